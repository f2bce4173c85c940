// gap_b200_main: the reference's command-line power flow (src/main/main.cpp) over the B200
// libraries, with the same options, flow and summary:
//   read the network through the IO module, build the admittance matrix, set the LU solver,
//   solve, write the results.
// The modules are loaded the way the reference's BackendFactory loads its GPU backends
// (dlopen of the bare library name + dlsym of the factory, src/core/backend_factory.cpp:26-96,
// 125-132; found through this executable's $ORIGIN rpath): libgap_io_pgm.so
// (create_pgm_io_module: PGM JSON input with loads as consumption), libgap_admittance_gpu.so,
// libgap_lu_gpu.so and libgap_powerflow_gpu.so.  Only the GPU backend exists here ("-b cpu" is
// refused).  One option is added: --base-power VA (PowerFlowConfig::base_power, default
// 100e6 as the reference's).
#include <dlfcn.h>

#include <chrono>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>

#include "gap_b200/gap_interfaces.hpp"

using namespace gap;

namespace {

struct AppConfig {
    std::string input_file, output_file;
    solver::PowerFlowConfig pf;
    bool verbose = false, benchmark = false;
};

void usage(const char* prog) {
    std::cout << "Usage: " << prog << " [OPTIONS]\n\nOPTIONS:\n"
              << "  -i, --input FILE      Input file path (PGM JSON, required)\n"
              << "  -o, --output FILE     Output file path (required)\n"
              << "  -b, --backend TYPE    Backend type: gpu (the only one in this build)\n"
              << "  -t, --tolerance VAL   Convergence tolerance (default: 1e-6)\n"
              << "  -m, --max-iter NUM    Maximum iterations (default: 50)\n"
              << "  --base-power VA       Per-unit power base (default: 100e6)\n"
              << "  -v, --verbose         Enable verbose output\n"
              << "  --benchmark           Enable benchmarking\n"
              << "  --flat-start          Use flat start initialization\n"
              << "  -h, --help            Show this help message\n";
}

AppConfig parse(int argc, char** argv) {
    AppConfig c;
    auto next = [&](int& i, const char* what) -> std::string {
        if (i + 1 >= argc) throw std::invalid_argument(std::string("Missing ") + what + " argument");
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-h" || a == "--help") {
            usage(argv[0]);
            std::exit(0);
        } else if (a == "-i" || a == "--input") {
            c.input_file = next(i, "input file");
        } else if (a == "-o" || a == "--output") {
            c.output_file = next(i, "output file");
        } else if (a == "-b" || a == "--backend") {
            const std::string b = next(i, "backend");
            if (b != "gpu") throw std::invalid_argument("Invalid backend type for this build: " + b);
        } else if (a == "-t" || a == "--tolerance") {
            c.pf.tolerance = std::stod(next(i, "tolerance"));
        } else if (a == "-m" || a == "--max-iter") {
            c.pf.max_iterations = std::stoi(next(i, "max iterations"));
        } else if (a == "--base-power") {
            c.pf.base_power = std::stod(next(i, "base power"));
        } else if (a == "-v" || a == "--verbose") {
            c.verbose = c.pf.verbose = true;
        } else if (a == "--benchmark") {
            c.benchmark = true;
        } else if (a == "--flat-start") {
            c.pf.use_flat_start = true;
        } else {
            throw std::invalid_argument("Unknown argument: " + a);
        }
    }
    if (c.input_file.empty()) throw std::invalid_argument("Input file is required");
    if (c.output_file.empty()) throw std::invalid_argument("Output file is required");
    return c;
}

template <typename T>
T* create(const char* lib, const char* sym) {
    void* h = dlopen(lib, RTLD_LAZY);  // never closed, as BackendFactory does
    if (!h) throw std::runtime_error(std::string("cannot load ") + lib + ": " + dlerror());
    auto f = reinterpret_cast<T* (*)()>(dlsym(h, sym));
    if (!f) throw std::runtime_error(std::string(lib) + " has no " + sym);
    return f();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc == 1) {
        std::cout << "GAP Power Flow Calculator (B200)\n\nAvailable backends: GPU\n\n";
        usage(argv[0]);
        return 0;
    }
    try {
        const AppConfig cfg = parse(argc, argv);
        const auto t0 = std::chrono::high_resolution_clock::now();
        std::unique_ptr<io::IIOModule> io(create<io::IIOModule>("libgap_io_pgm.so", "create_pgm_io_module"));
        std::unique_ptr<admittance::IAdmittanceMatrix> adm(create<admittance::IAdmittanceMatrix>(
            "libgap_admittance_gpu.so", "create_gpu_admittance_matrix"));
        std::shared_ptr<solver::ILUSolver> lu(
            create<solver::ILUSolver>("libgap_lu_gpu.so", "create_gpu_lu_solver"));
        std::unique_ptr<solver::IPowerFlowSolver> pf(create<solver::IPowerFlowSolver>(
            "libgap_powerflow_gpu.so", "create_gpu_powerflow_solver"));
        if (cfg.verbose) std::cout << "Reading network data...\n";
        if (!io->validate_input_format(cfg.input_file))
            throw std::runtime_error("not a PGM input dataset: " + cfg.input_file);
        const NetworkData net = io->read_network_data(cfg.input_file);
        if (cfg.verbose) std::cout << "Building admittance matrix...\n";
        const auto Y = adm->build_admittance_matrix(net);
        pf->set_lu_solver(lu);
        if (cfg.verbose) std::cout << "Solving power flow...\n";
        const solver::PowerFlowResult r = pf->solve_power_flow(net, *Y, cfg.pf);
        if (cfg.verbose) std::cout << "Writing results...\n";
        io->write_results(cfg.output_file, r.bus_voltages, r.converged, r.iterations);
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::high_resolution_clock::now() - t0)
                            .count();
        std::cout << "\nPower Flow Solution Summary:\n"
                  << "  Status: " << (r.converged ? "CONVERGED" : "NOT CONVERGED") << "\n"
                  << "  Iterations: " << r.iterations << "\n"
                  << "  Final mismatch: " << r.final_mismatch << "\n"
                  << "  Bus voltages: " << r.bus_voltages.size() << "\n";
        if (cfg.benchmark) std::cout << "  Execution time: " << ms << " ms\n";
        return r.converged ? 0 : 1;
    } catch (std::exception const& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
