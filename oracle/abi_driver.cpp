// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// A caller built exactly like the reference's own binaries: compiled against the reference's
// headers (include/gap/...) with the reference CPU backends included from their sources (as
// src/core/backend_factory.cpp:14-17 does).  It loads the B200 plugin libraries the way
// BackendFactory does (dlopen + dlsym of create_gpu_*, src/core/backend_factory.cpp:26-96) and
// compares them with the reference CPU backends through the reference's own interfaces.
//
//   abi_driver <plugin_dir> <network.txt>
//   abi_driver --io <plugin_dir> <pgm_input.json>
//
// --io loads libgap_io_pgm.so (create_pgm_io_module) as an IIOModule and prints the NetworkData
// it reads ("bus id u_rated type u_pu", "br id from to status r1 x1 g1 b1 k theta i_n sn",
// "app id node status type p_specified q_specified g1 b1 u_ref"), so the reader is checked
// through the reference's own NetworkData layout.
//
// network.txt: "n" then n lines "id u_rated type u_pu p q"; "m" then m lines
// "id from to status r1 x1 g1 b1 k theta"; "a" then a lines "id node status type p q g1 b1";
// finally "tol max_iter base_power".  Prints "key value..." lines.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>

#include <iomanip>

#include "gap/io/io_interface.h"
#include "src/admittance/cpu/cpu_admittance_matrix.cpp"
#include "src/solver/lu/cpu/cpu_lu_solver.cpp"
#include "src/solver/powerflow/cpu/cpu_newton_raphson.cpp"

using namespace gap;

template <typename F>
static F load(std::string const& dir, const char* lib, const char* sym) {
    void* h = dlopen((dir + "/" + lib).c_str(), RTLD_LAZY);
    if (!h) {
        std::cerr << "dlopen " << lib << ": " << dlerror() << "\n";
        std::exit(2);
    }
    void* f = dlsym(h, sym);
    if (!f) {
        std::cerr << "dlsym " << sym << "\n";
        std::exit(2);
    }
    return reinterpret_cast<F>(f);
}

static int read_with_io_module(std::string const& dir, std::string const& file) {
    using CI = io::IIOModule* (*)();
    std::unique_ptr<io::IIOModule> m(load<CI>(dir, "libgap_io_pgm.so", "create_pgm_io_module")());
    std::cout << std::setprecision(17) << "valid " << m->validate_input_format(file) << "\n";
    NetworkData net = m->read_network_data(file);
    std::cout << "counts " << net.num_buses << " " << net.num_branches << " "
              << net.num_appliances << " " << net.buses.size() << " " << net.branches.size()
              << " " << net.appliances.size() << "\n";
    for (auto const& b : net.buses)
        std::cout << "bus " << b.id << " " << b.u_rated << " " << static_cast<int>(b.bus_type)
                  << " " << b.u_pu << "\n";
    for (auto const& b : net.branches)
        std::cout << "br " << b.id << " " << b.from_bus << " " << b.to_bus << " "
                  << static_cast<int>(b.status) << " " << b.r1 << " " << b.x1 << " " << b.g1
                  << " " << b.b1 << " " << b.k << " " << b.theta << " " << b.i_n << " " << b.sn
                  << "\n";
    for (auto const& a : net.appliances)
        std::cout << "app " << a.id << " " << a.node << " " << static_cast<int>(a.status) << " "
                  << static_cast<int>(a.type) << " " << a.p_specified << " " << a.q_specified
                  << " " << a.g1 << " " << a.b1 << " " << a.u_ref << "\n";
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    gap::logging::Logger::getInstance().configure(gap::logging::LogLevel::OFF,
                                                  gap::logging::LogOutput::NONE);
    if (std::string(argv[1]) == "--io") return argc < 4 ? 2 : read_with_io_module(argv[2], argv[3]);
    std::ifstream in(argv[2]);
    NetworkData net;
    int n, m, a;
    in >> n;
    net.buses.resize(n);
    for (auto& b : net.buses) {
        int t;
        in >> b.id >> b.u_rated >> t >> b.u_pu >> b.active_power >> b.reactive_power;
        b.bus_type = static_cast<BusType>(t);
        b.energized = 1;
    }
    in >> m;
    net.branches.resize(m);
    for (auto& br : net.branches) {
        int st;
        in >> br.id >> br.from_bus >> br.to_bus >> st >> br.r1 >> br.x1 >> br.g1 >> br.b1 >> br.k >>
            br.theta;
        br.status = static_cast<int8_t>(st);
        br.from_status = br.to_status = 1;
    }
    in >> a;
    net.appliances.resize(a);
    for (auto& ap : net.appliances) {
        int st, t;
        in >> ap.id >> ap.node >> st >> t >> ap.p_specified >> ap.q_specified >> ap.g1 >> ap.b1;
        ap.status = static_cast<int8_t>(st);
        ap.type = static_cast<ApplianceType>(t);
    }
    solver::PowerFlowConfig cfg;
    in >> cfg.tolerance >> cfg.max_iterations >> cfg.base_power;
    net.num_buses = n;
    net.num_branches = m;
    net.num_appliances = a;
    std::string dir = argv[1];

    using CA = admittance::IAdmittanceMatrix* (*)();
    using CL = solver::ILUSolver* (*)();
    using CP = solver::IPowerFlowSolver* (*)();
    std::unique_ptr<admittance::IAdmittanceMatrix> gy(
        load<CA>(dir, "libgap_admittance_gpu.so", "create_gpu_admittance_matrix")());
    std::shared_ptr<solver::ILUSolver> glu(load<CL>(dir, "libgap_lu_gpu.so", "create_gpu_lu_solver")());
    std::unique_ptr<solver::IPowerFlowSolver> gnr(
        load<CP>(dir, "libgap_powerflow_gpu.so", "create_gpu_powerflow_solver")());
    std::cout << "backend " << static_cast<int>(gy->get_backend_type()) << " "
              << static_cast<int>(glu->get_backend_type()) << " "
              << static_cast<int>(gnr->get_backend_type()) << "\n";

    // Y-bus
    admittance::CPUAdmittanceMatrix cy;
    auto Yc = cy.build_admittance_matrix(net);
    auto Yg = gy->build_admittance_matrix(net);
    bool pat = Yc->row_ptr == Yg->row_ptr && Yc->col_idx == Yg->col_idx && Yc->nnz == Yg->nnz &&
               Yc->num_rows == Yg->num_rows;
    double dy = 0.0;
    bool bits = pat;
    for (int i = 0; pat && i < Yc->nnz; ++i) {
        dy = std::max(dy, std::abs(Yc->values[i] - Yg->values[i]));
        bits = bits && Yc->values[i] == Yg->values[i];
    }
    std::cout << "ybus_pattern_equal " << pat << "\nybus_values_equal " << bits
              << "\nybus_max_abs_diff " << dy << "\n";

    // update_admittance_matrix: the first branch out of service
    if (m > 0) {
        std::vector<BranchData> ch = {net.branches[0]};
        ch[0].status = 0;
        auto Uc = cy.update_admittance_matrix(*Yc, ch);
        auto Ug = gy->update_admittance_matrix(*Yc, ch);
        double du = 0.0, scale = 0.0;
        for (int i = 0; i < Uc->nnz; ++i) {
            du = std::max(du, std::abs(Uc->values[i] - Ug->values[i]));
            scale = std::max(scale, std::abs(Uc->values[i]));
        }
        std::cout << "update_rel_diff " << (scale > 0 ? du / scale : du) << "\n";
    }

    // Newton-Raphson: reference CPU (CPU LU) vs plugin (plugin LU attached, as the bindings do)
    solver::CPUNewtonRaphson cnr;
    cnr.set_lu_solver(std::make_shared<solver::CPULUSolver>());
    auto rc = cnr.solve_power_flow(net, *Yc, cfg);
    gnr->set_lu_solver(glu);
    auto rg = gnr->solve_power_flow(net, *Yg, cfg);
    double dv = 0.0, da = 0.0;
    for (int i = 0; i < n; ++i) {
        dv = std::max(dv, std::abs(std::abs(rc.bus_voltages[i]) - std::abs(rg.bus_voltages[i])));
        da = std::max(da, std::abs(std::arg(rc.bus_voltages[i]) - std::arg(rg.bus_voltages[i])));
    }
    // bus_injections of the plugin (the reference leaves it empty) against S = V conj(Y V)
    // from the reference's Y-bus at the plugin's voltages, per unit
    double dinj = rg.bus_injections.size() == static_cast<size_t>(n) ? 0.0 : 1e300, sinj = 0.0;
    if (dinj == 0.0) {
        const double zb = net.buses[0].u_rated * net.buses[0].u_rated / cfg.base_power;
        for (int i = 0; i < n; ++i) {
            Complex cur(0.0, 0.0);
            for (int p = Yc->row_ptr[i]; p < Yc->row_ptr[i + 1]; ++p)
                cur += Yc->values[p] * zb * rg.bus_voltages[Yc->col_idx[p]];
            const Complex sref = rg.bus_voltages[i] * std::conj(cur);
            dinj = std::max(dinj, std::abs(sref - rg.bus_injections[i]));
            sinj = std::max(sinj, std::abs(sref));
        }
    }
    std::cout << "nr_bus_injections " << rc.bus_injections.size() << " " << dinj << " " << sinj
              << "\n";
    std::cout << "nr_converged " << rc.converged << " " << rg.converged << "\nnr_iterations "
              << rc.iterations << " " << rg.iterations << "\nnr_max_dv " << dv << "\nnr_max_dangle "
              << da << "\nnr_final_mismatch " << rc.final_mismatch << " " << rg.final_mismatch
              << "\n";

    // calculate_mismatches at the CPU solution
    auto mc = cnr.calculate_mismatches(net, rc.bus_voltages, *Yc);
    auto mg = gnr->calculate_mismatches(net, rc.bus_voltages, *Yg);
    double dm = 0.0, sm = 0.0;
    for (size_t i = 0; i < mc.size() && i < mg.size(); ++i) {
        dm = std::max(dm, std::abs(mc[i] - mg[i]));
        sm = std::max(sm, std::abs(mc[i]));
    }
    std::cout << "mismatch_sizes " << mc.size() << " " << mg.size() << "\nmismatch_max_abs_diff "
              << dm << " " << sm << "\n";

    // iteration-state capture: per-iteration states of both solvers along their trajectories
    // (differences relative to each quantity's largest magnitude over the run), and the
    // capturing solve's result against the plain one
    solver::IPowerFlowSolver& cbase = cnr;  // the capture methods are public on the interface
    cbase.enable_state_capture(true);
    gnr->enable_state_capture(true);
    cnr.solve_power_flow(net, *Yc, cfg);
    auto rg2 = gnr->solve_power_flow(net, *Yg, cfg);
    auto const& sc = cbase.get_iteration_states();
    auto const& sg = gnr->get_iteration_states();
    auto rel = [](std::vector<Complex> const& a, std::vector<Complex> const& b) {
        double d = 0.0, s = 0.0;
        for (size_t i = 0; i < a.size() && i < b.size(); ++i) {
            d = std::max(d, std::abs(a[i] - b[i]));
            s = std::max(s, std::abs(a[i]));
        }
        return a.size() == b.size() ? (s > 0 ? d / s : d) : 1e300;
    };
    double cv = 0.0, ci = 0.0, cs = 0.0, cm = 0.0, cx = 0.0, m0 = 0.0;
    int idx_ok = 1;
    for (auto const& st : sc) m0 = std::max(m0, st.max_mismatch);
    for (size_t k = 0; k < sc.size() && k < sg.size(); ++k) {
        idx_ok &= sc[k].iteration == static_cast<int>(k) && sg[k].iteration == static_cast<int>(k);
        cv = std::max(cv, rel(sc[k].voltages, sg[k].voltages));
        ci = std::max(ci, rel(sc[k].currents, sg[k].currents));
        cs = std::max(cs, rel(sc[k].power_injections, sg[k].power_injections));
        if (sc[k].mismatches.size() != sg[k].mismatches.size()) cm = 1e300;
        for (size_t i = 0; i < sc[k].mismatches.size() && i < sg[k].mismatches.size(); ++i)
            cm = std::max(cm, std::abs(sc[k].mismatches[i] - sg[k].mismatches[i]));
        cx = std::max(cx, std::abs(sc[k].max_mismatch - sg[k].max_mismatch));
    }
    double dsame = 0.0;
    for (int i = 0; i < n; ++i) dsame = std::max(dsame, std::abs(rg2.bus_voltages[i] - rg.bus_voltages[i]));
    std::cout << "capture_counts " << sc.size() << " " << sg.size() << "\ncapture_iteration_index "
              << idx_ok << "\ncapture_rel_diff " << cv << " " << ci << " " << cs
              << "\ncapture_mismatch_abs_diff " << cm << " " << cx << " " << m0
              << "\ncapture_result " << (rg2.iterations == rg.iterations) << " "
              << (rg2.converged == rg.converged) << " " << dsame << "\n";
    gnr->clear_iteration_states();
    std::cout << "capture_cleared " << gnr->get_iteration_states().size() << "\n";
    gnr->enable_state_capture(false);
    cbase.enable_state_capture(false);

    // LU: Y (duplicate entries summed, since the reference LU treats duplicates inconsistently:
    // last one wins on its dense path, both kept on its sparse path) with a dominant diagonal
    // added; reference CPU LU vs plugin LU
    SparseMatrix A;
    A.num_rows = A.num_cols = n;
    A.row_ptr.assign(1, 0);
    for (int i = 0; i < n; ++i) {
        for (int p = Yc->row_ptr[i]; p < Yc->row_ptr[i + 1]; ++p) {
            int c = Yc->col_idx[p];
            bool merged = false;
            for (int q = A.row_ptr[i]; q < static_cast<int>(A.col_idx.size()); ++q)
                if (A.col_idx[q] == c) {
                    A.values[q] += Yc->values[p];
                    merged = true;
                }
            if (!merged) {
                A.col_idx.push_back(c);
                A.values.push_back(Yc->values[p]);
            }
        }
        A.row_ptr.push_back(static_cast<int>(A.col_idx.size()));
    }
    A.nnz = static_cast<int>(A.values.size());
    double ymax = 0.0;
    for (auto const& v : A.values) ymax = std::max(ymax, std::abs(v));
    for (int i = 0; i < n; ++i)
        for (int p = A.row_ptr[i]; p < A.row_ptr[i + 1]; ++p)
            if (A.col_idx[p] == i) A.values[p] += Complex(ymax, 0.5 * ymax);
    ComplexVector b(n);
    for (int i = 0; i < n; ++i) b[i] = Complex(std::sin(i + 1.0), std::cos(3.0 * i));
    solver::CPULUSolver clu;
    bool fc = clu.factorize(A), fg = glu->factorize(A);
    double dx = 0.0, sx = 0.0;
    if (fc && fg) {
        auto xc = clu.solve(b);
        auto xg = glu->solve(b);
        for (int i = 0; i < n; ++i) {
            dx = std::max(dx, std::abs(xc[i] - xg[i]));
            sx = std::max(sx, std::abs(xc[i]));
        }
    }
    std::cout << "lu_factorized " << fc << " " << fg << " " << glu->is_factorized()
              << "\nlu_rel_diff " << (sx > 0 ? dx / sx : dx) << "\n";
    bool threw = false;
    try {
        glu->solve(ComplexVector(n + 1));
    } catch (std::runtime_error const&) {
        threw = true;
    }
    std::cout << "lu_bad_rhs_throws " << threw << "\n";
    return 0;
}
