// gap_interfaces.hpp -- the reference's C++ plugin ABI, restated for the B200 plugins.
//
// The reference loads GPU backends with dlopen("libgap_*_gpu.so") + dlsym("create_gpu_*")
// (src/core/backend_factory.cpp:26-96) and calls them through three abstract classes.  A
// drop-in replacement must therefore present the same class layouts and the same virtual
// function order.  This header declares them again, member for member and in the same order,
// after:
//   include/gap/core/types.h:15-66, 204-357   (Float, Complex, enums, SparseMatrix,
//                                              BusData, BranchData, ApplianceData,
//                                              NetworkData, BackendType)
//   include/gap/admittance/admittance_interface.h:12-38   (IAdmittanceMatrix)
//   include/gap/solver/lu_solver_interface.h:12-48        (ILUSolver)
//   include/gap/solver/powerflow_interface.h:13-108       (PowerFlowConfig, IterationState,
//                                                           PowerFlowResult, IPowerFlowSolver)
//   include/gap/io/io_interface.h:8-44                    (IIOModule)
// Only layout-relevant declarations are repeated (no inline helpers, no GPU mirror structs).
// tests/test_gpu_plugins.py loads the plugins from a driver compiled against the reference's
// own headers, which checks that the two agree.
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace gap {

using Float = double;
using Complex = std::complex<Float>;
using ComplexVector = std::vector<Complex>;

enum class BusType { PQ = 0, PV = 1, SLACK = 2 };
enum class ApplianceType { SOURCE = 0, LOADGEN = 1, SHUNT = 2 };
enum class BranchType { LINE = 0, TRAFO = 1, GENERIC = 2 };
enum class BackendType { CPU, GPU_CUDA };

struct SparseMatrix {
    std::vector<int> row_ptr;
    std::vector<int> col_idx;
    std::vector<Complex> values;
    int num_rows;
    int num_cols;
    int nnz;
};

struct BusData {
    int id;
    Float u_rated;
    BusType bus_type{BusType::PQ};
    int8_t energized{0};
    Float u{0.0};
    Float u_pu{0.0};
    Float u_angle{0.0};
    Float active_power{0.0};
    Float reactive_power{0.0};
};

struct BranchData {
    int id;
    int from_bus;
    int8_t from_status;
    int to_bus;
    int8_t to_status;
    int8_t status;
    BranchType branch_type{BranchType::LINE};
    Float p_from{0.0}, p_to{0.0}, q_from{0.0}, q_to{0.0}, s_from{0.0}, s_to{0.0};
    Float i_from{0.0}, i_from_angle{0.0}, i_to{0.0}, i_to_angle{0.0}, loading{0.0};
    Float r1{1e-6}, x1{1e-6}, g1{0.0}, b1{0.0}, k{1.0}, theta{0.0}, sn{0.0};
    Float i_n{1000.0};
};

struct ApplianceData {
    int id;
    int node;
    int8_t status;
    ApplianceType type;
    Float p{0.0}, q{0.0}, i{0.0}, s{0.0};
    Float u_ref{1.0}, u_ref_angle{0.0}, sk{1e10}, rx_ratio{0.1};
    Float p_specified{0.0}, q_specified{0.0};
    Float g1{0.0}, b1{0.0};
};

struct NetworkData {
    std::vector<BusData> buses;
    std::vector<BranchData> branches;
    std::vector<ApplianceData> appliances;
    int num_buses;
    int num_branches;
    int num_appliances;
    std::string version{"1.0"};
    std::string type{"input"};
    bool is_batch{false};
};

namespace admittance {
class IAdmittanceMatrix {
  public:
    virtual ~IAdmittanceMatrix() = default;
    virtual std::unique_ptr<SparseMatrix> build_admittance_matrix(
        NetworkData const& network_data) = 0;
    virtual std::unique_ptr<SparseMatrix> update_admittance_matrix(
        SparseMatrix const& matrix, std::vector<BranchData> const& branch_changes) = 0;
    virtual BackendType get_backend_type() const noexcept = 0;
};
}  // namespace admittance

namespace solver {
class ILUSolver {
  public:
    virtual ~ILUSolver() = default;
    virtual bool factorize(SparseMatrix const& matrix) = 0;
    virtual ComplexVector solve(ComplexVector const& rhs) = 0;
    virtual bool update_factorization(SparseMatrix const& matrix) = 0;
    virtual BackendType get_backend_type() const noexcept = 0;
    virtual bool is_factorized() const noexcept = 0;
};

struct PowerFlowConfig {
    Float tolerance = 1e-6;
    int max_iterations = 50;
    bool use_flat_start = true;
    Float acceleration_factor = 1.0;
    bool verbose = false;
    Float base_power = 100e6;
};

struct IterationState {
    int iteration;
    std::vector<Complex> voltages;
    std::vector<Complex> currents;
    std::vector<Complex> power_injections;
    std::vector<double> mismatches;
    double max_mismatch;
};

struct PowerFlowResult {
    bool converged = false;
    int iterations = 0;
    Float final_mismatch = 0.0;
    ComplexVector bus_voltages;
    ComplexVector bus_injections;
};

class IPowerFlowSolver {
  public:
    virtual ~IPowerFlowSolver() = default;
    virtual PowerFlowResult solve_power_flow(NetworkData const& network_data,
                                             SparseMatrix const& admittance_matrix,
                                             PowerFlowConfig const& config = PowerFlowConfig{}) = 0;
    virtual void set_lu_solver(std::shared_ptr<ILUSolver> lu_solver) = 0;
    virtual std::vector<Float> calculate_mismatches(NetworkData const& network_data,
                                                    ComplexVector const& bus_voltages,
                                                    SparseMatrix const& admittance_matrix) = 0;
    virtual BackendType get_backend_type() const noexcept = 0;
    virtual void enable_state_capture(bool enable) { (void)enable; }
    virtual std::vector<IterationState> const& get_iteration_states() const {
        static std::vector<IterationState> empty;
        return empty;
    }
    virtual void clear_iteration_states() {}
};
}  // namespace solver

namespace io {
class IIOModule {
  public:
    virtual ~IIOModule() = default;
    virtual NetworkData read_network_data(std::string const& filename) = 0;
    virtual void write_results(std::string const& filename, ComplexVector const& bus_voltages,
                               bool converged, int iterations) = 0;
    virtual bool validate_input_format(std::string const& filename) = 0;
};
}  // namespace io

}  // namespace gap
