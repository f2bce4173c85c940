// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// A thin extern "C" driver over the reference's own CPU power-flow path, compiled from the
// reference sources where they lie (see oracle/Makefile).  Only tests/, the smoke check and the
// cpu_baseline leg of bench.py load the resulting oracle/_ref/libgapref.so, and only as the
// checker.  Nothing here is used by the GPU engine.
//
// The reference classes live in .cpp files without headers; the reference's own
// BackendFactory includes those .cpp files directly (src/core/backend_factory.cpp:14-17), and
// this driver does the same.
//
//   CPUAdmittanceMatrix  src/admittance/cpu/cpu_admittance_matrix.cpp:13-304
//   CPUNewtonRaphson     src/solver/powerflow/cpu/cpu_newton_raphson.cpp:13-777
//   CPULUSolver          src/solver/lu/cpu/cpu_lu_solver.cpp:25-828

#include "src/admittance/cpu/cpu_admittance_matrix.cpp"
#include "src/solver/lu/cpu/cpu_lu_solver.cpp"
#include "src/solver/powerflow/cpu/cpu_newton_raphson.cpp"

#include <cstring>

extern "C" {

// Flat description of gap::NetworkData (include/gap/core/types.h:204-352).
struct gapref_net {
    int n_bus;
    const int* bus_id;
    const double* u_rated;
    const int* bus_type;  // 0 PQ, 1 PV, 2 SLACK
    const double* u_pu;
    const double* p_w;    // BusData::active_power
    const double* q_var;  // BusData::reactive_power
    int n_branch;
    const int* br_id;
    const int* from_id;
    const int* to_id;
    const int* status;
    const double* r1;
    const double* x1;
    const double* g1;
    const double* b1;
    const double* k;
    const double* theta;
    int n_app;
    const int* app_id;
    const int* app_node;
    const int* app_status;
    const int* app_type;  // 0 SOURCE, 1 LOADGEN, 2 SHUNT
    const double* app_p;
    const double* app_q;
    const double* app_g1;
    const double* app_b1;
};

static gap::NetworkData to_network(gapref_net const* n) {
    gap::NetworkData net;
    net.num_buses = n->n_bus;
    net.num_branches = n->n_branch;
    net.num_appliances = n->n_app;
    net.buses.resize(n->n_bus);
    for (int i = 0; i < n->n_bus; ++i) {
        auto& b = net.buses[i];
        b.id = n->bus_id[i];
        b.u_rated = n->u_rated[i];
        b.bus_type = static_cast<gap::BusType>(n->bus_type[i]);
        b.energized = 1;
        b.u_pu = n->u_pu[i];
        b.u_angle = 0.0;
        b.active_power = n->p_w[i];
        b.reactive_power = n->q_var[i];
    }
    net.branches.resize(n->n_branch);
    for (int i = 0; i < n->n_branch; ++i) {
        auto& br = net.branches[i];
        br.id = n->br_id[i];
        br.from_bus = n->from_id[i];
        br.to_bus = n->to_id[i];
        br.from_status = 1;
        br.to_status = 1;
        br.status = static_cast<int8_t>(n->status[i]);
        br.r1 = n->r1[i];
        br.x1 = n->x1[i];
        br.g1 = n->g1[i];
        br.b1 = n->b1[i];
        br.k = n->k[i];
        br.theta = n->theta[i];
    }
    net.appliances.resize(n->n_app);
    for (int i = 0; i < n->n_app; ++i) {
        auto& a = net.appliances[i];
        a.id = n->app_id[i];
        a.node = n->app_node[i];
        a.status = static_cast<int8_t>(n->app_status[i]);
        a.type = static_cast<gap::ApplianceType>(n->app_type[i]);
        a.p_specified = n->app_p[i];
        a.q_specified = n->app_q[i];
        a.g1 = n->app_g1[i];
        a.b1 = n->app_b1[i];
    }
    return net;
}

void gapref_quiet(void) {
    gap::logging::Logger::getInstance().configure(gap::logging::LogLevel::OFF,
                                                  gap::logging::LogOutput::NONE);
}

// Y-bus in Siemens, exactly as CPUAdmittanceMatrix::build_admittance_matrix returns it.
// values are interleaved (re, im).  Returns nnz, or -(needed capacity) when cap is too small.
int gapref_ybus(gapref_net const* n, int cap, int* row_ptr, int* col_idx, double* values) {
    gapref_quiet();
    auto net = to_network(n);
    gap::admittance::CPUAdmittanceMatrix builder;
    auto Y = builder.build_admittance_matrix(net);
    if (Y->nnz > cap) return -Y->nnz;
    std::memcpy(row_ptr, Y->row_ptr.data(), sizeof(int) * Y->row_ptr.size());
    std::memcpy(col_idx, Y->col_idx.data(), sizeof(int) * Y->nnz);
    for (int i = 0; i < Y->nnz; ++i) {
        values[2 * i] = Y->values[i].real();
        values[2 * i + 1] = Y->values[i].imag();
    }
    return Y->nnz;
}

// update_admittance_matrix on a Y built from the same network; the changes are branches given
// by (from_id, to_id, status, r1, x1, g1, b1) in the same flat form.
int gapref_ybus_update(gapref_net const* n, gapref_net const* changes, int cap, int* row_ptr,
                       int* col_idx, double* values) {
    gapref_quiet();
    auto net = to_network(n);
    auto ch = to_network(changes);
    gap::admittance::CPUAdmittanceMatrix builder;
    auto Y = builder.build_admittance_matrix(net);
    auto Y2 = builder.update_admittance_matrix(*Y, ch.branches);
    if (Y2->nnz > cap) return -Y2->nnz;
    std::memcpy(row_ptr, Y2->row_ptr.data(), sizeof(int) * Y2->row_ptr.size());
    std::memcpy(col_idx, Y2->col_idx.data(), sizeof(int) * Y2->nnz);
    for (int i = 0; i < Y2->nnz; ++i) {
        values[2 * i] = Y2->values[i].real();
        values[2 * i + 1] = Y2->values[i].imag();
    }
    return Y2->nnz;
}

// Full reference NR: Y-bus build + CPUNewtonRaphson with CPULUSolver, as the reference's
// Python binding wires them (bindings/solver_bindings.cpp:134-160).
// v_out holds n_bus complex voltages (re, im) in per unit.
int gapref_solve(gapref_net const* n, double tol, int max_iter, double base_power,
                 double* v_out, int* converged, int* iterations, double* final_mismatch) {
    gapref_quiet();
    try {
        auto net = to_network(n);
        gap::admittance::CPUAdmittanceMatrix builder;
        auto Y = builder.build_admittance_matrix(net);
        gap::solver::CPUNewtonRaphson nr;
        nr.set_lu_solver(std::make_shared<gap::solver::CPULUSolver>());
        gap::solver::PowerFlowConfig cfg;
        cfg.tolerance = tol;
        cfg.max_iterations = max_iter;
        cfg.base_power = base_power;
        cfg.use_flat_start = true;
        auto res = nr.solve_power_flow(net, *Y, cfg);
        for (int i = 0; i < n->n_bus; ++i) {
            v_out[2 * i] = res.bus_voltages[i].real();
            v_out[2 * i + 1] = res.bus_voltages[i].imag();
        }
        *converged = res.converged ? 1 : 0;
        *iterations = res.iterations;
        *final_mismatch = res.final_mismatch;
        return 0;
    } catch (std::exception const&) {
        return -1;
    }
}

// The same solve with iteration-state capture on (IPowerFlowSolver::enable_state_capture,
// cpu_newton_raphson.cpp:95-149): per captured iteration k < cap, max_mis[k] and the voltages
// v_states[k][n_bus] (re, im), currents i_states and power injections s_states likewise (each
// nullable).  Returns the number of states captured, or -1 when the solve throws.
int gapref_solve_states(gapref_net const* n, double tol, int max_iter, double base_power,
                        int cap, double* max_mis, double* v_states, double* i_states,
                        double* s_states) {
    gapref_quiet();
    try {
        auto net = to_network(n);
        gap::admittance::CPUAdmittanceMatrix builder;
        auto Y = builder.build_admittance_matrix(net);
        gap::solver::CPUNewtonRaphson nr;
        nr.set_lu_solver(std::make_shared<gap::solver::CPULUSolver>());
        gap::solver::IPowerFlowSolver& base = nr;
        base.enable_state_capture(true);
        gap::solver::PowerFlowConfig cfg;
        cfg.tolerance = tol;
        cfg.max_iterations = max_iter;
        cfg.base_power = base_power;
        cfg.use_flat_start = true;
        nr.solve_power_flow(net, *Y, cfg);
        auto const& st = base.get_iteration_states();
        const int nb = n->n_bus;
        const int k_n = static_cast<int>(st.size());
        auto put = [nb](double* dst, int k, std::vector<gap::Complex> const& x) {
            if (!dst) return;
            for (int i = 0; i < nb && i < static_cast<int>(x.size()); ++i) {
                dst[(static_cast<size_t>(k) * nb + i) * 2] = x[i].real();
                dst[(static_cast<size_t>(k) * nb + i) * 2 + 1] = x[i].imag();
            }
        };
        for (int k = 0; k < k_n && k < cap; ++k) {
            if (max_mis) max_mis[k] = st[k].max_mismatch;
            put(v_states, k, st[k].voltages);
            put(i_states, k, st[k].currents);
            put(s_states, k, st[k].power_injections);
        }
        return k_n;
    } catch (std::exception const&) {
        return -1;
    }
}

// IPowerFlowSolver::calculate_mismatches (Watts, base 100 MVA) for a given voltage vector,
// using the reference-built Y-bus.
int gapref_mismatch(gapref_net const* n, double const* v, int cap, double* out) {
    gapref_quiet();
    auto net = to_network(n);
    gap::admittance::CPUAdmittanceMatrix builder;
    auto Y = builder.build_admittance_matrix(net);
    gap::ComplexVector V(n->n_bus);
    for (int i = 0; i < n->n_bus; ++i) V[i] = gap::Complex(v[2 * i], v[2 * i + 1]);
    gap::solver::CPUNewtonRaphson nr;
    auto mm = nr.calculate_mismatches(net, V, *Y);
    if (static_cast<int>(mm.size()) > cap) return -static_cast<int>(mm.size());
    for (size_t i = 0; i < mm.size(); ++i) out[i] = mm[i];
    return static_cast<int>(mm.size());
}

// CPULUSolver factorize + solve on a complex CSR matrix.  Returns 0 on success, 1 when
// factorize() reports failure, -1 when solve() throws.
int gapref_lu_solve(int n, int nnz, int const* row_ptr, int const* col_idx, double const* vals,
                    double const* rhs, double* x_out) {
    gapref_quiet();
    gap::SparseMatrix A;
    A.num_rows = A.num_cols = n;
    A.nnz = nnz;
    A.row_ptr.assign(row_ptr, row_ptr + n + 1);
    A.col_idx.assign(col_idx, col_idx + nnz);
    A.values.resize(nnz);
    for (int i = 0; i < nnz; ++i) A.values[i] = gap::Complex(vals[2 * i], vals[2 * i + 1]);
    gap::solver::CPULUSolver lu;
    if (!lu.factorize(A)) return 1;
    gap::ComplexVector b(n);
    for (int i = 0; i < n; ++i) b[i] = gap::Complex(rhs[2 * i], rhs[2 * i + 1]);
    try {
        auto x = lu.solve(b);
        for (int i = 0; i < n; ++i) {
            x_out[2 * i] = x[i].real();
            x_out[2 * i + 1] = x[i].imag();
        }
    } catch (std::exception const&) {
        return -1;
    }
    return 0;
}

}  // extern "C"
