// libgap_powerflow_gpu.so -- IPowerFlowSolver on the B200 Newton-Raphson engine.
//
// Replaces src/solver/powerflow/gpu/gpu_newton_raphson.cu (factory at :631-637) with the
// semantics of the reference CPU solver (src/solver/powerflow/cpu/cpu_newton_raphson.cpp:
// 33-240): per unit on buses[0].u_rated and config.base_power, specified power from the buses
// and their in-service SOURCE/LOADGEN appliances, flat start (SLACK/PV at u_pu, PQ at 0.98),
// the damped and clamped polar update, convergence on max |mismatch| < tolerance.  The whole
// loop runs on the device; the plan (ordering, symbolic factorisation) is cached per Y pattern
// and bus-type vector and rebuilt when either changes.  config.acceleration_factor is ignored,
// as by the reference CPU solver.  set_lu_solver() is accepted but the device engine always
// factorises with its own block LU.  With state capture enabled the same device loop is stepped
// from the host, one synchronisation per iteration.
#include <cmath>
#include <unordered_map>

#include "common.hpp"

namespace gapb200 {

class B200NewtonRaphson final : public gap::solver::IPowerFlowSolver {
  public:
    ~B200NewtonRaphson() override { reset(); }

    gap::solver::PowerFlowResult solve_power_flow(gap::NetworkData const& net,
                                                  gap::SparseMatrix const& Y,
                                                  gap::solver::PowerFlowConfig const& cfg) override {
        gap::solver::PowerFlowResult res;
        const int n = static_cast<int>(net.buses.size());
        res.bus_voltages.assign(n, gap::Complex(0.0, 0.0));
        if (n == 0 || cfg.max_iterations <= 0) {
            res.converged = n == 0 && cfg.max_iterations > 0;
            res.iterations = cfg.max_iterations > 0 ? 1 : 0;
            return res;
        }
        if (Y.num_rows != n || static_cast<int>(Y.row_ptr.size()) != n + 1)
            throw std::runtime_error("admittance matrix does not match the network");
        ensure_plan(net, Y);
        const double vb = net.buses[0].u_rated;
        const double zb = (vb * vb) / cfg.base_power;
        std::vector<gap::Complex> ypu(Y.nnz);
        for (int i = 0; i < Y.nnz; ++i) ypu[i] = Y.values[i] * zb;
        auto s = specified_power(net, cfg.base_power);
        std::vector<double> upu(n);
        for (int i = 0; i < n; ++i) upu[i] = net.buses[i].u_pu;
        gapk_nr_inputs in{};
        in.d_y = reinterpret_cast<const double*>(d_y_.upload(ypu));
        in.d_s_spec = reinterpret_cast<const double*>(d_s_.upload(s));
        in.d_u_pu = d_u_.upload(upu);
        if (!cfg.use_flat_start) {
            // the reference never initialises V without a flat start: it stays zero
            in.d_v_init = reinterpret_cast<const double*>(d_v_.upload(res.bus_voltages));
        }
        in.tolerance = cfg.tolerance;
        in.max_iterations = cfg.max_iterations;
        in.policy = GAPK_POLICY_REFERENCE;
        in.refine = 0;
        gapk_nr_outputs out{};
        out.d_v = static_cast<double*>(d_vo_.ensure(static_cast<size_t>(n) * 16));
        out.d_iterations = static_cast<int*>(d_it_.ensure(4));
        out.d_status = static_cast<int*>(d_st_.ensure(4));
        out.d_final_mismatch = static_cast<double*>(d_fm_.ensure(8));
        if (capture_)
            solve_capturing(in, out, n, cfg.max_iterations);
        else
            check(gapk_nr_solve(batch_, &in, &out, nullptr), "gapk_nr_solve");
        check_cuda(cudaMemcpy(res.bus_voltages.data(), out.d_v, static_cast<size_t>(n) * 16,
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy D2H");
        int it = 0, st = 0;
        double fm = 0.0;
        check_cuda(cudaMemcpy(&it, out.d_iterations, 4, cudaMemcpyDeviceToHost), "D2H");
        check_cuda(cudaMemcpy(&st, out.d_status, 4, cudaMemcpyDeviceToHost), "D2H");
        check_cuda(cudaMemcpy(&fm, out.d_final_mismatch, 8, cudaMemcpyDeviceToHost), "D2H");
        if (capture_ && st == GAPK_SCEN_SINGULAR) {
            // the device loop stops a scenario whose Jacobian does not factorise; the reference
            // keeps V and runs on to max_iterations (cpu_newton_raphson.cpp:416-419), recording
            // the same state each time
            while (!states_.empty() && static_cast<int>(states_.size()) < it) {
                gap::solver::IterationState s = states_.back();
                s.iteration = static_cast<int>(states_.size());
                states_.push_back(std::move(s));
            }
        }
        res.converged = st == GAPK_SCEN_CONVERGED;
        res.iterations = it;
        res.final_mismatch = fm;
        // bus_injections (declared by powerflow_interface.h:37-43, never filled by the
        // reference): S = V conj(Y V) at the final voltages, per unit like bus_voltages
        double* ds = static_cast<double*>(d_sb_.ensure(static_cast<size_t>(n) * 16));
        check(gapk_nr_get_state(batch_, nullptr, nullptr, ds, nullptr), "gapk_nr_get_state");
        d_sb_.download(res.bus_injections, n);
        return res;
    }

    void set_lu_solver(std::shared_ptr<gap::solver::ILUSolver> lu) override { lu_ = std::move(lu); }

    // Reference public method (cpu_newton_raphson.cpp:225-240): mismatches in the reference's
    // equation order, computed with the admittance matrix as given and a fixed 100 MVA base,
    // returned in W / var.
    std::vector<gap::Float> calculate_mismatches(gap::NetworkData const& net,
                                                 gap::ComplexVector const& V,
                                                 gap::SparseMatrix const& Y) override {
        const int n = static_cast<int>(net.buses.size());
        if (n == 0) return {};
        ensure_plan(net, Y);
        const double base = 100e6;
        auto s = specified_power(net, base);
        gapk_nr_inputs in{};
        in.d_y = reinterpret_cast<const double*>(d_y_.upload(Y.values));
        in.d_s_spec = reinterpret_cast<const double*>(d_s_.upload(s));
        in.d_v_init = reinterpret_cast<const double*>(d_v_.upload(V));
        in.max_iterations = 1;
        in.policy = GAPK_POLICY_NEWTON;
        check(gapk_nr_stage_load(batch_, &in, nullptr), "gapk_nr_stage_load");
        check(gapk_nr_stage_mismatch(batch_, nullptr), "gapk_nr_stage_mismatch");
        gapk_nr_plan_info info{};
        gapk_nr_plan_get_info(plan_, &info);
        double* df = static_cast<double*>(d_f_.ensure(static_cast<size_t>(info.n_vars) * 8 + 8));
        check(gapk_nr_stage_get_mismatch(batch_, df, nullptr), "gapk_nr_stage_get_mismatch");
        std::vector<double> f;
        d_f_.download(f, info.n_vars);
        for (auto& x : f) x *= base;
        return f;
    }

    gap::BackendType get_backend_type() const noexcept override {
        return gap::BackendType::GPU_CUDA;
    }

    // Iteration-state capture (powerflow_interface.h:83-107): with capture enabled, each solve
    // records, per iteration, the voltages the mismatch is taken at, I = Y V, S = V conj(I),
    // the mismatches (per unit, in the reference's equation order) and their maximum, as
    // gpu_newton_raphson.cu:452-490 and cpu_newton_raphson.cpp:125-149 do.
    void enable_state_capture(bool enable) override { capture_ = enable; }
    std::vector<gap::solver::IterationState> const& get_iteration_states() const override {
        return states_;
    }
    void clear_iteration_states() override { states_.clear(); }

  private:
    // The device loop stepped one iteration at a time (the trajectory of gapk_nr_solve) with
    // the state copied out before each step and the step's mismatch after it.
    void solve_capturing(gapk_nr_inputs const& in, gapk_nr_outputs const& out, int n,
                         int max_iterations) {
        states_.clear();
        check(gapk_nr_stage_load(batch_, &in, nullptr), "gapk_nr_stage_load");
        gapk_nr_plan_info info{};
        check(gapk_nr_plan_get_info(plan_, &info), "gapk_nr_plan_get_info");
        double* dv = static_cast<double*>(d_cap_.ensure(static_cast<size_t>(n) * 48));
        double* df = static_cast<double*>(d_f_.ensure(static_cast<size_t>(info.n_vars) * 8 + 8));
        std::vector<gap::Complex> vis;
        for (int it = 0; it < max_iterations; ++it) {
            check(gapk_nr_get_state(batch_, dv, dv + 2 * n, dv + 4 * n, nullptr),
                  "gapk_nr_get_state");
            int active = 0;
            check(gapk_nr_step(batch_, &active, nullptr), "gapk_nr_step");
            check(gapk_nr_stage_get_mismatch(batch_, df, nullptr), "gapk_nr_stage_get_mismatch");
            gap::solver::IterationState s;
            s.iteration = it;
            d_cap_.download(vis, static_cast<size_t>(3) * n);
            s.voltages.assign(vis.begin(), vis.begin() + n);
            s.currents.assign(vis.begin() + n, vis.begin() + 2 * n);
            s.power_injections.assign(vis.begin() + 2 * n, vis.end());
            d_f_.download(s.mismatches, info.n_vars);
            s.max_mismatch = 0.0;
            for (double x : s.mismatches) s.max_mismatch = std::max(s.max_mismatch, std::abs(x));
            states_.push_back(std::move(s));
            if (!active) break;
        }
        check(gapk_nr_get_outputs(batch_, &out, nullptr), "gapk_nr_get_outputs");
    }

    // get_specified_power_at_bus (cpu_newton_raphson.cpp:346-377), per unit of `base`
    static std::vector<gap::Complex> specified_power(gap::NetworkData const& net, double base) {
        const int n = static_cast<int>(net.buses.size());
        std::vector<gap::Complex> s(n);
        std::unordered_map<int, std::vector<int>> by_id;
        for (int i = 0; i < n; ++i) {
            s[i] = gap::Complex(net.buses[i].active_power, net.buses[i].reactive_power);
            by_id[net.buses[i].id].push_back(i);
        }
        for (auto const& a : net.appliances) {
            if (a.status != 1) continue;
            if (a.type != gap::ApplianceType::SOURCE && a.type != gap::ApplianceType::LOADGEN)
                continue;
            auto it = by_id.find(a.node);
            if (it == by_id.end()) continue;
            for (int i : it->second) s[i] += gap::Complex(a.p_specified, a.q_specified);
        }
        if (base > 0.0)
            for (auto& x : s) x /= base;
        return s;
    }

    void ensure_plan(gap::NetworkData const& net, gap::SparseMatrix const& Y) {
        const int n = static_cast<int>(net.buses.size());
        std::vector<int> bt(n);
        for (int i = 0; i < n; ++i) bt[i] = static_cast<int>(net.buses[i].bus_type);
        std::vector<int> ci(Y.col_idx.begin(), Y.col_idx.begin() + Y.nnz);
        if (plan_ && bt == bt_ && Y.row_ptr == rp_ && ci == ci_) return;
        reset();
        gapk_nr_plan_options po{GAPK_JAC_REFERENCE, GAPK_ORDER_MINDEG, 0};
        check(gapk_nr_plan_create(n, Y.nnz, Y.row_ptr.data(), ci.data(), bt.data(), &po, &plan_),
              "gapk_nr_plan_create");
        gapk_nr_batch_options bo{GAPK_PREC_FP64, 1, 1, 0, 1};
        check(gapk_nr_batch_create(plan_, 1, &bo, &batch_), "gapk_nr_batch_create");
        bt_ = bt;
        rp_ = Y.row_ptr;
        ci_ = ci;
    }

    void reset() {
        if (batch_) gapk_nr_batch_destroy(batch_);
        if (plan_) gapk_nr_plan_destroy(plan_);
        batch_ = nullptr;
        plan_ = nullptr;
    }

    std::shared_ptr<gap::solver::ILUSolver> lu_;
    gapk_nr_plan plan_ = nullptr;
    gapk_nr_batch batch_ = nullptr;
    std::vector<int> bt_, rp_, ci_;
    bool capture_ = false;
    std::vector<gap::solver::IterationState> states_;
    DeviceBuffer d_y_, d_s_, d_u_, d_v_, d_vo_, d_it_, d_st_, d_fm_, d_f_, d_cap_, d_sb_;
};

}  // namespace gapb200

extern "C" {
gap::solver::IPowerFlowSolver* create_gpu_powerflow_solver() {
    return new gapb200::B200NewtonRaphson();
}
void destroy_gpu_powerflow_solver(gap::solver::IPowerFlowSolver* instance) { delete instance; }
}
