// Host side of the Newton-Raphson engine: plan upload, batch state, the device-resident
// iteration loop (CUDA graph with a conditional while node), and the gapk_nr_* C ABI.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/gapk.h"
#include "internal.h"
#include "nr_kernels.cuh"

namespace gapk {

namespace {
thread_local std::string g_err = "no error";
}
void set_error(std::string const& msg) { g_err = msg; }

#define GAPK_CUDA_TRY(expr)                                                         \
    do {                                                                            \
        cudaError_t e__ = (expr);                                                   \
        if (e__ != cudaSuccess) {                                                   \
            set_error(std::string(#expr) + ": " + cudaGetErrorString(e__));         \
            return e__ == cudaErrorMemoryAllocation ? GAPK_ENOMEM : GAPK_ECUDA;     \
        }                                                                           \
    } while (0)

// ---- device buffers -------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(DevBuf const&) = delete;
    DevBuf& operator=(DevBuf const&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = n;
        if (n == 0) return GAPK_OK;
        GAPK_CUDA_TRY(cudaMalloc(&p, n));
        return GAPK_OK;
    }
    template <typename V>
    int upload(std::vector<V> const& v) {
        int rc = alloc(v.size() * sizeof(V));
        if (rc) return rc;
        if (!v.empty()) GAPK_CUDA_TRY(cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice));
        return GAPK_OK;
    }
    template <typename P>
    P* as() const {
        return reinterpret_cast<P*>(p);
    }
};

}  // namespace gapk

using namespace gapk;

struct gapk_nr_plan_s {
    NRPlanHost h;
    std::vector<int> y_row_ptr, y_col;
    // device copy (current device at first upload)
    bool uploaded = false;
    int device = -1;
    DevBuf d_yrp, d_ycol, d_bt, d_nob, d_si, d_ss, d_sa, d_lp, d_ln, d_fa, d_tg, d_pr, d_fb,
        d_sc, d_lptr, d_lidx, d_rptr, d_rl, d_arp, d_ar, d_var, d_eq, d_schur, d_aslots, d_acp, d_ac;
    PlanDev dev{};

    int upload() {
        if (uploaded) return GAPK_OK;
        int rc = 0;
        auto up = [&](DevBuf& b, std::vector<int> const& v) {
            if (!rc) rc = b.upload(v);
        };
        up(d_yrp, y_row_ptr);
        up(d_ycol, y_col);
        up(d_bt, h.bus_type);
        up(d_nob, h.node_of_bus);
        up(d_si, h.slot_info);
        up(d_ss, h.slot_src);
        up(d_sa, h.slot_a);
        up(d_lp, h.level_ptr);
        up(d_ln, h.level_nodes);
        up(d_fa, h.fa_ptr);
        up(d_tg, h.targets);
        up(d_pr, h.pairs);
        up(d_fb, h.fb_ptr);
        up(d_sc, h.scale);
        up(d_lptr, h.lptr);
        up(d_lidx, h.lidx);
        up(d_rptr, h.rptr);
        up(d_rl, h.rlist);
        up(d_arp, h.arow_ptr);
        up(d_ar, h.arow);
        up(d_var, h.var_of_comp);
        up(d_eq, h.eq_of_comp);
        up(d_schur, h.schur);
        up(d_aslots, h.a_slots);
        up(d_acp, h.acol_ptr);
        up(d_ac, h.acol);
        if (rc) return rc;
        cudaGetDevice(&device);
        dev.n_bus = h.n_bus;
        dev.nb = h.nb;
        dev.nnz_y = h.nnz_y;
        dev.n_slots = h.n_slots;
        dev.nnz_l = h.nnz_l;
        dev.n_levels = h.n_levels;
        dev.n_a = h.n_a;
        dev.jac_mode = h.jac_mode;
        dev.ns = h.ns;
        dev.n_tail = h.n_tail;
        dev.n_schur = static_cast<int>(h.schur.size() / 4);
        dev.schur = d_schur.as<int4>();
        dev.a_slots = d_aslots.as<int>();
        dev.acol_ptr = d_acp.as<int>();
        dev.acol = d_ac.as<int2>();
        dev.y_row_ptr = d_yrp.as<int>();
        dev.y_col = d_ycol.as<int>();
        dev.bus_type = d_bt.as<int>();
        dev.node_of_bus = d_nob.as<int>();
        dev.slot_info = d_si.as<int4>();
        dev.slot_src = d_ss.as<int>();
        dev.slot_a = d_sa.as<int>();
        dev.level_ptr = d_lp.as<int>();
        dev.level_nodes = d_ln.as<int>();
        dev.fa_ptr = d_fa.as<int>();
        dev.targets = d_tg.as<int4>();
        dev.pairs = d_pr.as<int2>();
        dev.fb_ptr = d_fb.as<int>();
        dev.scale = d_sc.as<int2>();
        dev.lptr = d_lptr.as<int>();
        dev.lidx = d_lidx.as<int>();
        dev.rptr = d_rptr.as<int>();
        dev.rlist = d_rl.as<int2>();
        dev.arow_ptr = d_arp.as<int>();
        dev.arow = d_ar.as<int2>();
        uploaded = true;
        return GAPK_OK;
    }
};

struct gapk_nr_batch_s {
    gapk_nr_plan plan = nullptr;
    int n_scen = 0, sw = 8, G = 0, precision = 0, y_shared = 1, threads = 256, use_graph = 1;
    int dense_fused = 0;
    DevBuf V, Sspec, Scalc, Y, F, A64, rhs, dx, res, X, Dt, mis, state, solving, singular,
        iters, status, fmis, gsolve, giter, grefine, gfactor, ctrl, tol;
    int dense_w = 0;          // panel width of the one-CTA-per-scenario dense LU (0: not used)
    size_t dense_smem = 0;    // its dynamic shared memory
    bool dense_split = false; // factorise the tail with the split kernels
    bool dense_tc = false;    // FP32 tail: trailing updates on the tensor cores (either LU path)
    BatchDev dev{};
    // graph cache
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_refine = -1;
    int cur_refine = 0;
    ~gapk_nr_batch_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

inline unsigned blocks_for(long items, int threads) {
    return static_cast<unsigned>((items + threads - 1) / threads);
}

template <typename T, int SW>
void launch_solve(gapk_nr_batch b, cudaStream_t st, const double2* rhs, double2* out, int acc) {
    PlanDev const& P = b->plan->dev;
    BatchDev const& B = b->dev;
    k_solve_fwd<T, SW><<<b->G, b->threads, 0, st>>>(P, B, rhs, acc);
    if (P.n_tail > 0)
        k_dense_solve<T, SW><<<b->G * SW, 256, dense_solve_smem(P.n_tail, sizeof(T)), st>>>(P, B, out, acc);
    k_solve_bwd<T, SW><<<b->G, b->threads, 0, st>>>(P, B, out, acc);
}

template <typename T, int SW>
void launch_factor(gapk_nr_batch b, cudaStream_t st) {
    PlanDev const& P = b->plan->dev;
    BatchDev const& B = b->dev;
    k_factor<T, SW><<<b->G, b->threads, 0, st>>>(P, B);
    if (P.n_tail > 0) {
        dim3 gs(blocks_for((long)P.n_schur * SW, 256), b->G);
        k_schur<T, SW><<<gs, 256, 0, st>>>(P, B);
        if (b->dense_split)
            launch_dense_lu_split<T>(b->G * SW, st, B, 2 * P.n_tail, b->dense_tc);
        else
            launch_dense_lu<T>(b->dense_w, b->G * SW, b->dense_smem, st, B, 2 * P.n_tail, b->dense_tc);
    }
}

template <typename T, int SW>
void launch_body(gapk_nr_batch b, cudaStream_t st, int use_cond, cudaGraphConditionalHandle h) {
    PlanDev const& P = b->plan->dev;
    BatchDev const& B = b->dev;
    const int G = b->G;
    k_mismatch<SW><<<mismatch_grid<SW>(P, G), 256, 0, st>>>(P, B);
    k_check<SW><<<1, 1024, 0, st>>>(B, use_cond, h);
    dim3 gj(blocks_for((long)P.n_a * SW, 256), G);
    k_jfill<T, SW><<<gj, 256, 0, st>>>(P, B);
    launch_factor<T, SW>(b, st);
    launch_solve<T, SW>(b, st, B.rhs, B.dx, 0);
    for (int r = 0; r < b->cur_refine; ++r) {
        dim3 gr(blocks_for((long)P.nb * SW, 256), G);
        k_residual<SW><<<gr, 256, 0, st>>>(P, B);
        launch_solve<T, SW>(b, st, B.res, B.dx, 1);
    }
    dim3 gu(blocks_for((long)P.n_bus * SW, 256), G);
    k_update<SW><<<gu, 256, 0, st>>>(P, B);
}

template <int SW>
void launch_load(gapk_nr_batch b, const gapk_nr_inputs* in, cudaStream_t st) {
    PlanDev const& P = b->plan->dev;
    dim3 g(blocks_for((long)P.n_bus * SW, 256), b->G);
    k_load<SW><<<g, 256, 0, st>>>(P, b->dev, reinterpret_cast<const double2*>(in->d_y),
                                  reinterpret_cast<const double2*>(in->d_s_spec),
                                  reinterpret_cast<const double2*>(in->d_v_init), in->d_u_pu,
                                  in->v_init_shared);
}

template <int SW>
void launch_store(gapk_nr_batch b, const gapk_nr_outputs* out, cudaStream_t st) {
    PlanDev const& P = b->plan->dev;
    long total = (long)b->n_scen * P.n_bus;
    k_store<SW><<<blocks_for(total, 256), 256, 0, st>>>(
        P, b->dev, reinterpret_cast<double2*>(out->d_v), out->d_iterations, out->d_status,
        out->d_final_mismatch);
}

// dispatch on (precision, lanes)
template <template <typename, int> class F, typename... A>
int dispatch_tsw(int precision, int sw, A&&... a) {
#define GAPK_CASE(T, S) F<T, S>::run(std::forward<A>(a)...)
    if (precision == GAPK_PREC_FP64) {
        switch (sw) {
            case 1: GAPK_CASE(double, 1); return 0;
            case 2: GAPK_CASE(double, 2); return 0;
            case 4: GAPK_CASE(double, 4); return 0;
            case 8: GAPK_CASE(double, 8); return 0;
        }
    } else {
        switch (sw) {
            case 1: GAPK_CASE(float, 1); return 0;
            case 2: GAPK_CASE(float, 2); return 0;
            case 4: GAPK_CASE(float, 4); return 0;
            case 8: GAPK_CASE(float, 8); return 0;
        }
    }
#undef GAPK_CASE
    return -1;
}

template <typename T, int SW>
struct BodyOp {
    static void run(gapk_nr_batch b, cudaStream_t st, int uc, cudaGraphConditionalHandle h) {
        launch_body<T, SW>(b, st, uc, h);
    }
};
template <typename T, int SW>
struct LoadOp {
    static void run(gapk_nr_batch b, const gapk_nr_inputs* in, cudaStream_t st) {
        launch_load<SW>(b, in, st);
    }
};
template <typename T, int SW>
struct StoreOp {
    static void run(gapk_nr_batch b, const gapk_nr_outputs* out, cudaStream_t st) {
        launch_store<SW>(b, out, st);
    }
};
template <typename T, int SW>
struct StageOp {
    static void run(gapk_nr_batch b, int which, cudaStream_t st) {
        PlanDev const& P = b->plan->dev;
        BatchDev const& B = b->dev;
        const int G = b->G;
        switch (which) {
            case 0:
                k_mismatch<SW><<<mismatch_grid<SW>(P, G), 256, 0, st>>>(P, B);
                break;
            case 1: {
                dim3 gj(blocks_for((long)P.n_a * SW, 256), G);
                k_jfill<T, SW><<<gj, 256, 0, st>>>(P, B);
                break;
            }
            case 2:
                launch_factor<T, SW>(b, st);
                break;
            case 3:
                launch_solve<T, SW>(b, st, B.rhs, B.dx, 0);
                for (int r = 0; r < b->cur_refine; ++r) {
                    dim3 gr(blocks_for((long)P.nb * SW, 256), G);
                    k_residual<SW><<<gr, 256, 0, st>>>(P, B);
                    launch_solve<T, SW>(b, st, B.res, B.dx, 1);
                }
                break;
            case 4: {
                dim3 gu(blocks_for((long)P.n_bus * SW, 256), G);
                k_update<SW><<<gu, 256, 0, st>>>(P, B);
                break;
            }
        }
    }
};
template <typename T, int SW>
struct KernelOp {
    static void run(gapk_nr_batch b, int which, cudaStream_t st) {
        PlanDev const& P = b->plan->dev;
        BatchDev const& B = b->dev;
        const int G = b->G;
        switch (which) {
            case 0: k_mismatch<SW><<<mismatch_grid<SW>(P, G), 256, 0, st>>>(P, B); break;
            case 1: k_jfill<T, SW><<<dim3(blocks_for((long)P.n_a * SW, 256), G), 256, 0, st>>>(P, B); break;
            case 2: k_factor<T, SW><<<G, b->threads, 0, st>>>(P, B); break;
            case 3:
                if (P.n_tail > 0)
                    k_schur<T, SW><<<dim3(blocks_for((long)P.n_schur * SW, 256), G), 256, 0, st>>>(P, B);
                break;
            case 4:
                if (P.n_tail > 0)
                    if (b->dense_split)
                        launch_dense_lu_split<T>(G * SW, st, B, 2 * P.n_tail, b->dense_tc);
                    else
                        launch_dense_lu<T>(b->dense_w, G * SW, b->dense_smem, st, B, 2 * P.n_tail, b->dense_tc);
                break;
            case 5: k_solve_fwd<T, SW><<<G, b->threads, 0, st>>>(P, B, B.rhs, 0); break;
            case 6:
                if (P.n_tail > 0)
                    k_dense_solve<T, SW><<<G * SW, 256, dense_solve_smem(P.n_tail, sizeof(T)), st>>>(P, B, B.dx, 0);
                break;
            case 7: k_solve_bwd<T, SW><<<G, b->threads, 0, st>>>(P, B, B.dx, 0); break;
            case 8: k_update<SW><<<dim3(blocks_for((long)P.n_bus * SW, 256), G), 256, 0, st>>>(P, B); break;
            case 9:
                if (B.A64) k_residual<SW><<<dim3(blocks_for((long)P.nb * SW, 256), G), 256, 0, st>>>(P, B);
                break;
        }
    }
};
template <typename T, int SW>
void launch_solve_t(gapk_nr_batch b, cudaStream_t st, const double2* rhs, double2* out, int acc) {
    PlanDev const& P = b->plan->dev;
    BatchDev const& B = b->dev;
    k_solve_fwd_t<T, SW><<<b->G, b->threads, 0, st>>>(P, B, rhs);
    if (P.n_tail > 0)
        k_dense_solve_t<T, SW><<<b->G * SW, 256, 2 * P.n_tail * sizeof(T), st>>>(P, B, out, acc);
    k_solve_bwd_t<T, SW><<<b->G, b->threads, 0, st>>>(P, B, out, acc);
}

template <typename T, int SW>
struct AdjointOp {
    static void run(gapk_nr_batch b, const double* dvm, const double* dva, double* dp, double* dq,
                    cudaStream_t st) {
        PlanDev const& P = b->plan->dev;
        BatchDev const& B = b->dev;
        const int G = b->G;
        k_adj_prep<SW><<<blocks_for((long)G * SW, 256), 256, 0, st>>>(B);
        k_mismatch<SW><<<mismatch_grid<SW>(P, G), 256, 0, st>>>(P, B);
        k_jfill<T, SW><<<dim3(blocks_for((long)P.n_a * SW, 256), G), 256, 0, st>>>(P, B);
        launch_factor<T, SW>(b, st);
        k_adj_rhs<SW><<<dim3(blocks_for((long)P.n_bus * SW, 256), G), 256, 0, st>>>(P, B, dvm, dva);
        launch_solve_t<T, SW>(b, st, B.rhs, B.dx, 0);
        if (B.A64) {
            k_residual_t<SW><<<dim3(blocks_for((long)P.nb * SW, 256), G), 256, 0, st>>>(P, B);
            launch_solve_t<T, SW>(b, st, B.res, B.dx, 1);
        }
        k_adj_out<SW><<<blocks_for((long)b->n_scen * P.n_bus, 256), 256, 0, st>>>(P, B, dp, dq);
    }
};
template <typename T, int SW>
struct AdjBranchOp {
    static void run(gapk_nr_batch b, int m, const int* f, const int* t, const double* brp, double* dr,
                    double* dx, cudaStream_t st) {
        k_adj_branch<SW><<<blocks_for((long)b->n_scen * m, 256), 256, 0, st>>>(
            b->plan->dev, b->dev, m, f, t, brp, dr, dx);
    }
};

template <typename T, int SW>
struct ToRefOp {
    static void run(gapk_nr_batch b, const double2* src, const int* map, int n_out, double sign,
                    double* dst, cudaStream_t st) {
        PlanDev const& P = b->plan->dev;
        long total = (long)b->n_scen * P.nb;
        if (total == 0) return;
        k_node_to_ref<SW><<<blocks_for(total, 256), 256, 0, st>>>(src, P.nb, b->n_scen, n_out,
                                                                   map, sign, dst);
    }
};

template <typename T, int SW>
struct StateOp {
    static void run(gapk_nr_batch b, double2* v, double2* i, double2* s, cudaStream_t st) {
        long total = (long)b->n_scen * b->plan->dev.n_bus;
        if (total == 0) return;
        k_state<SW><<<blocks_for(total, 256), 256, 0, st>>>(b->plan->dev, b->dev, v, i, s);
    }
};

int check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    return GAPK_OK;
}

int build_graph(gapk_nr_batch b, cudaStream_t st) {
    if (b->exec && b->graph_refine == b->cur_refine) return GAPK_OK;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    GAPK_CUDA_TRY(cudaGraphCreate(&b->graph, 0));
    cudaGraphConditionalHandle h;
    GAPK_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, b->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    GAPK_CUDA_TRY(cudaGraphAddNode(&node, b->graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    // capture the iteration body into the while node's graph
    cudaStream_t cs;
    GAPK_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        set_error(std::string("cudaStreamBeginCaptureToGraph: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    dispatch_tsw<BodyOp>(b->precision, b->sw, b, cs, 1, h);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        set_error(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    GAPK_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_refine = b->cur_refine;
    (void)st;
    return GAPK_OK;
}

int validate_inputs(gapk_nr_batch b, const gapk_nr_inputs* in) {
    if (!in || !in->d_y || !in->d_s_spec) {
        set_error("inputs: d_y and d_s_spec are required");
        return GAPK_EINVAL;
    }
    if (in->max_iterations < 0 || in->refine < 0 || in->refine > 8 ||
        (in->policy < GAPK_POLICY_REFERENCE || in->policy > GAPK_POLICY_CLAMPED)) {
        set_error("inputs: bad max_iterations / refine / policy");
        return GAPK_EINVAL;
    }
    if (in->refine > 0 && !b->A64.p) {
        set_error("inputs: refine > 0 needs a batch created with precision FP32");
        return GAPK_EINVAL;
    }
    if (!(in->refine_below >= 0.0) || !(in->reuse_below >= 0.0)) {
        set_error("inputs: refine_below and reuse_below must be >= 0");
        return GAPK_EINVAL;
    }
    if (in->reuse_below > 0.0 && in->refine < 1) {
        set_error("inputs: reuse_below > 0 needs refine >= 1");
        return GAPK_EINVAL;
    }
    return GAPK_OK;
}

int load_inputs(gapk_nr_batch b, const gapk_nr_inputs* in, cudaStream_t st) {
    if (!in || !in->d_y || !in->d_s_spec) {
        set_error("inputs: d_y and d_s_spec are required");
        return GAPK_EINVAL;
    }
    if (in->max_iterations < 0 || in->refine < 0 || in->refine > 8 ||
        (in->policy < GAPK_POLICY_REFERENCE || in->policy > GAPK_POLICY_CLAMPED)) {
        set_error("inputs: bad max_iterations / refine / policy");
        return GAPK_EINVAL;
    }
    if (in->refine > 0 && !b->A64.p) {
        set_error("inputs: refine > 0 needs a batch created with precision FP32");
        return GAPK_EINVAL;
    }
    b->cur_refine = in->refine;
    // iteration, max iterations, loop flag, step policy, iterations run, device wait error
    int ctrl[6] = {0, in->max_iterations, 1, in->policy, 0, 0};
    GAPK_CUDA_TRY(cudaMemcpyAsync(b->ctrl.p, ctrl, sizeof(ctrl), cudaMemcpyHostToDevice, st));
    if (!(in->refine_below >= 0.0) || !(in->reuse_below >= 0.0)) {
        set_error("inputs: refine_below and reuse_below must be >= 0");
        return GAPK_EINVAL;
    }
    if (in->reuse_below > 0.0 && in->refine < 1) {
        set_error("inputs: reuse_below > 0 needs refine >= 1");
        return GAPK_EINVAL;
    }
    double tol[3] = {in->tolerance, in->refine_below, in->reuse_below};
    GAPK_CUDA_TRY(cudaMemcpyAsync(b->tol.p, tol, sizeof(tol), cudaMemcpyHostToDevice, st));
    dispatch_tsw<LoadOp>(b->precision, b->sw, b, in, st);
    return check_launch();
}

}  // namespace

extern "C" {

const char* gapk_last_error(void) { return g_err.c_str(); }
int gapk_version(void) { return 100; }
int gapk_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int gapk_nr_plan_create(int n_bus, int nnz_y, const int* h_y_row_ptr, const int* h_y_col_idx,
                        const int* h_bus_type, const gapk_nr_plan_options* opt,
                        gapk_nr_plan* out) {
    TraceRange tr("gapk_nr_plan_create: ordering and symbolic analysis");
    if (!out || n_bus < 0 || nnz_y < 0 || !h_y_row_ptr || (nnz_y && !h_y_col_idx) ||
        (n_bus && !h_bus_type)) {
        set_error("gapk_nr_plan_create: bad arguments");
        return GAPK_EINVAL;
    }
    int jac = opt ? opt->jacobian_mode : GAPK_JAC_REFERENCE;
    int ord = opt ? opt->ordering : GAPK_ORDER_MINDEG;
    int dmin = opt ? opt->dense_min : 0;
    if (dmin == 0) dmin = 16;
    if ((jac != 0 && jac != 1) || (ord != 0 && ord != 1)) {
        set_error("gapk_nr_plan_create: bad options");
        return GAPK_EINVAL;
    }
    auto p = std::make_unique<gapk_nr_plan_s>();
    try {
        if (!analyze_nr(n_bus, nnz_y, h_y_row_ptr, h_y_col_idx, h_bus_type, jac, ord, dmin, p->h))
            return GAPK_EINVAL;
    } catch (std::bad_alloc const&) {
        set_error("gapk_nr_plan_create: host allocation failed");
        return GAPK_ENOMEM;
    }
    p->y_row_ptr.assign(h_y_row_ptr, h_y_row_ptr + n_bus + 1);
    p->y_col.assign(h_y_col_idx, h_y_col_idx + nnz_y);
    *out = p.release();
    return GAPK_OK;
}

int gapk_nr_plan_destroy(gapk_nr_plan p) {
    delete p;
    return GAPK_OK;
}

int gapk_nr_plan_get_info(gapk_nr_plan p, gapk_nr_plan_info* info) {
    if (!p || !info) {
        set_error("gapk_nr_plan_get_info: null argument");
        return GAPK_EINVAL;
    }
    auto const& h = p->h;
    info->n_bus = h.n_bus;
    info->n_block = h.nb;
    info->n_pq = h.n_pq;
    info->n_pv = h.n_pv;
    info->n_slack = h.n_slack;
    info->n_vars = h.n_vars;
    info->nnz_y = h.nnz_y;
    info->nnz_l_blocks = h.nnz_l;
    info->n_slots = h.n_slots;
    info->n_a_blocks = h.n_a;
    info->n_levels = h.n_levels;
    info->n_pairs = h.n_pairs;
    info->n_rows_pairs = h.nnz_l;
    info->max_level_width = h.max_level_width;
    info->n_tail = h.n_tail;
    int64_t sp = 0;
    for (size_t t = 0; t + 3 < h.schur.size(); t += 4) sp += h.schur[t + 2] - h.schur[t + 1];
    info->n_schur_pairs = sp;
    return GAPK_OK;
}

int64_t gapk_nr_plan_export(gapk_nr_plan p, int what, int* h_buf) {
    if (!p) return GAPK_EINVAL;
    auto const& h = p->h;
    std::vector<int> const* v = nullptr;
    switch (what) {
        case 0: v = &h.bus_of_node; break;
        case 1: v = &h.node_pq; break;
        case 2: v = &h.lptr; break;
        case 3: v = &h.lidx; break;
        case 4: v = &h.level_ptr; break;
        case 5: v = &h.level_nodes; break;
        case 6: v = &h.slot_info; break;
        case 7: {
            // slot_src_ptr derived from slot_info
            int64_t n = h.n_slots + 1;
            if (h_buf) {
                for (int s = 0; s < h.n_slots; ++s) h_buf[s] = h.slot_info[4 * s + 2];
                h_buf[h.n_slots] = static_cast<int>(h.slot_src.size());
            }
            return n;
        }
        case 8: v = &h.slot_src; break;
        case 9: v = &h.fa_ptr; break;
        case 10: v = &h.targets; break;
        case 11: v = &h.pairs; break;
        case 12: v = &h.fb_ptr; break;
        case 13: v = &h.scale; break;
        case 14: v = &h.rptr; break;
        case 15: v = &h.rlist; break;
        case 16: v = &h.var_of_comp; break;
        case 17: v = &h.eq_of_comp; break;
        case 18: v = &h.slot_a; break;
        case 19: v = &h.arow_ptr; break;
        case 20: v = &h.arow; break;
        case 21: v = &h.schur; break;
        default:
            set_error("gapk_nr_plan_export: unknown selector");
            return GAPK_EINVAL;
    }
    if (h_buf && !v->empty()) std::memcpy(h_buf, v->data(), v->size() * sizeof(int));
    return static_cast<int64_t>(v->size());
}

int gapk_nr_batch_create(gapk_nr_plan p, int n_scen, const gapk_nr_batch_options* opt,
                         gapk_nr_batch* out) {
    TraceRange tr("gapk_nr_batch_create");
    if (!p || !out || n_scen <= 0) {
        set_error("gapk_nr_batch_create: bad arguments");
        return GAPK_EINVAL;
    }
    auto b = std::make_unique<gapk_nr_batch_s>();
    b->plan = p;
    b->n_scen = n_scen;
    b->precision = opt ? opt->precision : GAPK_PREC_FP64;
    b->y_shared = opt ? (opt->y_shared ? 1 : 0) : 1;
    int lanes = opt ? opt->lanes : 0;
    if (lanes == 0) lanes = n_scen >= 8 ? 8 : (n_scen >= 4 ? 4 : (n_scen >= 2 ? 2 : 1));
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) {
        set_error("gapk_nr_batch_create: lanes must be 1, 2, 4 or 8");
        return GAPK_EINVAL;
    }
    if (b->precision != GAPK_PREC_FP64 && b->precision != GAPK_PREC_FP32) {
        set_error("gapk_nr_batch_create: bad precision");
        return GAPK_EINVAL;
    }
    b->sw = lanes;
    int thr = opt ? opt->threads : 0;
    if (thr == 0) thr = lanes == 1 ? 512 : 256;
    if (thr < 32 || thr > 1024 || thr % 32) {
        set_error("gapk_nr_batch_create: threads must be a multiple of 32 in [32, 1024]");
        return GAPK_EINVAL;
    }
    b->threads = thr;
    b->use_graph = opt ? opt->use_graph : 1;
    b->dense_fused = opt ? opt->dense_fused : 0;
    int rc = p->upload();
    if (rc) return rc;
    auto const& h = p->h;
    const size_t G = (n_scen + lanes - 1) / lanes;
    b->G = static_cast<int>(G);
    const size_t L = G * lanes;
    const size_t esz = b->precision == GAPK_PREC_FP64 ? 8 : 4;
    const size_t n = h.n_bus, nb = h.nb;
    auto A = [&](DevBuf& d, size_t bytes) {
        if (!rc) rc = d.alloc(bytes < 16 ? 16 : bytes);
    };
    A(b->V, L * n * 16);
    A(b->Sspec, L * n * 16);
    A(b->Scalc, L * n * 16);
    A(b->Y, (b->y_shared ? (size_t)h.nnz_y : L * h.nnz_y) * 16);
    A(b->F, L * (size_t)h.n_slots * 4 * esz);
    if (b->precision == GAPK_PREC_FP32) A(b->A64, L * (size_t)h.n_a * 32);
    A(b->rhs, L * nb * 16);
    A(b->dx, L * nb * 16);
    A(b->res, L * nb * 16);
    A(b->X, L * nb * 2 * esz);
    if (h.n_tail > 0) {
        // Dense-tail LU: one CTA per scenario (k_dense_lu, the panel in shared memory) when
        // there are enough scenarios to fill the GPU (or the caller says that concurrent
        // batches will, dense_fused) and the panel fits; otherwise the split kernels, which
        // spread each scenario's trailing update over many CTAs and have no shared-memory
        // limit on the tail size.
        const size_t N = 2 * (size_t)h.n_tail;
        const size_t smem_max = 232448 - 1024;  // opt-in shared memory per block, less static
        b->dense_w = 0;
        for (int w : {32, 16, 8}) {
            size_t bytes = dense_lu_elems((int)N, w) * esz;
            if (bytes <= smem_max && (w < 32 || esz == 4 || N <= 200)) {
                b->dense_w = w;
                b->dense_smem = bytes;
                break;
            }
        }
        int dev = 0, n_sm = 148;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        b->dense_split = b->dense_w == 0 || (L < 2 * (size_t)n_sm && !b->dense_fused);
        // FP32 tails have their trailing updates on the tensor cores unless the caller asks for
        // CUDA-core FMA: k_dense_lu_tc one CTA per scenario (panel width 32), k_dlu_update_tc
        // on the split path
        b->dense_tc = !(opt && opt->dense_fma) && b->precision == GAPK_PREC_FP32 &&
                      (b->dense_split || b->dense_w == 32);
        A(b->Dt, L * N * dense_ld((int)N) * esz);
        cudaError_t e = cudaSuccess;
        if (!b->dense_split)
            e = b->precision == GAPK_PREC_FP64
                    ? dense_lu_attributes<double>(b->dense_w, b->dense_smem, false)
                    : dense_lu_attributes<float>(b->dense_w, b->dense_smem, b->dense_tc);
        else if (b->dense_tc)
            e = split_lu_attributes();
        if (e != cudaSuccess) {
            set_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
            return GAPK_ECUDA;
        }
    }
    A(b->mis, L * 8);
    A(b->state, L * 4);
    A(b->solving, L * 4);
    A(b->singular, L * 4);
    A(b->iters, L * 4);
    A(b->status, L * 4);
    A(b->fmis, L * 8);
    A(b->gsolve, G * 4);
    A(b->giter, G * 4);
    A(b->ctrl, 8 * 4);
    A(b->grefine, G * 4);
    A(b->gfactor, G * 4);
    A(b->tol, 24);
    if (rc) return rc;
    // per-group flags start true (any non-zero byte pattern): callers that factorise without
    // a load (the general LU) refine and refactorise as before
    GAPK_CUDA_TRY(cudaMemset(b->grefine.p, 1, b->grefine.bytes));
    GAPK_CUDA_TRY(cudaMemset(b->gfactor.p, 1, b->gfactor.bytes));
    // control words: [5] the tensor-core LU's wait error, [6] its wait test (both off)
    GAPK_CUDA_TRY(cudaMemset(b->ctrl.p, 0, b->ctrl.bytes));
    BatchDev& d = b->dev;
    d.n_scen = n_scen;
    d.n_groups = b->G;
    d.sw = lanes;
    d.y_shared = b->y_shared;
    d.V = b->V.as<double2>();
    d.Sspec = b->Sspec.as<double2>();
    d.Scalc = b->Scalc.as<double2>();
    d.Y = b->Y.as<double2>();
    d.F = b->F.p;
    d.A64 = b->A64.as<double>();
    d.rhs = b->rhs.as<double2>();
    d.dx = b->dx.as<double2>();
    d.res = b->res.as<double2>();
    d.X = b->X.p;
    d.Dt = b->Dt.p;
    d.mis_bits = b->mis.as<unsigned long long>();
    d.state = b->state.as<int>();
    d.solving = b->solving.as<int>();
    d.singular = b->singular.as<int>();
    d.iters = b->iters.as<int>();
    d.status = b->status.as<int>();
    d.final_mis = b->fmis.as<double>();
    d.gsolve = b->gsolve.as<int>();
    d.giter = b->giter.as<int>();
    d.ctrl = b->ctrl.as<int>();
    d.tol = b->tol.as<double>();
    d.grefine = b->grefine.as<int>();
    d.gfactor = b->gfactor.as<int>();
    *out = b.release();
    return GAPK_OK;
}

int gapk_nr_batch_destroy(gapk_nr_batch b) {
    delete b;
    return GAPK_OK;
}

int gapk_nr_batch_lanes(gapk_nr_batch b) { return b ? b->sw : 0; }

int64_t gapk_nr_batch_device_bytes(gapk_nr_batch b) {
    if (!b) return 0;
    int64_t s = 0;
    for (DevBuf* d : {&b->V, &b->Sspec, &b->Scalc, &b->Y, &b->F, &b->A64, &b->rhs, &b->dx,
                      &b->res, &b->X, &b->Dt, &b->mis, &b->state, &b->solving, &b->singular, &b->iters,
                      &b->status, &b->fmis, &b->gsolve, &b->giter, &b->grefine, &b->gfactor, &b->ctrl, &b->tol})
        s += static_cast<int64_t>(d->bytes);
    return s;
}

int gapk_nr_solve(gapk_nr_batch b, const gapk_nr_inputs* in, const gapk_nr_outputs* out,
                  void* stream) {
    TraceRange tr("gapk_nr_solve");
    if (!b) {
        set_error("gapk_nr_solve: null batch");
        return GAPK_EINVAL;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = load_inputs(b, in, st);
    if (rc) return rc;
    if (in->max_iterations > 0) {
        if (b->use_graph) {
            rc = build_graph(b, st);
            if (rc) return rc;
            GAPK_CUDA_TRY(cudaGraphLaunch(b->exec, st));
        } else {
            // host-driven loop: one synchronisation per iteration
            for (int it = 0; it < in->max_iterations; ++it) {
                dispatch_tsw<BodyOp>(b->precision, b->sw, b, st, 0,
                                     cudaGraphConditionalHandle{});
                rc = check_launch();
                if (rc) return rc;
                int any = 0;
                GAPK_CUDA_TRY(cudaMemcpyAsync(&any, b->dev.ctrl + 2, sizeof(int),
                                              cudaMemcpyDeviceToHost, st));
                GAPK_CUDA_TRY(cudaStreamSynchronize(st));
                if (!any) break;
            }
        }
    }
    if (out) {
        dispatch_tsw<StoreOp>(b->precision, b->sw, b, out, st);
        rc = check_launch();
        if (rc) return rc;
    }
    return GAPK_OK;
}

int gapk_nr_last_loop_count(gapk_nr_batch b, void* stream, int* h_loops) {
    if (!b || !h_loops) return GAPK_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GAPK_CUDA_TRY(cudaMemcpyAsync(h_loops, b->dev.ctrl + 4, sizeof(int), cudaMemcpyDeviceToHost,
                                  st));
    GAPK_CUDA_TRY(cudaStreamSynchronize(st));
    return GAPK_OK;
}

int gapk_nr_stage_load(gapk_nr_batch b, const gapk_nr_inputs* in, void* stream) {
    if (!b) return GAPK_EINVAL;
    return load_inputs(b, in, static_cast<cudaStream_t>(stream));
}

static int stage(gapk_nr_batch b, int which, void* stream) {
    if (!b) {
        set_error("stage: null batch");
        return GAPK_EINVAL;
    }
    static const char* names[] = {"gapk stage: mismatch", "gapk stage: jacobian",
                                  "gapk stage: factor", "gapk stage: solve", "gapk stage: update"};
    TraceRange tr(which >= 0 && which < 5 ? names[which] : "gapk stage");
    dispatch_tsw<StageOp>(b->precision, b->sw, b, which, static_cast<cudaStream_t>(stream));
    return check_launch();
}
int gapk_nr_stage_mismatch(gapk_nr_batch b, void* s) { return stage(b, 0, s); }
int gapk_nr_stage_jacobian(gapk_nr_batch b, void* s) { return stage(b, 1, s); }
int gapk_nr_stage_factor(gapk_nr_batch b, void* s) { return stage(b, 2, s); }
int gapk_nr_stage_solve(gapk_nr_batch b, void* s) { return stage(b, 3, s); }

int gapk_nr_stage_kernel(gapk_nr_batch b, int kernel, void* stream) {
    if (!b || kernel < 0 || kernel > 9) {
        set_error("gapk_nr_stage_kernel: bad arguments");
        return GAPK_EINVAL;
    }
    dispatch_tsw<KernelOp>(b->precision, b->sw, b, kernel, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int gapk_nr_adjoint(gapk_nr_batch b, const double* d_dl_dvm, const double* d_dl_dva,
                    double* d_dl_dp, double* d_dl_dq, void* stream) {
    if (!b || !d_dl_dvm || !d_dl_dva) {
        set_error("gapk_nr_adjoint: bad arguments");
        return GAPK_EINVAL;
    }
    dispatch_tsw<AdjointOp>(b->precision, b->sw, b, d_dl_dvm, d_dl_dva, d_dl_dp, d_dl_dq,
                            static_cast<cudaStream_t>(stream));
    return check_launch();
}

int gapk_nr_adjoint_branch(gapk_nr_batch b, int n_branch, const int* d_from, const int* d_to,
                           const double* d_branch_pu, double* d_dl_dr, double* d_dl_dx,
                           void* stream) {
    if (!b || n_branch < 0 || (n_branch > 0 && (!d_from || !d_to || !d_branch_pu || !d_dl_dr ||
                                                !d_dl_dx))) {
        set_error("gapk_nr_adjoint_branch: bad arguments");
        return GAPK_EINVAL;
    }
    if (n_branch == 0) return GAPK_OK;
    dispatch_tsw<AdjBranchOp>(b->precision, b->sw, b, n_branch, d_from, d_to, d_branch_pu,
                              d_dl_dr, d_dl_dx, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int gapk_nr_stage_get_correction(gapk_nr_batch b, double* d_dx, void* stream) {
    if (!b || !d_dx) return GAPK_EINVAL;
    dispatch_tsw<ToRefOp>(b->precision, b->sw, b, b->dev.dx, b->plan->d_var.as<int>(),
                          b->plan->h.n_vars, 1.0, d_dx, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int gapk_nr_stage_get_mismatch(gapk_nr_batch b, double* d_f, void* stream) {
    if (!b || !d_f) return GAPK_EINVAL;
    dispatch_tsw<ToRefOp>(b->precision, b->sw, b, b->dev.rhs, b->plan->d_eq.as<int>(),
                          b->plan->h.n_vars, -1.0, d_f, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int gapk_nr_step(gapk_nr_batch b, int* h_active, void* stream) {
    TraceRange tr("gapk_nr_step: one Newton iteration");
    if (!b || !h_active) {
        set_error("gapk_nr_step: bad arguments");
        return GAPK_EINVAL;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    dispatch_tsw<BodyOp>(b->precision, b->sw, b, st, 0, cudaGraphConditionalHandle{});
    int rc = check_launch();
    if (rc) return rc;
    GAPK_CUDA_TRY(cudaMemcpyAsync(h_active, b->dev.ctrl + 2, sizeof(int),
                                  cudaMemcpyDeviceToHost, st));
    GAPK_CUDA_TRY(cudaStreamSynchronize(st));
    return GAPK_OK;
}

int gapk_nr_get_state(gapk_nr_batch b, double* d_v, double* d_i, double* d_s, void* stream) {
    if (!b) {
        set_error("gapk_nr_get_state: null batch");
        return GAPK_EINVAL;
    }
    dispatch_tsw<StateOp>(b->precision, b->sw, b, reinterpret_cast<double2*>(d_v),
                          reinterpret_cast<double2*>(d_i), reinterpret_cast<double2*>(d_s),
                          static_cast<cudaStream_t>(stream));
    return check_launch();
}

static int64_t sparse_trace_size(gapk_nr_batch b) {
    return 3 * static_cast<int64_t>(b->G) * (b->plan->h.n_levels + 2);
}
// the panel trace exists when the one-CTA-per-scenario dense LU factorises the tail
static int64_t dense_trace_size(gapk_nr_batch b) {
    const int N = 2 * b->plan->h.n_tail;
    if (N == 0 || b->dense_split || b->dense_w <= 0) return 0;
    return static_cast<int64_t>(b->G) * b->sw * (1 + 3 * ((N + b->dense_w - 1) / b->dense_w));
}

int64_t gapk_nr_level_trace_size(gapk_nr_batch b) {
    if (!b) return 0;
    return sparse_trace_size(b) + dense_trace_size(b);
}

int gapk_nr_batch_device_error(gapk_nr_batch b) {
    if (!b || !b->ctrl.p) return 0;
    int w = 0;
    if (cudaMemcpy(&w, b->ctrl.as<int>() + 5, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("gapk_nr_batch_device_error: cudaMemcpy failed");
        return GAPK_ECUDA;
    }
    return w ? 1 : 0;
}

int gapk_nr_batch_set_wait_test(gapk_nr_batch b, int skip) {
    if (!b || !b->ctrl.p) {
        set_error("gapk_nr_batch_set_wait_test: null batch");
        return GAPK_EINVAL;
    }
    const int v = skip ? 1 : 0;
    GAPK_CUDA_TRY(cudaMemcpy(b->ctrl.as<int>() + 6, &v, sizeof(int), cudaMemcpyHostToDevice));
    return GAPK_OK;
}

int gapk_nr_dense_trace_panels(gapk_nr_batch b) {
    if (!b || dense_trace_size(b) == 0) return 0;
    const int N = 2 * b->plan->h.n_tail;
    return (N + b->dense_w - 1) / b->dense_w;
}

int gapk_nr_set_level_trace(gapk_nr_batch b, unsigned long long* d_stamps, int64_t n_stamps) {
    if (!b || (d_stamps && n_stamps < gapk_nr_level_trace_size(b))) {
        set_error("gapk_nr_set_level_trace: null batch or stamp buffer too small");
        return GAPK_EINVAL;
    }
    b->dev.lvl_ts = d_stamps;
    b->dev.dlu_ts = d_stamps && dense_trace_size(b) ? d_stamps + sparse_trace_size(b) : nullptr;
    // the solve graph holds the previous setting: rebuild it on the next gapk_nr_solve
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return GAPK_OK;
}

int gapk_nr_get_outputs(gapk_nr_batch b, const gapk_nr_outputs* out, void* stream) {
    if (!b || !out) {
        set_error("gapk_nr_get_outputs: bad arguments");
        return GAPK_EINVAL;
    }
    dispatch_tsw<StoreOp>(b->precision, b->sw, b, out, static_cast<cudaStream_t>(stream));
    return check_launch();
}

}  // extern "C"

// ===========================================================================================
// Heterogeneous batches in one graph launch: every batch's whole solve (options, load, the
// Newton loop in a device-side while node, optionally a retry loop for the scenarios that
// did not converge, results out) is one branch of a single CUDA graph; the branches share no
// edges, so the device runs them concurrently and one cudaGraphLaunch solves them all.
// ===========================================================================================
namespace gapk {
namespace {

template <typename T, int SW>
struct InitOp {
    static void run(gapk_nr_batch b, const gapk_nr_inputs* in, cudaStream_t st) {
        k_init_ctrl<<<1, 32, 0, st>>>(b->dev, in->max_iterations, in->policy, in->tolerance,
                                     in->refine_below, in->reuse_below);
    }
};
template <typename T, int SW>
struct RetryOp {
    static void run(gapk_nr_batch b, const gapk_nr_inputs* in, int policy,
                    cudaGraphConditionalHandle h, cudaStream_t st) {
        PlanDev const& P = b->plan->dev;
        k_retry_flags<SW><<<1, 1024, 0, st>>>(b->dev, policy, h);
        dim3 g(blocks_for((long)P.n_bus * SW, 256), b->G);
        k_retry_v<SW><<<g, 256, 0, st>>>(P, b->dev, reinterpret_cast<const double2*>(in->d_v_init),
                                         in->d_u_pu, in->v_init_shared);
    }
};

// Adds a while node after the capture's current dependencies on `cs` and captures the batch's
// loop body into it on `body_stream`; the capture on `cs` then continues after the node.
int add_loop(gapk_nr_batch b, cudaStream_t cs, cudaStream_t body_stream, unsigned dflt,
             cudaGraphConditionalHandle* h_out) {
    cudaStreamCaptureStatus stat;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    GAPK_CUDA_TRY(cudaStreamGetCaptureInfo(cs, &stat, nullptr, &g, &deps, &nd));
    if (stat != cudaStreamCaptureStatusActive) {
        set_error("mix graph: capture not active");
        return GAPK_ECUDA;
    }
    cudaGraphConditionalHandle h;
    GAPK_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, dflt, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    std::vector<cudaGraphNode_t> dv(nd);
    for (size_t k = 0; k < nd; ++k) dv[k] = deps[k];
    cudaGraphNode_t node;
    GAPK_CUDA_TRY(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &np));
    GAPK_CUDA_TRY(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    cudaError_t e = cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        set_error(std::string("mix graph body capture: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    dispatch_tsw<BodyOp>(b->precision, b->sw, b, body_stream, 1, h);
    cudaGraph_t captured = nullptr;
    GAPK_CUDA_TRY(cudaStreamEndCapture(body_stream, &captured));
    *h_out = h;
    return GAPK_OK;
}

}  // namespace
}  // namespace gapk

struct gapk_nr_mix_s {
    std::vector<gapk_nr_batch> batches;
    // the inputs / outputs the graph was built for, as bytes (the C structs are unnamed)
    std::vector<unsigned char> in_bytes, out_bytes;
    int retry = -2;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = nullptr, body = nullptr;
    ~gapk_nr_mix_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cs) cudaStreamDestroy(cs);
        if (body) cudaStreamDestroy(body);
    }
    int build(const gapk_nr_inputs* ins, const gapk_nr_outputs* outs, int retry_policy) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        if (!cs) GAPK_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        if (!body) GAPK_CUDA_TRY(cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking));
        GAPK_CUDA_TRY(cudaGraphCreate(&graph, 0));
        for (size_t i = 0; i < batches.size(); ++i) {
            gapk_nr_batch b = batches[i];
            b->cur_refine = ins[i].refine;
            cudaError_t e = cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0,
                                                          cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) {
                set_error(std::string("mix graph capture: ") + cudaGetErrorString(e));
                return GAPK_ECUDA;
            }
            int rc = GAPK_OK;
            dispatch_tsw<InitOp>(b->precision, b->sw, b, &ins[i], cs);
            dispatch_tsw<LoadOp>(b->precision, b->sw, b, &ins[i], cs);
            cudaGraphConditionalHandle h{};
            if (ins[i].max_iterations > 0) rc = add_loop(b, cs, body, 1, &h);
            if (!rc && retry_policy >= 0 && ins[i].max_iterations > 0) {
                cudaGraphConditionalHandle r{};
                // the retry loop's condition starts false; k_retry_flags sets it
                rc = add_loop_after(b, &ins[i], retry_policy, &r);
            }
            if (!rc) dispatch_tsw<StoreOp>(b->precision, b->sw, b, &outs[i], cs);
            cudaGraph_t captured = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(cs, &captured);
            if (rc) return rc;
            if (e2 != cudaSuccess) {
                set_error(std::string("mix graph capture end: ") + cudaGetErrorString(e2));
                return GAPK_ECUDA;
            }
        }
        GAPK_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
        in_bytes.resize(batches.size() * sizeof(gapk_nr_inputs));
        out_bytes.resize(batches.size() * sizeof(gapk_nr_outputs));
        std::memcpy(in_bytes.data(), ins, in_bytes.size());
        std::memcpy(out_bytes.data(), outs, out_bytes.size());
        retry = retry_policy;
        return GAPK_OK;
    }
    // retry: flags + start voltages (handle r, default 0), then a second loop on handle r
    int add_loop_after(gapk_nr_batch b, const gapk_nr_inputs* in, int policy,
                       cudaGraphConditionalHandle* r_out) {
        cudaStreamCaptureStatus stat;
        cudaGraph_t g = nullptr;
        GAPK_CUDA_TRY(cudaStreamGetCaptureInfo(cs, &stat, nullptr, &g, nullptr, nullptr));
        cudaGraphConditionalHandle r;
        GAPK_CUDA_TRY(cudaGraphConditionalHandleCreate(&r, g, 0, cudaGraphCondAssignDefault));
        dispatch_tsw<RetryOp>(b->precision, b->sw, b, in, policy, r, cs);
        // the while node reads the condition k_retry_flags set
        cudaStreamCaptureStatus stat2;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        GAPK_CUDA_TRY(cudaStreamGetCaptureInfo(cs, &stat2, nullptr, &g, &deps, &nd));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = r;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        std::vector<cudaGraphNode_t> dv(nd);
    for (size_t k = 0; k < nd; ++k) dv[k] = deps[k];
        cudaGraphNode_t node;
        GAPK_CUDA_TRY(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &np));
        GAPK_CUDA_TRY(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t bg = np.conditional.phGraph_out[0];
        cudaError_t e = cudaStreamBeginCaptureToGraph(body, bg, nullptr, nullptr, 0,
                                                      cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            set_error(std::string("mix graph retry body capture: ") + cudaGetErrorString(e));
            return GAPK_ECUDA;
        }
        dispatch_tsw<BodyOp>(b->precision, b->sw, b, body, 1, r);
        cudaGraph_t captured = nullptr;
        GAPK_CUDA_TRY(cudaStreamEndCapture(body, &captured));
        *r_out = r;
        return GAPK_OK;
    }
};

extern "C" {

int gapk_nr_mix_create(int n, const gapk_nr_batch* batches, gapk_nr_mix* out) {
    if (!out || n <= 0 || !batches) {
        set_error("gapk_nr_mix_create: bad arguments");
        return GAPK_EINVAL;
    }
    auto m = std::make_unique<gapk_nr_mix_s>();
    for (int i = 0; i < n; ++i) {
        if (!batches[i]) {
            set_error("gapk_nr_mix_create: null batch");
            return GAPK_EINVAL;
        }
        for (int j = 0; j < i; ++j)
            if (batches[j] == batches[i]) {
                set_error("gapk_nr_mix_create: a batch appears twice");
                return GAPK_EINVAL;
            }
        m->batches.push_back(batches[i]);
    }
    *out = m.release();
    return GAPK_OK;
}

int gapk_nr_mix_destroy(gapk_nr_mix m) {
    delete m;
    return GAPK_OK;
}

int gapk_nr_mix_solve(gapk_nr_mix m, const gapk_nr_inputs* in, const gapk_nr_outputs* out,
                      int retry_policy, void* stream) {
    TraceRange tr("gapk_nr_mix_solve");
    if (!m || !in || !out ||
        (retry_policy != -1 &&
         (retry_policy < GAPK_POLICY_REFERENCE || retry_policy > GAPK_POLICY_CLAMPED))) {
        set_error("gapk_nr_mix_solve: bad arguments");
        return GAPK_EINVAL;
    }
    const size_t n = m->batches.size();
    for (size_t i = 0; i < n; ++i) {
        int rc = validate_inputs(m->batches[i], &in[i]);
        if (rc) return rc;
    }
    const bool same = m->exec && m->retry == retry_policy &&
                      m->in_bytes.size() == n * sizeof(gapk_nr_inputs) &&
                      std::memcmp(m->in_bytes.data(), in, m->in_bytes.size()) == 0 &&
                      std::memcmp(m->out_bytes.data(), out, m->out_bytes.size()) == 0;
    if (!same) {
        int rc = m->build(in, out, retry_policy);
        if (rc) return rc;
    }
    GAPK_CUDA_TRY(cudaGraphLaunch(m->exec, static_cast<cudaStream_t>(stream)));
    return GAPK_OK;
}

}  // extern "C"

// ===========================================================================================
// General sparse LU (ILUSolver): complex a + jb handled as the 2x2 real block [a -b; b a], so
// the Newton engine's analysis, level-scheduled factor, dense tail and solves are reused.
// ===========================================================================================
namespace gapk {

__global__ void k_cfill(PlanDev P, BatchDev B, const double2* __restrict__ vals,
                        const int* __restrict__ val_map) {
    const int a_idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (a_idx >= P.n_a) return;
    const int slot = P.a_slots[a_idx];
    const int4 si = P.slot_info[slot];
    double re = 0.0, im = 0.0;
    for (int e = si.z; e < si.w; ++e) {
        const double2 v = vals[val_map[P.slot_src[e]]];
        re += v.x;
        im += v.y;
    }
    stb(reinterpret_cast<Blk<double>*>(B.F) + slot, Blk<double>{re, -im, im, re});
}

__global__ void k_crhs(int nb, const int* __restrict__ bus_of_node, const int* __restrict__ rp,
                       const double2* __restrict__ b, double2* rhs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nb) rhs[k] = b[rp[bus_of_node[k]]];
}

__global__ void k_csol(int nb, const int* __restrict__ bus_of_node, const double2* __restrict__ x,
                       double2* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nb) out[bus_of_node[k]] = x[k];
}

}  // namespace gapk

struct gapk_splu_s {
    gapk_nr_plan_s plan;
    std::vector<int> rp, val_map;
    gapk_nr_batch batch = nullptr;
    DevBuf d_valmap, d_rp, d_bon;
    bool factorized = false;
    ~gapk_splu_s() {
        if (batch) gapk_nr_batch_destroy(batch);
    }
    int ready() {
        if (batch) return GAPK_OK;
        gapk_nr_batch_options o{GAPK_PREC_FP64, 1, 1, 512, 0};
        int rc = gapk_nr_batch_create(&plan, 1, &o, &batch);
        if (rc) return rc;
        rc = d_valmap.upload(val_map);
        if (!rc) rc = d_rp.upload(rp);
        if (!rc) rc = d_bon.upload(plan.h.bus_of_node);
        return rc;
    }
};

extern "C" {

int gapk_splu_create(int n, int nnz, const int* h_row_ptr, const int* h_col_idx,
                     gapk_splu* out) {
    if (!out || !h_row_ptr || (nnz > 0 && !h_col_idx)) {
        set_error("gapk_splu_create: bad arguments");
        return GAPK_EINVAL;
    }
    auto s = std::make_unique<gapk_splu_s>();
    try {
        if (!analyze_general(n, nnz, h_row_ptr, h_col_idx, 16, s->plan.h, s->rp, s->val_map))
            return GAPK_EINVAL;
    } catch (std::bad_alloc const&) {
        set_error("gapk_splu_create: host allocation failed");
        return GAPK_ENOMEM;
    }
    // the plan's "Y" pattern is the row-permuted matrix
    s->plan.y_row_ptr.assign(n + 1, 0);
    s->plan.y_col.clear();
    for (int i = 0; i < n; ++i) {
        const int r = s->rp[i];
        for (int p = h_row_ptr[r]; p < h_row_ptr[r + 1]; ++p) s->plan.y_col.push_back(h_col_idx[p]);
        s->plan.y_row_ptr[i + 1] = static_cast<int>(s->plan.y_col.size());
    }
    *out = s.release();
    return GAPK_OK;
}

int gapk_splu_destroy(gapk_splu s) {
    delete s;
    return GAPK_OK;
}

int gapk_splu_factorize(gapk_splu s, const double* d_values, void* stream) {
    if (!s || !d_values) {
        set_error("gapk_splu_factorize: bad arguments");
        return GAPK_EINVAL;
    }
    s->factorized = false;
    int rc = s->ready();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    gapk_nr_batch b = s->batch;
    const int one[2] = {1, 0};
    GAPK_CUDA_TRY(cudaMemcpyAsync(b->dev.gsolve, one, sizeof(int), cudaMemcpyHostToDevice, st));
    GAPK_CUDA_TRY(cudaMemcpyAsync(b->dev.solving, one, sizeof(int), cudaMemcpyHostToDevice, st));
    GAPK_CUDA_TRY(cudaMemcpyAsync(b->dev.singular, one + 1, sizeof(int), cudaMemcpyHostToDevice, st));
    PlanDev const& P = s->plan.dev;
    k_cfill<<<blocks_for((long)P.n_a, 256), 256, 0, st>>>(
        P, b->dev, reinterpret_cast<const double2*>(d_values), s->d_valmap.as<int>());
    launch_factor<double, 1>(b, st);
    rc = check_launch();
    if (rc) return rc;
    int sing = 0;
    GAPK_CUDA_TRY(cudaMemcpyAsync(&sing, b->dev.singular, sizeof(int), cudaMemcpyDeviceToHost, st));
    GAPK_CUDA_TRY(cudaStreamSynchronize(st));
    if (sing) {
        set_error("gapk_splu_factorize: pivot below 1e-14 (numerically singular under static "
                  "pivoting)");
        return GAPK_ESINGULAR;
    }
    s->factorized = true;
    return GAPK_OK;
}

int gapk_splu_solve(gapk_splu s, const double* d_rhs, double* d_x, void* stream) {
    if (!s || !d_rhs || !d_x) {
        set_error("gapk_splu_solve: bad arguments");
        return GAPK_EINVAL;
    }
    if (!s->factorized) {
        set_error("gapk_splu_solve: matrix not factorized");
        return GAPK_ESTATE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    gapk_nr_batch b = s->batch;
    const int nb = s->plan.h.nb;
    k_crhs<<<blocks_for(nb, 256), 256, 0, st>>>(nb, s->d_bon.as<int>(), s->d_rp.as<int>(),
                                                  reinterpret_cast<const double2*>(d_rhs),
                                                  b->dev.rhs);
    launch_solve<double, 1>(b, st, b->dev.rhs, b->dev.dx, 0);
    k_csol<<<blocks_for(nb, 256), 256, 0, st>>>(nb, s->d_bon.as<int>(), b->dev.dx,
                                                  reinterpret_cast<double2*>(d_x));
    return check_launch();
}

int gapk_splu_size(gapk_splu s) { return s ? s->plan.h.nb : GAPK_EINVAL; }

}  // extern "C"

// ===========================================================================================
// Allocation-free single-scenario solve.
//
// Some callers cannot call cudaMalloc at solve time: hosts that hand out device memory only
// from their own pools, and real-time loops that must not touch the allocator (cudaMalloc and
// cudaFree can block on the whole device).  gapk_nr_solve_noalloc serves them: it solves one
// scenario in FP64 with the same kernels as gapk_nr_solve, but every buffer it needs (a copy
// of the plan's index lists and the whole Newton state) is carved out of one file-scope device
// array of fixed size.  The caller passes only inputs and outputs.
// ===========================================================================================
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB, held by every device
                                                             // that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code the array's name
// is only a host-side stand-in, so the address must come from cudaGetSymbolAddress, once per
// device, with that device current.
int noalloc_scratch_ptr(void** out) {
    int dev = 0;
    GAPK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("gapk_nr_solve_noalloc: device index out of range");
        return GAPK_EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        GAPK_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        for (int w : {32, 16, 8})
            GAPK_CUDA_TRY(dense_lu_attributes<double>(w, 232448 - 1024, false));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return GAPK_OK;
}

struct Carver {
    size_t off = 0;
    size_t take(size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~size_t(255);
        return o;
    }
};

}  // namespace

extern "C" int gapk_nr_solve_noalloc(gapk_nr_plan p, const gapk_nr_inputs* in,
                                     const gapk_nr_outputs* out, void* stream) {
    if (!p || !in || !in->d_y || !in->d_s_spec) {
        set_error("gapk_nr_solve_noalloc: plan, d_y and d_s_spec are required");
        return GAPK_EINVAL;
    }
    if (in->max_iterations < 0 || in->refine != 0 ||
        (in->policy < GAPK_POLICY_REFERENCE || in->policy > GAPK_POLICY_CLAMPED)) {
        set_error("gapk_nr_solve_noalloc: bad max_iterations / policy, or refine != 0 "
                  "(this entry point solves in FP64 only)");
        return GAPK_EINVAL;
    }
    auto const& h = p->h;
    const size_t n = h.n_bus, nb = h.nb, nnz = h.nnz_y, N = 2 * (size_t)h.n_tail;
    // plan index lists copied into the scratch, in this order
    std::vector<int> const* lists[] = {&p->y_row_ptr, &p->y_col, &h.bus_type, &h.node_of_bus,
                                       &h.slot_info, &h.slot_src, &h.slot_a, &h.level_ptr,
                                       &h.level_nodes, &h.fa_ptr, &h.targets, &h.pairs,
                                       &h.fb_ptr, &h.scale, &h.lptr, &h.lidx, &h.rptr,
                                       &h.rlist, &h.arow_ptr, &h.arow, &h.schur, &h.a_slots};
    constexpr int kLists = sizeof(lists) / sizeof(lists[0]);
    Carver c;
    size_t loff[kLists];
    for (int i = 0; i < kLists; ++i) loff[i] = c.take(lists[i]->size() * sizeof(int));
    const size_t oV = c.take(n * 16), oS = c.take(n * 16), oSc = c.take(n * 16),
                 oY = c.take(nnz * 16), oF = c.take((size_t)h.n_slots * 32),
                 oRhs = c.take(nb * 16), oDx = c.take(nb * 16), oRes = c.take(nb * 16),
                 oX = c.take(nb * 16), oDt = c.take(N * dense_ld((int)N) * 8), oMis = c.take(8),
                 oState = c.take(4), oSolv = c.take(4), oSing = c.take(4), oIt = c.take(4),
                 oSt = c.take(4), oFm = c.take(8), oGs = c.take(4), oGi = c.take(4),
                 oCtrl = c.take(8 * 4), oTol = c.take(8);
    if (c.off > kNoAllocScratchBytes) {
        set_error("gapk_nr_solve_noalloc: this grid needs " + std::to_string(c.off) +
                  " bytes of working memory; the static scratch holds " +
                  std::to_string(kNoAllocScratchBytes) + " bytes (32 MiB)");
        return GAPK_ERANGE;
    }
    size_t dense_smem = 0;
    int dense_w = 0;
    if (h.n_tail > 0) {
        // the panel width rule of gapk_nr_batch_create for FP64 tails
        for (int w : {32, 16, 8}) {
            size_t bytes = dense_lu_elems((int)N, w) * 8;
            if (bytes <= 232448 - 1024 && (w < 32 || N <= 200)) {
                dense_w = w;
                dense_smem = bytes;
                break;
            }
        }
        if (!dense_w) {
            set_error("gapk_nr_solve_noalloc: dense tail exceeds the shared-memory panel limit");
            return GAPK_ERANGE;
        }
    }
    void* base = nullptr;
    int rc = noalloc_scratch_ptr(&base);
    if (rc) return rc;
    unsigned char* B0 = static_cast<unsigned char*>(base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int i = 0; i < kLists; ++i)
        if (!lists[i]->empty())
            GAPK_CUDA_TRY(cudaMemcpyAsync(B0 + loff[i], lists[i]->data(),
                                          lists[i]->size() * sizeof(int),
                                          cudaMemcpyHostToDevice, st));
    auto L = [&](int i) { return reinterpret_cast<const int*>(B0 + loff[i]); };
    PlanDev P{};
    P.n_bus = h.n_bus;
    P.nb = h.nb;
    P.nnz_y = h.nnz_y;
    P.n_slots = h.n_slots;
    P.nnz_l = h.nnz_l;
    P.n_levels = h.n_levels;
    P.n_a = h.n_a;
    P.jac_mode = h.jac_mode;
    P.ns = h.ns;
    P.n_tail = h.n_tail;
    P.n_schur = static_cast<int>(h.schur.size() / 4);
    P.y_row_ptr = L(0);
    P.y_col = L(1);
    P.bus_type = L(2);
    P.node_of_bus = L(3);
    P.slot_info = reinterpret_cast<const int4*>(L(4));
    P.slot_src = L(5);
    P.slot_a = L(6);
    P.level_ptr = L(7);
    P.level_nodes = L(8);
    P.fa_ptr = L(9);
    P.targets = reinterpret_cast<const int4*>(L(10));
    P.pairs = reinterpret_cast<const int2*>(L(11));
    P.fb_ptr = L(12);
    P.scale = reinterpret_cast<const int2*>(L(13));
    P.lptr = L(14);
    P.lidx = L(15);
    P.rptr = L(16);
    P.rlist = reinterpret_cast<const int2*>(L(17));
    P.arow_ptr = L(18);
    P.arow = reinterpret_cast<const int2*>(L(19));
    P.schur = reinterpret_cast<const int4*>(L(20));
    P.a_slots = L(21);
    BatchDev D{};
    D.n_scen = 1;
    D.n_groups = 1;
    D.sw = 1;
    D.y_shared = 1;
    D.V = reinterpret_cast<double2*>(B0 + oV);
    D.Sspec = reinterpret_cast<double2*>(B0 + oS);
    D.Scalc = reinterpret_cast<double2*>(B0 + oSc);
    D.Y = reinterpret_cast<double2*>(B0 + oY);
    D.F = B0 + oF;
    D.A64 = nullptr;
    D.rhs = reinterpret_cast<double2*>(B0 + oRhs);
    D.dx = reinterpret_cast<double2*>(B0 + oDx);
    D.res = reinterpret_cast<double2*>(B0 + oRes);
    D.X = B0 + oX;
    D.Dt = B0 + oDt;
    D.mis_bits = reinterpret_cast<unsigned long long*>(B0 + oMis);
    D.state = reinterpret_cast<int*>(B0 + oState);
    D.solving = reinterpret_cast<int*>(B0 + oSolv);
    D.singular = reinterpret_cast<int*>(B0 + oSing);
    D.iters = reinterpret_cast<int*>(B0 + oIt);
    D.status = reinterpret_cast<int*>(B0 + oSt);
    D.final_mis = reinterpret_cast<double*>(B0 + oFm);
    D.gsolve = reinterpret_cast<int*>(B0 + oGs);
    D.giter = reinterpret_cast<int*>(B0 + oGi);
    D.ctrl = reinterpret_cast<int*>(B0 + oCtrl);
    D.tol = reinterpret_cast<double*>(B0 + oTol);
    // control words and state start fresh on every call (the scratch keeps the last call's)
    int ctrl[8] = {0, in->max_iterations, 1, in->policy, 0, 0, 0, 0};
    GAPK_CUDA_TRY(cudaMemcpyAsync(D.ctrl, ctrl, sizeof(ctrl), cudaMemcpyHostToDevice, st));
    double tol = in->tolerance;
    GAPK_CUDA_TRY(cudaMemcpyAsync(D.tol, &tol, sizeof(double), cudaMemcpyHostToDevice, st));
    k_load<1><<<blocks_for((long)n, 256), 256, 0, st>>>(
        P, D, reinterpret_cast<const double2*>(in->d_y),
        reinterpret_cast<const double2*>(in->d_s_spec),
        reinterpret_cast<const double2*>(in->d_v_init), in->d_u_pu, 0);
    rc = check_launch();
    if (rc) return rc;
    const int thr = 512;
    for (int it = 0; it < in->max_iterations; ++it) {
        k_mismatch<1><<<mismatch_grid<1>(P, 1), 256, 0, st>>>(P, D);
        k_check<1><<<1, 1024, 0, st>>>(D, 0, cudaGraphConditionalHandle{});
        k_jfill<double, 1><<<blocks_for((long)h.n_a, 256), 256, 0, st>>>(P, D);
        k_factor<double, 1><<<1, thr, 0, st>>>(P, D);
        if (h.n_tail > 0) {
            k_schur<double, 1><<<blocks_for((long)P.n_schur, 256), 256, 0, st>>>(P, D);
            launch_dense_lu<double>(dense_w, 1, dense_smem, st, D, (int)N, false);
        }
        k_solve_fwd<double, 1><<<1, thr, 0, st>>>(P, D, D.rhs, 0);
        if (h.n_tail > 0)
            k_dense_solve<double, 1><<<1, 256, dense_solve_smem(P.n_tail, sizeof(double)), st>>>(P, D, D.dx, 0);
        k_solve_bwd<double, 1><<<1, thr, 0, st>>>(P, D, D.dx, 0);
        k_update<1><<<blocks_for((long)n, 256), 256, 0, st>>>(P, D);
        rc = check_launch();
        if (rc) return rc;
        int any = 0;
        GAPK_CUDA_TRY(cudaMemcpyAsync(&any, D.ctrl + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
        GAPK_CUDA_TRY(cudaStreamSynchronize(st));
        if (!any) break;
    }
    if (out) {
        k_store<1><<<blocks_for((long)n, 256), 256, 0, st>>>(
            P, D, reinterpret_cast<double2*>(out->d_v), out->d_iterations, out->d_status,
            out->d_final_mismatch);
        rc = check_launch();
        if (rc) return rc;
    }
    // the outputs are read from the shared scratch: wait for them, so that a later call from
    // this thread (on any stream) cannot overwrite the scratch before they are written
    GAPK_CUDA_TRY(cudaStreamSynchronize(st));
    return GAPK_OK;
}

// NVTX range helper of internal.h
gapk::TraceRange::TraceRange(const char* name) { nvtxRangePushA(name); }
gapk::TraceRange::~TraceRange() { nvtxRangePop(); }
