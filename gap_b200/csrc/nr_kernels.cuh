// Device kernels of the Newton-Raphson loop.
//
// Layout: scenarios sharing one plan are packed in groups of SW ("lanes"); every per-bus,
// per-node and per-slot quantity is stored [group][item][lane], so the SW threads that
// handle the same item for the SW scenarios of a group touch one contiguous run of memory
// (SW*16 B for a complex FP64 value, SW*16 B for an FP32 2x2 block).  Index lists (CSR of
// Y, factor schedule) are shared by all lanes and read once per warp.
//
// Reference semantics restated (src/solver/powerflow/cpu/cpu_newton_raphson.cpp):
//   mismatch   :243-337  S = V conj(Y V), Delta = S - S_spec, P rows for non-slack buses, Q
//                        rows for PQ buses, converged when max |Delta| < tol (:115-157)
//   Jacobian   :546-727  polar partial derivatives; |V| < 1e-6 replaced by 1 (:578)
//   update     :438-504  damped (0.9) and clamped polar update (policy REFERENCE)
#pragma once
#include <cuda_runtime.h>

#include "blocks.cuh"

namespace gapk {

enum { BUS_PQ = 0, BUS_PV = 1, BUS_SLACK = 2 };
enum { SC_CONVERGED = 0, SC_MAXITER = 1, SC_SINGULAR = 2, SC_NONFINITE = 3 };

struct PlanDev {
    int n_bus, nb, nnz_y, n_slots, nnz_l, n_levels, n_a;
    int jac_mode;  // 0: reference (last duplicate, |x| <= 1e-12 dropped), 1: exact
    int ns, n_tail, n_schur;  // sparse nodes, dense-tail nodes, Schur targets (= n_tail^2)
    const int4* schur;        // (slot, pair_begin, pair_end, position r*n_tail+c | hasval<<30)
    const int* a_slots;       // slots holding Jacobian values (the only ones the fill writes)
    const int* acol_ptr;      // A blocks by block column: (a index, row node)
    const int2* acol;
    const int* y_row_ptr;
    const int* y_col;
    const int* bus_type;
    const int* node_of_bus;
    const int4* slot_info;
    const int* slot_src;
    const int* slot_a;
    const int* level_ptr;
    const int* level_nodes;
    const int* fa_ptr;
    const int4* targets;
    const int2* pairs;
    const int* fb_ptr;
    const int2* scale;
    const int* lptr;
    const int* lidx;
    const int* rptr;
    const int2* rlist;
    const int* arow_ptr;
    const int2* arow;
};

// Per-batch device state.  q = group*SW + lane indexes per-scenario arrays.
struct BatchDev {
    int n_scen, n_groups, sw, y_shared;
    double2* V;       // [G][n_bus][SW]
    double2* Sspec;   // [G][n_bus][SW]
    double2* Scalc;   // [G][n_bus][SW]
    double2* Y;       // [nnz] (shared) or [G][nnz][SW]
    void* F;          // factor blocks [G][n_slots][SW]
    double* A64;      // FP64 Jacobian blocks [G][n_a][SW][4] (iterative refinement) or null
    double2* rhs;     // -Delta per node [G][nb][SW]
    double2* dx;      // Newton correction per node [G][nb][SW]
    double2* res;     // refinement residual [G][nb][SW]
    void* X;          // triangular-solve work vector [G][nb][SW] (T2)
    void* Dt;         // dense tail per scenario [G*SW][2*n_tail][dense_ld] (T), row-major
    unsigned long long* mis_bits;  // [G*SW] max |Delta| bits of the current iteration
    int* state;       // [G*SW] 0 iterating, 1 done
    int* solving;     // [G*SW] correction + update this iteration
    int* singular;    // [G*SW]
    int* iters;       // [G*SW]
    int* status;      // [G*SW]
    double* final_mis;  // [G*SW]
    int* gsolve;      // [G]
    int* giter;       // [G]
    int* ctrl;        // [0] iteration, [1] max_iter, [2] any iterating, [3] policy, [4] loops,
                      // [5] tensor-core LU wait ran out, [6] wait test (skip the MMAs)
    double* tol;      // [0] tolerance, [1] refine below, [2] reuse the factors below this mismatch
                      //     (0: never); the allocation-free path has [0] only
    int* grefine;     // [G] refinement pass runs for the group this iteration (null: always)
    int* gfactor;     // [G] the group refactorises this iteration (null: always); else the
                      //     previous factors precondition the refined solve
    unsigned long long* lvl_ts;  // level trace (null: off): %globaltimer stamps
                                 // [3 kernels: factor, forward, backward][G][n_levels + 2]
    unsigned long long* dlu_ts;  // dense-tail panel trace of k_dense_lu (null: off)
                                 // [G*SW][1 + 3 * panels]: start, then per panel the ends of
                                 // the diagonal block, the L21/U12 solves, the trailing update
};

// nanosecond clock of the level trace (PTX special register %globaltimer)
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// stamp j of kernel `which` for group g: 0 = start, 1 + h = level h done (in execution order),
// n_levels + 1 = end; one thread per CTA, after a barrier
__device__ __forceinline__ void lvl_stamp(BatchDev const& B, int n_levels, int which, int g,
                                          int j) {
    if (threadIdx.x == 0)
        B.lvl_ts[((size_t)which * B.n_groups + g) * (n_levels + 2) + j] = gtimer();
}

// ---------------------------------------------------------------------------------------
// load: interleave inputs, flat start, reset state
// ---------------------------------------------------------------------------------------
template <int SW>
__global__ void k_load(PlanDev P, BatchDev B, const double2* __restrict__ y_in,
                       const double2* __restrict__ s_in, const double2* __restrict__ v_in,
                       const double* __restrict__ u_pu, int v_shared) {
    const int g = blockIdx.y;
    const int n = P.n_bus;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(tid / SW), lane = (int)(tid % SW);
    int q = g * SW + lane;
    int src = q < B.n_scen ? q : g * SW;  // padding lanes mirror the group's first scenario
    if (i < n) {
        size_t o = ((size_t)g * n + i) * SW + lane;
        B.Sspec[o] = s_in[(size_t)src * n + i];
        double2 v;
        if (v_in) {
            v = v_in[(size_t)(v_shared ? 0 : src) * n + i];
        } else {
            // flat start (cpu_newton_raphson.cpp:77-88): SLACK/PV at u_pu, PQ at 0.98, angle 0
            int t = P.bus_type[i];
            double m = (t == BUS_PQ) ? 0.98 : (u_pu ? u_pu[i] : 1.0);
            v = make_double2(m, 0.0);
        }
        B.V[o] = v;
    }
    if (i < n) {
        if (!B.y_shared) {
            for (int p = i; p < P.nnz_y; p += n)
                B.Y[((size_t)g * P.nnz_y + p) * SW + lane] = y_in[(size_t)src * P.nnz_y + p];
        } else if (g == 0 && lane == 0) {
            for (int p = i; p < P.nnz_y; p += n) B.Y[p] = y_in[p];
        }
    }
    if (i == 0) {
        B.mis_bits[q] = 0ull;
        B.state[q] = q < B.n_scen ? 0 : 1;
        B.solving[q] = q < B.n_scen ? 1 : 0;
        B.singular[q] = 0;
        B.iters[q] = 0;
        B.status[q] = SC_MAXITER;
        B.final_mis[q] = 0.0;
        if (lane == 0) {
            B.gsolve[g] = 1;
            B.giter[g] = 1;
            if (B.grefine) B.grefine[g] = 1;  // the stage API refines unless k_check says not
            if (B.gfactor) B.gfactor[g] = 1;
        }
    }
}

// ---------------------------------------------------------------------------------------
// in-graph control: solve options as kernel arguments, and the retry of unconverged lanes
// ---------------------------------------------------------------------------------------
// Loop control words and tolerances of one solve, written on the device (a graph that holds
// several batches' loops sets each batch's options without host copies).
__global__ void k_init_ctrl(BatchDev B, int max_iter, int policy, double tol, double refine_below,
                            double reuse_below) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        B.ctrl[0] = 0;
        B.ctrl[1] = max_iter;
        B.ctrl[2] = 1;
        B.ctrl[3] = policy;
        B.ctrl[4] = 0;
        B.ctrl[5] = 0;  // set by a tensor-core LU whose bounded wait ran out during the solve
        B.tol[0] = tol;
        B.tol[1] = refine_below;
        B.tol[2] = reuse_below;
    }
}

// Retry after the loop (one CTA): every scenario that ended at max_iterations or with a
// non-finite mismatch starts again with the step policy `policy` (its other scenarios stay
// done); the groups holding one iterate again, refactorising and refining.  Sets the retry
// loop's condition to whether any scenario retries.
template <int SW>
__global__ void k_retry_flags(BatchDev B, int policy, cudaGraphConditionalHandle handle) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    const int total = B.n_groups * SW;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const bool again = q < B.n_scen && (B.status[q] == SC_MAXITER || B.status[q] == SC_NONFINITE);
        if (again) {
            B.state[q] = 0;
            B.solving[q] = 1;
            B.singular[q] = 0;
            B.iters[q] = 0;
            B.status[q] = SC_MAXITER;
            B.mis_bits[q] = 0ull;
            B.final_mis[q] = 0.0;
            any = 1;  // benign race: every writer stores 1
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < B.n_groups; g += blockDim.x) {
        int iv = 0;
        for (int l = 0; l < SW; ++l) {
            const int q = g * SW + l;
            iv |= q < B.n_scen && B.state[q] == 0;
        }
        B.gsolve[g] = iv;
        B.giter[g] = iv;
        if (B.grefine) B.grefine[g] = 1;
        if (B.gfactor) B.gfactor[g] = 1;
    }
    if (threadIdx.x == 0) {
        B.ctrl[0] = 0;
        B.ctrl[2] = any;
        B.ctrl[3] = policy;
        cudaGraphSetConditional(handle, any ? 1u : 0u);
    }
}

// The retried scenarios' voltages back at their start (as k_load sets them).
template <int SW>
__global__ void k_retry_v(PlanDev P, BatchDev B, const double2* __restrict__ v_in,
                          const double* __restrict__ u_pu, int v_shared) {
    const int g = blockIdx.y;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(tid / SW), lane = (int)(tid % SW);
    const int q = g * SW + lane;
    if (i >= P.n_bus || q >= B.n_scen || B.state[q] != 0) return;
    double2 v;
    if (v_in) {
        v = v_in[(size_t)(v_shared ? 0 : q) * P.n_bus + i];
    } else {
        const int t = P.bus_type[i];
        v = make_double2((t == BUS_PQ) ? 0.98 : (u_pu ? u_pu[i] : 1.0), 0.0);
    }
    B.V[((size_t)g * P.n_bus + i) * SW + lane] = v;
}

// ---------------------------------------------------------------------------------------
// mismatch: fused Y*V SpMV, S = V conj(I), Delta, rhs, per-scenario max |Delta|
// ---------------------------------------------------------------------------------------
// Each CTA covers MM_TILES consecutive tiles of 256 / SW buses (x SW lanes); the per-scenario
// maxima are reduced within the CTA (shuffles, then shared memory) before one atomicMax per
// lane, so a group's scenarios see n / (MM_TILES * 256 / SW) atomics instead of one per warp
// (same-address atomics serialise in L2).
constexpr int MM_TILES = 4;

template <int SW>
__global__ void __launch_bounds__(256, 8) k_mismatch(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.giter[g]) return;
    const int n = P.n_bus;
    const int lane = threadIdx.x % SW;
    const double2* Vg = B.V + (size_t)g * n * SW;
    const double2* Yg = B.y_shared ? B.Y : B.Y + (size_t)g * P.nnz_y * SW;
    const int ys = B.y_shared ? 0 : 1;  // Y value of entry p at Yg[p * (ys ? SW : 1) + ys * lane]
    double m = 0.0;
    // S = V conj(Y V) and the mismatch of bus i from its accumulated current (vi, sp, t, node:
    // the bus's own voltage, specified power, type and block node).  Loading these before the
    // gathers needs more than the 32 registers of 8 CTAs per SM and measured slower.
    auto finish = [&](int i, double ir, double ii, double2 vi, double2 sp, int t, int node) {
        const size_t o = ((size_t)g * n + i) * SW + lane;
        const double2 s = make_double2(fma(vi.x, ir, vi.y * ii), fma(vi.y, ir, -vi.x * ii));
        B.Scalc[o] = s;
        if (t != BUS_SLACK) {
            const double dp = s.x - sp.x;
            const double dq = (t == BUS_PQ) ? s.y - sp.y : 0.0;
            B.rhs[((size_t)g * P.nb + node) * SW + lane] = make_double2(-dp, -dq);
            m = nmax(m, nmax(fabs(dp), fabs(dq)));
        }
    };
    // two tiles at a time: the rows of buses i0 and i1 = i0 + 256 / SW are walked together, so
    // that each thread keeps two independent column -> V gather chains in flight
#pragma unroll 1
    for (int tile = 0; tile < MM_TILES; tile += 2) {
        const int i0 = ((blockIdx.x * MM_TILES + tile) * blockDim.x + threadIdx.x) / SW;
        const int i1 = i0 + (int)blockDim.x / SW;
        if (i0 >= n) break;
        const bool a1 = i1 < n;
        int p0 = P.y_row_ptr[i0], p1 = a1 ? P.y_row_ptr[i1] : 0;
        const int e0 = P.y_row_ptr[i0 + 1], e1 = a1 ? P.y_row_ptr[i1 + 1] : 0;
        double r0 = 0.0, q0 = 0.0, r1 = 0.0, q1 = 0.0;
        while (p0 < e0 || p1 < e1) {
            if (p0 < e0) {
                const double2 y = ys ? Yg[(size_t)p0 * SW + lane] : Yg[p0];
                const double2 v = Vg[(size_t)P.y_col[p0] * SW + lane];
                r0 = fma(y.x, v.x, r0);
                r0 = fma(-y.y, v.y, r0);
                q0 = fma(y.x, v.y, q0);
                q0 = fma(y.y, v.x, q0);
                ++p0;
            }
            if (p1 < e1) {
                const double2 y = ys ? Yg[(size_t)p1 * SW + lane] : Yg[p1];
                const double2 v = Vg[(size_t)P.y_col[p1] * SW + lane];
                r1 = fma(y.x, v.x, r1);
                r1 = fma(-y.y, v.y, r1);
                q1 = fma(y.x, v.y, q1);
                q1 = fma(y.y, v.x, q1);
                ++p1;
            }
        }
        finish(i0, r0, q0, Vg[(size_t)i0 * SW + lane], B.Sspec[((size_t)g * n + i0) * SW + lane],
               P.bus_type[i0], P.node_of_bus[i0]);
        if (a1)
            finish(i1, r1, q1, Vg[(size_t)i1 * SW + lane], B.Sspec[((size_t)g * n + i1) * SW + lane],
                   P.bus_type[i1], P.node_of_bus[i1]);
    }
#pragma unroll
    for (int off = SW; off < 32; off <<= 1) m = nmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    __shared__ double red[8][8];  // [warp][lane] (blockDim 256, SW <= 8)
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) < SW) red[w][lane] = m;
    __syncthreads();
    if (threadIdx.x < SW) {
        double r = red[0][threadIdx.x];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = nmax(r, red[k][threadIdx.x]);
        if (r != 0.0)
            atomicMax(&B.mis_bits[g * SW + threadIdx.x], (unsigned long long)__double_as_longlong(r));
    }
}

// Grid of k_mismatch for G lane groups.
template <int SW>
inline dim3 mismatch_grid(PlanDev const& P, int G) {
    const long per = (long)MM_TILES * 256;
    return dim3((unsigned)(((long)P.n_bus * SW + per - 1) / per), (unsigned)G);
}

// ---------------------------------------------------------------------------------------
// convergence test and loop control (one CTA)
// ---------------------------------------------------------------------------------------
template <int SW>
__global__ void k_check(BatchDev B, int use_cond, cudaGraphConditionalHandle handle) {
    __shared__ int any_iter;
    if (threadIdx.x == 0) any_iter = 0;
    __syncthreads();
    const int it = B.ctrl[0];
    const int max_iter = B.ctrl[1];
    const double tol = B.tol[0];
    const int total = B.n_groups * SW;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        if (q >= B.n_scen || B.state[q] != 0) {
            B.solving[q] = 0;
            continue;
        }
        const double m = __longlong_as_double((long long)B.mis_bits[q]);
        B.mis_bits[q] = 0ull;
        B.final_mis[q] = m;
        if (!isfinite(m)) {
            B.state[q] = 1;
            B.status[q] = SC_NONFINITE;
            B.iters[q] = it + 1;
            B.solving[q] = 0;
        } else if (m < tol) {
            B.state[q] = 1;
            B.status[q] = SC_CONVERGED;
            B.iters[q] = it + 1;
            B.solving[q] = 0;
        } else {
            B.solving[q] = 1;
            if (it + 1 >= max_iter) {
                B.state[q] = 1;
                B.status[q] = SC_MAXITER;
                B.iters[q] = max_iter;
            }
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < B.n_groups; g += blockDim.x) {
        int sv = 0, iv = 0;
        for (int l = 0; l < SW; ++l) {
            const int q = g * SW + l;
            if (q < B.n_scen) {
                sv |= B.solving[q];
                iv |= (B.state[q] == 0);
            }
        }
        B.gsolve[g] = sv;
        B.giter[g] = iv;
        if (B.grefine) {
            // refinement only once some iterating lane of the group is close to convergence
            const double rb = B.tol[1];
            int rv = rb <= 0.0;
            for (int l = 0; l < SW && !rv; ++l) {
                const int q = g * SW + l;
                if (q < B.n_scen && B.solving[q] && B.final_mis[q] < rb) rv = 1;
            }
            // the factors are reused once every iterating lane of the group is below [2];
            // the solve is then refined against the current FP64 Jacobian
            const double rf = B.tol[2];
            int fv = 1;
            if (B.gfactor && rf > 0.0 && sv) {
                fv = 0;
                for (int l = 0; l < SW; ++l) {
                    const int q = g * SW + l;
                    if (q < B.n_scen && B.solving[q] && !(B.final_mis[q] < rf)) fv = 1;
                }
            }
            if (B.gfactor) B.gfactor[g] = fv;
            B.grefine[g] = rv || !fv;
        }
        if (iv) atomicOr(&any_iter, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        B.ctrl[0] = it + 1;
        B.ctrl[2] = any_iter;
        B.ctrl[4] = it + 1;
        if (use_cond) cudaGraphSetConditional(handle, any_iter ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------------------
// Jacobian value fill on the fixed factor pattern (fill-in slots are zeroed)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void polar_parts(double2 v, double& vmr, double& c, double& s) {
    const double vm = hypot(v.x, v.y);
    if (vm > 0.0) {
        const double inv = 1.0 / vm;  // one division for both direction cosines
        c = v.x * inv;
        s = v.y * inv;
    } else {
        c = 1.0;
        s = 0.0;
    }
    vmr = vm < 1e-6 ? 1.0 : vm;
}

template <typename T, int SW>
__global__ void __launch_bounds__(256) k_jfill(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.gsolve[g]) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int a_idx = tid / SW, lane = tid % SW;
    if (a_idx >= P.n_a) return;
    const int slot = P.a_slots[a_idx];
    const int4 si = P.slot_info[slot];
    const int n = P.n_bus;
    Blk<double> J = {0.0, 0.0, 0.0, 0.0};
    const bool diag = si.x == si.y;
    if (diag || si.z < si.w) {
        double G = 0.0, Bv = 0.0;
#pragma unroll 4
        for (int e = si.z; e < si.w; ++e) {
            const int p = P.slot_src[e];
            const double2 y = B.y_shared ? B.Y[p] : B.Y[((size_t)g * P.nnz_y + p) * SW + lane];
            G += y.x;
            Bv += y.y;
        }
        const double2* Vg = B.V + (size_t)g * n * SW;
        const bool pqi = P.bus_type[si.x] == BUS_PQ;
        double vmi, ci, sni;
        polar_parts(Vg[(size_t)si.x * SW + lane], vmi, ci, sni);
        if (diag) {
            const double2 S = B.Scalc[((size_t)g * n + si.x) * SW + lane];
            J.a = -S.y - Bv * vmi * vmi;
            const double ivm = 1.0 / vmi;
            J.b = S.x * ivm + G * vmi;
            J.c = S.x - G * vmi * vmi;
            J.d = S.y * ivm - Bv * vmi;
            if (!pqi) {
                J.b = 0.0;
                J.c = 0.0;
                J.d = 1.0;
            }
        } else {
            const bool pqj = P.bus_type[si.y] == BUS_PQ;
            double vmj, cj, snj;
            polar_parts(Vg[(size_t)si.y * SW + lane], vmj, cj, snj);
            // u = |V_i| e^{j(theta_i - theta_j)}
            const double uc = vmi * (ci * cj + sni * snj);
            const double ud = vmi * (sni * cj - ci * snj);
            const double gcbd = G * uc + Bv * ud;
            const double gdbc = G * ud - Bv * uc;
            J.a = vmj * gdbc;
            J.b = gcbd;
            J.c = -vmj * gcbd;
            J.d = gdbc;
            if (!pqi) {
                J.c = 0.0;
                J.d = 0.0;
            }
            if (!pqj) {
                J.b = 0.0;
                J.d = 0.0;
            }
        }
    }
    if (P.jac_mode == 0) {
        // convert_to_sparse_matrix drops |x| <= 1e-12 (cpu_newton_raphson.cpp:754)
        if (fabs(J.a) <= 1e-12) J.a = 0.0;
        if (fabs(J.b) <= 1e-12) J.b = 0.0;
        if (fabs(J.c) <= 1e-12) J.c = 0.0;
        if (fabs(J.d) <= 1e-12 && !(diag && J.d == 1.0)) J.d = 0.0;
    }
    if (!B.gfactor || B.gfactor[g]) {  // a group that reuses its factors keeps them
        Blk<T>* F = reinterpret_cast<Blk<T>*>(B.F) + ((size_t)g * P.n_slots + slot) * SW + lane;
        stb(F, Blk<T>{(T)J.a, (T)J.b, (T)J.c, (T)J.d});
    }
    // the FP64 copy feeds only the refinement residual: skipped for groups that do not
    // refine this iteration
    if (B.A64 && (!B.grefine || B.grefine[g])) {
        Blk<double>* A = reinterpret_cast<Blk<double>*>(B.A64) +
                         ((size_t)g * P.n_a + a_idx) * SW + lane;
        stb(A, J);
    }
}

// ---------------------------------------------------------------------------------------
// numeric block LU (left-looking Crout), one CTA per group, level by level
// ---------------------------------------------------------------------------------------
template <typename T, int SW>
__global__ void k_factor(PlanDev P, BatchDev B) {
    const int g = blockIdx.x;
    if (!B.gsolve[g] || (B.gfactor && !B.gfactor[g])) return;
    Blk<T>* F = reinterpret_cast<Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    const int lane = threadIdx.x % SW;
    const int e0 = threadIdx.x / SW, ne = blockDim.x / SW;
    bool bad = false;
    if (B.lvl_ts) lvl_stamp(B, P.n_levels, 0, g, 0);
    for (int h = 0; h < P.n_levels; ++h) {
        const int ta = P.fa_ptr[h], tb = P.fa_ptr[h + 1];
        // two targets per worker at a time (targets of one level are independent), so that
        // their gathers overlap in memory
        for (int t = ta + e0; t < tb; t += 2 * ne) {
            const bool two = t + ne < tb;
            const int4 tg = P.targets[t];
            const int4 tg2 = two ? P.targets[t + ne] : make_int4(0, 0, 0, 0);
            Blk<T> acc = (tg.w & 2) ? ldb(F + (size_t)tg.x * SW + lane) : Blk<T>{0, 0, 0, 0};
            Blk<T> acc2 = (tg2.w & 2) ? ldb(F + (size_t)tg2.x * SW + lane) : Blk<T>{0, 0, 0, 0};
            const int nb = min(tg.z - tg.y, tg2.z - tg2.y);
#pragma unroll 2
            for (int i = 0; i < nb; ++i) {
                const int2 pr = P.pairs[tg.y + i];
                const int2 pr2 = P.pairs[tg2.y + i];
                msub(acc, ldb(F + (size_t)pr.x * SW + lane), ldb(F + (size_t)pr.y * SW + lane));
                msub(acc2, ldb(F + (size_t)pr2.x * SW + lane), ldb(F + (size_t)pr2.y * SW + lane));
            }
#pragma unroll 4
            for (int p = tg.y + nb; p < tg.z; ++p) {
                const int2 pr = P.pairs[p];
                msub(acc, ldb(F + (size_t)pr.x * SW + lane), ldb(F + (size_t)pr.y * SW + lane));
            }
#pragma unroll 4
            for (int p = tg2.y + nb; p < tg2.z; ++p) {
                const int2 pr = P.pairs[p];
                msub(acc2, ldb(F + (size_t)pr.x * SW + lane), ldb(F + (size_t)pr.y * SW + lane));
            }
            if (tg.w & 1) {
                bool ok;
                acc = inv2(acc, ok);
                bad |= !ok;
            }
            stb(F + (size_t)tg.x * SW + lane, acc);
            if (two) {
                if (tg2.w & 1) {
                    bool ok;
                    acc2 = inv2(acc2, ok);
                    bad |= !ok;
                }
                stb(F + (size_t)tg2.x * SW + lane, acc2);
            }
        }
        __syncthreads();
        const int sa = P.fb_ptr[h], sb = P.fb_ptr[h + 1];
        if (sb > sa) {
            for (int t = sa + e0; t < sb; t += ne) {
                const int2 sc = P.scale[t];
                Blk<T>* Lp = F + (size_t)sc.x * SW + lane;
                stb(Lp, mul(ldb(Lp), ldb(F + (size_t)sc.y * SW + lane)));
            }
            __syncthreads();
        }
        if (B.lvl_ts) lvl_stamp(B, P.n_levels, 0, g, h + 1);
    }
    if (B.lvl_ts) lvl_stamp(B, P.n_levels, 0, g, P.n_levels + 1);
    if (bad) B.singular[g * SW + lane] = 1;
}

// ---------------------------------------------------------------------------------------
// dense tail: Schur-complement gather from the sparse part, blocked dense LU, dense solves
// ---------------------------------------------------------------------------------------
// Row stride of the dense tail: N rounded up to 8, so that every 8-column group that starts
// on a multiple of 8 stays inside its (padded) row.
__host__ __device__ __forceinline__ int dense_ld(int N) { return (N + 7) & ~7; }

template <typename T>
struct V4 {
    T v[4];
};
__device__ __forceinline__ V4<float> ld4(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return {{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, V4<float> const& a) {
    *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ void st4(double* p, V4<double> const& a) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a.v[0], a.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(a.v[2], a.v[3]);
}

template <typename T, int SW>
__global__ void __launch_bounds__(256) k_schur(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.gsolve[g] || (B.gfactor && !B.gfactor[g])) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = tid / SW, lane = tid % SW;
    if (t >= P.n_schur) return;
    const int q = g * SW + lane;
    const Blk<T>* F = reinterpret_cast<const Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    const int4 tg = P.schur[t];
    Blk<T> acc = (tg.w >> 30) ? ldb(F + (size_t)tg.x * SW + lane) : Blk<T>{0, 0, 0, 0};
#pragma unroll 4
    for (int p = tg.y; p < tg.z; ++p) {
        const int2 pr = P.pairs[p];
        msub(acc, ldb(F + (size_t)pr.x * SW + lane), ldb(F + (size_t)pr.y * SW + lane));
    }
    const int N = 2 * P.n_tail, ld = dense_ld(N);
    const int pos = tg.w & ((1 << 30) - 1);
    const int r = 2 * (pos / P.n_tail), c = 2 * (pos % P.n_tail);
    T* D = reinterpret_cast<T*>(B.Dt) + (size_t)q * N * ld;
    D[(size_t)r * ld + c] = acc.a;
    D[(size_t)r * ld + c + 1] = acc.b;
    D[(size_t)(r + 1) * ld + c] = acc.c;
    D[(size_t)(r + 1) * ld + c + 1] = acc.d;
}

// Asynchronous global -> shared copies (cp.async): the copies of one thread are all in flight
// together, so a staging loop costs one memory latency instead of one per element.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES)
                     : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// Hint: bring the line holding p into L2 (no register result, nothing to wait for).
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Right-looking blocked LU without pivoting of one scenario's N x N tail (row-major, row
// stride dense_ld(N), in place), panels of W columns (W = 8, 16 or 32; compile time):
//   A. warp 0 factors the W x W diagonal block in registers (lane r holds row r; the pivot
//      row is broadcast with shuffles) and publishes U11 (transposed, in the panel buffer),
//      L11 (row-major) and 1/diag(U11) in shared memory;
//   B. every thread then solves whole rows of L21 (x U11 = a) and whole columns of U12
//      (L11 y = a), register resident and independent of each other -- two barriers per panel
//      in all; the L21 rows also go to the transposed panel buffer PT[c][r] for the trailing
//      update;
//   C. the trailing update streams U12 through a double-buffered shared-memory chunk of DCW
//      columns (cp.async prefetch of chunk i+1 during chunk i, one barrier per chunk); each
//      thread owns 8x8 register tiles and per k reads 8 rows of L21 and 8 columns of U12 (four
//      vector loads) for 64 FMAs.  The trailing matrix is read and written once per panel.
// Rows and columns past the last partial panel are padded with the identity, which leaves the
// factors unchanged.  A pivot below 1e-14 in magnitude (the reference LU's tolerance) marks the
// scenario singular.  Shared memory: dense_lu_elems(N, W) elements.  The register-resident
// steps A and B are separate (non-inlined) functions: each then gets the full register budget
// for its unrolled W-element row, instead of sharing it with the trailing-update tiles.
constexpr int DCW = 128;

__host__ __device__ __forceinline__ size_t dense_lu_elems(int N, int W) {
    return (size_t)W * dense_ld(N) + 2 * (size_t)W * DCW + (size_t)W * (W + 4) + (size_t)W;
}

// A: factor the diagonal block A[k0.., k0..] (w <= W rows and columns) in the lanes of one warp.
// Returns 1 if a pivot is below the tolerance.
template <typename T, int W>
__device__ __noinline__ int dense_diag_block(T* A, int ld, int k0, int w, T* PT, int pld, T* SL,
                                             T* SD) {
    const int r = threadIdx.x & 31;
    T a[W];
    if (r < w) {
        const T* row = A + (size_t)(k0 + r) * ld + k0;
#pragma unroll
        for (int c4 = 0; c4 < W; c4 += 4) {
            // columns up to ld - 1 lie inside the padded row
            const V4<T> v = k0 + c4 < ld ? ld4(row + c4) : V4<T>{{T(0), T(0), T(0), T(0)}};
#pragma unroll
            for (int t = 0; t < 4; ++t) a[c4 + t] = c4 + t < w ? v.v[t] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < W; ++c) a[c] = c == r ? T(1) : T(0);
    }
    int badl = 0;
#pragma unroll
    for (int kk = 0; kk < W; ++kk) {
        const T piv = __shfl_sync(0xffffffffu, a[kk], kk);
        if (kk < w && !(fabs(piv) >= T(1e-14))) badl = 1;
        const T inv = T(1) / piv;
        if (r == 0) SD[kk] = inv;
        const bool below = r > kk;
        const T l = a[kk] * inv;
        if (below) a[kk] = l;
#pragma unroll
        for (int c = kk + 1; c < W; ++c) {
            const T u = __shfl_sync(0xffffffffu, a[c], kk);
            if (below) a[c] = fma(-l, u, a[c]);
        }
    }
    if (r < W) {
#pragma unroll
        for (int c = 0; c < W; ++c) PT[c * pld + r] = a[c];  // U11 read as PT[c][k], k <= c
    }
    if (r < w) {
        T* row = A + (size_t)(k0 + r) * ld + k0;
        if (w == W) {
#pragma unroll
            for (int c4 = 0; c4 < W; c4 += 4) st4(row + c4, V4<T>{{a[c4], a[c4 + 1], a[c4 + 2], a[c4 + 3]}});
        } else {
#pragma unroll
            for (int c = 0; c < W; ++c)
                if (c < w) row[c] = a[c];
        }
    }
    if (r < W) {
#pragma unroll
        for (int c = 0; c < W; ++c) SL[r * (W + 4) + c] = a[c];  // L11 row-major, stride W + 4
    }
    return badl;
}

// B, one row of L21: x U11 = a for the row at `row` (W values; U11 transposed in PT with row
// stride pld), written back and, when PTr is given, to PTr[c * pld].
template <typename T, int W>
__device__ __noinline__ void dense_l21_row(T* row, const T* PT, int pld, const T* SD, T* PTr) {
    T x[W];
#pragma unroll
    for (int c4 = 0; c4 < W; c4 += 4) {
        const V4<T> v = ld4(row + c4);
#pragma unroll
        for (int t = 0; t < 4; ++t) x[c4 + t] = v.v[t];
    }
#pragma unroll
    for (int c = 0; c < W; ++c) {
        T s0 = x[c], s1 = T(0);
#pragma unroll
        for (int k4 = 0; k4 < c; k4 += 4) {
            const V4<T> u = ld4(PT + c * pld + k4);
#pragma unroll
            for (int t = 0; t < 4; ++t)
                if (k4 + t < c) {
                    if (t & 1) s1 = fma(-x[k4 + t], u.v[t], s1);
                    else s0 = fma(-x[k4 + t], u.v[t], s0);
                }
        }
        x[c] = (s0 + s1) * SD[c];
    }
    if (PTr) {
#pragma unroll
        for (int c = 0; c < W; ++c) PTr[c * pld] = x[c];
    }
#pragma unroll
    for (int c4 = 0; c4 < W; c4 += 4) st4(row + c4, V4<T>{{x[c4], x[c4 + 1], x[c4 + 2], x[c4 + 3]}});
}

// B, one column of U12: L11 y = a (unit lower) for the column at `col` (W values, stride ld),
// in place; L11 row-major in SL with row stride W + 4.
template <typename T, int W>
__device__ __noinline__ void dense_u12_col(T* col, const T* SL, int ld) {
    T y[W];
#pragma unroll
    for (int i = 0; i < W; ++i) y[i] = col[(size_t)i * ld];
#pragma unroll
    for (int i = 1; i < W; ++i) {
        T s0 = y[i], s1 = T(0);
#pragma unroll
        for (int k4 = 0; k4 < i; k4 += 4) {
            const V4<T> l = ld4(SL + i * (W + 4) + k4);
#pragma unroll
            for (int t = 0; t < 4; ++t)
                if (k4 + t < i) {
                    if (t & 1) s1 = fma(-l.v[t], y[k4 + t], s1);
                    else s0 = fma(-l.v[t], y[k4 + t], s0);
                }
        }
        y[i] = s0 + s1;
    }
#pragma unroll
    for (int i = 0; i < W; ++i) col[(size_t)i * ld] = y[i];
}

template <typename T, int W>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_dense_lu(BatchDev B, int N) {
    static_assert(W == 8 || W == 16 || W == 32, "panel width");
    const int q = blockIdx.x;
    if (q >= B.n_scen || !B.solving[q] || (B.gfactor && !B.gfactor[q / B.sw])) return;
    const int ld = dense_ld(N);
    T* A = reinterpret_cast<T*>(B.Dt) + (size_t)q * N * ld;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* PT = reinterpret_cast<T*>(smraw);        // [W][ld]: PT[c*ld + r] = panel (r, c)
    T* Ub0 = PT + (size_t)W * ld;               // [W][DCW] U12 chunk, two buffers
    T* Ub1 = Ub0 + W * DCW;
    T* SL = Ub1 + W * DCW;                      // [W][W + 4] L11 row-major
    T* SD = SL + W * (W + 4);                         // [W] 1 / U11 diagonal
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x;
    constexpr int VE = 16 / sizeof(T);
    if (tid == 0) bad = 0;
    // panel trace stamp j of this scenario (the address is rebuilt from the kernel
    // parameters at each stamp, so that the trace holds no registers across the loop)
    auto stamp = [&](int j, bool copy_prev) {
        if (B.dlu_ts && tid == 0) {
            unsigned long long* t = B.dlu_ts + (size_t)q * (1 + 3 * ((N + W - 1) / W)) + j;
            *t = copy_prev ? t[-1] : gtimer();
        }
    };
    stamp(0, false);
    for (int k0 = 0; k0 < N; k0 += W) {
        const int w = min(W, N - k0);
        const int m = N - k0;
        const int n2 = m - w;  // > 0 only for full panels
        // ---- A: diagonal block, warp 0
        if (tid < 32) {
            if (dense_diag_block<T, W>(A, ld, k0, w, PT, ld, SL, SD)) bad = 1;
        }
        __syncthreads();
        stamp(1 + 3 * (k0 / W), false);
        if (n2 > 0) {
            // ---- B: rows of L21 and columns of U12, one per thread at a time
            for (int it = tid; it < 2 * n2; it += nt) {
                if (it < n2) {
                    const int r = W + it;
                    dense_l21_row<T, W>(A + (size_t)(k0 + r) * ld + k0, PT, ld, SD, PT + r);
                } else {
                    dense_u12_col<T, W>(A + (size_t)k0 * ld + k0 + W + (it - n2), SL, ld);
                }
            }
            __syncthreads();
            stamp(2 + 3 * (k0 / W), false);
            // ---- C: trailing update, U12 in double-buffered chunks
            const int nch = (n2 + DCW - 1) / DCW;
            auto stage = [&](int ch, T* buf) {
                const int c0 = ch * DCW;
                const int cwp = (min(DCW, n2 - c0) + 7) & ~7;
                const int vpr = cwp / VE;
                // the columns past N are row padding and only ever feed padding columns
                for (int e2 = tid; e2 < W * vpr; e2 += nt) {
                    const int r = e2 / vpr, c = (e2 % vpr) * VE;
                    cp_async<16>(buf + r * DCW + c, A + (size_t)(k0 + r) * ld + k0 + W + c0 + c);
                }
            };
            stage(0, Ub0);
            cp_async_wait_all();
            __syncthreads();
            for (int ch = 0; ch < nch; ++ch) {
                T* cur = (ch & 1) ? Ub1 : Ub0;
                if (ch + 1 < nch) stage(ch + 1, (ch & 1) ? Ub0 : Ub1);
                const int c0 = ch * DCW;
                const int tcn = ((min(DCW, n2 - c0) + 7) & ~7) / 8;
                const int tr8 = (n2 + 7) / 8;
                const int ntile = tr8 * tcn;
                for (int tix = tid; tix < ntile; tix += nt) {
                    const int i0 = W + (tix / tcn) * 8, cc0 = (tix % tcn) * 8;
                    if (tix + nt < ntile) {
                        // the thread's next tile goes to L2 while this one computes
                        const int j0 = W + ((tix + nt) / tcn) * 8, dc0 = ((tix + nt) % tcn) * 8;
                        const T* pf = A + (size_t)(k0 + j0) * ld + k0 + W + c0 + dc0;
#pragma unroll
                        for (int ii = 0; ii < 8; ++ii)
                            if (j0 + ii < m) prefetch_l2(pf + (size_t)ii * ld);
                    }
                    T acc[8][8];
#pragma unroll
                    for (int ii = 0; ii < 8; ++ii) {
                        if (i0 + ii < m) {
                            const T* row = A + (size_t)(k0 + i0 + ii) * ld + k0 + W + c0 + cc0;
                            const V4<T> a = ld4(row), b = ld4(row + 4);
#pragma unroll
                            for (int c = 0; c < 4; ++c) { acc[ii][c] = a.v[c]; acc[ii][c + 4] = b.v[c]; }
                        } else {
#pragma unroll
                            for (int c = 0; c < 8; ++c) acc[ii][c] = T(0);
                        }
                    }
#pragma unroll 2
                    for (int r = 0; r < W; ++r) {
                        const V4<T> l0 = ld4(PT + r * ld + i0), l1 = ld4(PT + r * ld + i0 + 4);
                        const V4<T> u0 = ld4(cur + r * DCW + cc0), u1 = ld4(cur + r * DCW + cc0 + 4);
#pragma unroll
                        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                acc[ii][c] = fma(-l0.v[ii], u0.v[c], acc[ii][c]);
                                acc[ii][c + 4] = fma(-l0.v[ii], u1.v[c], acc[ii][c + 4]);
                                acc[ii + 4][c] = fma(-l1.v[ii], u0.v[c], acc[ii + 4][c]);
                                acc[ii + 4][c + 4] = fma(-l1.v[ii], u1.v[c], acc[ii + 4][c + 4]);
                            }
                    }
#pragma unroll
                    for (int ii = 0; ii < 8; ++ii) {
                        if (i0 + ii < m) {
                            T* row = A + (size_t)(k0 + i0 + ii) * ld + k0 + W + c0 + cc0;
                            st4(row, V4<T>{{acc[ii][0], acc[ii][1], acc[ii][2], acc[ii][3]}});
                            st4(row + 4, V4<T>{{acc[ii][4], acc[ii][5], acc[ii][6], acc[ii][7]}});
                        }
                    }
                }
                cp_async_wait_all();
                __syncthreads();
            }
        } else {
            stamp(2 + 3 * (k0 / W), true);
        }
        stamp(3 + 3 * (k0 / W), false);
    }
    if (tid == 0 && bad) B.singular[q] = 1;
}

}  // namespace gapk

#include "dense_lu_tc.cuh"

namespace gapk {

// Host side: opt in to the kernel's shared memory and launch it for panel width W.  With `tc`
// (FP32, W = 32) the tail is factorised by k_dense_lu_tc instead, the trailing update on the
// tensor cores; its shared memory does not depend on N.
template <typename T>
cudaError_t dense_lu_attributes(int W, size_t smem, bool tc) {
    auto set = [&](auto fn, size_t bytes) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return e;
    };
    if constexpr (sizeof(T) == 4) {
        if (tc) return W == 32 ? set(k_dense_lu_tc, dense_lu_tc_smem()) : cudaErrorInvalidValue;
    }
    switch (W) {
        case 32: return set(k_dense_lu<T, 32>, smem);
        case 16: return set(k_dense_lu<T, 16>, smem);
        case 8: return set(k_dense_lu<T, 8>, smem);
    }
    return cudaErrorInvalidValue;
}

template <typename T>
void launch_dense_lu(int W, int grid, size_t smem, cudaStream_t st, BatchDev const& B, int N, bool tc) {
    if constexpr (sizeof(T) == 4) {
        if (tc) {
            k_dense_lu_tc<<<grid, 256, dense_lu_tc_smem(), st>>>(B, N);
            return;
        }
    }
    switch (W) {
        case 32: k_dense_lu<T, 32><<<grid, 256, smem, st>>>(B, N); break;
        case 16: k_dense_lu<T, 16><<<grid, 256, smem, st>>>(B, N); break;
        case 8: k_dense_lu<T, 8><<<grid, 256, smem, st>>>(B, N); break;
    }
}

// Split dense LU (the batch path): the same right-looking factorisation as k_dense_lu, one
// panel of W = 32 columns at a time, as two launches per panel so that the rank-W trailing
// update of every scenario is spread over many small CTAs instead of one CTA per scenario:
//   k_dlu_panel  one CTA per scenario: steps A and B (diagonal block in one warp, whole L21 rows
//                and U12 columns per thread), written back to the tail in global memory;
//   k_dlu_update one CTA per (scenario, 64 x 64 tile of the trailing matrix): the tile's L21
//                rows (transposed) and U12 columns staged in shared memory, 8x8 register tiles
//                per thread, C -= L21 U12 in place.
// No dynamic shared memory, so the tail size is limited only by device memory.
constexpr int DLU_W = 32, DLU_TILE = 64;

template <typename T>
__global__ void __launch_bounds__(128) k_dlu_panel(BatchDev B, int N, int k0) {
    constexpr int W = DLU_W;
    const int q = blockIdx.x;
    if (q >= B.n_scen || !B.solving[q] || (B.gfactor && !B.gfactor[q / B.sw])) return;
    const int ld = dense_ld(N);
    T* A = reinterpret_cast<T*>(B.Dt) + (size_t)q * N * ld;
    __shared__ __align__(16) T U11[W * (W + 4)];  // transposed: U11[c][k], stride W + 4
    __shared__ __align__(16) T SL[W * (W + 4)];   // L11 row-major, stride W + 4
    __shared__ __align__(16) T SD[W];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int w = min(W, N - k0);
    const int n2 = N - k0 - w;
    if (tid < 32) {
        if (dense_diag_block<T, W>(A, ld, k0, w, U11, W + 4, SL, SD)) B.singular[q] = 1;
    }
    __syncthreads();
    for (int it = tid; it < 2 * n2; it += nt) {
        if (it < n2)
            dense_l21_row<T, W>(A + (size_t)(k0 + W + it) * ld + k0, U11, W + 4, SD, nullptr);
        else
            dense_u12_col<T, W>(A + (size_t)k0 * ld + k0 + W + (it - n2), SL, ld);
    }
}

template <typename T>
__global__ void __launch_bounds__(64, sizeof(T) == 4 ? 8 : 4)
    k_dlu_update(BatchDev B, int N, int k0, int tiles_j) {
    constexpr int W = DLU_W, TS = DLU_TILE;
    const int q = blockIdx.y;
    if (q >= B.n_scen || !B.solving[q] || (B.gfactor && !B.gfactor[q / B.sw])) return;
    const int ld = dense_ld(N);
    T* A = reinterpret_cast<T*>(B.Dt) + (size_t)q * N * ld;
    const int n2 = N - k0 - W;
    const int i0 = (blockIdx.x / tiles_j) * TS, j0 = (blockIdx.x % tiles_j) * TS;
    __shared__ __align__(16) T LT[W][TS];  // LT[c][r] = L21(i0 + r, c)
    __shared__ __align__(16) T UT[W][TS];  // UT[r][c] = U12(r, j0 + c)
    const int tid = threadIdx.x;
    T* base = A + (size_t)(k0 + W) * ld + k0 + W;  // trailing matrix origin
    {
        // one L21 row per thread (TS rows, TS threads); rows past the matrix are zero
        const int r = tid;
        if (i0 + r < n2) {
            const T* row = A + (size_t)(k0 + W + i0 + r) * ld + k0;
#pragma unroll
            for (int c4 = 0; c4 < W; c4 += 4) {
                const V4<T> v = ld4(row + c4);
#pragma unroll
                for (int t = 0; t < 4; ++t) LT[c4 + t][r] = v.v[t];
            }
        } else {
#pragma unroll
            for (int c = 0; c < W; ++c) LT[c][r] = T(0);
        }
        // U12 rows 0..W-1, columns j0..j0+TS-1 in groups of 4; a group that starts inside the
        // matrix ends inside the padded row (k0 + W and ld are multiples of 8)
        for (int e = tid; e < W * (TS / 4); e += TS) {
            const int r2 = e / (TS / 4), c = (e % (TS / 4)) * 4;
            const V4<T> v = j0 + c < n2 ? ld4(A + (size_t)(k0 + r2) * ld + k0 + W + j0 + c)
                                        : V4<T>{{T(0), T(0), T(0), T(0)}};
            st4(&UT[r2][c], v);
        }
    }
    __syncthreads();
    const int r0 = (tid / 8) * 8, c0 = (tid % 8) * 8;
    if (i0 + r0 >= n2 || j0 + c0 >= n2) return;
    T acc[8][8];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
        if (i0 + r0 + ii < n2) {
            const T* row = base + (size_t)(i0 + r0 + ii) * ld + j0 + c0;
            const V4<T> a = ld4(row), b = ld4(row + 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                acc[ii][c] = a.v[c];
                acc[ii][c + 4] = b.v[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[ii][c] = T(0);
        }
    }
#pragma unroll 2
    for (int r = 0; r < W; ++r) {
        const V4<T> l0 = ld4(&LT[r][r0]), l1 = ld4(&LT[r][r0 + 4]);
        const V4<T> u0 = ld4(&UT[r][c0]), u1 = ld4(&UT[r][c0 + 4]);
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                acc[ii][c] = fma(-l0.v[ii], u0.v[c], acc[ii][c]);
                acc[ii][c + 4] = fma(-l0.v[ii], u1.v[c], acc[ii][c + 4]);
                acc[ii + 4][c] = fma(-l1.v[ii], u0.v[c], acc[ii + 4][c]);
                acc[ii + 4][c + 4] = fma(-l1.v[ii], u1.v[c], acc[ii + 4][c + 4]);
            }
    }
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
        if (i0 + r0 + ii < n2) {
            T* row = base + (size_t)(i0 + r0 + ii) * ld + j0 + c0;
            st4(row, V4<T>{{acc[ii][0], acc[ii][1], acc[ii][2], acc[ii][3]}});
            st4(row + 4, V4<T>{{acc[ii][4], acc[ii][5], acc[ii][6], acc[ii][7]}});
        }
    }
}

// Host side: the split factorisation of every scenario's N x N tail (grid = padded scenarios).
// With `tc` (FP32) the trailing updates of at least one full 128 x 128 tile run on the tensor
// cores (k_dlu_update_tc; its shared memory opted in by split_lu_attributes); smaller trailing
// blocks, mostly empty as tensor-core tiles, keep the 64 x 64 CUDA-core tiles.
template <typename T>
void launch_dense_lu_split(int grid, cudaStream_t st, BatchDev const& B, int N, bool tc) {
    for (int k0 = 0; k0 < N; k0 += DLU_W) {
        k_dlu_panel<T><<<grid, 128, 0, st>>>(B, N, k0);
        const int n2 = N - k0 - DLU_W;
        if (n2 > 0) {
            if constexpr (sizeof(T) == 4) {
                if (tc && n2 >= TC_N) {
                    const int tt = (n2 + TC_N - 1) / TC_N;
                    k_dlu_update_tc<<<dim3(tt * tt, grid), 256, TC_OPER_BYTES, st>>>(B, N, k0, tt);
                    continue;
                }
            }
            const int tj = (n2 + DLU_TILE - 1) / DLU_TILE;
            k_dlu_update<T><<<dim3(tj * tj, grid), DLU_TILE, 0, st>>>(B, N, k0, tj);
        }
    }
}
inline cudaError_t split_lu_attributes() {
    return cudaFuncSetAttribute(k_dlu_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TC_OPER_BYTES);
}

// Forward (unit L) then backward (U) substitution on one scenario's tail vector, blocked by
// 32 rows.  Per block, the dot products of its rows with the solved part stream the factor:
// warp w takes rows w, w + 8, w + 16, w + 24 of the block together, each lane reading one
// 4-element vector per row per step (128 columns per warp-wide load), so every thread keeps
// four vector loads in flight; the block's 32 x 32 triangle is staged in shared memory by the
// whole CTA (one vector per thread) at the same time, and warp 0 then solves it with shuffles.
// At <= 36 registers, seven CTAs fit on an SM, so a 1024-scenario batch runs in one wave.  y
// lives in shared memory, ld = dense_ld(N) entries, zero beyond N (the factor's padding
// columns hold no values and are masked).
template <typename T>
__device__ __forceinline__ void dense_dot4(const T* __restrict__ A, int ld, int r0, int wid,
                                           int ln, int cb, int ce, int N, const T* y, T acc[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = T(0);
#pragma unroll 1
    for (int c = cb + 4 * ln; c < ce; c += 128) {
        const V4<T> yv = ld4(y + c);
        V4<T> a[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = r0 + wid + 8 * i;
            a[i] = row < N ? ld4(A + (size_t)row * ld + c) : V4<T>{{T(0), T(0), T(0), T(0)}};
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int t = 0; t < 4; ++t) acc[i] = fma(c + t < N ? a[i].v[t] : T(0), yv.v[t], acc[i]);
    }
}

// The 32 x 32 diagonal block at (r0, r0) into tri[32][33], one 4-vector per thread of the
// first 256 (a vector that starts inside the padded row ends inside it, ld % 8 == 0).
template <typename T>
__device__ __forceinline__ void dense_stage_tri(const T* __restrict__ A, int ld, int r0, int N,
                                                T (*tri)[33]) {
    const int t = threadIdx.x;
    if (t < 256) {
        const int r = t >> 3, c = (t & 7) * 4;
        const V4<T> v = r0 + r < N && r0 + c < ld ? ld4(A + (size_t)(r0 + r) * ld + r0 + c)
                                                 : V4<T>{{T(0), T(0), T(0), T(0)}};
#pragma unroll
        for (int k = 0; k < 4; ++k) tri[r][c + k] = v.v[k];
    }
}

template <typename T, int SW>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 7 : 4) k_dense_solve(PlanDev P, BatchDev B, double2* out,
                                                        int accumulate) {
    const int q = blockIdx.x;
    if (q >= B.n_scen || !B.solving[q]) return;
    const int g = q / SW, lane = q % SW;
    if (accumulate && B.grefine && !B.grefine[g]) return;
    const int N = 2 * P.n_tail, ld = dense_ld(N);
    const T* A = reinterpret_cast<const T*>(B.Dt) + (size_t)q * N * ld;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* y = reinterpret_cast<T*>(smraw);
    __shared__ T tri[32][33];
    const int tid = threadIdx.x, wid = tid >> 5, ln = tid & 31;
    for (int i = tid; i < ld / 2; i += blockDim.x) {
        const Vec2<T> v = i < P.n_tail ? ldv(X + (size_t)(P.ns + i) * SW + lane) : Vec2<T>{T(0), T(0)};
        y[2 * i] = v.x;
        y[2 * i + 1] = v.y;
    }
    __syncthreads();
    // L y = b, unit lower
    for (int r0 = 0; r0 < N; r0 += 32) {
        dense_stage_tri<T>(A, ld, r0, N, tri);
        if (r0 > 0) {
            T acc[4];
            // blockDim is 256: 8 warps x 4 rows = the 32 rows of the block
            dense_dot4<T>(A, ld, r0, wid, ln, 0, r0, N, y, acc);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
#pragma unroll
                for (int off = 16; off; off >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
            }
            if (ln == 0) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (r0 + wid + 8 * i < N) y[r0 + wid + 8 * i] -= acc[i];
            }
        }
        __syncthreads();
        if (wid == 0) {
            const int row = r0 + ln;
            T v = row < N ? y[row] : T(0);
            for (int j = 0; j < 32; ++j) {
                const T vj = __shfl_sync(0xffffffffu, v, j);
                if (ln > j && row < N && r0 + j < N) v = fma(-tri[ln][j], vj, v);
            }
            if (row < N) y[row] = v;
        }
        __syncthreads();
    }
    // U x = y
    const int last = ((N - 1) / 32) * 32;
    for (int r0 = last; r0 >= 0; r0 -= 32) {
        const int r1 = min(r0 + 32, N);
        dense_stage_tri<T>(A, ld, r0, N, tri);
        if (r1 < N) {
            T acc[4];
            dense_dot4<T>(A, ld, r0, wid, ln, r1, ld, N, y, acc);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
#pragma unroll
                for (int off = 16; off; off >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
            }
            if (ln == 0) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (r0 + wid + 8 * i < N) y[r0 + wid + 8 * i] -= acc[i];
            }
        }
        __syncthreads();
        if (wid == 0) {
            const int row = r0 + ln;
            T v = row < N ? y[row] : T(0);
            for (int j = 31; j >= 0; --j) {
                if (r0 + j < N) {
                    if (ln == j) v = v / tri[j][j];
                    const T vj = __shfl_sync(0xffffffffu, v, j);
                    if (ln < j && row < N) v = fma(-tri[ln][j], vj, v);
                }
            }
            if (row < N) y[row] = v;
        }
        __syncthreads();
    }
    double2* O = out + (size_t)g * P.nb * SW;
    for (int i = tid; i < P.n_tail; i += blockDim.x) {
        const int k = P.ns + i;
        stv(X + (size_t)k * SW + lane, Vec2<T>{y[2 * i], y[2 * i + 1]});
        double2* o = O + (size_t)k * SW + lane;
        if (accumulate) {
            const double2 old = *o;
            *o = make_double2(old.x + (double)y[2 * i], old.y + (double)y[2 * i + 1]);
        } else {
            *o = make_double2((double)y[2 * i], (double)y[2 * i + 1]);
        }
    }
}

// Dynamic shared memory of k_dense_solve / k_dense_solve_t: the tail vector, padded to ld.
__host__ __forceinline__ size_t dense_solve_smem(int n_tail, size_t esz) {
    return (size_t)dense_ld(2 * n_tail) * esz;
}

// ---------------------------------------------------------------------------------------
// sparse triangular solves: L y = b (unit lower) over the sparse levels, then every tail
// node gathers its sparse contributions; U x = y over the sparse levels (descending) once
// the dense tail is solved.  x is written as FP64 (optionally added to `out`).
// ---------------------------------------------------------------------------------------
// Levels with few nodes split every row over s sub-slots (s a power of two, up to 32): the
// sub-slots of one warp reduce with shuffles, the warps of one row through shared memory.
// split_factor: the largest s <= 32 with c * s <= ne (at least 1).
__device__ __forceinline__ int split_factor(int c, int ne) {
    int s = 1;
    while (s < 32 && c * s * 2 <= ne) s *= 2;
    return s;
}

// Sum `acc` over the s sub-slots of each row (slot e0 = row * s + sub); the result is valid in
// sub-slot 0.  Every thread of the block calls this (uniform s).
template <typename T, int SW>
__device__ __forceinline__ Vec2<T> split_reduce(Vec2<T> acc, int s, int sub, int row, int lane,
                                                Vec2<T>* red) {
    constexpr int S = 32 / SW;  // slots per warp
    const int sw = s < S ? s : S;
    for (int d = 1; d < sw; d *= 2) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, d * SW);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, d * SW);
    }
    if (s > S) {
        const int parts = s / S;
        if (sub % S == 0) red[(row * parts + sub / S) * SW + lane] = acc;
        __syncthreads();
        if (sub == 0) {
            acc = red[(row * parts) * SW + lane];
            for (int w = 1; w < parts; ++w) {
                const Vec2<T> v = red[(row * parts + w) * SW + lane];
                acc.x += v.x;
                acc.y += v.y;
            }
        }
    }
    return acc;
}

template <typename T, int SW>
__global__ void k_solve_fwd(PlanDev P, BatchDev B, const double2* __restrict__ rhs,
                            int refine_pass) {
    const int g = blockIdx.x;
    if (!B.gsolve[g] || (refine_pass && B.grefine && !B.grefine[g])) return;
    __shared__ Vec2<T> red[256];  // (blockDim / (32 / SW)) partial sums, <= 256 for SW <= 8
    const Blk<T>* F = reinterpret_cast<const Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    const double2* R = rhs + (size_t)g * P.nb * SW;
    const int lane = threadIdx.x % SW;
    const int e0 = threadIdx.x / SW, ne = blockDim.x / SW;
    if (B.lvl_ts) lvl_stamp(B, P.n_levels, 1, g, 0);
    for (int h = 0; h < P.n_levels; ++h) {
        const int lb = P.level_ptr[h], c = P.level_ptr[h + 1] - lb;
        const int s = split_factor(c, ne);
        if (s == 1) {
            // two nodes per worker at a time (nodes of one level are independent)
            for (int t = lb + e0; t < lb + c; t += 2 * ne) {
                const bool two = t + ne < lb + c;
                const int k = P.level_nodes[t];
                const int k2 = two ? P.level_nodes[t + ne] : k;
                const double2 b = R[(size_t)k * SW + lane];
                const double2 b2 = R[(size_t)k2 * SW + lane];
                Vec2<T> acc = {(T)b.x, (T)b.y}, acc2 = {(T)b2.x, (T)b2.y};
                const int qa = P.rptr[k], qe = P.rptr[k + 1];
                const int qa2 = two ? P.rptr[k2] : 0, qe2 = two ? P.rptr[k2 + 1] : 0;
                const int nb = min(qe - qa, qe2 - qa2);
#pragma unroll 2
                for (int i = 0; i < nb; ++i) {
                    const int2 r = P.rlist[qa + i];
                    const int2 r2 = P.rlist[qa2 + i];
                    msubv(acc, ldb(F + (size_t)r.x * SW + lane), ldv(X + (size_t)r.y * SW + lane));
                    msubv(acc2, ldb(F + (size_t)r2.x * SW + lane), ldv(X + (size_t)r2.y * SW + lane));
                }
#pragma unroll 4
                for (int q = qa + nb; q < qe; ++q) {
                    const int2 r = P.rlist[q];
                    msubv(acc, ldb(F + (size_t)r.x * SW + lane), ldv(X + (size_t)r.y * SW + lane));
                }
#pragma unroll 4
                for (int q = qa2 + nb; q < qe2; ++q) {
                    const int2 r = P.rlist[q];
                    msubv(acc2, ldb(F + (size_t)r.x * SW + lane), ldv(X + (size_t)r.y * SW + lane));
                }
                stv(X + (size_t)k * SW + lane, acc);
                if (two) stv(X + (size_t)k2 * SW + lane, acc2);
            }
        } else {
            const int j = e0 / s, sub = e0 % s;
            const int k = j < c ? P.level_nodes[lb + j] : 0;
            Vec2<T> acc = {T(0), T(0)};
            if (j < c) {
#pragma unroll 4
                for (int q = P.rptr[k] + sub; q < P.rptr[k + 1]; q += s) {
                    const int2 r = P.rlist[q];
                    msubv(acc, ldb(F + (size_t)r.x * SW + lane), ldv(X + (size_t)r.y * SW + lane));
                }
            }
            acc = split_reduce<T, SW>(acc, s, sub, j, lane, red);
            if (j < c && sub == 0) {
                const double2 b = R[(size_t)k * SW + lane];
                stv(X + (size_t)k * SW + lane, Vec2<T>{(T)b.x + acc.x, (T)b.y + acc.y});
            }
        }
        __syncthreads();
        if (B.lvl_ts) lvl_stamp(B, P.n_levels, 1, g, h + 1);
    }
    {
        // tail rows gather long sparse rows: 4 sub-slots per row (a shuffle reduction within
        // the warp, 4 <= 32 / SW), rounds uniform across the block
        constexpr int TS = 4;
        const int sub = e0 % TS, per = ne / TS;
        for (int base = P.ns; base < P.nb; base += per) {
            const int k = base + e0 / TS;
            Vec2<T> acc = {T(0), T(0)};
            if (k < P.nb) {
#pragma unroll 4
                for (int q = P.rptr[k] + sub; q < P.rptr[k + 1]; q += TS) {
                    const int2 r = P.rlist[q];
                    msubv(acc, ldb(F + (size_t)r.x * SW + lane), ldv(X + (size_t)r.y * SW + lane));
                }
            }
            acc = split_reduce<T, SW>(acc, TS, sub, 0, lane, red);
            if (k < P.nb && sub == 0) {
                const double2 b = R[(size_t)k * SW + lane];
                stv(X + (size_t)k * SW + lane, Vec2<T>{(T)b.x + acc.x, (T)b.y + acc.y});
            }
        }
    }
    if (B.lvl_ts) {
        __syncthreads();
        lvl_stamp(B, P.n_levels, 1, g, P.n_levels + 1);
    }
}

template <typename T, int SW>
__global__ void k_solve_bwd(PlanDev P, BatchDev B, double2* out, int accumulate) {
    const int g = blockIdx.x;
    if (!B.gsolve[g] || (accumulate && B.grefine && !B.grefine[g])) return;
    __shared__ Vec2<T> red[256];
    const Blk<T>* F = reinterpret_cast<const Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    double2* O = out + (size_t)g * P.nb * SW;
    const int lane = threadIdx.x % SW;
    const int e0 = threadIdx.x / SW, ne = blockDim.x / SW;
    const int Ub = P.nb + P.nnz_l;
    auto finish = [&](int k, Vec2<T> acc) {
        const Vec2<T> x = mulv(ldb(F + (size_t)k * SW + lane), acc);
        stv(X + (size_t)k * SW + lane, x);
        double2* o = O + (size_t)k * SW + lane;
        if (accumulate) {
            const double2 old = *o;
            *o = make_double2(old.x + (double)x.x, old.y + (double)x.y);
        } else {
            *o = make_double2((double)x.x, (double)x.y);
        }
    };
    if (B.lvl_ts) lvl_stamp(B, P.n_levels, 2, g, 0);
    for (int h = P.n_levels - 1; h >= 0; --h) {
        const int lb = P.level_ptr[h], c = P.level_ptr[h + 1] - lb;
        const int s = split_factor(c, ne);
        if (s == 1) {
            // two nodes per worker at a time (nodes of one level are independent)
            for (int t = lb + e0; t < lb + c; t += 2 * ne) {
                const bool two = t + ne < lb + c;
                const int k = P.level_nodes[t];
                const int k2 = two ? P.level_nodes[t + ne] : k;
                Vec2<T> acc = ldv(X + (size_t)k * SW + lane);
                Vec2<T> acc2 = ldv(X + (size_t)k2 * SW + lane);
                const int pa = P.lptr[k], pe = P.lptr[k + 1];
                const int pa2 = two ? P.lptr[k2] : 0, pe2 = two ? P.lptr[k2 + 1] : 0;
                const int nb = min(pe - pa, pe2 - pa2);
#pragma unroll 2
                for (int i = 0; i < nb; ++i) {
                    msubv(acc, ldb(F + (size_t)(Ub + pa + i) * SW + lane),
                          ldv(X + (size_t)P.lidx[pa + i] * SW + lane));
                    msubv(acc2, ldb(F + (size_t)(Ub + pa2 + i) * SW + lane),
                          ldv(X + (size_t)P.lidx[pa2 + i] * SW + lane));
                }
#pragma unroll 4
                for (int p = pa + nb; p < pe; ++p) {
                    msubv(acc, ldb(F + (size_t)(Ub + p) * SW + lane),
                          ldv(X + (size_t)P.lidx[p] * SW + lane));
                }
#pragma unroll 4
                for (int p = pa2 + nb; p < pe2; ++p) {
                    msubv(acc2, ldb(F + (size_t)(Ub + p) * SW + lane),
                          ldv(X + (size_t)P.lidx[p] * SW + lane));
                }
                finish(k, acc);
                if (two) finish(k2, acc2);
            }
        } else {
            const int j = e0 / s, sub = e0 % s;
            const int k = j < c ? P.level_nodes[lb + j] : 0;
            Vec2<T> acc = {T(0), T(0)};
            if (j < c) {
#pragma unroll 4
                for (int p = P.lptr[k] + sub; p < P.lptr[k + 1]; p += s) {
                    msubv(acc, ldb(F + (size_t)(Ub + p) * SW + lane),
                          ldv(X + (size_t)P.lidx[p] * SW + lane));
                }
            }
            acc = split_reduce<T, SW>(acc, s, sub, j, lane, red);
            if (j < c && sub == 0) {
                const Vec2<T> xk = ldv(X + (size_t)k * SW + lane);
                finish(k, Vec2<T>{xk.x + acc.x, xk.y + acc.y});
            }
        }
        __syncthreads();
        if (B.lvl_ts) lvl_stamp(B, P.n_levels, 2, g, P.n_levels - h);
    }
    if (B.lvl_ts) lvl_stamp(B, P.n_levels, 2, g, P.n_levels + 1);
}

// refinement residual: res = rhs - J dx with the FP64 Jacobian blocks
template <int SW>
__global__ void __launch_bounds__(256, 8) k_residual(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.gsolve[g] || (B.grefine && !B.grefine[g])) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = tid / SW, lane = tid % SW;
    if (k >= P.nb) return;
    const size_t base = (size_t)g * P.nb * SW;
    const double2 b = B.rhs[base + (size_t)k * SW + lane];
    Vec2<double> acc = {b.x, b.y};
    const Blk<double>* A = reinterpret_cast<const Blk<double>*>(B.A64) + (size_t)g * P.n_a * SW;
#pragma unroll 4
    for (int e = P.arow_ptr[k]; e < P.arow_ptr[k + 1]; ++e) {
        const int2 ac = P.arow[e];
        const double2 x = B.dx[base + (size_t)ac.y * SW + lane];
        msubv(acc, ldb(A + (size_t)ac.x * SW + lane), Vec2<double>{x.x, x.y});
    }
    B.res[base + (size_t)k * SW + lane] = make_double2(acc.x, acc.y);
}

// ---------------------------------------------------------------------------------------
// voltage update
// ---------------------------------------------------------------------------------------
template <int SW>
__global__ void __launch_bounds__(256, 8) k_update(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.gsolve[g]) return;
    const int n = P.n_bus;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = tid / SW, lane = tid % SW;
    if (i >= n) return;
    const int q = g * SW + lane;
    // the loads that do not depend on the flags below go first (padding lanes have storage),
    // so that one memory latency covers them and the flags
    const int node = P.node_of_bus[i];
    const size_t o = ((size_t)g * n + i) * SW + lane;
    double2 v = B.V[o];
    const bool pq = P.bus_type[i] == BUS_PQ;
    const double2 d = node >= 0 ? B.dx[((size_t)g * P.nb + node) * SW + lane] : make_double2(0.0, 0.0);
    if (q >= B.n_scen) return;  // padding lanes are never updated
    {
        if (B.singular[q]) {
            // the reference keeps V unchanged when factorize() fails and runs to max_iter
            if (i == 0 && B.solving[q]) {
                B.state[q] = 1;
                B.status[q] = SC_SINGULAR;
                B.iters[q] = B.ctrl[1];
                B.solving[q] = 0;
            }
            return;
        }
        if (!B.solving[q]) return;
    }
    if (node < 0) return;
    if (B.ctrl[3] != 1) {
        // reference policy (cpu_newton_raphson.cpp:457-503): damping 0.9 and the clamps;
        // clamped policy: the same clamps and order with the full step
        const double damp = B.ctrl[3] == 0 ? 0.9 : 1.0;
        const double vm = hypot(v.x, v.y);
        double a = damp * d.x;
        if (fabs(a) > 0.15) a = 0.15 * (a > 0 ? 1.0 : -1.0);
        double sn, cs;
        sincos(atan2(v.y, v.x) + a, &sn, &cs);
        v = make_double2(vm * cs, vm * sn);
        if (pq) {
            const double vm0 = hypot(v.x, v.y);
            double c = damp * d.y;
            if (fabs(c) > 0.08) c = 0.08 * (c > 0 ? 1.0 : -1.0);
            double vmn = vm0 + c;
            vmn = (vmn < 0.5) ? 0.5 : vmn;
            vmn = (1.5 < vmn) ? 1.5 : vmn;
            sincos(atan2(v.y, v.x), &sn, &cs);
            v = make_double2(vmn * cs, vmn * sn);
        }
    } else {
        // Newton step in polar form, |V| e^{j theta} -> (|V| + d|V|) e^{j (theta + dtheta)}:
        // V rotated by dtheta and scaled by (|V| + d|V|) / |V|, one sincos of the (small)
        // correction instead of atan2 and a sincos of the full angle
        const double vm = hypot(v.x, v.y);
        double sn, cs;
        sincos(d.x, &sn, &cs);
        if (vm > 0.0) {
            const double sc = pq ? (vm + d.y) / vm : 1.0;
            v = make_double2(sc * fma(v.x, cs, -v.y * sn), sc * fma(v.x, sn, v.y * cs));
        } else {
            const double m = pq ? d.y : 0.0;  // from V = 0 the angle is the correction's
            v = make_double2(m * cs, m * sn);
        }
    }
    B.V[o] = v;
}

// ---------------------------------------------------------------------------------------
// results out (scenario-major) and reference-order views of the stage vectors
// ---------------------------------------------------------------------------------------
template <int SW>
__global__ void k_store(PlanDev P, BatchDev B, double2* v_out, int* it_out, int* st_out,
                        double* fm_out) {
    const int n = P.n_bus;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)B.n_scen * n;
    if (tid < total) {
        const int s = (int)(tid / n), i = (int)(tid % n);
        const int g = s / SW, lane = s % SW;
        if (v_out) v_out[tid] = B.V[((size_t)g * n + i) * SW + lane];
        if (i == 0) {
            if (it_out) it_out[s] = B.iters[s];
            if (st_out) st_out[s] = B.status[s];
            if (fm_out) fm_out[s] = B.final_mis[s];
        }
    }
}

// current state per scenario in bus order: V, I = Y V and S = V conj(I), per unit
// (IterationState of powerflow_interface.h:28-35, filled as cpu_newton_raphson.cpp:125-149)
template <int SW>
__global__ void k_state(PlanDev P, BatchDev B, double2* v_out, double2* i_out,
                        double2* s_out) {
    const int n = P.n_bus;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)B.n_scen * n) return;
    const int s = (int)(tid / n), i = (int)(tid % n);
    const int g = s / SW, lane = s % SW;
    const double2* Vg = B.V + (size_t)g * n * SW;
    const double2* Yg = B.y_shared ? B.Y : B.Y + (size_t)g * P.nnz_y * SW;
    const size_t ys = B.y_shared ? 1 : SW;
    const size_t yl = B.y_shared ? 0 : lane;
    double ir = 0.0, ii = 0.0;
    for (int p = P.y_row_ptr[i]; p < P.y_row_ptr[i + 1]; ++p) {
        const double2 y = Yg[(size_t)p * ys + yl];
        const double2 v = Vg[(size_t)P.y_col[p] * SW + lane];
        ir = fma(y.x, v.x, ir);
        ir = fma(-y.y, v.y, ir);
        ii = fma(y.x, v.y, ii);
        ii = fma(y.y, v.x, ii);
    }
    const double2 vi = Vg[(size_t)i * SW + lane];
    if (v_out) v_out[tid] = vi;
    if (i_out) i_out[tid] = make_double2(ir, ii);
    if (s_out) s_out[tid] = make_double2(fma(vi.x, ir, vi.y * ii), fma(vi.y, ir, -vi.x * ii));
}

// node vector [G][nb][SW] -> reference order [n_scen][n_vars]; map[node*2+c] gives the
// reference index (or -1); sign multiplies the value
template <int SW>
__global__ void k_node_to_ref(const double2* __restrict__ src, int nb, int n_scen, int n_vars,
                              const int* __restrict__ map, double sign, double* dst) {
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)n_scen * nb) return;
    const int s = (int)(tid / nb), k = (int)(tid % nb);
    const int g = s / SW, lane = s % SW;
    const double2 v = src[((size_t)g * nb + k) * SW + lane];
    const int a = map[2 * k], b = map[2 * k + 1];
    if (a >= 0) dst[(size_t)s * n_vars + a] = sign * v.x;
    if (b >= 0) dst[(size_t)s * n_vars + b] = sign * v.y;
}

// ---------------------------------------------------------------------------------------
// adjoint: J^T lambda = dL/dx with the factors of J = L U
//   U^T z = g   : sparse forward sweep with U slots transposed (D^-T on sparse nodes), the
//                 tail gathers its sparse contributions, then a dense U_tt^T solve
//   L^T lam = z : dense L_tt^T solve, then a sparse backward sweep with L slots transposed
// ---------------------------------------------------------------------------------------
template <int SW>
__global__ void k_adj_prep(BatchDev B) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= B.n_groups * SW) return;
    B.solving[q] = q < B.n_scen ? 1 : 0;
    B.singular[q] = 0;
    if (q % SW == 0) {
        B.gsolve[q / SW] = 1;
        B.giter[q / SW] = 1;
    }
}

// g per node: (dL/dtheta, dL/d|V| for PQ buses); inputs scenario-major [n_scen][n_bus]
template <int SW>
__global__ void k_adj_rhs(PlanDev P, BatchDev B, const double* __restrict__ dvm,
                          const double* __restrict__ dva) {
    const int g = blockIdx.y;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = tid / SW, lane = tid % SW;
    if (i >= P.n_bus) return;
    const int node = P.node_of_bus[i];
    if (node < 0) return;
    const int q = g * SW + lane;
    const int src = q < B.n_scen ? q : g * SW;
    const double gt = dva[(size_t)src * P.n_bus + i];
    const double gv = P.bus_type[i] == BUS_PQ ? dvm[(size_t)src * P.n_bus + i] : 0.0;
    B.rhs[((size_t)g * P.nb + node) * SW + lane] = make_double2(gt, gv);
}

template <typename T, int SW>
__global__ void k_solve_fwd_t(PlanDev P, BatchDev B, const double2* __restrict__ rhs) {
    const int g = blockIdx.x;
    if (!B.gsolve[g]) return;
    const Blk<T>* F = reinterpret_cast<const Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    const double2* R = rhs + (size_t)g * P.nb * SW;
    const int lane = threadIdx.x % SW;
    const int e0 = threadIdx.x / SW, ne = blockDim.x / SW;
    for (int h = 0; h < P.n_levels; ++h) {
        for (int t = P.level_ptr[h] + e0; t < P.level_ptr[h + 1]; t += ne) {
            const int j = P.level_nodes[t];
            const double2 b = R[(size_t)j * SW + lane];
            Vec2<T> acc = {(T)b.x, (T)b.y};
#pragma unroll 4
            for (int q = P.rptr[j]; q < P.rptr[j + 1]; ++q) {
                const int2 r = P.rlist[q];  // (L slot of (j,k), k); U(k,j) sits nnz_l further
                msubtv(acc, ldb(F + (size_t)(r.x + P.nnz_l) * SW + lane),
                       ldv(X + (size_t)r.y * SW + lane));
            }
            stv(X + (size_t)j * SW + lane, multv(ldb(F + (size_t)j * SW + lane), acc));
        }
        __syncthreads();
    }
    for (int j = P.ns + e0; j < P.nb; j += ne) {
        const double2 b = R[(size_t)j * SW + lane];
        Vec2<T> acc = {(T)b.x, (T)b.y};
#pragma unroll 4
        for (int q = P.rptr[j]; q < P.rptr[j + 1]; ++q) {
            const int2 r = P.rlist[q];
            msubtv(acc, ldb(F + (size_t)(r.x + P.nnz_l) * SW + lane),
                   ldv(X + (size_t)r.y * SW + lane));
        }
        stv(X + (size_t)j * SW + lane, acc);
    }
}

template <typename T, int SW>
__global__ void __launch_bounds__(256) k_dense_solve_t(PlanDev P, BatchDev B, double2* out,
                                                       int accumulate) {
    const int q = blockIdx.x;
    if (q >= B.n_scen || !B.solving[q]) return;
    const int g = q / SW, lane = q % SW;
    const int N = 2 * P.n_tail, ld = dense_ld(N);
    const T* A = reinterpret_cast<const T*>(B.Dt) + (size_t)q * N * ld;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* y = reinterpret_cast<T*>(smraw);
    const int tid = threadIdx.x, wid = tid >> 5, ln = tid & 31, nw = blockDim.x >> 5;
    for (int i = tid; i < P.n_tail; i += blockDim.x) {
        const Vec2<T> v = ldv(X + (size_t)(P.ns + i) * SW + lane);
        y[2 * i] = v.x;
        y[2 * i + 1] = v.y;
    }
    __syncthreads();
    // U^T w = y (lower triangular with U's diagonal)
    for (int r0 = 0; r0 < N; r0 += 32) {
        for (int rr = wid; rr < 32; rr += nw) {
            const int row = r0 + rr;
            if (row >= N) continue;
            T acc = T(0);
            for (int c = ln; c < r0; c += 32) acc = fma(A[(size_t)c * ld + row], y[c], acc);
#pragma unroll
            for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
            if (ln == 0) y[row] -= acc;
        }
        __syncthreads();
        if (wid == 0) {
            const int row = r0 + ln;
            T v = row < N ? y[row] : T(0);
            for (int j = 0; j < 32; ++j) {
                if (r0 + j >= N) break;
                if (ln == j) v = v / A[(size_t)row * ld + row];
                const T vj = __shfl_sync(0xffffffffu, v, j);
                if (ln > j && row < N) v = fma(-A[(size_t)(r0 + j) * ld + row], vj, v);
            }
            if (row < N) y[row] = v;
        }
        __syncthreads();
    }
    // L^T lam = w (unit upper triangular)
    const int last = ((N - 1) / 32) * 32;
    for (int r0 = last; r0 >= 0; r0 -= 32) {
        const int r1 = min(r0 + 32, N);
        for (int rr = wid; rr < 32; rr += nw) {
            const int row = r0 + rr;
            if (row >= N) continue;
            T acc = T(0);
            for (int c = r1 + ln; c < N; c += 32) acc = fma(A[(size_t)c * ld + row], y[c], acc);
#pragma unroll
            for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
            if (ln == 0) y[row] -= acc;
        }
        __syncthreads();
        if (wid == 0) {
            const int row = r0 + ln;
            T v = row < N ? y[row] : T(0);
            for (int j = 31; j >= 0; --j) {
                if (r0 + j >= N) continue;
                const T vj = __shfl_sync(0xffffffffu, v, j);
                if (ln < j && row < N) v = fma(-A[(size_t)(r0 + j) * ld + row], vj, v);
            }
            if (row < N) y[row] = v;
        }
        __syncthreads();
    }
    double2* O = out + (size_t)g * P.nb * SW;
    for (int i = tid; i < P.n_tail; i += blockDim.x) {
        const int k = P.ns + i;
        stv(X + (size_t)k * SW + lane, Vec2<T>{y[2 * i], y[2 * i + 1]});
        double2* o = O + (size_t)k * SW + lane;
        if (accumulate) {
            const double2 old = *o;
            *o = make_double2(old.x + (double)y[2 * i], old.y + (double)y[2 * i + 1]);
        } else {
            *o = make_double2((double)y[2 * i], (double)y[2 * i + 1]);
        }
    }
}

template <typename T, int SW>
__global__ void k_solve_bwd_t(PlanDev P, BatchDev B, double2* out, int accumulate) {
    const int g = blockIdx.x;
    if (!B.gsolve[g]) return;
    const Blk<T>* F = reinterpret_cast<const Blk<T>*>(B.F) + (size_t)g * P.n_slots * SW;
    Vec2<T>* X = reinterpret_cast<Vec2<T>*>(B.X) + (size_t)g * P.nb * SW;
    double2* O = out + (size_t)g * P.nb * SW;
    const int lane = threadIdx.x % SW;
    const int e0 = threadIdx.x / SW, ne = blockDim.x / SW;
    for (int h = P.n_levels - 1; h >= 0; --h) {
        for (int t = P.level_ptr[h] + e0; t < P.level_ptr[h + 1]; t += ne) {
            const int k = P.level_nodes[t];
            Vec2<T> acc = ldv(X + (size_t)k * SW + lane);
#pragma unroll 4
            for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) {
                msubtv(acc, ldb(F + (size_t)(P.nb + p) * SW + lane),
                       ldv(X + (size_t)P.lidx[p] * SW + lane));
            }
            stv(X + (size_t)k * SW + lane, acc);
            double2* o = O + (size_t)k * SW + lane;
            if (accumulate) {
                const double2 old = *o;
                *o = make_double2(old.x + (double)acc.x, old.y + (double)acc.y);
            } else {
                *o = make_double2((double)acc.x, (double)acc.y);
            }
        }
        __syncthreads();
    }
}

// res = g - J^T lam with the FP64 Jacobian blocks, by block column
template <int SW>
__global__ void __launch_bounds__(256) k_residual_t(PlanDev P, BatchDev B) {
    const int g = blockIdx.y;
    if (!B.gsolve[g]) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = tid / SW, lane = tid % SW;
    if (c >= P.nb) return;
    const size_t base = (size_t)g * P.nb * SW;
    const double2 b = B.rhs[base + (size_t)c * SW + lane];
    Vec2<double> acc = {b.x, b.y};
    const Blk<double>* A = reinterpret_cast<const Blk<double>*>(B.A64) + (size_t)g * P.n_a * SW;
#pragma unroll 4
    for (int e = P.acol_ptr[c]; e < P.acol_ptr[c + 1]; ++e) {
        const int2 ar = P.acol[e];
        const double2 x = B.dx[base + (size_t)ar.y * SW + lane];
        msubtv(acc, ldb(A + (size_t)ar.x * SW + lane), Vec2<double>{x.x, x.y});
    }
    B.res[base + (size_t)c * SW + lane] = make_double2(acc.x, acc.y);
}

// dL/dP_spec = lambda_P, dL/dQ_spec = lambda_Q (PQ buses), per bus, scenario-major
template <int SW>
__global__ void k_adj_out(PlanDev P, BatchDev B, double* dp, double* dq) {
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)B.n_scen * P.n_bus) return;
    const int s = (int)(tid / P.n_bus), i = (int)(tid % P.n_bus);
    const int g = s / SW, lane = s % SW;
    const int node = P.node_of_bus[i];
    double a = 0.0, b = 0.0;
    if (node >= 0) {
        const double2 l = B.dx[((size_t)g * P.nb + node) * SW + lane];
        a = l.x;
        b = P.bus_type[i] == BUS_PQ ? l.y : 0.0;
    }
    if (dp) dp[tid] = a;
    if (dq) dq[tid] = b;
}

// dL/dr, dL/dx per branch (per unit): -lambda^T dF/dp through the branch's pi stamps with
// y = 1/(r + jx), dy/dr = -y^2, dy/dx = -j y^2; brp = (r, x, g, b, k, theta) per unit
template <int SW>
__global__ void k_adj_branch(PlanDev P, BatchDev B, int m, const int* __restrict__ from,
                             const int* __restrict__ to, const double* __restrict__ brp,
                             double* dr, double* dxo) {
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)B.n_scen * m) return;
    const int s = (int)(tid / m), b = (int)(tid % m);
    const int g = s / SW, lane = s % SW;
    const int f = from[b], t = to[b];
    double gr = 0.0, gx = 0.0;
    const double* q = brp + (size_t)b * 6;
    const double r = q[0], x = q[1], k = q[4], th = q[5];
    const double z2 = r * r + x * x;
    if (f >= 0 && t >= 0 && z2 > 0.0) {
        const double yr = r / z2, yi = -x / z2;
        const double y2r = yr * yr - yi * yi, y2i = 2.0 * yr * yi;  // y^2
        double sn, cs;
        sincos(th, &sn, &cs);
        const double tr = k * cs, ti = k * sn, k2 = k * k;
        const double2 vf = B.V[((size_t)g * P.n_bus + f) * SW + lane];
        const double2 vt = B.V[((size_t)g * P.n_bus + t) * SW + lane];
        const int nf = P.node_of_bus[f], nt = P.node_of_bus[t];
        const double2 lf = nf >= 0 ? B.dx[((size_t)g * P.nb + nf) * SW + lane] : make_double2(0, 0);
        const double2 lt = nt >= 0 ? B.dx[((size_t)g * P.nb + nt) * SW + lane] : make_double2(0, 0);
        const double lqf = P.bus_type[f] == BUS_PQ ? lf.y : 0.0;
        const double lqt = P.bus_type[t] == BUS_PQ ? lt.y : 0.0;
        for (int which = 0; which < 2; ++which) {
            // dy: -y^2 (r) or -j y^2 (x)
            const double dyr = which == 0 ? -y2r : y2i, dyi = which == 0 ? -y2i : -y2r;
            // dYff = dy/k^2, dYtt = dy, dYft = -dy*t/k^2, dYtf = -dy*conj(t)/k^2
            const double ffr = dyr / k2, ffi = dyi / k2;
            const double ftr = -(dyr * tr - dyi * ti) / k2, fti = -(dyr * ti + dyi * tr) / k2;
            const double tfr = -(dyr * tr + dyi * ti) / k2, tfi = -(dyi * tr - dyr * ti) / k2;
            // dI_f = dYff vf + dYft vt ; dI_t = dYtf vf + dYtt vt
            const double ifr = ffr * vf.x - ffi * vf.y + ftr * vt.x - fti * vt.y;
            const double ifi = ffr * vf.y + ffi * vf.x + ftr * vt.y + fti * vt.x;
            const double itr = tfr * vf.x - tfi * vf.y + dyr * vt.x - dyi * vt.y;
            const double iti = tfr * vf.y + tfi * vf.x + dyr * vt.y + dyi * vt.x;
            // dS = V conj(dI)
            const double sfr = vf.x * ifr + vf.y * ifi, sfi = vf.y * ifr - vf.x * ifi;
            const double str = vt.x * itr + vt.y * iti, sti = vt.y * itr - vt.x * iti;
            const double adj = lf.x * sfr + lqf * sfi + lt.x * str + lqt * sti;
            if (which == 0)
                gr = -adj;
            else
                gx = -adj;
        }
    }
    dr[tid] = gr;
    dxo[tid] = gx;
}

}  // namespace gapk
