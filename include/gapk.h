/*
 * gapk.h -- C ABI of the B200 Newton-Raphson power-flow engine (libgapk.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  Device pointers are
 * marked d_*, host pointers h_*.  Complex numbers are two interleaved doubles (re, im).
 * Every call that launches GPU work takes a cudaStream_t (passed as void*; NULL = the legacy
 * default stream) and does not synchronise unless it says so.
 *
 * Which reference interface each group replaces (paths inside the reference project):
 *
 *   gapk_ybus_*      gap::admittance::IAdmittanceMatrix::build_admittance_matrix /
 *                    update_admittance_matrix (include/gap/admittance/admittance_interface.h:21-31),
 *                    GPU implementation src/admittance/gpu/gpu_admittance_matrix.cu:243-410,
 *                    CPU semantics src/admittance/cpu/cpu_admittance_matrix.cpp:44-301.
 *   gapk_nr_*        gap::solver::IPowerFlowSolver::solve_power_flow
 *                    (include/gap/solver/powerflow_interface.h:59-61), GPU implementation
 *                    src/solver/powerflow/gpu/gpu_newton_raphson.cu:392-570 and its kernels
 *                    src/solver/powerflow/gpu/gpu_powerflow_kernels.cu:16-538, CPU semantics
 *                    src/solver/powerflow/cpu/cpu_newton_raphson.cpp:33-727.
 *   gapk_splu_*      gap::solver::ILUSolver::factorize / solve / update_factorization
 *                    (include/gap/solver/lu_solver_interface.h:21-35), GPU implementation
 *                    src/solver/lu/gpu/gpu_cudss_solver.cu:167-479.
 *   gapk_nr_adjoint  no counterpart in the reference (gradients through the converged state).
 *
 * The C++ plugin libraries libgap_{admittance,lu,powerflow}_gpu.so export the reference's
 * factory symbols (create_gpu_* / destroy_gpu_*) and call these functions.
 */
#ifndef GAPK_H
#define GAPK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
#define GAPK_OK 0
#define GAPK_EINVAL (-1)   /* bad argument (message in gapk_last_error)                   */
#define GAPK_ECUDA (-2)    /* CUDA runtime error                                          */
#define GAPK_ENOMEM (-3)   /* device allocation failed                                    */
#define GAPK_ESTATE (-4)   /* call out of order (e.g. solve before factorize)             */
#define GAPK_ESINGULAR (-5) /* zero / non-finite pivot                                    */
#define GAPK_ERANGE (-6)   /* size beyond a documented maximum                            */

/* per-scenario solve status */
#define GAPK_SCEN_CONVERGED 0
#define GAPK_SCEN_MAXITER 1
#define GAPK_SCEN_SINGULAR 2
#define GAPK_SCEN_NONFINITE 3

/* bus types, as gap::BusType (include/gap/core/types.h:30-34) */
#define GAPK_BUS_PQ 0
#define GAPK_BUS_PV 1
#define GAPK_BUS_SLACK 2

/* Message for the last failing call on this thread (never NULL). */
const char* gapk_last_error(void);
/* ABI version: major*10000 + minor*100 + patch. */
int gapk_version(void);
/* Number of CUDA devices visible (0 when none); never fails. */
int gapk_device_count(void);

/* ==== Y-bus ============================================================================
 * The CSR pattern is built on the host once per topology, bit-identical to the reference's
 * stable-sorted triplet order (duplicates from parallel branches kept, diagonal of every bus
 * present).  Values are assembled on the device as a deterministic segmented reduction: each
 * diagonal sums its shunt and branch-end stamps in the reference's order, without atomics.
 */
typedef struct gapk_ybus_s* gapk_ybus;

/* from_idx / to_idx are bus positions (0..n_bus-1); in_service != 0 marks branches that enter
 * the matrix (the caller resolves IDs and drops invalid branches, as the reference does).
 * shunt_bus lists the bus position of every shunt in appliance order. */
int gapk_ybus_create(int n_bus, int n_branch, const int* h_from_idx, const int* h_to_idx,
                     const int* h_in_service, int n_shunt, const int* h_shunt_bus,
                     gapk_ybus* out);
int gapk_ybus_destroy(gapk_ybus y);
int gapk_ybus_nnz(gapk_ybus y);
/* Copies the pattern out: h_row_ptr[n_bus+1], h_col_idx[nnz]. */
int gapk_ybus_pattern(gapk_ybus y, int* h_row_ptr, int* h_col_idx);

#define GAPK_YBUS_REFERENCE 0 /* ignore tap k and shift theta, as the reference builder   */
#define GAPK_YBUS_TAPS 1      /* pi model with tap k*exp(j theta) on the from side        */

/* Assemble values for n_scen scenarios.
 *   d_branch : doubles [n_scen][n_branch][6] = (r1, x1, g1, b1, k, theta) per branch,
 *              scenario stride branch_stride doubles (0 = shared by all scenarios)
 *   d_shunt  : doubles [n_scen][n_shunt][2] = (g1, b1), stride shunt_stride (0 = shared)
 *   d_values : complex [n_scen][nnz], stride values_stride complex entries
 *   scale    : every value is multiplied by scale (1.0 = Siemens; Z_base = per unit)
 */
int gapk_ybus_assemble(gapk_ybus y, int n_scen, const double* d_branch, int64_t branch_stride,
                       const double* d_shunt, int64_t shunt_stride, int mode, double scale,
                       double* d_values, int64_t values_stride, void* stream);

/* Branch status changes on existing Y values (IAdmittanceMatrix::update_admittance_matrix,
 * include/gap/admittance/admittance_interface.h:24-31; reference semantics
 * src/admittance/cpu/cpu_admittance_matrix.cpp:204-301).  A change sets one branch's status:
 * its stamps are added (status 1) or removed (status 0).  Changes are applied per CSR slot in
 * change order, one device thread per touched slot, so the result equals the sequential
 * application's.
 *   h_pos[i*4..]    : CSR indices of (diag from, diag to, (from,to), (to,from)) or -1, as
 *                     located in the pattern by the caller (host memory)
 *   d_params[i*7..] : (r1, x1, g1, b1, k, theta, status) in Ohm / S (device)
 *   mode            : GAPK_DELTA_REFERENCE  the reference's update, bit for bit: diagonals
 *                                           change by y + g1 + j b1 + j b1/2 (its build stamps
 *                                           y + g1 + j b1/2), taps ignored
 *                     GAPK_DELTA_FIXED      the builder's own stamps (y + g1 + j b1/2), taps
 *                                           ignored: update(build(net)) = build(changed net)
 *                     GAPK_DELTA_FIXED_TAPS the builder's pi-model stamps with the tap
 *                                           (GAPK_YBUS_TAPS)
 * gapk_ybus_apply_changes applies one change list to one value vector; the delta plan below
 * applies per-scenario change lists to a batch. */
#define GAPK_DELTA_REFERENCE 0
#define GAPK_DELTA_FIXED 1
#define GAPK_DELTA_FIXED_TAPS 2
int gapk_ybus_apply_changes(int n_changes, const int* h_pos, const double* d_params, int mode,
                            double* d_values, void* stream);

/* Batched branch changes (no reference counterpart; contingency screening): scenario s applies
 * changes h_change_ptr[s] .. h_change_ptr[s+1]-1 (positions h_pos as above) to its own value
 * vector d_values + s * values_stride (complex entries), every delta multiplied by scale
 * (1 = Siemens, Z_base = per unit).  The plan (the touched slots of every scenario, each with
 * its changes in order) is built once on the host and reused for any parameters. */
typedef struct gapk_ybus_delta_s* gapk_ybus_delta;
int gapk_ybus_delta_create(int n_scen, const int* h_change_ptr, const int* h_pos,
                           gapk_ybus_delta* out);
int gapk_ybus_delta_destroy(gapk_ybus_delta d);
int gapk_ybus_delta_apply(gapk_ybus_delta d, const double* d_params, int mode, double scale,
                          double* d_values, int64_t values_stride, void* stream);

/* Branch results of solved scenarios: fills, per scenario and branch, the BranchData result
 * fields p_from, q_from, i_from, s_from, p_to, q_to, i_to, s_to, loading
 * (include/gap/core/types.h:233-243), which the reference declares but never computes; the
 * definitions are power-grid-model's line outputs (W, var, A, VA; |I| = |S| / (sqrt(3)|U|);
 * loading = max(i_from, i_to) / i_n, or max(s_from, s_to) / sn where i_n is absent or 0).
 *   d_from, d_to : bus index per branch, -1 for an out-of-service branch (its row is zero)
 *   d_branch     : (r1, x1, g1, b1, k, theta) per branch in Ohm / S, as gapk_ybus_assemble;
 *                  branch_stride doubles between scenarios (0 = shared)
 *   d_v          : complex per-unit voltages [n_scen][n_bus]; u_base the voltage base (V)
 *   d_i_n, d_sn  : rated current (A) / power (VA) per branch, or NULL
 *   mode         : GAPK_YBUS_REFERENCE (taps ignored, as the reference's Y-bus) or _TAPS
 *   d_out        : [n_scen][n_branch][9] doubles */
int gapk_branch_flows(int n_scen, int n_bus, int n_branch, const int* d_from, const int* d_to,
                      const double* d_branch, int64_t branch_stride, const double* d_v,
                      double base_power, double u_base, const double* d_i_n, const double* d_sn,
                      int mode, double* d_out, void* stream);

/* ==== Newton-Raphson engine ===========================================================
 * A plan holds everything that depends only on the Y pattern and the bus types: the
 * 2x2-block Jacobian pattern, a minimum-degree ordering, the symbolic block-LU
 * factorisation, its level schedule and the Y->Jacobian scatter map.  Plans are built on the
 * host and uploaded to the current device on first use.  A batch holds the device state of
 * n_scen scenarios that share one plan.
 */
typedef struct gapk_nr_plan_s* gapk_nr_plan;
typedef struct gapk_nr_batch_s* gapk_nr_batch;

#define GAPK_JAC_REFERENCE 0 /* duplicate Y entries: last one wins (reference dense G/B)  */
#define GAPK_JAC_EXACT 1     /* duplicate Y entries summed (true derivative)              */

#define GAPK_ORDER_MINDEG 0  /* minimum degree on the bus graph                            */
#define GAPK_ORDER_NATURAL 1 /* bus order                                                  */

typedef struct {
    int jacobian_mode; /* GAPK_JAC_*                                                       */
    int ordering;      /* GAPK_ORDER_*                                                     */
    int dense_min;     /* trailing fully-dense block of at least this many nodes is
                          factorised densely (0 = default 16, < 0 = never)                 */
} gapk_nr_plan_options;

typedef struct {
    int n_bus, n_block;   /* buses; block unknowns (non-slack buses)                       */
    int n_pq, n_pv, n_slack;
    int n_vars;           /* reference Newton unknowns: (n_bus - n_slack) + n_pq            */
    int nnz_y;
    int nnz_l_blocks;     /* strictly-lower blocks of L (= of U^T)                          */
    int n_slots;          /* n_block + 2 * nnz_l_blocks                                     */
    int n_a_blocks;       /* blocks of the Jacobian pattern itself                          */
    int n_levels;         /* elimination-tree height + 1                                    */
    int64_t n_pairs;      /* block multiply-adds of one numeric factorisation               */
    int64_t n_rows_pairs; /* block multiply-adds of one forward solve                       */
    int max_level_width;
    int n_tail;           /* nodes in the dense trailing block (0 = none)                   */
    int64_t n_schur_pairs; /* block multiply-adds of the sparse part into the dense block   */
} gapk_nr_plan_info;

int gapk_nr_plan_create(int n_bus, int nnz_y, const int* h_y_row_ptr, const int* h_y_col_idx,
                        const int* h_bus_type, const gapk_nr_plan_options* opt,
                        gapk_nr_plan* out);
int gapk_nr_plan_destroy(gapk_nr_plan p);
int gapk_nr_plan_get_info(gapk_nr_plan p, gapk_nr_plan_info* info);

/* Export host-side schedule arrays (for inspection and CPU-side checking).  `what` selects:
 *   0 bus_of_node[n_block]   1 node_pq[n_block]      2 lptr[n_block+1]   3 lidx[nnz_l]
 *   4 level_ptr[n_levels+1]  5 level_nodes[n_block]  6 slot_info[n_slots*4]
 *   7 slot_src_ptr[n_slots+1] 8 slot_src[...]        9 fa_ptr[n_levels+1]
 *  10 targets[n_targets*4]  11 pairs[n_pairs*2]     12 fb_ptr[n_levels+1] 13 scale[n_b*2]
 *  14 rptr[n_block+1]       15 rlist[...*2]     16 var_of_comp[2*n_block]
 *  17 eq_of_comp[2*n_block]  18 slot_a[n_slots]   19 arow_ptr[n_block+1] 20 arow[...*2]
 *  21 schur[n_tail^2*4] (slot, pair_begin, pair_end, block position)
 * Returns the number of ints written (or needed when h_buf is NULL). */
int64_t gapk_nr_plan_export(gapk_nr_plan p, int what, int* h_buf);

#define GAPK_PREC_FP64 0  /* factor and triangular solves in FP64                          */
#define GAPK_PREC_FP32 1  /* factor and triangular solves in FP32 (mismatch, update and
                             convergence stay FP64)                                        */

typedef struct {
    int precision;      /* GAPK_PREC_*                                                     */
    int y_shared;       /* 1: one Y for all scenarios; 0: one Y per scenario               */
    int lanes;          /* scenarios interleaved per thread group: 1, 2, 4 or 8 (0 = auto) */
    int threads;        /* threads per CTA of the factor / solve kernels (0 = auto)        */
    int use_graph;      /* 1: NR loop as a CUDA graph with a device-side while node        */
    int dense_fused;    /* 1: one-CTA-per-scenario dense-tail LU even for a batch too small
                           to fill the GPU alone (batches that run concurrently on several
                           streams); 0: chosen by the batch size                           */
    int dense_fma;      /* FP32 tails have the trailing updates of their dense LU on the tensor
                           cores (tcgen05, three TF32 products accumulated in FP32:
                           k_dense_lu_tc one CTA per scenario, k_dlu_update_tc on the split
                           path) unless this is 1: then on CUDA-core FMA.  FP64 tails always
                           use CUDA cores.                                                   */
} gapk_nr_batch_options;

int gapk_nr_batch_create(gapk_nr_plan p, int n_scen, const gapk_nr_batch_options* opt,
                         gapk_nr_batch* out);
int gapk_nr_batch_destroy(gapk_nr_batch b);
/* Device bytes held by the batch. */
int64_t gapk_nr_batch_device_bytes(gapk_nr_batch b);
/* Scenarios per lane group (the interleave width the batch was created with, or chose). */
int gapk_nr_batch_lanes(gapk_nr_batch b);

#define GAPK_POLICY_REFERENCE 0 /* damping 0.9, |dtheta|<=0.15, |d|V||<=0.08, |V| in [0.5,1.5]
                                   (cpu_newton_raphson.cpp:438-504)                         */
#define GAPK_POLICY_NEWTON 1    /* full Newton step                                         */
#define GAPK_POLICY_CLAMPED 2   /* full Newton step with the reference policy's clamps and |V| clip  */

typedef struct {
    const double* d_y;      /* complex Y (per unit): [nnz] if y_shared else [n_scen][nnz] */
    const double* d_s_spec; /* complex specified injections (per unit) [n_scen][n_bus]    */
    const double* d_v_init; /* complex start voltages [n_scen][n_bus], or NULL = flat start */
    const double* d_u_pu;   /* flat-start |V| of SLACK/PV buses [n_bus] (NULL = 1.0)        */
    double tolerance;       /* on max |mismatch| in per unit                                */
    int max_iterations;
    int policy;             /* GAPK_POLICY_*                                                */
    int refine;             /* extra iterative-refinement steps on each Newton correction  */
    double refine_below;    /* refine only in iterations where some iterating scenario of a
                               lane group has max |mismatch| below this (0 = every iteration);
                               far from the solution the FP32 step error does not slow Newton */
    double reuse_below;     /* once every iterating scenario of a lane group has max |mismatch|
                               below this, the group keeps its previous LU factors instead of
                               refactorising, and the (refined, refine >= 1) solve uses them
                               against the current FP64 Jacobian (0 = refactorise every time) */
    int v_init_shared;      /* != 0: d_v_init is one start vector [n_bus] for every scenario */
} gapk_nr_inputs;

typedef struct {
    double* d_v;              /* complex [n_scen][n_bus] (may be NULL)                    */
    int* d_iterations;        /* [n_scen] (may be NULL)                                   */
    int* d_status;            /* [n_scen] GAPK_SCEN_* (may be NULL)                       */
    double* d_final_mismatch; /* [n_scen] (may be NULL)                                   */
} gapk_nr_outputs;

/* Runs the whole Newton-Raphson loop on the device.  Asynchronous on `stream`. */
int gapk_nr_solve(gapk_nr_batch b, const gapk_nr_inputs* in, const gapk_nr_outputs* out,
                  void* stream);

/* ==== Heterogeneous batches in one launch (no reference counterpart) ======================
 * Batches of different plans (load scenarios of one grid, its N-1 contingencies sharing that
 * grid's plan, independent grids of any size) solved by ONE cudaGraphLaunch: each batch's whole
 * solve -- its options, its inputs loaded, its Newton loop as a device-side while node, results
 * written -- is one branch of a single graph, and the branches run concurrently.  Per-scenario
 * status words as gapk_nr_solve's.  With retry_policy >= 0 (a GAPK_POLICY_*), the scenarios
 * that end at max_iterations or with a non-finite mismatch restart from their start vector
 * under that policy, inside the same launch (a second while node per branch whose condition
 * the device sets); their iteration count is then the retry's.  The graph is built on the first
 * call and rebuilt only when an input/output pointer or option changes; a batch belongs to at
 * most one mix at a time and is not solved on its own while the mix runs. */
typedef struct gapk_nr_mix_s* gapk_nr_mix;
int gapk_nr_mix_create(int n_batches, const gapk_nr_batch* batches, gapk_nr_mix* out);
int gapk_nr_mix_destroy(gapk_nr_mix m);
/* in[i] / out[i] for batch i (as for gapk_nr_solve); asynchronous on `stream`. */
int gapk_nr_mix_solve(gapk_nr_mix m, const gapk_nr_inputs* in, const gapk_nr_outputs* out,
                      int retry_policy, void* stream);

/* ==== Stepping, for iteration-state capture ===============================================
 * IPowerFlowSolver::enable_state_capture / get_iteration_states
 * (include/gap/solver/powerflow_interface.h:28-35,83-107; recorded per iteration by
 * src/solver/powerflow/gpu/gpu_newton_raphson.cu:452-490).  After gapk_nr_stage_load, each
 * gapk_nr_step runs one iteration of the loop gapk_nr_solve runs (mismatch, convergence test,
 * Jacobian, factorisation, solve, update) on every scenario still iterating, synchronises the
 * stream and sets *h_active to 1 while some scenario is still iterating.  At most
 * max_iterations steps do work; gapk_nr_get_outputs then writes what gapk_nr_solve writes.
 * The trajectory is the one gapk_nr_solve takes. */
int gapk_nr_step(gapk_nr_batch b, int* h_active, void* stream);
/* The batch's current state in bus order, per unit, complex [n_scen][n_bus] each (any may be
 * NULL): the voltages V, the current injections I = Y V and the power injections
 * S = V conj(I).  Called before a step, it is the state that step's mismatch is taken at. */
int gapk_nr_get_state(gapk_nr_batch b, double* d_v, double* d_i, double* d_s, void* stream);
int gapk_nr_get_outputs(gapk_nr_batch b, const gapk_nr_outputs* out, void* stream);

/* ==== Level trace (per-level latency of the level-scheduled kernels) ======================
 * No counterpart in the reference (its only timers are host std::chrono phase totals,
 * src/solver/powerflow/cpu/cpu_newton_raphson.cpp:23-30,181-206).  With d_stamps set (device
 * memory of gapk_nr_level_trace_size(b) uint64 values), the sparse factorisation and the
 * sparse forward and backward solves write %globaltimer stamps (ns) into
 * [kernel: 0 factor, 1 forward, 2 backward][lane group][j], j = 0 at the kernel's start,
 * 1 + i when the i-th level in execution order is done, n_levels + 1 at the end; one CTA per
 * lane group writes its own row.  When the batch factorises its dense tail with the
 * one-CTA-per-scenario kernel, a panel trace follows: [scenario (padded to whole lane
 * groups)][1 + 3 * panels], the kernel's start, then per panel of gapk_nr_dense_trace_panels
 * the ends of the diagonal-block factorisation, of the L21 / U12 solves and of the trailing
 * update.  NULL switches the trace off.  Changing the setting makes the next gapk_nr_solve
 * rebuild its graph. */
int64_t gapk_nr_level_trace_size(gapk_nr_batch b);
int gapk_nr_dense_trace_panels(gapk_nr_batch b);
int gapk_nr_set_level_trace(gapk_nr_batch b, unsigned long long* d_stamps, int64_t n_stamps);

/* ==== Bounded waits of the tensor-core dense LU ==========================================
 * k_dense_lu_tc and k_dlu_update_tc wait for their MMAs on an mbarrier with a bounded number
 * of polls.  When a wait runs out the CTA marks its scenario SINGULAR, sets the batch's device
 * error word, frees its tensor memory and returns; the next solve starts with the word clear.
 * gapk_nr_batch_device_error returns the word (1: a wait ran out during the last solve), after
 * waiting for the device.  gapk_nr_batch_set_wait_test is a test hook: with skip = 1 the two
 * kernels issue no MMAs, so that every wait runs out (a factorising scenario then ends
 * SINGULAR); 0 restores normal operation.  Set it between solves (it is read on the device,
 * so graphs already built follow it). */
int gapk_nr_batch_device_error(gapk_nr_batch b);
int gapk_nr_batch_set_wait_test(gapk_nr_batch b, int skip);

/* ==== Adjoint (gradients through the converged state; no counterpart in the reference) ====
 * With the batch holding a converged state (after gapk_nr_solve, or gapk_nr_stage_load with
 * the solution as d_v_init), refactorises the Jacobian at that state and solves
 * J^T lambda = dL/dx, x = (theta of non-slack buses, |V| of PQ buses), with the same block
 * factors transposed (plus one FP64 refinement step for FP32 batches).  Inputs are dL/d|V|
 * and dL/dtheta per bus ([n_scen][n_bus]); entries of fixed quantities (slack angle and
 * magnitude, PV magnitudes) are ignored.  Outputs dL/dP_spec and dL/dQ_spec per bus
 * ([n_scen][n_bus], per unit; zero where the injection does not enter the equations).  Use a
 * plan created with GAPK_JAC_EXACT so that the factors are those of the true Jacobian. */
int gapk_nr_adjoint(gapk_nr_batch b, const double* d_dl_dvm, const double* d_dl_dva,
                    double* d_dl_dp, double* d_dl_dq, void* stream);
/* After gapk_nr_adjoint: dL/dr and dL/dx per branch and scenario ([n_scen][n_branch], per
 * unit), the implicit part -lambda^T dF/d(r, x) through the pi-model stamps.  d_from/d_to are
 * bus positions (-1 for branches not in the matrix); d_branch_pu = (r, x, g, b, k, theta) per
 * branch in per unit, as used to build Y. */
int gapk_nr_adjoint_branch(gapk_nr_batch b, int n_branch, const int* d_from, const int* d_to,
                           const double* d_branch_pu, double* d_dl_dr, double* d_dl_dx,
                           void* stream);

/* ==== General sparse LU (ILUSolver) =====================================================
 * Complex square CSR matrices (values interleaved re, im).  Analysis once per pattern on the
 * host: a row permutation giving a zero-free diagonal (maximum transversal), minimum-degree
 * ordering of the symmetrised pattern, symbolic factorisation; numeric factorisation and
 * solves on the device with static pivoting (a pivot below 1e-14 reports GAPK_ESINGULAR,
 * as CPULUSolver's pivot tolerance, src/solver/lu/cpu/cpu_lu_solver.cpp:65).  Duplicate
 * entries are summed.  Replaces ILUSolver::factorize / solve / update_factorization
 * (include/gap/solver/lu_solver_interface.h:21-35). */
typedef struct gapk_splu_s* gapk_splu;
int gapk_splu_create(int n, int nnz, const int* h_row_ptr, const int* h_col_idx, gapk_splu* out);
int gapk_splu_destroy(gapk_splu s);
int gapk_splu_size(gapk_splu s);
/* Factorises d_values (complex [nnz], device); synchronises the stream to report the result. */
int gapk_splu_factorize(gapk_splu s, const double* d_values, void* stream);
/* x = A^-1 b for complex device vectors of length n. */
int gapk_splu_solve(gapk_splu s, const double* d_rhs, double* d_x, void* stream);

/* Allocation-free variant of gapk_nr_solve for ONE scenario in FP64 (no counterpart in the
 * reference).  For callers that may not allocate device memory while they solve: hosts that
 * own all device memory through their own pools and hand none to plugins, and real-time
 * loops that must not call into the allocator (cudaMalloc / cudaFree can block on the whole
 * device).  It calls no cudaMalloc, cudaFree or allocating library routine: the plan's index
 * lists are copied into, and the whole Newton state lives in, one static 32 MiB device array
 * that every GPU loading the library holds until the process exits.  Grids whose plan and
 * state need more than 32 MiB (beyond about 15k buses of the transmission-like generator;
 * 10k-bus grids fit) are rejected with GAPK_ERANGE.  `in` as for gapk_nr_solve with
 * refine = 0 (d_y shared, d_s_spec / d_v_init / outputs for one scenario).  The loop is driven
 * from the host: the call copies the plan's index lists from host memory, waits for `stream`
 * once per Newton iteration and once more after writing the outputs, so the outputs are ready
 * when it returns; pass a stream created with cudaStreamNonBlocking so that these waits do
 * not also wait for work on the legacy default stream.  The first call on a device looks up
 * the array's device address and sets a kernel attribute; make that first call before any
 * stream capture.  All calls share the one array, so calls that overlap on the GPU (from
 * several host threads at once) race and corrupt each other; the array keeps the last call's
 * contents, and every call reinitialises what it reads. */
int gapk_nr_solve_noalloc(gapk_nr_plan p, const gapk_nr_inputs* in, const gapk_nr_outputs* out,
                          void* stream);

/* Device counters of the last solve, copied to the host (synchronises the stream):
 * h_counters[0] = Newton iterations run by the device loop (max over scenarios). */
int gapk_nr_last_loop_count(gapk_nr_batch b, void* stream, int* h_loops);

/* ---- building blocks, one launch each (used for timing and for tests) ----------------- */
/* Copy inputs into the batch and flat-start; afterwards the kernels below may be run. */
int gapk_nr_stage_load(gapk_nr_batch b, const gapk_nr_inputs* in, void* stream);
int gapk_nr_stage_mismatch(gapk_nr_batch b, void* stream);
int gapk_nr_stage_jacobian(gapk_nr_batch b, void* stream);
int gapk_nr_stage_factor(gapk_nr_batch b, void* stream);
int gapk_nr_stage_solve(gapk_nr_batch b, void* stream);
/* One kernel of the loop body, for per-kernel timing and profiling:
 *   0 mismatch  1 jacobian fill  2 sparse factor  3 Schur gather  4 dense LU
 *   5 sparse forward solve  6 dense solve  7 sparse backward solve  8 update
 *   9 refinement residual (FP32 batches)
 * Kernels 3, 4 and 6 do nothing when the plan has no dense tail. */
int gapk_nr_stage_kernel(gapk_nr_batch b, int kernel, void* stream);
/* Newton correction of the last stage_solve, [n_scen][n_vars] doubles in the reference's
 * variable order (theta of non-slack buses, then |V| of PQ buses). */
int gapk_nr_stage_get_correction(gapk_nr_batch b, double* d_dx, void* stream);
/* Mismatch of the last stage_mismatch, [n_scen][n_vars] in the reference's equation order. */
int gapk_nr_stage_get_mismatch(gapk_nr_batch b, double* d_f, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GAPK_H */
