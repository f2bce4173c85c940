"""Benchmark: power-flow solves/s on B200 -- batched mixed-precision Newton-Raphson.

Workload (one "step"): 1024 load scenarios (per-bus lognormal sigma 0.1) of the seeded
10k-bus transmission-like grid (mean degree 2.8, 10 % tap / phase-shift transformers, 20 % PV,
2 % shunts), solved together to max |mismatch| < 1e-8 pu: FP32 Jacobian factor and triangular
solves (two FP64 iterative-refinement steps and factor reuse below 1e-2 pu), FP64 mismatch /
update / convergence, the whole Newton loop on the device (CUDA graph with a device-side while
node).  Weak scaling: under torchrun the global batch holds world x 1024 scenarios and each
rank solves its contiguous shard of 1024 (gap_b200.sharding), with no collective inside the
Newton loop; statuses are gathered once after the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload mixed     # the mixed batch below, one JSON line
    python bench.py --workload large     # the 100k-bus grid below, one JSON line
    python bench.py --workload adjoint   # loss gradients on 256 scenarios, one JSON line
    python bench.py --workload feeder    # the 200-bus feeder, with the reference's CPU time

Prints one JSON line (rank 0).  `value` times the solve with inputs resident in HBM; `e2e`
times the same call with host (pinned) inputs and results copied inside the timed region.
The plain FP64 single-scenario solve of the same grid is reported beside it.

Supplementary workloads (one GPU, not the headline):
  mixed  1024 load scenarios of a 2k-bus grid of the same generator, 256 N-1 branch outages
         of that grid (distinct non-bridge branches, one plan shared with the load scenarios),
         and 64 independent grids with n log-uniform in [500, 20000], all solved by one CUDA
         graph launch (one branch per study, lanes/threads autotuned per study; unconverged
         scenarios retried with the clamped step policy in the same launch).
  large  32 load scenarios of a 100k-bus grid of the same generator (accuracy against the
         FP64 oracle: tests/test_gpu_large.py).
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Power-flow solves/s on 1 B200: batched mixed-precision vs plain FP64 at 1e-8 pu"
from gap_b200.workloads import (BASE, GRID_SEED, MAX_ITER, N_BUS, REFINE_BELOW,  # noqa: E402
                                REFINE_STEPS, REUSE_BELOW, SIGMA, TOL)
from gap_b200 import workloads  # noqa: E402

N_SCEN = workloads.N_SCEN
# per-bus load scale of the large (100k-bus) workload
LARGE_LOAD_SCALE = 0.025


def workload(rank: int, world: int = 1):
    """This rank's shard of the global batch: world x N_SCEN scenarios, block b drawn with seed
    1 + b, split contiguously by sharding.shard (rank r solves block r)."""
    from gap_b200.sharding import shard

    idx = shard(world * N_SCEN, world, rank)
    assert idx[0] == rank * N_SCEN and len(idx) == N_SCEN
    net, s_spec, v0 = workloads.headline(rank, N_SCEN)
    return net, s_spec, v0, idx


def config(extra=None):
    c = {"workload": f"{N_SCEN} load scenarios x {N_BUS}-bus transmission grid (seed {GRID_SEED})",
         "n_bus": N_BUS, "scenarios_per_gpu": N_SCEN, "load_sigma": SIGMA, "tol_pu": TOL,
         "max_iter": MAX_ITER,
         "precision": "fp32 factor+solve, fp64 mismatch/update; below 1e-2 pu: 2 refinement "
                      "steps, factors reused",
         "policy": "newton", "start": "dc angles", "l2": "inputs larger than L2 (state > 300 MB)",
         "generator_deviations": dict(workloads.DEVIATIONS)}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------------------------------
# CPU baseline: the oracle's FP64 restatement (sparse LU), one scenario per process
# ------------------------------------------------------------------------------------------

def _cpu_solve(idx):
    import numpy as np

    from oracle import restate

    net, s_spec, v0 = _CPU_STATE
    o = restate.nr_solve(net, Y=_CPU_Y, tol=TOL, max_iter=MAX_ITER, base_power=BASE,
                         policy="newton", jac="exact", s_spec=s_spec[idx], v0=v0)
    return bool(o["converged"])


def _cpu_init():
    global _CPU_STATE, _CPU_Y
    from oracle import restate

    _CPU_STATE = workload(0)[:3]
    _CPU_Y = restate.ybus_pi(_CPU_STATE[0])


def _warm(i):
    time.sleep(0.5)
    return i


def make_ready(pool, cores):
    """Runs one sleeping task per worker so every worker has finished its initializer
    (workload build) before anything is timed."""
    pool.map(_warm, range(cores), chunksize=1)


def cpu_run(pool, sample_idx):
    t0 = time.perf_counter()
    ok = sum(pool.map(_cpu_solve, sample_idx))
    return ok, time.perf_counter() - t0


def make_pool():
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    return ctx.Pool(cores, initializer=_cpu_init), cores


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        import statistics

        self.f.flush()
        rows = []
        try:
            with open(self.f.name) as fh:
                for line in fh:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------
# algorithmic bytes per kernel launch: every operand read once and every result written once
# ------------------------------------------------------------------------------------------

# DRAM bytes per scenario per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one
# ncu --set full capture of the kernels on 320 scenarios of the same grid, scaled by scenarios
# (each scenario's work and bytes are independent of the others).
MEASURED_TRAFFIC_PER_SCENARIO = {"dense_lu": (1665.719e6 + 1626.506e6) / 320,  # k_dense_lu_tc
                                 "dense_lu_fma": (1451.877e6 + 1568.291e6) / 320,  # k_dense_lu
                                 "schur": (103.909e6 + 277.920e6) / 320,
                                 "factor_sparse": (248.066e6 + 205.772e6) / 320}


def algorithmic_bytes(kernel, info, n_scen, esz):
    n, nb, nnz = info["n_bus"], info["n_block"], info["nnz_y"]
    ns_slots = info["n_slots"]
    T = info["n_tail"]
    N = 2 * T
    nnzl = info["nnz_l_blocks"]
    blk = 4 * esz
    S = n_scen
    if kernel == "mismatch":
        return nnz * 20 + 4 * (n + 1) + S * (n * 16 * 3 + nb * 16)
    if kernel == "jacobian":
        return nnz * 16 + ns_slots * 16 + S * (n * 32 + ns_slots * blk + info["n_a_blocks"] * 32)
    if kernel == "schur":
        # read the tail slots and the sparse-part blocks that feed them once, write the dense tail
        return S * (T * T * blk + nnzl * blk + N * N * esz)
    if kernel == "dense_lu":
        return S * 2 * N * N * esz
    if kernel == "dense_solve":
        return S * N * N * esz
    if kernel == "factor_sparse":
        return S * 2 * (ns_slots - T * T) * blk
    if kernel in ("solve_fwd", "solve_bwd"):
        return S * (nnzl * blk + nb * 16 * 2)
    if kernel == "residual":
        # FP64 Jacobian blocks, the correction and the right-hand side read, the residual written
        return S * (info["n_a_blocks"] * 32 + nb * 16 * 3)
    if kernel == "update":
        return S * (n * 32 + nb * 16)
    return 0


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------

def run_ours(args, rank, world, device):
    import numpy as np
    import torch

    from gap_b200 import _native as N
    from gap_b200.engine import (HostPipeline, NRBatch, NRPlan, YbusPlan, branch_params,
                                 shunt_params)

    dist = world > 1
    if dist:
        import torch.distributed as tdist

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.SUM)
        return float(t.item())

    pool = cores = None
    if rank == 0 and world == 1 and not args.no_cpu:
        pool, cores = make_pool()  # spawn context: safe beside the CUDA context
        make_ready(pool, cores)

    net, s_np, v_np, shard_idx = workload(rank, world)
    zb = float(net.u_rated[0]) ** 2 / BASE
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=N.YBUS_TAPS,
                    scale=zb)[0]
    t0 = time.perf_counter()
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    plan_s = time.perf_counter() - t0
    info = plan.info
    batch = NRBatch(plan, N_SCEN, use_graph=not args.host_loop, dense_fma=args.dense_fma,
                    **workloads.batch_kwargs())
    s_dev = torch.as_tensor(s_np, device="cuda")
    v_dev = torch.as_tensor(v_np, device="cuda")

    def step():
        return batch.solve(y, s_dev, v_init=v_dev, **workloads.solve_kwargs())

    for _ in range(args.warmup):
        r = step()
    torch.cuda.synchronize()
    loops = batch.loop_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(device) as clk:
        barrier()
        e0.record()
        for _ in range(args.steps):
            r = step()
        e1.record()
        torch.cuda.synchronize()
        barrier()
    ms = allmax(e0.elapsed_time(e1))
    status = r.status.cpu().numpy()
    iters = r.iterations.cpu().numpy()
    conv = int((status == 0).sum())
    if dist:
        from gap_b200.sharding import gather

        full = gather(shard_idx, {"status": status, "iterations": iters}, world * N_SCEN)
        conv_all = int((full["status"] == 0).sum())
    else:
        conv_all = conv
    value = conv_all * args.steps / (ms / 1e3)

    # e2e: host (pinned) inputs -> device -> solve -> host results, every step
    s_h = torch.as_tensor(s_np).pin_memory()
    v_h = torch.as_tensor(v_np).pin_memory()
    vo_h = torch.empty((N_SCEN, net.n_bus), dtype=torch.complex128).pin_memory()
    st_h = torch.empty(N_SCEN, dtype=torch.int32).pin_memory()
    it_h = torch.empty(N_SCEN, dtype=torch.int32).pin_memory()
    fm_h = torch.empty(N_SCEN, dtype=torch.float64).pin_memory()

    # four parts on four streams: one part's copies overlap the other parts' solves (each part
    # keeps the one-CTA-per-scenario dense LU, dense_fused)
    pipe = HostPipeline(plan, N_SCEN, chunks=4, **workloads.batch_kwargs())

    def e2e_step():
        pipe.solve(y, s_h, v_h, vo_h, st_h, it_h, fm_h, **workloads.solve_kwargs())

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = allmax(e0.elapsed_time(e1))
    conv_e2e = allsum(int((st_h.numpy() == 0).sum()))
    # S_spec of every scenario, and the shared start vector once per pipeline part
    h2d = N_SCEN * net.n_bus * 16 + len(pipe.ranges) * net.n_bus * 16
    d2h = N_SCEN * net.n_bus * 16 + N_SCEN * (4 + 4 + 8)

    # per-kernel times (CUDA events on the launching stream), after a fresh Jacobian
    batch.stage_load(y, s_dev, v_init=v_dev, refine=1)
    batch.stage("mismatch")
    kt = {}
    for name in NRBatch.KERNELS:
        ts = []
        for _ in range(3):
            batch.stage("jacobian")
            if name in ("schur", "dense_lu"):
                batch.kernel("factor_sparse")
            if name == "dense_lu":
                batch.kernel("schur")
            if name in ("solve_fwd", "dense_solve", "solve_bwd"):
                batch.stage("factor")
            torch.cuda.synchronize()
            e0.record()
            batch.kernel(name)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        kt[name] = sorted(ts)[1]
    # per-level latency of the level-scheduled kernels (%globaltimer stamps, one launch each)
    lt = batch.level_trace(y, s_dev, v_init=v_dev)

    def level_summary(d):
        med = np.median(d["level_us"], axis=0)  # per level, median over lane groups
        return {"total_us": float(np.median(d["total_us"])),
                "per_level_us_median": float(np.median(med)) if med.size else 0.0,
                "slowest_level_us": float(med.max()) if med.size else 0.0}

    lu_levels = {"critical_path_levels": info["n_levels"], "dense_tail_order": 2 * info["n_tail"],
                 "max_level_width": info["max_level_width"],
                 "factor_sparse": level_summary(lt["factor"]),
                 "solve_fwd": level_summary(lt["forward"]),
                 "solve_bwd": level_summary(lt["backward"]),
                 "source": "%globaltimer stamps at each level barrier, median over lane groups"}
    if "dense" in lt:
        ph = np.median(lt["dense"]["phase_us"], axis=0)  # [panels, 3], median over scenarios
        st = lt["dense"]["stamps"]
        lu_levels["dense_lu"] = {
            "panels": int(ph.shape[0]), "total_us": float(np.median(st[:, -1] - st[:, 0]) / 1e3),
            "diagonal_blocks_us": float(ph[:, 0].sum()), "l21_u12_solves_us": float(ph[:, 1].sum()),
            "trailing_updates_us": float(ph[:, 2].sum()),
            "source": "per-panel stamps of one CTA (one scenario), median over scenarios; "
                      "CTAs run 2 per SM in 3.5 waves"}
    per_iter = {"mismatch": 1, "jacobian": 1, "factor_sparse": 1, "schur": 1, "dense_lu": 1,
                "solve_fwd": 2, "dense_solve": 2, "solve_bwd": 2, "update": 1, "residual": 1}
    if info["n_tail"] == 0:
        for k in ("schur", "dense_lu", "dense_solve"):
            per_iter[k] = 0
    share = {k: kt[k] * per_iter[k] for k in kt}
    dom = max(share, key=share.get)
    esz = 4
    alg = algorithmic_bytes(dom, info, N_SCEN, esz)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg / (kt[dom] / 1e3) / 1e9
    tps = MEASURED_TRAFFIC_PER_SCENARIO.get(
        "dense_lu_fma" if dom == "dense_lu" and args.dense_fma else dom)
    traffic = tps * N_SCEN if tps else None
    # the dense LU's FP32-accurate flop rate (2/3 N^3 flops per scenario over its time)
    fma_tflops = (N_SCEN * 2.0 / 3.0 * (2 * info["n_tail"]) ** 3 / (kt["dense_lu"] / 1e3) / 1e12
                  if info["n_tail"] and dom == "dense_lu" else None)
    # every kernel of the loop against the same HBM roof (algorithmic bytes / CUDA-event time)
    kernel_roofline = {}
    for k in kt:
        b = algorithmic_bytes(k, info, N_SCEN, esz)
        if b and kt[k] > 0:
            gbs = b / (kt[k] / 1e3) / 1e9
            kernel_roofline[k] = {"ms": kt[k], "algorithmic_bytes": b, "achieved_gbs": gbs,
                                  "frac": gbs / hbm}
    launches_per_iter = 6 + 3 * 2 + 1 + 1 if info["n_tail"] else 4 + 2 * 2 + 1 + 1
    gpu_launches = args.steps * (2 + loops * launches_per_iter)

    # plain FP64 single-scenario path on the same grid
    single = NRBatch(plan, 1, precision="fp64", lanes=1, threads=512)
    s1 = s_dev[:1].contiguous()
    v1 = v_dev[None].contiguous()
    for _ in range(args.warmup):
        rs = single.solve(y, s1, v_init=v1, tol=TOL, max_iter=MAX_ITER, policy="newton")
    torch.cuda.synchronize()
    reps = max(args.steps, 5)
    e0.record()
    for _ in range(reps):
        rs = single.solve(y, s1, v_init=v1, tol=TOL, max_iter=MAX_ITER, policy="newton")
    e1.record()
    torch.cuda.synchronize()
    single_ms = e0.elapsed_time(e1) / reps
    single_ok = int(rs.status[0].item()) == 0
    plain = {"value": (1.0 if single_ok else 0.0) * 1e3 / single_ms, "unit": "solves/s",
             "ms_per_solve": single_ms, "iterations": int(rs.iterations[0].item()),
             "converged": single_ok}

    cpu = None
    if pool is not None:
        sample = list(range(2 * cores)) if cores <= 8 else list(range(cores))
        ok, wall = cpu_run(pool, sample)
        cpu = {"value": ok / wall, "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": f"{len(sample)} scenarios of the same workload, FP64 restatement "
                         f"(scipy sparse LU), one process per core, {wall:.1f} s wall"}
        pool.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
            "data": "synthetic (seeded generator, no external dataset)",
            "config": config({"parallelism": f"scenario shards x{world}",
                              "newton_loop": "host" if args.host_loop else "cuda graph",
                              "dense_lu_trailing_update": "cuda-core fma (device batch)"
                                                          if args.dense_fma else "tensor cores",
                              "converged_per_step": conv_all,
                              "max_iterations_run": int(iters.max()), "plan_seconds": plan_s}),
            "e2e": {"value": conv_e2e * args.steps / (e2e_ms / 1e3), "unit": "solves/s",
                    "api": "HostPipeline: 4 x 256 scenarios on 4 streams, pinned host buffers "
                           "(S_spec per scenario, one shared start vector)",
                    "h2d_bytes_per_step": h2d * world, "d2h_bytes_per_step": d2h * world},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg,
                         "traffic_source": "ncu capture on 320 scenarios, scaled by scenarios"
                         if traffic else None,
                         "dense_lu_effective_tflops": fma_tflops,
                         "launch_ms": kt[dom], "peak_source": "measured" if peaks else "fallback"},
            "kernel_ms": kt, "kernel_share_ms_per_iter": share, "lu_levels": lu_levels,
            "kernel_roofline": kernel_roofline,
            "plain_fp64_single": plain,
            "batched_over_plain_fp64": value / plain["value"] if plain["value"] else None,
            "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": gpu_launches,
        }
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# reference arm: the reference path on host cores (CPU restatement; see module docstring)
# ------------------------------------------------------------------------------------------

REF_NOTE = ("the reference's own CPU backend (dense Jacobian, unordered LU, ~n^4) cannot finish "
            "one 10k-bus solve in bounded time (1000 buses: 134 s per LU factorisation), so the "
            "reference arm runs the FP64 CPU restatement of its algorithm with a sparse LU")


def run_reference(args, rank, world):
    if rank != 0:
        return
    pool, cores = make_pool()
    make_ready(pool, cores)
    for w in range(args.warmup):
        cpu_run(pool, [w])
    tot_ok = 0
    tot_t = 0.0
    for s in range(args.steps):
        idx = [(s * cores + i) % N_SCEN for i in range(cores)]
        ok, t = cpu_run(pool, idx)
        tot_ok += ok
        tot_t += t
    pool.close()
    v = tot_ok / tot_t
    line = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_t / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, no external dataset)", "config": config(),
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} scenarios per step, one process per core; {REF_NOTE}"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# supplementary workloads
# ------------------------------------------------------------------------------------------

def run_mixed(args):
    import numpy as np
    import torch

    from gap_b200 import studies, synth

    t0 = time.perf_counter()
    net = synth.transmission_grid(GRID_SEED, n=2000)
    v0 = synth.dc_start(net, BASE)
    s_load = synth.load_scenarios(net, 1024, sigma=SIGMA, seed=1, base_power=BASE)
    load = studies.load_study("load", net, s_load, v0, base_power=BASE)
    outs = synth.n_minus_1(net, 256)
    cont = studies.contingency_study("n-1", net, outs, net.specified_power(BASE), v0,
                                     base_power=BASE, plan=load.plan)
    grids = []
    for i, n in enumerate(synth.grid_sizes(64)):
        g = synth.transmission_grid(100 + i, n=int(n))
        grids.append(studies.load_study(f"grid{i}", g, g.specified_power(BASE)[None],
                                        synth.dc_start(g, BASE), base_power=BASE))
    setup_s = time.perf_counter() - t0
    all_st = [load, cont] + grids
    kw = dict(tol=TOL, max_iter=MAX_ITER, policy="newton", refine=REFINE_STEPS,
              refine_below=REFINE_BELOW,
              reuse_below=REUSE_BELOW)
    t1 = time.perf_counter()
    for st in all_st:
        studies.autotune(st, **kw)
    tune_s = time.perf_counter() - t1
    with Clocks(0) as clk:
        # one graph launch for the whole mix; unconverged scenarios retried with the clamped
        # step policy inside the same launch
        ms, conv, wall = studies.timed_mixed(all_st, steps=args.steps,
                                             warmup=max(args.warmup, 1), retry="clamped", **kw)
    # the same studies as separate graphs on one stream each (the launch-per-study baseline)
    ms_streams, conv_streams, _ = studies.timed_concurrent(all_st, steps=args.steps,
                                                           warmup=max(args.warmup, 1), **kw)
    studies.solve_mixed(all_st, retry="clamped", **kw)
    torch.cuda.synchronize()
    n_sys = sum(st.n_scen for st in all_st)
    not_conv = {st.name: int((st.result.status != 0).sum().item()) for st in all_st
                if int((st.result.status != 0).sum().item())}
    picks = {}
    for st in all_st:
        key = f"{st.lanes}x{st.threads}"
        picks[key] = picks.get(key, 0) + 1
    # each study alone, for the concurrency gain
    seq = 0.0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for st in all_st:
        e0.record()
        st.batch.solve(st.y, st.s_spec, v_init=st.v0, **kw)
        e1.record()
        torch.cuda.synchronize()
        seq += e0.elapsed_time(e1)
    line = {
        "metric": "Power-flow solves/s on 1 B200, mixed batch (load scenarios + N-1 + "
                  "independent grids) at 1e-8 pu",
        "workload": "mixed", "value": conv / (ms / 1e3), "unit": "solves/s", "n_gpus": 1,
        "steps": args.steps, "ms_per_step": ms, "converged_per_step": conv,
        "systems_per_step": n_sys, "not_converged": not_conv, "higher_is_better": True,
        "launch": "one CUDA graph launch for all studies (gapk_nr_mix_solve), clamped-policy "
                  "retry of unconverged scenarios inside it",
        "per_study_streams": {"value": conv_streams / (ms_streams / 1e3), "ms_per_step": ms_streams,
                              "converged_per_step": conv_streams,
                              "note": "one graph launch per study on its own stream, no retry"},
        "dtype": "fp32+fp64",
        "data": "synthetic (seeded generator, no external dataset)",
        "config": {"workload": "1024 load scenarios + 256 N-1 outages of a 2000-bus grid "
                               "+ 64 independent grids, n log-uniform in [500, 20000]",
                   "grid_sizes": [int(g.net.n_bus) for g in grids],
                   "tol_pu": TOL, "max_iter": MAX_ITER, "policy": "newton",
                   "precision": "fp32 factor+solve, fp64 mismatch/update; below 1e-2 pu: 2 "
                                                   "refinement steps, factors reused",
                   "streams": len(all_st), "autotuned_lanes_x_threads": picks,
                   "autotuned_load_and_n-1": [f"{st.lanes}x{st.threads}" for st in all_st[:2]]},
        "sequential_ms": seq, "concurrency_gain": seq / ms,
        "host_wall_ms_per_step": wall * 1e3, "setup_seconds": setup_s,
        "autotune_seconds": tune_s, "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_large(args):
    import numpy as np
    import torch

    from gap_b200 import studies, synth

    t0 = time.perf_counter()
    # at 100k buses the headline's loading (p ~ U[0,1] x 0.05 pu) has no solution reachable
    # from the DC start (FP64 and FP32 alike cycle at 4-11 pu); half of it converges
    net = synth.transmission_grid(GRID_SEED, n=args.large_buses, load_scale=LARGE_LOAD_SCALE)
    v0 = synth.dc_start(net, BASE)
    S = 32
    s_load = synth.load_scenarios(net, S, sigma=SIGMA, seed=1, base_power=BASE)
    gen_s = time.perf_counter() - t0
    t1 = time.perf_counter()
    st = studies.load_study("large", net, s_load, v0, base_power=BASE)
    plan_s = time.perf_counter() - t1
    st.lanes, st.threads = 8, 1024
    b = st.make_batch()
    # full Newton steps with the reference's clamps: pure Newton diverges on a few of these
    # scenarios from the DC start (as the FP64 oracle does), the clamped steps converge
    kw = dict(tol=TOL, max_iter=30, policy="clamped", refine=REFINE_STEPS,
              refine_below=REFINE_BELOW,
              reuse_below=REUSE_BELOW)
    r = b.solve(st.y, st.s_spec, v_init=st.v0, **kw)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record()
        for _ in range(args.steps):
            r = b.solve(st.y, st.s_spec, v_init=st.v0, **kw)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    status = r.status.cpu().numpy()
    iters = r.iterations.cpu().numpy()
    info = st.plan.info
    line = {
        "metric": f"Power-flow solves/s on 1 B200, {args.large_buses}-bus grid, FP32 factor + "
                  "FP64 refinement at 1e-8 pu",
        "workload": "large", "value": int((status == 0).sum()) / (ms / 1e3),
        "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "fp32+fp64",
        "data": "synthetic (seeded generator, no external dataset)",
        "config": {"workload": f"32 load scenarios x {args.large_buses}-bus transmission grid "
                               f"(seed {GRID_SEED}, load scale {LARGE_LOAD_SCALE})",
                   "policy": "clamped Newton",
                   "max_iter": 30,
                   "n_tail": info["n_tail"], "nnz_l_blocks": info["nnz_l_blocks"],
                   "n_pairs": info["n_pairs"], "n_schur_pairs": info["n_schur_pairs"]},
        "converged": int((status == 0).sum()), "iterations_max": int(iters.max()),
        "device_bytes": b.device_bytes,
        "generate_seconds": gen_s, "plan_seconds": plan_s, "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_adjoint(args):
    import numpy as np
    import torch

    from gap_b200 import synth
    from gap_b200.autograd import DifferentiablePowerFlow, branch_losses_mw

    net = synth.transmission_grid(GRID_SEED, n=N_BUS)
    S = 256
    s = synth.load_scenarios(net, S, sigma=SIGMA, seed=1, base_power=BASE)
    out = {}
    for prec in ("fp64", "fp32"):
        model = DifferentiablePowerFlow(net, S, base_power=BASE, precision=prec, tol=1e-10,
                                        max_iter=30)
        p = torch.tensor(s.real, device="cuda", requires_grad=True)
        q = torch.tensor(s.imag, device="cuda", requires_grad=True)
        r = model.branch[:, 0].clone().requires_grad_(True)
        x = model.branch[:, 1].clone().requires_grad_(True)

        def step():
            for t in (p, q, r, x):
                t.grad = None
            vm, va = model(p, q, r, x)
            L = ((vm - 1.0) ** 2).sum() + branch_losses_mw(vm, va, r, x, model).sum()
            L.backward()
            return L

        for _ in range(max(args.warmup, 1)):
            step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            L = step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out[prec] = {"ms_per_step": ms, "gradients_per_s": S / (ms / 1e3),
                     "loss": float(L.item()),
                     "grad_norms": [float(t.grad.norm().item()) for t in (p, q, r, x)]}
    line = {
        "metric": "Loss gradients/s on 1 B200 (power flow + adjoint, dL/dP, dL/dQ per bus and "
                  "dL/dr, dL/dx per branch)",
        "workload": "adjoint", "value": out["fp64"]["gradients_per_s"], "unit": "gradients/s",
        "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded generator, no external dataset)",
        "config": {"workload": f"{S} load scenarios x {N_BUS}-bus transmission grid "
                               f"(seed {GRID_SEED})",
                   "loss": "sum_bus (|V|-1)^2 + sum_branch P_loss [MW]", "tol_pu": 1e-10},
        "fp64": out["fp64"], "fp32_factor_refined": out["fp32"],
    }
    print(json.dumps(line), flush=True)


def run_feeder(args):
    """The 200-bus meshed feeder, the one size where the reference's own CPU backend finishes.
    Reference step policy (the reference's damped, clamped update), tol 1e-8 pu, flat start."""
    import numpy as np
    import torch

    from gap_b200 import _native as N
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    base = 1e6
    net = synth.feeder_grid(0)
    zb = float(net.u_rated[0]) ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=N.YBUS_REFERENCE,
                    scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type)
    u = torch.as_tensor(net.u_pu.astype(np.float64), device="cuda")
    kw = dict(tol=1e-8, max_iter=20, policy="reference", u_pu=u)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    res = {}
    for name, S in (("single_fp64", 1), ("batched_fp64", 1024)):
        s = (net.specified_power(base)[None] if S == 1 else
             synth.load_scenarios(net, S, sigma=SIGMA, seed=1, base_power=base))
        st = torch.as_tensor(s, device="cuda")
        b = NRBatch(plan, S, precision="fp64", lanes=1 if S == 1 else 8,
                    threads=256 if S == 1 else 512)
        for _ in range(max(args.warmup, 1)):
            r = b.solve(y, st, **kw)
        torch.cuda.synchronize()
        reps = max(args.steps, 5)
        e0.record()
        for _ in range(reps):
            r = b.solve(y, st, **kw)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        conv = int((r.status == 0).sum().item())
        res[name] = {"solves_per_s": conv / (ms / 1e3), "ms_per_batch": ms, "scenarios": S,
                     "converged": conv, "iterations_max": int(r.iterations.max().item())}
    cpu = None
    try:
        from oracle import refnet  # the reference's own CPU backend, built from its sources

        if refnet.available():
            refnet.solve(net, tol=1e-8, max_iter=20, base_power=base)  # warm-up
            t0 = time.perf_counter()
            o = refnet.solve(net, tol=1e-8, max_iter=20, base_power=base)
            wall = time.perf_counter() - t0
            cpu = {"value": 1.0 / wall if o["converged"] else 0.0, "unit": "solves/s",
                   "cores": 1, "kind": "reference",
                   "sample": f"one solve of the same feeder by the reference's CPU backend "
                             f"(dense Jacobian, its LU), {o['iterations']} iterations, "
                             f"{wall:.2f} s"}
    except Exception as e:  # the compiled reference is optional on a box without it
        cpu = {"unavailable": str(e)[:200]}
    line = {
        "metric": "Power-flow solves/s on 1 B200, 200-bus meshed feeder (reference step "
                  "policy, FP64) at 1e-8 pu",
        "workload": "feeder", "value": res["batched_fp64"]["solves_per_s"], "unit": "solves/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded generator, no external dataset)",
        "config": {"workload": "200-bus meshed feeder (seed 0); 1024 lognormal load scenarios "
                               "for the batched line", "policy": "reference", "tol_pu": 1e-8,
                   "start": "flat"},
        "single_fp64": res["single_fp64"], "batched_fp64": res["batched_fp64"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    global N_SCEN
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenarios", type=int, default=N_SCEN,
                    help="scenarios per GPU (profiling runs use fewer; the headline uses 1024)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling)")
    ap.add_argument("--workload", default="transmission",
                    choices=["transmission", "mixed", "large", "adjoint", "feeder"],
                    help="transmission: the headline; mixed / large: supplementary lines")
    ap.add_argument("--large-buses", type=int, default=100_000,
                    help="grid size of --workload large")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the Newton loop from the host instead of one CUDA graph with a "
                         "conditional node (same kernels and work; lets ncu see every launch)")
    ap.add_argument("--dense-fma", action="store_true",
                    help="device-resident batch only: the dense-tail LU's trailing update on "
                         "CUDA-core FMA (k_dense_lu) instead of the tensor cores (k_dense_lu_tc)")
    args = ap.parse_args()
    N_SCEN = args.scenarios
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch

    torch.cuda.set_device(local)
    if args.workload != "transmission":
        {"mixed": run_mixed, "large": run_large, "adjoint": run_adjoint,
         "feeder": run_feeder}[args.workload](args)
        return
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as tdist

            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
