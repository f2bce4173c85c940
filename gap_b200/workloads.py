"""The headline workload: one definition shared by the benchmark and the parity tests.

1024 load scenarios (per-bus lognormal factors, sigma 0.1) of the seeded 10,000-bus
transmission-like grid (`synth.transmission_grid(0)`), solved together to max |mismatch| <
1e-8 pu: FP32 Jacobian factor and triangular solves, FP64 mismatch / update / convergence; once
a lane group's max |mismatch| is below 1e-2 pu it refines every correction twice in FP64 and
keeps its previous LU factors.  Pure Newton steps from one DC-flow start shared by every
scenario; 8 scenario lanes per group and 1024-thread level-scheduled kernels, which puts the
dense tail (order 506) on the one-CTA-per-scenario LU.

`DEVIATIONS` lists where the generator fixes what the workload's written specification leaves
open or cannot meet (the specified loading has no power-flow solution on this grid).
"""

from __future__ import annotations

N_BUS = 10_000
GRID_SEED = 0
N_SCEN = 1024
SIGMA = 0.1
TOL = 1e-8
MAX_ITER = 20
BASE = 1e8  # 100 MVA
PRECISION = "fp32"
LANES = 8
THREADS = 1024
POLICY = "newton"
# FP64 refinement steps per Newton correction once a lane group's max |mismatch| < 1e-2 pu
REFINE_STEPS = 2
REFINE_BELOW = 1e-2
# ... and below the same mismatch the lane group keeps its previous LU factors
REUSE_BELOW = 1e-2

DEVIATIONS = {
    "load_scale": "loads p ~ U[0,1] x 0.05 pu, q = U[0.1,0.4] p (the written p ~ U[0,1] pu has "
                  "no solution: the load-scale continuation of the FP64 oracle stops at its "
                  "nose point, tests/test_workload_loading.py)",
    "transformers": "10 % of branches, drawn from the bridge branches first, b = 0",
    "pv": "20 % PV buses, placed so every bus is within 2 hops of voltage control; each PV bus "
          "generates the load of the buses nearest to it (local dispatch)",
    "start": "DC-flow angles, |V| at the PV / slack setpoints, 1.0 pu elsewhere (one start "
             "vector shared by every scenario)",
}


def solve_kwargs():
    """Keyword arguments of NRBatch.solve for the headline solve."""
    return dict(tol=TOL, max_iter=MAX_ITER, policy=POLICY, refine=REFINE_STEPS,
                refine_below=REFINE_BELOW, reuse_below=REUSE_BELOW)


def batch_kwargs():
    """Keyword arguments of NRBatch for the headline batch."""
    return dict(precision=PRECISION, lanes=LANES, threads=THREADS)


def headline(rank: int = 0, n_scen: int = N_SCEN):
    """(network, S_spec complex128 [n_scen, n_bus] per unit, shared start vector [n_bus]).
    Rank r of a multi-GPU run draws its own scenarios (seed 1 + r)."""
    from . import synth

    net = synth.transmission_grid(GRID_SEED, n=N_BUS)
    s_spec = synth.load_scenarios(net, n_scen, sigma=SIGMA, seed=1 + rank, base_power=BASE)
    return net, s_spec, synth.dc_start(net, BASE)
