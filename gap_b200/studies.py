"""Mixed batches of power-flow studies on one GPU (no counterpart in the reference).

A *study* is one NRPlan (one Y pattern and bus-type vector) with its own batch of scenarios.
Three kinds of study are built here, and any number of them run concurrently, each on its own
CUDA stream, with the Newton loop of every study captured once as a CUDA graph:

* load scenarios of one grid: one Y shared by every scenario, per-scenario S_spec;
* N-1 branch contingencies of one grid: the grid's own Y pattern, one Y value set per
  scenario: the base values with the outaged branch's stamps removed on the device (a
  batched, fixed version of the reference's update_admittance_matrix,
  src/admittance/cpu/cpu_admittance_matrix.cpp:204-301), so the outage leaves (near-)zeros in
  place of the branch's entries and every contingency shares the base grid's symbolic
  analysis;
* independent grids: one study per grid.

`autotune` picks the scenario-lane count and the thread count of the level-scheduled kernels
for a study by timing candidates on the study's own inputs.
"""

from __future__ import annotations

import time
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .engine import (NRBatch, NRMix, NRPlan, NRResult, YbusDelta, YbusPlan, branch_params,
                     shunt_params)
from .network import Network


def _torch():
    import torch

    return torch


# ----------------------------------------------------------------------------------------
# contingencies (outage candidates: synth.n_minus_1, the non-bridge in-service branches)
# ----------------------------------------------------------------------------------------

def contingency_branch_params(net: Network, outages) -> np.ndarray:
    """[S, m, 6] branch parameters (r1, x1, g1, b1, k, theta), scenario s with branch
    outages[s] stamped as zero admittance."""
    base = branch_params(net)
    outages = np.asarray(outages, dtype=np.int64)
    out = np.repeat(base[None], len(outages), axis=0)
    out[np.arange(len(outages)), outages, 0:4] = 0.0
    return out


def outage_network(net: Network, branch: int) -> Network:
    """Copy of `net` with one branch out of service (status 0)."""
    import dataclasses

    st = net.status.copy()
    st[branch] = 0
    return dataclasses.replace(net, status=st)


# ----------------------------------------------------------------------------------------
# studies
# ----------------------------------------------------------------------------------------

@dataclass
class Study:
    """One plan with its scenarios, ready to solve: y is [nnz] (shared) or [S, nnz]."""
    name: str
    net: Network
    plan: NRPlan
    y: object
    s_spec: object
    v0: object
    precision: str = "fp32"
    lanes: int = 0
    threads: int = 0
    batch: NRBatch | None = None
    stream: object = None
    result: NRResult | None = None
    info: dict = field(default_factory=dict)

    @property
    def n_scen(self) -> int:
        return int(self.s_spec.shape[0])

    @property
    def y_shared(self) -> bool:
        return self.y.dim() == 1

    def make_batch(self):
        if self.batch is None:
            self.batch = NRBatch(self.plan, self.n_scen, precision=self.precision,
                                 y_shared=self.y_shared, lanes=self.lanes,
                                 threads=self.threads)
        return self.batch


def _ybus(net: Network, base_power: float, branch=None, taps=True):
    torch = _torch()
    zb = float(net.u_rated[0]) ** 2 / base_power
    yp = YbusPlan.from_network(net)
    br = torch.as_tensor(branch_params(net) if branch is None else branch, device="cuda")
    y = yp.assemble(br, torch.as_tensor(shunt_params(net), device="cuda"),
                    mode=N.YBUS_TAPS if taps else N.YBUS_REFERENCE, scale=zb)
    return yp, y


def load_study(name, net: Network, s_spec, v0, base_power=1e8, precision="fp32",
               plan: NRPlan | None = None) -> Study:
    """Load scenarios of one grid: s_spec [S, n] per unit, v0 [n] or [S, n]."""
    torch = _torch()
    yp, y = _ybus(net, base_power)
    if plan is None:
        plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    s = torch.as_tensor(np.asarray(s_spec, np.complex128), device="cuda")
    v = np.asarray(v0, np.complex128)
    if v.ndim == 1:
        v = np.repeat(v[None], s.shape[0], axis=0)
    return Study(name, net, plan, y[0], s, torch.as_tensor(v, device="cuda"), precision)


def contingency_study(name, net: Network, outages, s_spec, v0, base_power=1e8,
                      precision="fp32", plan: NRPlan | None = None) -> Study:
    """N-1 branch outages of one grid, one scenario per outage, sharing the grid's plan.  The
    scenarios' Y values are the base grid's with the outaged branch's stamps removed on the
    device (YbusDelta, builder's pi-model stamps): its entries stay in the pattern as
    (near-)zeros, so every scenario keeps the base symbolic analysis."""
    torch = _torch()
    yp, y0 = _ybus(net, base_power)
    if plan is None:
        plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    S = len(outages)
    y = y0.repeat(S, 1).contiguous()
    delta = YbusDelta(yp, [[int(b)] for b in outages])
    zb = float(net.u_rated[0]) ** 2 / base_power
    delta.apply(y, delta.params(branch_params(net), 0.0), mode="fixed_taps", scale=zb)
    s = np.asarray(s_spec, np.complex128)
    if s.ndim == 1:
        s = np.repeat(s[None], S, axis=0)
    v = np.asarray(v0, np.complex128)
    if v.ndim == 1:
        v = np.repeat(v[None], S, axis=0)
    st = Study(name, net, plan, y, torch.as_tensor(s, device="cuda"),
               torch.as_tensor(v, device="cuda"), precision)
    st.info["outages"] = np.asarray(outages)
    return st


# ----------------------------------------------------------------------------------------
# autotuning and concurrent solves
# ----------------------------------------------------------------------------------------

CANDIDATES = ((8, 1024), (4, 1024), (8, 512), (4, 512), (2, 512), (1, 512), (1, 256))
_TUNED: "weakref.WeakKeyDictionary[NRPlan, dict]" = weakref.WeakKeyDictionary()


def autotune(study: Study, tol=1e-8, max_iter=20, policy="newton", refine=1,
             candidates=CANDIDATES, reps=2, refine_below=0.0, reuse_below=0.0):
    """Time each (lanes, threads) candidate on the study's own inputs (CUDA events, after a
    warm-up solve) and keep the fastest batch in the study.  Candidates whose lane count
    exceeds the scenario count are skipped; results are cached per (plan, S, precision,
    shared Y)."""
    torch = _torch()
    cache = _TUNED.setdefault(study.plan, {})
    key = (study.n_scen, study.precision, study.y_shared)
    if key in cache:
        study.lanes, study.threads = cache[key]
        study.batch = None
        study.make_batch()
        return cache[key]
    best = None
    times = {}
    for lanes, threads in candidates:
        if lanes > max(1, study.n_scen):
            continue
        b = NRBatch(study.plan, study.n_scen, precision=study.precision,
                    y_shared=study.y_shared, lanes=lanes, threads=threads)
        b.solve(study.y, study.s_spec, v_init=study.v0, tol=tol, max_iter=max_iter,
                policy=policy, refine=refine, refine_below=refine_below,
                reuse_below=reuse_below)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            b.solve(study.y, study.s_spec, v_init=study.v0, tol=tol, max_iter=max_iter,
                    policy=policy, refine=refine, refine_below=refine_below,
                reuse_below=reuse_below)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        times[(lanes, threads)] = ms
        if best is None or ms < best[0]:
            best = (ms, lanes, threads, b)
        else:
            del b
    _, study.lanes, study.threads, study.batch = best
    study.info["autotune_ms"] = times
    cache[key] = (study.lanes, study.threads)
    return study.lanes, study.threads


def solve_concurrent(studies, tol=1e-8, max_iter=20, policy="newton", refine=1,
                     refine_below=0.0, reuse_below=0.0):
    """Launch every study on its own CUDA stream (inputs made visible to it first) and wait
    for all of them.  Each study's result lands in `study.result`."""
    torch = _torch()
    cur = torch.cuda.current_stream()
    for st in studies:
        st.make_batch()
        if st.stream is None:
            st.stream = torch.cuda.Stream()
        st.stream.wait_stream(cur)
    for st in studies:
        with torch.cuda.stream(st.stream):
            st.result = st.batch.solve(st.y, st.s_spec, v_init=st.v0, tol=tol,
                                       max_iter=max_iter, policy=policy, refine=refine,
                                       stream=st.stream, refine_below=refine_below,
                                       reuse_below=reuse_below)
    for st in studies:
        cur.wait_stream(st.stream)
    return [st.result for st in studies]


def timed_concurrent(studies, steps=3, warmup=1, **kw):
    """Device time (ms, CUDA events on the current stream, which waits for every study) of
    `steps` rounds of solve_concurrent after `warmup` rounds, and the converged count of the
    last round."""
    torch = _torch()
    for _ in range(warmup):
        solve_concurrent(studies, **kw)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    for _ in range(steps):
        solve_concurrent(studies, **kw)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    conv = sum(int((st.result.status == 0).sum().item()) for st in studies)
    return e0.elapsed_time(e1) / steps, conv, wall / steps


# ----------------------------------------------------------------------------------------
# one launch for the whole mix
# ----------------------------------------------------------------------------------------

_MIXES: "weakref.WeakValueDictionary" = weakref.WeakValueDictionary()


class _MixHolder:
    def __init__(self, mix):
        self.mix = mix


def solve_mixed(studies, tol=1e-8, max_iter=20, policy="newton", refine=1, refine_below=0.0,
                reuse_below=0.0, retry="clamped", stream=None):
    """Every study solved by ONE graph launch (engine.NRMix over the studies' batches): each
    study's solve is a branch of the graph; with `retry`, scenarios that end unconverged restart
    from their start vector under that step policy inside the same launch.  Results land in
    `study.result` (the same tensors on every call; asynchronous on the stream)."""
    for st in studies:
        st.make_batch()
    key = tuple(id(st.batch) for st in studies)
    holder = _MIXES.get(key)
    if holder is None:
        holder = _MixHolder(NRMix([st.batch for st in studies]))
        _MIXES[key] = holder
        for st in studies:
            st.info["_mix"] = holder  # keeps the mix alive as long as its studies
    res = holder.mix.solve([st.y for st in studies], [st.s_spec for st in studies],
                           [st.v0 for st in studies], tol=tol, max_iter=max_iter, policy=policy,
                           refine=refine, refine_below=refine_below, reuse_below=reuse_below,
                           retry=retry, stream=stream)
    for st, r in zip(studies, res):
        st.result = r
    return res


def timed_mixed(studies, steps=3, warmup=1, **kw):
    """Device time (ms, CUDA events) of `steps` one-launch solves of the whole mix after
    `warmup` solves, the converged count of the last solve and the host wall time per step."""
    torch = _torch()
    for _ in range(warmup):
        solve_mixed(studies, **kw)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    for _ in range(steps):
        solve_mixed(studies, **kw)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    conv = sum(int((st.result.status == 0).sum().item()) for st in studies)
    return e0.elapsed_time(e1) / steps, conv, wall / steps
