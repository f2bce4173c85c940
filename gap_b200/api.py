"""Reference-facing Python API of the B200 power-flow engine.

Mirrors the reference's interfaces for the Newton-Raphson path:

* `PowerFlowConfig`, `PowerFlowResult`       include/gap/solver/powerflow_interface.h:13-43
* `AdmittanceMatrix.build_admittance_matrix`  include/gap/admittance/admittance_interface.h:21
* `NewtonRaphson.solve_power_flow` / `.calculate_mismatches`
                                              include/gap/solver/powerflow_interface.h:59-79
* `IterationState`, `NewtonRaphson.enable_state_capture` / `.get_iteration_states` /
  `.clear_iteration_states`                   include/gap/solver/powerflow_interface.h:28-35,
                                              83-107
* `solve_simple_power_flow`                   bindings/solver_bindings.cpp:56-217 (same
                                              argument lists, same output rows)

Everything computes on the GPU through libgapk.so; `backend` values other than the GPU
ones raise, as the reference raises for an unavailable backend.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .engine import NRBatch, NRPlan, YbusPlan, branch_params, require_cuda, shunt_params
from .network import PQ, PV, SLACK, Network


@dataclass
class PowerFlowConfig:
    """gap::solver::PowerFlowConfig (powerflow_interface.h:13-20) plus engine options."""

    tolerance: float = 1e-6
    max_iterations: int = 50
    use_flat_start: bool = True
    acceleration_factor: float = 1.0  # accepted for compatibility; the reference CPU path
    verbose: bool = False             # ignores it and so does this engine
    base_power: float = 100e6
    # engine options (no reference counterpart)
    policy: str = "reference"   # "reference" (damped, clamped) or "newton"
    jacobian: str = "reference"  # "reference" (last duplicate) or "exact"
    precision: str = "fp64"      # "fp64" or "fp32" (mixed: FP32 factor, FP64 mismatch/update)
    refine: int = 0              # iterative-refinement steps per correction (fp32 only)
    ybus_taps: bool = False      # apply transformer tap / phase shift (the reference ignores)


@dataclass
class PowerFlowResult:
    """gap::solver::PowerFlowResult (powerflow_interface.h:37-43)."""

    converged: bool = False
    iterations: int = 0
    final_mismatch: float = 0.0
    bus_voltages: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex128))
    bus_injections: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex128))
    status: int = N.SCEN_MAXITER


@dataclass
class IterationState:
    """gap::solver::IterationState (powerflow_interface.h:28-35): the state one iteration's
    mismatch is taken at, per unit; mismatches in the reference's equation order."""

    iteration: int
    voltages: np.ndarray
    currents: np.ndarray
    power_injections: np.ndarray
    mismatches: np.ndarray
    max_mismatch: float


class AdmittanceMatrix:
    """GPU Y-bus builder (IAdmittanceMatrix).  Returns the CSR triple in Siemens."""

    def __init__(self, taps: bool = False):
        self.mode = N.YBUS_TAPS if taps else N.YBUS_REFERENCE
        self._cache = {}

    def plan(self, net: Network) -> YbusPlan:
        f, t, valid = net.branch_index()
        sb, _, _ = net.shunt_index()
        key = (net.n_bus, np.where(valid, f, -1).tobytes(), np.where(valid, t, -1).tobytes(),
               np.asarray(sb).tobytes())
        p = self._cache.get(key)
        if p is None:
            p = YbusPlan.from_network(net)
            self._cache = {key: p}
        return p

    def build_device(self, net: Network, scale: float = 1.0):
        """Values on the device (complex128 [nnz]) and the plan."""
        import torch

        require_cuda()
        p = self.plan(net)
        br = torch.as_tensor(branch_params(net), device="cuda")
        sh = torch.as_tensor(shunt_params(net), device="cuda")
        return p, p.assemble(br, sh, mode=self.mode, scale=scale)[0]

    def build_admittance_matrix(self, net: Network):
        p, vals = self.build_device(net)
        return p.row_ptr.copy(), p.col_idx.copy(), vals.cpu().numpy()

    def get_backend_type(self):
        return "GPU_CUDA"


class NewtonRaphson:
    """GPU Newton-Raphson solver (IPowerFlowSolver).  Plans are cached per (Y pattern, bus
    types, Jacobian mode) and rebuilt when any of them changes."""

    def __init__(self):
        self._plans = {}
        self._batches = {}
        self._capture = False
        self._states = []

    def _plan(self, row_ptr, col_idx, bus_type, jac):
        key = (np.asarray(row_ptr, np.int32).tobytes(), np.asarray(col_idx, np.int32).tobytes(),
               np.asarray(bus_type, np.int32).tobytes(), jac)
        p = self._plans.get(key)
        if p is None:
            p = NRPlan(row_ptr, col_idx, bus_type, jacobian=jac)
            if len(self._plans) > 8:
                self._plans.clear()
                self._batches.clear()
            self._plans[key] = p
        return p

    def _batch(self, plan, precision):
        key = (id(plan), precision)
        b = self._batches.get(key)
        if b is None:
            b = NRBatch(plan, 1, precision=precision, y_shared=True, lanes=1)
            self._batches[key] = b
        return b

    def solve_power_flow(self, net: Network, admittance_matrix=None,
                         config: PowerFlowConfig = PowerFlowConfig()) -> PowerFlowResult:
        """IPowerFlowSolver::solve_power_flow.  admittance_matrix: (row_ptr, col_idx, values)
        in Siemens, or None to build it on the GPU.  Per unit on buses[0].u_rated and
        config.base_power (cpu_newton_raphson.cpp:46-58)."""
        import torch

        require_cuda()
        if net.n_bus == 0:
            return PowerFlowResult(converged=True, iterations=1)
        zb = float(net.u_rated[0]) * float(net.u_rated[0]) / config.base_power
        if admittance_matrix is None:
            yp, y = AdmittanceMatrix(config.ybus_taps).build_device(net, scale=zb)
            row_ptr, col_idx = yp.row_ptr, yp.col_idx
        else:
            row_ptr, col_idx, vals = admittance_matrix
            v = np.asarray(vals, np.complex128)
            ypu = np.empty_like(v)
            ypu.real = v.real * zb
            ypu.imag = v.imag * zb
            y = torch.as_tensor(ypu, device="cuda")
        plan = self._plan(row_ptr, col_idx, net.bus_type, config.jacobian)
        batch = self._batch(plan, config.precision)
        s = torch.as_tensor(net.specified_power(config.base_power)[None, :], device="cuda")
        u = torch.as_tensor(net.u_pu, dtype=torch.float64, device="cuda")
        kw = dict(u_pu=u, tol=config.tolerance, max_iter=config.max_iterations,
                  policy=config.policy, refine=config.refine)
        if self._capture:
            r, states = batch.solve_captured(y, s, **kw)
            torch.cuda.synchronize()
            self._states = [IterationState(
                iteration=int(x["iteration"]), voltages=x["v"][0].cpu().numpy(),
                currents=x["i"][0].cpu().numpy(), power_injections=x["s"][0].cpu().numpy(),
                mismatches=x["mismatch"][0].cpu().numpy(),
                max_mismatch=float(x["max_mismatch"][0].item())) for x in states]
            if int(r.status[0].item()) == N.SCEN_SINGULAR:
                # the device loop stops a scenario whose Jacobian does not factorise; the
                # reference keeps V and runs on to max_iterations (cpu_newton_raphson.cpp:
                # 416-419), recording the same state each time
                while self._states and len(self._states) < int(r.iterations[0].item()):
                    last = self._states[-1]
                    self._states.append(IterationState(len(self._states), last.voltages,
                                                       last.currents, last.power_injections,
                                                       last.mismatches, last.max_mismatch))
        else:
            r = batch.solve(y, s, **kw)
            torch.cuda.synchronize()
        st = int(r.status[0].item())
        # bus_injections, which the reference declares but never fills: S = V conj(Y V) at
        # the final voltages, per unit of base_power like bus_voltages
        _, _, s_bus = batch.state()
        return PowerFlowResult(converged=st == N.SCEN_CONVERGED,
                               iterations=int(r.iterations[0].item()),
                               final_mismatch=float(r.final_mismatch[0].item()),
                               bus_voltages=r.v[0].cpu().numpy(),
                               bus_injections=s_bus[0].cpu().numpy(), status=st)

    def calculate_mismatches(self, net: Network, bus_voltages, admittance_matrix=None):
        """IPowerFlowSolver::calculate_mismatches: reference equation order, in Watts / var
        on the fixed 100 MVA base the reference's public method uses
        (cpu_newton_raphson.cpp:225-240)."""
        import torch

        require_cuda()
        base = 100e6
        if admittance_matrix is None:
            yp, y = AdmittanceMatrix().build_device(net)
            row_ptr, col_idx = yp.row_ptr, yp.col_idx
        else:
            row_ptr, col_idx, vals = admittance_matrix
            y = torch.as_tensor(np.asarray(vals, np.complex128), device="cuda")
        plan = self._plan(row_ptr, col_idx, net.bus_type, "reference")
        batch = self._batch(plan, "fp64")
        s = torch.as_tensor(net.specified_power(base)[None, :], device="cuda")
        v = torch.as_tensor(np.asarray(bus_voltages, np.complex128)[None, :], device="cuda")
        batch.stage_load(y, s, v_init=v)
        batch.stage("mismatch")
        f = batch.mismatch()
        torch.cuda.synchronize()
        return f[0].cpu().numpy() * base

    def enable_state_capture(self, enable: bool):
        """Record an IterationState per iteration of each following solve (the device loop is
        then stepped from the host, one synchronisation per iteration; same trajectory).  The
        states of the last solve replace the previous ones, as gpu_newton_raphson.cu:402-405."""
        self._capture = bool(enable)

    def get_iteration_states(self):
        return self._states

    def clear_iteration_states(self):
        self._states = []

    def set_lu_solver(self, lu_solver):
        """Accepted for interface compatibility: the device-resident engine factorises the
        Jacobian with its own block LU and never hands it to a host-side solver."""
        self._lu = lu_solver

    def get_backend_type(self):
        return "GPU_CUDA"


def network_from_simple_lists(bus_data, branch_data) -> Network:
    """List conversion of solve_simple_power_flow (bindings/solver_bindings.cpp:67-111):
    bus rows [id, u_rated, bus_type, u_pu, u_angle, p, q] (>= 7 entries), branch rows
    [id, from, to, r, x, (b)] (>= 5 entries); every branch in service, g1 = 0, k = 1."""
    for row in bus_data:
        if len(row) < 7:
            raise RuntimeError("Bus data must have at least 7 elements: [id, u_rated, bus_type, "
                               "u_pu, u_angle, p, q]")
    for row in branch_data:
        if len(row) < 5:
            raise RuntimeError("Branch data must have at least 5 elements: [id, from_bus, "
                               "to_bus, r, x]")
    nb = len(bus_data)
    m = len(branch_data)
    bus = np.zeros((nb, 7))
    for i, row in enumerate(bus_data):
        bus[i] = [float(x) for x in row[:7]]
    br = np.zeros((m, 6))
    for i, row in enumerate(branch_data):
        br[i, :5] = [float(x) for x in row[:5]]
        br[i, 5] = float(row[5]) if len(row) > 5 else 0.0
    return Network.build(bus_id=bus[:, 0].astype(np.int64).astype(np.int32), u_rated=bus[:, 1],
                         bus_type=bus[:, 2].astype(np.int32), u_pu=bus[:, 3], p=bus[:, 5],
                         q=bus[:, 6], br_id=br[:, 0].astype(np.int32),
                         from_id=br[:, 1].astype(np.int32), to_id=br[:, 2].astype(np.int32),
                         r1=br[:, 3], x1=br[:, 4], b1=br[:, 5])


_GPU_NAMES = ("gpu", "GPU", "cuda", "CUDA")
_default_solver = None


def solve_simple_power_flow(bus_data, branch_data, tolerance=1e-6, max_iterations=50,
                            verbose=False, base_power=100e6, backend="gpu"):
    """bindings/solver_bindings.cpp:56-217.  Returns one row [re, im, |V|, arg V] per bus
    and a last row [converged, iterations, final_mismatch, 0]."""
    global _default_solver
    if backend not in _GPU_NAMES:
        raise RuntimeError(f"Simple power flow solution failed: Requested backend '{backend}' "
                           "is not available (gap_b200 provides the GPU backend)")
    try:
        net = network_from_simple_lists(bus_data, branch_data)
        cfg = PowerFlowConfig(tolerance=tolerance, max_iterations=max_iterations,
                              verbose=verbose, base_power=base_power)
        if _default_solver is None:
            _default_solver = NewtonRaphson()
        ybuilder = AdmittanceMatrix()
        Y = ybuilder.build_admittance_matrix(net) if net.n_bus else None
        res = _default_solver.solve_power_flow(net, Y, cfg)
    except Exception as e:  # same wrapping as the reference binding (:178-181)
        raise RuntimeError(f"Simple power flow solution failed: {e}") from e
    out = []
    for v in res.bus_voltages:
        out.append([v.real, v.imag, abs(v), math.atan2(v.imag, v.real)])
    out.append([1.0 if res.converged else 0.0, float(res.iterations), res.final_mismatch, 0.0])
    return out


def is_cuda_available() -> bool:
    """gap_solver.is_cuda_available (bindings/cuda_bindings.cpp)."""
    try:
        return N.lib().gapk_device_count() > 0
    except Exception:
        return False
