"""Python host layer over libgapk.so: Y-bus builder, Newton-Raphson plans and batches.

Device memory and streams come from PyTorch (tensors on cuda, torch's current stream); all
compute runs in the library's sm_100a kernels.  There is no CPU fallback: on a machine
without the library or without a GPU these classes raise.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .network import PQ, PV, SLACK, Network


def _torch():
    import torch

    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def require_cuda():
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("gap_b200 needs a CUDA device (no CPU fallback on the product path)")
    N.lib()


# ----------------------------------------------------------------------------------------
# Y-bus
# ----------------------------------------------------------------------------------------


class YbusPlan:
    """CSR pattern of one topology (host, built once) + device value assembly.

    Replaces IAdmittanceMatrix::build_admittance_matrix
    (include/gap/admittance/admittance_interface.h:21-22): the pattern equals the reference's
    stable-sorted triplet order (src/admittance/cpu/cpu_admittance_matrix.cpp:100-186)."""

    def __init__(self, n_bus, from_idx, to_idx, in_service, shunt_bus=()):
        L = N.lib()
        self.n_bus = int(n_bus)
        f = N.i32(from_idx)
        t = N.i32(to_idx)
        s = N.i32(in_service)
        sb = N.i32(shunt_bus)
        self.n_branch = int(f.size)
        self.n_shunt = int(sb.size)
        self.from_idx, self.to_idx, self.in_service = f, t, s
        h = C.c_void_p()
        N.check(L.gapk_ybus_create(C.c_int(self.n_bus), C.c_int(self.n_branch), N.iptr(f),
                                   N.iptr(t), N.iptr(s), C.c_int(self.n_shunt), N.iptr(sb),
                                   C.byref(h)))
        self._h = h
        self.nnz = int(L.gapk_ybus_nnz(h))
        self.row_ptr = np.zeros(self.n_bus + 1, np.int32)
        self.col_idx = np.zeros(self.nnz, np.int32)
        N.check(L.gapk_ybus_pattern(h, N.iptr(self.row_ptr), N.iptr(self.col_idx)))

    @staticmethod
    def from_network(net: Network) -> "YbusPlan":
        f, t, valid = net.branch_index()
        sb, _, _ = net.shunt_index()
        return YbusPlan(net.n_bus, np.where(valid, f, 0), np.where(valid, t, 0),
                        valid.astype(np.int32), sb)

    def assemble(self, branch, shunt=None, mode=N.YBUS_REFERENCE, scale=1.0, stream=None):
        """branch: cuda float64 [m, 6] or [S, m, 6] = (r1, x1, g1, b1, k, theta);
        shunt: [n_shunt, 2] or [S, n_shunt, 2] = (g1, b1).  Returns complex128 [S, nnz]
        (S = 1 for unbatched input)."""
        torch = _torch()
        br = branch.contiguous()
        S = br.shape[0] if br.dim() == 3 else 1
        bst = self.n_branch * 6 if br.dim() == 3 else 0
        if shunt is None:
            shunt = torch.zeros((max(self.n_shunt, 1), 2), dtype=torch.float64, device=br.device)
        sh = shunt.contiguous()
        sst = self.n_shunt * 2 if sh.dim() == 3 else 0
        out = torch.empty((S, self.nnz), dtype=torch.complex128, device=br.device)
        N.check(N.lib().gapk_ybus_assemble(self._h, S, _dptr(br), bst, _dptr(sh), sst, mode,
                                           float(scale), _dptr(out), self.nnz,
                                           _stream_ptr(stream)))
        return out

    def branch_positions(self) -> np.ndarray:
        """[n_branch, 4] int32: the CSR indices of each in-service branch's own stamps
        (diagonal from, diagonal to, (from, to), (to, from)); -1 rows for out-of-service
        branches.  The pattern keeps the duplicates of parallel branches, in branch order
        (src/admittance/cpu/cpu_admittance_matrix.cpp:151-186), so the k-th branch joining
        two buses owns the k-th duplicate of their off-diagonal entries."""
        rp, ci = self.row_ptr, self.col_idx
        out = np.full((self.n_branch, 4), -1, np.int32)
        diag = np.full(self.n_bus, -1, np.int64)
        rows = np.repeat(np.arange(self.n_bus), np.diff(rp))
        d = np.nonzero(ci == rows)[0]
        diag[rows[d][::-1]] = d[::-1]  # first diagonal entry of each row
        seen = {}
        for b in range(self.n_branch):
            if not self.in_service[b]:
                continue
            f, t = int(self.from_idx[b]), int(self.to_idx[b])
            if f == t:
                raise ValueError(f"branch {b} connects bus {f} to itself")
            out[b, 0], out[b, 1] = diag[f], diag[t]
            for role, (r, c) in ((2, (f, t)), (3, (t, f))):
                k = seen.get((r, c), 0)
                seen[(r, c)] = k + 1
                hits = rp[r] + np.nonzero(ci[rp[r]:rp[r + 1]] == c)[0]
                out[b, role] = hits[k]
        return out

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_ybus_destroy(self._h)
                self._h = None
        except Exception:
            pass


class YbusDelta:
    """Branch status changes for a batch of scenarios on one Y pattern, applied on the device
    one thread per touched entry (gapk_ybus_delta_*; the reference applies one change list
    sequentially, src/admittance/cpu/cpu_admittance_matrix.cpp:204-301).

    changes: one list of branch indices per scenario.  positions: [n_branch, 4] CSR indices
    per branch (default: each branch's own entries, YbusPlan.branch_positions)."""

    MODES = {"reference": N.DELTA_REFERENCE, "fixed": N.DELTA_FIXED,
             "fixed_taps": N.DELTA_FIXED_TAPS}

    def __init__(self, yplan: YbusPlan, changes, positions=None):
        pos = yplan.branch_positions() if positions is None else np.asarray(positions, np.int32)
        self.branches = [np.asarray(c, np.int64).reshape(-1) for c in changes]
        self.n_scen = len(self.branches)
        ptr = np.zeros(self.n_scen + 1, np.int32)
        ptr[1:] = np.cumsum([len(c) for c in self.branches])
        flat = np.concatenate(self.branches) if ptr[-1] else np.zeros(0, np.int64)
        self.change_branch = flat
        hp = N.i32(pos[flat].reshape(-1)) if len(flat) else np.zeros(4, np.int32)
        h = C.c_void_p()
        N.check(N.lib().gapk_ybus_delta_create(C.c_int(self.n_scen), N.iptr(ptr), N.iptr(hp),
                                               C.byref(h)))
        self._h = h
        self.nnz = yplan.nnz

    def params(self, branch: np.ndarray, status) -> np.ndarray:
        """[n_changes, 7] (r1, x1, g1, b1, k, theta, status) from branch_params rows and the
        new status per change (scalar or [n_changes])."""
        prm = np.zeros((len(self.change_branch), 7))
        prm[:, :6] = np.asarray(branch)[self.change_branch]
        prm[:, 6] = status
        return prm

    def apply(self, values, params, mode="fixed_taps", scale=1.0, stream=None):
        """values: complex128 [n_scen, nnz] on the device, changed in place; params: float64
        [n_changes, 7] (device tensor or host array)."""
        torch = _torch()
        prm = torch.as_tensor(np.asarray(params, np.float64) if not torch.is_tensor(params)
                              else params, device=values.device).contiguous()
        N.check(N.lib().gapk_ybus_delta_apply(self._h, _dptr(prm), self.MODES[mode],
                                              float(scale), _dptr(values),
                                              values.stride(0) if values.dim() == 2 else 0,
                                              _stream_ptr(stream)))
        return values

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_ybus_delta_destroy(self._h)
                self._h = None
        except Exception:
            pass


def branch_params(net: Network) -> np.ndarray:
    """[m, 6] float64 = (r1, x1, g1, b1, k, theta) per branch, in the network's units."""
    return np.stack([net.r1, net.x1, net.g1, net.b1, net.k, net.theta], axis=1).astype(np.float64)


def shunt_params(net: Network) -> np.ndarray:
    sb, g, b = net.shunt_index()
    if len(sb) == 0:
        return np.zeros((1, 2))
    return np.stack([np.asarray(g, np.float64), np.asarray(b, np.float64)], axis=1)


BRANCH_RESULT_FIELDS = ("p_from", "q_from", "i_from", "s_from", "p_to", "q_to", "i_to", "s_to",
                        "loading")


def branch_flows(net: Network, v, base_power, taps=True, i_n=None, sn=None, branch=None,
                 stream=None):
    """Branch results on the device (gapk_branch_flows): v complex128 per-unit voltages
    [S, n_bus] (cuda); branch (r1, x1, g1, b1, k, theta) [m, 6] or [S, m, 6] (cuda, default the
    network's own).  Returns float64 [S, m, 9] in BRANCH_RESULT_FIELDS order (W, var, A, VA,
    loading); out-of-service branches give zero rows."""
    torch = _torch()
    v = v.contiguous()
    S = v.shape[0]
    f, t, valid = net.branch_index()
    dev = v.device
    fi = torch.as_tensor(np.where(valid, f, -1).astype(np.int32), device=dev)
    ti = torch.as_tensor(np.where(valid, t, -1).astype(np.int32), device=dev)
    br = (torch.as_tensor(branch_params(net), device=dev) if branch is None else branch).contiguous()
    bst = net.n_branch * 6 if br.dim() == 3 else 0
    inn = None if i_n is None else torch.as_tensor(np.asarray(i_n, np.float64), device=dev)
    snn = None if sn is None else torch.as_tensor(np.asarray(sn, np.float64), device=dev)
    out = torch.zeros((S, net.n_branch, 9), dtype=torch.float64, device=dev)
    N.check(N.lib().gapk_branch_flows(S, net.n_bus, net.n_branch, _dptr(fi), _dptr(ti),
                                      _dptr(br), bst, _dptr(v), float(base_power),
                                      float(net.u_rated[0]), _dptr(inn), _dptr(snn),
                                      N.YBUS_TAPS if taps else N.YBUS_REFERENCE, _dptr(out),
                                      _stream_ptr(stream)))
    return out


# ----------------------------------------------------------------------------------------
# Newton-Raphson
# ----------------------------------------------------------------------------------------

_EXPORT = dict(bus_of_node=0, node_pq=1, lptr=2, lidx=3, level_ptr=4, level_nodes=5,
               slot_info=6, slot_src_ptr=7, slot_src=8, fa_ptr=9, targets=10, pairs=11,
               fb_ptr=12, scale=13, rptr=14, rlist=15, var_of_comp=16, eq_of_comp=17,
               slot_a=18, arow_ptr=19, arow=20, schur=21)


class NRPlan:
    """Symbolic analysis of one (Y pattern, bus types) pair; shared by every batch and every
    scenario with that pattern.  Host-only until a batch uploads it."""

    def __init__(self, row_ptr, col_idx, bus_type, jacobian="reference", ordering="mindeg",
                 dense_min=0):
        L = N.lib()
        rp = N.i32(row_ptr)
        ci = N.i32(col_idx)
        bt = N.i32(bus_type)
        opt = N.PlanOptions(N.JAC_REFERENCE if jacobian == "reference" else N.JAC_EXACT,
                            N.ORDER_MINDEG if ordering == "mindeg" else N.ORDER_NATURAL,
                            int(dense_min))
        h = C.c_void_p()
        N.check(L.gapk_nr_plan_create(C.c_int(len(rp) - 1), C.c_int(len(ci)), N.iptr(rp),
                                      N.iptr(ci), N.iptr(bt), C.byref(opt), C.byref(h)))
        self._h = h
        self.row_ptr, self.col_idx, self.bus_type = rp, ci, bt
        info = N.PlanInfo()
        N.check(L.gapk_nr_plan_get_info(h, C.byref(info)))
        self.info = info.as_dict()

    def export(self, name):
        L = N.lib()
        w = _EXPORT[name]
        n = L.gapk_nr_plan_export(self._h, w, None)
        if n < 0:
            N.check(int(n))
        buf = np.zeros(max(int(n), 1), np.int32)
        L.gapk_nr_plan_export(self._h, w, N.iptr(buf))
        return buf[: int(n)]

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_nr_plan_destroy(self._h)
                self._h = None
        except Exception:
            pass


@dataclass
class NRResult:
    v: "object"            # complex128 [S, n_bus] (torch, cuda)
    iterations: "object"   # int32 [S]
    status: "object"       # int32 [S]
    final_mismatch: "object"  # float64 [S]

    @property
    def converged(self):
        return self.status == N.SCEN_CONVERGED


class NRBatch:
    """Device state for n_scen scenarios sharing one NRPlan."""

    def __init__(self, plan: NRPlan, n_scen: int, precision="fp64", y_shared=True, lanes=0,
                 threads=0, use_graph=True, dense_fused=False, dense_fma=False):
        require_cuda()
        self.plan = plan
        self.n_scen = int(n_scen)
        self.precision = precision
        self.y_shared = bool(y_shared)
        opt = N.BatchOptions(N.PREC_FP64 if precision == "fp64" else N.PREC_FP32,
                             1 if y_shared else 0, int(lanes), int(threads),
                             1 if use_graph else 0, 1 if dense_fused else 0,
                             1 if dense_fma else 0)
        h = C.c_void_p()
        N.check(N.lib().gapk_nr_batch_create(plan._h, C.c_int(self.n_scen), C.byref(opt),
                                             C.byref(h)))
        self._h = h

    @property
    def device_bytes(self):
        return int(N.lib().gapk_nr_batch_device_bytes(self._h))

    def device_error(self) -> bool:
        """True when a bounded wait of the tensor-core dense LU ran out during the last solve
        (its scenarios end SINGULAR); waits for the device."""
        rc = int(N.lib().gapk_nr_batch_device_error(self._h))
        if rc < 0:
            N.check(rc)
        return rc == 1

    def set_wait_test(self, skip: bool):
        """Test hook: with skip the tensor-core dense LU issues no MMAs, so that its bounded
        waits run out (gapk_nr_batch_set_wait_test)."""
        N.check(N.lib().gapk_nr_batch_set_wait_test(self._h, C.c_int(1 if skip else 0)))

    def _inputs(self, y, s_spec, v_init, u_pu, tol, max_iter, policy, refine, refine_below=0.0,
                reuse_below=0.0):
        pol = {"reference": N.POLICY_REFERENCE, "newton": N.POLICY_NEWTON,
               "clamped": N.POLICY_CLAMPED}[policy]
        shared = 1 if v_init is not None and v_init.dim() == 1 else 0
        return N.Inputs(_dptr(y), _dptr(s_spec), _dptr(v_init), _dptr(u_pu), float(tol),
                        int(max_iter), pol, int(refine), float(refine_below),
                        float(reuse_below), shared)

    def solve(self, y, s_spec, v_init=None, u_pu=None, tol=1e-8, max_iter=20,
              policy="reference", refine=0, out=None, stream=None,
              refine_below=0.0, reuse_below=0.0) -> NRResult:
        """y: complex128 per-unit Y values, [nnz] (y_shared) or [S, nnz]; s_spec: complex128
        [S, n_bus]; v_init: complex128 [S, n_bus], [n_bus] (one start for every scenario) or
        None (flat start); u_pu: float64
        [n_bus] flat-start |V| of SLACK/PV buses.  refine_below > 0 runs the `refine`
        refinement steps only in iterations where a scenario of the lane group has max
        |mismatch| below it.  reuse_below > 0 keeps a group's previous LU factors once all
        its iterating scenarios are below it (the refined solve then corrects against the
        current Jacobian; needs refine >= 1)."""
        torch = _torch()
        n = self.plan.info["n_bus"]
        dev = s_spec.device
        if out is None:
            out = NRResult(torch.empty((self.n_scen, n), dtype=torch.complex128, device=dev),
                           torch.empty(self.n_scen, dtype=torch.int32, device=dev),
                           torch.empty(self.n_scen, dtype=torch.int32, device=dev),
                           torch.empty(self.n_scen, dtype=torch.float64, device=dev))
        inp = self._inputs(y, s_spec, v_init, u_pu, tol, max_iter, policy, refine, refine_below,
                           reuse_below)
        o = N.Outputs(_dptr(out.v), _dptr(out.iterations), _dptr(out.status),
                      _dptr(out.final_mismatch))
        N.check(N.lib().gapk_nr_solve(self._h, C.byref(inp), C.byref(o), _stream_ptr(stream)))
        return out

    def solve_captured(self, y, s_spec, v_init=None, u_pu=None, tol=1e-8, max_iter=20,
                       policy="reference", refine=0, stream=None, refine_below=0.0,
                       reuse_below=0.0):
        """solve() stepped one iteration at a time, recording per iteration what
        IPowerFlowSolver's state capture records (powerflow_interface.h:28-35,
        gpu_newton_raphson.cu:452-490): the voltages that iteration's mismatch is taken at,
        I = Y V, S = V conj(I) (complex128 [S, n_bus], per unit), the mismatch in the
        reference's equation order ([S, n_vars]) and its max |.| per scenario.  The trajectory
        is solve()'s.  Returns (NRResult, list of dicts with keys iteration, v, i, s,
        mismatch, max_mismatch)."""
        torch = _torch()
        n = self.plan.info["n_bus"]
        dev = s_spec.device
        sp = _stream_ptr(stream)
        inp = self._inputs(y, s_spec, v_init, u_pu, tol, max_iter, policy, refine, refine_below,
                           reuse_below)
        N.check(N.lib().gapk_nr_stage_load(self._h, C.byref(inp), sp))
        states = []
        active = C.c_int(0)
        for it in range(int(max_iter)):
            v, i, s = (torch.empty((self.n_scen, n), dtype=torch.complex128, device=dev)
                       for _ in range(3))
            N.check(N.lib().gapk_nr_get_state(self._h, _dptr(v), _dptr(i), _dptr(s), sp))
            N.check(N.lib().gapk_nr_step(self._h, C.byref(active), sp))
            f = self.mismatch(stream)
            states.append(dict(iteration=it, v=v, i=i, s=s, mismatch=f,
                               max_mismatch=f.abs().amax(dim=1) if f.shape[1] else
                               torch.zeros(self.n_scen, dtype=torch.float64, device=dev)))
            if not active.value:
                break
        out = NRResult(torch.empty((self.n_scen, n), dtype=torch.complex128, device=dev),
                       torch.empty(self.n_scen, dtype=torch.int32, device=dev),
                       torch.empty(self.n_scen, dtype=torch.int32, device=dev),
                       torch.empty(self.n_scen, dtype=torch.float64, device=dev))
        o = N.Outputs(_dptr(out.v), _dptr(out.iterations), _dptr(out.status),
                      _dptr(out.final_mismatch))
        N.check(N.lib().gapk_nr_get_outputs(self._h, C.byref(o), sp))
        return out, states

    # stage access (tests, profiling)
    def stage_load(self, y, s_spec, v_init=None, u_pu=None, refine=0, stream=None,
                   policy="newton"):
        inp = self._inputs(y, s_spec, v_init, u_pu, 0.0, 1, policy, refine)
        N.check(N.lib().gapk_nr_stage_load(self._h, C.byref(inp), _stream_ptr(stream)))

    def stage(self, name, stream=None):
        fn = {"mismatch": "gapk_nr_stage_mismatch", "jacobian": "gapk_nr_stage_jacobian",
              "factor": "gapk_nr_stage_factor", "solve": "gapk_nr_stage_solve"}[name]
        N.check(getattr(N.lib(), fn)(self._h, _stream_ptr(stream)))

    KERNELS = ("mismatch", "jacobian", "factor_sparse", "schur", "dense_lu", "solve_fwd",
               "dense_solve", "solve_bwd", "update", "residual")

    def kernel(self, name, stream=None):
        """Launch one kernel of the loop body (timing / profiling)."""
        N.check(N.lib().gapk_nr_stage_kernel(self._h, self.KERNELS.index(name),
                                             _stream_ptr(stream)))

    def state(self, stream=None):
        """The batch's current state (after solve(): the solution), per unit, complex128
        [n_scen, n_bus] each: V, the current injections I = Y V and the power injections
        S = V conj(I) (gapk_nr_get_state)."""
        torch = _torch()
        n = self.plan.info["n_bus"]
        v, i, s = (torch.empty((self.n_scen, n), dtype=torch.complex128, device="cuda")
                   for _ in range(3))
        N.check(N.lib().gapk_nr_get_state(self._h, _dptr(v), _dptr(i), _dptr(s),
                                          _stream_ptr(stream)))
        return v, i, s

    def level_trace(self, y, s_spec, v_init=None, u_pu=None, stream=None):
        """Per-level latency of the level-scheduled kernels at the state (y, s_spec, v_init):
        one mismatch and Jacobian, then the sparse factorisation, Schur gather, dense LU and
        the three solves, each launched once with the level trace on
        (gapk_nr_set_level_trace).  Returns, per kernel ("factor", "forward", "backward"),
        dict(stamps = %globaltimer ns [n_groups, n_levels + 2], level_us = duration of each
        level in execution order [n_groups, n_levels], total_us [n_groups]); and, when the
        one-CTA-per-scenario dense LU runs, "dense": dict(stamps [n_scen, 1 + 3 * panels],
        phase_us [n_scen, panels, 3] = diagonal block, L21/U12 solves, trailing update)."""
        torch = _torch()
        L = N.lib()
        n = int(L.gapk_nr_level_trace_size(self._h))
        buf = torch.zeros(n, dtype=torch.int64, device=s_spec.device)
        self.stage_load(y, s_spec, v_init=v_init, u_pu=u_pu, stream=stream)
        self.kernel("mismatch", stream)
        self.kernel("jacobian", stream)
        N.check(L.gapk_nr_set_level_trace(self._h, _dptr(buf), n))
        try:
            for k in ("factor_sparse", "schur", "dense_lu", "solve_fwd", "dense_solve",
                      "solve_bwd"):
                self.kernel(k, stream)
            torch.cuda.synchronize()
        finally:
            N.check(L.gapk_nr_set_level_trace(self._h, None, 0))
        lv = self.plan.info["n_levels"]
        host = buf.cpu().numpy()
        ns = 3 * (n_groups := self._groups()) * (lv + 2)
        ts = host[:ns].reshape(3, n_groups, lv + 2)
        out = {name: dict(stamps=ts[i], level_us=np.diff(ts[i][:, :lv + 1], axis=1) / 1e3,
                          total_us=(ts[i][:, -1] - ts[i][:, 0]) / 1e3)
               for i, name in enumerate(("factor", "forward", "backward"))}
        npan = int(L.gapk_nr_dense_trace_panels(self._h))
        if npan:
            d = host[ns:].reshape(-1, 1 + 3 * npan)[:self.n_scen]
            out["dense"] = dict(stamps=d, phase_us=np.diff(d, axis=1).reshape(-1, npan, 3) / 1e3)
        return out

    def _groups(self):
        """Lane groups of the batch: ceil(n_scen / lanes)."""
        sw = int(N.lib().gapk_nr_batch_lanes(self._h))
        return -(-self.n_scen // sw)

    def correction(self, stream=None):
        torch = _torch()
        nv = self.plan.info["n_vars"]
        out = torch.zeros((self.n_scen, nv), dtype=torch.float64, device="cuda")
        N.check(N.lib().gapk_nr_stage_get_correction(self._h, _dptr(out), _stream_ptr(stream)))
        return out

    def mismatch(self, stream=None):
        torch = _torch()
        nv = self.plan.info["n_vars"]
        out = torch.zeros((self.n_scen, nv), dtype=torch.float64, device="cuda")
        N.check(N.lib().gapk_nr_stage_get_mismatch(self._h, _dptr(out), _stream_ptr(stream)))
        return out

    def loop_count(self, stream=None):
        v = C.c_int(0)
        N.check(N.lib().gapk_nr_last_loop_count(self._h, _stream_ptr(stream), C.byref(v)))
        return v.value

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_nr_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass


class NRMix:
    """Batches of any plans solved together by ONE graph launch (gapk_nr_mix_*): each batch's
    whole solve is one branch of a single CUDA graph, the branches run concurrently, and with
    `retry` the scenarios that end unconverged restart from their start vector under that step
    policy inside the same launch.  The graph is built on the first solve and reused while the
    input tensors and options stay the same; results land in the same tensors every time
    (self.results)."""

    def __init__(self, batches):
        require_cuda()
        self.batches = list(batches)
        arr = (C.c_void_p * len(self.batches))(*[b._h.value for b in self.batches])
        h = C.c_void_p()
        N.check(N.lib().gapk_nr_mix_create(len(self.batches), arr, C.byref(h)))
        self._h = h
        torch = _torch()
        self.results = []
        for b in self.batches:
            n = b.plan.info["n_bus"]
            self.results.append(NRResult(
                torch.empty((b.n_scen, n), dtype=torch.complex128, device="cuda"),
                torch.empty(b.n_scen, dtype=torch.int32, device="cuda"),
                torch.empty(b.n_scen, dtype=torch.int32, device="cuda"),
                torch.empty(b.n_scen, dtype=torch.float64, device="cuda")))

    def solve(self, ys, s_specs, v_inits=None, u_pus=None, tol=1e-8, max_iter=20,
              policy="newton", refine=0, refine_below=0.0, reuse_below=0.0, retry=None,
              stream=None):
        """ys / s_specs / v_inits / u_pus: one entry per batch, as NRBatch.solve takes them
        (keep the same tensors between calls to reuse the graph); retry: None or a step policy
        name.  Returns self.results (NRResult per batch), written asynchronously on the
        stream."""
        nb = len(self.batches)
        v_inits = v_inits if v_inits is not None else [None] * nb
        u_pus = u_pus if u_pus is not None else [None] * nb
        ins = (N.Inputs * nb)(*[b._inputs(y, s, v, u, tol, max_iter, policy, refine,
                                          refine_below, reuse_below)
                                for b, y, s, v, u in zip(self.batches, ys, s_specs, v_inits,
                                                         u_pus)])
        outs = (N.Outputs * nb)(*[N.Outputs(_dptr(r.v), _dptr(r.iterations), _dptr(r.status),
                                            _dptr(r.final_mismatch)) for r in self.results])
        pol = -1 if retry is None else {"reference": N.POLICY_REFERENCE,
                                        "newton": N.POLICY_NEWTON,
                                        "clamped": N.POLICY_CLAMPED}[retry]
        self._keep = (ys, s_specs, v_inits, u_pus)
        N.check(N.lib().gapk_nr_mix_solve(self._h, ins, outs, pol, _stream_ptr(stream)))
        return self.results

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_nr_mix_destroy(self._h)
                self._h = None
        except Exception:
            pass


class HostPipeline:
    """Batched solves from and to host memory with the copies overlapped: the scenarios are
    split into `chunks` contiguous parts (multiples of the lane count), each with its own
    NRBatch and CUDA stream, so the device solves one part while the next part's inputs and the
    previous part's results cross PCIe.  Host tensors should be pinned for the copies to be
    asynchronous."""

    def __init__(self, plan: NRPlan, n_scen: int, chunks=2, precision="fp32", lanes=8,
                 threads=1024):
        torch = _torch()
        require_cuda()
        n_scen = int(n_scen)
        chunks = max(1, min(int(chunks), n_scen))
        step = -(-n_scen // chunks)
        step = -(-step // max(1, lanes)) * max(1, lanes)
        self.ranges = [(a, min(a + step, n_scen)) for a in range(0, n_scen, step)]
        # the parts run concurrently and together fill the GPU: each keeps the
        # one-CTA-per-scenario dense LU even when it alone would not
        self.batches = [NRBatch(plan, b - a, precision=precision, lanes=lanes, threads=threads,
                                dense_fused=len(self.ranges) > 1)
                        for a, b in self.ranges]
        self.streams = [torch.cuda.Stream() for _ in self.ranges]
        self.plan = plan
        self.n_scen = n_scen

    def solve(self, y, s_host, v_host, out_v, out_status=None, out_iterations=None,
              out_mismatch=None, **kw):
        """y: device per-unit Y [nnz]; s_host: host complex128 [S, n_bus]; v_host: host
        complex128 [S, n_bus], or [n_bus] for one start vector shared by every scenario (copied
        once per part); results into the host tensors out_v [S, n_bus] (and optionally status,
        iterations, final mismatch [S]).  Returns after every part's results are on the
        host."""
        torch = _torch()
        cur = torch.cuda.current_stream()
        for st in self.streams:
            st.wait_stream(cur)
        for (a, b), bt, st in zip(self.ranges, self.batches, self.streams):
            with torch.cuda.stream(st):
                sd = s_host[a:b].to("cuda", non_blocking=True)
                vd = (v_host if v_host.dim() == 1 else v_host[a:b]).to("cuda", non_blocking=True)
                r = bt.solve(y, sd, v_init=vd, stream=st, **kw)
                out_v[a:b].copy_(r.v, non_blocking=True)
                for host, dev in ((out_status, r.status), (out_iterations, r.iterations),
                                  (out_mismatch, r.final_mismatch)):
                    if host is not None:
                        host[a:b].copy_(dev, non_blocking=True)
        for st in self.streams:
            st.synchronize()


# ----------------------------------------------------------------------------------------
# General sparse LU
# ----------------------------------------------------------------------------------------


class SparseLU:
    """Complex square sparse LU on the device (ILUSolver, include/gap/solver/
    lu_solver_interface.h:21-35): host analysis once per pattern, device factorisation with
    static pivoting (after a zero-free-diagonal row matching) and device solves."""

    def __init__(self, row_ptr, col_idx):
        rp = N.i32(row_ptr)
        ci = N.i32(col_idx)
        h = C.c_void_p()
        N.check(N.lib().gapk_splu_create(C.c_int(len(rp) - 1), C.c_int(len(ci)), N.iptr(rp),
                                         N.iptr(ci), C.byref(h)))
        self._h = h
        self.n = int(N.lib().gapk_splu_size(h))

    def factorize(self, values, stream=None) -> bool:
        """values: complex128 [nnz] on the device.  False when a pivot is (numerically)
        zero; other failures raise."""
        require_cuda()
        rc = N.lib().gapk_splu_factorize(self._h, _dptr(values), _stream_ptr(stream))
        if rc == -5:
            return False
        N.check(rc)
        return True

    def solve(self, rhs, stream=None):
        torch = _torch()
        x = torch.empty_like(rhs)
        N.check(N.lib().gapk_splu_solve(self._h, _dptr(rhs), _dptr(x), _stream_ptr(stream)))
        return x

    def __del__(self):
        try:
            if self._h:
                N.lib().gapk_splu_destroy(self._h)
                self._h = None
        except Exception:
            pass
