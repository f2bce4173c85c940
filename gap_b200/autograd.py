"""Differentiable batched power flow (no counterpart in the reference).

`DifferentiablePowerFlow(net, n_scen)(p, q, r, x) -> (vm, va)` solves n_scen scenarios on the
device and is a `torch.autograd` function of the per-bus specified injections (p, q per unit,
[n_scen, n_bus]) and the branch resistances / reactances (r, x in Ohm, [n_branch], shared by
the scenarios).  The backward pass is the adjoint of the converged state: the device
refactorises the exact Jacobian at the solution and solves J^T lambda = dL/dx with the same
block factors (gapk_nr_adjoint), then contracts lambda with dF/d(r, x) branch by branch
(gapk_nr_adjoint_branch).  Gradients are those of the solution map, so they do not depend on
the Newton step policy used to get there.

`branch_losses_mw(vm, va, r, x, model)` gives the branch real-power losses as a torch function
of the same quantities, for losses that depend on the branch parameters directly.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from .engine import NRBatch, NRPlan, YbusPlan, _dptr, _stream_ptr, branch_params, shunt_params
from .network import Network


class DifferentiablePowerFlow:
    def __init__(self, net: Network, n_scen: int, base_power: float = 1e8,
                 precision: str = "fp64", taps: bool = True, tol: float = 1e-10,
                 max_iter: int = 30, v_init=None, lanes: int = 0):
        self.net = net
        self.n_scen = int(n_scen)
        self.base_power = float(base_power)
        self.zb = float(net.u_rated[0]) ** 2 / self.base_power
        self.tol = tol
        self.max_iter = max_iter
        self.precision = precision
        self.mode = N.YBUS_TAPS if taps else N.YBUS_REFERENCE
        self.yp = YbusPlan.from_network(net)
        self.plan = NRPlan(self.yp.row_ptr, self.yp.col_idx, net.bus_type, jacobian="exact")
        self.batch = NRBatch(self.plan, self.n_scen, precision=precision, lanes=lanes)
        dev = "cuda"
        self.branch = torch.as_tensor(branch_params(net), device=dev)
        self.shunt = torch.as_tensor(shunt_params(net), device=dev)
        f, t, valid = net.branch_index()
        self.from_idx = torch.as_tensor(np.where(valid, f, -1).astype(np.int32), device=dev)
        self.to_idx = torch.as_tensor(np.where(valid, t, -1).astype(np.int32), device=dev)
        self.valid = torch.as_tensor(valid, device=dev)
        if v_init is None:
            from .synth import dc_start

            v_init = dc_start(net, self.base_power)
        v = np.asarray(v_init, np.complex128)
        if v.ndim == 1:
            v = np.repeat(v[None], self.n_scen, axis=0)
        self.v0 = torch.as_tensor(v, device=dev)

    def branch_tensor(self, r, x):
        br = self.branch.clone()
        br[:, 0] = r
        br[:, 1] = x
        return br

    def __call__(self, p, q, r=None, x=None):
        if r is None:
            r = self.branch[:, 0].clone()
        if x is None:
            x = self.branch[:, 1].clone()
        return _PowerFlowFn.apply(p, q, r, x, self)


class _PowerFlowFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p, q, r, x, model):
        br = model.branch_tensor(r, x)
        y = model.yp.assemble(br, model.shunt, mode=model.mode, scale=model.zb)[0]
        s = torch.complex(p.contiguous(), q.contiguous())
        refine = 1 if model.precision == "fp32" else 0
        res = model.batch.solve(y, s, v_init=model.v0, tol=model.tol, max_iter=model.max_iter,
                                policy="newton", refine=refine)
        st = res.status.cpu().numpy()
        if (st != N.SCEN_CONVERGED).any():
            raise RuntimeError(f"power flow did not converge for scenarios "
                               f"{np.nonzero(st != 0)[0].tolist()[:8]}")
        v = res.v
        ctx.save_for_backward(v, y, s, r, x)
        ctx.model = model
        return v.abs(), v.angle()

    @staticmethod
    def backward(ctx, gvm, gva):
        v, y, s, r, x = ctx.saved_tensors
        model = ctx.model
        b = model.batch
        S, n = v.shape
        gvm = torch.zeros((S, n), dtype=torch.float64, device=v.device) if gvm is None \
            else gvm.contiguous().to(torch.float64)
        gva = torch.zeros((S, n), dtype=torch.float64, device=v.device) if gva is None \
            else gva.contiguous().to(torch.float64)
        b.stage_load(y, s, v_init=v.contiguous(), refine=1 if model.precision == "fp32" else 0)
        dp = torch.empty((S, n), dtype=torch.float64, device=v.device)
        dq = torch.empty_like(dp)
        L = N.lib()
        N.check(L.gapk_nr_adjoint(b._h, _dptr(gvm), _dptr(gva), _dptr(dp), _dptr(dq),
                                  _stream_ptr()))
        gr = gx = None
        if ctx.needs_input_grad[2] or ctx.needs_input_grad[3]:
            m = model.branch.shape[0]
            brp = model.branch_tensor(r, x).clone()
            brp[:, 0] = brp[:, 0] / model.zb
            brp[:, 1] = brp[:, 1] / model.zb
            brp[:, 2] = brp[:, 2] * model.zb
            brp[:, 3] = brp[:, 3] * model.zb
            if model.mode == N.YBUS_REFERENCE:
                brp[:, 4] = 1.0
                brp[:, 5] = 0.0
            brp = brp.contiguous()
            dr = torch.empty((S, m), dtype=torch.float64, device=v.device)
            dxx = torch.empty_like(dr)
            N.check(L.gapk_nr_adjoint_branch(b._h, C.c_int(m), _dptr(model.from_idx),
                                             _dptr(model.to_idx), _dptr(brp), _dptr(dr),
                                             _dptr(dxx), _stream_ptr()))
            # per unit -> Ohm: r_pu = r / Z_base
            gr = dr.sum(0) / model.zb
            gx = dxx.sum(0) / model.zb
        return dp, dq, gr, gx, None



def branch_losses_mw(vm, va, r, x, model: DifferentiablePowerFlow):
    """Real-power loss of every in-service branch, Re(S_from + S_to), in MW, as a torch
    function of the solution (vm, va: [S, n]) and the branch parameters (r, x in Ohm).
    Stamps as the Y-bus builder's pi model (taps unless the model was built without)."""
    zb = model.zb
    br = model.branch_tensor(r, x)
    keep = model.valid
    f = model.from_idx[keep].long()
    t = model.to_idx[keep].long()
    rp = br[keep, 0] / zb
    xp = br[keep, 1] / zb
    y = 1.0 / torch.complex(rp, xp)
    ysh = torch.complex(br[keep, 2] * zb, br[keep, 3] * zb / 2.0)
    if model.mode == N.YBUS_TAPS:
        tap = torch.polar(br[keep, 4], br[keep, 5])
    else:
        tap = torch.ones_like(y)
    yff = (y + ysh) / (tap.abs() ** 2)
    ytt = y + ysh
    yft = -y / tap.conj()
    ytf = -y / tap
    v = torch.polar(vm, va)
    vf, vt = v[:, f], v[:, t]
    i_f = yff * vf + yft * vt
    i_t = ytf * vf + ytt * vt
    loss = (vf * i_f.conj() + vt * i_t.conj()).real
    return loss * (model.base_power / 1e6)
