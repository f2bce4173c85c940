"""Adjoint gradients through the converged power flow (gap_b200.autograd) against the
oracle's FP64 implicit-function gradient and central finite differences.

Loss (the C4 workload's): L = sum_bus (|V|-1)^2 + sum_branch P_loss[MW].  Relative error
criterion per coordinate: |g - g_ref| <= 1e-6 * max(|g_ref|, 1e-3 * max|g_ref|)."""

import numpy as np
import pytest

from oracle import restate

pytestmark = pytest.mark.gpu
REL = 1e-6


def _rel_ok(g, ref, rel=REL):
    g = np.asarray(g)
    ref = np.asarray(ref)
    floor = 1e-3 * np.max(np.abs(ref))
    err = np.abs(g - ref) / np.maximum(np.abs(ref), floor)
    return float(np.max(err))


def _setup(n=300, S=3, precision="fp64", seed=6, tol=1e-11):
    import torch

    from gap_b200 import synth
    from gap_b200.autograd import DifferentiablePowerFlow

    net = synth.transmission_grid(seed, n=n)
    base = 1e8
    s = synth.load_scenarios(net, S, sigma=0.1, seed=seed, base_power=base)
    model = DifferentiablePowerFlow(net, S, base_power=base, precision=precision, tol=tol)
    p = torch.tensor(s.real, device="cuda", requires_grad=True)
    q = torch.tensor(s.imag, device="cuda", requires_grad=True)
    r = model.branch[:, 0].clone().requires_grad_(True)
    x = model.branch[:, 1].clone().requires_grad_(True)
    return net, s, model, p, q, r, x


def _loss(model, p, q, r, x):
    from gap_b200.autograd import branch_losses_mw

    vm, va = model(p, q, r, x)
    return ((vm - 1.0) ** 2).sum() + branch_losses_mw(vm, va, r, x, model).sum(), vm, va


def test_adjoint_matches_fp64_implicit_function_gradient():
    net, s, model, p, q, r, x = _setup()
    L, vm, va = _loss(model, p, q, r, x)
    L.backward()
    v = (vm.detach() * __import__("torch").exp(1j * va.detach())).cpu().numpy()
    dr_tot = np.zeros(net.n_branch)
    dx_tot = np.zeros(net.n_branch)
    for k in range(s.shape[0]):
        o = restate.adjoint_gradients(net, v[k], base_power=model.base_power, taps=True)
        assert _rel_ok(p.grad[k].cpu().numpy(), o["dP"]) < REL
        assert _rel_ok(q.grad[k].cpu().numpy(), o["dQ"]) < REL
        dr_tot += o["dr"]
        dx_tot += o["dx"]
    assert _rel_ok(r.grad.cpu().numpy(), dr_tot) < REL
    assert _rel_ok(x.grad.cpu().numpy(), dx_tot) < REL


def test_adjoint_matches_central_finite_differences():
    """Central differences: h = 1e-6 per unit for P; 1e-4 per unit for Q and 1e-4 of the value
    for r / x, whose gradients are smaller, so that the difference stays above the loss's
    rounding floor: the summed loss is O(10-100) MW, so its ~1e-12 rounding noise over 2h swamps
    small reactive gradients (the FP64 oracle alone shows FD errors ~7e-6 at h = 1e-6 on Q)."""
    import torch

    net, s, model, p, q, r, x = _setup(S=2, seed=8, tol=1e-13)
    L, vm, va = _loss(model, p, q, r, x)
    L.backward()
    rng = np.random.default_rng(0)

    def L_at(args):
        with torch.no_grad():
            return float(_loss(model, *args)[0].item())

    base = [p.detach(), q.detach(), r.detach(), x.detach()]
    nonslack = np.nonzero(net.bus_type != 2)[0]
    pq = np.nonzero(net.bus_type == 0)[0]
    results = {}
    for j, name in enumerate(("p", "q", "r", "x")):
        grad = (p, q, r, x)[j].grad
        gs, fs = [], []
        for _ in range(8 if j < 2 else 6):
            idx = ((int(rng.integers(0, 2)), int(rng.choice(nonslack if j == 0 else pq)))
                   if j < 2 else (int(rng.integers(0, net.n_branch)),))
            h = (1e-6, 1e-4)[j] if j < 2 else 1e-4 * abs(float(base[j][idx]))
            d = torch.zeros_like(base[j])
            d[idx] = h
            plus = list(base)
            minus = list(base)
            plus[j] = base[j] + d
            minus[j] = base[j] - d
            fs.append((L_at(plus) - L_at(minus)) / (2 * h))
            gs.append(float(grad[idx]))
        floor = 1e-3 * float(grad.abs().max())
        err = np.abs(np.array(gs) - np.array(fs)) / np.maximum(np.abs(fs), floor)
        results[name] = float(err.max())
    # the difference quotient's own noise (solves converged to 1e-13 pu, loss rounding) moves
    # the Q estimates by a few 1e-6 with the solve's rounding; the exact check is the
    # implicit-function gradient test above
    assert results["p"] < 1e-6 and results["q"] < 5e-6, results
    assert results["r"] < 1e-5 and results["x"] < 1e-5, results


def test_fp32_factors_with_refinement_match_fp64_gradients():
    import torch

    outs = []
    for prec in ("fp64", "fp32"):
        net, s, model, p, q, r, x = _setup(S=9, precision=prec, seed=10)
        L, vm, va = _loss(model, p, q, r, x)
        L.backward()
        outs.append([t.grad.cpu().numpy() for t in (p, q, r, x)])
    for a, b in zip(*outs):
        assert _rel_ok(b, a) < REL


def test_adjoint_at_transmission_scale():
    """The C4 setting on fewer scenarios: 10k-bus grid, gradients of the same loss against
    the FP64 oracle's implicit-function gradient (1e-6 relative)."""
    import torch

    net, s, model, p, q, r, x = _setup(n=10_000, S=2, seed=0, tol=1e-10)
    L, vm, va = _loss(model, p, q, r, x)
    L.backward()
    v = (vm.detach() * torch.exp(1j * va.detach())).cpu().numpy()
    dr_tot = np.zeros(net.n_branch)
    dx_tot = np.zeros(net.n_branch)
    for k in range(s.shape[0]):
        o = restate.adjoint_gradients(net, v[k], base_power=model.base_power, taps=True)
        assert _rel_ok(p.grad[k].cpu().numpy(), o["dP"]) < REL
        assert _rel_ok(q.grad[k].cpu().numpy(), o["dQ"]) < REL
        dr_tot += o["dr"]
        dx_tot += o["dx"]
    assert _rel_ok(r.grad.cpu().numpy(), dr_tot) < REL
    assert _rel_ok(x.grad.cpu().numpy(), dx_tot) < REL
