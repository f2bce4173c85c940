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
    import torch

    net, s, model, p, q, r, x = _setup(S=2, seed=8, tol=1e-13)
    L, vm, va = _loss(model, p, q, r, x)
    L.backward()
    rng = np.random.default_rng(0)
    h = 1e-6

    def L_at(pp, qq, rr, xx):
        with torch.no_grad():
            return float(_loss(model, pp, qq, rr, xx)[0].item())

    nonslack = np.nonzero(net.bus_type != 2)[0]
    pq = np.nonzero(net.bus_type == 0)[0]
    checks = []
    for _ in range(6):
        k, i = int(rng.integers(0, 2)), int(rng.choice(nonslack))
        dp = torch.zeros_like(p)
        dp[k, i] = h
        fd = (L_at(p.detach() + dp, q.detach(), r.detach(), x.detach())
              - L_at(p.detach() - dp, q.detach(), r.detach(), x.detach())) / (2 * h)
        checks.append((float(p.grad[k, i]), fd))
    for _ in range(5):
        k, i = int(rng.integers(0, 2)), int(rng.choice(pq))
        dq = torch.zeros_like(q)
        dq[k, i] = h
        fd = (L_at(p.detach(), q.detach() + dq, r.detach(), x.detach())
              - L_at(p.detach(), q.detach() - dq, r.detach(), x.detach())) / (2 * h)
        checks.append((float(q.grad[k, i]), fd))
    for which, t in (("r", r), ("x", x)):
        for _ in range(5):
            b = int(rng.integers(0, net.n_branch))
            hb = h * abs(float(t[b]))
            d = torch.zeros_like(t)
            d[b] = hb
            args_p = [p.detach(), q.detach(), r.detach(), x.detach()]
            args_m = [p.detach(), q.detach(), r.detach(), x.detach()]
            j = 2 if which == "r" else 3
            args_p[j] = args_p[j] + d
            args_m[j] = args_m[j] - d
            fd = (L_at(*args_p) - L_at(*args_m)) / (2 * hb)
            checks.append((float(t.grad[b]), fd))
    g = np.array([c[0] for c in checks])
    f = np.array([c[1] for c in checks])
    scale = np.max(np.abs(f))
    err = np.abs(g - f) / np.maximum(np.abs(f), 1e-3 * scale)
    assert np.max(err) < 1e-5, (err, g, f)


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
