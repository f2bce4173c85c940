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


H_PQ, H_R, H_X = 4e-3, 5e-2, 2e-2
UNIT = (1, -1, 2, -2, 4, -4)


def _fd_check(net, s, kw, n_pq, n_rx, seed):
    """Adjoint gradients of L = sum over the scenarios of sum_bus (|V|-1)^2 + sum_branch
    P_loss[MW] against central differences on n_pq P and n_pq Q injections (random scenarios
    and buses) and n_rx r and n_rx x values (random branches, shared by every scenario).

    The difference quotient is extrapolated twice (Richardson), D = (64 D(h) - 20 D(2h) +
    D(4h)) / 45 with D(h) = (L(+h) - L(-h)) / 2h, h = 4e-3 pu for P / Q and 5e-2 (r), 2e-2
    (x) of the value for the branch parameters: its truncation error is O(h^6) (x, which sets
    |z|, is the more nonlinear of the two).  The perturbed solves run a fixed 12 Newton
    iterations (tolerance 0), which takes every scenario to its rounding floor.  The steps are
    large because the loss of a converged solve carries rounding noise that differs from solve
    to solve (the Newton fixed point moves with the last bits of the mismatch, times the
    Jacobian's inverse; ~1e-11 at 10k buses): over 2h = 2e-6 that is ~1e-5 of the gradient,
    ~1e-4 relative for the small reactive and branch gradients, and the batch loss that r and
    x move sums one such noise per scenario.  The plain central difference at h = 1e-6 (no
    extrapolation) is reported beside it.  Returns {kind: (Richardson error, plain error, max
    |gradient|)}, errors relative as _rel_ok measures them."""
    import math

    import torch

    from gap_b200.autograd import DifferentiablePowerFlow, branch_losses_mw

    S = s.shape[0]
    model = DifferentiablePowerFlow(net, S, **kw)

    def losses(m, vm, va, r, x):
        return ((vm - 1.0) ** 2).sum(1) + branch_losses_mw(vm, va, r, x, m).sum(1)

    def losses_at_floor(m, p, q, r, x):
        y = m.yp.assemble(m.branch_tensor(r, x), m.shunt, mode=m.mode, scale=m.zb)[0]
        res = m.batch.solve(y, torch.complex(p.contiguous(), q.contiguous()), v_init=m.v0,
                            tol=0.0, max_iter=12, policy="newton")
        assert (res.final_mismatch < 1e-12).all()
        return losses(m, res.v.abs(), res.v.angle(), r, x).cpu().numpy()

    p = torch.tensor(s.real, device="cuda", requires_grad=True)
    q = torch.tensor(s.imag, device="cuda", requires_grad=True)
    r = model.branch[:, 0].clone().requires_grad_(True)
    x = model.branch[:, 1].clone().requires_grad_(True)
    vm, va = model(p, q, r, x)
    losses(model, vm, va, r, x).sum().backward()
    rng = np.random.default_rng(seed)
    nonslack = np.nonzero(net.bus_type != 2)[0]
    pq = np.nonzero(net.bus_type == 0)[0]
    inservice = np.nonzero(net.branch_index()[2])[0]
    inj = ([("p", int(rng.integers(0, S)), int(rng.choice(nonslack))) for _ in range(n_pq)] +
           [("q", int(rng.integers(0, S)), int(rng.choice(pq))) for _ in range(n_pq)])
    brs = ([("r", int(rng.choice(inservice))) for _ in range(n_rx)] +
           [("x", int(rng.choice(inservice))) for _ in range(n_rx)])

    def step(kind):
        return {"p": H_PQ, "q": H_PQ, "r": H_R, "x": H_X}[kind]

    def steps(kind):
        return [u * step(kind) for u in UNIT] + [1e-6, -1e-6]

    fd, fd_plain, ad, kinds = [], [], [], []

    def record(kind, L8, scale, grad):
        H = step(kind)
        d1 = (L8[0] - L8[1]) / (2 * H * scale)
        d2 = (L8[2] - L8[3]) / (4 * H * scale)
        d4 = (L8[4] - L8[5]) / (8 * H * scale)
        fd.append((64 * d1 - 20 * d2 + d4) / 45)
        fd_plain.append((L8[6] - L8[7]) / (2e-6 * scale))
        ad.append(grad)
        kinds.append(kind)

    r0, x0 = r.detach(), x.detach()
    with torch.no_grad():
        # P / Q: every perturbed evaluation is one scenario of a second batch
        ne = len(UNIT) + 2
        m2 = DifferentiablePowerFlow(net, len(inj) * ne, **kw)
        rows = [c[1] for c in inj for _ in range(ne)]
        p2 = p.detach()[rows].clone()
        q2 = q.detach()[rows].clone()
        for k, (kind, sc, bus) in enumerate(inj):
            for e, h in enumerate(steps(kind)):
                (p2 if kind == "p" else q2)[k * ne + e, bus] += h
        Lv = losses_at_floor(m2, p2, q2, r0, x0)
        for k, (kind, sc, bus) in enumerate(inj):
            record(kind, Lv[k * ne:(k + 1) * ne], 1.0,
                   float((p if kind == "p" else q).grad[sc, bus]))
        # r / x: shared by every scenario, so each evaluation is a solve of the whole batch
        for kind, b in brs:
            base_val = float((r0 if kind == "r" else x0)[b])
            Ls = []
            for h in steps(kind):
                rr, xx = r0.clone(), x0.clone()
                (rr if kind == "r" else xx)[b] += h * base_val
                Ls.append(math.fsum(losses_at_floor(model, p.detach(), q.detach(), rr,
                                                    xx).tolist()))
            record(kind, Ls, base_val, float((r if kind == "r" else x).grad[b]))
    fd, fd_plain, ad, kinds = map(np.array, (fd, fd_plain, ad, kinds))
    worst = {}
    for kind in ("p", "q", "r", "x"):
        m = kinds == kind
        worst[kind] = (_rel_ok(ad[m], fd[m]), _rel_ok(ad[m], fd_plain[m]),
                       float(np.max(np.abs(ad[m]))))
    return worst


def test_adjoint_matches_central_finite_differences():
    """300-bus grid, 3 scenarios: 8 P, 8 Q, 6 r and 6 x coordinates within 1e-6 of the
    extrapolated central differences (_fd_check)."""
    from gap_b200 import synth

    net = synth.transmission_grid(8, n=300)
    s = synth.load_scenarios(net, 3, sigma=0.1, seed=8, base_power=1e8)
    worst = _fd_check(net, s, dict(base_power=1e8, precision="fp64", tol=1e-12, max_iter=30),
                      n_pq=8, n_rx=6, seed=0)
    print("300-bus adjoint vs central differences (Richardson, plain h=1e-6, max |gradient|):",
          worst)
    assert all(v[0] < REL for v in worst.values()), worst


def test_adjoint_c4_scale_central_differences():
    """The C4 workload: 256 load scenarios of the 10k-bus grid, L summed over the batch; 64
    seeded coordinates (24 P, 24 Q, 8 r, 8 x) within 1e-6 of the extrapolated central
    differences (_fd_check)."""
    from gap_b200 import synth

    net = synth.transmission_grid(0, n=10_000)
    s = synth.load_scenarios(net, 256, sigma=0.1, seed=1, base_power=1e8)
    worst = _fd_check(net, s, dict(base_power=1e8, precision="fp64", tol=1e-12, max_iter=30),
                      n_pq=24, n_rx=8, seed=42)
    print("C4 adjoint vs central differences (Richardson, plain h=1e-6, max |gradient|):", worst)
    assert all(v[0] < REL for v in worst.values()), worst
