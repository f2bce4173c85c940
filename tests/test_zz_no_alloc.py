"""The allocation-free solve, gapk_nr_solve_noalloc, checked against gapk_nr_solve.

gapk_nr_solve_noalloc exists for callers that may not allocate device memory while they
solve (hosts that hand out device memory only from their own pools, real-time loops kept away
from the allocator, whose cudaMalloc / cudaFree can block on the whole device).  It keeps every
working buffer in one static 32 MiB device array.  These tests call it through the C ABI
twice in a row -- on two different grids, so the second call reuses memory the first one left
behind -- and compare each result with the regular batched entry point on a one-scenario FP64
batch, within the parity tolerance of the other GPU tests (|V| and angle within 1e-8, same
iteration count and status).  This file is named to run after every other test file.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_V = 1e-8


def _case(kind):
    import torch

    from gap_b200 import synth
    from gap_b200.engine import NRPlan, YbusPlan, branch_params, shunt_params

    if kind == "feeder":
        net, base, mode, jac, policy, v0 = synth.feeder_grid(2), 1e6, 0, "reference", "reference", None
    elif kind == "isolated":
        from helpers import network_of

        net, _ = network_of("kat_four_bus_isolated")
        base, mode, jac, policy, v0 = 1e6, 0, "reference", "reference", None
    else:
        n = 10_000 if kind == "transmission10k" else 2000
        net, base, mode, jac, policy = synth.transmission_grid(3, n=n), 1e8, 1, "exact", "newton"
        v0 = synth.dc_start(net, base)
    zb = float(net.u_rated[0]) ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=mode, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian=jac)
    s = torch.as_tensor(net.specified_power(base)[None], device="cuda")
    u = torch.as_tensor(net.u_pu, device="cuda")
    v = None if v0 is None else torch.as_tensor(v0[None], device="cuda")
    return plan, y, s, u, v, policy


def _noalloc(plan, y, s, u, v, policy, max_iter=30):
    import torch

    from gap_b200 import _native as N
    from gap_b200.engine import _dptr, _stream_ptr

    n = plan.info["n_bus"]
    vo = torch.zeros((1, n), dtype=torch.complex128, device="cuda")
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    fm = torch.zeros(1, dtype=torch.float64, device="cuda")
    inp = N.Inputs(_dptr(y), _dptr(s), _dptr(v), _dptr(u), 1e-8, max_iter,
                   N.POLICY_REFERENCE if policy == "reference" else N.POLICY_NEWTON, 0)
    out = N.Outputs(_dptr(vo), _dptr(it), _dptr(st), _dptr(fm))
    rc = N.lib().gapk_nr_solve_noalloc(plan._h, C.byref(inp), C.byref(out), _stream_ptr())
    torch.cuda.synchronize()
    return rc, vo[0].cpu().numpy(), int(it.item()), int(st.item())


def _regular(plan, y, s, u, v, policy, max_iter=30):
    import torch

    from gap_b200.engine import NRBatch

    b = NRBatch(plan, 1, precision="fp64", lanes=1)
    r = b.solve(y, s, v_init=v, u_pu=u, tol=1e-8, max_iter=max_iter, policy=policy)
    torch.cuda.synchronize()
    return r.v[0].cpu().numpy(), int(r.iterations[0].item()), int(r.status[0].item())


def test_noalloc_matches_regular_solve_on_two_calls_in_a_row():
    cases = [_case("feeder"), _case("transmission")]
    for args in cases:  # two calls in a row, different grids sharing the static scratch
        rc, v, it, st = _noalloc(*args)
        assert rc == 0, rc
        vr, itr, str_ = _regular(*args)
        assert st == str_ == 0
        assert it == itr
        assert np.max(np.abs(np.abs(v) - np.abs(vr))) < TOL_V
        assert np.max(np.abs(np.angle(v) - np.angle(vr))) < TOL_V
    # and the first grid again, after the second one overwrote the scratch
    rc, v, it, st = _noalloc(*cases[0])
    vr, itr, _ = _regular(*cases[0])
    assert rc == 0 and st == 0 and it == itr
    assert np.max(np.abs(v - vr)) < TOL_V


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    from gap_b200 import _native as N

    plan, y, s, u, v, policy = _case("transmission")
    big = None
    from gap_b200 import synth
    from gap_b200.engine import NRPlan, YbusPlan

    net = synth.transmission_grid(0, n=20000)
    yp = YbusPlan.from_network(net)
    big = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    rc, *_ = _noalloc(big, y, s, u, v, policy)
    assert rc == -6  # GAPK_ERANGE
    assert b"32 MiB" in N.lib().gapk_last_error()


@pytest.mark.parametrize("max_iter", [0, 2])
def test_noalloc_unconverged_runs_match_regular_solve(max_iter):
    """max_iter = 0 returns the start vector; max_iter = 2 stops before convergence: status
    (MAXITER), iteration count and voltages as the regular entry point's."""
    args = _case("transmission")
    rc, v, it, st = _noalloc(*args, max_iter=max_iter)
    vr, itr, str_ = _regular(*args, max_iter=max_iter)
    assert rc == 0
    assert st == str_ == 1  # SCEN_MAXITER
    assert it == itr
    assert np.max(np.abs(v - vr)) < TOL_V


def test_noalloc_singular_jacobian_status_matches_regular_solve():
    """An isolated PQ bus makes the Jacobian singular: both entry points stop the scenario with
    status SINGULAR, iterations = max_iterations and the voltages unchanged."""
    args = _case("isolated")
    rc, v, it, st = _noalloc(*args)
    vr, itr, str_ = _regular(*args)
    assert rc == 0
    assert st == str_ == 2  # SCEN_SINGULAR
    assert it == itr
    assert np.max(np.abs(v - vr)) < TOL_V


def test_noalloc_fits_the_10k_bus_grid():
    """The documented size: a 10,000-bus grid of the transmission generator fits the 32 MiB
    scratch and solves as the regular entry point does."""
    args = _case("transmission10k")
    rc, v, it, st = _noalloc(*args)
    assert rc == 0, rc
    vr, itr, str_ = _regular(*args)
    assert st == str_ == 0 and it == itr
    assert np.max(np.abs(v - vr)) < TOL_V
