"""GPU parity: the sm_100a path (through libgapk.so's C ABI) against the oracle and the
reference's golden outputs.

Tolerances (from the engine's parity contract): CSR pattern and reference-mode Y-bus values
bit-exact; tap-mode Y-bus 1e-14 relative; converged |V| and angle within 1e-8 pu / rad of the
reference CPU solver and iteration count within +-1; mismatch 1e-9 relative; FP64 Newton
correction 1e-10 relative."""

import numpy as np
import pytest

from helpers import fixture_names, load, network_of, parity_fixtures
from oracle import restate

pytestmark = pytest.mark.gpu

FIX = [n for n in parity_fixtures() if n != "kat_update"]


def _torch():
    import torch

    return torch


@pytest.mark.parametrize("name", FIX)
def test_ybus_device_values_bit_exact(name):
    from gap_b200.api import AdmittanceMatrix

    net, d = network_of(name)
    rp, ci, va = AdmittanceMatrix().build_admittance_matrix(net)
    assert np.array_equal(rp, d["y_row_ptr"]) and np.array_equal(ci, d["y_col_idx"])
    assert np.array_equal(va, d["y_values"])


def test_ybus_taps_mode_matches_pi_model():
    from gap_b200 import synth
    from gap_b200.api import AdmittanceMatrix

    net = synth.transmission_grid(2, n=600)
    rp, ci, va = AdmittanceMatrix(taps=True).build_admittance_matrix(net)
    rp2, ci2, vb = restate.ybus_pi(net)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)
    scale = np.max(np.abs(vb))
    assert np.max(np.abs(va - vb)) <= 1e-14 * scale


def test_ybus_batched_scenarios():
    """Per-scenario branch parameters (here: outages as zero admittance rows) in one launch."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(4, n=300)
    yp = YbusPlan.from_network(net)
    br = np.repeat(branch_params(net)[None], 5, axis=0)
    rng = np.random.default_rng(0)
    br[:, :, 0] *= rng.uniform(0.9, 1.1, size=br.shape[:2])
    out = yp.assemble(torch.as_tensor(br, device="cuda"),
                      torch.as_tensor(shunt_params(net), device="cuda"), mode=1).cpu().numpy()
    for s in range(5):
        n2 = synth.transmission_grid(4, n=300)
        n2.r1 = br[s, :, 0].copy()
        _, _, ref = restate.ybus_pi(n2)
        assert np.max(np.abs(out[s] - ref)) <= 1e-14 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", fixture_names("pgm_"))
def test_solve_simple_power_flow_pgm(name):
    """The reference's pytest contract (test_pgm_validation.py:213-252) plus parity with the
    reference CPU solver on the same lists."""
    from gap_b200.api import solve_simple_power_flow

    d = load(name)
    out = solve_simple_power_flow(d["bus_data"].tolist(), d["branch_data"].tolist(),
                                  tolerance=1e-8, max_iterations=20, verbose=False,
                                  base_power=float(d["base_power"]), backend="gpu")
    meta = out[-1]
    rows = np.array(out[:-1])
    assert bool(meta[0]) and bool(d["ref_converged"])
    assert abs(int(meta[1]) - int(d["ref_iterations"])) <= 1
    assert np.max(np.abs(rows[:, 2] - d["pgm_u_pu"])) < 5e-6
    assert np.max(np.abs(rows[:, 2] - np.abs(d["ref_v"]))) < 1e-8
    assert np.max(np.abs(rows[:, 3] - np.angle(d["ref_v"]))) < 1e-8


@pytest.mark.parametrize("name", fixture_names("c0_") + fixture_names("kat_"))
def test_nr_fp64_matches_reference(name):
    if name == "kat_update":
        pytest.skip("no solve")
    from gap_b200.api import NewtonRaphson, PowerFlowConfig

    net, d = network_of(name)
    cfg = PowerFlowConfig(tolerance=1e-8, max_iterations=20, base_power=float(d["base_power"]))
    Y = (d["y_row_ptr"], d["y_col_idx"], d["y_values"])
    r = NewtonRaphson().solve_power_flow(net, Y, cfg)
    assert r.converged == bool(d["ref_converged"])
    assert abs(r.iterations - int(d["ref_iterations"])) <= 1
    # bus_injections (never filled by the reference): S = V conj(Y V) per unit at the result
    zb = float(net.u_rated[0]) ** 2 / cfg.base_power
    s_ref = restate.power_injections(Y[0], Y[1], Y[2] * zb, r.bus_voltages)
    assert np.max(np.abs(r.bus_injections - s_ref)) <= 1e-12 * max(1.0, np.max(np.abs(s_ref)))
    if r.converged:
        assert np.max(np.abs(np.abs(r.bus_voltages) - np.abs(d["ref_v"]))) < 1e-8
        assert np.max(np.abs(np.angle(r.bus_voltages) - np.angle(d["ref_v"]))) < 1e-8
    else:
        # singular Jacobian (isolated bus): V stays where the reference leaves it
        np.testing.assert_allclose(r.bus_voltages, d["ref_v"], atol=1e-12)
        assert r.final_mismatch == pytest.approx(float(d["ref_final_mismatch"]), rel=1e-9)


@pytest.mark.parametrize("name", [n for n in fixture_names("kat_") if n != "kat_update"])
def test_mismatch_matches_reference(name):
    from gap_b200.api import NewtonRaphson

    net, d = network_of(name)
    nr = NewtonRaphson()
    for k in ("0", "1"):
        f = nr.calculate_mismatches(net, d["mm_v" + k])
        np.testing.assert_allclose(f, d["mm_f" + k], rtol=1e-9, atol=1e-6)


@pytest.mark.parametrize("precision,lanes", [("fp64", 1), ("fp64", 4), ("fp32", 8)])
def test_newton_correction_matches_sparse_solve(precision, lanes):
    """One Jacobian build + factor + solve on the device vs scipy on the oracle Jacobian."""
    torch = _torch()
    import scipy.sparse.linalg as spla

    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(7, n=1000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    S = 6
    rng = np.random.default_rng(3)
    v = np.stack([restate.flat_start(net) * np.exp(1j * rng.normal(0, 0.03, net.n_bus))
                  for _ in range(S)])
    s_spec = np.repeat(net.specified_power(base)[None], S, axis=0)
    b = NRBatch(plan, S, precision=precision, lanes=lanes)
    b.stage_load(y, torch.as_tensor(s_spec, device="cuda"),
                 v_init=torch.as_tensor(v, device="cuda"), refine=1 if precision == "fp32" else 0)
    for st in ("mismatch", "jacobian", "factor", "solve"):
        b.stage(st)
    dx = b.correction().cpu().numpy()
    f = b.mismatch().cpu().numpy()
    ypu = y.cpu().numpy()
    for s in range(S):
        sc = restate.power_injections(yp.row_ptr, yp.col_idx, ypu, v[s])
        fr = restate.mismatch(net.bus_type, sc, s_spec[s])
        np.testing.assert_allclose(f[s], fr, rtol=1e-9, atol=1e-11)
        J = restate.jacobian(yp.row_ptr, yp.col_idx, ypu, v[s], net.bus_type, mode="exact",
                             drop=False)
        xr = spla.spsolve(J.tocsc(), -fr)
        tol = 1e-10 if precision == "fp64" else 1e-6
        assert np.max(np.abs(dx[s] - xr)) <= tol * np.max(np.abs(xr))


@pytest.mark.parametrize("precision,refine", [("fp64", 0), ("fp32", 1)])
def test_batched_scenarios_match_oracle(precision, refine):
    """Load scenarios of a transmission grid (taps, PV, shunts) in one batch, Newton policy,
    against the FP64 oracle solved to the same tolerance."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(1, n=2000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    S = 19  # not a multiple of the lane count: exercises padding lanes
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=5, base_power=base)
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    b = NRBatch(plan, S, precision=precision, lanes=8)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    r = b.solve(y, torch.as_tensor(s_spec, device="cuda"),
                v_init=torch.as_tensor(v0, device="cuda"), tol=1e-10, max_iter=30,
                policy="newton", refine=refine)
    torch.cuda.synchronize()
    st = r.status.cpu().numpy()
    assert (st == 0).all(), st
    V = r.v.cpu().numpy()
    Y = restate.ybus_pi(net)
    for s in (0, 7, 8, 18):
        o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
        assert o["converged"]
        assert np.max(np.abs(np.abs(V[s]) - np.abs(o["v"]))) < 1e-8
        assert np.max(np.abs(np.angle(V[s]) - np.angle(o["v"]))) < 1e-8


def test_graph_and_host_loop_agree():
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.feeder_grid(3)
    zb = net.u_rated[0] ** 2 / 1e6
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type)
    s = torch.as_tensor(net.specified_power(1e6)[None], device="cuda")
    outs = []
    for g in (True, False):
        b = NRBatch(plan, 1, lanes=1, use_graph=g)
        r = b.solve(y, s, tol=1e-8, max_iter=20)
        torch.cuda.synchronize()
        outs.append((r.v.cpu().numpy(), int(r.iterations[0]), b.loop_count()))
    assert outs[0][1] == outs[1][1] == outs[0][2]
    np.testing.assert_array_equal(outs[0][0], outs[1][0])


@pytest.mark.parametrize("name", [n for n in fixture_names("kat_") if n != "kat_update"]
                         + fixture_names("c0_")[:2] + fixture_names("pgm_")[:4])
def test_iteration_state_capture_matches_reference(name):
    """enable_state_capture / get_iteration_states (powerflow_interface.h:83-107): one
    IterationState per iteration, state by state against the reference's own capture
    (cpu_newton_raphson.cpp:125-149), and the capturing solve's result equal to the plain
    solve's."""
    from gap_b200.api import NewtonRaphson, PowerFlowConfig

    net, d = network_of(name)
    cfg = PowerFlowConfig(tolerance=1e-8, max_iterations=20, base_power=float(d["base_power"]))
    Y = (d["y_row_ptr"], d["y_col_idx"], d["y_values"])
    nr = NewtonRaphson()
    plain = nr.solve_power_flow(net, Y, cfg)
    assert nr.get_iteration_states() == []
    nr.enable_state_capture(True)
    r = nr.solve_power_flow(net, Y, cfg)
    st = nr.get_iteration_states()
    assert (r.converged, r.iterations) == (plain.converged, plain.iterations)
    np.testing.assert_array_equal(r.bus_voltages, plain.bus_voltages)
    assert len(st) == r.iterations
    ref_m = d["cap_max_mis"]
    assert abs(len(st) - len(ref_m)) <= 1
    m0 = max(1.0, float(np.max(ref_m)))
    for k in range(min(len(st), len(ref_m))):
        assert st[k].iteration == k
        assert abs(st[k].max_mismatch - ref_m[k]) <= 1e-9 * m0
        assert st[k].max_mismatch == np.max(np.abs(st[k].mismatches), initial=0.0)
        assert np.max(np.abs(st[k].voltages - d["cap_v"][k])) < 1e-9
        if "cap_i" in d:
            si = max(1.0, float(np.max(np.abs(d["cap_i"][k]))))
            ss = max(1.0, float(np.max(np.abs(d["cap_s"][k]))))
            assert np.max(np.abs(st[k].currents - d["cap_i"][k])) <= 1e-9 * si
            assert np.max(np.abs(st[k].power_injections - d["cap_s"][k])) <= 1e-9 * ss
    nr.clear_iteration_states()
    assert nr.get_iteration_states() == []


def test_stepped_batch_matches_oracle_states():
    """gapk_nr_step / gapk_nr_get_state on a lane-interleaved FP64 batch: every scenario's
    recorded states against the oracle's, and the outputs equal to gapk_nr_solve's."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.feeder_grid(1)
    zb = net.u_rated[0] ** 2 / 1e6
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type)
    S = 6
    rng = np.random.default_rng(5)
    s0 = net.specified_power(1e6)
    sc = s0[None, :] * rng.uniform(0.6, 1.3, size=(S, 1))
    s = torch.as_tensor(sc, device="cuda")
    b = NRBatch(plan, S, precision="fp64", lanes=4)
    ref = b.solve(y, s, tol=1e-8, max_iter=20)
    r, states = b.solve_captured(y, s, tol=1e-8, max_iter=20)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.v.cpu().numpy(), ref.v.cpu().numpy())
    np.testing.assert_array_equal(r.iterations.cpu().numpy(), ref.iterations.cpu().numpy())
    its = r.iterations.cpu().numpy()
    assert len(states) == int(its.max())
    rp, ci, va = restate.ybus_reference(net)
    for q in range(S):
        o = restate.nr_solve(net, Y=(rp, ci, va), tol=1e-8, max_iter=20, base_power=1e6,
                             s_spec=sc[q], states=True)
        assert abs(o["iterations"] - int(its[q])) <= 1
        m0 = max(1.0, o["states"][0]["max_mismatch"])
        for k in range(min(int(its[q]), len(o["states"]))):
            g, w = states[k], o["states"][k]
            assert np.max(np.abs(g["v"][q].cpu().numpy() - w["v"])) < 1e-9
            assert np.max(np.abs(g["mismatch"][q].cpu().numpy() - w["mismatch"])) <= 1e-9 * m0
            si = max(1.0, float(np.max(np.abs(w["i"]))))
            assert np.max(np.abs(g["i"][q].cpu().numpy() - w["i"])) <= 1e-9 * si
            assert np.max(np.abs(g["s"][q].cpu().numpy() - w["s"])) <= 1e-9 * si


def test_max_iterations_semantics():
    """max_iterations reached: iterations == max, not converged, final mismatch from the last
    evaluation (cpu_newton_raphson.cpp:100-174)."""
    from gap_b200 import synth
    from gap_b200.api import NewtonRaphson, PowerFlowConfig

    net = synth.feeder_grid(0)
    r = NewtonRaphson().solve_power_flow(net, None, PowerFlowConfig(tolerance=1e-8,
                                                                    max_iterations=3,
                                                                    base_power=1e6))
    o = restate.nr_solve(net, tol=1e-8, max_iter=3, base_power=1e6)
    assert not r.converged and r.iterations == 3 and not o["converged"]
    assert r.final_mismatch == pytest.approx(o["final_mismatch"], rel=1e-9)
    np.testing.assert_allclose(r.bus_voltages, o["v"], atol=1e-12)


@pytest.mark.parametrize("precision,lanes,dense_min", [("fp64", 1, 0), ("fp32", 8, 0),
                                                       ("fp64", 2, -1)])
def test_dense_tail_correction_matches_sparse_solve(precision, lanes, dense_min):
    """A grid whose elimination order ends in a large dense block (dense tail on the device)
    against scipy; dense_min=-1 runs the same grid fully on the sparse schedule."""
    torch = _torch()
    import scipy.sparse.linalg as spla

    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(9, n=4000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact", dense_min=dense_min)
    assert (plan.info["n_tail"] > 50) == (dense_min == 0)
    S = 3
    rng = np.random.default_rng(11)
    v = np.stack([synth.dc_start(net, base) * np.exp(1j * rng.normal(0, 0.01, net.n_bus))
                  for _ in range(S)])
    s_spec = np.repeat(net.specified_power(base)[None], S, axis=0)
    b = NRBatch(plan, S, precision=precision, lanes=lanes)
    b.stage_load(y, torch.as_tensor(s_spec, device="cuda"),
                 v_init=torch.as_tensor(v, device="cuda"), refine=1 if precision == "fp32" else 0)
    for st in ("mismatch", "jacobian", "factor", "solve"):
        b.stage(st)
    dx = b.correction().cpu().numpy()
    ypu = y.cpu().numpy()
    for s in range(S):
        sc = restate.power_injections(yp.row_ptr, yp.col_idx, ypu, v[s])
        fr = restate.mismatch(net.bus_type, sc, s_spec[s])
        J = restate.jacobian(yp.row_ptr, yp.col_idx, ypu, v[s], net.bus_type, mode="exact",
                             drop=False)
        xr = spla.spsolve(J.tocsc(), -fr)
        tol = 1e-10 if precision == "fp64" else 1e-6
        assert np.max(np.abs(dx[s] - xr)) <= tol * np.max(np.abs(xr))


def test_level_trace_stamps_and_unchanged_results():
    """gapk_nr_set_level_trace: per-group stamps ordered in time for the factorisation and both
    solves, and the correction computed with the trace on equal to the one computed without."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(9, n=4000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    assert plan.info["n_tail"] > 50
    S = 304  # >= 2 per SM: the one-CTA-per-scenario dense LU, which writes the panel trace
    rng = np.random.default_rng(3)
    v0 = synth.dc_start(net, base)
    v = torch.as_tensor(v0[None] * np.exp(1j * rng.normal(0, 0.01, (S, net.n_bus))),
                        device="cuda")
    s = torch.as_tensor(np.repeat(net.specified_power(base)[None], S, axis=0), device="cuda")
    b = NRBatch(plan, S, precision="fp32", lanes=8)
    b.stage_load(y, s, v_init=v)
    for st in ("mismatch", "jacobian", "factor", "solve"):
        b.stage(st)
    dx0 = b.correction()
    lt = b.level_trace(y, s, v_init=v)
    dx1 = b.correction()
    assert torch.equal(dx0, dx1)
    L = plan.info["n_levels"]
    for k in ("factor", "forward", "backward"):
        st = lt[k]["stamps"]
        assert st.shape == (S // 8, L + 2)
        assert (st[:, 0] > 0).all() and (np.diff(st, axis=1) >= 0).all()
        assert lt[k]["level_us"].shape == (S // 8, L)
        assert (lt[k]["total_us"] > 0).all() and (lt[k]["total_us"] < 1e5).all()
    d = lt["dense"]["stamps"]
    npan = -(-2 * plan.info["n_tail"] // 32)
    assert d.shape == (S, 1 + 3 * npan)
    assert (d[:, 0] > 0).all() and (np.diff(d, axis=1) >= 0).all()
    assert lt["dense"]["phase_us"].shape == (S, npan, 3)
    # trace off afterwards: a plain solve is unaffected and writes no stamps
    r = b.solve(y, s, v_init=v, tol=1e-8, max_iter=20, policy="newton", refine=1)
    torch.cuda.synchronize()
    assert bool((r.status == 0).all())


def _csr(A):
    rows, cols = np.nonzero(A)
    rp = np.zeros(A.shape[0] + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp).astype(np.int32), cols.astype(np.int32), A[rows, cols]


@pytest.mark.parametrize("name", fixture_names("lu_"))
def test_sparse_lu_matches_reference_lu(name):
    torch = _torch()
    from gap_b200.engine import SparseLU

    d = load(name)
    lu = SparseLU(d["row_ptr"], d["col_idx"])
    assert lu.factorize(torch.as_tensor(d["values"], device="cuda"))
    x = lu.solve(torch.as_tensor(d["rhs"], device="cuda")).cpu().numpy()
    np.testing.assert_allclose(x, d["ref_x"], rtol=1e-10, atol=1e-12)


def test_sparse_lu_reference_unit_matrices_and_pivoting_cases():
    """The matrices of tests/unit/test_lu_solver.cpp (2x2, 3x3 tridiagonal, diagonal,
    identity) plus systems that need the row matching (zero diagonal) and a dense tail."""
    torch = _torch()
    from gap_b200.engine import SparseLU

    rng = np.random.default_rng(5)
    mats = [np.array([[2, 1], [1, 2]], complex), np.array([[2, 1, 0], [1, 3, 1], [0, 1, 2]], complex),
            np.diag([2.0, 3.0, 4.0]).astype(complex), np.eye(3, dtype=complex),
            np.array([[0, 2], [3, 0]], complex)]
    n = 300
    A = ((rng.random((n, n)) < 0.02) * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))))
    P = np.eye(n)[rng.permutation(n)]
    A = P @ (A + np.diag(5 + rng.random(n)))  # rows shuffled: diagonal mostly zero
    mats.append(A)
    for A in mats:
        rp, ci, va = _csr(A)
        lu = SparseLU(rp, ci)
        assert lu.factorize(torch.as_tensor(va, device="cuda"))
        b = rng.normal(size=A.shape[0]) + 1j * rng.normal(size=A.shape[0])
        x = lu.solve(torch.as_tensor(b, device="cuda")).cpu().numpy()
        # the reference's own GPU LU tests accept 1e-9 on their denser system
        # (tests/unit/test_gpu_lu_solver.cpp:247); static pivoting on the shuffled 300 x 300
        # system leaves residuals near 1e-10
        np.testing.assert_allclose(A @ x, b, rtol=1e-9, atol=1e-9)
    # numerically singular under static pivoting -> factorize reports failure
    rp, ci, va = _csr(np.array([[1, 1], [1, 1]], complex))
    assert not SparseLU(rp, ci).factorize(torch.as_tensor(va, device="cuda"))


def test_clamped_policy_matches_oracle_from_flat_start():
    """Full Newton steps with the reference's clamps, from the flat start (where the clamps
    bind), against the oracle's same policy: same iteration count, voltages to 1e-8."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(2, n=2000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    S = 4
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=3, base_power=base)
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    b = NRBatch(plan, S, precision="fp64", lanes=4)
    u = torch.as_tensor(net.u_pu.astype(np.float64), device="cuda")
    r = b.solve(y, torch.as_tensor(s_spec, device="cuda"), u_pu=u, tol=1e-10, max_iter=40,
                policy="clamped")
    torch.cuda.synchronize()
    assert (r.status.cpu().numpy() == 0).all()
    V = r.v.cpu().numpy()
    it = r.iterations.cpu().numpy()
    Y = restate.ybus_pi(net)
    for s in range(S):
        o = restate.nr_solve(net, Y=Y, tol=1e-10, max_iter=40, base_power=base,
                             policy="clamped", jac="exact", s_spec=s_spec[s])
        assert o["converged"]
        assert abs(int(it[s]) - o["iterations"]) <= 1
        assert np.max(np.abs(V[s] - o["v"])) < 1e-8


def test_refinement_only_near_convergence_matches_oracle():
    """FP32 factor with the refinement step run only once a group is near convergence
    (refine_below): same converged voltages as the FP64 oracle, and refinement does run
    (results differ from no refinement at all only through convergence, not accuracy)."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(1, n=2000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    S = 11
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=6, base_power=base)
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    b = NRBatch(plan, S, precision="fp32", lanes=4)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    s_t = torch.as_tensor(s_spec, device="cuda")
    v_t = torch.as_tensor(v0, device="cuda")
    r = b.solve(y, s_t, v_init=v_t, tol=1e-10, max_iter=30, policy="newton", refine=1,
                refine_below=1e-4)
    torch.cuda.synchronize()
    assert (r.status.cpu().numpy() == 0).all()
    V = r.v.cpu().numpy()
    Y = restate.ybus_pi(net)
    for s in (0, 5, 10):
        o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
        assert np.max(np.abs(np.abs(V[s]) - np.abs(o["v"]))) < 1e-8
        assert np.max(np.abs(np.angle(V[s]) - np.angle(o["v"]))) < 1e-8
    with pytest.raises(Exception):
        b.solve(y, s_t, v_init=v_t, tol=1e-10, max_iter=30, policy="newton", refine=1,
                refine_below=-1.0)


def test_dense_tail_paths_agree():
    """The dense tail is factorised by one CTA per scenario when a batch fills the GPU (here
    300 scenarios) and by the split panel/update kernels otherwise (8 scenarios): both give
    the same converged voltages, and the same as the FP64 oracle."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(3, n=3000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    assert plan.info["n_tail"] > 32
    S = 300
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=8, base_power=base)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    kw = dict(tol=1e-10, max_iter=30, policy="newton", refine=1)
    big = NRBatch(plan, S, precision="fp32", lanes=8)
    rb = big.solve(y, torch.as_tensor(s_spec, device="cuda"),
                   v_init=torch.as_tensor(v0, device="cuda"), **kw)
    small = NRBatch(plan, 8, precision="fp32", lanes=8)
    rs = small.solve(y, torch.as_tensor(s_spec[:8], device="cuda"),
                     v_init=torch.as_tensor(v0[:8], device="cuda"), **kw)
    torch.cuda.synchronize()
    assert (rb.status.cpu().numpy() == 0).all() and (rs.status.cpu().numpy() == 0).all()
    Vb, Vs = rb.v.cpu().numpy(), rs.v.cpu().numpy()
    assert np.max(np.abs(Vb[:8] - Vs)) < 1e-9
    # dense_fused: the small batch on the one-CTA-per-scenario kernel (as the parts of a
    # HostPipeline run) gives the large batch's voltages
    fused = NRBatch(plan, 8, precision="fp32", lanes=8, dense_fused=True)
    rf = fused.solve(y, torch.as_tensor(s_spec[:8], device="cuda"),
                     v_init=torch.as_tensor(v0[:8], device="cuda"), **kw)
    assert (rf.status.cpu().numpy() == 0).all()
    assert np.max(np.abs(rf.v.cpu().numpy() - Vb[:8])) < 1e-12
    Y = restate.ybus_pi(net)
    for s in (0, 299):
        o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
        assert np.max(np.abs(Vb[s] - o["v"])) < 1e-8


def test_dense_lu_tensor_core_trailing_update():
    """The one-CTA-per-scenario FP32 dense-tail LU with its rank-32 trailing updates on the
    tensor cores (k_dense_lu_tc: tcgen05, three TF32 products per tile accumulated in FP32; the
    default) converges like the CUDA-core kernel (dense_fma): every scenario converged,
    iteration counts within one, voltages within 1e-9 of each other and within 1e-8 of the
    FP64 oracle."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(3, n=6000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    # several 128 x 128 trailing tiles in the first panels, ragged last tile and panel
    assert 2 * plan.info["n_tail"] > 256 and (2 * plan.info["n_tail"]) % 32
    S = 300
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=8, base_power=base)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    kw = dict(tol=1e-10, max_iter=30, policy="newton", refine=1)
    out = {}
    for fma in (False, True):
        r = NRBatch(plan, S, precision="fp32", lanes=8, dense_fma=fma).solve(
            y, torch.as_tensor(s_spec, device="cuda"),
            v_init=torch.as_tensor(v0, device="cuda"), **kw)
        torch.cuda.synchronize()
        assert (r.status.cpu().numpy() == 0).all()
        out[fma] = (r.v.cpu().numpy(), r.iterations.cpu().numpy())
    assert np.max(np.abs(out[True][0] - out[False][0])) < 1e-9
    assert np.max(np.abs(out[True][1] - out[False][1])) <= 1
    Y = restate.ybus_pi(net)
    for s in (0, 299):
        o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
        assert np.max(np.abs(out[False][0][s] - o["v"])) < 1e-8


def test_split_dense_lu_tensor_core_update():
    """Batches too small to fill the GPU factorise the dense tail with the split kernels (a
    panel launch per 32 columns, then one CTA per 128 x 128 trailing tile and scenario); in
    FP32 the tile update runs on the tensor cores (k_dlu_update_tc).  Against the CUDA-core
    update (dense_fma): every scenario converged, iterations within one, voltages within 1e-9;
    against the FP64 oracle within 1e-8."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(3, n=6000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    assert 2 * plan.info["n_tail"] > 256 and (2 * plan.info["n_tail"]) % 32
    S = 8
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=9, base_power=base)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    kw = dict(tol=1e-10, max_iter=30, policy="newton", refine=1)
    out = {}
    for fma in (False, True):
        r = NRBatch(plan, S, precision="fp32", lanes=8, dense_fma=fma).solve(
            y, torch.as_tensor(s_spec, device="cuda"),
            v_init=torch.as_tensor(v0, device="cuda"), **kw)
        torch.cuda.synchronize()
        assert (r.status.cpu().numpy() == 0).all()
        out[fma] = (r.v.cpu().numpy(), r.iterations.cpu().numpy())
    assert np.max(np.abs(out[True][0] - out[False][0])) < 1e-9
    assert np.max(np.abs(out[True][1] - out[False][1])) <= 1
    Y = restate.ybus_pi(net)
    for s in (0, S - 1):
        o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
        assert np.max(np.abs(out[False][0][s] - o["v"])) < 1e-8


def test_host_pipeline_equals_one_batch():
    """Solving from pinned host buffers in two stream-overlapped parts gives bit-identical
    results to one device batch (the parts keep the lane groups)."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import HostPipeline, NRBatch, NRPlan, YbusPlan, branch_params, \
        shunt_params

    net = synth.transmission_grid(5, n=1200)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    S = 48
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=4, base_power=base)
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    kw = dict(tol=1e-10, max_iter=30, policy="newton", refine=1, refine_below=1e-4)
    # the pipeline's parts use the one-CTA-per-scenario dense LU (dense_fused); so does the
    # reference batch here
    one = NRBatch(plan, S, precision="fp32", lanes=8, threads=1024, dense_fused=True).solve(
        y, torch.as_tensor(s_spec, device="cuda"), v_init=torch.as_tensor(v0, device="cuda"),
        **kw)
    s_h = torch.as_tensor(s_spec).pin_memory()
    v_h = torch.as_tensor(v0).pin_memory()
    vo = torch.empty((S, net.n_bus), dtype=torch.complex128).pin_memory()
    st = torch.empty(S, dtype=torch.int32).pin_memory()
    it = torch.empty(S, dtype=torch.int32).pin_memory()
    pipe = HostPipeline(plan, S, chunks=2, precision="fp32", lanes=8)
    assert pipe.ranges == [(0, 24), (24, 48)]
    for _ in range(2):
        pipe.solve(y, s_h, v_h, vo, st, it, **kw)
        assert torch.equal(vo, one.v.cpu())
        assert torch.equal(st, one.status.cpu()) and (st.numpy() == 0).all()
        assert torch.equal(it, one.iterations.cpu())
    # one start vector shared by every scenario (v_init_shared): the same results, from the
    # pipeline and from a device batch
    v_h1 = torch.as_tensor(v0[0]).pin_memory()
    pipe.solve(y, s_h, v_h1, vo, st, it, **kw)
    assert torch.equal(vo, one.v.cpu()) and torch.equal(it, one.iterations.cpu())
    shared = NRBatch(plan, S, precision="fp32", lanes=8, threads=1024, dense_fused=True).solve(
        y, torch.as_tensor(s_spec, device="cuda"), v_init=torch.as_tensor(v0[0], device="cuda"),
        **kw)
    assert torch.equal(shared.v, one.v) and torch.equal(shared.iterations, one.iterations)


def test_factor_reuse_near_convergence_matches_oracle():
    """Below reuse_below a lane group keeps its previous LU factors and the refined solve
    corrects against the current FP64 Jacobian: converged voltages as the FP64 oracle's, and
    the option is refused without refinement."""
    torch = _torch()
    from gap_b200 import synth
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(1, n=2000)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    S = 13
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=7, base_power=base)
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    v0 = np.repeat(synth.dc_start(net, base)[None], S, axis=0)
    s_t = torch.as_tensor(s_spec, device="cuda")
    v_t = torch.as_tensor(v0, device="cuda")
    Y = restate.ybus_pi(net)
    for lanes, n_sc in ((4, S), (8, 320)):
        b = NRBatch(plan, n_sc, precision="fp32", lanes=lanes)
        ss = s_t if n_sc == S else s_t.repeat((n_sc + S - 1) // S, 1)[:n_sc].contiguous()
        vv = v_t if n_sc == S else v_t.repeat((n_sc + S - 1) // S, 1)[:n_sc].contiguous()
        r = b.solve(y, ss, v_init=vv, tol=1e-10, max_iter=30, policy="newton", refine=1,
                    refine_below=1e-3, reuse_below=1e-3)
        torch.cuda.synchronize()
        assert (r.status.cpu().numpy() == 0).all()
        V = r.v.cpu().numpy()
        for s in (0, 6, 12):
            o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=base,
                                 policy="newton", jac="exact", s_spec=s_spec[s], v0=v0[s])
            assert np.max(np.abs(V[s] - o["v"])) < 1e-8
    with pytest.raises(Exception):
        b.solve(y, ss, v_init=vv, tol=1e-10, max_iter=30, policy="newton", refine=0,
                reuse_below=1e-3)
