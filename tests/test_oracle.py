"""The oracle (CPU restatement) pinned against the reference's own outputs: golden vectors
generated by tests/golden/make_golden.py from the reference CPU path and from the
power-grid-model outputs shipped with the reference's tests."""

import numpy as np
import pytest

from helpers import fixture_names, load, network_of, net_from, parity_fixtures
from oracle import restate

FIX = [n for n in parity_fixtures() if n != "kat_update"]


@pytest.mark.parametrize("name", FIX)
def test_ybus_restatement_bit_exact(name):
    net, d = network_of(name)
    rp, ci, va = restate.ybus_reference(net)
    assert np.array_equal(rp, d["y_row_ptr"])
    assert np.array_equal(ci, d["y_col_idx"])
    assert np.array_equal(va.view(np.float64), d["y_values"].view(np.float64))


@pytest.mark.parametrize("name", FIX)
def test_nr_restatement_matches_reference(name):
    net, d = network_of(name)
    base = float(d["base_power"])
    r = restate.nr_solve(net, tol=1e-8, max_iter=20, base_power=base)
    assert r["converged"] == bool(d["ref_converged"])
    assert abs(r["iterations"] - int(d["ref_iterations"])) <= 1
    if r["converged"]:
        assert np.max(np.abs(np.abs(r["v"]) - np.abs(d["ref_v"]))) < 1e-10
        assert np.max(np.abs(np.angle(r["v"]) - np.angle(d["ref_v"]))) < 1e-10


@pytest.mark.parametrize("name", FIX)
def test_iteration_states_match_reference_capture(name):
    """IterationState per iteration (cpu_newton_raphson.cpp:125-149, captured from the
    reference by tests/golden/make_golden.py): the restatement's trajectory state by state."""
    net, d = network_of(name)
    r = restate.nr_solve(net, tol=1e-8, max_iter=20, base_power=float(d["base_power"]),
                         states=True)
    st = r["states"]
    ref_m = d["cap_max_mis"]
    assert len(ref_m) == int(d["ref_iterations"])
    assert len(st) == r["iterations"]
    m0 = max(1.0, float(np.max(ref_m)))
    for k in range(min(len(st), len(ref_m))):
        assert st[k]["iteration"] == k
        assert abs(st[k]["max_mismatch"] - ref_m[k]) <= 1e-10 * m0
        assert np.max(np.abs(st[k]["v"] - d["cap_v"][k])) < 1e-10
        assert st[k]["max_mismatch"] == np.max(np.abs(st[k]["mismatch"]), initial=0.0)
        if "cap_i" in d:
            si = max(1.0, float(np.max(np.abs(d["cap_i"][k]))))
            ss = max(1.0, float(np.max(np.abs(d["cap_s"][k]))))
            assert np.max(np.abs(st[k]["i"] - d["cap_i"][k])) <= 1e-10 * si
            assert np.max(np.abs(st[k]["s"] - d["cap_s"][k])) <= 1e-10 * ss


@pytest.mark.parametrize("name", fixture_names("pgm_"))
def test_reference_and_restatement_vs_power_grid_model(name):
    """The reference's own acceptance criterion (tests/pgm_validation/test_pgm_validation.py:38-43):
    |V| within 5e-6 pu of the power-grid-model solution."""
    net, d = network_of(name)
    assert np.max(np.abs(np.abs(d["ref_v"]) - d["pgm_u_pu"])) < 5e-6
    r = restate.nr_solve(net, tol=1e-8, max_iter=20, base_power=float(d["base_power"]))
    assert np.max(np.abs(np.abs(r["v"]) - d["pgm_u_pu"])) < 5e-6


@pytest.mark.parametrize("name", fixture_names("kat_"))
def test_mismatch_restatement(name):
    if name == "kat_update":
        pytest.skip("no mismatch vectors")
    net, d = network_of(name)
    Y = restate.ybus_reference(net)
    s_spec = net.specified_power(100e6)
    for k in ("0", "1"):
        v = d["mm_v" + k]
        f = restate.mismatch(net.bus_type, restate.power_injections(*Y, v), s_spec) * 100e6
        np.testing.assert_allclose(f, d["mm_f" + k], rtol=1e-12, atol=1e-9)


def test_ybus_update_restatement():
    d = load("kat_update")
    net = net_from(d)
    ch = net_from(d, "ch_")
    Y = restate.ybus_reference(net)
    rp, ci, va = restate.ybus_update_reference(Y, ch)
    assert np.array_equal(rp, d["y_row_ptr"]) and np.array_equal(ci, d["y_col_idx"])
    np.testing.assert_allclose(va, d["y_values"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("name", fixture_names("lu_"))
def test_lu_reference_solutions(name):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    d = load(name)
    n = len(d["row_ptr"]) - 1
    A = sp.csr_matrix((d["values"], d["col_idx"], d["row_ptr"]), shape=(n, n))
    x = spla.spsolve(A.tocsc(), d["rhs"])
    assert int(d["ref_status"]) == 0
    np.testing.assert_allclose(x, d["ref_x"], rtol=1e-10, atol=1e-12)


def test_c0_generator_matches_fixture():
    from gap_b200 import synth

    for seed in range(5):
        d = load(f"c0_seed{seed}")
        net = synth.feeder_grid(seed)
        for f in ("from_id", "to_id", "r1", "x1", "p", "q", "bus_type"):
            assert np.array_equal(getattr(net, f), d["net_" + f]), f


@pytest.mark.parametrize("name", fixture_names("pgm_"))
def test_branch_flows_match_power_grid_model(name):
    """Branch results at power-grid-model's own node voltages against its line results (the
    reference's PGM validation outputs; PGM prints node angles in degrees): the pi-model flows
    agree to 1e-6 of each quantity's largest value."""
    net, d = network_of(name)
    v = d["pgm_u_pu"] * np.exp(1j * np.deg2rad(d["pgm_u_angle"]))
    out, idx = restate.branch_flows(net, v, float(d["base_power"]), i_n=d["pgm_line_i_n"],
                                    taps=False)
    ref = d["pgm_line"]
    assert out.shape == ref.shape
    scale = np.max(np.abs(ref), axis=0)
    err = np.max(np.abs(out - ref), axis=0) / np.where(scale > 0, scale, 1.0)
    assert np.all(err < 1e-6), err


PGM_JSON = ("pgm_radial_1feeder_2nodepf", "pgm_radial_2feeder_8nodepf", "pgm_radial_3feeder_8nodepf")


def _pgm_json(d):
    import zlib

    return zlib.decompress(d["pgm_input_json_z"].tobytes()).decode()


@pytest.mark.parametrize("name", PGM_JSON)
def test_pgm_reader_solves_to_power_grid_model(name):
    """PGM input JSON -> Network (loads as negative injections) -> FP64 oracle solve: node
    voltages within the reference's acceptance criterion of power-grid-model's (5e-6 pu), and
    the same network data as the reference parser's conversion in the fixture."""
    from gap_b200 import pgm

    _, d = network_of(name)
    net, extra = pgm.read_input(_pgm_json(d))
    base = float(d["base_power"])
    r = restate.nr_solve(net, tol=1e-8, max_iter=20, base_power=base)
    assert r["converged"]
    assert np.max(np.abs(np.abs(r["v"]) - d["pgm_u_pu"])) < 5e-6
    assert np.max(np.abs(np.angle(r["v"]) - np.deg2rad(d["pgm_u_angle"]))) < 5e-6
    br = d["branch_data"]
    assert np.allclose(net.r1, br[:, 3], rtol=1e-12) and np.allclose(net.x1, br[:, 4], rtol=1e-12)
    assert np.allclose(net.b1, br[:, 5], rtol=1e-9)
    assert np.array_equal(extra["i_n"], d["pgm_line_i_n"])


@pytest.mark.parametrize("name", PGM_JSON)
def test_pgm_writer_reproduces_power_grid_model_output(name):
    """pgm.write_output on the oracle's solution (voltages, bus injections, branch results)
    against power-grid-model's whole output dataset: node, line, sym_load and source results."""
    from gap_b200 import pgm
    from helpers import compare_pgm_output, pgm_output

    _, d = network_of(name)
    net, extra = pgm.read_input(_pgm_json(d))
    base = float(d["base_power"])
    r = restate.nr_solve(net, tol=1e-12, max_iter=30, base_power=base)
    assert r["converged"]
    rp, ci, va = restate.ybus_reference(net)
    zb = float(net.u_rated[0]) ** 2 / base
    s_bus = restate.power_injections(rp, ci, va * zb, r["v"])
    fl, idx = restate.branch_flows(net, r["v"], base, i_n=extra["i_n"], taps=False)
    flows = np.zeros((net.n_branch, 9))
    flows[idx] = fl
    ours = pgm.write_output(net, extra, r["v"], s_bus, flows, base)
    worst = compare_pgm_output(ours, pgm_output(d), rtol=1e-9)
    assert {"node", "line", "sym_load", "source"} <= {c for c, _ in worst}


def test_pgm_update_dataset_to_scenarios():
    """A batch update (row and columnar forms) gives per-scenario S_spec with the updated
    loads (as negative injections) and the other appliances unchanged."""
    import json

    from gap_b200 import pgm

    _, d = network_of("pgm_radial_3feeder_8nodepf")
    doc = json.loads(_pgm_json(d))
    net, _ = pgm.read_input(doc)
    loads = doc["data"]["sym_load"]
    scale = [0.5, 1.0, 1.7]
    rows = [{"sym_load": [{"id": ld["id"], "p_specified": f * ld["p_specified"]}
                          for ld in loads]} for f in scale]
    cols = {"sym_load": [r["sym_load"] for r in rows]}
    base = float(d["base_power"])
    for upd in (rows, cols):
        s = pgm.read_update(net, upd, base)
        assert s.shape == (3, net.n_bus)
        s0 = net.specified_power(base)
        for i, f in enumerate(scale):
            assert np.allclose(s[i].real, f * s0.real, rtol=1e-12, atol=0)
            assert np.allclose(s[i].imag, s0.imag, rtol=1e-12, atol=0)


def test_pgm_writer_components_and_balances():
    """pgm.write_output on a PGM input with every component kind the reader takes (line,
    transformer, generic_branch, source, sym_load, sym_gen, shunt): each result lands under its
    component, node injections equal the node's appliances (source + generation - load), and
    the branch results at each end sum to the node injections less the shunts' power."""
    from gap_b200 import pgm

    doc = {"data": {
        "node": [{"id": 1, "u_rated": 10500.0}, {"id": 2, "u_rated": 10500.0},
                 {"id": 3, "u_rated": 10500.0}, {"id": 4, "u_rated": 10500.0}],
        "line": [{"id": 10, "from_node": 1, "to_node": 2, "from_status": 1, "to_status": 1,
                  "r1": 0.3, "x1": 0.4, "c1": 1e-7, "tan1": 0.0, "i_n": 500.0}],
        "transformer": [{"id": 11, "from_node": 2, "to_node": 3, "from_status": 1,
                         "to_status": 1, "u1": 10500.0, "u2": 10500.0, "sn": 2e6, "uk": 0.06,
                         "pk": 2e4, "i0": 0.0, "p0": 0.0, "rx_ratio": 0.1}],
        "generic_branch": [{"id": 12, "from_node": 3, "to_node": 4, "from_status": 1,
                            "to_status": 1, "r1": 0.2, "x1": 0.5, "g1": 0.0, "b1": 0.0,
                            "k": 1.0, "shift": 0.0, "sn": 1e6}],
        "source": [{"id": 20, "node": 1, "status": 1, "u_ref": 1.02}],
        "sym_load": [{"id": 30, "node": 3, "status": 1, "type": 0, "p_specified": 4e5,
                      "q_specified": 1e5}, {"id": 31, "node": 4, "status": 1, "type": 0,
                                            "p_specified": 3e5, "q_specified": 5e4}],
        "sym_gen": [{"id": 40, "node": 2, "status": 1, "type": 0, "p_specified": 1e5,
                     "q_specified": 0.0}],
        "shunt": [{"id": 50, "node": 4, "status": 1, "g1": 0.0, "b1": 1e-4}],
    }}
    net, extra = pgm.read_input(doc)
    base = 1e6
    r = restate.nr_solve(net, tol=1e-12, max_iter=30, base_power=base, policy="newton",
                         Y=restate.ybus_pi(net), jac="exact")
    assert r["converged"]
    rp, ci, va = restate.ybus_pi(net)
    zb = float(net.u_rated[0]) ** 2 / base
    s_bus = restate.power_injections(rp, ci, va * zb, r["v"])
    fl, idx = restate.branch_flows(net, r["v"], base, i_n=extra["i_n"], sn=extra["sn"])
    flows = np.zeros((net.n_branch, 9))
    flows[idx] = fl
    out = pgm.write_output(net, extra, r["v"], s_bus, flows, base)
    assert {c: len(v) for c, v in out.items()} == {"node": 4, "line": 1, "transformer": 1,
                                                   "generic_branch": 1, "source": 1,
                                                   "sym_load": 2, "sym_gen": 1}
    node = {n["id"]: n for n in out["node"]}
    src = out["source"][0]
    assert src["p"] == pytest.approx(node[1]["p"], rel=1e-12)
    assert node[2]["p"] == pytest.approx(1e5, rel=1e-9)
    assert node[3]["p"] == pytest.approx(-4e5, rel=1e-9)
    assert node[4]["q"] == pytest.approx(-5e4, rel=1e-9)
    assert out["sym_load"][0]["p"] == 4e5 and out["sym_gen"][0]["p"] == 1e5
    assert src["i"] == pytest.approx(np.hypot(src["p"], src["q"]) /
                                     (np.sqrt(3) * node[1]["u"]), rel=1e-12)
    # every node's injection flows out through its branch ends (the shunt's power is inside
    # the node injection's Y V), so with the shunt at bus 4 its reactive balance closes on Y
    ends = {1: [("line", "from")], 2: [("line", "to"), ("transformer", "from")],
            3: [("transformer", "to"), ("generic_branch", "from")],
            4: [("generic_branch", "to")]}
    for nid, lst in ends.items():
        p_out = sum(out[c][0]["p_" + e] for c, e in lst)
        assert p_out == pytest.approx(node[nid]["p"], rel=1e-9, abs=1e-3)
    gb = out["generic_branch"][0]
    assert gb["loading"] == pytest.approx(max(gb["i_from"], gb["i_to"]) / extra["i_n"][2],
                                          rel=1e-12)


def test_ybus_delta_fixed_restatement_equals_fresh_build():
    """The fixed update (the builder's own stamps) takes build(net) to build(changed net):
    branch outages, a parallel pair (one reversed) and a re-closure in one change list, with
    and without taps, within 1e-14 of the largest entry."""
    import dataclasses

    from gap_b200 import synth
    from gap_b200.engine import YbusPlan, branch_params
    from helpers import dense_of, with_parallel_branches

    net = with_parallel_branches(synth.transmission_grid(2, n=300), [0, 5, 9], reverse=[5])
    m0 = net.n_branch - 3
    yp = YbusPlan.from_network(net)
    pos = yp.branch_positions()
    changes = [3, 5, m0 + 1, 9, 3]  # out, out, out (parallel to 5), out, back in
    status = [0, 0, 0, 0, 1]
    prm = np.zeros((len(changes), 7))
    prm[:, :6] = branch_params(net)[changes]
    prm[:, 6] = status
    st = net.status.copy()
    for b, s in zip(changes, status):
        st[b] = s
    changed = dataclasses.replace(net, status=st)
    for mode, build in (("fixed_taps", restate.ybus_pi), ("fixed", restate.ybus_reference)):
        base = build(net)
        rp, ci, va = base
        assert np.array_equal(rp, yp.row_ptr) and np.array_equal(ci, yp.col_idx)
        upd = restate.ybus_delta(va, pos[changes], prm, mode)
        a, b = dense_of((rp, ci, upd)), dense_of(build(changed))
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b)), mode


def test_ybus_delta_reference_restatement_matches_reference_update():
    """The batched update's reference mode, restated, against the reference's own update."""
    d = load("kat_update")
    net = net_from(d)
    ch = net_from(d, "ch_")
    Y = restate.ybus_reference(net)
    rp, ci, va = Y
    pos, prm = [], []
    for b in range(ch.n_branch):
        f, t = int(ch.from_id[b]), int(ch.to_id[b])

        def find(r, c):
            hit = np.nonzero(ci[rp[r]:rp[r + 1]] == c)[0]
            return int(rp[r] + hit[0]) if len(hit) else -1
        pos.append([find(f, f), find(t, t), find(f, t), find(t, f)])
        prm.append([ch.r1[b], ch.x1[b], ch.g1[b], ch.b1[b], 1.0, 0.0, float(ch.status[b])])
    out = restate.ybus_delta(va, np.array(pos), np.array(prm), "reference")
    np.testing.assert_allclose(out, d["y_values"], rtol=1e-14, atol=1e-14)
