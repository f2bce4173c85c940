"""Host-side logic of libgapk.so, no GPU needed: the C ABI exports, the Y-bus pattern, and the
symbolic block-LU schedule (executed on the CPU exactly as the kernels walk it)."""

import os
import re

import numpy as np
import pytest

import schedule_emu as E
from helpers import network_of, parity_fixtures
from oracle import restate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gapk_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    from gap_b200 import _native as N

    L = N.lib()
    names = declared("gapk.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.gapk_version() >= 100


@pytest.mark.parametrize("name", [n for n in parity_fixtures() if n != "kat_update"])
def test_ybus_pattern_bit_exact(name):
    from gap_b200.engine import YbusPlan

    net, d = network_of(name)
    p = YbusPlan.from_network(net)
    assert np.array_equal(p.row_ptr, d["y_row_ptr"])
    assert np.array_equal(p.col_idx, d["y_col_idx"])


def _nets():
    from gap_b200 import synth

    out = [("c0", synth.feeder_grid(0), 1e6), ("tr300", synth.transmission_grid(3, n=300), 1e8)]
    for n in ("kat_three_bus_pv", "kat_parallel_branches", "kat_appliances"):
        net, d = network_of(n)
        out.append((n, net, 1e6))
    return out


@pytest.mark.parametrize("case", _nets(), ids=lambda c: c[0])
@pytest.mark.parametrize("jac", ["reference", "exact"])
@pytest.mark.parametrize("ordering", ["mindeg", "natural"])
@pytest.mark.parametrize("dense_min", [0, 4, -1])
def test_block_lu_schedule_solves_jacobian(case, jac, ordering, dense_min):
    from gap_b200.engine import NRPlan

    name, net, base = case
    rp, ci, vals = restate.ybus_pi(net)
    ypu = vals * (net.u_rated[0] ** 2 / base)
    plan = NRPlan(rp, ci, net.bus_type, jacobian=jac, ordering=ordering, dense_min=dense_min)
    if dense_min == -1:
        assert plan.info["n_tail"] == 0
    info = plan.info
    assert info["n_vars"] == (net.n_bus - np.sum(net.bus_type == 2)) + np.sum(net.bus_type == 0)
    rng = np.random.default_rng(0)
    v = restate.flat_start(net) * np.exp(1j * rng.normal(0, 0.05, net.n_bus))
    J, F, var, eq = E.jacobian_blocks(plan, rp, ci, ypu, v, net.bus_type, jac)
    Ff = E.factor(plan, F)
    b = rng.normal(size=J.shape[0])
    nb = info["n_block"]
    rhs = np.zeros((nb, 2))
    for k in range(nb):
        for c in range(2):
            if eq[k, c] >= 0:
                rhs[k, c] = b[eq[k, c]]
    X = E.solve(plan, Ff, rhs)
    x = np.zeros(J.shape[0])
    for k in range(nb):
        for c in range(2):
            if var[k, c] >= 0:
                x[var[k, c]] = X[k, c]
    xr = np.linalg.solve(J, b)
    assert np.max(np.abs(x - xr)) <= 1e-9 * np.max(np.abs(xr))


@pytest.mark.parametrize("seed", range(30))
def test_block_lu_schedule_on_random_networks(seed):
    """Fuzzing the symbolic analysis: the block-LU schedule (sparse levels and dense tail,
    executed on the CPU as the kernels walk it) solves the Jacobian of seeded random networks
    (parallel and out-of-service branches, PV buses, shunts, taps)."""
    from gap_b200.engine import NRPlan
    from helpers import random_network

    net = random_network(seed)
    rp, ci, vals = restate.ybus_pi(net)
    ypu = vals * (net.u_rated[0] ** 2 / 1e6)
    rng = np.random.default_rng(seed)
    v = restate.flat_start(net) * np.exp(1j * rng.normal(0, 0.05, net.n_bus))
    for dense_min in (0, 4, -1):
        plan = NRPlan(rp, ci, net.bus_type, jacobian="exact", dense_min=dense_min)
        J, F, var, eq = E.jacobian_blocks(plan, rp, ci, ypu, v, net.bus_type, "exact")
        X = E.solve(plan, E.factor(plan, F), _rhs(eq, b := rng.normal(size=J.shape[0])))
        x = np.zeros(J.shape[0])
        for k in range(plan.info["n_block"]):
            for c in range(2):
                if var[k, c] >= 0:
                    x[var[k, c]] = X[k, c]
        xr = np.linalg.solve(J, b)
        assert np.max(np.abs(x - xr)) <= 1e-9 * np.max(np.abs(xr))


def _rhs(eq, b):
    rhs = np.zeros((eq.shape[0], 2))
    for k in range(eq.shape[0]):
        for c in range(2):
            if eq[k, c] >= 0:
                rhs[k, c] = b[eq[k, c]]
    return rhs


def test_schedule_levels_respect_dependencies():
    """Every factor pair reads slots owned by strictly lower elimination-tree levels."""
    from gap_b200 import synth
    from gap_b200.engine import NRPlan

    net = synth.transmission_grid(5, n=800)
    rp, ci, _ = restate.ybus_reference(net)
    plan = NRPlan(rp, ci, net.bus_type, dense_min=4)
    nb = plan.info["n_block"]
    nnzl = plan.info["nnz_l_blocks"]
    lptr = plan.export("lptr")
    lidx = plan.export("lidx")
    lp = plan.export("level_ptr")
    ln = plan.export("level_nodes")
    level = np.zeros(nb, int)
    for h in range(len(lp) - 1):
        level[ln[lp[h]:lp[h + 1]]] = h
    col_of = np.repeat(np.arange(nb), np.diff(lptr))
    ns = nb - plan.info["n_tail"]
    level[ns:] = 10**6
    owner = np.concatenate([np.arange(nb), col_of, col_of])  # slot -> node whose level owns it
    fa = plan.export("fa_ptr")
    tg = plan.export("targets").reshape(-1, 4)
    pr = plan.export("pairs").reshape(-1, 2)
    for h in range(len(fa) - 1):
        for t in range(fa[h], fa[h + 1]):
            assert level[owner[tg[t, 0]]] == h
            for p in range(tg[t, 1], tg[t, 2]):
                assert level[owner[pr[p, 0]]] < h and level[owner[pr[p, 1]]] < h
    # parents are above children
    for k in range(ns):
        if lptr[k + 1] > lptr[k]:
            assert level[lidx[lptr[k]]] > level[k]
    # Schur targets are tail slots and read only sparse-part slots
    sch = plan.export("schur").reshape(-1, 4)
    assert len(sch) == plan.info["n_tail"] ** 2
    assert plan.info["n_tail"] > 0
    for slot, pb, pe, pos in sch:
        assert owner[slot] >= ns
        for p in range(pb, pe):
            assert owner[pr[p, 0]] < ns and owner[pr[p, 1]] < ns


def test_plan_rejects_bad_input():
    from gap_b200 import _native as N
    from gap_b200.engine import NRPlan

    with pytest.raises(N.GapkError):
        NRPlan(np.array([0, 1, 3]), np.array([0, 5, 1]), np.array([2, 0]))
    with pytest.raises(N.GapkError):
        NRPlan(np.array([0, 1, 2]), np.array([0, 1]), np.array([2, 7]))


def test_synth_generators_deterministic():
    from gap_b200 import synth

    a = synth.transmission_grid(11, n=400)
    b = synth.transmission_grid(11, n=400)
    for f in ("from_id", "to_id", "r1", "x1", "b1", "k", "theta", "p", "q", "bus_type", "u_pu"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    assert abs(a.n_branch - 1.4 * 400) <= 2
    assert np.sum(a.bus_type == 1) == 80 and np.sum(a.bus_type == 2) == 1
    f, t, valid = a.branch_index()
    br = synth.bridges(a.n_bus, f, t)
    out = synth.n_minus_1(a, 20)
    assert len(out) == 20 and not br[out].any()


def test_sparse_lu_analysis_matching_and_errors():
    from gap_b200 import _native as N
    from gap_b200.engine import SparseLU

    # zero diagonal: [[0, 1], [1, 0]] needs the row matching
    lu = SparseLU([0, 1, 2], [1, 0])
    assert lu.n == 2
    # structurally singular: both rows only in column 0
    with pytest.raises(N.GapkError):
        SparseLU([0, 1, 2], [0, 0])
    # empty / non-square-like patterns are rejected (reference: factorize() returns false)
    with pytest.raises(N.GapkError):
        SparseLU([0, 0, 0], [])
    rng = np.random.default_rng(4)
    for n in (5, 40, 200):
        A = (rng.random((n, n)) < 0.05)
        perm = rng.permutation(n)
        np.fill_diagonal(A, False)
        A[perm, np.arange(n)] = True   # a transversal exists, mostly off the diagonal
        rows, cols = np.nonzero(A)
        rp = np.zeros(n + 1, np.int32)
        np.add.at(rp, rows + 1, 1)
        assert SparseLU(np.cumsum(rp), cols).n == n


def test_contingency_params_equal_branch_outage():
    """An N-1 outage expressed as zero r1/x1/g1/b1 (the Y-bus builder's zero-admittance
    branch) gives the Y values of the network with that branch out of service, and the
    candidates are exactly the non-bridge branches (checked by removing each one)."""
    import dataclasses

    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components

    from gap_b200 import studies, synth

    net = synth.transmission_grid(6, n=120)
    outs = synth.n_minus_1(net, 10, seed=4)
    params = studies.contingency_branch_params(net, outs)
    f, t, valid = net.branch_index()
    for s, b in enumerate(outs):
        keep = valid.copy()
        keep[b] = False
        g = sp.coo_matrix((np.ones(keep.sum()), (f[keep], t[keep])), shape=(net.n_bus,) * 2)
        assert connected_components(g, directed=False)[0] == 1
        zeroed = dataclasses.replace(net, r1=params[s, :, 0], x1=params[s, :, 1],
                                     g1=params[s, :, 2], b1=params[s, :, 3])
        rp, ci, va = restate.ybus_pi(zeroed)
        A = sp.csr_matrix((va, ci, rp), shape=(net.n_bus,) * 2).toarray()
        rp2, ci2, va2 = restate.ybus_pi(studies.outage_network(net, b))
        B = sp.csr_matrix((va2, ci2, rp2), shape=(net.n_bus,) * 2).toarray()
        assert np.array_equal(A, B)
        others = np.delete(np.arange(net.n_branch), b)
        assert np.array_equal(params[s, others], studies.branch_params(net)[others])
    # every non-candidate in-service branch is a bridge
    br = synth.bridges(net.n_bus, f[valid], t[valid])
    for e in np.nonzero(valid)[0][br][:5]:
        keep = valid.copy()
        keep[e] = False
        g = sp.coo_matrix((np.ones(keep.sum()), (f[keep], t[keep])), shape=(net.n_bus,) * 2)
        assert connected_components(g, directed=False)[0] > 1


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The Python binding's ctypes structures have the C header's layout: every field at the
    offset and every struct of the size that a C compiler gives include/gapk.h."""
    import ctypes as C
    import shutil
    import subprocess

    from gap_b200 import _native as N

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"gapk_nr_plan_options": N.PlanOptions, "gapk_nr_plan_info": N.PlanInfo,
               "gapk_nr_batch_options": N.BatchOptions, "gapk_nr_inputs": N.Inputs,
               "gapk_nr_outputs": N.Outputs}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "gapk.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out.splitlines()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
