"""Shared test helpers: golden fixtures -> Network objects."""

import glob
import os

import numpy as np

from gap_b200.network import Network

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def net_from(d, prefix="net_"):
    kw = {k[len(prefix):]: d[k] for k in d if k.startswith(prefix)}
    return Network(**kw)


def pgm_network(d):
    from gap_b200.api import network_from_simple_lists

    return network_from_simple_lists(d["bus_data"].tolist(), d["branch_data"].tolist())


def network_of(name):
    d = load(name)
    if name.startswith("pgm_"):
        return pgm_network(d), d
    return net_from(d), d


def parity_fixtures():
    return fixture_names("kat_") + fixture_names("c0_") + fixture_names("pgm_")


def pgm_output(d):
    """power-grid-model's output dataset stored with a PGM fixture (zlib-compressed JSON)."""
    import json
    import zlib

    return json.loads(zlib.decompress(d["pgm_output_json_z"].tobytes()).decode())


def compare_pgm_output(ours, ref, rtol):
    """Largest relative difference per (component, attribute) between two PGM output datasets
    (matched by id; relative to the attribute's largest magnitude in `ref`); asserts every
    component and record of `ref` is present and each difference is below rtol."""
    worst = {}
    for comp, recs in ref.items():
        if comp == "meta" or not isinstance(recs, list):
            continue
        mine = {r["id"]: r for r in ours.get(comp, [])}
        assert set(mine) == {r["id"] for r in recs}, comp
        for key in recs[0]:
            if key in ("id",):
                continue
            if key == "energized":
                assert all(bool(mine[r["id"]][key]) == bool(r[key]) for r in recs), comp
                continue
            a = np.array([float(mine[r["id"]][key]) for r in recs])
            b = np.array([float(r[key]) for r in recs])
            scale = max(float(np.max(np.abs(b))), 1e-30)
            worst[(comp, key)] = float(np.max(np.abs(a - b))) / scale
    bad = {k: w for k, w in worst.items() if not w < rtol}
    assert not bad, bad
    return worst


def random_network(seed, n_max=40):
    """A seeded random small network for fuzzing the device path against the oracle: a random
    tree plus extra branches (parallel duplicates and an out-of-service one among them), 10 kV
    per-unit-like impedances, a few transformers with taps / phase shifts, shunts, PV buses
    (about 20%), one slack (bus 0), light loads and generation, bus IDs shuffled."""
    from gap_b200.network import LOADGEN, PQ, PV, SHUNT, SLACK, Network

    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(3, n_max + 1))
    ids = rng.permutation(np.arange(10, 10 + 3 * n, 3))[:n]
    frm, to = [], []
    for i in range(1, n):
        frm.append(int(rng.integers(0, i)))
        to.append(i)
    for _ in range(int(rng.integers(0, max(2, n // 3)))):
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        frm.append(a)
        to.append(b)
    if len(frm) > 2 and rng.random() < 0.5:  # a parallel duplicate of an existing branch
        j = int(rng.integers(0, len(frm)))
        frm.append(frm[j])
        to.append(to[j])
    m = len(frm)
    zb = 10e3 ** 2 / 1e6
    x = rng.uniform(0.02, 0.12, m) * zb
    r = x * rng.uniform(0.1, 0.5, m)
    b = rng.uniform(0.0, 0.02, m) / zb
    k = np.ones(m)
    th = np.zeros(m)
    tr = rng.random(m) < 0.15
    k[tr] = rng.uniform(0.95, 1.05, tr.sum())
    th[tr] = rng.uniform(0.0, 0.1, tr.sum())
    status = np.ones(m, np.int32)
    if m > n:  # an extra branch out of service (the tree stays connected)
        status[int(rng.integers(n - 1, m))] = 0
    bt = np.full(n, PQ, np.int32)
    bt[0] = SLACK
    pv = rng.random(n) < 0.2
    pv[0] = False
    bt[pv] = PV
    u_pu = np.ones(n)
    u_pu[0] = rng.uniform(1.0, 1.05)
    u_pu[pv] = rng.uniform(0.99, 1.04, pv.sum())
    p = np.zeros(n)
    q = np.zeros(n)
    load = rng.uniform(0.0, 0.25e6, n)
    p[1:] = -load[1:]
    q[1:] = -load[1:] * rng.uniform(0.1, 0.4, n - 1)
    p[pv] = rng.uniform(0.05e6, 0.3e6, pv.sum())
    app_node, app_type, app_g1, app_b1 = [], [], [], []
    for i in np.nonzero(rng.random(n) < 0.15)[0]:
        app_node.append(int(ids[i]))
        app_type.append(SHUNT)
        app_g1.append(0.0)
        app_b1.append(float(rng.uniform(-0.02, 0.02) / zb))
    return Network.build(bus_id=ids, u_rated=np.full(n, 10e3), bus_type=bt, u_pu=u_pu, p=p, q=q,
                         from_id=ids[frm], to_id=ids[to], r1=r, x1=x, b1=b, k=k, theta=th,
                         status=status, app_node=app_node, app_type=app_type, app_g1=app_g1,
                         app_b1=app_b1)


def with_parallel_branches(net, branches, reverse=()):
    """Copy of `net` with a duplicate of each listed branch appended (new ids; the copies of
    the branches in `reverse` run to -> from), so that the Y pattern holds duplicate entries."""
    import dataclasses

    branches = list(branches)
    rev = np.isin(branches, list(reverse))
    kw = {}
    for name in ("r1", "x1", "g1", "b1", "k", "theta", "status"):
        a = getattr(net, name)
        kw[name] = np.concatenate([a, a[branches]])
    f = net.from_id[branches]
    t = net.to_id[branches]
    kw["from_id"] = np.concatenate([net.from_id, np.where(rev, t, f)]).astype(net.from_id.dtype)
    kw["to_id"] = np.concatenate([net.to_id, np.where(rev, f, t)]).astype(net.to_id.dtype)
    start = int(max(np.max(net.br_id), np.max(net.bus_id), np.max(net.app_id, initial=0))) + 1
    kw["br_id"] = np.concatenate([net.br_id, np.arange(start, start + len(branches))]).astype(
        net.br_id.dtype)
    return dataclasses.replace(net, **kw)


def dense_of(Y):
    """CSR (row_ptr, col_idx, values) with duplicates summed, as a dense complex matrix."""
    import scipy.sparse as sp

    rp, ci, va = Y
    n = len(rp) - 1
    return sp.csr_matrix((np.array(va), np.array(ci), np.array(rp)), shape=(n, n)).toarray()
