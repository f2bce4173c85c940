"""Seeded synthetic power-flow workloads.

All generators draw from numpy's PCG64 (`np.random.default_rng(seed)`) in the fixed order
documented per function, so a (generator, seed, size) triple names one network bit for bit.

* `feeder_grid`      -- 10 kV meshed ring feeder: random recursive tree plus 10 % tie lines,
                        one slack, constant-power loads, no PV (the 200-bus CPU-runnable case).
* `transmission_grid`-- transmission-like random geometric grid on a 100 MVA base: spanning
                        tree plus nearest-neighbour ties (mean degree ~2.8), 10 % transformers
                        with tap and phase shift, 20 % PV buses, 2 % shunts.
* `load_scenarios`   -- per-bus lognormal load scaling of a base case.
* `n_minus_1`        -- branch outages that keep the grid connected (non-bridge branches).
"""

from __future__ import annotations

import math

import numpy as np

from .network import LOADGEN, PQ, PV, SHUNT, SLACK, Network


def feeder_grid(seed: int = 0, n: int = 200, tie_frac: float = 0.10) -> Network:
    """Meshed 10 kV feeder.  Draw order: parents (i=1..n-1, parent ~ U{0..i-1}); tie pairs
    (rejection-sampled until round(tie_frac*n) distinct new non-self pairs); r1 ~ U[0.05,0.5]
    Ohm and x1 ~ U[0.05,0.4] Ohm for all branches (tree branches first, then ties); load
    p ~ U[0.05,0.5] MW for buses 1..n-1, q = 0.3 p.  Bus 0 is the slack at u_ref = 1.0 pu.
    Loads are negative bus injections (W / var), as the reference's Python tests pass them."""
    rng = np.random.default_rng(seed)
    parent = np.array([rng.integers(0, i) for i in range(1, n)], dtype=np.int64)
    edges = {(min(i, int(p)), max(i, int(p))) for i, p in zip(range(1, n), parent)}
    frm = list(range(1, n))
    to = [int(p) for p in parent]
    n_tie = int(round(tie_frac * n))
    ties = 0
    while ties < n_tie:
        a, b = (int(v) for v in rng.integers(0, n, size=2))
        if a == b:
            continue
        key = (min(a, b), max(a, b))
        if key in edges:
            continue
        edges.add(key)
        frm.append(a)
        to.append(b)
        ties += 1
    m = len(frm)
    r1 = rng.uniform(0.05, 0.5, size=m)
    x1 = rng.uniform(0.05, 0.4, size=m)
    p_mw = rng.uniform(0.05, 0.5, size=n - 1)
    p = np.zeros(n)
    q = np.zeros(n)
    p[1:] = -p_mw * 1e6
    q[1:] = -0.3 * p_mw * 1e6
    bt = np.full(n, PQ, np.int32)
    bt[0] = SLACK
    return Network.build(bus_id=np.arange(n), u_rated=np.full(n, 10e3), bus_type=bt,
                         u_pu=np.ones(n), p=p, q=q, from_id=frm, to_id=to, r1=r1, x1=x1)


TRANSMISSION_KV = 138.0
BASE_MVA = 100.0
# Per-bus loads are p ~ U[0,1] * LOAD_SCALE pu.  With LOAD_SCALE = 1 (0-100 MW at every bus of
# a 100 MVA-base grid with x ~ U[0.01,0.2]) no power-flow solution exists at 10k buses: a
# load-scale continuation of the 10k-bus base case ends at its nose point near 0.23
# (tests/test_workload_loading.py), and lognormal scenarios (sigma 0.1) around 0.2 already
# fail; 0.05 leaves every scenario solvable.
LOAD_SCALE = 0.05


def transmission_grid(seed: int = 0, n: int = 10_000, mean_degree: float = 2.8,
                      trafo_frac: float = 0.10, pv_frac: float = 0.20,
                      shunt_frac: float = 0.02, load_scale: float = LOAD_SCALE,
                      cover_hops: int = 2) -> Network:
    """Transmission-like grid, per-unit data on a 100 MVA base converted to Ohm / S at
    138 kV so that the reference's single-voltage-base per-unit step recovers them.

    Draw order: bus coordinates (n x 2 uniform); tree attachment (bus i, in index order,
    joins the nearest of the buses 0..i-1 among its k-nearest candidates, else a random
    earlier bus); extra ties (random bus, random one of its 6 nearest neighbours, until
    m = round(mean_degree*n/2)); per branch x ~ U[0.01,0.2], r = x / U[5,15], b ~ U[0,0.05];
    transformer set (round(trafo_frac*m) branches drawn from the bridges first, then from the
    other branches), tap ~ U[0.95,1.05], shift ~ U[0,10] deg (transformers carry b = 0); PV placement (random order, a bus becomes PV while it is more than
    cover_hops hops from every voltage-controlled bus, then random top-up to pv_frac of the
    buses) and |V| setpoints ~ U[0.98,1.05]; shunt set (shunt_frac of buses) with
    b ~ U[-0.05,0.05] pu; loads p ~ U[0,1] pu * load_scale, q = U[0.1,0.4] p.  PV generation
    is local: each bus's load is assigned to its nearest voltage-controlled bus (multi-source
    BFS in hops) and every PV bus generates its region's load; the slack supplies its own
    region and the losses.  The slack is the bus closest to the centre of the square, at
    1.0 pu."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    xy = rng.random((n, 2))
    tree = cKDTree(xy)
    frm, to = [], []
    edges = set()
    # spanning tree: nearest earlier bus among 16 nearest neighbours, else random earlier bus
    kq = min(16, n)
    _, nbr = tree.query(xy, k=kq)
    nbr = np.atleast_2d(nbr)
    fallback = rng.random(n)
    for i in range(1, n):
        cand = [int(j) for j in nbr[i] if j < i]
        j = cand[0] if cand else int(fallback[i] * i)
        frm.append(i)
        to.append(j)
        edges.add((min(i, j), max(i, j)))
    m_target = int(round(mean_degree * n / 2))
    k6 = min(7, n)
    _, nb6 = tree.query(xy, k=k6)
    nb6 = np.atleast_2d(nb6)
    guard = 0
    while len(frm) < m_target and guard < 50 * n:
        guard += 1
        a = int(rng.integers(0, n))
        b = int(nb6[a][int(rng.integers(1, k6))]) if k6 > 1 else a
        if a == b:
            continue
        key = (min(a, b), max(a, b))
        if key in edges:
            continue
        edges.add(key)
        frm.append(a)
        to.append(b)
    m = len(frm)
    x_pu = rng.uniform(0.01, 0.2, size=m)
    r_pu = x_pu / rng.uniform(5.0, 15.0, size=m)
    b_pu = rng.uniform(0.0, 0.05, size=m)
    # transformers sit on radial connections: drawn from the bridge branches (a phase shift
    # there rotates the angles behind it instead of driving loop flow), then from the rest
    is_br = bridges(n, frm, to)
    n_tr = int(round(trafo_frac * m))
    cand = rng.permutation(np.nonzero(is_br)[0])
    other = rng.permutation(np.nonzero(~is_br)[0])
    pick = np.concatenate([cand, other])[:n_tr]
    is_tr = np.zeros(m, bool)
    is_tr[pick] = True
    tap = np.where(is_tr, rng.uniform(0.95, 1.05, size=m), 1.0)
    shift = np.where(is_tr, np.deg2rad(rng.uniform(0.0, 10.0, size=m)), 0.0)
    b_pu = np.where(is_tr, 0.0, b_pu)
    slack = int(np.argmin(np.sum((xy - 0.5) ** 2, axis=1)))
    adj = [[] for _ in range(n)]
    for a, b in zip(frm, to):
        adj[a].append(b)
        adj[b].append(a)
    # PV placement: buses in random order become PV while they are more than `cover_hops`
    # hops from every voltage-controlled bus (slack included), then the PV set is topped up
    # to pv_frac of the buses at random.
    n_pv = int(round(pv_frac * n))
    dist = np.full(n, np.iinfo(np.int64).max)
    is_pv = np.zeros(n, bool)

    def cover(src):
        dist[src] = 0
        frontier = [src]
        for d in range(1, cover_hops + 1):
            nxt = []
            for u in frontier:
                for w in adj[u]:
                    if dist[w] > d:
                        dist[w] = d
                        nxt.append(w)
            frontier = nxt

    cover(slack)
    order = rng.permutation(n)
    placed = 0
    for v in order:
        if placed >= n_pv:
            break
        if v != slack and dist[v] > cover_hops:
            is_pv[v] = True
            placed += 1
            cover(int(v))
    rest = np.array([v for v in rng.permutation(n) if v != slack and not is_pv[v]], np.int64)
    is_pv[rest[: max(0, n_pv - int(is_pv.sum()))]] = True
    pv = np.nonzero(is_pv)[0]
    bt = np.full(n, PQ, np.int32)
    bt[pv] = PV
    bt[slack] = SLACK
    vset = np.ones(n)
    vset[pv] = rng.uniform(0.98, 1.05, size=len(pv))
    n_sh = int(round(shunt_frac * n))
    sh_bus = rng.permutation(n)[:n_sh]
    sh_b = rng.uniform(-0.05, 0.05, size=n_sh)
    p_load = rng.uniform(0.0, 1.0, size=n) * load_scale
    q_load = rng.uniform(0.1, 0.4, size=n) * p_load
    p_load[slack] = 0.0
    q_load[slack] = 0.0
    # local dispatch: every bus's load is served by its nearest (in hops) voltage-controlled
    # bus; each PV bus generates the load of its region, the slack covers its own region and
    # the losses
    owner = np.full(n, -1, np.int64)
    src = [slack] + [int(v) for v in pv]
    for s_ in src:
        owner[s_] = s_
    frontier = list(src)
    while frontier:
        nxt = []
        for u in frontier:
            for w in adj[u]:
                if owner[w] < 0:
                    owner[w] = owner[u]
                    nxt.append(w)
        frontier = nxt
    owner[owner < 0] = slack
    region = np.zeros(n)
    np.add.at(region, owner, p_load)
    p_gen = np.zeros(n)
    p_gen[pv] = region[pv]
    u = TRANSMISSION_KV * 1e3
    zb = u * u / (BASE_MVA * 1e6)
    sbase = BASE_MVA * 1e6
    p = (p_gen - p_load) * sbase
    q = -q_load * sbase
    return Network.build(
        bus_id=np.arange(n), u_rated=np.full(n, u), bus_type=bt, u_pu=vset, p=p, q=q,
        from_id=frm, to_id=to, r1=r_pu * zb, x1=x_pu * zb, b1=b_pu / zb, k=tap, theta=shift,
        app_node=sh_bus, app_type=np.full(n_sh, SHUNT), app_b1=sh_b / zb,
        app_g1=np.zeros(n_sh))


def load_scenarios(net: Network, n_scen: int, sigma: float = 0.1, seed: int = 1,
                   base_power: float = BASE_MVA * 1e6):
    """S_spec (per unit, complex128 [n_scen, n_bus]) for n_scen load scenarios: every bus's
    load (negative part of P and Q) scaled by its own lognormal(0, sigma) factor per
    scenario; generation unchanged.  Scenario 0 draws its factors like the others."""
    rng = np.random.default_rng(seed)
    s0 = net.specified_power(base_power)
    load = np.minimum(s0.real, 0.0) + 1j * np.minimum(s0.imag, 0.0)
    gen = s0 - load
    f = rng.lognormal(0.0, sigma, size=(n_scen, net.n_bus))
    return gen[None, :] + f * load[None, :]


def bridges(n: int, frm, to) -> np.ndarray:
    """Boolean mask of bridge edges (Tarjan, iterative)."""
    frm = np.asarray(frm)
    to = np.asarray(to)
    m = len(frm)
    adj = [[] for _ in range(n)]
    for e in range(m):
        adj[frm[e]].append((to[e], e))
        adj[to[e]].append((frm[e], e))
    disc = [-1] * n
    low = [0] * n
    is_bridge = np.zeros(m, bool)
    t = 0
    for root in range(n):
        if disc[root] >= 0:
            continue
        stack = [(root, -1, iter(adj[root]))]
        disc[root] = low[root] = t
        t += 1
        while stack:
            u, pe, it = stack[-1]
            adv = False
            for w, e in it:
                if e == pe:
                    continue
                if disc[w] < 0:
                    disc[w] = low[w] = t
                    t += 1
                    stack.append((w, e, iter(adj[w])))
                    adv = True
                    break
                low[u] = min(low[u], disc[w])
            if not adv:
                stack.pop()
                if stack:
                    p = stack[-1][0]
                    low[p] = min(low[p], low[u])
                    if low[u] > disc[p]:
                        is_bridge[pe] = True
    return is_bridge


def n_minus_1(net: Network, count: int, seed: int = 2) -> np.ndarray:
    """Indices of `count` distinct in-service non-bridge branches (outage candidates)."""
    f, t, valid = net.branch_index()
    br = bridges(net.n_bus, f[valid], t[valid])
    cand = np.nonzero(valid)[0][~br]
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(cand, size=min(count, len(cand)), replace=False))


def grid_sizes(count: int, lo: int = 500, hi: int = 20_000, seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))).astype(int)


def dc_start(net: Network, base_power: float = BASE_MVA * 1e6, s_spec=None) -> np.ndarray:
    """Initial voltages for the transmission workloads: angles from a DC power flow
    (B' theta = P + phase-shift injections, x scaled by the tap ratio, slack angle 0),
    magnitudes at the SLACK/PV setpoints and 1.0 for PQ buses.  Host-side input preparation
    (scipy sparse solve); returns complex128 [n_bus]."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    f, t, valid = net.branch_index()
    zb = float(net.u_rated[0]) ** 2 / base_power
    ff, tt = f[valid], t[valid]
    x = net.x1[valid] / zb * net.k[valid]
    x = np.where(np.abs(x) > 1e-9, x, 1e-9)
    b = 1.0 / x
    sh = net.theta[valid]
    n = net.n_bus
    B = sp.coo_matrix((np.r_[b, b, -b, -b], (np.r_[ff, tt, ff, tt], np.r_[ff, tt, tt, ff])),
                      shape=(n, n)).tocsr()
    P = (net.specified_power(base_power) if s_spec is None else np.asarray(s_spec)).real
    Ps = np.zeros(n)
    np.add.at(Ps, ff, b * sh)
    np.add.at(Ps, tt, -b * sh)
    keep = net.bus_type != SLACK
    ang = np.zeros(n)
    if keep.any():
        ang[keep] = spla.spsolve(B[keep][:, keep].tocsc(), (P + Ps)[keep])
    vm = np.where(net.bus_type == PQ, 1.0, net.u_pu)
    return vm * np.exp(1j * ang)
