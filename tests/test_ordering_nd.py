"""Why the 10k-bus transmission grid is ordered by minimum degree, not nested dissection.

The plan factorises its sparse nodes on a level schedule and its trailing fully-dense block
(the "tail") with a dense LU per scenario.  Nested dissection orders each part before the
separator that splits it; here the parts are split by the Fiedler vector of the graph Laplacian
at the median (from a seeded start vector), the separator is the cut's boundary on either
side, and parts of fewer than 200 nodes (and every separator) are ordered by the library's
minimum degree.  The permuted pattern goes through the same analysis with the natural order,
so both orders are scored by the plan's own statistics and by a per-scenario cost model from
B200 FP32 timings of the kernels at 1024 scenarios: dense LU 2/3 N^3 flops at 18.5 TFLOP/s,
2.72 ps per Schur block pair (the model the analysis sizes the tail with) and 1.89 ps per
sparse-factor block pair (k_factor 0.85 ms for 439,290 pairs).

On this grid the top separator alone (285 nodes) is larger than minimum degree's whole tail
(253).  Dissection can shrink the dense tail (to 72 nodes with one side's boundary), but the
separator nodes that stay in the sparse part carry long columns: 2.5-180 M sparse-factor
pairs against 0.44 M, so every variant costs several times more, with 2-33x the levels."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.slow


def _model_cost(info):
    n = 2 * info["n_tail"]
    return (2.0 / 3.0 * n ** 3 / 18.5e12 + 2.72e-12 * info["n_schur_pairs"]
            + 1.89e-12 * info["n_pairs"])


def test_minimum_degree_beats_nested_dissection():
    from gap_b200 import synth
    from gap_b200 import workloads as W
    from gap_b200.engine import NRPlan, YbusPlan

    net = synth.transmission_grid(W.GRID_SEED, n=W.N_BUS)
    yp = YbusPlan.from_network(net)
    rp, ci = np.asarray(yp.row_ptr), np.asarray(yp.col_idx)
    n = len(rp) - 1
    bt = np.asarray(net.bus_type)
    P = sp.csr_matrix((np.ones(len(ci)), ci, rp), shape=(n, n))
    G = ((P + P.T) > 0).astype(float).tocsr()
    G.setdiag(0)
    G.eliminate_zeros()

    def split(nodes, side=0):
        sub = G[nodes][:, nodes].tocsr()
        lap = sp.diags(np.asarray(sub.sum(axis=1)).ravel()) - sub
        v0 = np.random.default_rng(0).random(len(nodes))
        vals, vecs = spla.eigsh(lap + 1e-6 * sp.eye(len(nodes)), k=2, sigma=0, which="LM",
                                v0=v0)
        f = vecs[:, np.argsort(vals)[1]]
        left = (f < np.median(f)) != bool(side)
        sep = np.zeros(len(nodes), bool)
        for i in np.where(left)[0]:
            if np.any(~left[sub.indices[sub.indptr[i]:sub.indptr[i + 1]]]):
                sep[i] = True
        return nodes[left & ~sep], nodes[~left], nodes[sep]

    def mindeg(nodes):
        sub = (G[nodes][:, nodes] + sp.eye(len(nodes))).tocsr()
        sub.sort_indices()
        p = NRPlan(sub.indptr, sub.indices, np.zeros(len(nodes), np.int32), jacobian="exact",
                   dense_min=-1)
        return nodes[p.export("bus_of_node")]

    def nd(nodes, depth, side):
        if depth == 0 or len(nodes) < 200:
            return mindeg(nodes)
        a, b, s = split(nodes, side)
        return np.concatenate([nd(a, depth - 1, side), nd(b, depth - 1, side), mindeg(s)])

    md = NRPlan(rp, ci, bt, jacobian="exact").info
    nonslack = np.where(bt != 2)[0]
    top = split(nonslack)[2]
    print(f"minimum degree: tail {md['n_tail']}, levels {md['n_levels']}, sparse pairs "
          f"{md['n_pairs']}, model {_model_cost(md) * 1e6:.2f} us; top separator {len(top)} nodes")
    assert len(top) > md["n_tail"]
    for depth, side in ((1, 0), (1, 1), (2, 0), (2, 1)):
        order = np.concatenate([nd(nonslack, depth, side), np.where(bt == 2)[0]])
        Pp = P[order][:, order].tocsr()
        Pp.sort_indices()
        info = NRPlan(Pp.indptr, Pp.indices, bt[order], jacobian="exact",
                      ordering="natural").info
        print(f"nested dissection depth {depth} side {side}: tail {info['n_tail']}, levels "
              f"{info['n_levels']}, sparse pairs {info['n_pairs']}, "
              f"model {_model_cost(info) * 1e6:.2f} us")
        assert _model_cost(info) > 2 * _model_cost(md)
        assert info["n_levels"] > 1.5 * md["n_levels"]
