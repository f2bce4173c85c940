"""Test helper: executes an NRPlan's exported factor / solve schedule on the CPU in numpy,
exactly as the device kernels walk it (level by level, phase A then phase B), so the host
symbolic analysis can be checked without a GPU."""

import numpy as np

from oracle import restate


def jacobian_blocks(plan, row_ptr, col_idx, ypu, v, bus_type, mode):
    """Reference-order Jacobian (oracle) scattered into the plan's slot storage."""
    J = restate.jacobian(row_ptr, col_idx, ypu, v, bus_type, mode=mode, drop=False).toarray()
    info = plan.info
    nb, ns = info["n_block"], info["n_slots"]
    si = plan.export("slot_info").reshape(ns, 4)
    ssp = plan.export("slot_src_ptr")
    node_of_bus = np.full(len(bus_type), -1)
    bon = plan.export("bus_of_node")
    node_of_bus[bon] = np.arange(nb)
    var = plan.export("var_of_comp").reshape(nb, 2)
    eq = plan.export("eq_of_comp").reshape(nb, 2)
    F = np.zeros((ns, 2, 2))
    for s in range(ns):
        rb, cb, b, e = si[s]
        rn, cn = node_of_bus[rb], node_of_bus[cb]
        blk = np.zeros((2, 2))
        if b < e or rb == cb:
            for r in range(2):
                for c in range(2):
                    er, vc = eq[rn, r], var[cn, c]
                    if er >= 0 and vc >= 0:
                        blk[r, c] = J[er, vc]
            if rb == cb and eq[rn, 1] < 0:
                blk[1, 1] = 1.0
        F[s] = blk
    return J, F, var, eq


def factor(plan, F):
    """Returns (F, D): factored slot storage of the sparse part and the dense tail's LU
    (unit-lower L below the diagonal, U on and above it; None when there is no tail)."""
    F = F.copy()
    info = plan.info
    L = info["n_levels"]
    fa = plan.export("fa_ptr")
    tg = plan.export("targets").reshape(-1, 4)
    pr = plan.export("pairs").reshape(-1, 2)
    fb = plan.export("fb_ptr")
    sc = plan.export("scale").reshape(-1, 2)
    for h in range(L):
        for t in range(fa[h], fa[h + 1]):
            slot, pb, pe, isd = tg[t]
            acc = F[slot].copy()
            for p in range(pb, pe):
                acc -= F[pr[p, 0]] @ F[pr[p, 1]]
            if isd & 1:
                acc = np.linalg.inv(acc)
            F[slot] = acc
        for t in range(fb[h], fb[h + 1]):
            F[sc[t, 0]] = F[sc[t, 0]] @ F[sc[t, 1]]
    T = info["n_tail"]
    if T == 0:
        return F, None
    D = np.zeros((2 * T, 2 * T))
    for slot, pb, pe, pos in plan.export("schur").reshape(-1, 4):
        acc = F[slot].copy() if (pos >> 30) & 1 else np.zeros((2, 2))
        for p in range(pb, pe):
            acc -= F[pr[p, 0]] @ F[pr[p, 1]]
        r, c = divmod(pos & ((1 << 30) - 1), T)
        D[2 * r:2 * r + 2, 2 * c:2 * c + 2] = acc
    n = 2 * T
    for j in range(n):
        D[j + 1:, j] /= D[j, j]
        D[j + 1:, j + 1:] -= np.outer(D[j + 1:, j], D[j, j + 1:])
    return F, D


def solve(plan, FD, rhs_nodes):
    F, D = FD
    info = plan.info
    nb = info["n_block"]
    nnzl = info["nnz_l_blocks"]
    T = info["n_tail"]
    ns = nb - T
    L = info["n_levels"]
    lp = plan.export("level_ptr")
    ln = plan.export("level_nodes")
    rptr = plan.export("rptr")
    rl = plan.export("rlist").reshape(-1, 2)
    lptr = plan.export("lptr")
    lidx = plan.export("lidx")
    X = rhs_nodes.copy()
    for h in range(L):
        for t in range(lp[h], lp[h + 1]):
            k = ln[t]
            acc = X[k].copy()
            for q in range(rptr[k], rptr[k + 1]):
                acc -= F[rl[q, 0]] @ X[rl[q, 1]]
            X[k] = acc
    if T:
        for k in range(ns, nb):
            acc = X[k].copy()
            for q in range(rptr[k], rptr[k + 1]):
                acc -= F[rl[q, 0]] @ X[rl[q, 1]]
            X[k] = acc
        y = X[ns:].reshape(-1).copy()
        n = 2 * T
        for i in range(n):
            y[i] -= D[i, :i] @ y[:i]
        for i in range(n - 1, -1, -1):
            y[i] = (y[i] - D[i, i + 1:] @ y[i + 1:]) / D[i, i]
        X[ns:] = y.reshape(T, 2)
    for h in range(L - 1, -1, -1):
        for t in range(lp[h], lp[h + 1]):
            k = ln[t]
            acc = X[k].copy()
            for p in range(lptr[k], lptr[k + 1]):
                acc -= F[nb + nnzl + p] @ X[lidx[p]]
            X[k] = F[k] @ acc
    return X
