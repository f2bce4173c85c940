"""ORACLE TEST INFRASTRUCTURE -- FP64 CPU restatement of the reference's Newton-Raphson path.

Test-only: imported by tests/, by the smoke check and by bench.py's CPU-baseline leg, as the
checker; the product never calls it.  Each function names the reference lines it restates.
Where the reference is silent or cannot run (transformer tap/phase-shift stamps, PV buses at
scale, batched scenarios, gradients) the restatement extends it with textbook formulas, and
says so; those parts are checked against physics (power balance, finite differences) instead.

Pinning: the reference-mode functions are checked against the reference's own CPU code built
from source (oracle/_ref/libgapref.so) and against the golden PGM outputs under tests/golden/.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from gap_b200.network import PQ, PV, SLACK, Network

# ----------------------------------------------------------------------------------------
# Y-bus
# ----------------------------------------------------------------------------------------


def ybus_reference(net: Network):
    """CPUAdmittanceMatrix::build_admittance_matrix
    (src/admittance/cpu/cpu_admittance_matrix.cpp:44-202), bit for bit.

    Shunt appliances first (:88-97), then branch stamps in input order (:100-140): series
    y = (r - jx)/(r^2 + x^2) (0 when r^2 + x^2 <= 1e-12), both diagonals += y + g1 + j b1/2,
    off-diagonals -y at (f,t) and (t,f); tap k and shift theta ignored; duplicates kept;
    diagonal triplets appended last (:143-145); stable (row, col) sort (:151-154); CSR.
    Returns (row_ptr int32[n+1], col_idx int32[nnz], values complex128[nnz]) in Siemens."""
    n = net.n_bus
    f, t, valid = net.branch_index()
    dre = [0.0] * n
    dim = [0.0] * n
    sb, sg, sbb = net.shunt_index()
    for i, g, b in zip(sb.tolist(), np.asarray(sg).tolist(), np.asarray(sbb).tolist()):
        dre[i] += g
        dim[i] += b
    rows, cols, vre, vim = [], [], [], []
    r1 = net.r1.tolist()
    x1 = net.x1.tolist()
    g1 = net.g1.tolist()
    b1 = net.b1.tolist()
    for b in range(net.n_branch):
        if not valid[b]:
            continue
        fb, tb = int(f[b]), int(t[b])
        r, x = r1[b], x1[b]
        z2 = r * r + x * x
        if z2 > 1e-12:
            yr, yi = r / z2, -x / z2
        else:
            yr, yi = 0.0, 0.0
        sre = (yr + g1[b]) + 0.0
        sim = (yi + 0.0) + b1[b] / 2.0
        dre[fb] += sre
        dim[fb] += sim
        dre[tb] += sre
        dim[tb] += sim
        rows += [fb, tb]
        cols += [tb, fb]
        vre += [-yr, -yr]
        vim += [-yi, -yi]
    rows += list(range(n))
    cols += list(range(n))
    vre += dre
    vim += dim
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    order = np.argsort(rows * max(n, 1) + cols, kind="stable")
    rows, cols = rows[order], cols[order]
    # keep exact component values (no complex arithmetic on them)
    vals = np.empty(len(order), np.complex128)
    vals.real = np.asarray(vre, np.float64)[order]
    vals.imag = np.asarray(vim, np.float64)[order]
    row_ptr = np.zeros(n + 1, np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    return row_ptr, cols.astype(np.int32), vals


def ybus_pi(net: Network):
    """Y-bus with transformer taps and phase shifts (NOT in the reference, which ignores
    BranchData::k / ::theta, types.h:250-251).  Standard pi model with the off-nominal tap
    t = k*exp(j*theta) on the from side:  Y_ff = (y + ysh)/k^2, Y_tt = y + ysh,
    Y_ft = -y/conj(t), Y_tf = -y/t, with ysh = g1 + j*b1/2 per end (the reference's end
    stamp).  Same CSR pattern and order as ybus_reference; for k == 1 and theta == 0 the values
    equal the reference's bit for bit (the reference arithmetic is used for those branches)."""
    row_ptr, col_idx, vals = ybus_reference(net)
    n = net.n_bus
    f, t, valid = net.branch_index()
    # recompute with taps: rebuild diagonal from scratch in the same accumulation order
    dre = [0.0] * n
    dim = [0.0] * n
    sb, sg, sbb = net.shunt_index()
    for i, g, b in zip(sb.tolist(), np.asarray(sg).tolist(), np.asarray(sbb).tolist()):
        dre[i] += g
        dim[i] += b
    off = {}
    order_keys = []
    for b in range(net.n_branch):
        if not valid[b]:
            continue
        fb, tb = int(f[b]), int(t[b])
        r, x = float(net.r1[b]), float(net.x1[b])
        z2 = r * r + x * x
        yr, yi = (r / z2, -x / z2) if z2 > 1e-12 else (0.0, 0.0)
        kk, th = float(net.k[b]), float(net.theta[b])
        sre = (yr + float(net.g1[b])) + 0.0
        sim = (yi + 0.0) + float(net.b1[b]) / 2.0
        if kk == 1.0 and th == 0.0:
            ff = (sre, sim)
            tt = (sre, sim)
            ft = (-yr, -yi)
            tf = (-yr, -yi)
        else:
            y = complex(yr, yi)
            tap = kk * complex(math.cos(th), math.sin(th))
            yff = complex(sre, sim) / (kk * kk)
            yft = -y / tap.conjugate()
            ytf = -y / tap
            ff = (yff.real, yff.imag)
            tt = (sre, sim)
            ft = (yft.real, yft.imag)
            tf = (ytf.real, ytf.imag)
        dre[fb] += ff[0]
        dim[fb] += ff[1]
        dre[tb] += tt[0]
        dim[tb] += tt[1]
        order_keys.append(((fb, tb), ft))
        order_keys.append(((tb, fb), tf))
    # off-diagonal entries appear in CSR in branch order within each (row, col)
    out = vals.copy()
    slot = {}
    for i in range(n):
        for p in range(row_ptr[i], row_ptr[i + 1]):
            j = int(col_idx[p])
            if j == i:
                continue
            slot.setdefault((i, j), []).append(p)
    used = {}
    for key, v in order_keys:
        if key[0] == key[1]:
            continue
        k = used.get(key, 0)
        p = slot[key][k]
        used[key] = k + 1
        out[p] = complex(v[0], v[1])
    # diagonal: the diagonal triplet is the last (i,i) entry of row i in CSR order (self-loop
    # branch triplets precede it thanks to the stable sort)
    for i in range(n):
        ps = [p for p in range(row_ptr[i], row_ptr[i + 1]) if col_idx[p] == i]
        if ps:
            out[ps[-1]] = complex(dre[i], dim[i])
    return row_ptr, col_idx, out


# ----------------------------------------------------------------------------------------
# Newton-Raphson
# ----------------------------------------------------------------------------------------


def var_maps(bus_type):
    """Variable / equation maps of CPUNewtonRaphson (cpu_newton_raphson.cpp:530-541,
    603-627): columns are theta of every non-slack bus in bus order, then |V| of every PQ bus
    in bus order; rows are, per non-slack bus in bus order, P then (PQ only) Q.  All SLACK
    buses are treated as fixed (the reference excludes only the first SLACK from the angle
    variables, which makes its system non-square when several SLACK buses exist)."""
    bt = np.asarray(bus_type)
    n = bt.shape[0]
    ang = np.full(n, -1, np.int64)
    mag = np.full(n, -1, np.int64)
    nonslack = np.nonzero(bt != SLACK)[0]
    ang[nonslack] = np.arange(len(nonslack))
    pq = np.nonzero(bt == PQ)[0]
    mag[pq] = len(nonslack) + np.arange(len(pq))
    # equation rows
    peq = np.full(n, -1, np.int64)
    qeq = np.full(n, -1, np.int64)
    r = 0
    for i in range(n):
        if bt[i] == SLACK:
            continue
        peq[i] = r
        r += 1
        if bt[i] == PQ:
            qeq[i] = r
            r += 1
    return ang, mag, peq, qeq, r


def power_injections(row_ptr, col_idx, vals, v):
    """S = V * conj(Y V), summing duplicate entries (cpu_newton_raphson.cpp:296-337)."""
    n = len(row_ptr) - 1
    Y = sp.csr_matrix((vals, col_idx, row_ptr), shape=(n, n))
    return v * np.conj(Y @ v)


def mismatch(bus_type, s_calc, s_spec):
    """Delta = S_calc - S_spec in the reference's interleaved order
    (cpu_newton_raphson.cpp:268-289)."""
    ang, mag, peq, qeq, ne = var_maps(bus_type)
    d = np.zeros(ne)
    ok = peq >= 0
    d[peq[ok]] = (s_calc.real - s_spec.real)[ok]
    okq = qeq >= 0
    d[qeq[okq]] = (s_calc.imag - s_spec.imag)[okq]
    return d


def _dedupe(row_ptr, col_idx, vals, mode):
    """COO of Y with duplicate (i, j) entries resolved: 'reference' keeps the LAST entry in
    CSR order (the dense G/B copy of cpu_newton_raphson.cpp:585-597 overwrites), 'exact'
    sums them (the true derivative of the SpMV the mismatch uses)."""
    n = len(row_ptr) - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    cols = np.asarray(col_idx, np.int64)
    key = rows * n + cols
    if mode == "exact":
        uk, inv = np.unique(key, return_inverse=True)
        v = np.zeros(len(uk), np.complex128)
        np.add.at(v, inv, vals)
        return uk // n, uk % n, v
    # last occurrence
    rk = key[::-1]
    uk, first_in_rev = np.unique(rk, return_index=True)
    last = len(key) - 1 - first_in_rev
    return uk // n, uk % n, np.asarray(vals)[last]


def jacobian(row_ptr, col_idx, vals, v, bus_type, mode="reference", drop=True):
    """Polar Jacobian (cpu_newton_raphson.cpp:546-557, 559-727) as a scipy CSR matrix in the
    reference's row/column order.  |V| < 1e-6 is replaced by 1 (:578).  With drop=True
    entries with |x| <= 1e-12 are removed as convert_to_sparse_matrix does (:754)."""
    n = len(row_ptr) - 1
    ang, mag, peq, qeq, ne = var_maps(bus_type)
    s = power_injections(row_ptr, col_idx, vals, v)
    P, Q = s.real, s.imag
    vm = np.abs(v)
    va = np.angle(v)
    vm = np.where(vm < 1e-6, 1.0, vm)
    I, J, Yv = _dedupe(row_ptr, col_idx, vals, mode)
    G, B = Yv.real, Yv.imag
    rr, cc, xx = [], [], []

    def add(r, c, x, mask):
        m = mask & (r >= 0) & (c >= 0)
        rr.append(r[m])
        cc.append(c[m])
        xx.append(x[m])

    off = I != J
    i, j = I[off], J[off]
    g, b = G[off], B[off]
    th = va[i] - va[j]
    sn, cs = np.sin(th), np.cos(th)
    Vi, Vj = vm[i], vm[j]
    t = np.ones(len(i), bool)
    add(peq[i], ang[j], Vi * Vj * (g * sn - b * cs), t)
    add(peq[i], mag[j], Vi * (g * cs + b * sn), t)
    add(qeq[i], ang[j], -Vi * Vj * (g * cs + b * sn), t)
    add(qeq[i], mag[j], Vi * (g * sn - b * cs), t)
    # diagonal (G_ii, B_ii from the (deduplicated) diagonal entry, else 0)
    Gd = np.zeros(n)
    Bd = np.zeros(n)
    dm = I == J
    Gd[I[dm]] = G[dm]
    Bd[I[dm]] = B[dm]
    k = np.arange(n)
    t = np.ones(n, bool)
    add(peq, ang, -Q - Bd * vm * vm, t)
    add(peq, mag, P / vm + Gd * vm, t)
    add(qeq, ang, P - Gd * vm * vm, t)
    add(qeq, mag, Q / vm - Bd * vm, t)
    r = np.concatenate(rr)
    c = np.concatenate(cc)
    x = np.concatenate(xx)
    if drop:
        keep = np.abs(x) > 1e-12
        r, c, x = r[keep], c[keep], x[keep]
    return sp.csr_matrix((x, (r, c)), shape=(ne, ne))


def flat_start(net: Network):
    """cpu_newton_raphson.cpp:77-88: SLACK and PV at u_pu (angle 0), PQ at 0.98."""
    v = np.where(net.bus_type == PQ, 0.98, net.u_pu).astype(np.complex128)
    return v


def update_reference(bus_type, v, dx, damping=0.9):
    """update_voltage_estimates (cpu_newton_raphson.cpp:438-504): damping 0.9, |dtheta|
    clamp 0.15 rad, |d|V|| clamp 0.08, |V| clipped to [0.5, 1.5]; angles first (every
    non-slack bus in bus order), then magnitudes (PQ buses in bus order).  damping=1.0 is the
    engine's 'clamped' policy (full step, same clamps)."""
    ang, mag, peq, qeq, ne = var_maps(bus_type)
    v = v.copy()
    n = len(v)
    for i in range(n):
        if ang[i] >= 0:
            vm = abs(v[i])
            a = damping * dx[ang[i]]
            if abs(a) > 0.15:
                a = 0.15 * (1.0 if a > 0 else -1.0)
            va = math.atan2(v[i].imag, v[i].real) + a
            v[i] = complex(vm * math.cos(va), vm * math.sin(va))
    for i in range(n):
        if mag[i] >= 0:
            vm0 = abs(v[i])
            c = damping * dx[mag[i]]
            if abs(c) > 0.08:
                c = 0.08 * (1.0 if c > 0 else -1.0)
            vm = min(max(vm0 + c, 0.5), 1.5)
            va = math.atan2(v[i].imag, v[i].real)
            v[i] = complex(vm * math.cos(va), vm * math.sin(va))
    return v


def update_newton(bus_type, v, dx):
    """Pure Newton step in polar coordinates (no damping, no clamps)."""
    ang, mag, peq, qeq, ne = var_maps(bus_type)
    vm = np.abs(v)
    va = np.angle(v)
    m = ang >= 0
    va[m] += dx[ang[m]]
    m = mag >= 0
    vm[m] += dx[mag[m]]
    return vm * np.exp(1j * va)


def nr_solve(net: Network, Y=None, tol=1e-8, max_iter=20, base_power=1e6,
             policy="reference", jac="reference", s_spec=None, v0=None, history=False,
             states=False):
    """CPUNewtonRaphson::solve_power_flow (cpu_newton_raphson.cpp:33-218) with a sparse LU.

    policy 'reference' = the reference's damped, clamped update; 'newton' = pure Newton;
    'clamped' = full Newton step with the reference's clamps.
    jac 'reference' = last-wins duplicates and the 1e-12 drop; 'exact' = summed duplicates.
    Y defaults to the reference Y-bus (Siemens).  Returns dict(v, converged, iterations,
    final_mismatch[, trace][, states]); states=True records IterationState per iteration as
    cpu_newton_raphson.cpp:125-149 does (v, i = Y_pu v, s = v conj(i), mismatch, max)."""
    if Y is None:
        Y = ybus_reference(net)
    row_ptr, col_idx, vals = Y
    zb = float(net.u_rated[0]) ** 2 / base_power
    ypu = np.empty(len(vals), np.complex128)
    ypu.real = np.real(vals) * zb
    ypu.imag = np.imag(vals) * zb
    if s_spec is None:
        s_spec = net.specified_power(base_power)
    v = flat_start(net) if v0 is None else np.asarray(v0, np.complex128).copy()
    bt = net.bus_type
    res = dict(converged=False, iterations=0, final_mismatch=0.0)
    trace = []
    rec = []
    for it in range(max_iter):
        s = power_injections(row_ptr, col_idx, ypu, v)
        d = mismatch(bt, s, s_spec)
        mx = float(np.max(np.abs(d))) if d.size else 0.0
        res["final_mismatch"] = mx
        trace.append(mx)
        if states:
            n = len(row_ptr) - 1
            cur = sp.csr_matrix((ypu, col_idx, row_ptr), shape=(n, n)) @ v
            rec.append(dict(iteration=it, v=v.copy(), i=cur, s=v * np.conj(cur),
                            mismatch=d.copy(), max_mismatch=mx))
        if mx < tol:
            res["converged"] = True
            res["iterations"] = it + 1
            break
        Jm = jacobian(row_ptr, col_idx, ypu, v, bt, mode=jac, drop=(jac == "reference"))
        try:
            dx = spla.splu(Jm.tocsc()).solve(-d)
        except RuntimeError:
            # factorize() failed: the reference continues with zero corrections
            # (cpu_newton_raphson.cpp:416-419)
            dx = np.zeros(len(d))
        if policy == "reference":
            v = update_reference(bt, v, dx)
        elif policy == "clamped":
            v = update_reference(bt, v, dx, damping=1.0)
        else:
            v = update_newton(bt, v, dx)
    if not res["converged"]:
        res["iterations"] = max_iter
    res["v"] = v
    if history:
        res["trace"] = trace
    if states:
        res["states"] = rec
    return res


# ----------------------------------------------------------------------------------------
# Branch losses and adjoint gradients (beyond the reference)
# ----------------------------------------------------------------------------------------


def branch_stamps(net: Network, zb: float, taps=True):
    """Per in-service branch the four pi-model stamps (per unit) used by ybus_pi."""
    f, t, valid = net.branch_index()
    idx = np.nonzero(valid)[0]
    r = net.r1[idx] / zb
    x = net.x1[idx] / zb
    z2 = r * r + x * x
    y = np.where(z2 > 1e-12, (r - 1j * x) / np.where(z2 > 1e-12, z2, 1.0), 0.0)
    ysh = net.g1[idx] * zb + 1j * net.b1[idx] * zb / 2.0
    if taps:
        tap = net.k[idx] * np.exp(1j * net.theta[idx])
    else:
        tap = np.ones(len(idx), np.complex128)
    yff = (y + ysh) / np.abs(tap) ** 2
    ytt = y + ysh
    yft = -y / np.conj(tap)
    ytf = -y / tap
    return idx, f[idx], t[idx], y, yff, ytt, yft, ytf, tap


def loss_value(net: Network, v, zb, base_power, taps=True):
    """L = sum_bus (|V|-1)^2 + sum_branch P_loss[MW] with P_loss = Re(S_from + S_to)."""
    idx, f, t, y, yff, ytt, yft, ytf, tap = branch_stamps(net, zb, taps)
    i_f = yff * v[f] + yft * v[t]
    i_t = ytf * v[f] + ytt * v[t]
    ploss = np.real(v[f] * np.conj(i_f) + v[t] * np.conj(i_t))
    return float(np.sum((np.abs(v) - 1.0) ** 2) + np.sum(ploss) * base_power / 1e6)


def adjoint_gradients(net: Network, v, base_power=1e6, taps=True):
    """Implicit-function gradients of loss_value at a converged state v (FP64, exact
    Jacobian).  Returns dict(dP, dQ) per bus (w.r.t. S_spec in per unit) and (dr, dx) per
    branch (w.r.t. r1, x1 in Ohm; zeros for out-of-service branches)."""
    zb = float(net.u_rated[0]) ** 2 / base_power
    Y = ybus_pi(net) if taps else ybus_reference(net)
    row_ptr, col_idx, vals = Y
    ypu = vals * zb
    bt = net.bus_type
    n = net.n_bus
    ang, mag, peq, qeq, ne = var_maps(bt)
    Jm = jacobian(row_ptr, col_idx, ypu, v, bt, mode="exact", drop=False)
    vm = np.abs(v)
    idx, f, t, y, yff, ytt, yft, ytf, tap = branch_stamps(net, zb, taps)
    w = base_power / 1e6
    # dL/dx (x = theta_nonslack, |V|_PQ); V_i = |V_i| e^{j th_i}
    g = np.zeros(ne)
    dvm = 2.0 * (vm - 1.0)
    m = mag >= 0
    g[mag[m]] += dvm[m]
    # branch loss derivative w.r.t. complex V: loss = Re(V^H Yb V) restricted to the branch
    # d loss / d th_i = Re(conj(dL/dV_i) * j V_i) * 2 ... computed via Wirtinger: for
    # f(V) = Re(sum_k V_k conj(I_k)), df = Re(dV^H (I + Yb^H V)) for each branch.
    vf, vt = v[f], v[t]
    i_f = yff * vf + yft * vt
    i_t = ytf * vf + ytt * vt
    # gradient vector gV_k = I_k + sum_l conj(Yb_lk) V_l   (so that df = Re(conj(gV) . dV))
    gvf = i_f + np.conj(yff) * vf + np.conj(ytf) * vt
    gvt = i_t + np.conj(yft) * vf + np.conj(ytt) * vt
    gV = np.zeros(n, np.complex128)
    np.add.at(gV, f, gvf * w)
    np.add.at(gV, t, gvt * w)
    # dV/dth = j V ; dV/d|V| = V/|V|
    dth = np.real(np.conj(gV) * 1j * v)
    dmag = np.real(np.conj(gV) * v / np.where(vm > 0, vm, 1.0))
    a = ang >= 0
    g[ang[a]] += dth[a]
    g[mag[m]] += dmag[m]
    lam = spla.splu(Jm.T.tocsc()).solve(g)
    dP = np.zeros(n)
    dQ = np.zeros(n)
    p = peq >= 0
    dP[p] = lam[peq[p]]
    q = qeq >= 0
    dQ[q] = lam[qeq[q]]
    # parameter gradients: dL/dp = dL/dp|direct - lam^T dF/dp, F_k = S_calc,k - S_spec,k
    m_br = net.n_branch
    dr = np.zeros(m_br)
    dxg = np.zeros(m_br)
    r = net.r1[idx] / zb
    x = net.x1[idx] / zb
    for which, dy in (("r", -(y * y)), ("x", -1j * (y * y))):
        # stamp derivatives w.r.t. y
        a2 = np.abs(tap) ** 2
        dyff = dy / a2
        dytt = dy
        dyft = -dy / np.conj(tap)
        dytf = -dy / tap
        di_f = dyff * vf + dyft * vt
        di_t = dytf * vf + dytt * vt
        dsf = vf * np.conj(di_f)
        dst = vt * np.conj(di_t)
        # direct loss term
        direct = np.real(dsf + dst) * w
        # -lam^T dF
        adj = np.zeros(len(idx))
        pf, pt_ = peq[f], peq[t]
        qf, qt_ = qeq[f], qeq[t]
        adj += np.where(pf >= 0, lam[np.maximum(pf, 0)] * dsf.real, 0.0)
        adj += np.where(pt_ >= 0, lam[np.maximum(pt_, 0)] * dst.real, 0.0)
        adj += np.where(qf >= 0, lam[np.maximum(qf, 0)] * dsf.imag, 0.0)
        adj += np.where(qt_ >= 0, lam[np.maximum(qt_, 0)] * dst.imag, 0.0)
        grad_pu = direct - adj
        if which == "r":
            dr[idx] = grad_pu / zb
        else:
            dxg[idx] = grad_pu / zb
    return dict(dP=dP, dQ=dQ, dr=dr, dx=dxg, lam=lam)


def ybus_update_reference(Y, changes: Network):
    """CPUAdmittanceMatrix::update_admittance_matrix (cpu_admittance_matrix.cpp:204-301):
    for each changed branch, from/to taken as matrix indices (shifted down by one when both
    are positive and one exceeds the matrix size), delta = y + g1 + j b1 (+ j b1/2) added to
    both diagonals, -y to the first (f,t) and (t,f) entries; negated when status is 0."""
    row_ptr, col_idx, vals = Y
    out = np.array(vals, np.complex128).copy()
    nrows = len(row_ptr) - 1
    for b in range(changes.n_branch):
        f, t = int(changes.from_id[b]), int(changes.to_id[b])
        if f > 0 and t > 0 and (f > nrows or t > nrows):
            f -= 1
            t -= 1
        if f < 0 or f >= nrows or t < 0 or t >= nrows:
            continue
        r, x = float(changes.r1[b]), float(changes.x1[b])
        z2 = r * r + x * x
        ys = complex(r / z2, -x / z2) if z2 > 1e-12 else 0j
        tot = ys + complex(float(changes.g1[b]), float(changes.b1[b]))
        sh = complex(0.0, float(changes.b1[b]) / 2.0)
        if not changes.status[b]:
            tot, ys, sh = -tot, -ys, -sh
        for bus in (f, t):
            for p in range(row_ptr[bus], row_ptr[bus + 1]):
                if col_idx[p] == bus:
                    out[p] += tot + sh
                    break
        for a, c in ((f, t), (t, f)):
            for p in range(row_ptr[a], row_ptr[a + 1]):
                if col_idx[p] == c:
                    out[p] -= ys
                    break
    return row_ptr, col_idx, out


def change_stamps(prm, taps):
    """The Y-bus builder's four stamps (ff, tt, ft, tf) of one branch, prm = (r1, x1, g1, b1,
    k, theta, ...): y = 1/(r + jx) (0 when |z|^2 <= 1e-12), end stamp y + g1 + j b1/2
    (cpu_admittance_matrix.cpp:120-139), and with taps the pi model of ybus_pi."""
    r, x, g, b, kk, th = (float(v) for v in prm[:6])
    z2 = r * r + x * x
    yr, yi = (r / z2, -x / z2) if z2 > 1e-12 else (0.0, 0.0)
    end = complex((yr + g) + 0.0, (yi + 0.0) + b / 2.0)
    y = complex(yr, yi)
    if not taps or (kk == 1.0 and th == 0.0):
        return end, end, -y, -y
    tap = kk * complex(math.cos(th), math.sin(th))
    return end / (kk * kk), end, -y / tap.conjugate(), -y / tap


def ybus_delta(values, positions, params, mode, scale=1.0):
    """Branch status changes applied to Y values in change order (the batched device update's
    restatement).  positions [c, 4] = CSR indices (diag from, diag to, (from,to), (to,from)) or
    -1; params [c, 7] = (r1, x1, g1, b1, k, theta, status).  mode 'reference': the reference's
    update (cpu_admittance_matrix.cpp:238-297: diagonals y + g1 + j b1 + j b1/2, off-diagonals
    -y, taps ignored); 'fixed': the builder's stamps without taps; 'fixed_taps': with taps.
    Deltas are added for status 1 and subtracted for status 0, multiplied by scale."""
    out = np.array(values, np.complex128).copy()
    for c in range(len(params)):
        q = params[c]
        if mode == "reference":
            r, x, g, b = (float(v) for v in q[:4])
            z2 = r * r + x * x
            ys = complex(r / z2, -x / z2) if z2 > 1e-12 else 0j
            diag = (ys + complex(g, b)) + complex(0.0, b / 2.0)
            d = (diag, diag, -ys, -ys)
        else:
            d = change_stamps(q, taps=(mode == "fixed_taps"))
        sign = 1.0 if q[6] != 0.0 else -1.0
        for role in range(4):
            p = int(positions[c][role])
            if p >= 0:
                out[p] += sign * d[role] * scale
    return out


def branch_flows(net: Network, v, base_power, i_n=None, sn=None, taps=True):
    """Branch results of a solved network, in the units of the reference's BranchData result
    fields (include/gap/core/types.h:233-243: p/q in W/var, s in VA, i in A, loading), which
    the reference declares but never fills; definitions as power-grid-model's line output
    (the reference's PGM validation data): S_from = V_f conj(I_f) with I_f = Y_ff V_f + Y_ft V_t
    the current into the branch at its from end (pi model of the Y-bus builder), likewise at
    the to end; |I| = |S| / (sqrt(3) |U|) with U the line-to-line voltage; loading =
    max(i_from, i_to) / i_n, or max(s_from, s_to) / sn for a branch with sn > 0 and no i_n.
    Returns ([m_in_service, 9] = p_from, q_from, i_from, s_from, p_to, q_to, i_to, s_to,
    loading; the in-service branch indices)."""
    zb = float(net.u_rated[0]) ** 2 / base_power
    idx, f, t, y, yff, ytt, yft, ytf, tap = branch_stamps(net, zb, taps)
    v = np.asarray(v, np.complex128)
    vf, vt = v[f], v[t]
    i_f = yff * vf + yft * vt
    i_t = ytf * vf + ytt * vt
    s_f = vf * np.conj(i_f) * base_power
    s_t = vt * np.conj(i_t) * base_power
    ub = float(net.u_rated[0])
    sq3 = math.sqrt(3.0)
    a_f = np.abs(s_f) / (sq3 * np.abs(vf) * ub)
    a_t = np.abs(s_t) / (sq3 * np.abs(vt) * ub)
    load = np.zeros(len(idx))
    if i_n is not None:
        inn = np.asarray(i_n, np.float64)[idx] if len(i_n) == net.n_branch else np.asarray(i_n)
        load = np.where(inn > 0, np.maximum(a_f, a_t) / np.where(inn > 0, inn, 1.0), 0.0)
    if sn is not None:
        snn = np.asarray(sn, np.float64)[idx] if len(sn) == net.n_branch else np.asarray(sn)
        use = (snn > 0) & (load == 0)
        load = np.where(use, np.maximum(np.abs(s_f), np.abs(s_t)) / np.where(snn > 0, snn, 1.0),
                        load)
    out = np.stack([s_f.real, s_f.imag, a_f, np.abs(s_f), s_t.real, s_t.imag, a_t, np.abs(s_t),
                    load], axis=1)
    return out, idx
