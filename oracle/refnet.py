"""ORACLE TEST INFRASTRUCTURE -- ctypes access to the reference's own CPU path.

Loads oracle/_ref/libgapref.so (built by oracle/Makefile from the reference sources plus
oracle/ref_driver.cpp).  Used only by tests/, the smoke check and bench.py's CPU-baseline leg,
as the checker.  `available()` is False when the library was not built (e.g. when the
reference checkout was absent at build time).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_LIB = None
_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libgapref.so")


class _Net(C.Structure):
    _fields_ = [
        ("n_bus", C.c_int), ("bus_id", C.c_void_p), ("u_rated", C.c_void_p),
        ("bus_type", C.c_void_p), ("u_pu", C.c_void_p), ("p_w", C.c_void_p),
        ("q_var", C.c_void_p),
        ("n_branch", C.c_int), ("br_id", C.c_void_p), ("from_id", C.c_void_p),
        ("to_id", C.c_void_p), ("status", C.c_void_p), ("r1", C.c_void_p), ("x1", C.c_void_p),
        ("g1", C.c_void_p), ("b1", C.c_void_p), ("k", C.c_void_p), ("theta", C.c_void_p),
        ("n_app", C.c_int), ("app_id", C.c_void_p), ("app_node", C.c_void_p),
        ("app_status", C.c_void_p), ("app_type", C.c_void_p), ("app_p", C.c_void_p),
        ("app_q", C.c_void_p), ("app_g1", C.c_void_p), ("app_b1", C.c_void_p),
    ]


def available() -> bool:
    return os.path.exists(_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError(f"reference oracle not built: {_PATH} (run make -C oracle)")
        _LIB = C.CDLL(_PATH)
        _LIB.gapref_quiet()
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a.size else None


def _pack(net):
    keep = []

    def k(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return _ptr(a)

    s = _Net()
    s.n_bus = net.n_bus
    s.bus_id = k(net.bus_id, np.int32)
    s.u_rated = k(net.u_rated, np.float64)
    s.bus_type = k(net.bus_type, np.int32)
    s.u_pu = k(net.u_pu, np.float64)
    s.p_w = k(net.p, np.float64)
    s.q_var = k(net.q, np.float64)
    s.n_branch = net.n_branch
    s.br_id = k(net.br_id, np.int32)
    s.from_id = k(net.from_id, np.int32)
    s.to_id = k(net.to_id, np.int32)
    s.status = k(net.status, np.int32)
    for f in ("r1", "x1", "g1", "b1", "k", "theta"):
        setattr(s, f, k(getattr(net, f), np.float64))
    s.n_app = net.n_app
    s.app_id = k(net.app_id, np.int32)
    s.app_node = k(net.app_node, np.int32)
    s.app_status = k(net.app_status, np.int32)
    s.app_type = k(net.app_type, np.int32)
    for f in ("app_p", "app_q", "app_g1", "app_b1"):
        setattr(s, f, k(getattr(net, f), np.float64))
    return s, keep


def ybus(net):
    """Reference Y-bus (Siemens): (row_ptr int32, col_idx int32, values complex128)."""
    L = lib()
    s, keep = _pack(net)
    cap = net.n_bus + 2 * net.n_branch + 8
    rp = np.zeros(net.n_bus + 1, np.int32)
    ci = np.zeros(cap, np.int32)
    va = np.zeros(2 * cap, np.float64)
    nnz = L.gapref_ybus(C.byref(s), C.c_int(cap), _ptr(rp), _ptr(ci), _ptr(va))
    if nnz < 0:
        raise RuntimeError("capacity")
    return rp, ci[:nnz].copy(), va[: 2 * nnz].view(np.complex128).copy()


def ybus_update(net, changes):
    L = lib()
    s, keep = _pack(net)
    c, keep2 = _pack(changes)
    cap = net.n_bus + 2 * net.n_branch + 8
    rp = np.zeros(net.n_bus + 1, np.int32)
    ci = np.zeros(cap, np.int32)
    va = np.zeros(2 * cap, np.float64)
    nnz = L.gapref_ybus_update(C.byref(s), C.byref(c), C.c_int(cap), _ptr(rp), _ptr(ci),
                               _ptr(va))
    return rp, ci[:nnz].copy(), va[: 2 * nnz].view(np.complex128).copy()


def solve(net, tol=1e-8, max_iter=20, base_power=1e6):
    """Reference NR.  Returns dict(v=complex128[n], converged, iterations, final_mismatch)."""
    L = lib()
    s, keep = _pack(net)
    v = np.zeros(2 * net.n_bus, np.float64)
    conv = C.c_int(0)
    it = C.c_int(0)
    fm = C.c_double(0.0)
    rc = L.gapref_solve(C.byref(s), C.c_double(tol), C.c_int(max_iter), C.c_double(base_power),
                        _ptr(v), C.byref(conv), C.byref(it), C.byref(fm))
    if rc != 0:
        raise RuntimeError("reference solve threw")
    return dict(v=v.view(np.complex128).copy(), converged=bool(conv.value),
                iterations=int(it.value), final_mismatch=float(fm.value))


def solve_states(net, tol=1e-8, max_iter=20, base_power=1e6):
    """Reference CPUNewtonRaphson with iteration-state capture on: a list, per iteration, of
    dict(max_mismatch, v, i, s) (complex per-unit vectors over the buses)."""
    L = lib()
    s, keep = _pack(net)
    n = net.n_bus
    cap = max(int(max_iter), 1)
    mm = np.zeros(cap, np.float64)
    vs, cs, ss = (np.zeros((cap, n, 2), np.float64) for _ in range(3))
    k = L.gapref_solve_states(C.byref(s), C.c_double(tol), C.c_int(max_iter),
                              C.c_double(base_power), C.c_int(cap), _ptr(mm), _ptr(vs),
                              _ptr(cs), _ptr(ss))
    if k < 0:
        raise RuntimeError("reference solve threw")
    k = min(k, cap)
    return [dict(max_mismatch=float(mm[j]), v=vs[j].view(np.complex128)[:, 0].copy(),
                 i=cs[j].view(np.complex128)[:, 0].copy(),
                 s=ss[j].view(np.complex128)[:, 0].copy()) for j in range(k)]


def mismatch(net, v):
    L = lib()
    s, keep = _pack(net)
    vv = np.ascontiguousarray(np.asarray(v, np.complex128)).view(np.float64)
    out = np.zeros(2 * net.n_bus + 2, np.float64)
    n = L.gapref_mismatch(C.byref(s), _ptr(vv), C.c_int(out.size), _ptr(out))
    return out[:n].copy()


def lu_solve(row_ptr, col_idx, vals, rhs):
    """Reference CPULUSolver.  Returns (status, x); status 0 ok, 1 factorize failed,
    -1 solve threw."""
    L = lib()
    n = len(row_ptr) - 1
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    va = np.ascontiguousarray(np.asarray(vals, np.complex128)).view(np.float64)
    b = np.ascontiguousarray(np.asarray(rhs, np.complex128)).view(np.float64)
    x = np.zeros(2 * n, np.float64)
    st = L.gapref_lu_solve(C.c_int(n), C.c_int(len(ci)), _ptr(rp), _ptr(ci), _ptr(va), _ptr(b),
                           _ptr(x))
    return int(st), x.view(np.complex128).copy()
