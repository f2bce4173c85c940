"""power-grid-model (PGM) JSON input and batch-update datasets -> Network / scenarios.

The reference reads PGM JSON in C++ (src/io/json_io.cpp:113-382, convertPgm* and
inferBusTypes) and in its Python validation tooling.  This reader produces the same
NetworkData content for the components of the power-flow path, with the reference's load sign
corrected: a PGM sym_load's p_specified / q_specified are consumption, so they enter S_spec as
negative injections (the reference copies them as positive LOADGEN injections,
json_io.cpp:195-209, and its bindings' callers have to flip the sign,
bindings/solver_bindings.cpp:196-197); sym_gen values are injections as given.

Components read (PGM input format, one dataset):
  node            -> bus (id, u_rated)
  line            -> branch: r1, x1; b1 = 2 pi 50 c1, g1 = b1 tan1 (json_io.cpp:143-147 and
                     BranchData::set_from_pgm_capacitive_params); i_n
  transformer     -> branch as json_io.cpp:216-268: z = uk u1^2 / sn split by rx_ratio,
                     k = u1 / u2 (x (1 + tap_pos tap_size / 1e5)), theta = clock x 30 deg,
                     i_n = sn / (sqrt 3 min(u1, u2)); taps and shifts reach the Y-bus only in
                     the engine's taps mode (the reference ignores them)
  generic_branch  -> branch: r1, x1, g1, b1, k, shift (json_io.cpp:273-309)
  source          -> SOURCE appliance; its bus becomes SLACK at u_ref (inferBusTypes)
  sym_load        -> LOADGEN appliance with -p_specified, -q_specified
  sym_gen         -> LOADGEN appliance with p_specified, q_specified
  shunt           -> SHUNT appliance (g1, b1)
A branch is in service when both from_status and to_status are set.

write_output formats solved scenarios as a PGM output dataset (node, line, transformer,
generic_branch, sym_load, sym_gen, source), the results the reference's write_results leaves
unimplemented (json_io.cpp:507-517).
"""

from __future__ import annotations

import dataclasses
import json
import math

import numpy as np

from .network import LOADGEN, PQ, SHUNT, SLACK, SOURCE, Network


def _data(doc):
    if isinstance(doc, (str, bytes)) and not str(doc).lstrip().startswith("{"):
        with open(doc) as fh:
            doc = json.load(fh)
    elif isinstance(doc, (str, bytes)):
        doc = json.loads(doc)
    return doc.get("data", doc) if isinstance(doc, dict) else doc


BRANCH_KINDS = ("line", "transformer", "generic_branch")
APPLIANCE_KINDS = ("source", "sym_load", "sym_gen", "shunt")


def read_input(doc):
    """PGM input dataset (path, JSON text or parsed dict) -> (Network in SI units,
    {"i_n": rated current per branch (A), "sn": rated power per branch (VA), "branch_kind":
    index into BRANCH_KINDS per branch, "appliance_kind": index into APPLIANCE_KINDS per
    appliance})."""
    d = _data(doc)
    nodes = d.get("node", [])
    bus_id = np.array([int(n["id"]) for n in nodes], np.int64)
    u_rated = np.array([float(n["u_rated"]) for n in nodes])
    br = []  # (id, from, to, status, r1, x1, g1, b1, k, theta, i_n, sn)
    br_kind = []
    for ln in d.get("line", []):
        c1, tan1 = float(ln.get("c1", 0.0)), float(ln.get("tan1", 0.0))
        b1 = 2.0 * math.pi * 50.0 * c1 if c1 > 0 else 0.0
        br.append((int(ln["id"]), int(ln["from_node"]), int(ln["to_node"]),
                   int(bool(ln.get("from_status", 1)) and bool(ln.get("to_status", 1))),
                   float(ln["r1"]), float(ln["x1"]), b1 * tan1, b1, 1.0, 0.0,
                   float(ln.get("i_n", 1000.0)), 0.0))
        br_kind.append(0)
    for tr in d.get("transformer", []):
        u1, u2, sn, uk = (float(tr[k]) for k in ("u1", "u2", "sn", "uk"))
        z = uk * u1 * u1 / sn
        xr = 1.0 / float(tr["rx_ratio"]) if "rx_ratio" in tr else 10.0
        rf = 1.0 / math.sqrt(1.0 + xr * xr)
        k = u1 / u2
        if "tap_pos" in tr and "tap_size" in tr:
            k *= 1.0 + float(tr["tap_pos"]) * float(tr["tap_size"]) / 100000.0
        theta = float(tr.get("clock", 0.0)) * math.pi / 6.0
        br.append((int(tr["id"]), int(tr["from_node"]), int(tr["to_node"]),
                   int(bool(tr.get("from_status", 1)) and bool(tr.get("to_status", 1))),
                   z * rf, z * xr * rf, 0.0, 0.0, k, theta, sn / (math.sqrt(3.0) * min(u1, u2)),
                   sn))
        br_kind.append(1)
    for gb in d.get("generic_branch", []):
        sn = float(gb.get("sn", 0.0))
        i_n = float(gb["i_n"]) if "i_n" in gb else (sn / (math.sqrt(3.0) * 20000.0) if sn > 0
                                                      else 1000.0)
        br.append((int(gb["id"]), int(gb["from_node"]), int(gb["to_node"]),
                   int(bool(gb.get("from_status", 1)) and bool(gb.get("to_status", 1))),
                   float(gb["r1"]), float(gb["x1"]), float(gb.get("g1", 0.0)),
                   float(gb.get("b1", 0.0)), float(gb.get("k", 1.0)),
                   float(gb.get("shift", 0.0)), i_n, sn))
        br_kind.append(2)
    br = np.array(br, np.float64).reshape(-1, 12)
    apps = []  # (id, node, status, type, p, q, g1, b1)
    app_kind = []
    u_ref = {}
    for s in d.get("source", []):
        apps.append((int(s["id"]), int(s["node"]), int(s.get("status", 1)), SOURCE, 0, 0, 0, 0))
        app_kind.append(0)
        if int(s.get("status", 1)):
            u_ref[int(s["node"])] = float(s.get("u_ref", 1.0))
    for ld in d.get("sym_load", []):
        apps.append((int(ld["id"]), int(ld["node"]), int(ld.get("status", 1)), LOADGEN,
                     -float(ld.get("p_specified", 0.0)), -float(ld.get("q_specified", 0.0)), 0, 0))
        app_kind.append(1)
    for g in d.get("sym_gen", []):
        apps.append((int(g["id"]), int(g["node"]), int(g.get("status", 1)), LOADGEN,
                     float(g.get("p_specified", 0.0)), float(g.get("q_specified", 0.0)), 0, 0))
        app_kind.append(2)
    for sh in d.get("shunt", []):
        apps.append((int(sh["id"]), int(sh["node"]), int(sh.get("status", 1)), SHUNT, 0, 0,
                     float(sh.get("g1", 0.0)), float(sh.get("b1", 0.0))))
        app_kind.append(3)
    apps = np.array(apps, np.float64).reshape(-1, 8)
    bus_type = np.full(len(bus_id), PQ, np.int32)
    u_pu = np.ones(len(bus_id))
    pos = {int(b): i for i, b in enumerate(bus_id)}
    for node, u in u_ref.items():
        if node in pos:
            bus_type[pos[node]] = SLACK
            u_pu[pos[node]] = u
    net = Network.build(
        bus_id=bus_id, u_rated=u_rated, bus_type=bus_type, u_pu=u_pu,
        br_id=br[:, 0].astype(np.int64), from_id=br[:, 1].astype(np.int64),
        to_id=br[:, 2].astype(np.int64), status=br[:, 3].astype(np.int32), r1=br[:, 4],
        x1=br[:, 5], g1=br[:, 6], b1=br[:, 7], k=br[:, 8], theta=br[:, 9],
        app_id=apps[:, 0].astype(np.int64), app_node=apps[:, 1].astype(np.int64),
        app_status=apps[:, 2].astype(np.int32), app_type=apps[:, 3].astype(np.int32),
        app_p=apps[:, 4], app_q=apps[:, 5], app_g1=apps[:, 6], app_b1=apps[:, 7])
    net_i_n = br[:, 10].copy()
    net_sn = br[:, 11].copy()
    return net, {"i_n": net_i_n, "sn": net_sn, "branch_kind": np.array(br_kind, np.int32),
                 "appliance_kind": np.array(app_kind, np.int32)}


def read_update(net: Network, doc, base_power: float) -> np.ndarray:
    """PGM batch update dataset (a list of per-scenario update datasets, or the columnar
    {"sym_load": [[...scenario 0...], [...scenario 1...]]} form) applied to `net`'s
    appliances: per scenario, the updated sym_load / sym_gen p_specified / q_specified (and
    status) replace the input's.  Returns S_spec per unit, complex128 [n_scen, n_bus], ready
    for a batched solve."""
    d = _data(doc)
    if isinstance(d, dict):
        n = max((len(v) for v in d.values()), default=0)
        scen = [{k: v[i] for k, v in d.items()} for i in range(n)]
    else:
        scen = list(d)
    idx = {int(a): i for i, a in enumerate(net.app_id)}
    out = np.empty((len(scen), net.n_bus), np.complex128)
    for s, upd in enumerate(scen):
        p, q, st = net.app_p.copy(), net.app_q.copy(), net.app_status.copy()
        for comp, sign in (("sym_load", -1.0), ("sym_gen", 1.0)):
            for u in upd.get(comp, []):
                i = idx[int(u["id"])]
                if "p_specified" in u:
                    p[i] = sign * float(u["p_specified"])
                if "q_specified" in u:
                    q[i] = sign * float(u["q_specified"])
                if "status" in u:
                    st[i] = int(u["status"])
        out[s] = dataclasses.replace(net, app_p=p, app_q=q, app_status=st).specified_power(
            base_power)
    return out


def _host(x):
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)


def write_output(net: Network, extra, v, s_bus, flows, base_power: float, angle="deg",
                 u_rated=None):
    """Solved scenarios -> PGM output dataset(s), the component results of the reference's
    validation data (tests/pgm_validation/test_data/*/output.json):

      node            id, energized, u_pu, u_angle, u (V), p, q (injection, W / var)
      line, transformer, generic_branch
                      id, energized, loading, p_from, q_from, i_from, s_from, p_to, q_to,
                      i_to, s_to (the device branch results, gapk_branch_flows)
      sym_load        id, energized, p, q (consumption), s, pf
      sym_gen         id, energized, p, q, s, pf
      source          id, energized, p, q, s, pf, i: the node's injection less the node's
                      other appliances

    v: complex per-unit voltages [n_bus] or [S, n_bus]; s_bus: per-unit power injections
    S = V conj(Y V) of the same shape (NRBatch.state()); flows: [.., n_branch, 9] as
    engine.branch_flows returns (W, var, A, VA); extra: read_input's second result.  angle
    "deg" (the unit of the reference's validation data) or "rad".  Returns one dict per
    scenario (a list when v has a scenario axis)."""
    v, s_bus, flows = _host(v), _host(s_bus), _host(flows)
    if v.ndim == 2:
        return [write_output(net, extra, v[k], s_bus[k], flows[k], base_power, angle, u_rated)
                for k in range(v.shape[0])]
    ur = np.asarray(net.u_rated if u_rated is None else u_rated, np.float64)
    ang = np.angle(v)
    if angle == "deg":
        ang = np.degrees(ang)
    s_w = s_bus * base_power
    out = {"node": [{"id": int(net.bus_id[i]), "energized": bool(abs(v[i]) > 0.0),
                     "u_pu": float(abs(v[i])), "u_angle": float(ang[i]),
                     "u": float(abs(v[i]) * ur[i]), "p": float(s_w[i].real),
                     "q": float(s_w[i].imag)} for i in range(net.n_bus)]}
    fields = ("p_from", "q_from", "i_from", "s_from", "p_to", "q_to", "i_to", "s_to")
    kinds = extra.get("branch_kind", np.zeros(net.n_branch, np.int32))
    for b in range(net.n_branch):
        rec = {"id": int(net.br_id[b]), "energized": bool(net.status[b]),
               "loading": float(flows[b][8])}
        rec.update({f: float(flows[b][j]) for j, f in enumerate(fields)})
        out.setdefault(BRANCH_KINDS[int(kinds[b])], []).append(rec)
    pos = {int(bid): i for i, bid in enumerate(net.bus_id)}
    akind = extra.get("appliance_kind", np.where(net.app_type == SOURCE, 0, 1))
    on = (net.app_status == 1)
    # appliance injections (W / var) per node, sources excluded
    other = np.zeros(net.n_bus, np.complex128)
    for a in range(net.n_app):
        if on[a] and net.app_type[a] == LOADGEN and int(net.app_node[a]) in pos:
            other[pos[int(net.app_node[a])]] += complex(net.app_p[a], net.app_q[a])
    for a in range(net.n_app):
        kind = APPLIANCE_KINDS[int(akind[a])]
        i = pos.get(int(net.app_node[a]))
        live = bool(on[a]) and i is not None and abs(v[i]) > 0.0
        if kind == "shunt":
            continue
        if kind == "source":
            sp = (s_w[i] - other[i]) if live else 0j
        elif kind == "sym_load":
            sp = -complex(net.app_p[a], net.app_q[a]) if live else 0j
        else:
            sp = complex(net.app_p[a], net.app_q[a]) if live else 0j
        s_abs = abs(sp)
        rec = {"id": int(net.app_id[a]), "energized": live, "p": float(sp.real),
               "q": float(sp.imag), "s": float(s_abs),
               "pf": float(sp.real / s_abs) if s_abs > 0 else 0.0}
        if kind == "source":
            rec["i"] = float(s_abs / (math.sqrt(3.0) * abs(v[i]) * ur[i])) if live else 0.0
        out.setdefault(kind, []).append(rec)
    return out
