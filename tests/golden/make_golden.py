"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout that has the reference project next to it and
the reference oracle built (make -C oracle):

    python tests/golden/make_golden.py --ref <path of the reference checkout>

Fixtures (all small .npz files):
  pgm_<case>.npz   the reference's PGM validation cases (tests/pgm_validation/test_data, the
                   ones under 100 KB, as the reference's pytest selects them,
                   test_pgm_validation.py:49-63), converted to the solve_simple_power_flow
                   lists exactly as the reference's pytest converts them (:160-206), with the
                   power-grid-model outputs (u_pu, u_angle) and the reference CPU solver's
                   result on the same lists.
  c0_seed<k>.npz   the 200-bus meshed feeder (seeds 0..4) with the reference Y-bus and the
                   reference CPU NR result (tol 1e-8, max 20, base 1 MVA).
  kat_<name>.npz   small hand-built networks restating the reference's unit-test topologies
                   (tests/unit/test_admittance.cpp, test_newton_raphson_functions.cpp) plus
                   edge cases (parallel branches, out-of-service branch, unknown bus ID,
                   isolated bus, shunts, PV bus), with reference Y-bus, mismatch and NR.
  lu_<name>.npz    complex sparse systems solved by the reference CPULUSolver.
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gap_b200 import synth  # noqa: E402
from gap_b200.network import LOADGEN, PQ, PV, SHUNT, SLACK, SOURCE, Network  # noqa: E402
from oracle import refnet  # noqa: E402


def net_arrays(net: Network, prefix="net_"):
    return {prefix + k: getattr(net, k) for k in net.__dataclass_fields__}


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def ref_all(net, tol=1e-8, max_iter=20, base=1e6):
    rp, ci, va = refnet.ybus(net)
    sol = refnet.solve(net, tol, max_iter, base)
    # iteration-state capture of the same solve (IterationState per iteration,
    # cpu_newton_raphson.cpp:125-149): max |mismatch| and V; I = Y V and S = V conj(I) too on
    # grids of up to 64 buses (they follow from V and Y, so larger grids keep V only)
    st = refnet.solve_states(net, tol, max_iter, base)
    cap = dict(cap_max_mis=np.array([x["max_mismatch"] for x in st]),
               cap_v=np.array([x["v"] for x in st]).reshape(len(st), net.n_bus))
    if net.n_bus <= 64:
        cap["cap_i"] = np.array([x["i"] for x in st]).reshape(len(st), net.n_bus)
        cap["cap_s"] = np.array([x["s"] for x in st]).reshape(len(st), net.n_bus)
    return dict(y_row_ptr=rp, y_col_idx=ci, y_values=va, ref_v=sol["v"],
                ref_converged=np.int32(sol["converged"]), ref_iterations=np.int32(sol["iterations"]),
                ref_final_mismatch=np.float64(sol["final_mismatch"]), **cap)


def simple_lists_to_network(bus_data, branch_data):
    """solve_simple_power_flow's list conversion (bindings/solver_bindings.cpp:67-111)."""
    bus = np.asarray(bus_data, np.float64)
    br = np.asarray(branch_data, np.float64).reshape(-1, max(len(branch_data[0]), 5) if branch_data else 5)
    b1 = br[:, 5] if br.shape[1] > 5 else np.zeros(len(br))
    return Network.build(bus_id=bus[:, 0].astype(int), u_rated=bus[:, 1],
                         bus_type=bus[:, 2].astype(int), u_pu=bus[:, 3], p=bus[:, 5],
                         q=bus[:, 6], br_id=br[:, 0].astype(int), from_id=br[:, 1].astype(int),
                         to_id=br[:, 2].astype(int), r1=br[:, 3], x1=br[:, 4], b1=b1)


PGM_JSON_CASES = ("radial_1feeder_2nodepf", "radial_2feeder_8nodepf", "radial_3feeder_8nodepf")


def make_pgm(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "tests", "pgm_validation"))
    from json_io.gap_json_parser import PGMJSONParser  # reference code, used only here

    data = os.path.join(ref_root, "tests", "pgm_validation", "test_data")
    made = []
    for case in sorted(os.listdir(data)):
        d = os.path.join(data, case)
        inp, outp = os.path.join(d, "input.json"), os.path.join(d, "output.json")
        if not (os.path.exists(inp) and os.path.exists(outp)):
            continue
        if os.path.getsize(inp) >= 100000:
            continue
        meta = json.load(open(os.path.join(d, "metadata.json")))
        parser = PGMJSONParser(base_power=meta.get("base_power", 1e6))
        net = parser.parse_network(inp)
        ref = json.load(open(outp))
        nodes = {n["id"]: n for n in ref["node"]}
        ids = sorted(nodes)
        pgm_u = np.array([nodes[i]["u_pu"] for i in ids])
        pgm_a = np.array([nodes[i]["u_angle"] for i in ids])
        bus_data, branch_data = [], []
        for i in range(net.n_node):
            if i in net.source_node:
                bt, vpu = 2, float(net.u_ref_pu[net.source_node == i][0])
            else:
                bt, vpu = 0, 1.0
            p = q = 0.0
            if i in net.load_node:
                for li in np.nonzero(net.load_node == i)[0]:
                    if net.load_status[li]:
                        p -= net.p_load_pu[li] * net.base_power
                        q -= net.q_load_pu[li] * net.base_power
            bus_data.append([int(net.node_ids[i]), float(net.u_rated[i]), bt, vpu, 0.0, p, q])
        zb = (net.u_rated[0] ** 2) / net.base_power
        for i in range(net.n_branch):
            if net.branch_status[i]:
                branch_data.append([int(net.branch_ids[i]), int(net.from_node[i]),
                                    int(net.to_node[i]), float(net.r_pu[i]) * zb,
                                    float(net.x_pu[i]) * zb, float(net.b_pu[i]) / zb, 1])
        gnet = simple_lists_to_network(bus_data, branch_data)
        sol = ref_all(gnet, 1e-8, 20, net.base_power)
        # power-grid-model's line results, in branch_data order (in-service branches), and the
        # lines' rated currents from the input: the branch-flow golden vectors
        lines_out = {ln["id"]: ln for ln in ref.get("line", [])}
        lines_in = {ln["id"]: ln for ln in json.load(open(inp))["data"].get("line", [])}
        keys = ("p_from", "q_from", "i_from", "s_from", "p_to", "q_to", "i_to", "s_to", "loading")
        bids = [int(b[0]) for b in branch_data]
        extra = {}
        if bids and all(b in lines_out and b in lines_in for b in bids):
            extra["pgm_line"] = np.array([[float(lines_out[b][kk]) for kk in keys] for b in bids])
            extra["pgm_line_i_n"] = np.array([float(lines_in[b]["i_n"]) for b in bids])
        if case in PGM_JSON_CASES:
            # the PGM input itself (zlib-compressed JSON text), for the PGM reader's tests
            import zlib

            extra["pgm_input_json_z"] = np.frombuffer(zlib.compress(open(inp, "rb").read(), 9),
                                                      np.uint8)
            # and power-grid-model's whole output dataset, for the PGM writer's tests
            extra["pgm_output_json_z"] = np.frombuffer(
                zlib.compress(open(outp, "rb").read(), 9), np.uint8)
        save("pgm_" + case, bus_data=np.asarray(bus_data), branch_data=np.asarray(branch_data),
             base_power=np.float64(net.base_power), pgm_u_pu=pgm_u, pgm_u_angle=pgm_a,
             **sol, **extra)
        made.append(case)
    return made


def make_c0():
    for seed in range(5):
        net = synth.feeder_grid(seed)
        save(f"c0_seed{seed}", **net_arrays(net), base_power=np.float64(1e6), **ref_all(net))


def kat_networks():
    """Small networks; IDs, units and values follow the reference unit tests where named."""
    k = {}
    # 2-bus, test_admittance.cpp:89-151 (230 kV, r=0.02, x=0.06, b=0.05; 100 MW / 50 Mvar load)
    k["two_bus"] = Network.build(bus_id=[1, 2], u_rated=[230e3, 230e3], bus_type=[SLACK, PQ],
                                 u_pu=[1.0, 1.0], p=[0.0, -100e6], q=[0.0, -50e6],
                                 from_id=[1], to_id=[2], r1=[0.02 * 529], x1=[0.06 * 529],
                                 b1=[0.05 / 529])
    # 3-bus triangle with a PV bus (test_admittance.cpp:153-233 topology)
    k["three_bus_pv"] = Network.build(
        bus_id=[0, 1, 2], u_rated=[10e3] * 3, bus_type=[SLACK, PV, PQ], u_pu=[1.0, 1.02, 1.0],
        p=[0.0, 0.3e6, -0.8e6], q=[0.0, 0.0, -0.3e6], from_id=[0, 1, 0], to_id=[1, 2, 2],
        r1=[0.3, 0.4, 0.5], x1=[0.6, 0.5, 0.9], b1=[1e-6, 0.0, 2e-6])
    # 4 buses: isolated bus 3 has a shunt only; branch 2 out of service (test_admittance.cpp:616-812)
    k["four_bus_isolated"] = Network.build(
        bus_id=[0, 1, 2, 3], u_rated=[10e3] * 4, bus_type=[SLACK, PQ, PQ, PQ],
        u_pu=[1.0] * 4, p=[0, -0.2e6, -0.1e6, 0.0], q=[0, -0.05e6, -0.02e6, 0.0],
        from_id=[0, 1, 0], to_id=[1, 2, 2], status=[1, 1, 0], r1=[0.2, 0.3, 0.4],
        x1=[0.4, 0.5, 0.6], app_node=[3, 2], app_type=[SHUNT, SHUNT], app_g1=[0.0, 0.0],
        app_b1=[-0.03, 0.001])
    # parallel branches between buses 1 and 2 (duplicates kept in the CSR) + an unknown bus ID
    k["parallel_branches"] = Network.build(
        bus_id=[0, 1, 2], u_rated=[10e3] * 3, bus_type=[SLACK, PQ, PQ], u_pu=[1.0] * 3,
        p=[0, -0.3e6, -0.4e6], q=[0, -0.1e6, -0.1e6], from_id=[0, 1, 2, 1, 7],
        to_id=[1, 2, 1, 0, 1], r1=[0.2, 0.3, 0.35, 0.25, 0.1], x1=[0.4, 0.5, 0.55, 0.45, 0.2],
        g1=[0.0, 1e-5, 0.0, 0.0, 0.0], b1=[0.0, 1e-6, 2e-6, 0.0, 0.0])
    # appliances: loads/sources summed into S_spec (cpu_newton_raphson.cpp:359-369), one off
    k["appliances"] = Network.build(
        bus_id=[10, 11, 12], u_rated=[10e3] * 3, bus_type=[SLACK, PQ, PQ], u_pu=[1.0] * 3,
        p=[0, -0.1e6, 0.0], q=[0, 0.0, 0.0], from_id=[10, 11], to_id=[11, 12], r1=[0.2, 0.3],
        x1=[0.4, 0.5], app_node=[11, 12, 12, 12, 10],
        app_type=[LOADGEN, LOADGEN, LOADGEN, SOURCE, SHUNT],
        app_p=[-0.05e6, -0.2e6, -0.5e6, 0.0, 0.0], app_q=[-0.01e6, -0.05e6, -0.1e6, 0.0, 0.0],
        app_status=[1, 1, 0, 1, 1], app_b1=[0.0, 0.0, 0.0, 0.0, 0.002])
    # zero-impedance branch (y = 0 below |z|^2 <= 1e-12) next to a normal one
    k["zero_impedance"] = Network.build(
        bus_id=[0, 1, 2], u_rated=[10e3] * 3, bus_type=[SLACK, PQ, PQ], u_pu=[1.0] * 3,
        p=[0, -0.1e6, -0.1e6], q=[0, 0, 0], from_id=[0, 1, 0], to_id=[1, 2, 2],
        r1=[0.2, 0.0, 0.3], x1=[0.4, 1e-7, 0.5])
    return k


def make_kats():
    for name, net in kat_networks().items():
        out = dict(**net_arrays(net), base_power=np.float64(1e6), **ref_all(net))
        # mismatch at flat start and at a perturbed point, reference public API (Watts,
        # base 100 MVA; cpu_newton_raphson.cpp:225-240)
        v0 = np.where(net.bus_type == PQ, 0.98, net.u_pu).astype(np.complex128)
        v1 = v0 * np.exp(1j * 0.01 * np.arange(net.n_bus))
        out["mm_v0"] = v0
        out["mm_f0"] = refnet.mismatch(net, v0)
        out["mm_v1"] = v1
        out["mm_f1"] = refnet.mismatch(net, v1)
        save("kat_" + name, **out)
    # Y-bus update (update_admittance_matrix, cpu_admittance_matrix.cpp:204-301): take branch
    # 1 of the triangle out of service
    net = kat_networks()["three_bus_pv"]
    ch = Network.build(bus_id=[0], u_rated=[10e3], bus_type=[SLACK], from_id=[1], to_id=[2],
                       status=[0], r1=[0.4], x1=[0.5], b1=[0.0])
    rp, ci, va = refnet.ybus_update(net, ch)
    save("kat_update", **net_arrays(net), **net_arrays(ch, "ch_"), y_row_ptr=rp,
         y_col_idx=ci, y_values=va)


def make_lu():
    rng = np.random.default_rng(7)
    cases = {}
    # 3x3 KAT of test_lu_solver.cpp:94-140 style plus random diagonally dominant systems
    for n, dens in ((3, 1.0), (10, 0.3), (60, 0.08), (120, 0.04)):
        A = (rng.random((n, n)) < dens) * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
        A += np.diag(n * (1.0 + rng.random(n)) + 0j)
        rows, cols = np.nonzero(A)
        rp = np.zeros(n + 1, np.int32)
        np.add.at(rp, rows + 1, 1)
        rp = np.cumsum(rp).astype(np.int32)
        vals = A[rows, cols]
        b = rng.normal(size=n) + 1j * rng.normal(size=n)
        st, x = refnet.lu_solve(rp, cols.astype(np.int32), vals, b)
        cases[f"n{n}"] = dict(row_ptr=rp, col_idx=cols.astype(np.int32), values=vals, rhs=b,
                              ref_status=np.int32(st), ref_x=x)
    for k, v in cases.items():
        save("lu_" + k, **v)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True,
                    help="the reference checkout (its PGM validation cases are read from it)")
    a = ap.parse_args()
    if not refnet.available():
        raise SystemExit("build the reference oracle first: make -C oracle REF=" + a.ref)
    print("pgm:", make_pgm(a.ref))
    make_c0()
    make_kats()
    make_lu()
    print("done")
