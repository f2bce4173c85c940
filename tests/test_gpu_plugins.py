"""The drop-in boundary: the B200 plugin libraries loaded by a caller compiled against the
reference's own headers (oracle/_ref/abi_driver, built from oracle/abi_driver.cpp) and
compared, through the reference's interfaces, with the reference CPU backends."""

import os
import subprocess

import numpy as np
import pytest

from helpers import fixture_names, network_of

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "abi_driver")
LIBDIR = os.path.join(ROOT, "gap_b200", "lib")


def write_net(net, path, tol=1e-8, max_iter=20, base=1e6):
    def f(x):
        return repr(float(x))

    def i(x):
        return str(int(x))

    lines = [i(net.n_bus)]
    for k in range(net.n_bus):
        lines.append(" ".join([i(net.bus_id[k]), f(net.u_rated[k]), i(net.bus_type[k]),
                               f(net.u_pu[k]), f(net.p[k]), f(net.q[k])]))
    lines.append(i(net.n_branch))
    for b in range(net.n_branch):
        lines.append(" ".join([i(net.br_id[b]), i(net.from_id[b]), i(net.to_id[b]),
                               i(net.status[b])] + [f(getattr(net, a)[b]) for a in
                                                    ("r1", "x1", "g1", "b1", "k", "theta")]))
    lines.append(i(net.n_app))
    for a in range(net.n_app):
        lines.append(" ".join([i(net.app_id[a]), i(net.app_node[a]), i(net.app_status[a]),
                               i(net.app_type[a])] + [f(getattr(net, c)[a]) for c in
                                                      ("app_p", "app_q", "app_g1", "app_b1")]))
    lines.append(" ".join([f(tol), i(max_iter), f(base)]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def run_driver(net, tmp_path, base):
    p = tmp_path / "net.txt"
    write_net(net, p, base=base)
    r = subprocess.run([DRIVER, LIBDIR, str(p)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        k, *v = line.split()
        out[k] = [float(x) for x in v]
    return out


pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(DRIVER), reason="abi driver not built")]


@pytest.mark.parametrize("name", [n for n in fixture_names("kat_") if n != "kat_update"]
                         + ["c0_seed0", "c0_seed3", "pgm_radial_3feeder_8nodepf"])
def test_plugins_drop_in_against_reference_backends(name, tmp_path):
    net, d = network_of(name)
    o = run_driver(net, tmp_path, float(d["base_power"]))
    assert o["backend"] == [1, 1, 1]  # BackendType::GPU_CUDA from all three
    assert o["ybus_pattern_equal"] == [1] and o["ybus_values_equal"] == [1]
    assert o["update_rel_diff"][0] <= 1e-14
    cc, cg = o["nr_converged"]
    assert cc == cg
    ic, ig = o["nr_iterations"]
    assert abs(ic - ig) <= 1
    if cc:
        assert o["nr_max_dv"][0] < 1e-8 and o["nr_max_dangle"][0] < 1e-8
    # bus_injections: empty from the reference, S = V conj(Y V) per unit from the plugin
    n_ref_inj, d_inj, s_inj = o["nr_bus_injections"]
    assert n_ref_inj == 0 and d_inj <= 1e-12 * max(s_inj, 1.0)
    assert o["mismatch_sizes"][0] == o["mismatch_sizes"][1]
    dm, sm = o["mismatch_max_abs_diff"]
    assert dm <= 1e-9 * sm + 1e-6
    # iteration-state capture: one state per iteration on both sides, the same states along
    # the trajectory, and the capturing solve's result equal to the plain one
    nc, ng = o["capture_counts"]
    assert nc == ic and ng == ig
    assert o["capture_iteration_index"] == [1]
    if cc:
        assert max(o["capture_rel_diff"]) < 1e-9
        cm, cx, m0 = o["capture_mismatch_abs_diff"]
        assert cm <= 1e-9 * max(m0, 1.0) and cx <= 1e-9 * max(m0, 1.0)
    assert o["capture_result"] == [1, 1, 0.0]
    assert o["capture_cleared"] == [0]
    assert o["lu_factorized"] == [1, 1, 1]
    assert o["lu_rel_diff"][0] < 1e-10
    assert o["lu_bad_rhs_throws"] == [1]
