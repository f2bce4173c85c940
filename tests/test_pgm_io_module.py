"""The C++ PGM reader behind the reference's IO interface (libgap_io_pgm.so,
create_pgm_io_module), read through a driver compiled against the reference's own headers
(oracle/_ref/abi_driver --io): the NetworkData it produces -- buses, branches, appliances,
bus types -- must equal what the Python reader (gap_b200.pgm.read_input) makes of the same
file, with loads as negative injections.  No GPU: the reader is host code."""

import json
import os
import subprocess
import zlib

import numpy as np
import pytest

from helpers import fixture_names, load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "abi_driver")
LIB = os.path.join(ROOT, "gap_b200", "lib")

pytestmark = pytest.mark.skipif(
    not (os.path.exists(DRIVER) and os.path.exists(os.path.join(LIB, "libgap_io_pgm.so"))),
    reason="reference-built driver or libgap_io_pgm.so not built")

CASES = [n for n in fixture_names("pgm_") if "pgm_input_json_z" in load(n)]

# every component the reader knows, with statuses off, taps, clocks and defaults exercised
SYNTHETIC = {
    "version": "1.0", "type": "input", "is_batch": False, "attributes": {},
    "data": {
        "node": [{"id": 1, "u_rated": 10500.0}, {"id": 2, "u_rated": 10500.0},
                 {"id": 3, "u_rated": 10500.0}, {"id": 7, "u_rated": 400.0}],
        "line": [{"id": 10, "from_node": 1, "to_node": 2, "from_status": 1, "to_status": 1,
                  "r1": 0.25, "x1": 0.2, "c1": 1e-6, "tan1": 0.001, "i_n": 420.0},
                 {"id": 11, "from_node": 2, "to_node": 3, "from_status": 1, "to_status": 0,
                  "r1": 0.3, "x1": 0.1}],
        "transformer": [{"id": 20, "from_node": 3, "to_node": 7, "from_status": 1,
                         "to_status": 1, "u1": 10500.0, "u2": 400.0, "sn": 630e3,
                         "uk": 0.06, "rx_ratio": 0.15, "tap_pos": 2, "tap_size": 250.0,
                         "clock": 5}],
        "generic_branch": [{"id": 30, "from_node": 1, "to_node": 3, "from_status": 1,
                            "to_status": 1, "r1": 0.5, "x1": 0.7, "g1": 1e-6, "b1": 2e-6,
                            "k": 1.02, "shift": 0.05, "sn": 1e6}],
        "source": [{"id": 40, "node": 1, "status": 1, "u_ref": 1.02, "u_ref_angle": 0.0,
                    "sk": 1e9, "rx_ratio": 0.1}],
        "sym_load": [{"id": 50, "node": 2, "status": 1, "type": 0, "p_specified": 1e5,
                      "q_specified": 3e4},
                     {"id": 51, "node": 7, "status": 0, "type": 0, "p_specified": 2e4,
                      "q_specified": 1e4}],
        "sym_gen": [{"id": 60, "node": 3, "status": 1, "type": 0, "p_specified": 5e4,
                     "q_specified": -1e4}],
        "shunt": [{"id": 70, "node": 2, "status": 1, "g1": 1e-5, "b1": 2e-4}],
    },
}


def _read(path):
    out = subprocess.run([DRIVER, "--io", LIB, path], capture_output=True, text=True,
                         timeout=60)
    assert out.returncode == 0, out.stderr
    rows = {"bus": [], "br": [], "app": []}
    head = {}
    for line in out.stdout.splitlines():
        k, *v = line.split()
        if k in rows:
            rows[k].append([float(x) for x in v])
        else:
            head[k] = [int(x) for x in v]
    return head, {k: np.array(v).reshape(len(v), -1) for k, v in rows.items()}


def _compare(path, doc):
    from gap_b200 import pgm

    head, r = _read(path)
    net, extra = pgm.read_input(doc)
    assert head["valid"] == [1]
    assert head["counts"] == [net.n_bus, net.n_branch, net.n_app] * 2
    bus, br, app = r["bus"], r["br"], r["app"]
    assert np.array_equal(bus[:, 0], net.bus_id) and np.allclose(bus[:, 1], net.u_rated, rtol=1e-15)
    assert np.array_equal(bus[:, 2], net.bus_type)
    assert np.allclose(bus[:, 3], net.u_pu, rtol=1e-15)
    if net.n_branch:
        assert np.array_equal(br[:, 0], net.br_id)
        assert np.array_equal(br[:, 1], net.from_id) and np.array_equal(br[:, 2], net.to_id)
        assert np.array_equal(br[:, 3], net.status)
        for col, a in zip(range(4, 10), (net.r1, net.x1, net.g1, net.b1, net.k, net.theta)):
            np.testing.assert_allclose(br[:, col], a, rtol=1e-14, atol=1e-300)
        np.testing.assert_allclose(br[:, 10], extra["i_n"], rtol=1e-14)
        np.testing.assert_allclose(br[:, 11], extra["sn"], rtol=1e-14)
    if net.n_app:
        assert np.array_equal(app[:, 0], net.app_id) and np.array_equal(app[:, 1], net.app_node)
        assert np.array_equal(app[:, 2], net.app_status)
        assert np.array_equal(app[:, 3], net.app_type)
        for col, a in zip(range(4, 8), (net.app_p, net.app_q, net.app_g1, net.app_b1)):
            np.testing.assert_allclose(app[:, col], a, rtol=1e-15, atol=1e-300)
    return net


@pytest.mark.parametrize("name", CASES)
def test_io_module_reads_pgm_cases_as_the_python_reader(name, tmp_path):
    d = load(name)
    text = zlib.decompress(d["pgm_input_json_z"].tobytes()).decode()
    path = tmp_path / "input.json"
    path.write_text(text)
    net = _compare(str(path), json.loads(text))
    # loads are consumption: negative injections on every loaded bus
    loads = net.app_type == 1
    assert (net.app_p[loads] <= 0).all() and (net.app_p[loads] < 0).any()


def test_io_module_reads_every_component(tmp_path):
    path = tmp_path / "synthetic.json"
    path.write_text(json.dumps(SYNTHETIC))
    net = _compare(str(path), SYNTHETIC)
    # the source's bus is the slack at u_ref, every other bus PQ (no PV inference from loads)
    assert list(net.bus_type) == [2, 0, 0, 0] and net.u_pu[0] == 1.02


def test_io_module_rejects_non_pgm_files(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"data": {"line": []}}')
    out = subprocess.run([DRIVER, "--io", LIB, str(bad)], capture_output=True, text=True,
                         timeout=60)
    assert out.stdout.startswith("valid 0")
