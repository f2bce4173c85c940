"""The command-line flow of the reference (src/main/main.cpp: IO module -> admittance matrix ->
LU solver -> power-flow solver -> write_results) over the B200 libraries: gap_b200_main reads
the reference's PGM validation inputs through libgap_io_pgm.so (loads as consumption), solves
them on the GPU through the reference-ABI plugins and writes a PGM output dataset whose node
voltages must match power-grid-model's within the reference's own criterion, 5e-6 pu
(tests/pgm_validation/test_pgm_validation.py:38-43)."""

import json
import os
import subprocess
import zlib

import numpy as np
import pytest

from helpers import fixture_names, load, pgm_output

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gap_b200", "lib", "gap_b200_main")
CASES = [n for n in fixture_names("pgm_") if "pgm_input_json_z" in load(n)]


@pytest.mark.parametrize("name", CASES)
def test_cli_solves_pgm_input_like_power_grid_model(name, tmp_path):
    d = load(name)
    inp = tmp_path / "input.json"
    out = tmp_path / "output.json"
    inp.write_text(zlib.decompress(d["pgm_input_json_z"].tobytes()).decode())
    r = subprocess.run([CLI, "-i", str(inp), "-o", str(out), "-b", "gpu", "-t", "1e-8", "-m",
                        "20", "--base-power", str(float(d["base_power"])), "--benchmark"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Status: CONVERGED" in r.stdout
    res = json.loads(out.read_text())
    assert res["type"] == "sym_output" and res["converged"] is True
    mine = {n["id"]: n["u_pu"] for n in res["data"]["node"]}
    ref = {n["id"]: n["u_pu"] for n in pgm_output(d)["node"]}
    assert set(mine) == set(ref)
    err = max(abs(mine[k] - ref[k]) for k in ref)
    print(f"{name}: CLI u_pu vs power-grid-model {err:.2e}")
    assert err < 5e-6


def test_cli_refuses_the_cpu_backend(tmp_path):
    r = subprocess.run([CLI, "-i", "x.json", "-o", "y.json", "-b", "cpu"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "Invalid backend" in r.stderr
