"""Branch results on the device (gapk_branch_flows) against the oracle's restatement and
power-grid-model's own line outputs (the reference's PGM validation data)."""

import numpy as np
import pytest

from helpers import fixture_names, network_of
from oracle import restate

pytestmark = pytest.mark.gpu


def _rel(a, b):
    scale = np.max(np.abs(b), axis=0)
    return np.max(np.abs(a - b), axis=0) / np.where(scale > 0, scale, 1.0)


@pytest.mark.parametrize("name", fixture_names("pgm_"))
def test_branch_flows_pgm_cases(name):
    import torch

    from gap_b200.engine import branch_flows

    net, d = network_of(name)
    base = float(d["base_power"])
    for v in (d["pgm_u_pu"] * np.exp(1j * np.deg2rad(d["pgm_u_angle"])), d["ref_v"]):
        out = branch_flows(net, torch.as_tensor(v[None], device="cuda"), base, taps=False,
                           i_n=d["pgm_line_i_n"]).cpu().numpy()[0]
        orc, idx = restate.branch_flows(net, v, base, i_n=d["pgm_line_i_n"], taps=False)
        assert np.all(_rel(out[idx], orc) < 1e-10)
        assert np.all(_rel(out[idx], d["pgm_line"]) < 1e-6)


def test_branch_flows_batched_taps_and_outages():
    import dataclasses

    import torch

    from gap_b200 import synth
    from gap_b200.engine import branch_flows

    net = synth.transmission_grid(9, n=500)
    st = net.status.copy()
    st[[3, 17]] = 0
    net = dataclasses.replace(net, status=st)
    base = 1e8
    rng = np.random.default_rng(2)
    S = 3
    V = np.stack([synth.dc_start(net, base) * (1 + 0.01 * rng.normal(size=net.n_bus))
                  for _ in range(S)])
    i_n = rng.uniform(500, 1500, net.n_branch)
    out = branch_flows(net, torch.as_tensor(V, device="cuda"), base, taps=True,
                       i_n=i_n).cpu().numpy()
    for s in range(S):
        orc, idx = restate.branch_flows(net, V[s], base, i_n=i_n, taps=True)
        assert np.all(_rel(out[s, idx], orc) < 1e-10)
        assert np.all(out[s, [3, 17]] == 0.0)
        # losses are non-negative on every in-service branch
        assert np.all(out[s, idx, 0] + out[s, idx, 4] > -1e-6 * np.abs(out[s, idx, 0]).max())
