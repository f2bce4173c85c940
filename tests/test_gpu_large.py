"""100k-bus grid, FP32 factor + FP64 refinement (about a minute, most of it host analysis).
A full FP64 oracle solve is out of reach at this size (one scipy SuperLU
factorisation of the 180k x 180k Jacobian takes minutes), so the check is the oracle's own FP64
mismatch at the device's solutions, and agreement of the mixed-precision solution with the
device's FP64 solve."""

import json

import numpy as np
import pytest

from oracle import restate

pytestmark = pytest.mark.gpu

BASE = 1e8


def test_100k_bus_mixed_precision_converges_and_matches_fp64():
    import torch

    from gap_b200 import studies, synth
    from gap_b200.engine import NRBatch

    net = synth.transmission_grid(0, n=100_000, load_scale=0.025)
    v0 = synth.dc_start(net, BASE)
    S = 8
    s_load = synth.load_scenarios(net, S, sigma=0.1, seed=1, base_power=BASE)
    st = studies.load_study("large", net, s_load, v0, base_power=BASE)
    kw = dict(tol=1e-8, max_iter=30, policy="clamped")
    b32 = NRBatch(st.plan, S, precision="fp32", lanes=8, threads=1024)
    r32 = b32.solve(st.y, st.s_spec, v_init=st.v0, refine=1, refine_below=1e-4, **kw)
    b64 = NRBatch(st.plan, S, precision="fp64", lanes=8, threads=1024)
    r64 = b64.solve(st.y, st.s_spec, v_init=st.v0, **kw)
    torch.cuda.synchronize()
    assert (r32.status.cpu().numpy() == 0).all() and (r64.status.cpu().numpy() == 0).all()
    V32, V64 = r32.v.cpu().numpy(), r64.v.cpu().numpy()
    rp, ci, va = restate.ybus_pi(net)
    ypu = va * (float(net.u_rated[0]) ** 2 / BASE)
    out = {"n_tail": st.plan.info["n_tail"], "iterations_fp32": r32.iterations.tolist(),
           "iterations_fp64": r64.iterations.tolist()}
    for s in range(S):
        for V in (V32[s], V64[s]):
            d = restate.mismatch(net.bus_type, restate.power_injections(rp, ci, ypu, V),
                                 s_load[s])
            assert np.max(np.abs(d)) < 1e-8
    out["max_dvm_fp32_vs_fp64"] = float(np.max(np.abs(np.abs(V32) - np.abs(V64))))
    out["max_dangle_fp32_vs_fp64"] = float(np.max(np.abs(np.angle(V32) - np.angle(V64))))
    assert out["max_dvm_fp32_vs_fp64"] < 1e-7 and out["max_dangle_fp32_vs_fp64"] < 1e-7
    print(json.dumps(out))
