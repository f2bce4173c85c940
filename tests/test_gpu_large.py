"""100k-bus grid, FP32 factor + FP64 refinement, against the FP64 oracle (minutes of host
analysis and oracle time: runs only with GAP_B200_LARGE=1)."""

import json
import os

import numpy as np
import pytest

from oracle import restate

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("GAP_B200_LARGE") != "1",
                                 reason="100k-bus case: set GAP_B200_LARGE=1")]

BASE = 1e8


def test_100k_bus_mixed_precision_matches_fp64_oracle():
    import torch

    from gap_b200 import studies, synth

    net = synth.transmission_grid(0, n=100_000)
    v0 = synth.dc_start(net, BASE)
    S = 8
    s_load = synth.load_scenarios(net, S, sigma=0.1, seed=1, base_power=BASE)
    st = studies.load_study("large", net, s_load, v0, base_power=BASE)
    st.lanes, st.threads = 8, 1024
    b = st.make_batch()
    r = b.solve(st.y, st.s_spec, v_init=st.v0, tol=1e-8, max_iter=30, policy="clamped",
                refine=1)
    torch.cuda.synchronize()
    assert (r.status.cpu().numpy() == 0).all()
    V = r.v.cpu().numpy()
    Y = restate.ybus_pi(net)
    out = {"n_tail": st.plan.info["n_tail"], "iterations": r.iterations.cpu().tolist()}
    for s in (0, S - 1):
        o = restate.nr_solve(net, Y=Y, tol=1e-8, max_iter=30, base_power=BASE,
                             policy="clamped", jac="exact", s_spec=s_load[s], v0=v0)
        assert o["converged"]
        dv = float(np.max(np.abs(np.abs(V[s]) - np.abs(o["v"]))))
        da = float(np.max(np.abs(np.angle(V[s]) - np.angle(o["v"]))))
        out[f"scenario{s}"] = {"oracle_iterations": o["iterations"], "max_dvm": dv,
                               "max_dangle": da}
        assert dv < 1e-7 and da < 1e-7
    print(json.dumps(out))
