"""Heterogeneous batches in one launch (gapk_nr_mix_*, studies.solve_mixed): load scenarios of
a grid, N-1 contingencies sharing that grid's plan, and independent grids of other sizes --
among them a 15,532-bus grid on which pure Newton from the DC start diverges -- solved by one
graph launch with the headline's FP32 + refinement settings, unconverged scenarios retried with
the clamped step policy inside the same launch.

Checks: every scenario converges; sampled scenarios of every study match the FP64 oracle to
1e-8 pu / rad (|V|, angle); the studies that converge without the retry give bit-for-bit the
voltages of their own batch solved alone."""

import dataclasses

import numpy as np
import pytest

from oracle import restate

pytestmark = pytest.mark.gpu

BASE = 1e8
KW = dict(tol=1e-8, max_iter=20, policy="newton", refine=2, refine_below=1e-2, reuse_below=1e-2)


def _studies():
    from gap_b200 import studies, synth

    net = synth.transmission_grid(5, n=1000)
    v0 = synth.dc_start(net, BASE)
    load = studies.load_study("load", net, synth.load_scenarios(net, 12, sigma=0.1, seed=3,
                                                                base_power=BASE), v0,
                              base_power=BASE)
    outs = synth.n_minus_1(net, 6)
    cont = studies.contingency_study("n-1", net, outs, net.specified_power(BASE), v0,
                                     base_power=BASE, plan=load.plan)
    grids = []
    sizes = synth.grid_sizes(64)
    for i in (33, 5, 12):  # grid 33 (15,532 buses) diverges under pure Newton from DC angles
        g = synth.transmission_grid(100 + i, n=int(sizes[i]))
        grids.append(studies.load_study(f"grid{i}", g, g.specified_power(BASE)[None],
                                        synth.dc_start(g, BASE), base_power=BASE))
    return [load, cont] + grids


def _check(v, net, s_spec, v0, Y, policy):
    o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=BASE, policy=policy,
                         jac="exact", s_spec=s_spec, v0=v0)
    assert o["converged"]
    dvm = float(np.max(np.abs(np.abs(v) - np.abs(o["v"]))))
    dva = float(np.max(np.abs(np.angle(v) - np.angle(o["v"]))))
    assert dvm <= 1e-8 and dva <= 1e-8, (dvm, dva)
    return max(dvm, dva)


def test_mixed_batch_one_launch_with_clamped_retry_matches_oracle():
    import torch

    from gap_b200 import studies
    from gap_b200.engine import NRBatch

    sts = _studies()
    for st in sts:
        st.lanes, st.threads = (8, 512) if st.n_scen >= 8 else (1, 512)
    # pure Newton alone leaves grid 33 unconverged
    alone = {}
    for st in sts:
        b = NRBatch(st.plan, st.n_scen, precision="fp32", y_shared=st.y_shared, lanes=st.lanes,
                    threads=st.threads)
        r = b.solve(st.y, st.s_spec, v_init=st.v0, **KW)
        torch.cuda.synchronize()
        alone[st.name] = (r.v.clone(), r.status.clone())
    assert int(alone["grid33"][1][0].item()) != 0
    res = studies.solve_mixed(sts, retry="clamped", **KW)
    torch.cuda.synchronize()
    for st, r in zip(sts, res):
        assert (r.status.cpu().numpy() == 0).all(), (st.name, r.status.cpu().numpy())
    # a second launch reuses the graph and gives the same results
    v_first = [r.v.clone() for r in res]
    res = studies.solve_mixed(sts, retry="clamped", **KW)
    torch.cuda.synchronize()
    for a, r in zip(v_first, res):
        assert torch.equal(a, r.v)
    # studies that converged on their own: bit for bit the batch solved alone
    for st, r in zip(sts, res):
        if (alone[st.name][1].cpu().numpy() == 0).all():
            assert torch.equal(alone[st.name][0], r.v), st.name
    worst = 0.0
    load, cont = sts[0], sts[1]
    Y = restate.ybus_pi(load.net)
    s_load = load.s_spec.cpu().numpy()
    v0 = load.v0[0].cpu().numpy()
    for s in (0, 11):
        worst = max(worst, _check(res[0].v[s].cpu().numpy(), load.net, s_load[s], v0, Y,
                                  "newton"))
    for k in (0, 5):
        b = int(cont.info["outages"][k])
        st_ = cont.net.status.copy()
        st_[b] = 0
        out_net = dataclasses.replace(cont.net, status=st_)
        worst = max(worst, _check(res[1].v[k].cpu().numpy(), out_net,
                                  cont.s_spec[k].cpu().numpy(), v0, restate.ybus_pi(out_net),
                                  "newton"))
    for st, r in zip(sts[2:], res[2:]):
        pol = "clamped" if st.name == "grid33" else "newton"
        worst = max(worst, _check(r.v[0].cpu().numpy(), st.net, st.s_spec[0].cpu().numpy(),
                                  st.v0[0].cpu().numpy(), restate.ybus_pi(st.net), pol))
    print(f"mixed batch, one launch: worst |dV| / dtheta vs FP64 oracle {worst:.2e}")
