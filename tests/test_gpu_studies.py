"""Mixed batches (load scenarios, N-1 contingencies sharing one plan, independent grids) run
concurrently on CUDA streams, against the FP64 oracle."""

import numpy as np
import pytest

from oracle import restate

pytestmark = pytest.mark.gpu

BASE = 1e8


def _check(V, net, s_spec, v0, Y, tol=1e-8):
    o = restate.nr_solve(net, Y=Y, tol=1e-12, max_iter=30, base_power=BASE, policy="newton",
                         jac="exact", s_spec=s_spec, v0=v0)
    assert o["converged"]
    assert np.max(np.abs(np.abs(V) - np.abs(o["v"]))) < tol
    assert np.max(np.abs(np.angle(V) - np.angle(o["v"]))) < tol


def test_mixed_studies_concurrent_match_oracle():
    import torch

    from gap_b200 import studies, synth

    net = synth.transmission_grid(4, n=600)
    v0 = synth.dc_start(net, BASE)
    s_load = synth.load_scenarios(net, 24, sigma=0.1, seed=9, base_power=BASE)
    load = studies.load_study("load", net, s_load, v0, base_power=BASE)
    outs = synth.n_minus_1(net, 12, seed=5)
    s0 = net.specified_power(BASE)
    cont = studies.contingency_study("n-1", net, outs, s0, v0, base_power=BASE, plan=load.plan)
    grids = []
    for i, n in enumerate((300, 800, 1500)):
        g = synth.transmission_grid(20 + i, n=n)
        grids.append(studies.load_study(f"grid{n}", g, g.specified_power(BASE)[None],
                                        synth.dc_start(g, BASE), base_power=BASE))
    lanes, threads = studies.autotune(load, tol=1e-10, max_iter=30,
                                      candidates=((8, 512), (4, 256), (1, 256)))
    assert (lanes, threads) in ((8, 512), (4, 256), (1, 256))
    assert studies.autotune(load, tol=1e-10, max_iter=30) == (lanes, threads)  # cached
    all_st = [load, cont] + grids
    studies.solve_concurrent(all_st, tol=1e-10, max_iter=30, policy="newton", refine=1)
    torch.cuda.synchronize()
    for st in all_st:
        assert (st.result.status.cpu().numpy() == 0).all(), st.name
    Y = restate.ybus_pi(net)
    V = load.result.v.cpu().numpy()
    for s in (0, 13, 23):
        _check(V[s], net, s_load[s], v0, Y)
    V = cont.result.v.cpu().numpy()
    for s in (0, 5, 11):
        nk = studies.outage_network(net, int(outs[s]))
        _check(V[s], nk, s0, v0, restate.ybus_pi(nk))
    # different outages give different solutions
    assert np.max(np.abs(V[0] - V[1])) > 1e-6
    for g in grids:
        Vg = g.result.v.cpu().numpy()[0]
        _check(Vg, g.net, g.s_spec.cpu().numpy()[0], g.v0.cpu().numpy()[0],
               restate.ybus_pi(g.net))
    # a second round reuses the batches and graphs and gives the same voltages
    first = [st.result.v.clone() for st in all_st]
    studies.solve_concurrent(all_st, tol=1e-10, max_iter=30, policy="newton", refine=1)
    torch.cuda.synchronize()
    for st, v in zip(all_st, first):
        assert torch.equal(st.result.v, v), st.name
