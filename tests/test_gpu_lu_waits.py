"""Bounded waits of the tensor-core dense LU, made to run out without a GPU fault.

k_dense_lu_tc (one CTA per scenario) and k_dlu_update_tc (the split path) wait for their MMAs on
an mbarrier with a bounded number of polls.  With the batch's wait test on
(gapk_nr_batch_set_wait_test) they issue no MMAs, so every such wait runs out: each factorising
scenario must end SINGULAR with its start voltages and iterations = max_iterations, the batch's
device error word must read 1, and with the test off the same batch (same graph) must solve
normally again -- the kernels freed their tensor memory and the context stays usable."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(n_bus, S, seed):
    import torch

    from gap_b200 import synth
    from gap_b200.engine import NRPlan, YbusPlan, branch_params, shunt_params

    net = synth.transmission_grid(seed, n=n_bus)
    base = 1e8
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    s = torch.as_tensor(synth.load_scenarios(net, S, sigma=0.1, seed=seed, base_power=base),
                        device="cuda")
    v0 = torch.as_tensor(synth.dc_start(net, base), device="cuda")
    return plan, y, s, v0


@pytest.mark.parametrize("fused", [True, False])
def test_tensor_core_lu_wait_runs_out_and_recovers(fused):
    import torch

    from gap_b200 import _native as N
    from gap_b200.engine import NRBatch

    # 6000 buses: a dense tail of order 282, so both kernels have full 128 x 128 tiles
    plan, y, s, v0 = _setup(6000, 8, 4)
    assert 2 * plan.info["n_tail"] >= 256
    kw = dict(tol=1e-8, max_iter=20, policy="newton", refine=1)
    b = NRBatch(plan, 8, precision="fp32", lanes=8, dense_fused=fused)
    good = b.solve(y, s, v_init=v0, **kw)
    torch.cuda.synchronize()
    assert (good.status.cpu().numpy() == N.SCEN_CONVERGED).all()
    assert not b.device_error()
    v_good = good.v.clone()

    b.set_wait_test(True)
    t0 = time.perf_counter()
    bad = b.solve(y, s, v_init=v0, **kw)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    st = bad.status.cpu().numpy()
    assert (st == N.SCEN_SINGULAR).all(), st
    assert (bad.iterations.cpu().numpy() == kw["max_iter"]).all()
    # the reference keeps V where it was when the factorisation fails: the start vector
    np.testing.assert_array_equal(bad.v.cpu().numpy(), np.broadcast_to(v0.cpu().numpy(),
                                                                       bad.v.shape))
    assert b.device_error()
    print(f"fused={fused}: waits ran out, solve returned after {elapsed:.1f} s")

    b.set_wait_test(False)
    again = b.solve(y, s, v_init=v0, **kw)
    torch.cuda.synchronize()
    assert (again.status.cpu().numpy() == N.SCEN_CONVERGED).all()
    assert not b.device_error()
    assert torch.equal(again.v, v_good)
