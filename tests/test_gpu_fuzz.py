"""Randomised parity: seeded random small networks (random topology with parallel and
out-of-service branches, PV buses, shunts, transformers with taps and phase shifts, shuffled
bus IDs) solved on the device and by the oracle."""

import numpy as np
import pytest

from helpers import random_network
from oracle import restate

pytestmark = pytest.mark.gpu

SEEDS = range(24)


@pytest.mark.parametrize("seed", SEEDS)
def test_reference_path_matches_oracle_on_random_networks(seed):
    """Reference Y-bus, reference step policy, FP64, through the Python API: same
    convergence flag, iterations within +-1, converged voltages within 1e-8."""
    from gap_b200.api import NewtonRaphson, PowerFlowConfig

    net = random_network(seed)
    cfg = PowerFlowConfig(tolerance=1e-8, max_iterations=50, base_power=1e6)
    r = NewtonRaphson().solve_power_flow(net, None, cfg)
    o = restate.nr_solve(net, tol=1e-8, max_iter=50, base_power=1e6)
    assert r.converged == o["converged"]
    if o["converged"]:
        assert abs(r.iterations - o["iterations"]) <= 1
        assert np.max(np.abs(np.abs(r.bus_voltages) - np.abs(o["v"]))) < 1e-8
        assert np.max(np.abs(np.angle(r.bus_voltages) - np.angle(o["v"]))) < 1e-8


@pytest.mark.parametrize("seed", SEEDS)
def test_batched_mixed_precision_matches_oracle_on_random_networks(seed):
    """Pi-model Y-bus with taps, Newton policy, 5 load scenarios in one FP32 batch with FP64
    refinement, against the FP64 oracle: voltages within 1e-8."""
    import torch

    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_params, shunt_params

    net = random_network(seed)
    base = 1e6
    zb = net.u_rated[0] ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type, jacobian="exact")
    rng = np.random.default_rng(seed)
    scale = rng.uniform(0.7, 1.2, 5)
    s_spec = np.stack([net.specified_power(base) * f for f in scale])
    u = torch.as_tensor(net.u_pu.astype(np.float64), device="cuda")
    b = NRBatch(plan, len(scale), precision="fp32", lanes=4)
    r = b.solve(y, torch.as_tensor(s_spec, device="cuda"), u_pu=u, tol=1e-10, max_iter=30,
                policy="newton", refine=1)
    torch.cuda.synchronize()
    V = r.v.cpu().numpy()
    st = r.status.cpu().numpy()
    Y = restate.ybus_pi(net)
    for s in range(len(scale)):
        o = restate.nr_solve(net, Y=Y, tol=1e-10, max_iter=30, base_power=base,
                             policy="newton", jac="exact", s_spec=s_spec[s])
        assert (st[s] == 0) == o["converged"]
        if o["converged"]:
            assert np.max(np.abs(V[s] - o["v"])) < 1e-8
