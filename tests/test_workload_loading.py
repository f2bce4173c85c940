"""Why the transmission workload's loading is 0.05 pu per bus, not the written U[0,1] pu.

The generator's loads (p ~ U[0,1] x load_scale pu, q proportional to p) and its local PV
dispatch (each PV bus generates its region's load) are linear in load_scale, so the written
loading is S_spec(1) = 20 x S_spec(0.05) of the same grid.  A load-scale continuation with the
FP64 oracle (pure Newton from the previous solution, step halved on failure down to 1e-3 of
the written loading) follows the solution branch from 0.05 up to its nose point, where it
ends: well below 1, so the written loading has no power-flow solution on this grid, and 0.05
sits at about a fifth of the loadability limit."""

import numpy as np
import pytest

from oracle import restate

pytestmark = pytest.mark.slow

BASE = 1e8


def test_written_loading_is_beyond_the_nose_point():
    from gap_b200 import synth
    from gap_b200 import workloads as W

    net = synth.transmission_grid(W.GRID_SEED, n=W.N_BUS)
    written = synth.transmission_grid(W.GRID_SEED, n=W.N_BUS, load_scale=1.0)
    s1 = written.specified_power(BASE)
    s05 = net.specified_power(BASE)
    # the same grid; only loads and PV dispatch scale, linearly
    assert np.array_equal(net.bus_type, written.bus_type) and np.array_equal(net.x1, written.x1)
    assert np.max(np.abs(synth.LOAD_SCALE * s1 - s05)) <= 1e-14 * np.max(np.abs(s05))
    Y = restate.ybus_pi(net)

    def solve(t, v0, max_iter):
        o = restate.nr_solve(net, Y=Y, tol=1e-8, max_iter=max_iter, base_power=BASE,
                             policy="newton", jac="exact", s_spec=t * s1, v0=v0)
        # a collapsed iterate (|V| -> 0) is not the high-voltage solution branch
        ok = o["converged"] and float(np.min(np.abs(o["v"]))) > 0.3
        return ok, o["v"]

    t = synth.LOAD_SCALE
    ok, v = solve(t, synth.dc_start(net, BASE), 20)
    assert ok
    h = 0.05
    while h > 1e-3 and t < 1.0:
        ok, v_new = solve(min(1.0, t + h), v, 12)
        if ok:
            t = min(1.0, t + h)
            v = v_new
            h *= 1.5
        else:
            h /= 2
    print(f"solution branch ends at load scale {t:.4f} (min |V| {np.min(np.abs(v)):.3f} pu)")
    assert t < 0.5
    assert t > 4 * synth.LOAD_SCALE
