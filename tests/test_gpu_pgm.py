"""PGM input JSON -> device engine -> PGM-style results: the node voltages and line results of
power-grid-model (the reference's PGM validation data) reproduced through the reader, a
batched device solve of a batch-update dataset, and the device branch results."""

import json
import zlib

import numpy as np
import pytest

from helpers import compare_pgm_output, network_of, pgm_output
from oracle import restate

pytestmark = pytest.mark.gpu

CASES = ("pgm_radial_2feeder_8nodepf", "pgm_radial_3feeder_8nodepf")


@pytest.mark.parametrize("name", CASES)
def test_pgm_json_batch_update_end_to_end(name):
    import torch

    from gap_b200 import pgm
    from gap_b200.engine import NRBatch, NRPlan, YbusPlan, branch_flows, branch_params, \
        shunt_params

    _, d = network_of(name)
    doc = json.loads(zlib.decompress(d["pgm_input_json_z"].tobytes()).decode())
    net, extra = pgm.read_input(doc)
    base = float(d["base_power"])
    scale = [1.0, 0.6, 1.3, 0.9]
    upd = [{"sym_load": [{"id": ld["id"], "p_specified": f * ld["p_specified"],
                          "q_specified": f * ld["q_specified"]}
                         for ld in doc["data"]["sym_load"]]} for f in scale]
    s_spec = pgm.read_update(net, upd, base)
    zb = float(net.u_rated[0]) ** 2 / base
    yp = YbusPlan.from_network(net)
    y = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                    torch.as_tensor(shunt_params(net), device="cuda"), mode=0, scale=zb)[0]
    plan = NRPlan(yp.row_ptr, yp.col_idx, net.bus_type)
    b = NRBatch(plan, len(scale), precision="fp64", lanes=4)
    u = torch.as_tensor(net.u_pu.astype(np.float64), device="cuda")
    r = b.solve(y, torch.as_tensor(s_spec, device="cuda"), u_pu=u, tol=1e-10, max_iter=30,
                policy="reference")
    torch.cuda.synchronize()
    assert (r.status.cpu().numpy() == 0).all()
    V = r.v.cpu().numpy()
    # scenario 0 is the input itself: power-grid-model's voltages and line results
    assert np.max(np.abs(np.abs(V[0]) - d["pgm_u_pu"])) < 5e-6
    assert np.max(np.abs(np.angle(V[0]) - np.deg2rad(d["pgm_u_angle"]))) < 5e-6
    flows = branch_flows(net, r.v, base, taps=False, i_n=extra["i_n"]).cpu().numpy()
    ref = d["pgm_line"]
    scale_ref = np.max(np.abs(ref), axis=0)
    assert np.all(np.max(np.abs(flows[0] - ref), axis=0) / scale_ref < 1e-7)
    # the whole PGM output dataset of the input scenario through the writer: node voltages and
    # injections (device state), line, load and source results
    _, _, s_bus = b.state()
    all_flows = branch_flows(net, r.v, base, taps=False, i_n=extra["i_n"])
    out = pgm.write_output(net, extra, r.v, s_bus, all_flows, base)
    assert len(out) == len(scale)
    compare_pgm_output(out[0], pgm_output(d), rtol=1e-7)
    # every scenario against the FP64 oracle on the same S_spec
    for s in range(len(scale)):
        o = restate.nr_solve(net, tol=1e-12, max_iter=40, base_power=base, s_spec=s_spec[s])
        assert o["converged"]
        assert np.max(np.abs(V[s] - o["v"])) < 1e-8
    # heavier loading, lower voltages at the feeder ends
    assert np.abs(V[2]).min() < np.abs(V[0]).min() < np.abs(V[1]).min()
