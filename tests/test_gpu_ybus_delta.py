"""Branch status changes on the device (gapk_ybus_apply_changes / gapk_ybus_delta_*): one
thread per touched CSR entry, each entry's changes in change order.

* reference mode: bit for bit the reference's update_admittance_matrix
  (src/admittance/cpu/cpu_admittance_matrix.cpp:204-301), golden output of the reference;
* fixed modes: update(build(net)) equals build(changed net) within 1e-14 of the largest entry
  (summing duplicate entries), for a batch of N-1 outages and for change lists that hit the
  same entries several times (a parallel pair, a re-closure), and agrees with the oracle's
  restatement of the sequential update."""

import ctypes as C
import dataclasses

import numpy as np
import pytest

from helpers import dense_of, load, net_from, with_parallel_branches
from oracle import restate

pytestmark = pytest.mark.gpu


def test_reference_mode_bit_exact_vs_reference_update():
    import torch

    from gap_b200 import _native as N

    d = load("kat_update")
    net = net_from(d)
    ch = net_from(d, "ch_")
    rp, ci, va = restate.ybus_reference(net)
    pos, prm = [], []
    for b in range(ch.n_branch):
        f, t = int(ch.from_id[b]), int(ch.to_id[b])

        def find(r, c):
            hit = np.nonzero(ci[rp[r]:rp[r + 1]] == c)[0]
            return int(rp[r] + hit[0]) if len(hit) else -1
        pos += [find(f, f), find(t, t), find(f, t), find(t, f)]
        prm.append([ch.r1[b], ch.x1[b], ch.g1[b], ch.b1[b], 1.0, 0.0, float(ch.status[b])])
    v = torch.as_tensor(va, device="cuda")
    p = torch.as_tensor(np.array(prm), device="cuda")
    hp = np.array(pos, np.int32)
    N.check(N.lib().gapk_ybus_apply_changes(len(prm), N.iptr(hp), C.c_void_p(p.data_ptr()),
                                            N.DELTA_REFERENCE, C.c_void_p(v.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.array_equal(v.cpu().numpy(), d["y_values"])


def _sparse(Y):
    import scipy.sparse as sp

    rp, ci, va = Y
    n = len(rp) - 1
    # copies: sum_duplicates sorts the index arrays in place, and csr_matrix shares them
    m = sp.csr_matrix((np.array(va), np.array(ci), np.array(rp)), shape=(n, n))
    m.sum_duplicates()
    return m


def test_n_minus_1_batch_fixed_taps_equals_fresh_build():
    import torch

    from gap_b200 import synth
    from gap_b200.engine import YbusDelta, YbusPlan, branch_params, shunt_params

    base = 1e8
    net = with_parallel_branches(synth.transmission_grid(1, n=2000), [2, 40], reverse=[40])
    zb = float(net.u_rated[0]) ** 2 / base
    yp = YbusPlan.from_network(net)
    outs = list(synth.n_minus_1(net, 256))
    m0 = net.n_branch - 2
    # multi-change scenarios: a parallel pair out, and out-then-back-in of the same branch
    lists = [[b] for b in outs] + [[2, m0], [40, m0 + 1, 40], [7, 7, 7]]
    status = [[0] for _ in outs] + [[0, 0], [0, 0, 1], [0, 1, 0]]
    S = len(lists)
    y0 = yp.assemble(torch.as_tensor(branch_params(net), device="cuda"),
                     torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)
    y = y0.repeat(S, 1).contiguous()
    delta = YbusDelta(yp, lists)
    prm = delta.params(branch_params(net), np.concatenate(status))
    delta.apply(y, prm, mode="fixed_taps", scale=zb)
    torch.cuda.synchronize()
    Y = y.cpu().numpy()
    rp, ci = yp.row_ptr, yp.col_idx
    pos = yp.branch_positions()
    ybase = restate.ybus_pi(net)[2] * zb
    worst_build = worst_seq = 0.0
    k = 0
    for s in range(S):
        n_c = len(lists[s])
        seq = restate.ybus_delta(ybase, pos[lists[s]], prm[k:k + n_c], "fixed_taps", scale=zb)
        k += n_c
        st = net.status.copy()
        for b, v in zip(lists[s], status[s]):
            st[b] = v
        fresh = restate.ybus_pi(dataclasses.replace(net, status=st))
        fresh = (fresh[0], fresh[1], fresh[2] * zb)
        ref = _sparse(fresh)
        scale = np.max(np.abs(ref.data))
        worst_build = max(worst_build, float(np.max(np.abs((_sparse((rp, ci, Y[s])) - ref).data),
                                                    initial=0.0)) / scale)
        worst_seq = max(worst_seq, float(np.max(np.abs(Y[s] - seq))) / scale)
    print(f"delta vs fresh build {worst_build:.2e}, vs sequential restatement {worst_seq:.2e}")
    assert worst_build <= 1e-14 and worst_seq <= 1e-14


def test_contingency_study_values_match_zero_admittance_assembly():
    """The N-1 study's device-built Y values (base minus the outaged branch's stamps) agree with
    assembling each outage as a zero-admittance branch."""
    import torch

    from gap_b200 import studies, synth
    from gap_b200.engine import YbusPlan, shunt_params

    base = 1e8
    net = synth.transmission_grid(3, n=1500)
    outs = synth.n_minus_1(net, 64)
    st = studies.contingency_study("n-1", net, outs, net.specified_power(base),
                                   synth.dc_start(net, base), base_power=base)
    zb = float(net.u_rated[0]) ** 2 / base
    yp = YbusPlan.from_network(net)
    ref = yp.assemble(torch.as_tensor(studies.contingency_branch_params(net, outs), device="cuda"),
                      torch.as_tensor(shunt_params(net), device="cuda"), mode=1, scale=zb)
    a, b = st.y.cpu().numpy(), ref.cpu().numpy()
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))
