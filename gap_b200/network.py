"""Host-side network description.

`Network` is a structure-of-arrays restatement of the reference's `gap::NetworkData`
(include/gap/core/types.h:204-352): buses (`BusData`, :204-219), branches (`BranchData`,
:224-274) and single-port appliances (`ApplianceData`, :284-310).  Units follow the reference:
voltages in V, impedances in Ohm, admittances in S, powers in W / var, angles in rad.

Bus, branch and appliance IDs are the user's IDs; buses are indexed by their position in the
arrays, and branches/appliances refer to buses by ID, as in the reference.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# gap::BusType (types.h:30-34)
PQ, PV, SLACK = 0, 1, 2
# gap::ApplianceType (types.h:40-44)
SOURCE, LOADGEN, SHUNT = 0, 1, 2
# gap::BranchType (types.h:50-54)
LINE, TRAFO, GENERIC = 0, 1, 2


def _f64(x, n, default=0.0):
    if x is None:
        return np.full(n, default, dtype=np.float64)
    a = np.ascontiguousarray(x, dtype=np.float64)
    if a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a


def _i32(x, n, default=0):
    if x is None:
        return np.full(n, default, dtype=np.int32)
    a = np.ascontiguousarray(x, dtype=np.int32)
    if a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a


@dataclass
class Network:
    bus_id: np.ndarray
    u_rated: np.ndarray
    bus_type: np.ndarray
    u_pu: np.ndarray
    p: np.ndarray  # BusData::active_power (W), generator direction
    q: np.ndarray  # BusData::reactive_power (var)
    br_id: np.ndarray
    from_id: np.ndarray
    to_id: np.ndarray
    status: np.ndarray
    r1: np.ndarray
    x1: np.ndarray
    g1: np.ndarray
    b1: np.ndarray
    k: np.ndarray
    theta: np.ndarray
    app_id: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    app_node: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    app_status: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    app_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    app_p: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    app_q: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    app_g1: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    app_b1: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))

    @staticmethod
    def build(bus_id, u_rated, bus_type, u_pu=None, p=None, q=None,
              from_id=(), to_id=(), r1=(), x1=(), g1=None, b1=None, k=None, theta=None,
              status=None, br_id=None,
              app_node=(), app_type=(), app_p=None, app_q=None, app_g1=None, app_b1=None,
              app_status=None, app_id=None) -> "Network":
        n = len(bus_id)
        m = len(from_id)
        a = len(app_node)
        return Network(
            bus_id=_i32(bus_id, n), u_rated=_f64(u_rated, n), bus_type=_i32(bus_type, n),
            u_pu=_f64(u_pu, n, 1.0), p=_f64(p, n), q=_f64(q, n),
            br_id=_i32(br_id if br_id is not None else np.arange(m), m),
            from_id=_i32(from_id, m), to_id=_i32(to_id, m), status=_i32(status, m, 1),
            r1=_f64(r1, m), x1=_f64(x1, m), g1=_f64(g1, m), b1=_f64(b1, m),
            k=_f64(k, m, 1.0), theta=_f64(theta, m, 0.0),
            app_id=_i32(app_id if app_id is not None else np.arange(a), a),
            app_node=_i32(app_node, a), app_status=_i32(app_status, a, 1),
            app_type=_i32(app_type, a), app_p=_f64(app_p, a), app_q=_f64(app_q, a),
            app_g1=_f64(app_g1, a), app_b1=_f64(app_b1, a))

    @property
    def n_bus(self) -> int:
        return int(self.bus_id.shape[0])

    @property
    def n_branch(self) -> int:
        return int(self.from_id.shape[0])

    @property
    def n_app(self) -> int:
        return int(self.app_node.shape[0])

    def id_to_index(self) -> np.ndarray:
        """Bus ID -> position lookup, as the reference builds it
        (src/admittance/cpu/cpu_admittance_matrix.cpp:56-73): sized max_id+1, -1 for unknown
        IDs, later duplicates overwrite earlier ones, negative IDs are never mapped."""
        max_id = int(self.bus_id.max()) if self.n_bus else -1
        lut = np.full(max_id + 1, -1, dtype=np.int64)
        for idx, bid in enumerate(self.bus_id.tolist()):
            if 0 <= bid <= max_id:
                lut[bid] = idx
        return lut

    def branch_index(self):
        """(from_idx, to_idx, valid) for every branch; valid is False for out-of-service
        branches and for branches naming unknown bus IDs, which the reference skips
        (cpu_admittance_matrix.cpp:100-118)."""
        lut = self.id_to_index()
        max_id = lut.shape[0] - 1

        def look(ids):
            ids = ids.astype(np.int64)
            ok = (ids >= 0) & (ids <= max_id)
            out = np.full(ids.shape, -1, dtype=np.int64)
            out[ok] = lut[ids[ok]]
            return out

        f = look(self.from_id)
        t = look(self.to_id)
        n = self.n_bus
        valid = (self.status != 0) & (f >= 0) & (f < n) & (t >= 0) & (t < n)
        return f, t, valid

    def shunt_index(self):
        """(bus_idx, g1, b1) of every SHUNT appliance the reference stamps into the Y-bus
        diagonal (cpu_admittance_matrix.cpp:88-97: all SHUNTs, whatever their status)."""
        lut = self.id_to_index()
        max_id = lut.shape[0] - 1
        sel = []
        for a in range(self.n_app):
            if self.app_type[a] != SHUNT:
                continue
            node = int(self.app_node[a])
            if 0 <= node <= max_id:
                bi = int(lut[node])
                if 0 <= bi < self.n_bus:
                    sel.append((a, bi))
        idx = np.array([s[1] for s in sel], dtype=np.int64)
        aa = np.array([s[0] for s in sel], dtype=np.int64)
        return idx, self.app_g1[aa] if len(aa) else np.zeros(0), \
            self.app_b1[aa] if len(aa) else np.zeros(0)

    def specified_power(self, base_power: float) -> np.ndarray:
        """S_spec per bus in per unit, as CPUNewtonRaphson::get_specified_power_at_bus
        (src/solver/powerflow/cpu/cpu_newton_raphson.cpp:346-377): the bus's own P/Q when
        either is non-zero, plus every in-service SOURCE/LOADGEN appliance whose node equals the
        bus ID, divided by base_power when base_power > 0."""
        s = (self.p + 1j * self.q).astype(np.complex128)
        if self.n_app:
            first = {}
            for i, bid in enumerate(self.bus_id.tolist()):
                first.setdefault(bid, []).append(i)
            for a in range(self.n_app):
                if self.app_status[a] == 1 and self.app_type[a] in (SOURCE, LOADGEN):
                    for i in first.get(int(self.app_node[a]), []):
                        s[i] += complex(self.app_p[a], self.app_q[a])
        if base_power > 0.0:
            # component-wise, as std::complex<double> /= double does
            s = (s.real / base_power) + 1j * (s.imag / base_power)
        return s
