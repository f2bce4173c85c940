"""Shared test helpers: golden fixtures -> Network objects."""

import glob
import os

import numpy as np

from gap_b200.network import Network

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def net_from(d, prefix="net_"):
    kw = {k[len(prefix):]: d[k] for k in d if k.startswith(prefix)}
    return Network(**kw)


def pgm_network(d):
    from gap_b200.api import network_from_simple_lists

    return network_from_simple_lists(d["bus_data"].tolist(), d["branch_data"].tolist())


def network_of(name):
    d = load(name)
    if name.startswith("pgm_"):
        return pgm_network(d), d
    return net_from(d), d


def parity_fixtures():
    return fixture_names("kat_") + fixture_names("c0_") + fixture_names("pgm_")


def pgm_output(d):
    """power-grid-model's output dataset stored with a PGM fixture (zlib-compressed JSON)."""
    import json
    import zlib

    return json.loads(zlib.decompress(d["pgm_output_json_z"].tobytes()).decode())


def compare_pgm_output(ours, ref, rtol):
    """Largest relative difference per (component, attribute) between two PGM output datasets
    (matched by id; relative to the attribute's largest magnitude in `ref`); asserts every
    component and record of `ref` is present and each difference is below rtol."""
    worst = {}
    for comp, recs in ref.items():
        if comp == "meta" or not isinstance(recs, list):
            continue
        mine = {r["id"]: r for r in ours.get(comp, [])}
        assert set(mine) == {r["id"] for r in recs}, comp
        for key in recs[0]:
            if key in ("id",):
                continue
            if key == "energized":
                assert all(bool(mine[r["id"]][key]) == bool(r[key]) for r in recs), comp
                continue
            a = np.array([float(mine[r["id"]][key]) for r in recs])
            b = np.array([float(r[key]) for r in recs])
            scale = max(float(np.max(np.abs(b))), 1e-30)
            worst[(comp, key)] = float(np.max(np.abs(a - b))) / scale
    bad = {k: w for k, w in worst.items() if not w < rtol}
    assert not bad, bad
    return worst
