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
