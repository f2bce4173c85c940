"""gap_b200 -- B200-native Newton-Raphson power flow.

A drop-in GPU backend for the reference's Newton-Raphson path (Y-bus assembly, fused
mismatch, Jacobian fill, sparse block LU, voltage update), computed by hand-written sm_100a
kernels in libgapk.so.  See `gap_b200.api` for the reference-facing functions and
`gap_b200.engine` for batched / mixed-precision solves, `gap_b200.autograd` for
differentiable ones and `gap_b200.studies` for mixed batches of grids and contingencies.
"""

from .network import GENERIC, LINE, LOADGEN, PQ, PV, SHUNT, SLACK, SOURCE, TRAFO, Network

__version__ = "0.1.0"


def __getattr__(name):
    # lazy: keep `import gap_b200` cheap and torch-free until a solver is used
    if name in ("PowerFlowConfig", "PowerFlowResult", "AdmittanceMatrix", "NewtonRaphson",
                "solve_simple_power_flow", "is_cuda_available", "network_from_simple_lists"):
        from . import api

        return getattr(api, name)
    raise AttributeError(name)
