"""canary_b200: B200 (sm_100a) nodal-DG hot path of CliMA/Canary.jl.

Host side of the drop-in: the reference's mesh/metric/operator setup mirrored
in numpy (operators, mesh, metric), the workload initial conditions (ic), and
the device API (dg) that runs the hand-written CUDA kernels of
libcanary_b200.so through its C-ABI, and the batched many-instance driver
(batch).  torch is imported only when a device
call is made.
"""
from . import batch, dg, ic, mesh, metric, operators  # noqa: F401
from ._lib import CanaryError  # noqa: F401

__all__ = ["ic", "mesh", "metric", "operators", "dg", "batch", "CanaryError"]
