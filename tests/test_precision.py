"""Precision form report on small cases: the FP32 form (FP32 state and
arithmetic, FP64 device geometry rounded once, per-field offsets) against
the FP64 form after the same steps.  Tolerance: 1e-5 relative L2 per field,
also for the viscous form of the orders that run the fused viscous passes
(with state offsets); 1e-4 for the viscous orders that run the unfused
passes (no offsets there).  Conservation sums (compensated FP64): relative
mass drift below 1e-6 in FP32 and 1e-12 in FP64 on the periodic meshes."""
from canary_b200.dg import viscous_fused
import pytest

from conftest import cuda_available
from canary_b200 import precision as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


# 3-D meshes fine enough for the Fourier state to stay smooth to t = 0.08
# (coarser ones, e.g. N=3 on 4^3 hexes, blow up before that on the oracle too)
@pytest.mark.parametrize("dim,N,n,visc", [(3, 4, 4, 0.0), (3, 5, 3, 0.0), (3, 3, 6, 0.0), (3, 4, 4, 1e-3),
                                          (2, 4, 10, 0.0), (2, 7, 10, 0.0)])
def test_precision_form_small(dim, N, n, visc):
    c = P.run_case(dim, N, n, 40, visc=visc)
    assert c["fp64"]["finite"] and c["fp32"]["finite"]
    assert c["max_rel_l2"] < (1e-4 if visc and not viscous_fused(dim, N) else 1e-5), c
    assert c["fp64"]["mass_drift_rel"] < 1e-12 and c["fp32"]["mass_drift_rel"] < 1e-6, c
