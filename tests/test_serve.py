"""Serving loop (continuous batching): each result is the same alone and in
the mix, the served FP64 results equal the one-at-a-time FP64 path, the FP32
served form stays within the precision-form tolerance of FP64, and admission
respects the HBM budget.

Tolerances: alone-vs-in-the-mix bit-identical; served FP64 vs one-at-a-time
FP64 1e-12 relative L2 per field (the oracle parity bar; FP64 batches use the
per-node geometry, like the one-at-a-time path); served FP32 vs FP64 1e-5 per
field for the inviscid requests and 1e-4 for the viscous ones (no state
offsets there; the FP32 batch runs the vortex requests' affine meshes with
the affine-element stage).  Rejected, cancelled and failed requests leave the
other requests' results unchanged.
"""
import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import relerr_fields
from canary_b200 import serve as S


def small_requests():
    R = S.Request
    return [R(0, "vortex", 3, 6, 0.05, 0.0, 4.0, 4.5, 5.5), R(1, "vortex", 6, 4, 0.08, 0.0, 2.0, 6.0, 3.0),
            R(2, "euler3d", 3, 4, 0.05, 0.0, seed=2), R(3, "vortex", 8, 3, 0.03, 0.0, 5.0, 5.0, 5.0),
            R(4, "ns3d", 3, 4, 0.04, 0.0, seed=4), R(5, "euler3d", 4, 4, 0.06, 0.0, seed=5),
            R(6, "vortex", 4, 8, 0.05, 0.0, 1.5, 3.0, 7.0), R(7, "euler3d", 5, 4, 0.03, 0.0, seed=7)]


def _serve(reqs, precision=32, budget=120e9, tick=3, realtime=False):
    srv = S.Server(precision, hbm_budget=budget, max_instances=64, tick_steps=tick)
    rep = srv.serve(reqs, realtime=realtime)
    srv.close()
    return rep


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("precision", [32, 64])
def test_result_same_alone_and_in_mix(precision):
    reqs = small_requests()
    mixed = _serve(reqs, precision)
    assert not mixed.failed
    for r in reqs:
        alone = _serve([r], precision)
        assert np.array_equal(alone.results[r.rid], mixed.results[r.rid]), (r.kind, r.rid)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_served_fp64_equals_one_at_a_time_and_fp32_within_tolerance():
    reqs = small_requests()
    served64 = _serve(reqs, 64)
    served32 = _serve(reqs, 32)
    seq = S.serve_one_at_a_time(reqs, 64)
    for r in reqs:
        assert max(relerr_fields(served64.results[r.rid], seq.results[r.rid])) < 1e-12, r.rid
        e32 = max(relerr_fields(served32.results[r.rid], seq.results[r.rid]))
        assert e32 < (1e-4 if r.kind == "ns3d" else 1e-5), (r.kind, e32)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_admission_respects_hbm_budget():
    reqs = small_requests()
    srv = S.Server(32, hbm_budget=1e9, max_instances=64, tick_steps=2)
    # a budget that holds every mesh but only the largest request's state at
    # a time, so the others queue for memory
    need = sorted(srv.request_bytes(r) for r in reqs)
    meshes = sum(S.MeshPool.nbytes(r.dim, r.N, r.n_side, 32) for r in reqs)
    srv.budget = meshes + need[-1]
    rep = srv.serve(reqs, realtime=False)
    srv.close()
    assert len(rep.latencies) == len(reqs)
    assert rep.peak_bytes <= srv.budget
    assert rep.max_live < len(reqs)  # some requests waited for memory
    full = _serve(reqs, 32)
    for r in reqs:  # queueing changes nothing in the results
        assert np.array_equal(rep.results[r.rid], full.results[r.rid])


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_realtime_stream_latencies():
    reqs = S.request_stream(12, rate=40.0, seed=3)
    for r in reqs:  # keep the test short: small meshes, short final times
        r.n_side = min(r.n_side, 8 if r.dim == 2 else 4)
        r.t_final = 0.02
    rep = _serve(reqs, 32, realtime=True)
    s = rep.summary()
    assert s["requests"] == 12 and s["p99_s"] >= s["p50_s"] > 0
    assert all(rep.latencies[r.rid] > 0 for r in reqs)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_unfittable_request_is_rejected_and_the_rest_complete():
    reqs = small_requests()[:4]
    big = S.Request(99, "vortex", 8, 64, 0.01, 0.0, 3.0, 5.0, 5.0)
    srv = S.Server(32, hbm_budget=1e9, max_instances=64, tick_steps=3)
    srv.budget = sum(S.MeshPool.nbytes(r.dim, r.N, r.n_side, 32) + srv.request_bytes(r) for r in reqs)
    assert srv.never_fits(big) and not any(srv.never_fits(r) for r in reqs)
    rep = srv.serve(reqs + [big], realtime=False)
    srv.close()
    assert set(rep.rejected) == {99} and 99 not in rep.results
    full = _serve(reqs, 32)
    for r in reqs:
        assert np.array_equal(rep.results[r.rid], full.results[r.rid])
    s = rep.summary()
    assert s["rejected"] == 1 and s["completed"] == len(reqs)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_cancelled_requests_leave_the_others_unchanged():
    reqs = small_requests()[:4]
    # a long solve that is still running when its client withdraws it, and
    # one withdrawn before it is admitted
    long = S.Request(50, "vortex", 8, 48, 4.0, 0.0, 3.0, 5.0, 5.0)
    early = S.Request(51, "vortex", 4, 8, 0.05, 0.0, 2.0, 4.0, 4.0)
    srv = S.Server(32, hbm_budget=120e9, max_instances=64, tick_steps=3)
    rep = srv.serve(reqs + [long, early], realtime=False, cancel={50: 0.5, 51: 0.0})
    srv.close()
    assert rep.cancelled == {50, 51}
    assert 50 not in rep.results and 51 not in rep.results
    full = _serve(reqs, 32)
    for r in reqs:
        assert np.array_equal(rep.results[r.rid], full.results[r.rid])
    s = rep.summary()
    assert s["cancelled"] == 2 and s["completed"] == len(reqs)


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_simulated_allocation_failure_waits_or_is_rejected():
    reqs = small_requests()[:4]
    full = _serve(reqs, 32)
    # second request: its set-up fails while the first is resident, so it
    # waits for memory and is admitted later, with an unchanged result
    srv = S.Server(32, hbm_budget=120e9, max_instances=64, tick_steps=3)
    srv.fail_alloc = {reqs[1].rid}
    rep = srv.serve(reqs, realtime=False)
    srv.close()
    assert not rep.rejected and not srv.fail_alloc
    for r in reqs:
        assert np.array_equal(rep.results[r.rid], full.results[r.rid])
    # first request: nothing else holds memory, so it is rejected
    srv = S.Server(32, hbm_budget=120e9, max_instances=64, tick_steps=3)
    srv.fail_alloc = {reqs[0].rid}
    rep = srv.serve(reqs, realtime=False)
    srv.close()
    assert set(rep.rejected) == {reqs[0].rid}
    for r in reqs[1:]:
        assert np.array_equal(rep.results[r.rid], full.results[r.rid])


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_normalised_3d_requests_complete():
    reqs = [S.Request(0, "euler3d", 3, 4, 0.6, 0.0, seed=3, vel_peak=0.1),
            S.Request(1, "ns3d", 4, 4, 0.5, 0.0, seed=4, vel_peak=0.1),
            S.Request(2, "euler3d", 5, 4, 0.5, 0.0, seed=5, vel_peak=0.1)]
    rep = _serve(reqs, 32)
    assert not rep.failed
    s = rep.summary()
    assert s["completed"] == 3 and s["per_kind"]["euler3d"]["completed"] == 2
