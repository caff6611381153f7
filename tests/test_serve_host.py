"""Host side of the serving loop (no GPU): the request stream and the time
step plan."""
import math

import numpy as np

from canary_b200 import serve as S


def test_request_stream_is_seeded_and_follows_the_mix():
    a = S.request_stream(2000, rate=50.0, seed=7)
    b = S.request_stream(2000, rate=50.0, seed=7)
    assert [(r.kind, r.N, r.n_side, r.t_final, r.arrival) for r in a] == \
           [(r.kind, r.N, r.n_side, r.t_final, r.arrival) for r in b]
    kinds = np.array([r.kind for r in a])
    assert abs(np.mean(kinds == "vortex") - 0.70) < 0.04
    assert abs(np.mean(kinds != "vortex") - 0.30) < 0.04
    for r in a:
        if r.kind == "vortex":
            assert 3 <= r.N <= 8 and 8 <= r.n_side <= 64 and 1 <= r.beta <= 5
            assert 2 <= r.xc <= 8 and 2 <= r.yc <= 8
        else:
            assert 3 <= r.N <= 7 and 4 <= r.n_side <= 16
        assert 0.5 <= r.t_final <= 2.0
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) >= 0)
    gaps = np.diff(arr)
    assert abs(gaps.mean() - 1 / 50.0) < 0.1 / 50.0  # Poisson rate 50/s
    assert all(r.arrival == 0.0 for r in S.request_stream(10, rate=0.0))


def test_plan_reaches_the_final_time():
    r = S.Request(0, "vortex", 8, 64, 1.3, 0.0)
    n, dt = S.plan(r, 2.9)
    assert abs(n * dt - 1.3) < 1e-12
    assert dt <= 0.2 * (10.0 / 64) / (64 * 2.9) + 1e-15
    r3 = S.Request(1, "euler3d", 7, 16, 0.5, 0.0)
    n3, dt3 = S.plan(r3, 1.3)
    assert n3 == math.ceil(0.5 / (0.2 * (2 * math.pi / 16) / (49 * 1.3)))


def test_mesh_pool_evicts_idle_meshes_least_recently_used_first():
    class _BM:
        closed = 0

        def close(self):
            _BM.closed += 1

    pool = S.MeshPool(device=None, stream=None)
    for k, (nbytes, users, last) in {"a": (40, 0, 3.0), "b": (30, 1, 1.0), "c": (20, 0, 2.0)}.items():
        pool.meshes[k] = S._Mesh(None, nbytes, {32: _BM()}, users, last)
    assert pool.resident_bytes() == 90
    assert pool.evict(need=5, budget=100, in_use=0)          # fits: nothing evicted
    assert set(pool.meshes) == {"a", "b", "c"}
    assert pool.evict(need=25, budget=100, in_use=0)         # drops "c" (idle, oldest idle)
    assert set(pool.meshes) == {"a", "b"} and _BM.closed == 1
    assert not pool.evict(need=80, budget=100, in_use=0)     # "b" is in use: cannot make room
    assert set(pool.meshes) == {"b"} and _BM.closed == 2
    assert S.MeshPool.nbytes(3, 3, 4, 32) > S.MeshPool.nbytes(3, 3, 4, 64) > 0


def test_report_counts_completed_requests_only():
    lat = {0: 1.0, 1: 2.0, 2: 30.0, 3: 4.0}
    kinds = {0: "vortex", 1: "vortex", 2: "euler3d", 3: "ns3d", 4: "euler3d", 5: "vortex"}
    rep = S.Report(lat, {}, 0.0, 10.0, 1e12, 0, 3, failed={2}, kinds=kinds, rejected={4: "too big"},
                   cancelled={5}, work={0: 1e10, 1: 2e10, 3: 3e10})
    s = rep.summary()
    assert s["requests"] == 6 and s["completed"] == 3
    assert s["failed"] == 1 and s["rejected"] == 1 and s["cancelled"] == 1
    assert s["solves_per_s"] == 3 / 10.0
    assert s["p50_s"] == 2.0 and s["p99_s"] < 4.0 + 1e-9  # the failed request's 30 s is not counted
    assert s["dof_stage_per_s"] == 1e11 and s["completed_dof_stage_per_s"] == 6e9
    pk = s["per_kind"]
    assert pk["vortex"]["completed"] == 2 and pk["vortex"]["cancelled"] == 1
    assert pk["euler3d"]["completed"] == 0 and pk["euler3d"]["failed"] == 1 and pk["euler3d"]["rejected"] == 1
    assert pk["euler3d"]["p50_s"] is None and pk["ns3d"]["p50_s"] == 4.0


def test_request_that_can_never_fit_is_recognised():
    import types
    srv = types.SimpleNamespace(precision=32, budget=2 * 10 ** 8)
    srv.request_bytes = lambda r: S.Server.request_bytes(srv, r)
    small = S.Request(0, "vortex", 3, 8, 0.5, 0.0)
    big = S.Request(1, "euler3d", 7, 16, 0.5, 0.0)
    assert not S.Server.never_fits(srv, small)
    assert S.Server.never_fits(srv, big)  # 16^3 N=7: state and mesh exceed 200 MB


def test_normalised_stream_scales_only_the_3d_requests():
    a = S.request_stream(50, rate=10.0, seed=1)
    b = S.request_stream(50, rate=10.0, seed=1, vel_peak=0.1)
    for r, q in zip(a, b):
        assert (r.kind, r.N, r.n_side, r.t_final, r.arrival) == (q.kind, q.N, q.n_side, q.t_final, q.arrival)
        assert r.vel_peak is None and q.vel_peak == (None if q.dim == 2 else 0.1)
