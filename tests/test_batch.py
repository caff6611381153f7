"""Batched LSRK(5,4) over many independent instances (cb_batch_*), against the
FP64 oracle run instance by instance, and the batching properties: a result
does not depend on what else is in the batch, on when the instance was
admitted, or on the group shape chosen by the tuner.

Tolerances: FP64 batch vs oracle 1e-12 relative L2 per field; FP32 batch vs
the FP64 oracle 1e-5; alone-vs-in-the-mix and variant 0-vs-1 bit-identical.
"""
import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import fourier_case, oracle_run, relerr_fields, vortex_case
from canary_b200 import batch as B
from canary_b200 import CanaryError, dg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _cases():
    """(mesh, Q, dt, nsteps) of a mixed set: 2-D vortices of several orders,
    sizes and parameters, and warped 3-D Fourier cubes."""
    out = []
    for N, n, beta, xc, yc, steps in [(3, 4, 5.0, 5.0, 5.0, 9), (5, 3, 2.0, 4.0, 6.0, 6),
                                      (8, 2, 3.5, 6.0, 3.0, 4), (4, 5, 1.5, 3.0, 7.0, 8),
                                      (1, 6, 5.0, 5.0, 5.0, 5), (6, 3, 4.0, 5.5, 4.5, 7)]:
        m, Q = vortex_case(N, n, beta, xc, yc)
        out.append((m, Q, 0.002, steps))
    # low orders take a fraction of the CFL step: the k <= 4 Fourier state is
    # under-resolved there (the oracle itself blows up at the full step)
    for N, n, steps, scale in [(3, 4, 5, 1.0), (7, 2, 3, 1.0), (2, 6, 6, 0.25), (1, 8, 5, 0.1)]:
        m, Q, dt = fourier_case(N, n)
        out.append((m, Q, dt * scale, steps))
    return out


@pytest.fixture(scope="module")
def cases():
    return _cases()


@pytest.fixture(scope="module")
def oracle_results(cases):
    return [oracle_run(m, Q, dt, k) for (m, Q, dt, k) in cases]


def _run_batch(cases, precision, idx=None, chunks=(2, 3, 100), variants=None, affine=None, used=False,
               concurrent=None):
    """Admit cases[idx] into one batch, run in the given chunks, return the
    final FP64 host states (and, with `used`, the variant each slot ran)."""
    idx = range(len(cases)) if idx is None else idx
    b = B.Batch(precision, max_instances=64)
    if affine is not None:
        b.set_affine(affine)
    if concurrent is not None:
        b.set_concurrent(concurrent)
    for (dim, N, v) in (variants or []):
        b.set_variant(dim, N, v)
    meshes, slots = [], []
    for i in idx:
        m, Q, dt, k = cases[i]
        bm = B.BatchMesh(dg.DeviceMesh.upload(m), precision)
        meshes.append(bm)
        slots.append(b.add_state(bm, Q, dt, k))
    ran = [b.slot_variant(s) for s in slots]
    for c in chunks:
        b.run(c)
    assert not b.status().any()
    out = [b.result(s) for s in slots]
    b.close()
    return (out, ran) if used else out


def test_batch_fp64_matches_oracle(cases, oracle_results):
    out = _run_batch(cases, 64)
    for (m, Q, dt, k), ref, got in zip(cases, oracle_results, out):
        err = max(relerr_fields(got, ref))
        assert err < 1e-12, (m.dim, m.N, m.nelem, err)


def test_batch_fp32_matches_oracle(cases, oracle_results):
    out = _run_batch(cases, 32)
    for (m, Q, dt, k), ref, got in zip(cases, oracle_results, out):
        err = max(relerr_fields(got, ref))
        assert err < 1e-5, (m.dim, m.N, m.nelem, err)


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_result_same_alone_and_in_mix(cases, precision):
    alone = [_run_batch(cases, precision, idx=[i], chunks=(100,))[0] for i in (0, 3, 7)]
    mixed = _run_batch(cases, precision, chunks=(1, 1, 5, 100))
    for a, i in zip(alone, (0, 3, 7)):
        assert np.array_equal(a, mixed[i])


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_variants_agree(cases, precision):
    """Grouped variants (1, 2) are bit-identical to each other, and so are the
    per-node pipelined ones (0, 3, 4, 6, 7, 8, 11: the same code at other
    occupancies, staging depth, group size or nodes per thread, or with only
    the state staged) and the
    affine ones (5, 9) on affine meshes; the families sum the contraction
    (padded rows) or form the geometry differently and agree to round-off:
    1e-13 (FP64) / 1e-5 (FP32) relative between the per-node families,
    1e-11 / 1e-5 for the affine stage.  A chosen variant runs as chosen: a
    per-node one is not replaced by the affine stage, an affine one falls back
    to the default per-node variant on a warped mesh."""
    orders = [(m.dim, m.N) for (m, Q, dt, k) in cases]
    probe = B.Batch(precision, 1)
    built = {}
    for d, N in orders:
        for v in B.VARIANTS:
            try:
                probe.set_variant(d, N, v)
                built[(d, N, v)] = True
            except CanaryError:
                built[(d, N, v)] = False
    probe.close()
    runs, used = {}, {}
    for v in B.VARIANTS:
        runs[v], used[v] = _run_batch(cases, precision, variants=[(d, N, v) for d, N in orders if built[(d, N, v)]],
                                      affine=True, used=True)
    tol = 1e-13 if precision == 64 else 1e-5
    tol_aff = 1e-11 if precision == 64 else 1e-5
    for i, (m, Q, dt, k) in enumerate(cases):
        affine = m.dim == 2  # uniform vortex meshes; the 3-D Fourier cubes are warped
        for v in B.VARIANTS:
            if built[(m.dim, m.N, v)] and v not in B.AFFINE:
                assert used[v][i] == v
            elif built[(m.dim, m.N, v)]:
                assert (used[v][i] == v) == affine
        if built[(m.dim, m.N, 2)]:
            assert np.array_equal(runs[1][i], runs[2][i])
        if built[(m.dim, m.N, 0)]:
            for v in B.PIPELINED:
                if built[(m.dim, m.N, v)]:
                    assert np.array_equal(runs[0][i], runs[v][i])
        if affine and built[(m.dim, m.N, 5)]:
            for v in B.AFFINE:
                if built[(m.dim, m.N, v)]:
                    assert np.array_equal(runs[5][i], runs[v][i])
        assert max(relerr_fields(runs[0][i], runs[1][i])) < tol
        if built[(m.dim, m.N, 5)]:
            assert max(relerr_fields(runs[5][i], runs[1][i])) < tol_aff


@pytest.mark.parametrize("precision", [64, 32])
def test_shape_order_in_the_step_graph_does_not_change_results(cases, precision):
    """Shapes as concurrent graph branches (default) or one after another:
    every instance's arithmetic is the same, so the states are bit-identical."""
    serial = _run_batch(cases, precision, concurrent=False)
    conc = _run_batch(cases, precision)
    for a, c in zip(serial, conc):
        assert np.array_equal(a, c)


def test_unbuilt_variant_is_rejected():
    b = B.Batch(64, 4)
    with pytest.raises(CanaryError):
        b.set_variant(3, 7, 2)  # 3-D N=7 groups of 1024 nodes are not built
    with pytest.raises(CanaryError):
        b.set_variant(3, 7, 3)  # 512-thread blocks are not built for three per SM
    b.close()


def test_continuous_batching_admit_and_release(cases):
    """Instances admitted while others run, released as they finish, slots
    reused and work lists compacted: each result equals the instance alone."""
    alone = [_run_batch(cases, 64, idx=[i], chunks=(100,))[0] for i in range(len(cases))]
    b = B.Batch(64, max_instances=3)
    meshes = {}
    pending = list(range(len(cases)))
    live = {}
    got = {}
    rounds = 0
    while pending or live:
        # admit while slots are free
        while pending and len(live) < 3:
            i = pending.pop(0)
            m, Q, dt, k = cases[i]
            bm = meshes.setdefault(i, B.BatchMesh(dg.DeviceMesh.upload(m), 64))
            live[b.add_state(bm, Q, dt, k)] = i
        b.run(2)
        rounds += 1
        for s in list(live):
            done, target = b.info(s)
            if done == target:
                got[live.pop(s)] = b.result(s)
    b.close()
    assert rounds > 3
    for i in range(len(cases)):
        assert np.array_equal(got[i], alone[i]), i


def test_many_small_instances_force_list_growth_and_compaction():
    """Hundreds of admissions and releases of small instances exercise work
    list growth, in-place compaction and generation tags."""
    m, Q = vortex_case(1, 40)  # N=1: 64 elements per group, 25 groups
    ref = _run_batch([(m, Q, 0.002, 3)], 64, chunks=(100,))[0]
    bm = B.BatchMesh(dg.DeviceMesh.upload(m), 64)
    b = B.Batch(64, max_instances=48)
    slots = [b.add_state(bm, Q, 0.002, 3) for _ in range(48)]
    for cycle in range(4):
        b.run(1)
        # release every other slot, re-admit into the freed slots
        for s in slots[cycle % 2::2]:
            b.release(s)
        for j in range(cycle % 2, 48, 2):
            slots[j] = b.add_state(bm, Q, 0.002, 3)
    b.run(10)
    for s in slots:
        assert np.array_equal(b.result(s), ref)
    b.close()


def test_nonfinite_state_flags_only_its_slot(cases):
    m, Q, dt, k = cases[0]
    bad = Q.copy(order="F")
    bad[:, 2, 0] = -1.0  # negative density: the pressure's sqrt gives NaN
    b = B.Batch(64, 8)
    bm = B.BatchMesh(dg.DeviceMesh.upload(m), 64)
    s_good = b.add_state(bm, Q, dt, k)
    s_bad = b.add_state(bm, bad, dt, k)
    b.run(k)
    st = b.status()
    assert st[s_bad] != 0 and st[s_good] == 0
    good = b.result(s_good)
    alone = _run_batch(cases, 64, idx=[0], chunks=(100,))[0]
    assert np.array_equal(good, alone)
    b.close()


def test_batch_matches_single_solver(cases):
    """Same instance through cb_lsrk_run (pipelined single-mesh kernel) and the
    batch (grouped kernel): same arithmetic up to round-off."""
    m, Q, dt, k = cases[7]  # 3-D N=7
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64)
    s.run(k, dt)
    single = s.state()
    s.close()
    got = _run_batch(cases, 64, idx=[7], chunks=(100,))[0]
    assert max(relerr_fields(got, single)) < 1e-13


def test_autotuner_picks_a_built_variant():
    tuned = B.autotune(32, [(2, 3), (3, 4)], nodes_target=20000, steps=1, repeat=1)
    b = B.Batch(32, 1)
    for (dim, N), v in tuned.items():
        b.set_variant(dim, N, v)  # raises if the chosen variant is not built
        assert b.variant(dim, N) == v
    b.close()
    assert (3, 4) in tuned and tuned[(3, 4)] in B.VARIANTS


def test_autotuner_on_the_workload_size_mix_reports_the_configuration():
    """Tuning on the workload's own instances of each shape (several mesh
    sizes) reports the chosen variant's elements per CTA, threads, nodes per
    thread, staging depth and CTAs per SM."""
    inst = [(2, 4, 6), (2, 4, 10), (2, 6, 4), (2, 4, 8), (2, 6, 12)]
    rep = {}
    tuned = B.autotune(32, [(2, 4), (2, 6)], nodes_target=50000, steps=1, repeat=1, instances=inst, report=rep)
    assert set(tuned) == {(2, 4), (2, 6)}
    assert rep[(2, 4)]["instances"] == 3 and rep[(2, 6)]["instances"] == 2
    for key, r in rep.items():
        c = r["config"]
        assert r["variant"] == tuned[key] and r["variant"] in r["ms_per_step"]
        assert c["threads_per_cta"] >= 32 and c["elements_per_cta"] >= 1 and c["ctas_per_sm"] >= 1
        assert c["nodes_per_thread"] >= 1 and c["staging_depth"] in (0, 1, 2)
    b = B.Batch(32, 1)
    # copies two groups ahead are built where they fit four FP32 blocks per SM (2-D N >= 6)
    assert b.variant_info(2, 6, B.VAR_DEEP)["staging_depth"] == 2
    with pytest.raises(CanaryError):
        b.variant_info(2, 4, B.VAR_DEEP)
    assert b.variant_info(2, 4, 0)["staging_depth"] == 1 and b.variant_info(2, 4, 1)["staging_depth"] == 0
    b.close()


def test_invalid_mesh_is_reported_at_first_use(cases):
    """cb_mesh_create does not wait for its set-up; the vmap / boundary-code
    validation is reported by the first use of the mesh."""
    m, Q, dt, k = cases[0]
    dm = dg.DeviceMesh.upload(m)
    dm.elemtobndy[0] = 7  # no such boundary condition
    bm = B.BatchMesh(dm, 64)
    with pytest.raises(CanaryError) as ei:
        bm.affine
    assert "boundary" in str(ei.value)
    b = B.Batch(64, 2)
    with pytest.raises(CanaryError):
        b.add_state(bm, Q, dt, k)
    b.close()
    bm.close()
