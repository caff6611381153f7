"""Known-answer tests of the reference (test/test_operators.jl,
test/test_mesh.jl, test/test_metric.jl), run against both the CPU oracle and
the product's host-side mirror of the setup API.  These pin the setup layer
(quadrature, operators, brick mesh, Hilbert partition, connectivity, vmaps,
metric terms) to what the reference's own tests pin."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O
from canary_b200 import mesh as HM
from canary_b200 import metric as HMT
from canary_b200 import operators as HOP


class OracleImpl:
    name = "oracle"
    legendre = staticmethod(O.legendre)
    legendre_coefs = staticmethod(O.legendre_coefs)
    custom_gauss_rule = staticmethod(lambda lo, hi, a, b, e, m: O.custom_gauss_rule(lo, hi, a, b, e, m))
    lglpoints = staticmethod(O.lglpoints)
    lgpoints = staticmethod(O.lgpoints)
    spectralderivative = staticmethod(O.spectralderivative)
    interpolationmatrix = staticmethod(O.interpolationmatrix)
    hilbertcode = staticmethod(O.hilbertcode)
    centroidtocode = staticmethod(O.centroidtocode)
    brickmesh = staticmethod(O.brickmesh)
    partition = staticmethod(O.partition)
    connectmesh = staticmethod(O.connectmesh)
    mappings = staticmethod(O.mappings)
    creategrid = staticmethod(O.creategrid)

    @staticmethod
    def computemetric(D, *X):
        return O.computemetric(D, *X)


class HostImpl:
    name = "host"
    legendre = staticmethod(HOP.legendre)
    legendre_coefs = staticmethod(HOP.legendre_coefs)
    custom_gauss_rule = staticmethod(lambda lo, hi, a, b, e, m: HOP.custom_gauss_rule(lo, hi, a, b, e, m))
    lglpoints = staticmethod(HOP.lglpoints)
    lgpoints = staticmethod(HOP.lgpoints)
    spectralderivative = staticmethod(HOP.spectralderivative)
    interpolationmatrix = staticmethod(HOP.interpolationmatrix)
    hilbertcode = staticmethod(HM.hilbertcode)
    centroidtocode = staticmethod(HM.centroidtocode)
    brickmesh = staticmethod(HM.brickmesh)
    partition = staticmethod(HM.partition)
    connectmesh = staticmethod(HM.connectmesh)
    mappings = staticmethod(HM.mappings)
    creategrid = staticmethod(HMT.creategrid)

    @staticmethod
    def computemetric(D, *X):
        if len(X) == 2:
            return HMT.computemetric2d(*X, D)
        return HMT.computemetric3d(*X, D)


IMPLS = [OracleImpl, HostImpl]


@pytest.fixture(params=IMPLS, ids=lambda c: c.name)
def impl(request):
    return request.param


# ------------------------------------------------ test/test_operators.jl:1-57
def test_gauss_quadrature_known_answers(impl):
    x, w = impl.legendre(1)
    assert np.all(x == 0) and np.allclose(w, [2.0])
    x, w = impl.legendre(1, "L")
    assert np.allclose(x, [-1.0]) and np.allclose(w, [2.0])
    x, w = impl.legendre(1, "R")
    assert np.allclose(x, [1.0]) and np.allclose(w, [2.0])
    x, w = impl.legendre(2, "L")
    assert np.allclose(x, [-1.0, 1 / 3]) and np.allclose(w, [0.5, 1.5])
    x, w = impl.legendre(2, "R")
    assert np.allclose(x, [-1 / 3, 1.0]) and np.allclose(w, [1.5, 0.5])


def test_gauss_quadrature_errors(impl):
    with pytest.raises(Exception, match="Must have at least two points for both ends."):
        impl.legendre(1, "B")
    a, b = impl.legendre_coefs(100)
    with pytest.raises(Exception, match="No convergence after 1 iterations"):
        impl.custom_gauss_rule(-1.0, 1.0, a, b, "B", 1)


# ------------------------------------------------ test/test_operators.jl:59-90
def _P5(r):
    return (15 * r - 70 * r ** 3 + 63 * r ** 5) / 8


def _P6(r):
    return (-5 + 105 * r ** 2 - 315 * r ** 4 + 231 * r ** 6) / 16


def _DP6(r):
    return (210 * r - 1260 * r ** 3 + 1386 * r ** 5) / 16


def test_operators_exactness(impl):
    N = 6
    r, w = impl.lglpoints(N)
    D = impl.spectralderivative(r)
    x = np.linspace(-1, 1, 101)
    I = impl.interpolationmatrix(r, x)
    assert np.isclose(np.sum(_P5(r) ** 2 * w), 2 / 11)
    assert np.allclose(D @ _P6(r), _DP6(r))
    assert np.allclose(I @ _P6(r), _P6(x))
    r, w = impl.lgpoints(N)
    D = impl.spectralderivative(r)
    assert np.isclose(np.sum(_P5(r) ** 2 * w), 2 / 11)
    assert np.isclose(np.sum(_P6(r) ** 2 * w), 2 / 13)
    assert np.allclose(D @ _P6(r), _DP6(r))


# ------------------------------------------------ test/test_mesh.jl:1-60
def test_linear_partition():
    assert HM.linearpartition(1, 1, 1) == range(1, 2)
    assert HM.linearpartition(20, 1, 1) == range(1, 21)
    assert HM.linearpartition(10, 1, 2) == range(1, 6)
    assert HM.linearpartition(10, 2, 2) == range(6, 11)


HILBERT_2BIT = [([0, 0], [0, 0]), ([1, 0], [0, 1]), ([1, 1], [0, 2]), ([0, 1], [0, 3]),
                ([0, 2], [1, 0]), ([0, 3], [1, 1]), ([1, 3], [1, 2]), ([1, 2], [1, 3]),
                ([2, 2], [2, 0]), ([2, 3], [2, 1]), ([3, 3], [2, 2]), ([3, 2], [2, 3]),
                ([3, 1], [3, 0]), ([2, 1], [3, 1]), ([2, 0], [3, 2]), ([3, 0], [3, 3])]


def test_hilbert_code(impl):
    for y, h in (([0, 0], [0, 0]), ([0, 1], [0, 1]), ([1, 1], [1, 0]), ([1, 0], [1, 1])):
        assert list(impl.hilbertcode(y, bits=1)) == h
    for y, h in HILBERT_2BIT:
        assert list(impl.hilbertcode(y, bits=2)) == h
    assert [int(v) for v in impl.hilbertcode([14, 3, 4], bits=64)] == [0, 0, 0xE25]


def test_mesh_to_hilbert_code(impl):
    etc = np.zeros((2, 4, 6), order="F")
    etc[:, :, 0] = [[2, 3, 2, 3], [4, 4, 5, 5]]
    etc[:, :, 1] = [[3, 4, 3, 4], [4, 4, 5, 5]]
    etc[:, :, 2] = [[4, 5, 4, 5], [4, 4, 5, 5]]
    etc[:, :, 3] = [[2, 3, 2, 3], [5, 5, 6, 6]]
    etc[:, :, 4] = [[3, 4, 3, 4], [5, 5, 6, 6]]
    etc[:, :, 5] = [[4, 5, 4, 5], [5, 5, 6, 6]]
    expect = np.array([[0x0, 0x1555555555555555, 0xffffffffffffffff, 0x5555555555555555,
                        0x6aaaaaaaaaaaaaaa, 0xaaaaaaaaaaaaaaaa],
                       [0x0, 0x5555555555555555, 0xffffffffffffffff, 0x5555555555555555,
                        0xaaaaaaaaaaaaaaaa, 0xaaaaaaaaaaaaaaaa]], dtype=np.uint64)
    assert np.array_equal(impl.centroidtocode(etc), expect)
    one = np.zeros((2, 4, 1), order="F")
    one[:, :, 0] = [[2, 3, 2, 3], [4, 4, 5, 5]]
    assert np.array_equal(impl.centroidtocode(one), np.zeros((2, 1), dtype=np.uint64))


def test_vertex_ordering():
    vs = O.vertsortandorder
    assert vs(1) == ((1,), 1)
    assert vs(1, 2) == ((1, 2), 1) and vs(2, 1) == ((1, 2), 2)
    for v, o in (((1, 2, 3), 1), ((3, 1, 2), 2), ((2, 3, 1), 3), ((2, 1, 3), 4), ((3, 2, 1), 5), ((1, 3, 2), 6)):
        assert vs(*v) == ((1, 2, 3), o)
    with pytest.raises(Exception, match=r"Problem finding vertex ordering \(1, 1, 2\)"):
        vs(2, 1, 1)
    for v, o in (((1, 2, 3, 4), 1), ((1, 3, 2, 4), 2), ((2, 1, 3, 4), 3), ((2, 4, 1, 3), 4),
                 ((3, 1, 4, 2), 5), ((3, 4, 1, 2), 6), ((4, 2, 3, 1), 7), ((4, 3, 2, 1), 8)):
        assert vs(*v) == ((1, 2, 3, 4), o)
        assert HM._sort_face(v) == ((1, 2, 3, 4), o)
    with pytest.raises(Exception, match="Problem finding vertex ordering"):
        vs(1, 3, 3, 1)


# ------------------------------------------------ test/test_mesh.jl:94-245
def test_brickmesh(impl):
    etv, etc, etb, fc = impl.brickmesh((np.arange(4, 8),), (False,))
    assert np.array_equal(etv, [[1, 2, 3], [2, 3, 4]])
    assert np.array_equal(etb, [[1, 0, 0], [0, 0, 1]])
    assert fc == []
    assert np.array_equal(etc[:, :, 0], [[4, 5]]) and np.array_equal(etc[:, :, 2], [[6, 7]])

    etv, etc, etb, fc = impl.brickmesh((np.arange(4, 8),), (True,))
    assert np.array_equal(etb, np.zeros((2, 3)))
    assert [list(map(int, r)) for r in fc] == [[3, 2, 1]]

    etv, etc, etb, fc = impl.brickmesh((np.arange(2, 6), np.arange(4, 7)), (False, True))
    assert np.array_equal(etv, np.array([[1, 2, 5, 6], [2, 3, 6, 7], [3, 4, 7, 8],
                                         [5, 6, 9, 10], [6, 7, 10, 11], [7, 8, 11, 12]]).T)
    assert np.array_equal(etb, [[1, 0, 0, 1, 0, 0], [0, 0, 1, 0, 0, 1],
                                [0, 0, 0, 0, 0, 0], [0, 0, 0, 0, 0, 0]])
    assert [list(map(int, r)) for r in fc] == [[4, 4, 1, 2], [5, 4, 2, 3], [6, 4, 3, 4]]
    assert np.array_equal(etc[:, :, 0], [[2, 3, 2, 3], [4, 4, 5, 5]])
    assert np.array_equal(etc[:, :, 4], [[3, 4, 3, 4], [5, 5, 6, 6]])

    etv, etc, etb, fc = impl.brickmesh((np.arange(-1, 2, 2), np.arange(-1, 2, 2), np.arange(-1, 2)),
                                       (True, True, True))
    assert np.array_equal(etv, np.array([[1, 2, 3, 4, 5, 6, 7, 8], [5, 6, 7, 8, 9, 10, 11, 12]]).T)
    assert np.array_equal(etb, np.zeros((6, 2)))
    assert [list(map(int, r)) for r in fc] == [[1, 2, 1, 3, 5, 7], [1, 4, 1, 2, 5, 6],
                                              [2, 2, 5, 7, 9, 11], [2, 4, 5, 6, 9, 10],
                                              [2, 6, 1, 2, 3, 4]]
    assert np.array_equal(etc[:, :, 0], [[-1, 1, -1, 1, -1, 1, -1, 1], [-1, -1, 1, 1, -1, -1, 1, 1],
                                         [-1, -1, -1, -1, 0, 0, 0, 0]])

    etv, etc, etb, fc = impl.brickmesh((np.arange(-1, 2),) * 3, (False,) * 3,
                                       boundary=np.array([[11, 13, 15], [12, 14, 16]]))
    assert np.array_equal(etb, [[11, 0, 11, 0, 11, 0, 11, 0], [0, 12, 0, 12, 0, 12, 0, 12],
                                [13, 13, 0, 0, 13, 13, 0, 0], [0, 0, 14, 14, 0, 0, 14, 14],
                                [15, 15, 15, 15, 0, 0, 0, 0], [0, 0, 0, 0, 16, 16, 16, 16]])


@pytest.mark.parametrize("x,p,b", [((np.arange(1, 1001),), (False,), [1, 2]),
                                   ((np.arange(-1, 11, 2), np.arange(-1, 2), np.arange(-4, 2)),
                                    (True, False, True), [[1, 3, 5], [2, 4, 6]])])
def test_brickmesh_parts(impl, x, p, b):
    b = np.array(b).reshape(2, -1)
    etv, etc, etb, _ = impl.brickmesh(x, p, boundary=b)
    parts = [impl.brickmesh(x, p, boundary=b, part=j, numparts=50) for j in range(1, 51)]
    assert np.array_equal(etv, np.concatenate([q[0] for q in parts], axis=1))
    assert np.array_equal(etc, np.concatenate([q[1] for q in parts], axis=2))
    assert np.array_equal(etb, np.concatenate([q[2] for q in parts], axis=1))


# ------------------------------------------------ test/test_mesh.jl:247-336
def test_connect(impl):
    m = impl.connectmesh(*impl.partition(*impl.brickmesh((np.arange(0, 11),), (True,))))
    for e in range(10):
        assert np.array_equal(m["elemtocoord"][:, :, e], [[e, e + 1]])
    assert np.array_equal(m["elemtoelem"], [[10, 1, 2, 3, 4, 5, 6, 7, 8, 9], [2, 3, 4, 5, 6, 7, 8, 9, 10, 1]])
    assert np.array_equal(m["elemtoface"], [[2] * 10, [1] * 10])
    assert np.all(m["elemtoordr"] == 1) and np.all(m["elemtobndy"] == 0)

    m = impl.connectmesh(*impl.partition(*impl.brickmesh((np.arange(0, 5), np.arange(5, 10)), (False, True))))
    coords = [[0, 1, 5, 6], [1, 2, 5, 6], [1, 2, 6, 7], [0, 1, 6, 7], [0, 1, 7, 8], [0, 1, 8, 9],
              [1, 2, 8, 9], [1, 2, 7, 8], [2, 3, 7, 8], [2, 3, 8, 9], [3, 4, 8, 9], [3, 4, 7, 8],
              [3, 4, 6, 7], [2, 3, 6, 7], [2, 3, 5, 6], [3, 4, 5, 6]]
    for e, (x0, x1, y0, y1) in enumerate(coords):
        assert np.array_equal(m["elemtocoord"][:, :, e], [[x0, x1, x0, x1], [y0, y0, y1, y1]])
    assert np.array_equal(m["elemtoelem"], [
        [1, 1, 4, 4, 5, 6, 6, 5, 8, 7, 10, 9, 14, 3, 2, 15],
        [2, 15, 14, 3, 8, 7, 10, 9, 12, 11, 11, 12, 13, 13, 16, 16],
        [6, 7, 2, 1, 4, 5, 8, 3, 14, 9, 12, 13, 16, 15, 10, 11],
        [4, 3, 8, 5, 6, 1, 2, 7, 10, 15, 16, 11, 12, 9, 14, 13]])
    assert np.array_equal(m["elemtoface"], [
        [1, 2, 2, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2],
        [1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 2],
        [4] * 16, [3] * 16])
    assert np.all(m["elemtoordr"] == 1)


# ------------------------------------------------ test/test_mesh.jl:337-436
def test_mappings(impl):
    m = impl.connectmesh(*impl.partition(*impl.brickmesh((np.arange(0, 5),), (True,))))
    vM, vP = impl.mappings(3, m["elemtoelem"], m["elemtoface"], m["elemtoordr"])
    assert list(vM.ravel(order="F")) == [1, 4, 5, 8, 9, 12, 13, 16]
    assert list(vP.ravel(order="F")) == [16, 5, 4, 9, 8, 13, 12, 1]

    m = impl.connectmesh(*impl.partition(*impl.brickmesh((np.arange(-1, 2), np.arange(0, 2)), (False, True))))
    vM, vP = impl.mappings(2, m["elemtoelem"], m["elemtoface"], m["elemtoordr"])
    assert list(vM.ravel(order="F")) == [1, 4, 7, 3, 6, 9, 1, 2, 3, 7, 8, 9,
                                         10, 13, 16, 12, 15, 18, 10, 11, 12, 16, 17, 18]
    assert list(vP.ravel(order="F")) == [1, 4, 7, 10, 13, 16, 7, 8, 9, 1, 2, 3,
                                         3, 6, 9, 12, 15, 18, 16, 17, 18, 10, 11, 12]

    m = impl.connectmesh(*impl.partition(*impl.brickmesh((np.arange(0, 2), np.arange(0, 2), np.arange(-1, 2)),
                                                         (False, True, False))))
    vM, vP = impl.mappings(2, m["elemtoelem"], m["elemtoface"], m["elemtoordr"])
    fmask = np.array([[1, 3, 1, 7, 1, 19], [4, 6, 2, 8, 2, 20], [7, 9, 3, 9, 3, 21],
                      [10, 12, 10, 16, 4, 22], [13, 15, 11, 17, 5, 23], [16, 18, 12, 18, 6, 24],
                      [19, 21, 19, 25, 7, 25], [22, 24, 20, 26, 8, 26], [25, 27, 21, 27, 9, 27]])
    Np = 27
    assert np.array_equal(vM.ravel(order="F"), np.concatenate([fmask.ravel(order="F"), fmask.ravel(order="F") + Np]))
    expectP = np.concatenate([fmask[:, 0], fmask[:, 1], fmask[:, 3], fmask[:, 2], fmask[:, 4],
                              fmask[:, 4] + Np, fmask[:, 0] + Np, fmask[:, 1] + Np, fmask[:, 3] + Np,
                              fmask[:, 2] + Np, fmask[:, 5], fmask[:, 5] + Np])
    assert np.array_equal(vP.ravel(order="F"), expectP)


# ------------------------------------------------ test/test_mesh.jl:457-464
def test_partition_identity(impl):
    etv, etc, etb, fc = impl.brickmesh((np.arange(-1, 2, 2), np.arange(-1, 2, 2), np.arange(-2, 3)), (True,) * 3)
    n = impl.partition(etv, etc, etb, fc)
    assert np.array_equal(etv, n[0]) and np.array_equal(etc, n[1]) and np.array_equal(etb, n[2])
    assert [list(map(int, r)) for r in fc] == [list(map(int, r)) for r in n[3]]


# ------------------------------------------------ test/test_metric.jl:8-41
def test_metric_1d():
    r, w = O.lglpoints(4)
    D = O.spectralderivative(r)
    e2c = np.zeros((1, 2, 2), order="F")
    e2c[:, :, 0] = [[-1, 0]]
    e2c[:, :, 1] = [[0, 10]]
    (x,) = O.creategrid(e2c, r)
    assert np.allclose(x[:, 0], (r - 1) / 2) and np.allclose(x[:, 1], 5 * (r + 1))
    m = O.computemetric(D, x)
    assert np.allclose(m["J"][:, 0], 0.5) and np.allclose(m["J"][:, 1], 5)
    assert np.allclose(m["xix"][:, 0], 2) and np.allclose(m["xix"][:, 1], 0.2)
    assert np.allclose(m["nx"][0, 0], -1) and np.allclose(m["nx"][0, 1], 1)
    assert np.allclose(m["sJ"], 1)


# ------------------------------------------------ test/test_metric.jl:43-300
def _f2(r, s):
    return (9 * r - (1 + r) * s ** 2 + (r - 1) ** 2 * (1 - s ** 2 + s ** 3),
            10 * s + r ** 4 * (1 - s) + r ** 2 * s * (1 + s))


def test_metric_2d_rotation(impl):
    N = 2
    r, w = impl.lglpoints(N)
    D = impl.spectralderivative(r)
    e2c = np.zeros((2, 4, 4), order="F")
    e2c[:, :, 0] = [[0, 2, 0, 2], [0, 0, 2, 2]]
    e2c[:, :, 1] = [[2, 2, 0, 0], [0, 2, 0, 2]]
    e2c[:, :, 2] = [[2, 0, 2, 0], [2, 2, 0, 0]]
    e2c[:, :, 3] = [[0, 0, 2, 2], [2, 0, 2, 0]]
    x, y = impl.creategrid(e2c, r)
    x1 = np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2]])
    y1 = np.array([[0, 1, 2], [0, 1, 2], [0, 1, 2]])
    rot = lambda a: np.rot90(a, -1)
    xe = [x1, rot(x1), rot(rot(x1)), rot(rot(rot(x1)))]
    ye = [y1, rot(y1), rot(rot(y1)), rot(rot(rot(y1)))]
    for e in range(4):
        assert np.allclose(x[:, :, e], xe[e]) and np.allclose(y[:, :, e], ye[e])
    m = impl.computemetric(D, x, y)
    assert np.allclose(m["J"], 1)
    xix = np.zeros(4); xix[0], xix[2] = 1, -1
    xiy = np.zeros(4); xiy[1], xiy[3] = 1, -1
    etax = np.zeros(4); etax[1], etax[3] = -1, 1
    etay = np.zeros(4); etay[0], etay[2] = 1, -1
    for e in range(4):
        assert np.allclose(m["xix"][:, :, e], xix[e]) and np.allclose(m["xiy"][:, :, e], xiy[e])
        assert np.allclose(m["etax"][:, :, e], etax[e]) and np.allclose(m["etay"][:, :, e], etay[e])
    assert np.allclose(m["sJ"], 1)
    nx = np.zeros((4, 4)); ny = np.zeros((4, 4))
    nx[0, 0], nx[1, 0], nx[2, 1], nx[3, 1], nx[0, 2], nx[1, 2], nx[2, 3], nx[3, 3] = -1, 1, 1, -1, 1, -1, -1, 1
    ny[2, 0], ny[3, 0], ny[0, 1], ny[1, 1], ny[2, 2], ny[3, 2], ny[0, 3], ny[1, 3] = -1, 1, -1, 1, 1, -1, 1, -1
    for e in range(4):
        for f in range(4):
            assert np.allclose(m["nx"][:, f, e], nx[f, e], atol=1e-15)
            assert np.allclose(m["ny"][:, f, e], ny[f, e], atol=1e-15)


def test_metric_2d_polynomial_and_constant_preservation(impl):
    N = 4
    r, w = impl.lglpoints(N)
    D = impl.spectralderivative(r)
    Nq = N + 1
    e2c = np.zeros((2, 4, 1), order="F")
    e2c[:, :, 0] = [[-1, 1, -1, 1], [-1, -1, 1, 1]]
    x, y = impl.creategrid(e2c, r)
    xr = 7 + y ** 2 - 2 * y ** 3 + 2 * x * (1 - y ** 2 + y ** 3)
    xs = -2 * (1 + x) * y + (-1 + x) ** 2 * y * (-2 + 3 * y)
    yr = -4 * x ** 3 * (-1 + y) + 2 * x * y * (1 + y)
    ys = 10 - x ** 4 + x ** 2 * (1 + 2 * y)
    J = xr * ys - xs * yr
    x, y = _f2(x, y)
    m = impl.computemetric(D, np.asfortranarray(x), np.asfortranarray(y))
    assert np.allclose(m["J"], J)
    assert np.allclose(m["xix"], ys / J) and np.allclose(m["etax"], -yr / J)
    assert np.allclose(m["xiy"], -xs / J) and np.allclose(m["etay"], xr / J)
    nx, ny, sJ = m["nx"], m["ny"], m["sJ"]
    assert np.allclose(np.hypot(nx, ny), 1)
    assert np.allclose(sJ[:, 0] * nx[:, 0], -ys[0]) and np.allclose(sJ[:, 0] * ny[:, 0], xs[0])
    assert np.allclose(sJ[:, 1] * nx[:, 1], ys[-1]) and np.allclose(sJ[:, 1] * ny[:, 1], -xs[-1])
    assert np.allclose(sJ[:, 2] * nx[:, 2], yr[:, 0]) and np.allclose(sJ[:, 2] * ny[:, 2], -xr[:, 0])
    assert np.allclose(sJ[:, 3] * nx[:, 3], -yr[:, -1]) and np.allclose(sJ[:, 3] * ny[:, 3], xr[:, -1])
    # constant preservation (test_metric.jl:246-300)
    Jm, xix, etax = m["J"][:, :, 0], m["xix"][:, :, 0], m["etax"][:, :, 0]
    Cx = np.zeros((Nq, Nq))
    for n in range(Nq):
        Cx[:, n] += D @ (Jm[:, n] * xix[:, n])
        Cx[n, :] += D @ (Jm[n, :] * etax[n, :])
    assert np.abs(Cx).max() <= 1000 * np.finfo(float).eps


def _f3(r, s, t):
    return (s + r * t - (r ** 2 * s ** 2 * t ** 2) / 4,
            t - ((r * s * t) / 2 + 0.5) ** 3 + 1,
            r + (r / 2 + 0.5) ** 6 * (s / 2 + 0.5) ** 6 * (t / 2 + 0.5) ** 6)


def _cube(n):
    e2c = np.zeros((3, 8, n), order="F")
    e2c[:, :, 0] = [[-1, 1, -1, 1, -1, 1, -1, 1], [-1, -1, 1, 1, -1, -1, 1, 1], [-1, -1, -1, -1, 1, 1, 1, 1]]
    return e2c


def test_metric_3d_rotation(impl):
    th1, th2, th3 = 2 * np.pi * 0.9, 2 * np.pi * -0.56, 2 * np.pi * 0.33
    Qm = np.array([[np.cos(th1), -np.sin(th1), 0], [np.sin(th1), np.cos(th1), 0], [0, 0, 1]])
    Qm = Qm @ np.array([[np.cos(th2), 0, -np.sin(th2)], [0, 1, 0], [np.sin(th2), 0, np.cos(th2)]])
    Qm = Qm @ np.array([[1, 0, 0], [0, np.cos(th3), -np.sin(th3)], [0, np.sin(th3), np.cos(th3)]])
    r, w = impl.lglpoints(2)
    D = impl.spectralderivative(r)
    e2c = np.zeros((3, 8, 1), order="F")
    e2c[:, :, 0] = Qm @ np.array([[0, 2, 0, 2, 0, 2, 0, 2], [0, 0, 2, 2, 0, 0, 2, 2], [0, 0, 0, 0, 2, 2, 2, 2]])
    x, y, z = impl.creategrid(e2c, r)
    m = impl.computemetric(D, x, y, z)
    assert np.allclose(m["J"], 1)
    for key, val in (("xix", Qm[0, 0]), ("xiy", Qm[1, 0]), ("xiz", Qm[2, 0]), ("etax", Qm[0, 1]),
                     ("etay", Qm[1, 1]), ("etaz", Qm[2, 1]), ("zetax", Qm[0, 2]), ("zetay", Qm[1, 2]),
                     ("zetaz", Qm[2, 2])):
        assert np.allclose(m[key], val)
    assert np.allclose(m["sJ"], 1)
    for f in range(6):
        sgn = -1 if f % 2 == 0 else 1
        assert np.allclose(m["nx"][:, f], sgn * Qm[0, f // 2])
        assert np.allclose(m["ny"][:, f], sgn * Qm[1, f // 2])
        assert np.allclose(m["nz"][:, f], sgn * Qm[2, f // 2])


def test_metric_3d_polynomial(impl):
    N = 9
    r, w = impl.lglpoints(N)
    D = impl.spectralderivative(r)
    x, y, z = impl.creategrid(_cube(1), r)
    xr, xs, xt = z - (x * y ** 2 * z ** 2) / 2, 1 - (x ** 2 * y * z ** 2) / 2, x - (x ** 2 * y ** 2 * z) / 2
    yr = -(3 * y * z * ((x * y * z) / 2 + 0.5) ** 2) / 2
    ys = -(3 * x * z * ((x * y * z) / 2 + 0.5) ** 2) / 2
    yt = 1 - (3 * x * y * ((x * y * z) / 2 + 0.5) ** 2) / 2
    a, b, c = x / 2 + 0.5, y / 2 + 0.5, z / 2 + 0.5
    zr, zs, zt = 3 * a ** 5 * b ** 6 * c ** 6 + 1, 3 * a ** 6 * b ** 5 * c ** 6, 3 * a ** 6 * b ** 6 * c ** 5
    J = xr * (ys * zt - yt * zs) + yr * (zs * xt - zt * xs) + zr * (xs * yt - xt * ys)
    exact = dict(xix=(ys * zt - yt * zs) / J, xiy=(zs * xt - zt * xs) / J, xiz=(xs * yt - xt * ys) / J,
                 etax=(yt * zr - yr * zt) / J, etay=(zt * xr - zr * xt) / J, etaz=(xt * yr - xr * yt) / J,
                 zetax=(yr * zs - ys * zr) / J, zetay=(zr * xs - zs * xr) / J, zetaz=(xr * ys - xs * yr) / J)
    X = [np.asfortranarray(v) for v in _f3(x, y, z)]
    m = impl.computemetric(D, *X)
    assert np.allclose(m["J"], J)
    for k, v in exact.items():
        assert np.allclose(m[k], v), k
    assert np.allclose(np.sqrt(m["nx"] ** 2 + m["ny"] ** 2 + m["nz"] ** 2), 1)


def test_metric_3d_constant_preservation(impl):
    N = 5
    Nq = N + 1
    r, w = impl.lglpoints(N)
    D = impl.spectralderivative(r)
    x, y, z = impl.creategrid(_cube(1), r)
    X = [np.asfortranarray(v) for v in _f3(x, y, z)]
    m = impl.computemetric(D, *X)
    J = m["J"][..., 0]
    C = np.zeros((3, Nq, Nq, Nq))
    for c, (a, b, d) in enumerate((("xix", "etax", "zetax"), ("xiy", "etay", "zetay"), ("xiz", "etaz", "zetaz"))):
        A, B, Dd = m[a][..., 0], m[b][..., 0], m[d][..., 0]
        for mm in range(Nq):
            for n in range(Nq):
                C[c][:, n, mm] += D @ (J[:, n, mm] * A[:, n, mm])
                C[c][n, :, mm] += D @ (J[n, :, mm] * B[n, :, mm])
                C[c][n, mm, :] += D @ (J[n, mm, :] * Dd[n, mm, :])
    assert np.abs(C).max() <= 1000 * np.finfo(float).eps
