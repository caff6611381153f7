"""Brick mesh and connectivity on the device (cb_brickmesh) against the host
mirror of brickmesh -> partition -> connectmesh -> mappings (itself pinned
to the reference's known answers in tests/test_reference_pins.py): the
element order (Hilbert code of the centroids), corner coordinates, boundary
codes and vmapM / vmapP must be identical, and so must the geometry that
cb_computegeometry builds from them.
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from canary_b200 import dg
from canary_b200.mesh import brickmesh, connectmesh, mappings, partition

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def host_maps(N, x, periodic, boundary=None):
    cm = connectmesh(*partition(*brickmesh(x, periodic, boundary=boundary)))
    vM, vP = mappings(N, cm["elemtoelem"], cm["elemtoface"], cm["elemtoordr"])
    return cm["elemtocoord"], cm["elemtobndy"], vM, vP


CASES = [
    (2, 4, (np.linspace(0, 10, 4), np.linspace(0, 10, 5)), (True, True), None),
    (2, 3, (np.linspace(0, 1, 6), np.array([0.0, 0.1, 0.5, 0.55, 1.0])), (False, True), [[1, 2], [3, 4]]),
    (2, 5, (np.linspace(0, 1, 2), np.linspace(-1, 1, 7)), (True, False), None),
    (2, 2, (np.linspace(0, 1, 3), np.linspace(0, 1, 3)), (True, True), None),
    (2, 8, (np.linspace(0, 10, 65), np.linspace(0, 10, 65)), (True, True), None),
    (3, 3, (np.linspace(0, 1, 3), np.linspace(0, 2, 4), np.linspace(0, 3, 5)), (True, False, True), None),
    (3, 2, (np.linspace(0, 1, 2), np.linspace(0, 1, 2), np.linspace(0, 1, 3)), (True, True, True), None),
    (3, 4, (np.linspace(0, 2 * math.pi, 17),) * 3, (True, True, True), None),
    (3, 5, (np.array([0, 0.3, 1.0]), np.linspace(0, 1, 4), np.geomspace(1, 2, 5)), (False, False, False),
     [[1, 1, 1], [1, 1, 1]]),
]


@pytest.mark.parametrize("dim,N,x,periodic,boundary", CASES)
def test_device_connectivity_matches_host(dim, N, x, periodic, boundary):
    etc, etb, vM, vP = host_maps(N, x, periodic, boundary)
    dm = dg.DeviceMesh.build(dim, N, x, periodic, boundary=boundary)
    assert np.array_equal(dg.from_device(dm.elemtocoord, etc.shape), etc)
    assert np.array_equal(dg.from_device(dm.elemtobndy, etb.shape), etb)
    assert np.array_equal(dg.from_device(dm.vmapM, vM.shape), vM)
    assert np.array_equal(dg.from_device(dm.vmapP, vP.shape), vP)
    hm = dg.DeviceMesh.build(dim, N, x, periodic, boundary=boundary, connect="host")
    assert bool((hm.vgeo == dm.vgeo).all()) and bool((hm.sgeo == dm.sgeo).all())
