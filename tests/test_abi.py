"""The C-ABI library loads on a machine without a GPU and exports every
symbol that include/canary_b200.h declares; argument validation answers
without touching the device."""
import ctypes as C
import os
import re

import pytest

from canary_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "canary_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cb_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "cb_volumerhs" in syms and "cb_lsrk_run" in syms
    assert set(syms) == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s


def test_version_and_orders():
    L = _lib.lib()
    assert L.cb_version() >= 1
    assert L.cb_max_order(2) >= 8 and L.cb_max_order(3) >= 10
    assert L.cb_max_order(4) == 0


def test_argument_validation_without_device():
    L = _lib.lib()
    phys = _lib.cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
    dummy = C.c_void_p(16)  # never dereferenced: validation fails first
    assert L.cb_volumerhs(4, 3, dummy, dummy, dummy, dummy, 1, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert "dim" in L.cb_last_error().decode()
    assert L.cb_volumerhs(3, 99, dummy, dummy, dummy, dummy, 1, C.byref(phys), None) == _lib.CB_ERR_UNSUPPORTED
    assert L.cb_volumerhs(3, 3, None, dummy, dummy, dummy, 1, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert L.cb_volumerhs(3, 3, dummy, dummy, dummy, dummy, -1, C.byref(phys), None) == _lib.CB_ERR_ARG
    h = C.c_void_p()
    assert L.cb_solver_create(C.byref(h), 3, 3, 16, 1, dummy, dummy, dummy, dummy, dummy, dummy,
                              dummy, dummy, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert L.cb_lsrk_run(None, 1, 0.1) == _lib.CB_ERR_ARG


def test_check_raises():
    with pytest.raises(_lib.CanaryError):
        L = _lib.lib()
        phys = _lib.cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
        _lib.check(L.cb_volumerhs(5, 3, None, None, None, None, 1, C.byref(phys), None))


def test_batch_argument_validation_without_device():
    L = _lib.lib()
    phys = _lib.cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
    negvisc = _lib.cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, -1e-3)
    dummy = C.c_void_p(16)
    h = C.c_void_p()
    # orders outside the batched range, bad dim / precision, null arrays
    assert L.cb_mesh_create(C.byref(h), 2, 9, 64, 4, dummy, dummy, dummy, dummy, dummy, dummy,
                            None) == _lib.CB_ERR_UNSUPPORTED
    assert L.cb_mesh_create(C.byref(h), 3, 8, 64, 4, dummy, dummy, dummy, dummy, dummy, dummy,
                            None) == _lib.CB_ERR_UNSUPPORTED
    assert L.cb_mesh_create(C.byref(h), 4, 3, 64, 4, dummy, dummy, dummy, dummy, dummy, dummy,
                            None) == _lib.CB_ERR_ARG
    assert L.cb_mesh_create(C.byref(h), 2, 3, 16, 4, dummy, dummy, dummy, dummy, dummy, dummy,
                            None) == _lib.CB_ERR_ARG
    assert L.cb_mesh_create(C.byref(h), 2, 3, 64, 4, None, dummy, dummy, dummy, dummy, dummy,
                            None) == _lib.CB_ERR_ARG
    assert L.cb_batch_create(C.byref(h), 16, 8, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert L.cb_batch_create(C.byref(h), 64, 0, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert L.cb_batch_create(C.byref(h), 64, 8, C.byref(negvisc), None) == _lib.CB_ERR_ARG
    assert "visc" in L.cb_last_error().decode()
    assert L.cb_batch_set_variant(None, 2, 3, 0) == _lib.CB_ERR_ARG
    assert L.cb_batch_run(None, 1) == _lib.CB_ERR_ARG
    assert L.cb_batch_release(None, 0) == _lib.CB_ERR_ARG
    assert L.cb_batch_info(None, 0, None, None) == _lib.CB_ERR_ARG
    assert L.cb_batch_destroy(None) == _lib.CB_OK and L.cb_mesh_destroy(None) == _lib.CB_OK


def test_partition_and_setup_argument_validation_without_device():
    """The stage / exchange API of the partitioned solve and the device brick
    mesh reject bad arguments before touching the device."""
    L = _lib.lib()
    phys = _lib.cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
    dummy = C.c_void_p(16)
    h = C.c_void_p()
    nxt = C.c_void_p()
    assert L.cb_solver_create_ghosted(C.byref(h), 3, 3, 64, 8, -1, dummy, dummy, dummy, dummy, dummy, dummy,
                                      dummy, dummy, C.byref(phys), None) == _lib.CB_ERR_ARG
    assert L.cb_solver_stage(None, 0, 1e-3, C.byref(nxt)) == _lib.CB_ERR_ARG
    assert L.cb_solver_stage_pass(None, 0, 1e-3, 0, C.byref(nxt)) == _lib.CB_ERR_ARG
    assert L.cb_solver_settle(None) == _lib.CB_ERR_ARG
    assert L.cb_solver_current(None, C.byref(nxt)) == _lib.CB_ERR_ARG
    assert L.cb_solver_pack(None, 0, dummy, 1, dummy) == _lib.CB_ERR_ARG
    assert L.cb_solver_unpack(None, 0, dummy, 0, 1) == _lib.CB_ERR_ARG
    n = (C.c_int64 * 3)(2, 2, 2)
    xs = (C.c_void_p * 3)(16, 16, 16)
    per = (C.c_int * 3)(1, 1, 1)
    assert L.cb_brickmesh(4, 3, n, xs, per, None, dummy, dummy, dummy, dummy, None) == _lib.CB_ERR_ARG
    bad = (C.c_int64 * 3)(2, 0, 2)
    assert L.cb_brickmesh(3, 3, bad, xs, per, None, dummy, dummy, dummy, dummy, None) == _lib.CB_ERR_ARG
    assert L.cb_mesh_affine(None, None) == _lib.CB_ERR_ARG
    assert L.cb_batch_set_affine(None, 1) == _lib.CB_ERR_ARG
    assert L.cb_batch_set_concurrent(None, 1) == _lib.CB_ERR_ARG
    assert L.cb_batch_slot_variant(None, 0, None) == _lib.CB_ERR_ARG

