"""ctypes binding of libcanary_b200.so (the C-ABI declared in
include/canary_b200.h).

The library is located next to this package (../lib/libcanary_b200.so) or
through $CANARY_B200_LIB.  Loading fails loudly when it is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CANARY_B200_LIB",
                          os.path.join(os.path.dirname(_HERE), "lib", "libcanary_b200.so"))

# status codes of include/canary_b200.h
CB_OK, CB_ERR_ARG, CB_ERR_UNSUPPORTED, CB_ERR_BC, CB_ERR_CUDA, CB_ERR_MESH, \
    CB_ERR_NONFINITE, CB_ERR_TIMEOUT, CB_ERR_NOMEM = range(9)

EXPORTS = (
    "cb_version", "cb_last_error", "cb_device_status", "cb_max_order",
    "cb_volumerhs", "cb_volumerhs_f32", "cb_fluxrhs", "cb_fluxrhs_f32",
    "cb_updatesolution", "cb_updatesolution_f32",
    "cb_volume_grad", "cb_flux_grad", "cb_update_gradQ", "cb_volume_div", "cb_flux_div",
    "cb_solver_create", "cb_lsrk_run", "cb_solver_set_offset", "cb_solver_sums",
    "cb_solver_destroy", "cb_solver_status_async", "cb_lsrk_stage_noalloc", "cb_noalloc_status",
    "cb_solver_reset_status", "cb_solver_test_timeout", "cb_solver_set_kernel", "cb_solver_get_kernel",
    "cb_solver_create_ghosted", "cb_solver_stage", "cb_solver_stage_pass", "cb_solver_current", "cb_solver_settle",
    "cb_solver_pack", "cb_solver_unpack", "cb_solver_pack_faces", "cb_solver_unpack_faces",
    "cb_solver_set_split", "cb_solver_stage_split",
    "cb_computegeometry", "cb_brickmesh", "cb_mesh_create", "cb_mesh_affine", "cb_mesh_destroy",
    "cb_batch_create", "cb_batch_set_variant", "cb_batch_get_variant", "cb_batch_set_affine",
    "cb_batch_set_concurrent", "cb_batch_slot_variant", "cb_batch_variant_info", "cb_batch_add",
    "cb_batch_run", "cb_batch_info", "cb_batch_release", "cb_batch_status", "cb_batch_status_async", "cb_batch_destroy",
)


class CanaryError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[canary_b200 error {code}] {msg}")
        self.code = code


class cb_phys(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("gamma", "R_gas", "c_p", "c_v", "gravity", "Pr", "lambda_", "visc")]


_lib = None

vp = C.c_void_p
i64 = C.c_int64
dbl = C.c_double


def lib() -> C.CDLL:
    """Load (once) and return the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libcanary_b200.so not found at {LIB_PATH}; build it with "
                           "`python canary.jl_b200/build.py` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    L.cb_last_error.restype = C.c_char_p
    for name in EXPORTS:
        getattr(L, name)  # raises AttributeError if a symbol is missing
    phys_p = C.POINTER(cb_phys)
    L.cb_volumerhs.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, phys_p, vp]
    L.cb_volumerhs_f32.argtypes = L.cb_volumerhs.argtypes
    L.cb_fluxrhs.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, vp, vp, vp, phys_p, vp]
    L.cb_fluxrhs_f32.argtypes = L.cb_fluxrhs.argtypes
    L.cb_updatesolution.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, dbl, dbl, dbl, dbl, vp]
    L.cb_updatesolution_f32.argtypes = L.cb_updatesolution.argtypes
    L.cb_volume_grad.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, phys_p, vp]
    L.cb_flux_grad.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, vp, vp, vp, phys_p, vp]
    L.cb_update_gradQ.argtypes = [C.c_int, C.c_int, vp, vp, vp, i64, vp]
    L.cb_volume_div.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, i64, phys_p, vp]
    L.cb_flux_div.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, i64, vp, vp, vp, phys_p, vp]
    L.cb_device_status.argtypes = [vp]
    L.cb_solver_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, i64, vp, vp, vp, vp,
                                   vp, vp, vp, vp, phys_p, vp]
    L.cb_lsrk_run.argtypes = [vp, i64, dbl]
    L.cb_solver_sums.argtypes = [vp, C.POINTER(C.c_double)]
    L.cb_solver_set_offset.argtypes = [vp, C.POINTER(C.c_double)]
    L.cb_solver_destroy.argtypes = [vp]
    L.cb_solver_create_ghosted.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, i64, i64, vp, vp, vp, vp,
                                           vp, vp, vp, vp, phys_p, vp]
    L.cb_solver_stage.argtypes = [vp, C.c_int, dbl, C.POINTER(vp)]
    L.cb_solver_stage_pass.argtypes = [vp, C.c_int, dbl, C.c_int, C.POINTER(vp)]
    L.cb_solver_current.argtypes = [vp, C.POINTER(vp)]
    L.cb_solver_settle.argtypes = [vp]
    L.cb_solver_pack.argtypes = [vp, C.c_int, vp, i64, vp]
    L.cb_solver_unpack.argtypes = [vp, C.c_int, vp, i64, i64]
    L.cb_solver_pack_faces.argtypes = [vp, C.c_int, vp, i64, vp]
    L.cb_solver_unpack_faces.argtypes = [vp, C.c_int, vp, i64, vp]
    L.cb_solver_set_split.argtypes = [vp, i64]
    L.cb_solver_stage_split.argtypes = [vp, C.c_int, dbl, C.c_int, C.POINTER(vp)]
    L.cb_lsrk_stage_noalloc.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, i64,
                                        phys_p, dbl, dbl, dbl, vp, vp]
    L.cb_noalloc_status.argtypes = [vp, C.POINTER(C.c_uint)]
    L.cb_computegeometry.argtypes = [C.c_int, C.c_int, i64, vp, dbl, vp, vp, vp, vp, vp, vp]
    L.cb_mesh_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, i64, vp, vp, vp, vp, vp, vp, vp]
    L.cb_mesh_destroy.argtypes = [vp]
    L.cb_brickmesh.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.cb_mesh_affine.argtypes = [vp, C.POINTER(C.c_int)]
    L.cb_batch_set_affine.argtypes = [vp, C.c_int]
    L.cb_batch_set_concurrent.argtypes = [vp, C.c_int]
    L.cb_batch_slot_variant.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
    L.cb_batch_variant_info.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(i64)]
    L.cb_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, phys_p, vp]
    L.cb_batch_set_variant.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.cb_batch_get_variant.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.cb_batch_add.argtypes = [vp, vp, vp, vp, dbl, i64, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.cb_batch_run.argtypes = [vp, i64]
    L.cb_batch_info.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64)]
    L.cb_batch_release.argtypes = [vp, C.c_int]
    L.cb_batch_status.argtypes = [vp, C.POINTER(C.c_uint)]
    L.cb_batch_destroy.argtypes = [vp]
    L.cb_batch_status_async.argtypes = [vp, vp]
    L.cb_solver_status_async.argtypes = [vp, vp]
    L.cb_solver_reset_status.argtypes = [vp]
    L.cb_solver_test_timeout.argtypes = [vp]
    L.cb_solver_set_kernel.argtypes = [vp, C.c_int]
    L.cb_solver_get_kernel.argtypes = [vp, C.POINTER(C.c_int)]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != CB_OK:
        raise CanaryError(rc, lib().cb_last_error().decode(errors="replace"))
