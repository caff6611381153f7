"""Build libcanary_b200.so (sm_100a) from csrc/ with nvcc.

    python canary.jl_b200/build.py [--force] [-j JOBS] [--ptxas-verbose]

Each translation unit is compiled to an object in csrc/_build/ (git-ignored)
and the objects are linked into lib/libcanary_b200.so next to this file.  The
CUDA runtime is linked statically so the library does not depend on the
runtime version that the host process (e.g. PyTorch) loads.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(CSRC, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcanary_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-I", INCLUDE] + ARCH


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
           if f.endswith((".cuh", ".h", ".inc"))]
    out.append(os.path.join(INCLUDE, "canary_b200.h"))
    out.append(os.path.abspath(__file__))  # the flags
    return out


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + _deps())


# per-file flags: the geometry follows the reference's arithmetic without
# multiply-add contraction; the FP32 form's kernels divide and take square
# roots with the hardware approximations (within 2 ulp of FP32 rounding,
# several instructions fewer each; the form's bar is 1e-5 relative L2)
_FP32_FAST = ["-prec-div=false", "-prec-sqrt=false"]
FILE_FLAGS = {"cb_geometry.cu": ["-fmad=false"], "cb_batch_2d_f32.cu": _FP32_FAST, "cb_batch_3d_f32.cu": _FP32_FAST,
              "cb_inst_2d_f32.cu": _FP32_FAST, "cb_inst_3d_f32.cu": _FP32_FAST}


def _compile(src: str, verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    extra = FILE_FLAGS.get(os.path.basename(src), [])
    cmd = [nvcc()] + NVCC_FLAGS + extra + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [s for s, o in zip(srcs, objs) if force or verbose or _stale(o, s)]
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
                logs.append(log)
    if todo or not os.path.exists(LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        subprocess.run(cmd, check=True)
    if verbose:
        sys.stderr.write("".join(logs))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.ptxas_verbose))


if __name__ == "__main__":
    main()
