"""Build the in-tree shared library ``sharpclaw_b200/libsharpclaw_b200.so``.

Every CUDA translation unit is compiled for sm_100a with nvcc (cross-compiles
without a GPU) and linked with the static CUDA runtime, so the library loads
with no dependency beyond the driver.  The FP64_STRICT unit is compiled with
``--fmad=false``: its arithmetic then follows the reference's written
evaluation order (no fused multiply-add contraction).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsharpclaw_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE,
          "--expt-relaxed-constexpr"]
FAST32 = ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]

UNITS = {
    "scl_capi.cu": [],
    "scl_frames.cu": [],
    "scl_noalloc.cu": [],
    "scl_batch.cu": [],
    "scl_adjoint.cu": ["--fmad=false"],
    "scl_prec_fp64.cu": ["--fmad=true"],
    "scl_prec_fp64s.cu": ["--fmad=false"],
    "scl_prec_mixed.cu": ["--fmad=true"] + FAST32,
    "scl_prec_fp32.cu": ["--fmad=true"] + FAST32,
    "scl_prec_fp64_2d.cu": ["--fmad=true"],
    "scl_prec_fp64s_2d.cu": ["--fmad=false"],
    "scl_prec_mixed_2d.cu": ["--fmad=true"] + FAST32,
    "scl_prec_fp32_2d.cu": ["--fmad=true"] + FAST32,
}


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(INCLUDE, "sharpclaw_cuda.h")]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(unit, extra, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
    if not _stale(obj, [src] + _deps()):
        return obj
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    # the large per-form units first, so the small ones fill the gaps
    order = sorted(UNITS.items(), key=lambda kv: not kv[0].startswith("scl_prec_"))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(12, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), order))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
