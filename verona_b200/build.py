"""Build libverona_b200.so in-tree with nvcc for sm_100a.

Translation units and their floating-point contract:
  vb_stage_f64.cu, vb_ref1d.cu, vb_api.cu  -fmad=false  (FP64 path rounds as
                                            the reference: no FMA contraction)
  vb_stage_f64c.cu                          -fmad=true   (the FP64 stage kernels with FMA
                                            contraction, namespace vb_f64c; tuning
                                            fp64_contract)
  vb_stage_f32.cu                           -fmad=true, approximate FP32 divide and
                                            square root, FTZ (FP32-bulk path; the
                                            FP64 con2prim in it stays IEEE)
  vb_mlp.cu                                 -fmad=true   (BF16 tensor-core MLP)
  vb_batch_f64.cu / vb_batch_f32.cu         as the FP64 / FP32 stage units (batched problems)
Objects go to verona_b200/_build/, the library to verona_b200/libverona_b200.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libverona_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -Werror=shadow: a local that shadows another (a loop counter named like a
# physical constant) is a build error
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Werror=shadow", "-I", CSRC,
          "-I", INC, "--expt-relaxed-constexpr"]
UNITS = {
    "vb_stage_f64.cu": ["-fmad=false"],
    "vb_stage_f64c.cu": ["-fmad=true"],
    "vb_ref1d.cu": ["-fmad=false"],
    "vb_api.cu": ["-fmad=false"],
    "vb_stage_f32.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_newer(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    heads = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    heads.append(os.path.join(INC, "verona_b200.h"))
    return any(os.path.getmtime(p) > t for p in [src] + heads)


def _compile(unit: str, flags: list[str], verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
    if _deps_newer(obj, src):
        cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    units = dict(UNITS)
    if os.path.exists(os.path.join(CSRC, "vb_mlp.cu")):
        units["vb_mlp.cu"] = ["-fmad=true"]  # the learned-guess Newton refinement is FP64 with FMA
    if os.path.exists(os.path.join(CSRC, "vb_batch.cu")):
        units["vb_batch.cu"] = ["-fmad=false"]
        units["vb_batch_f64.cu"] = ["-fmad=false"]
        units["vb_batch_f32.cu"] = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
    if os.path.exists(os.path.join(CSRC, "vb_grid.cu")):
        units["vb_grid.cu"] = ["-fmad=false"]
    if os.path.exists(os.path.join(CSRC, "vb_noalloc.cu")):
        units["vb_noalloc.cu"] = ["-fmad=false"]
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), units.items()))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
