"""Builds libtrench_b200.so in-tree with nvcc for sm_100a.

Each translation unit has its own flags: the reference-exact FP64 tracer is
compiled with -fmad=false (no fused multiply-add contraction), the others with
the default contraction.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
ROOT = HERE.parent
LIB = HERE / "libtrench_b200.so"
BUILD = ROOT / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
UNITS = {
    "tb_capi.cu": [],
    "tb_trace_f64.cu": ["-fmad=false"],
    "tb_trace_f32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "tb_poisson.cu": [],
    "tb_step.cu": ["-fmad=false"],
    "tb_bench.cu": [],
    "tb_inject.cu": [],
    "tb_adjoint.cu": ["-fmad=false"],
}


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found")
    return path


def sources():
    return [CSRC / u for u in UNITS] + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "trench_b200.h"]


def up_to_date():
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources())


def build(force=False, verbose=False, ptxas_info=False):
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    for unit, flags in UNITS.items():
        obj = BUILD / (unit + ".o")
        cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(CSRC / unit), "-o", str(obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
