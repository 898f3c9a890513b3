"""Builds libfluidstep.so (the product) for sm_100a with nvcc.

    python fluid-engine_b200/build.py [--verbose]

Device code is compiled with -fmad=false -prec-div=true -prec-sqrt=true
-ftz=false: every float operation rounds once, in source order, so the
kernels reproduce the host oracle bit for bit.  The library links the CUDA
runtime statically and exports only the C ABI of include/fluid_step.h.

A second library, libfluidstep_contract.so, is the same C ABI with the
physics kernels (fe_kernels.cu) compiled with -fmad=true: the compiler may
contract a multiply and an add into one fused multiply-add.  Its results
are checked against the FP64 evaluation of the step within a relative
tolerance instead of bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "fluid_step", "libfluidstep.so")
CONTRACT_OUT = os.path.join(HERE, "fluid_step", "libfluidstep_contract.so")
CONTRACT_SOURCES = ["fe_kernels.cu"]
BUILD = os.path.join(HERE, "_build")

SOURCES = ["fe_kernels.cu", "fe_sort.cu", "fe_api.cu", "fe_sort_noalloc.cu", "fe_mlp.cu", "fe_tune.cu",
           "fe_splat.cu", "fe_raymarch.cu",
           "fe_model.cu", "fe_learned.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true",
         "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "-Xptxas", "-v", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "fluid_step.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or newer(o, [s] + headers):
            cmd = [nvcc()] + ARCH + FLAGS + ["-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            log = r.stdout + r.stderr
            if r.returncode != 0:
                sys.stderr.write(log)
                raise RuntimeError(f"nvcc failed on {src}")
            with open(o + ".log", "w") as f:
                f.write(log)
            if verbose:
                sys.stdout.write(log)
    link(OUT, objs, force)
    # the contraction build: the physics kernels again with -fmad=true
    contract_flags = ["-fmad=true" if f == "-fmad=false" else f for f in FLAGS]
    cobjs = []
    for o, src in zip(objs, SOURCES):
        if src not in CONTRACT_SOURCES:
            cobjs.append(o)
            continue
        s = os.path.join(CSRC, src)
        co = os.path.join(BUILD, src.replace(".cu", "_contract.o"))
        cobjs.append(co)
        if force or newer(co, [s] + headers):
            cmd = [nvcc()] + ARCH + contract_flags + ["-c", s, "-o", co]
            r = subprocess.run(cmd, capture_output=True, text=True)
            log = r.stdout + r.stderr
            if r.returncode != 0:
                sys.stderr.write(log)
                raise RuntimeError(f"nvcc failed on {src} (contraction build)")
            with open(co + ".log", "w") as f:
                f.write(log)
    link(CONTRACT_OUT, cobjs, force)
    return OUT


def link(out: str, objs, force: bool) -> None:
    if force or newer(out, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", out] + objs + ["-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"link of {os.path.basename(out)} failed")


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
