"""Builds libfdtd_b200.so in-tree (sm_100a only).

    python -m fdtd3d_b200.build [--force]

Translation units and flags:
  csrc/setup.cpp          g++  -O2 -ffp-contract=off   host geometry/set-up (FP64, reference op order)
  csrc/plain_kernels.cu   nvcc --fmad=false            FP64 plain form + incident grid kernels
  csrc/fast_kernels.cu    nvcc                          FP32 / FP16-storage fused form, reductions
  csrc/fused3d.cu         nvcc                          3-D single-sweep E+H kernel (register-blocked)
  csrc/sweep3d.cu         nvcc                          3-D single-sweep E+H kernel (TMA-pipelined)
  csrc/sweep2.cu          nvcc                          3-D two-step (temporally blocked) sweep
  csrc/fdtd_api.cu        nvcc                          C ABI, context, launch sequence
  csrc/cli.cpp            g++ -> fdtd3d-b200            command-line drop-in over the C ABI
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
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfdtd_b200.so")
CLI = os.path.join(HERE, "fdtd3d-b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolchain is required to build libfdtd_b200.so")
    return cand


def _units():
    nvcc = _nvcc()
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-I", CSRC]
    units = [
        ("setup.cpp", ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", CSRC]),
        ("plain_kernels.cu", [nvcc] + common + ["--fmad=false"]),
        ("fast_kernels.cu", [nvcc] + common),
        ("fdtd_api.cu", [nvcc] + common),
    ]
    if os.path.exists(os.path.join(CSRC, "fused3d.cu")):
        units.append(("fused3d.cu", [nvcc] + common))
    for extra in ("sweep3d.cu", "sweep2.cu", "tfsf2.cu", "tmz_batch.cu", "adjoint.cu", "noalloc.cu", "ntff.cu"):
        if os.path.exists(os.path.join(CSRC, extra)):
            units.append((extra, [nvcc] + common))
    return units


def _deps_mtime() -> float:
    m = 0.0
    for root in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(root):
            m = max(m, os.path.getmtime(os.path.join(root, f)))
    return m


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    units = _units()

    def compile_one(u):
        name, cmd = u
        obj = os.path.join(BUILD, name + ".o")
        full = cmd + ["-c", os.path.join(CSRC, name), "-o", obj]
        r = subprocess.run(full, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(full)}\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(units)) as ex:
        objs = list(ex.map(compile_one, units))
    tmp = LIB + ".tmp"
    link = [_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(link)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    # the command-line drop-in, linked against the library next to it
    cli = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", os.path.join(CSRC, "cli.cpp"), "-o", CLI + ".tmp", "-L", HERE,
           "-lfdtd_b200", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cli, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"cli build failed: {' '.join(cli)}\n{r.stdout}\n{r.stderr}")
    os.replace(CLI + ".tmp", CLI)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
