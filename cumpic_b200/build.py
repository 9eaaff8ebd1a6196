"""Build recipe of the CUDA library (sm_100a) and of the CPU oracle.

``build_library()`` compiles the units in ``UNITS`` (cumpic_b200/csrc) with
nvcc and links them into cumpic_b200/libcumc_b200.so. FMA contraction is off
in the FP64 units so that they are bit-compatible with the FP64 restatement
used as the test oracle.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcumc_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
# FP64 path: no multiply-add contraction, IEEE division and square root, so
# that results are bit-compatible with the FP64 restatement of the reference.
FP64_FLAGS = ["--fmad=false"]
# mixed path: FMA contraction; IEEE-rounded FP32 division and square root (the
# approximate forms raise the density error at t_end from 1.06e-5 to 1.5e-5 on
# Orszag-Tang 256^3); the column walker compiled for 10 blocks a SM (96
# registers) instead of the FP64 unit's 8.
MIXED_FLAGS = ["--fmad=true", "-prec-div=true", "-prec-sqrt=true", "-DCUMC_WALK_MINB=10"]
UNITS = {"cumc_api.cu": FP64_FLAGS, "cumc_mixed.cu": MIXED_FLAGS, "cumc_static.cu": FP64_FLAGS}
NVCC_FLAGS = COMMON + FP64_FLAGS  # flags of the FP64 unit (kept for tools that print them)


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh"))] + [
        os.path.join(ROOT, "include", "cumc.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    if force or _stale(LIB, _sources()):
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for unit, flags in UNITS.items():
            obj = os.path.join(objdir, unit.replace(".cu", ".o"))
            cmd = ["nvcc", *COMMON, *flags, "-c", "-o", obj, os.path.join(CSRC, unit)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(obj)
        cmd = ["nvcc", *ARCH, "-shared", "-o", LIB + ".tmp", *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


DRIVER_SRC = os.path.join(HERE, "driver", "cumc_main.c")
DRIVER = os.path.join(HERE, "driver", "cumc_main")
# the C caller is plain C99 and must build warning-free against include/cumc.h
DRIVER_FLAGS = ["-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-pedantic"]


def build_driver(force: bool = False) -> str:
    """Compile the C program that drives the library with the reference main
    program's call sequence (cumpic_b200/driver/cumc_main.c) and link it
    against libcumc_b200.so."""
    lib = build_library()
    if force or _stale(DRIVER, [DRIVER_SRC, lib, os.path.join(ROOT, "include", "cumc.h")]):
        cmd = ["gcc", *DRIVER_FLAGS, "-o", DRIVER + ".tmp", DRIVER_SRC, "-L" + HERE, "-lcumc_b200",
               "-Wl,-rpath,$ORIGIN/.."]
        subprocess.run(cmd, check=True)
        os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


def build_oracle(force: bool = False) -> str:
    """Compile the FP64 CPU oracle (test infrastructure) via oracle/Makefile,
    and, where the reference sources are present, the mechanical translation
    of the reference into oracle/_ref/ (the oracle's own checker)."""
    args = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)
    # the reference's source tree: CUMC_REFERENCE, else the recipe's default
    override = [f"REFERENCE={os.environ['CUMC_REFERENCE']}"] if os.environ.get("CUMC_REFERENCE") else []
    reference = subprocess.run(args + ["print-reference", *override], check=True, capture_output=True,
                               text=True).stdout.strip()
    if reference and os.path.isdir(os.path.join(reference, "solver")):
        subprocess.run(args + ["ref", f"REFERENCE={reference}"], check=True)
    return os.path.join(ROOT, "oracle", "build", "libcumc_oracle.so")


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
    print(build_driver(force=True))
    print(build_oracle())
