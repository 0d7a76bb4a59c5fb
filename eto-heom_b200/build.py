"""Build libheom.so (C ABI + sm_100a kernels) and the heom_2des / heom_scan / heom_dynamics CLIs in-tree.

    python eto-heom_b200/build.py [--force]

Host C++ is compiled with -ffp-contract=off: the problem set-up (Hamiltonian sort,
orientation, coupling coefficients, pulse fields) must round exactly as the reference
does.  The bit-exact FP64 kernels are compiled with --fmad=false as a second guard
(they already use explicit __dmul_rn / __dadd_rn).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libheom.so")
CLIS = [(os.path.join(SRC, "heom_2des.cpp"), os.path.join(PKG, "heom_2des")),
        (os.path.join(SRC, "heom_scan.cpp"), os.path.join(PKG, "heom_scan")),
        (os.path.join(SRC, "heom_dynamics.cpp"), os.path.join(PKG, "heom_dynamics"))]

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOSTFLAGS = "-fPIC,-ffp-contract=off,-fno-fast-math,-Wall,-Wno-unused-function"
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", HOSTFLAGS, "-I" + os.path.join(ROOT, "include")]

UNITS = [
    ("problem.cpp", []),
    ("plan.cu", []),
    ("exact.cu", ["--fmad=false"]),
    ("scan.cu", ["-Xptxas", "-warn-spills"]),
    ("peak.cu", []),
    ("noalloc.cu", []),
    ("sg.cu", []),
    ("adjoint.cu", []),
]
HEADERS = ["heom_host.h", "kernels.h", "exact.cuh", "scan.h", "scan_pm.cuh", "scan_slots.cuh", "sg.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "heom.h")]
    objs = []
    for name, extra in UNITS:
        src = os.path.join(SRC, name)
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + hdrs + [__file__]):
            flags = list(extra)
            if verbose_ptxas and name.endswith(".cu"):
                flags += ["-Xptxas", "-v"]
            _run([NVCC, *ARCH, *COMMON, *flags, "-c", src, "-o", obj])
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    for cli_src, cli in CLIS:
        if force or _newer(cli, [cli_src, LIB, os.path.join(ROOT, "include", "heom.h")]):
            _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-Wall", "-I" + os.path.join(ROOT, "include"),
                  cli_src, "-o", cli, "-L" + PKG, "-lheom", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
