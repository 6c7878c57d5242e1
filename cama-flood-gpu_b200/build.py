"""Build libcmfb200.so (sm_100a) in-tree.

    python cama-flood-gpu_b200/build.py [--force]

Compiles the CUDA kernels, the C-ABI plan code and the host topology helpers
with nvcc for `-gencode arch=compute_100a,code=sm_100a` into
cama-flood-gpu_b200/cmfb200/lib/libcmfb200.so.  The CUDA runtime is linked
statically, so the library needs only the NVIDIA driver at run time.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
OUT_DIR = HERE / "cmfb200" / "lib"
OUT = OUT_DIR / "libcmfb200.so"
SOURCES = [CSRC / "cmf_plan.cu", CSRC / "cmf_adjoint.cu", CSRC / "cmf_forcing.cu", CSRC / "cmf_topology.cpp"]
DEPS = SOURCES + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "cmfb200.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    return any(p.stat().st_mtime > t for p in DEPS)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and not needs_build():
        return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    cmd = [
        nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
        "-Xcompiler", "-fPIC,-O2", "-shared", "-cudart", "static",
        f"-I{INCLUDE}", f"-I{CSRC}",
        *[str(s) for s in SOURCES],
        "-o", str(OUT),
    ]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = []
    if "--ptxas-v" in args:
        extra = ["-Xptxas", "-v"]
    build(force="--force" in args or bool(extra), verbose=True, extra=extra)
    print(OUT)
