"""Compile the reference CUDA launchers into oracle/_ref (test oracle only).

    python oracle/build_ref.py

Reads the reference sources where they lie (/root/reference/cmfgpu/phys/cuda,
or $CMF_REFERENCE_ROOT) -- nothing is copied into this repository -- and
links them with oracle/ref_binding.cpp into oracle/_ref/cmf_refcuda*.so for
sm_100a.  The output directory is git-ignored; the built module travels to the
GPU box with the rest of the tree.  Skips (returns None) when the reference
tree is absent, e.g. on the GPU box, which only uses the prebuilt module.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF = Path(os.environ.get("CMF_REFERENCE_ROOT", "/root/reference")) / "cmfgpu" / "phys" / "cuda"
UNITS = ("outflow.cu", "storage.cu", "adaptive_time.cu", "bifurcation.cu", "reservoir.cu", "levee.cu")


def built_module() -> Path | None:
    hits = sorted(OUT.glob("cmf_refcuda*.so"))
    return hits[0] if hits else None


def build(force: bool = False) -> Path | None:
    if not REF.exists():
        return built_module()
    sources = [HERE / "ref_binding.cpp"] + [REF / u for u in UNITS]
    mod = built_module()
    if mod and not force and all(s.stat().st_mtime <= mod.stat().st_mtime for s in sources):
        return mod
    OUT.mkdir(exist_ok=True)
    from torch.utils.cpp_extension import load
    load(
        name="cmf_refcuda",
        sources=[str(s) for s in sources],
        build_directory=str(OUT),
        extra_cflags=["-O2"],
        extra_cuda_cflags=["-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                           f"-I{REF}"],
        verbose=False,
        is_python_module=True,
    )
    return built_module()


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
