"""Compile the reference CUDA launchers into oracle/_ref (test oracle only).

    python oracle/build_ref.py

Reads the reference sources where they lie (cmfgpu/phys/cuda under the
checkout that oracle/refroot.py locates) -- nothing is copied into this
repository -- and
links them with oracle/ref_binding.cpp into oracle/_ref/cmf_refcuda*.so for
sm_100a.  The output directory is git-ignored; the built module travels to the
GPU box with the rest of the tree.  Skips (returns None) when the reference
tree is absent, e.g. on the GPU box, which only uses the prebuilt module.
"""
from __future__ import annotations

import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
try:
    from .refroot import reference_root
except ImportError:                      # run as a script
    sys.path.insert(0, str(HERE))
    from refroot import reference_root
_ROOT = reference_root()
REF = (_ROOT / "cmfgpu" / "phys" / "cuda") if _ROOT else HERE / "_ref" / "no-reference-checkout"
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
