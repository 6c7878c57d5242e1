"""Golden fixtures from the REFERENCE's own CUDA kernels (run on a B200).

    python tests/golden/make_ref_golden.py [out_dir]

Uses oracle/_ref (the reference cmfgpu/phys/cuda launchers compiled unmodified
for sm_100a by oracle/build_ref.py) through oracle/ref_cuda.py.  For each
feature case a small seeded network is routed for one simulated day from the
generator's cold state (state S1 is saved), then the CFL sub-step count of the
next day and ONE sub-step are run (n, dt and state S2 are saved).  The
fixtures pin the CPU oracle (tests/test_oracle_golden.py) and the CUDA product
(tests/test_gpu_golden.py) against the reference itself.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cama-flood-gpu_b200"))
sys.path.insert(0, str(ROOT / "tests"))

from cmfb200 import synthetic as syn  # noqa: E402
from oracle import oracle as O, ref_cuda as RC  # noqa: E402

import golden_cases as G  # noqa: E402


def main(out_dir: Path) -> None:
    import torch
    for case, spec in G.CASES.items():
        net = syn.generate(spec)
        fields = O.reference_fields(net.fields, net.opened_modules)
        ref = RC.RefCuda(fields, net.opened_modules)
        ref.set_runoff(syn.daily_runoff(net, 0))
        ref.step_advance(86400.0)
        s1 = ref.state()
        ref.set_runoff(syn.daily_runoff(net, 1))
        n = ref.adaptive_sub_steps(86400.0)
        ref.t["time_step"].fill_(86400.0 / n)
        ref.substep()
        torch.cuda.synchronize()
        s2 = ref.state()
        out = {"n": np.int32(n), "dt": np.float32(s2["time_step"][0])}
        for k in G.state_fields(net.opened_modules):
            out["in_" + k] = s1[k]
            out["out_" + k] = s2[k]
        for k in G.diag_fields(net.opened_modules):
            out["out_" + k] = s2[k]
        path = out_dir / f"ref_{case}.npz"
        np.savez_compressed(path, **out)
        print(case, "n", n, path, path.stat().st_size, flush=True)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE)
