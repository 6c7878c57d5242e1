"""Where the reference checkout lies on this machine -- for the recipes that
read its sources (oracle/build_ref.py, the golden-fixture generators under
tests/golden/).  No committed file names the path: it is $CMF_REFERENCE_ROOT,
else the first line of oracle/_ref/REFERENCE_ROOT (a local setting, not
committed; oracle/_ref/ is git-ignored).  None when neither names an existing
directory, as on a machine without the reference."""
from __future__ import annotations

import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
SETTING = HERE / "_ref" / "REFERENCE_ROOT"


def reference_root() -> Path | None:
    p = os.environ.get("CMF_REFERENCE_ROOT")
    if not p and SETTING.exists():
        lines = SETTING.read_text().strip().splitlines()
        p = lines[0].strip() if lines else ""
    if p and Path(p).is_dir():
        return Path(p)
    return None
