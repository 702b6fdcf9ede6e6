"""Loading of the golden fixtures recorded from the reference (tests/golden)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def fixture_names() -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.endswith("_summary"))


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def slices(offsets: np.ndarray, ids: np.ndarray):
    off = offsets.astype(np.int64)
    return [ids[off[j]:off[j + 1]] for j in range(len(off) - 1)]
