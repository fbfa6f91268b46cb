"""Generates the committed golden vectors under tests/golden/ from the
reference's own code compiled host-side (oracle/_ref, built by
`make -C oracle`). Run from the repository root:
    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

from oracle_lib import RefLib, _np_ptr  # noqa: E402


def sobol(ref: RefLib):
    rng = np.random.default_rng(2024)
    n = 512
    sample = np.concatenate([np.arange(128, dtype=np.uint32), rng.integers(0, 1 << 24, n - 128, dtype=np.uint32)])
    h = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    bounce = rng.integers(0, 16, n, dtype=np.uint32)
    dim = rng.integers(0, 9, n, dtype=np.uint32)
    out = {}
    for dims in (1, 2, 3):
        o = np.zeros(n * dims, np.float32)
        ref.lib.rbref_sobol(n, dims, _np_ptr(sample), _np_ptr(h), _np_ptr(bounce), _np_ptr(dim), _np_ptr(o))
        out[f"out{dims}"] = o
    np.savez_compressed(HERE / "sobol.npz", sample=sample, hash=h, bounce=bounce, dim=dim, **out)


if __name__ == "__main__":
    ref = RefLib()
    sobol(ref)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))
