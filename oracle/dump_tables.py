"""Oracle build step (test infrastructure): writes the reference's spectral
tables as plain data next to its LUT files, so that a process can read the
reference's inputs without loading any oracle library.

    python oracle/dump_tables.py oracle/_ref

reads the CIE 1931 XYZ curves and the RGB basis spectra from the compiled
reference (src/core/spectral.cpp through oracle/_ref/libratbite_ref.so) and
writes oracle/_ref/bin/spectra.npz with arrays `cie_xyz` and `basis_rgb`
(3 x 471 float32 each, 360-830 nm at 1 nm).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent / "tests"))


def main(out_dir: str) -> None:
    from oracle_lib import RefLib
    ref = RefLib(Path(out_dir) / "libratbite_ref.so")
    dst = Path(out_dir) / "bin" / "spectra.npz"
    dst.parent.mkdir(parents=True, exist_ok=True)
    np.savez(dst, cie_xyz=ref.cie_xyz(), basis_rgb=ref.basis_rgb())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(HERE / "_ref"))
