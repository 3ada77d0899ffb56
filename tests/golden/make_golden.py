"""Regenerates the golden fixtures under tests/golden/ from the reference tree.

dense_lattice_5x5x10.npz - the reference's own DenseLattice fixtures
    src/tests/DenseLattice/data/test1.bin, test2.bin and multtest_ddd.bin
    (DenseLattice::save format, DenseLattice.h:270, 396: a header of three
    float64 values h, w, d, then h*w*d float64 values, column-major per tab).
    denselatticemulttests.cpp:19-49 checks multtest_ddd = test1 * test2 tab by
    tab; the fixtures are stored here as the arrays A, B, C (shape h*w*d flat).

Usage: python tests/golden/make_golden.py [reference_root]
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def read_bin(path: Path):
    raw = np.fromfile(path, dtype=np.float64)
    h, w, d = (int(x) for x in raw[:3])
    data = raw[3:]
    assert data.size == h * w * d, (path, h, w, d, data.size)
    return (h, w, d), data


def main(ref_root: str = "/root/reference"):
    data_dir = Path(ref_root) / "src" / "tests" / "DenseLattice" / "data"
    (h, w, d), A = read_bin(data_dir / "test1.bin")
    (w2, wB, d2), B = read_bin(data_dir / "test2.bin")
    (h3, wB3, d3), Cm = read_bin(data_dir / "multtest_ddd.bin")
    assert (w2, d2) == (w, d) and (h3, wB3, d3) == (h, wB, d)
    np.savez(HERE / "dense_lattice_5x5x10.npz", A=A, B=B, C=Cm, shape=np.array([h, w, wB, d], np.int64))
    print("wrote", HERE / "dense_lattice_5x5x10.npz", (h, w, wB, d))


if __name__ == "__main__":
    main(*sys.argv[1:])
