"""Generates tests/golden/tiles_ref.npz by running the reference's own CPU
code (Tile_create and blockspmv_cpu compiled unmodified into
oracle/_ref/libmfref.so) on small seeded matrices.

Run from the repository root in a checkout that has the reference tree and
has built oracle/ (make -C oracle):  python tests/golden/make_golden.py
The inputs are stored next to the outputs, so the fixtures pin the oracle
without the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import _oracle as O  # noqa: E402


def poisson2d(N):
    rp = [0]
    ci, va = [], []
    for j in range(N):
        for i in range(N):
            r = i + N * j
            ent = []
            if j > 0: ent.append((r - N, -1.0))
            if i > 0: ent.append((r - 1, -1.0))
            ent.append((r, 4.0))
            if i < N - 1: ent.append((r + 1, -1.0))
            if j < N - 1: ent.append((r + N, -1.0))
            for c, v in ent:
                ci.append(c)
                va.append(v)
            rp.append(len(ci))
    return N * N, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va)


def random_csr(n, per_row, seed, unsorted=True, dense_row=None):
    rng = np.random.default_rng(seed)
    rp = [0]
    ci, va = [], []
    for r in range(n):
        k = int(rng.integers(0, per_row + 1))
        cols = set(rng.integers(0, n, size=k).tolist())
        cols.add(r)
        if dense_row is not None and r == dense_row:
            cols |= set(range(0, n, 1))
        cols = sorted(cols)
        if unsorted:
            rng.shuffle(cols)
        for c in cols:
            ci.append(c)
            va.append(float(rng.standard_normal()))
        rp.append(len(ci))
    return n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va)


CASES = {
    "poisson2d_32": lambda: (*poisson2d(32), None),
    "random_300_unsorted": lambda: (*random_csr(300, 12, 1), None),
    "random_257_odd": lambda: (*random_csr(257, 6, 2), None),
    "random_33_rowlen1": lambda: (*random_csr(33, 8, 3), None),
    "random_241_truncated_225": lambda: (*random_csr(241, 6, 4), 225),
    "dense_row_96": lambda: (*random_csr(96, 4, 5, dense_row=40), None),
}


def main():
    out = {}
    for name, make in CASES.items():
        n, rp, ci, va, rowA = make()
        rowA = n if rowA is None else rowA
        r = O.RefTiles(rowA, n, rp, ci, va)
        arrays = r.arrays()  # before the SpMV fills the nibble column array
        x = np.random.default_rng(7).standard_normal(n)
        y, p1, p2, rbb = r.spmv(x)
        out[f"{name}/rowA"] = np.array([rowA, n])
        out[f"{name}/row_ptr"] = rp
        out[f"{name}/col_idx"] = ci
        out[f"{name}/val"] = va
        out[f"{name}/x"] = x
        out[f"{name}/y"] = y
        out[f"{name}/ptroffset1"] = p1
        out[f"{name}/ptroffset2"] = p2
        out[f"{name}/rowblkblock"] = np.array([rbb])
        for k, v in arrays.items():
            out[f"{name}/{k}"] = v
        print(name, rowA, r.sizes["tilenum"])
    np.savez_compressed(os.path.join(HERE, "tiles_ref.npz"), **out)


if __name__ == "__main__":
    main()
