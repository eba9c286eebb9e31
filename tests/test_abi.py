"""CPU tests of the C ABI library: it loads, exports every declared entry
point, and its host-side code (generators, readers, writers) is right."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "mf.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text))
    return {n for n in names if n.startswith("mf_") or n in ("cg_solve_inc", "bicgstab")} - {"mf_"}


def test_library_exports_every_declared_symbol(mf):
    L = mf.lib()
    declared = _declared_functions()
    assert len(declared) >= 35
    for name in sorted(declared):
        assert hasattr(L, name), name
    assert set(mf.EXPORTED) <= declared


def test_generator_sizes(mf):
    A = mf.Matrix.poisson2d(256)
    assert A.info()[:3] == (65536, 65536, 326656)
    B = mf.Matrix.convdiff3d(16)
    n, nc, nnz, hb, _ = B.info()
    assert (n, nnz) == (4096, 7 * 4096 - 6 * 256) and hb
    C = mf.Matrix.varpoisson3d(8)
    n, _, nnz, hb, hx = C.info()
    assert n == 512 and nnz == 7 * 512 - 6 * 64 and hb and hx


def test_varpoisson_is_symmetric_diagonally_dominant(mf):
    import scipy.sparse as sp

    A = mf.Matrix.varpoisson3d(10, seed=3)
    rp, ci, v = A.csr()
    M = sp.csr_matrix((v, ci, rp), shape=(1000, 1000))
    assert abs(M - M.T).max() == 0
    d = M.diagonal()
    off = np.asarray(abs(M).sum(axis=1)).ravel() - d
    assert np.all(d >= off - 1e-12)
    b = A.b()
    assert np.allclose(M @ A.xstar(), b, rtol=1e-14, atol=1e-12)
    assert np.all((v[ci == np.repeat(np.arange(1000), np.diff(rp))] > 0))


def test_convdiff_coefficients(mf):
    A = mf.Matrix.convdiff3d(4)
    rp, ci, v = A.csr()
    # interior cell (1,1,1): index 1 + 4 + 16 = 21
    r = 21
    row = dict(zip(ci[rp[r]:rp[r + 1]], v[rp[r]:rp[r + 1]]))
    assert row == {21 - 16: -1.25, 21 - 4: -1.5, 20: -2.0, 21: 7.75, 22: -1.0, 25: -1.0, 37: -1.0}


def test_spd_random_is_spd(mf):
    import scipy.sparse as sp

    A = mf.Matrix.spd_random(800, 11)
    rp, ci, v = A.csr()
    M = sp.csr_matrix((v, ci, rp), shape=(800, 800))
    assert abs(M - M.T).max() < 1e-15
    w = np.linalg.eigvalsh(M.toarray())
    assert w.min() > 0
    assert np.all(np.diff(ci[rp[0]:rp[1]]) > 0)


def test_batch_sizes(mf):
    s = mf.batch_sizes(512, 1000, 200000, 2)
    assert s.min() >= 1000 and s.max() <= 200000
    assert 20000 < s.mean() < 60000


def test_mtx_reader_expands_symmetric_in_file_order(mf, tmp_path):
    p = tmp_path / "a.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% c\n3 3 4\n1 1 2.0\n2 1 -1.0\n3 2 -0.5\n3 3 4.0\n")
    n, nc, rp, ci, v = mf.read_Dmatrix_32(str(p))
    assert (n, nc) == (3, 3)
    assert list(rp) == [0, 2, 4, 6]
    assert list(ci) == [0, 1, 0, 2, 1, 2]
    assert list(v) == [2.0, -1.0, -1.0, -0.5, -0.5, 4.0]


def test_mtx_reader_pattern_and_general(mf, tmp_path):
    p = tmp_path / "b.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n2 3 3\n2 3\n1 1\n2 1\n")
    n, nc, rp, ci, v = mf.read_Dmatrix_32(str(p))
    assert (n, nc) == (2, 3) and list(rp) == [0, 1, 3] and list(ci) == [0, 2, 0] and list(v) == [1.0] * 3


def test_mtx_reader_matches_reference_reader(mf, O):
    if not O.ref_available() or O.ref_tree() is None:
        pytest.skip("reference harness not built, or its source tree absent")
    base = os.path.join(O.ref_tree(), "ginkgo-develop", "matrices", "test")
    files = [f for f in ("1138_bus.mtx", "ani1.mtx", "ani1_nonsymm.mtx", "isai_spd.mtx") if os.path.exists(os.path.join(base, f))]
    if not files:
        pytest.skip("reference matrices absent")
    for f in files:
        path = os.path.join(base, f)
        m, n, rp, ci, v = O.ref_read_mtx(path)
        mm, nn, rp2, ci2, v2 = mf.read_Dmatrix_32(path)
        assert (m, n) == (mm, nn), f
        assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2), f


def test_cbd_roundtrip(mf, tmp_path):
    A = mf.Matrix.convdiff3d(6)
    p = str(tmp_path / "a.cbd")
    A.write_cbd(p)
    B = mf.Matrix.read_cbd(p)
    for a, b in zip(A.csr(), B.csr()):
        assert np.array_equal(a, b)
    raw = open(p, "rb").read()
    rows, cols = np.frombuffer(raw[:8], np.int32)
    nnz = np.frombuffer(raw[8:16], np.int64)[0]
    assert (rows, cols, nnz) == (216, 216, A.nnz)
    assert len(raw) == 16 + 8 * 217 + 4 * nnz + 8 * nnz


def test_cbd_against_the_reference_biio(mf, O, tmp_path):
    """A .cbd written here reads back through the reference's own
    binary_read_csr (biio.h:22-72), and one written by its binary_write_csr
    (biio.h:74-97) reads back here: same sizes, row pointers, columns and
    values, and byte-identical files."""
    if not O.ref_available():
        pytest.skip("reference harness not built")
    A = mf.Matrix.varpoisson3d(7)
    rp, ci, v = A.csr()
    ours = str(tmp_path / "ours.cbd")
    A.write_cbd(ours)
    m, n, rp2, ci2, v2 = O.ref_read_cbd(ours)
    assert (m, n) == (A.n, A.n)
    assert np.array_equal(rp2, rp.astype(np.int64)) and np.array_equal(ci2, ci) and np.array_equal(v2, v)
    theirs = str(tmp_path / "theirs.cbd")
    O.ref_write_cbd(theirs, A.n, A.n, rp, ci, v)
    B = mf.Matrix.read_cbd(theirs)
    for a, b in zip(A.csr(), B.csr()):
        assert np.array_equal(a, b)
    assert open(ours, "rb").read() == open(theirs, "rb").read()


def test_errors_are_status_codes(mf):
    h = mf._p()
    assert mf.lib().mf_gen_poisson2d(0, mf.C.byref(h)) == mf.MF_ERR_ARG
    assert mf.lib().mf_read_mtx(b"/nonexistent.mtx", mf.C.byref(h)) == mf.MF_ERR_IO
    assert mf.lib().mf_status_str(mf.MF_ERR_TIMEOUT) == b"device wait timed out"
