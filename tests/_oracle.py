"""ctypes bindings of the CPU oracle (oracle/liboracle.so) and of the
reference's own CPU code compiled unmodified (oracle/_ref/libmfref.so).

Test infrastructure only: the product (libmf.so) never loads these.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libmfref.so")

_i = C.c_int
_p = C.c_void_p


class MfoTiles(C.Structure):
    _fields_ = [(n, _i) for n in ("rowA", "colA", "tilem", "tilen", "tilenum", "csrsize", "csrptrlen")] + [
        (n, C.POINTER(C.c_int)) for n in ("tile_ptr", "tile_columnidx", "tile_nnz", "blknnz", "csr_offset", "csrptr_offset")
    ] + [
        ("Format", C.POINTER(C.c_char)),
        ("blknnznnz", C.POINTER(C.c_ubyte)),
        ("Blockcsr_Val", C.POINTER(C.c_double)),
        ("Blockcsr_Val_Low", C.POINTER(C.c_float)),
        ("Tile_csr_Col", C.POINTER(C.c_ubyte)),
        ("Blockcsr_Ptr", C.POINTER(C.c_ubyte)),
        ("csr_compressedIdx", C.POINTER(C.c_ubyte)),
    ]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(ORACLE_SO)
        L = _lib
        L.mfo_tile_create.argtypes = [_i, _i, _p, _p, _p, C.POINTER(MfoTiles)]
        L.mfo_set_threads.argtypes = [_i]
        L.mfo_set_threads.restype = _i
        L.mfo_tiles_free.argtypes = [C.POINTER(MfoTiles)]
        L.mfo_blockspmv.argtypes = [C.POINTER(MfoTiles), _p, _p, _p, _p, _p]
        L.mfo_row_compress.argtypes = [C.POINTER(MfoTiles), _p, _p, _p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.mfo_row_compress.restype = _i
        L.mfo_balance_twopointer.argtypes = [C.POINTER(MfoTiles), _i, _i, _p, _p, _p, _p]
        L.mfo_balance_twopointer.restype = _i
        L.mfo_csr_spmv.argtypes = [_i, _p, _p, _p, _p, _p]
        L.mfo_dot.argtypes = [_i, _p, _p]
        L.mfo_dot.restype = C.c_double
        L.mfo_cg.argtypes = [C.POINTER(MfoTiles), _p, _p, C.c_double, _i, C.POINTER(C.c_double)]
        L.mfo_cg.restype = _i
        L.mfo_cg_dir32.argtypes = [C.POINTER(MfoTiles), _p, _p, C.c_double, _i, _i, C.POINTER(C.c_double)]
        L.mfo_cg_dir32.restype = _i
        L.mfo_pcg_jacobi.argtypes = [C.POINTER(MfoTiles), _p, _p, _p, C.c_double, _i, C.POINTER(C.c_double)]
        L.mfo_pcg_jacobi.restype = _i
        L.mfo_bicgstab.argtypes = [C.POINTER(MfoTiles), _p, _p, C.c_double, _i, C.POINTER(C.c_double)]
        L.mfo_bicgstab.restype = _i
        L.mfo_fp8_e4m3_encode.argtypes = [C.c_double]
        L.mfo_fp8_e4m3_encode.restype = C.c_uint8
        L.mfo_fp8_e4m3_decode.argtypes = [C.c_uint8]
        L.mfo_fp8_e4m3_decode.restype = C.c_double
        L.mfo_fp16_encode.argtypes = [C.c_double]
        L.mfo_fp16_encode.restype = C.c_uint16
        L.mfo_fp16_decode.argtypes = [C.c_uint16]
        L.mfo_fp16_decode.restype = C.c_double
        L.mfo_tile_scale.argtypes = [_i, C.c_double]
        L.mfo_tile_scale.restype = C.c_double
        L.mfo_mixed_spmv.argtypes = [C.POINTER(MfoTiles), _p, _p, _p]
        L.mfo_mlp_forward.argtypes = [_p] * 7 + [_i, _p]
        L.mfo_mlp_forward.restype = C.c_float
        L.mfo_mlp_grad.argtypes = [_p] * 8 + [_i] + [_p] * 6
        L.mfo_mlp_grad.restype = C.c_float
        L.mfo_gen_poisson2d.argtypes = [_i, C.POINTER(MfoSystem)]
        L.mfo_gen_convdiff3d.argtypes = [_i, C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(MfoSystem)]
        L.mfo_gen_varpoisson3d.argtypes = [_i, C.c_double, C.c_double, C.c_uint64, C.POINTER(MfoSystem)]
        for f in ("mfo_gen_poisson2d", "mfo_gen_convdiff3d", "mfo_gen_varpoisson3d"):
            getattr(L, f).restype = _i
        L.mfo_system_free.argtypes = [C.POINTER(MfoSystem)]
    return _lib


class MfoSystem(C.Structure):
    _fields_ = [("n", _i), ("nnz", _i), ("row_ptr", C.POINTER(C.c_int)), ("col_idx", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_double)), ("b", C.POINTER(C.c_double)), ("xstar", C.POINTER(C.c_double))]


class System:
    """A synthetic workload generated by the oracle (oracle/workloads.c):
    n, CSR (rp, ci, v), b and x* (None where the workload has none)."""

    def __init__(self, fn, *args):
        m = MfoSystem()
        rc = getattr(lib(), fn)(*args, C.byref(m))
        if rc != 0:
            raise ValueError(f"{fn}{args}: bad arguments")
        try:
            n, nnz = m.n, m.nnz
            self.n = n
            self.rp = np.ctypeslib.as_array(m.row_ptr, shape=(n + 1,)).copy()
            self.ci = np.ctypeslib.as_array(m.col_idx, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
            self.v = np.ctypeslib.as_array(m.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
            self.b = np.ctypeslib.as_array(m.b, shape=(n,)).copy()
            self.xstar = np.ctypeslib.as_array(m.xstar, shape=(n,)).copy() if m.xstar else None
        finally:
            lib().mfo_system_free(C.byref(m))

    def csr(self):
        return self.rp, self.ci, self.v


def gen_poisson2d(N):
    """2D 5-point Laplacian, N x N grid, b = A * ones."""
    return System("mfo_gen_poisson2d", N)


def gen_convdiff3d(N, v=(1.0, 0.5, 0.25), seed=0):
    """3D 7-point upwind convection-diffusion, N^3 grid, b ~ U[-1, 1]."""
    return System("mfo_gen_convdiff3d", N, v[0], v[1], v[2], seed)


def gen_varpoisson3d(N, klo=1e-3, khi=1e3, seed=1):
    """3D 7-point variable-coefficient Poisson, N^3 grid, faces logU[klo, khi],
    b = A x*, x* ~ U[0, 1]."""
    return System("mfo_gen_varpoisson3d", N, klo, khi, seed)


# MLP weight blocks inside the packed weight vector: W1[64][6], b1[64],
# W2[64][64], b2[64], W3[4][64], b3[4]
_MLP_BLOCKS = [(0, 384), (384, 448), (448, 4544), (4544, 4608), (4608, 4864), (4864, 4868)]


def mlp_forward(w, x):
    """Logits (n, 4) of the oracle's FP32 MLP for packed weights w."""
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    n = x.shape[0]
    out = np.zeros((n, 4), np.float32)
    parts = [w[a:b] for a, b in _MLP_BLOCKS]
    lib().mfo_mlp_forward(*[_ptr(q) for q in parts], _ptr(x), n, _ptr(out))
    return out


def mlp_grad(w, x, labels):
    """(packed gradient, loss) of the mean softmax cross-entropy."""
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(labels, np.int32)
    parts = [w[a:b] for a, b in _MLP_BLOCKS]
    g = np.zeros_like(w)
    gparts = [g[a:b] for a, b in _MLP_BLOCKS]
    loss = lib().mfo_mlp_grad(*[_ptr(q) for q in parts], _ptr(x), _ptr(y), x.shape[0], *[_ptr(q) for q in gparts])
    return g, float(loss)


def ref_available():
    return os.path.exists(REF_SO)


def ref_tree():
    """The reference's Performance-Comparison directory the harness was built
    from (recorded by oracle/Makefile), or None where it is absent."""
    try:
        with open(os.path.join(ROOT, "oracle", "_ref", "ref_dir.txt")) as f:
            d = f.read().strip()
        return d if os.path.isdir(d) else None
    except OSError:
        return None


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        R = _ref
        R.ref_tile_create.argtypes = [_i, _i, _i, _p, _p, _p]
        R.ref_tile_create.restype = _p
        R.ref_tile_sizes.argtypes = [_p, _p]
        R.ref_tile_array.argtypes = [_p, C.c_char_p, _p]
        R.ref_tile_array.restype = _i
        R.ref_blockspmv.argtypes = [_p, _p, _p, _p, _p, _p, _i]
        R.ref_tile_free.argtypes = [_p]
        R.ref_read_mtx.argtypes = [C.c_char_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i),
                                   C.POINTER(C.POINTER(_i)), C.POINTER(C.POINTER(_i)), C.POINTER(C.POINTER(C.c_double))]
        R.ref_read_mtx.restype = _i
        R.ref_free.argtypes = [_p]
        R.ref_read_cbd.argtypes = [C.c_char_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(C.c_int64),
                                   C.POINTER(C.POINTER(C.c_int64)), C.POINTER(C.POINTER(_i)),
                                   C.POINTER(C.POINTER(C.c_double))]
        R.ref_read_cbd.restype = _i
        R.ref_write_cbd.argtypes = [C.c_char_p, _i, _i, C.c_int64, _p, _p, _p]
    return _ref


ARRAY_SPECS = {
    # name: (dtype, length key)
    "tile_ptr": (np.int32, "tilem+1"),
    "tile_columnidx": (np.int32, "tilenum"),
    "tile_nnz": (np.int32, "tilenum+1"),
    "blknnz": (np.int32, "tilenum+1"),
    "csr_offset": (np.int32, "tilenum+1"),
    "csrptr_offset": (np.int32, "tilenum+1"),
    "Format": (np.int8, "tilenum"),
    "blknnznnz": (np.uint8, "tilenum+1"),
    "Blockcsr_Val": (np.float64, "csrsize"),
    "Blockcsr_Val_Low": (np.float32, "csrsize"),
    "Tile_csr_Col": (np.uint8, "csrsize"),
    "Blockcsr_Ptr": (np.uint8, "csrptrlen"),
    "csr_compressedIdx": (np.uint8, "csrhalf"),
}


def _length(key, s):
    return {
        "tilem+1": s["tilem"] + 1,
        "tilenum": s["tilenum"],
        "tilenum+1": s["tilenum"] + 1,
        "csrsize": s["csrsize"],
        "csrptrlen": s["csrptrlen"],
        "csrhalf": (s["csrsize"] + 1) // 2,
    }[key]


class OracleTiles:
    """Tile_create restated by the oracle (mfo_tile_create)."""

    def __init__(self, rowA, colA, rp, ci, val):
        self.rp = np.ascontiguousarray(rp, np.int32)
        self.ci = np.ascontiguousarray(ci, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        self.t = MfoTiles()
        rc = lib().mfo_tile_create(rowA, colA, _ptr(self.rp), _ptr(self.ci), _ptr(self.val), C.byref(self.t))
        assert rc == 0
        self.sizes = {k: getattr(self.t, k) for k in ("rowA", "colA", "tilem", "tilen", "tilenum", "csrsize", "csrptrlen")}

    def array(self, name):
        dt, key = ARRAY_SPECS[name]
        n = _length(key, self.sizes)
        p = getattr(self.t, name)
        raw = C.cast(p, C.POINTER(C.c_ubyte))
        buf = C.string_at(raw, n * np.dtype(dt).itemsize) if n > 0 else b""
        return np.frombuffer(buf, dtype=dt).copy()

    def arrays(self):
        return {k: self.array(k) for k in ARRAY_SPECS}

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.sizes["rowA"], np.float64)
        lib().mfo_blockspmv(C.byref(self.t), _ptr(x), _ptr(y), None, None, None)
        return y

    def offsets(self):
        n = self.sizes["tilenum"]
        p1 = np.zeros(max(n, 1), np.int32)
        p2 = np.zeros(max(n, 1), np.int32)
        rbb = np.zeros(1, np.int32)
        lib().mfo_blockspmv(C.byref(self.t), None, None, _ptr(p1), _ptr(p2), _ptr(rbb))
        return p1[:n], p2[:n], int(rbb[0])

    def mixed_spmv(self, prec, x):
        x = np.ascontiguousarray(x, np.float64)
        prec = np.ascontiguousarray(prec, np.uint8)
        y = np.zeros(self.sizes["rowA"], np.float64)
        lib().mfo_mixed_spmv(C.byref(self.t), _ptr(prec), _ptr(x), _ptr(y))
        return y

    def row_compress(self):
        s = self.sizes
        nz = np.zeros(s["tilenum"] + 1, np.int32)
        tr = np.zeros(max(s["tilenum"], 1), np.int32)
        bs = np.zeros(s["tilem"] + 1, np.int32)
        a = C.c_void_p()
        b = C.c_void_p()
        cnt = lib().mfo_row_compress(C.byref(self.t), _ptr(nz), _ptr(tr), _ptr(bs), C.byref(a), C.byref(b))
        rid = np.frombuffer(C.string_at(a, cnt + 1), np.uint8).copy()
        rpn = np.frombuffer(C.string_at(b, cnt + 1), np.uint8).copy()
        C.CDLL(None).free.argtypes = [_p]
        C.CDLL(None).free(a)
        C.CDLL(None).free(b)
        return dict(nonzero_row_new=nz, tile_rowidx=tr[: s["tilenum"]], block_signal=bs,
                    blockrowid_new=rid, blockcsr_ptr_new=rpn)

    def balance(self, block_nnz, block_per_warp=180):
        n = self.sizes["tilenum"]
        idx = lib().mfo_balance_twopointer(C.byref(self.t), block_nnz, block_per_warp, None, None, None, None)
        bp = np.zeros(idx + 1, np.int32)
        a = np.zeros(n + 1, np.int32)
        b = np.zeros(n + 1, np.int32)
        c = np.zeros(n + 1, np.int32)
        idx2 = lib().mfo_balance_twopointer(C.byref(self.t), block_nnz, block_per_warp, _ptr(bp), _ptr(a), _ptr(b), _ptr(c))
        assert idx2 == idx
        return idx, bp, a, b, c

    def cg(self, b, tol, maxiter, x0=None):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.sizes["rowA"]) if x0 is None else np.array(x0, np.float64)
        rel = C.c_double()
        it = lib().mfo_cg(C.byref(self.t), _ptr(b), _ptr(x), tol, maxiter, C.byref(rel))
        return it, x, rel.value

    def cg_dir32(self, b, tol, maxiter, replace=50, x0=None):
        """One column of the FP32-direction multi-right-hand-side CG."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.sizes["rowA"]) if x0 is None else np.array(x0, np.float64)
        rel = C.c_double()
        it = lib().mfo_cg_dir32(C.byref(self.t), _ptr(b), _ptr(x), tol, maxiter, replace, C.byref(rel))
        return it, x, rel.value

    def pcg_jacobi(self, diag, b, tol, maxiter, x0=None):
        diag = np.ascontiguousarray(diag, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.sizes["rowA"]) if x0 is None else np.array(x0, np.float64)
        rel = C.c_double()
        it = lib().mfo_pcg_jacobi(C.byref(self.t), _ptr(diag), _ptr(b), _ptr(x), tol, maxiter, C.byref(rel))
        return it, x, rel.value

    def bicgstab(self, b, tol, maxiter, x0=None):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.sizes["rowA"]) if x0 is None else np.array(x0, np.float64)
        rel = C.c_double()
        it = lib().mfo_bicgstab(C.byref(self.t), _ptr(b), _ptr(x), tol, maxiter, C.byref(rel))
        return it, x, rel.value

    def __del__(self):
        try:
            lib().mfo_tiles_free(C.byref(self.t))
        except Exception:
            pass


class RefTiles:
    """Tile_create of the reference itself (oracle/_ref/libmfref.so)."""

    def __init__(self, rowA, colA, rp, ci, val):
        self.rp = np.ascontiguousarray(rp, np.int32)
        self.ci = np.ascontiguousarray(ci, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        self.h = ref().ref_tile_create(rowA, colA, int(self.rp[rowA]), _ptr(self.rp), _ptr(self.ci), _ptr(self.val))
        s = np.zeros(7, np.int32)
        ref().ref_tile_sizes(self.h, _ptr(s))
        self.sizes = dict(zip(("tilem", "tilen", "tilenum", "csrsize", "csrptrlen", "rowA", "colA"), map(int, s)))

    def array(self, name):
        dt, key = ARRAY_SPECS[name]
        n = _length(key, self.sizes)
        a = np.zeros(max(n, 1), dt)
        assert ref().ref_tile_array(self.h, name.encode(), _ptr(a)) == 0
        return a[:n]

    def arrays(self):
        return {k: self.array(k) for k in ARRAY_SPECS}

    def spmv(self, x, fill_compressed=True):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.sizes["tilem"] * 16, np.float64)
        n = self.sizes["tilenum"]
        p1 = np.zeros(max(n, 1), np.int32)
        p2 = np.zeros(max(n, 1), np.int32)
        rbb = np.zeros(1, np.int32)
        ref().ref_blockspmv(self.h, _ptr(x), _ptr(y), _ptr(p1), _ptr(p2), _ptr(rbb), 1 if fill_compressed else 0)
        return y[: self.sizes["rowA"]], p1[:n], p2[:n], int(rbb[0])

    def __del__(self):
        try:
            ref().ref_tile_free(self.h)
        except Exception:
            pass


def set_threads(n):
    """OpenMP threads of the oracle's (and the reference code's) parallel
    loops on this thread; returns the count in effect."""
    return int(lib().mfo_set_threads(int(n)))


def ref_read_mtx(path):
    m, n, nnz = _i(), _i(), _i()
    rp = C.POINTER(_i)()
    ci = C.POINTER(_i)()
    va = C.POINTER(C.c_double)()
    ref().ref_read_mtx(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(va))
    R = np.ctypeslib.as_array(rp, shape=(m.value + 1,)).copy()
    CI = np.ctypeslib.as_array(ci, shape=(nnz.value,)).copy()
    V = np.ctypeslib.as_array(va, shape=(nnz.value,)).copy()
    for p in (rp, ci, va):
        ref().ref_free(C.cast(p, _p))
    return m.value, n.value, R, CI, V


def ref_read_cbd(path):
    """The reference's binary_read_csr: (rows, cols, row_ptr int64, col, val)."""
    m, n, nnz = _i(), _i(), C.c_int64()
    rp = C.POINTER(C.c_int64)()
    ci = C.POINTER(_i)()
    va = C.POINTER(C.c_double)()
    rc = ref().ref_read_cbd(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci),
                            C.byref(va))
    if rc != 0:
        raise OSError(f"binary_read_csr failed on {path}")
    R = np.ctypeslib.as_array(rp, shape=(m.value + 1,)).copy()
    CI = np.ctypeslib.as_array(ci, shape=(nnz.value,)).copy()
    V = np.ctypeslib.as_array(va, shape=(nnz.value,)).copy()
    for p in (rp, ci, va):
        ref().ref_free(C.cast(p, _p))
    return m.value, n.value, R, CI, V


def ref_write_cbd(path, m, n, rp, ci, v):
    """The reference's binary_write_csr of a CSR matrix (row_ptr widened to int64)."""
    rp64 = np.ascontiguousarray(rp, np.int64)
    ci = np.ascontiguousarray(ci, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    ref().ref_write_cbd(path.encode(), m, n, int(rp64[-1]), _ptr(rp64), _ptr(ci), _ptr(v))
