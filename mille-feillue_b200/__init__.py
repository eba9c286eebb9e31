"""Python binding of libmf.so, the B200-native tiled CG / BiCGSTAB solver.

The package name contains a hyphen; import it with
``importlib.import_module("mille-feillue_b200")``.

Everything here calls the C ABI declared in include/mf.h through ctypes;
there is no Python or CPU compute path. Loading fails loudly when the
shared library has not been built.

Reference-facing names mirror the Mille-feuille entry points:
  Tile_create      Performance-Comparison/csr2block.h:267
  blockspmv        Performance-Comparison/blockspmv_cpu.h:2 (SpMV part)
  cg_solve_inc     Performance-Comparison/Mille-feuille_CG_NVIDIA.cu:3979
  bicgstab         Performance-Comparison/Mille-feuille_BiCGSTAB_NVIDIA.cu:1476
  read_Dmatrix_32  Performance-Comparison/biio2.0/src/biio.h:153
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmf.so")

MF_OK = 0
MF_ERR_ARG = -1
MF_ERR_CUDA = -2
MF_ERR_TIMEOUT = -3
MF_ERR_NOT_CONVERGED = -4
MF_ERR_BREAKDOWN = -5
MF_ERR_IO = -6
MF_ERR_NOMEM = -7
MF_ERR_RESIDENCY = -8
MF_ERR_UNSUPPORTED = -9
PANEL_FP64 = 0  # multi-right-hand-side CG: every panel FP64 (each column the FP64 CG)
PANEL_FP32 = 1  # FP32 search directions and products, one persistent launch (default)

PREC_FP64, PREC_FP32, PREC_FP16, PREC_FP8 = 0, 1, 2, 3
MODE_FP64, MODE_MIXED_RULE, MODE_MIXED_MLP, MODE_FIXED = 0, 1, 2, 3
NOALLOC_MAX_ROWS = 131072  # MF_NOALLOC_MAX_ROWS

_i = C.c_int
_d = C.c_double
_p = C.c_void_p


class MfCsr(C.Structure):
    _fields_ = [("n", _i), ("ncols", _i), ("nnz", _i), ("row_ptr", _p), ("col_idx", _p), ("val", _p)]


class MfOptions(C.Structure):
    _fields_ = [
        ("precision_mode", _i), ("fixed_precision", _i), ("replace_every", _i), ("ctas_per_sm", _i),
        ("rb_per_slab", _i), ("slab_bytes", _i), ("timeout_s", _d), ("check_true_residual", _i),
        ("fixed_iterations", _i), ("mixed_tau", _d), ("device", _i), ("reserved", _i * 7),
    ]


class MfResult(C.Structure):
    _fields_ = [
        ("status", _i), ("iterations", _i), ("replacements", _i), ("level_switches", _i),
        ("rel_residual_true", _d), ("rel_residual_rec", _d), ("time_ms", _d), ("spmv_bytes", _d),
        ("spmv_bytes_fp64", _d), ("tile_frac", _d * 4), ("error_site", _i), ("iters_fp64", _i),
        ("iters_level", _i * 3), ("spmv_bytes_level", _d * 3), ("total_bytes", _d),
        ("fell_back_fp64", _i), ("selector_fallback", _i),
    ]

    def as_dict(self):
        return {
            "status": self.status, "iterations": self.iterations, "replacements": self.replacements,
            "level_switches": self.level_switches, "rel_residual_true": self.rel_residual_true,
            "rel_residual_rec": self.rel_residual_rec, "time_ms": self.time_ms,
            "spmv_bytes": self.spmv_bytes, "spmv_bytes_fp64": self.spmv_bytes_fp64,
            "tile_frac": list(self.tile_frac), "error_site": self.error_site, "iters_fp64": self.iters_fp64,
            "iters_level": list(self.iters_level), "spmv_bytes_level": list(self.spmv_bytes_level),
            "total_bytes": self.total_bytes, "fell_back_fp64": self.fell_back_fp64,
            "selector_fallback": self.selector_fallback,
        }


class MfTuneResult(C.Structure):
    _fields_ = [("slab_bytes", _i), ("rb_per_slab", _i), ("ms_best", _d), ("ms_default", _d), ("candidates", _i),
                ("cand_slab_bytes", _i * 16), ("cand_rb_per_slab", _i * 16), ("cand_ms", _d * 16)]


class MfMemoryReport(C.Structure):
    _fields_ = [("csr_bytes", _d), ("tile_index_bytes", _d), ("tile_value_bytes", _d * 4),
                ("tile_total_bytes", _d), ("slab_bytes_fp64", _d), ("slab_bytes_mixed", _d),
                ("workspace_bytes", _d), ("device_bytes", _d)]


class MfTileInfo(C.Structure):
    _fields_ = [(n, _i) for n in ("rowA", "colA", "tilem", "tilen", "tilenum", "csrsize", "csrptrlen",
                                  "cnt_non_new", "nslabs", "nctas")] + [
        ("layout_bytes", C.c_longlong), ("encode_ms", _d), ("layout_ms", _d)]


_ARRAY_FIELDS = [
    ("tile_ptr", np.int32, "tilem+1"), ("tile_columnidx", np.int32, "tilenum"),
    ("tile_nnz", np.int32, "tilenum+1"), ("blknnz", np.int32, "tilenum+1"),
    ("csr_offset", np.int32, "tilenum+1"), ("csrptr_offset", np.int32, "tilenum+1"),
    ("Format", np.int8, "tilenum"), ("blknnznnz", np.uint8, "tilenum+1"),
    ("Blockcsr_Val", np.float64, "csrsize"), ("Blockcsr_Val_Low", np.float32, "csrsize"),
    ("Tile_csr_Col", np.uint8, "csrsize"), ("Blockcsr_Ptr", np.uint8, "csrptrlen"),
    ("csr_compressedIdx", np.uint8, "csrhalf"), ("ptroffset1", np.int32, "tilenum"),
    ("ptroffset2", np.int32, "tilenum"), ("tile_rowidx", np.int32, "tilenum"),
    ("nonzero_row_new", np.int32, "tilenum+1"), ("block_signal", np.int32, "tilem+1"),
    ("blockrowid_new", np.uint8, "cnt+1"), ("blockcsr_ptr_new", np.uint8, "cnt+1"),
]


class MfTileArrays(C.Structure):
    _fields_ = [(name, _p) for name, _, _ in _ARRAY_FIELDS]


# C-ABI symbols declared in include/mf.h (checked by the CPU test suite).
EXPORTED = [
    "mf_status_str", "mf_options_default", "mf_gen_poisson2d", "mf_gen_convdiff3d", "mf_gen_varpoisson3d",
    "mf_gen_spd_random", "mf_gen_batch_sizes", "mf_read_mtx", "mf_read_cbd", "mf_write_cbd",
    "mf_matrix_from_csr", "mf_matrix_info", "mf_matrix_csr", "mf_matrix_b", "mf_matrix_xstar",
    "mf_matrix_set_b", "mf_matrix_free", "mf_encode", "mf_encode_dev", "mf_free", "mf_tiles_info",
    "mf_tiles_export", "mf_tiles_precisions", "mf_tiles_set_precisions", "mf_balance_twopointer", "mf_spmv",
    "mf_spmv_host", "mf_spmv_bench", "mf_solve_cg", "mf_solve_cg_dev", "mf_solve_bicgstab",
    "mf_solve_bicgstab_dev", "mf_true_residual", "cg_solve_inc", "bicgstab", "mf_version", "mf_last_error",
    "mf_spmv_level", "mf_spmv_bench_level", "mf_trace", "mf_batch_create", "mf_batch_solve_cg_dev",
    "mf_batch_solve_cg_each_dev", "mf_batch_results", "mf_batch_info", "mf_batch_free",
    "mf_solve_cg_dev_noalloc", "mf_mlp_set_weights", "mf_mlp_get_weights", "mf_tiles_features",
    "mf_tiles_select_mlp", "mf_mlp_forward_dev", "mf_mlp_grad_dev", "mf_mlp_train_dev", "mf_solve_pcg",
    "mf_solve_pcg_dev", "mf_memory_report", "mf_tiles_autotune", "mf_solve_cg_multi", "mf_solve_cg_multi_dev",
    "mf_solve_cg_multi_ex", "mf_solve_cg_multi_dev_ex", "mf_check_planner",
]
MLP_WEIGHTS = 4868
MLP_WEIGHTS_PATH = os.path.join(_HERE, "mlp_weights.bin")

_lib = None


def lib():
    """Loads libmf.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libmf.so not built at {LIB_PATH}; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    L.mf_status_str.restype = C.c_char_p
    L.mf_status_str.argtypes = [_i]
    L.mf_version.restype = C.c_char_p
    L.mf_last_error.restype = C.c_char_p
    L.mf_options_default.argtypes = [C.POINTER(MfOptions)]
    L.mf_gen_poisson2d.argtypes = [_i, C.POINTER(_p)]
    L.mf_gen_convdiff3d.argtypes = [_i, _d, _d, _d, C.c_uint64, C.POINTER(_p)]
    L.mf_gen_varpoisson3d.argtypes = [_i, _d, _d, C.c_uint64, C.POINTER(_p)]
    L.mf_gen_spd_random.argtypes = [_i, C.c_uint64, C.POINTER(_p)]
    L.mf_gen_batch_sizes.argtypes = [_i, _i, _i, C.c_uint64, _p]
    L.mf_read_mtx.argtypes = [C.c_char_p, C.POINTER(_p)]
    L.mf_read_cbd.argtypes = [C.c_char_p, C.POINTER(_p)]
    L.mf_write_cbd.argtypes = [_p, C.c_char_p]
    L.mf_matrix_from_csr.argtypes = [_i, _i, _i, _p, _p, _p, C.POINTER(_p)]
    L.mf_matrix_info.argtypes = [_p] + [C.POINTER(_i)] * 5
    L.mf_matrix_csr.argtypes = [_p, C.POINTER(MfCsr)]
    L.mf_matrix_b.argtypes = [_p]
    L.mf_matrix_b.restype = _p
    L.mf_matrix_xstar.argtypes = [_p]
    L.mf_matrix_xstar.restype = _p
    L.mf_matrix_set_b.argtypes = [_p, _p]
    L.mf_matrix_free.argtypes = [_p]
    L.mf_encode.argtypes = [C.POINTER(MfCsr), C.POINTER(MfOptions), C.POINTER(_p)]
    L.mf_encode_dev.argtypes = [_i, _i, _i, _p, _p, _p, C.POINTER(MfOptions), C.POINTER(_p)]
    L.mf_free.argtypes = [_p]
    L.mf_tiles_info.argtypes = [_p, C.POINTER(MfTileInfo)]
    L.mf_tiles_export.argtypes = [_p, C.POINTER(MfTileArrays)]
    L.mf_tiles_precisions.argtypes = [_p, _p, _p]
    L.mf_tiles_set_precisions.argtypes = [_p, _p]
    L.mf_balance_twopointer.argtypes = [_p, _i, _i, C.POINTER(_i), _p, _p, _p, _p]
    L.mf_spmv.argtypes = [_p, _p, _p, _p]
    L.mf_spmv_level.argtypes = [_p, _i, _p, _p]
    L.mf_spmv_host.argtypes = [_p, _p, _p]
    L.mf_spmv_bench.argtypes = [_p, _p, _p, _i, C.POINTER(_d), C.POINTER(_d)]
    L.mf_spmv_bench_level.argtypes = [_p, _i, _p, _p, _i, C.POINTER(_d), C.POINTER(_d)]
    for f in ("mf_solve_cg", "mf_solve_cg_dev", "mf_solve_bicgstab", "mf_solve_bicgstab_dev", "mf_solve_pcg",
              "mf_solve_pcg_dev",
              "mf_solve_cg_dev_noalloc"):
        getattr(L, f).argtypes = [_p, _p, _p, _d, _i, C.POINTER(MfOptions), C.POINTER(MfResult)]
    L.mf_true_residual.argtypes = [_p, _p, _p, C.POINTER(_d)]
    L.mf_check_planner.argtypes = [_i, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.mf_check_planner.restype = _i
    L.mf_memory_report.argtypes = [_p, C.POINTER(MfMemoryReport)]
    L.mf_tiles_autotune.argtypes = [_p, _i, C.POINTER(MfTuneResult)]
    L.mf_solve_cg_multi.argtypes = [C.POINTER(MfCsr), _i, _p, _p, _d, _i, _p, _p, C.POINTER(_d)]
    L.mf_solve_cg_multi_dev.argtypes = [_i, _p, _p, _p, _i, _p, _p, _d, _i, _p, _p, C.POINTER(_d)]
    L.mf_solve_cg_multi_ex.argtypes = [_i, C.POINTER(MfCsr), _i, _p, _p, _d, _i, _p, _p, C.POINTER(_d)]
    L.mf_solve_cg_multi_dev_ex.argtypes = [_i, _i, _p, _p, _p, _i, _p, _p, _d, _i, _p, _p, C.POINTER(_d)]
    L.mf_mlp_set_weights.argtypes = [_p]
    L.mf_mlp_get_weights.argtypes = [_p]
    L.mf_tiles_features.argtypes = [_p, _p]
    L.mf_tiles_select_mlp.argtypes = [_p, _i, _p, _p]
    L.mf_mlp_forward_dev.argtypes = [_p, _p, _i, _i, _p]
    L.mf_mlp_grad_dev.argtypes = [_p, _p, _p, _i, _p, C.POINTER(C.c_float)]
    L.mf_mlp_train_dev.argtypes = [_p, _p, _p, _i, _i, _i, C.c_float, C.POINTER(C.c_float)]
    L.mf_trace.argtypes = [_p, _p, _i]
    L.mf_batch_create.argtypes = [_i, _p, C.POINTER(MfOptions), _i, C.POINTER(_p)]
    L.mf_batch_solve_cg_dev.argtypes = [_p, _p, _p, _d, _i, C.POINTER(_d)]
    L.mf_batch_solve_cg_each_dev.argtypes = [_p, _p, _p, _d, _i, C.POINTER(_d)]
    L.mf_batch_results.argtypes = [_p, _p, _p, _p]
    L.mf_batch_info.argtypes = [_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(_i)]
    L.mf_batch_free.argtypes = [_p]
    L.cg_solve_inc.argtypes = [_p, _p, _p, _p, _p, _p, _i, C.POINTER(_i), _i, _d, C.c_char_p, _i, _i, _i]
    L.cg_solve_inc.restype = None
    L.bicgstab.argtypes = [_p, _p, _p, _p, _p, _i, C.c_char_p, _i, _i]
    _lib = L
    return L


class MfError(RuntimeError):
    def __init__(self, status, what=""):
        msg = lib().mf_status_str(status).decode()
        detail = lib().mf_last_error().decode()
        super().__init__(f"{what}: {msg} ({status}) {detail}".strip())
        self.status = status


def _check(rc, what):
    if rc != MF_OK:
        raise MfError(rc, what)


def _ptr(a):
    return a.ctypes.data_as(_p)


def solve_cg_multi(matrix, B, X0=None, tol=1e-10, maxiter=10000, panel=PANEL_FP32):
    """CG on the k <= 16 columns of B (n x k) at once, sharing each SpMM
    (panel: PANEL_FP32 or PANEL_FP64). Returns (X, iterations[k],
    rel_residual[k], device ms)."""
    B = np.asfortranarray(B, dtype=np.float64)
    n, k = B.shape
    X = np.asfortranarray(np.zeros((n, k)) if X0 is None else X0, dtype=np.float64)
    it = np.zeros(k, np.int32)
    rel = np.zeros(k)
    ms = _d()
    rc = lib().mf_solve_cg_multi_ex(panel, C.byref(matrix.csr_struct()), k, _ptr(B), _ptr(X), tol, maxiter,
                                    _ptr(it), _ptr(rel), C.byref(ms))
    if rc not in (MF_OK, MF_ERR_NOT_CONVERGED):
        _check(rc, "mf_solve_cg_multi")
    return X, it, rel, ms.value


def set_mlp_weights(w):
    """Process-wide selector weights (MLP_WEIGHTS floats); None clears them."""
    if w is None:
        _check(lib().mf_mlp_set_weights(None), "mf_mlp_set_weights")
        return
    a = np.ascontiguousarray(w, np.float32)
    if a.size != MLP_WEIGHTS:
        raise ValueError(f"selector weights need {MLP_WEIGHTS} floats, got {a.size}")
    _check(lib().mf_mlp_set_weights(_ptr(a)), "mf_mlp_set_weights")


def load_mlp_weights(path=None):
    """Loads selector weights (raw little-endian float32) and sets them."""
    w = np.fromfile(path or MLP_WEIGHTS_PATH, dtype="<f4")
    set_mlp_weights(w)
    return w


def options(**kw):
    """mf_options with the library defaults, overridden by keyword."""
    o = MfOptions()
    lib().mf_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


# ------------------------------------------------------------------ matrices
class Matrix:
    """Host CSR matrix owned by libmf (mf_matrix)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def _make(cls, fn, *args):
        h = _p()
        _check(fn(*args, C.byref(h)), fn.__name__)
        return cls(h)

    @classmethod
    def poisson2d(cls, N):
        return cls._make(lib().mf_gen_poisson2d, N)

    @classmethod
    def convdiff3d(cls, N, v=(1.0, 0.5, 0.25), seed=0):
        return cls._make(lib().mf_gen_convdiff3d, N, v[0], v[1], v[2], seed)

    @classmethod
    def varpoisson3d(cls, N, klo=1e-3, khi=1e3, seed=1):
        return cls._make(lib().mf_gen_varpoisson3d, N, klo, khi, seed)

    @classmethod
    def spd_random(cls, n, seed):
        return cls._make(lib().mf_gen_spd_random, n, seed)

    @classmethod
    def read_mtx(cls, path):
        return cls._make(lib().mf_read_mtx, path.encode())

    @classmethod
    def read_cbd(cls, path):
        return cls._make(lib().mf_read_cbd, path.encode())

    @classmethod
    def from_csr(cls, n, ncols, row_ptr, col_idx, val):
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        v = np.ascontiguousarray(val, np.float64)
        return cls._make(lib().mf_matrix_from_csr, n, ncols, int(rp[-1]), _ptr(rp), _ptr(ci), _ptr(v))

    def write_cbd(self, path):
        _check(lib().mf_write_cbd(self.h, path.encode()), "mf_write_cbd")

    def info(self):
        n, nc, nnz, hb, hx = _i(), _i(), _i(), _i(), _i()
        lib().mf_matrix_info(self.h, C.byref(n), C.byref(nc), C.byref(nnz), C.byref(hb), C.byref(hx))
        return n.value, nc.value, nnz.value, bool(hb.value), bool(hx.value)

    @property
    def n(self):
        return self.info()[0]

    @property
    def nnz(self):
        return self.info()[2]

    def csr_struct(self):
        c = MfCsr()
        lib().mf_matrix_csr(self.h, C.byref(c))
        return c

    def csr(self):
        """(row_ptr, col_idx, val) as numpy copies."""
        c = self.csr_struct()
        rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(_i)), shape=(c.n + 1,)).copy()
        if c.nnz == 0:
            return rp, np.zeros(0, np.int32), np.zeros(0)
        ci = np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(_i)), shape=(c.nnz,)).copy()
        v = np.ctypeslib.as_array(C.cast(c.val, C.POINTER(_d)), shape=(c.nnz,)).copy()
        return rp, ci, v

    def _vec(self, fn):
        p = fn(self.h)
        if not p:
            return None
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(_d)), shape=(self.n,)).copy()

    def b(self):
        return self._vec(lib().mf_matrix_b)

    def xstar(self):
        return self._vec(lib().mf_matrix_xstar)

    def __del__(self):
        try:
            if self.h:
                lib().mf_matrix_free(self.h)
                self.h = None
        except Exception:
            pass


def check_planner(on=None):
    """Switches the GPU slab planner's self-check (every layout built is also
    planned on the host and compared) and returns (checked, mismatches)."""
    c, m = C.c_longlong(), C.c_longlong()
    lib().mf_check_planner(-1 if on is None else int(bool(on)), C.byref(c), C.byref(m))
    return c.value, m.value


def batch_sizes(count=512, lo=1000, hi=200000, seed=2):
    out = np.zeros(count, np.int32)
    _check(lib().mf_gen_batch_sizes(count, lo, hi, seed, _ptr(out)), "mf_gen_batch_sizes")
    return out


# --------------------------------------------------------------------- tiles
class Tiles:
    """Device tile matrix (mf_tiles): the GPU csr2block encoding plus the
    solver's slab layout."""

    def __init__(self, matrix=None, opts=None, csr=None):
        self.h = _p()
        o = opts if opts is not None else options()
        if matrix is not None:
            c = matrix.csr_struct()
            self._keep = matrix
        else:
            n, ncols, rp, ci, v = csr
            self._keep = (np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                          np.ascontiguousarray(v, np.float64))
            c = MfCsr(n, ncols, int(self._keep[0][n]), _ptr(self._keep[0]), _ptr(self._keep[1]), _ptr(self._keep[2]))
        if o.precision_mode == MODE_MIXED_MLP and lib().mf_mlp_get_weights(None) != MF_OK:
            load_mlp_weights()  # the packaged selector, unless the caller set one
        _check(lib().mf_encode(C.byref(c), C.byref(o), C.byref(self.h)), "mf_encode")
        self.opts = o

    def autotune(self, reps=20):
        """Picks the slab geometry with the fastest solver SpMV; the handle keeps it."""
        r = MfTuneResult()
        _check(lib().mf_tiles_autotune(self.h, reps, C.byref(r)), "mf_tiles_autotune")
        k = r.candidates
        return {"slab_bytes": r.slab_bytes, "rb_per_slab": r.rb_per_slab, "ms_best": r.ms_best,
                "ms_default": r.ms_default,
                "candidates": [(r.cand_slab_bytes[i], r.cand_rb_per_slab[i], r.cand_ms[i]) for i in range(k)]}

    def memory_report(self):
        """Memory cost of the tile format vs CSR (the reference's study) and the device bytes held."""
        r = MfMemoryReport()
        _check(lib().mf_memory_report(self.h, C.byref(r)), "mf_memory_report")
        d = {f: getattr(r, f) for f, _ in r._fields_}
        d["tile_value_bytes"] = list(r.tile_value_bytes)
        return d

    def features(self):
        """Selector features f0..f5 of every tile, shape (tilenum, 6)."""
        n = self.info()["tilenum"]
        f = np.zeros((max(n, 1), 6), np.float32)
        _check(lib().mf_tiles_features(self.h, _ptr(f)), "mf_tiles_features")
        return f[:n]

    def select_mlp(self, rel_res):
        """Learned selector classes at the given residual levels, (levels, tilenum)."""
        n = self.info()["tilenum"]
        r = np.ascontiguousarray(rel_res, np.float64)
        p = np.zeros((len(r), max(n, 1)), np.uint8)
        _check(lib().mf_tiles_select_mlp(self.h, len(r), _ptr(r), _ptr(p)), "mf_tiles_select_mlp")
        return p[:, :n]

    def info(self):
        i = MfTileInfo()
        _check(lib().mf_tiles_info(self.h, C.byref(i)), "mf_tiles_info")
        return {f: getattr(i, f) for f, _ in i._fields_}

    def export(self, names=None):
        """Host copies of the Tile_create arrays (reference names)."""
        inf = self.info()
        sizes = {"tilem+1": inf["tilem"] + 1, "tilenum": inf["tilenum"], "tilenum+1": inf["tilenum"] + 1,
                 "csrsize": inf["csrsize"], "csrptrlen": inf["csrptrlen"], "csrhalf": (inf["csrsize"] + 1) // 2,
                 "cnt+1": inf["cnt_non_new"] + 1}
        arrs = MfTileArrays()
        out = {}
        for name, dt, key in _ARRAY_FIELDS:
            if names is not None and name not in names:
                continue
            a = np.zeros(max(sizes[key], 1), dt)
            out[name] = (a, sizes[key])
            setattr(arrs, name, _ptr(a))
        _check(lib().mf_tiles_export(self.h, C.byref(arrs)), "mf_tiles_export")
        return {k: a[:n] for k, (a, n) in out.items()}

    def precisions(self):
        n = self.info()["tilenum"]
        p = np.zeros(max(n, 1), np.uint8)
        s = np.zeros(max(n, 1), np.float32)
        _check(lib().mf_tiles_precisions(self.h, _ptr(p), _ptr(s)), "mf_tiles_precisions")
        return p[:n], s[:n]

    def set_precisions(self, prec):
        p = np.ascontiguousarray(prec, np.uint8)
        _check(lib().mf_tiles_set_precisions(self.h, _ptr(p)), "mf_tiles_set_precisions")

    def balance_twopointer(self, block_nnz, block_per_warp=180):
        idx = _i()
        _check(lib().mf_balance_twopointer(self.h, block_nnz, block_per_warp, C.byref(idx), None, None, None, None),
               "mf_balance_twopointer")
        n = self.info()["tilenum"]
        bp = np.zeros(idx.value + 1, np.int32)
        a, b, c = (np.zeros(n + 1, np.int32) for _ in range(3))
        _check(lib().mf_balance_twopointer(self.h, block_nnz, block_per_warp, C.byref(idx), _ptr(bp), _ptr(a),
                                           _ptr(b), _ptr(c)), "mf_balance_twopointer")
        return idx.value, bp, a, b, c

    def spmv(self, x):
        """y = A x through mf_spmv_host (host buffers)."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.info()["rowA"], np.float64)
        _check(lib().mf_spmv_host(self.h, _ptr(x), _ptr(y)), "mf_spmv_host")
        return y

    def spmv_dev(self, x_ptr, y_ptr, stream=None):
        _check(lib().mf_spmv(self.h, _p(x_ptr), _p(y_ptr), _p(stream or 0)), "mf_spmv")

    def spmv_level_dev(self, level, x_ptr, y_ptr):
        _check(lib().mf_spmv_level(self.h, level, _p(x_ptr), _p(y_ptr)), "mf_spmv_level")

    def spmv_bench(self, x_ptr, y_ptr, reps, level=-1):
        ms, nb = _d(), _d()
        _check(lib().mf_spmv_bench_level(self.h, level, _p(x_ptr), _p(y_ptr), reps, C.byref(ms), C.byref(nb)),
               "mf_spmv_bench")
        return ms.value, nb.value

    def _solve(self, fn, b, x0, tol, maxiter, opts):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.info()["rowA"]) if x0 is None else np.array(x0, np.float64)
        res = MfResult()
        o = opts if opts is not None else self.opts
        rc = fn(self.h, _ptr(b), _ptr(x), tol, maxiter, C.byref(o), C.byref(res))
        if rc not in (MF_OK, MF_ERR_NOT_CONVERGED, MF_ERR_BREAKDOWN):
            raise MfError(rc, fn.__name__)
        return x, res.as_dict()

    def solve_cg(self, b, x0=None, tol=1e-10, maxiter=10000, opts=None):
        return self._solve(lib().mf_solve_cg, b, x0, tol, maxiter, opts)

    def solve_bicgstab(self, b, x0=None, tol=1e-10, maxiter=10000, opts=None):
        return self._solve(lib().mf_solve_bicgstab, b, x0, tol, maxiter, opts)

    def solve_pcg(self, b, x0=None, tol=1e-10, maxiter=10000, opts=None):
        """Jacobi-preconditioned CG (FP64)."""
        return self._solve(lib().mf_solve_pcg, b, x0, tol, maxiter, opts)

    def solve_pcg_dev(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000, opts=None):
        return self._solve_dev(lib().mf_solve_pcg_dev, b_ptr, x_ptr, tol, maxiter, opts)

    def _solve_dev(self, fn, b_ptr, x_ptr, tol, maxiter, opts):
        res = MfResult()
        o = opts if opts is not None else self.opts
        rc = fn(self.h, _p(b_ptr), _p(x_ptr), tol, maxiter, C.byref(o), C.byref(res))
        if rc not in (MF_OK, MF_ERR_NOT_CONVERGED, MF_ERR_BREAKDOWN):
            raise MfError(rc, fn.__name__)
        return res.as_dict()

    def solve_cg_dev(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000, opts=None):
        return self._solve_dev(lib().mf_solve_cg_dev, b_ptr, x_ptr, tol, maxiter, opts)

    def solve_bicgstab_dev(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000, opts=None):
        return self._solve_dev(lib().mf_solve_bicgstab_dev, b_ptr, x_ptr, tol, maxiter, opts)

    def solve_cg_dev_noalloc(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000, opts=None):
        """FP64 CG with static device scratch (no allocation; n <= NOALLOC_MAX_ROWS)."""
        return self._solve_dev(lib().mf_solve_cg_dev_noalloc, b_ptr, x_ptr, tol, maxiter, opts)

    def trace(self, max_iters=4096):
        """Phase timestamps of the last traced CG solve, shape (iters, 8)."""
        buf = np.zeros(max_iters * 8, np.uint64)
        n = lib().mf_trace(self.h, _ptr(buf), max_iters)
        return buf[: max(n, 0) * 8].reshape(-1, 8)

    def __del__(self):
        try:
            if self.h:
                lib().mf_free(self.h)
                self.h = None
        except Exception:
            pass


def generate_spd_batch(sizes, seed=2, threads=16, index=None):
    """The random SPD systems of a batch (system s drawn with seed
    seed * 1000003 + s + 1), generated in parallel host threads. `index`
    gives each size's position in the whole batch (default 0, 1, ...), so a
    rank that holds a subset draws the same systems as a single process."""
    from concurrent.futures import ThreadPoolExecutor

    idx = list(range(len(sizes))) if index is None else [int(i) for i in index]
    if len(idx) != len(sizes):
        raise ValueError("index must give one position per size")
    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(lambda a: Matrix.spd_random(int(a[1]), seed * 1000003 + a[0] + 1), zip(idx, sizes)))


def split_systems(sizes, world):
    """Longest-processing-time split of a batch over `world` ranks: systems
    in decreasing size, each to the rank with the least load so far (ties to
    the lowest rank). Returns one ascending index list per rank; every rank
    computes the same split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for s in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        rk = min(range(world), key=lambda k: (loads[k], k))
        loads[rk] += float(sizes[s])
        parts[rk].append(s)
    return [sorted(p) for p in parts]


class Batch:
    """Many independent systems solved by one persistent launch (mf_batch)."""

    def __init__(self, matrices, opts=None, with_baseline=False):
        self._mats = list(matrices)
        arr = (MfCsr * len(self._mats))(*[m.csr_struct() for m in self._mats])
        self.h = _p()
        o = opts if opts is not None else options()
        _check(lib().mf_batch_create(len(self._mats), C.cast(arr, _p), C.byref(o), 1 if with_baseline else 0,
                                     C.byref(self.h)), "mf_batch_create")
        self.sizes = np.array([m.n for m in self._mats], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])

    def info(self):
        r, z, g = C.c_longlong(), C.c_longlong(), _i()
        lib().mf_batch_info(self.h, C.byref(r), C.byref(z), C.byref(g))
        return {"rows": r.value, "nnz": z.value, "grid": g.value}

    def solve_cg_dev(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000):
        ms = _d()
        rc = lib().mf_batch_solve_cg_dev(self.h, _p(b_ptr), _p(x_ptr), tol, maxiter, C.byref(ms))
        _check(rc, "mf_batch_solve_cg_dev")
        return ms.value

    def solve_cg_each_dev(self, b_ptr, x_ptr, tol=1e-10, maxiter=10000):
        ms = _d()
        _check(lib().mf_batch_solve_cg_each_dev(self.h, _p(b_ptr), _p(x_ptr), tol, maxiter, C.byref(ms)),
               "mf_batch_solve_cg_each_dev")
        return ms.value

    def results(self):
        n = len(self._mats)
        it = np.zeros(n, np.int32)
        st = np.zeros(n, np.int32)
        rel = np.zeros(n, np.float64)
        _check(lib().mf_batch_results(self.h, _ptr(it), _ptr(st), _ptr(rel)), "mf_batch_results")
        return it, st, rel

    def __del__(self):
        try:
            if self.h:
                lib().mf_batch_free(self.h)
                self.h = None
        except Exception:
            pass


# ------------------------------------------------ reference-interface mirror
def Tile_create(rowA, colA, row_ptr, col_idx, val):
    """GPU csr2block: the arrays of Tile_create (csr2block.h:267) as numpy."""
    t = Tiles(csr=(rowA, colA, row_ptr, col_idx, val))
    return t.export(), t


def blockspmv(tiles, x):
    """y = A x with the tiled GPU kernel, in blockspmv_cpu's summation order."""
    return tiles.spmv(x)


def cg_solve_inc(RowPtr, ColIdx, Val, x, b, n, maxiter=10000, threshold=1e-10, ori=None, block_nnz=0):
    """Drop-in of cg_solve_inc: solves on the first (n // 16) * 16 rows, writes
    the solution into x (numpy, in place) and returns the iteration count."""
    rp = np.ascontiguousarray(RowPtr, np.int32)
    ci = np.ascontiguousarray(ColIdx, np.int32)
    v = np.ascontiguousarray(Val, np.float64)
    low = v.astype(np.float32)
    bb = np.ascontiguousarray(b, np.float64)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    it = _i(0)
    lib().cg_solve_inc(_ptr(rp), _ptr(ci), _ptr(v), _ptr(low), _ptr(x), _ptr(bb), n, C.byref(it), maxiter,
                       threshold, b"", int(rp[n]) if n < len(rp) else int(rp[-1]), ori if ori else n, block_nnz)
    return it.value


def bicgstab(RowPtr, ColIdx, Val, rhs, x, n, block_nnz=0):
    """Drop-in of bicgstab: rhs is overwritten with A * ones, x with the
    solution; returns 0 on convergence, 1 otherwise (the reference's code)."""
    rp = np.ascontiguousarray(RowPtr, np.int32)
    ci = np.ascontiguousarray(ColIdx, np.int32)
    v = np.ascontiguousarray(Val, np.float64)
    assert rhs.dtype == np.float64 and x.dtype == np.float64
    return lib().bicgstab(_ptr(rp), _ptr(ci), _ptr(v), _ptr(rhs), _ptr(x), int(rp[-1]), b"", n, block_nnz)


def read_Dmatrix_32(path):
    """read_Dmatrix_32 semantics: (m, n, row_ptr, col_idx, val)."""
    m = Matrix.read_mtx(path)
    n, nc, _, _, _ = m.info()
    rp, ci, v = m.csr()
    return n, nc, rp, ci, v
