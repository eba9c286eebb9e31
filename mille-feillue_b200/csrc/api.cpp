// C ABI of libmf (declared in include/mf.h): handles, encoder entry points,
// exports of the Tile_create arrays, SpMV and the persistent solvers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "solver.h"
#include "tiles.h"

using namespace mf;

namespace mf {
int build_mixed_levels(mf_tiles *t, cudaStream_t s);                                  // precision.cu
int abs_range(const double *v, long long n, double *lo, double *hi, cudaStream_t s);  // precision.cu
}

template <class T>
static int d2h(T *dst, const T *src, size_t count) {
    if (!dst || count == 0) return MF_OK;
    MF_CUDA_TRY(cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost));
    return MF_OK;
}

extern "C" {

const char *mf_status_str(int s) {
    switch (s) {
        case MF_OK: return "ok";
        case MF_ERR_ARG: return "invalid argument";
        case MF_ERR_CUDA: return "CUDA error";
        case MF_ERR_TIMEOUT: return "device wait timed out";
        case MF_ERR_NOT_CONVERGED: return "not converged";
        case MF_ERR_BREAKDOWN: return "breakdown";
        case MF_ERR_IO: return "I/O error";
        case MF_ERR_NOMEM: return "out of memory";
        case MF_ERR_RESIDENCY: return "persistent grid cannot be co-resident";
        case MF_ERR_UNSUPPORTED: return "unsupported input";
        default: return "unknown status";
    }
}

const char *mf_version(void) { return "mf-b200 0.1 (sm_100a)"; }

const char *mf_last_error(void) { return mf::last_error().c_str(); }

void mf_options_default(mf_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->precision_mode = MF_MODE_FP64;
    o->fixed_precision = MF_PREC_FP64;
    o->replace_every = 50;
    o->ctas_per_sm = 0;
    o->rb_per_slab = 0;
    o->slab_bytes = 0;
    o->timeout_s = 2.0;
    o->check_true_residual = 1;
    o->fixed_iterations = 0;
    o->mixed_tau = 0.0;
    o->device = 0;
}

}  // extern "C"

namespace mf {
int ensure_host_tiles(const mf_tiles *t) {
    std::lock_guard<std::mutex> lock(t->host_tiles_mu);
    if (t->host_tiles) return MF_OK;
    t->h_tile_ptr.resize(t->tilem + 1);
    t->h_tile_col.resize(t->tilenum);
    std::vector<int> off(t->tilenum + 1);
    MF_CUDA_TRY(cudaMemcpy(t->h_tile_ptr.data(), t->tile_ptr.p, sizeof(int) * (t->tilem + 1), cudaMemcpyDeviceToHost));
    if (t->tilenum > 0)
        MF_CUDA_TRY(cudaMemcpy(t->h_tile_col.data(), t->tile_col.p, sizeof(int) * t->tilenum, cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(off.data(), t->tile_off.p, sizeof(int) * (t->tilenum + 1), cudaMemcpyDeviceToHost));
    t->h_tile_nnz.resize(t->tilenum);
    for (int k = 0; k < t->tilenum; ++k) t->h_tile_nnz[k] = off[k + 1] - off[k];
    t->host_tiles = true;
    return MF_OK;
}

// Encodes a device CSR; G > 0 forces the number of CTA ranges of the layout
// (1 for the batched solver, whose CTAs each own a whole system).
int encode_dev_impl(int n, int ncols, int nnz, const int *rp, const int *ci, const double *val,
                    const mf_options *opt, int G_force, mf_tiles **out) {
    if (!out || n <= 0 || ncols <= 0 || nnz < 0 || !rp || (nnz > 0 && (!ci || !val))) return MF_ERR_ARG;
    auto *t = new mf_tiles;
    if (opt) t->opt = *opt;
    else mf_options_default(&t->opt);
    int rc;
    MF_CUDA_TRY(cudaSetDevice(t->opt.device));
    t->device = t->opt.device;
    MF_CUDA_TRY(cudaDeviceGetAttribute(&t->nsm, cudaDevAttrMultiProcessorCount, t->device));
    if ((rc = kernel_config(t, &t->G)) != MF_OK) { delete t; return rc; }
    if (G_force > 0) t->G = G_force;
    cudaStream_t s = 0;
    if ((rc = encode_device(t, n, ncols, nnz, rp, ci, val, s)) != MF_OK) { delete t; return rc; }
    std::vector<uint8_t> prec(t->tilenum, MF_PREC_FP64);
    if ((rc = build_layout(t, t->L64, prec, s)) != MF_OK) { delete t; return rc; }
    if (t->opt.precision_mode != MF_MODE_FP64) {
        if ((rc = build_mixed_levels(t, s)) != MF_OK) { delete t; return rc; }
    }
    *out = t;
    return MF_OK;
}
}  // namespace mf

extern "C" {

int mf_encode_dev(int n, int ncols, int nnz, const int *rp, const int *ci, const double *val,
                  const mf_options *opt, mf_tiles **out) {
    return mf::encode_dev_impl(n, ncols, nnz, rp, ci, val, opt, 0, out);
}

int mf_encode(const mf_csr *A, const mf_options *opt, mf_tiles **out) {
    if (!A || !out || A->n <= 0 || A->ncols <= 0 || A->nnz < 0 || !A->row_ptr) return MF_ERR_ARG;
    if (A->row_ptr[0] != 0 || A->row_ptr[A->n] != A->nnz) return MF_ERR_ARG;
    // the column indices and the row pointers' order are checked on the GPU
    // by the encoder (as for mf_encode_dev)
    const int dev = opt ? opt->device : 0;
    MF_CUDA_TRY(cudaSetDevice(dev));
    DevArray<int> rp, ci;
    DevArray<double> v;
    if (rp.alloc(A->n + 1) || ci.alloc(A->nnz) || v.alloc(A->nnz)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpy(rp.p, A->row_ptr, sizeof(int) * (A->n + 1), cudaMemcpyHostToDevice));
    if (A->nnz > 0) {
        MF_CUDA_TRY(cudaMemcpy(ci.p, A->col_idx, sizeof(int) * A->nnz, cudaMemcpyHostToDevice));
        MF_CUDA_TRY(cudaMemcpy(v.p, A->val, sizeof(double) * A->nnz, cudaMemcpyHostToDevice));
    }
    return mf_encode_dev(A->n, A->ncols, A->nnz, rp.p, ci.p, v.p, opt, out);
}

void mf_free(mf_tiles *t) { delete t; }

int mf_tiles_info(const mf_tiles *t, mf_tile_info *info) {
    if (!t || !info) return MF_ERR_ARG;
    info->rowA = t->rowA;
    info->colA = t->colA;
    info->tilem = t->tilem;
    info->tilen = t->tilen;
    info->tilenum = t->tilenum;
    info->csrsize = t->csrsize;
    info->csrptrlen = t->csrptrlen;
    info->cnt_non_new = t->cnt_non_new;
    info->nslabs = t->L64.nslabs;
    info->nctas = t->G;
    info->layout_bytes = (long long)t->L64.bytes;
    info->encode_ms = t->encode_ms;
    info->layout_ms = t->layout_ms;
    return MF_OK;
}

extern "C++" {
namespace {
template <class T>
double dev_bytes(const DevArray<T> &a) {
    return (double)a.n * sizeof(T);
}
double layout_dev_bytes(const Layout &L) {
    return dev_bytes(L.slabs) + dev_bytes(L.head) + dev_bytes(L.cta_slab) + dev_bytes(L.cta_rb) +
           dev_bytes(L.cta_dep) + dev_bytes(L.prec_dev) + dev_bytes(L.scale_dev);
}
}  // namespace
}  // extern "C++"

// The reference's memory-cost study (Memory-Cost/memory_Mille_feillue.cu)
// counts the tile metadata (:659-668), the row-compression and per-entry
// column bytes (:859-863) and the value bytes of the precision mix (:916);
// its cuSPARSE counterpart counts CSR as (n+1) + nnz int32 and nnz FP64
// values (memory_cuSPARSE.cu:189-191). The same tallies here, for the
// level-0 precision mix, beside what this handle actually holds on the GPU.
int mf_memory_report(const mf_tiles *t, mf_memory_cost *r) {
    if (!t || !r) return MF_ERR_ARG;
    std::memset(r, 0, sizeof *r);
    if (int rc = mf::ensure_host_tiles(t)) return rc;
    const double tn = t->tilenum, tm = t->tilem;
    r->csr_bytes = (double)(t->rowA + 1) * 4 + (double)t->csrsize * (4 + 8);
    r->tile_index_bytes = (tm + 1) * 4 + tn * 4 + (tn + 1) * 1 + (tn + 1) * 4 + (tn + 1) * 4 + (tn + 3) * 4 +
                          2.0 * (t->cnt_non_new + 1) + tn + (double)t->csrsize + tn * 4;
    const std::vector<uint8_t> *prec = (t->mixed_ready && t->Lmix[0].built) ? &t->Lmix[0].prec : nullptr;
    for (int k = 0; k < t->tilenum; ++k) {
        const int p = prec ? (*prec)[k] : MF_PREC_FP64;
        r->tile_value_bytes[p] += (double)t->h_tile_nnz[k] * prec_width(p);
    }
    r->tile_total_bytes = r->tile_index_bytes;
    for (int p = 0; p < 4; ++p) r->tile_total_bytes += r->tile_value_bytes[p];
    r->slab_bytes_fp64 = (double)t->L64.bytes;
    for (int l = 0; l < MF_NLEVELS; ++l)
        if (t->Lmix[l].built) r->slab_bytes_mixed += (double)t->Lmix[l].bytes;
    double d = dev_bytes(t->tile_ptr) + dev_bytes(t->tile_col) + dev_bytes(t->tile_off) + dev_bytes(t->csrptr_off) +
               dev_bytes(t->val) + dev_bytes(t->val_low) + dev_bytes(t->col) + dev_bytes(t->ptr) +
               dev_bytes(t->blknnznnz) + dev_bytes(t->nonzero_row_new) + dev_bytes(t->tile_rowidx) +
               dev_bytes(t->block_signal) + dev_bytes(t->blockrowid_new) + dev_bytes(t->blockcsr_ptr_new) +
               dev_bytes(t->diag) + layout_dev_bytes(t->L64);
    for (int l = 0; l < MF_NLEVELS; ++l) d += layout_dev_bytes(t->Lmix[l]);
    d += layout_dev_bytes(t->Lbicg);
    r->workspace_bytes = dev_bytes(t->ws) + dev_bytes(t->sync) + dev_bytes(t->xpad) + dev_bytes(t->x32buf) +
                         dev_bytes(t->trace);
    r->device_bytes = d + r->workspace_bytes;
    return MF_OK;
}

int mf_tiles_export(const mf_tiles *t, mf_tile_arrays *h) {
    if (!t || !h) return MF_ERR_ARG;
    const size_t tn = (size_t)t->tilenum;
    int rc = MF_OK;
    rc |= d2h(h->tile_ptr, t->tile_ptr.p, (size_t)t->tilem + 1);
    rc |= d2h(h->tile_columnidx, t->tile_col.p, tn);
    rc |= d2h(h->tile_nnz, t->tile_off.p, tn + 1);
    rc |= d2h(h->blknnz, t->tile_off.p, tn + 1);
    rc |= d2h(h->csr_offset, t->tile_off.p, tn + 1);
    rc |= d2h(h->csrptr_offset, t->csrptr_off.p, tn + 1);
    rc |= d2h(h->blknnznnz, t->blknnznnz.p, tn + 1);
    rc |= d2h(h->Blockcsr_Val, t->val.p, (size_t)t->csrsize);
    rc |= d2h(h->Blockcsr_Val_Low, t->val_low.p, (size_t)t->csrsize);
    rc |= d2h(h->Tile_csr_Col, t->col.p, (size_t)t->csrsize);
    rc |= d2h(h->Blockcsr_Ptr, t->ptr.p, (size_t)t->csrptrlen);
    rc |= d2h(h->ptroffset1, t->tile_off.p, tn);
    rc |= d2h(h->ptroffset2, t->csrptr_off.p, tn);
    rc |= d2h(h->tile_rowidx, t->tile_rowidx.p, tn);
    rc |= d2h(h->nonzero_row_new, t->nonzero_row_new.p, tn + 1);
    rc |= d2h(h->block_signal, t->block_signal.p, (size_t)t->tilem + 1);
    rc |= d2h(h->blockrowid_new, t->blockrowid_new.p, (size_t)t->cnt_non_new + 1);
    rc |= d2h(h->blockcsr_ptr_new, t->blockcsr_ptr_new.p, (size_t)t->cnt_non_new + 1);
    if (rc != MF_OK) return MF_ERR_CUDA;
    if (h->Format) std::memset(h->Format, 0, tn);
    if (h->csr_compressedIdx) std::memset(h->csr_compressedIdx, 0, ((size_t)t->csrsize + 1) / 2);
    // A 1-row tail block: Tile_create's exclusive_scan_char leaves the row
    // count in the pointer and step 4 then copies no values for it
    // (csr2block.h:237-251, utils.h:52-53). The device keeps correct tiles;
    // the export reproduces the reference arrays.
    const int rl_last = t->rowA - (t->tilem - 1) * 16;
    if (rl_last == 1) {
        std::vector<int> tp(2), off(2);
        cudaMemcpy(tp.data(), t->tile_ptr.p + t->tilem - 1, 2 * sizeof(int), cudaMemcpyDeviceToHost);
        for (int k = tp[0]; k < tp[1]; ++k) {
            int o[2];
            cudaMemcpy(o, t->tile_off.p + k, 2 * sizeof(int), cudaMemcpyDeviceToHost);
            int cc = 0;
            cudaMemcpy(&cc, t->csrptr_off.p + k, sizeof(int), cudaMemcpyDeviceToHost);
            if (h->Blockcsr_Ptr) h->Blockcsr_Ptr[cc] = (unsigned char)(o[1] - o[0]);
            for (int q = o[0]; q < o[1]; ++q) {
                if (h->Blockcsr_Val) h->Blockcsr_Val[q] = 0.0;
                if (h->Blockcsr_Val_Low) h->Blockcsr_Val_Low[q] = 0.0f;
                if (h->Tile_csr_Col) h->Tile_csr_Col[q] = 0;
            }
        }
    }
    return MF_OK;
}

int mf_tiles_precisions(const mf_tiles *t, unsigned char *prec, float *scale) {
    if (!t) return MF_ERR_ARG;
    const Layout *L = &t->L64;
    for (int l = MF_NLEVELS - 1; l >= 0; --l)
        if (t->mixed_ready && t->Lmix[l].built) {
            L = &t->Lmix[0];
            break;
        }
    if (prec) std::memcpy(prec, L->prec.data(), L->prec.size());
    if (scale && t->tilenum > 0)
        MF_CUDA_TRY(cudaMemcpy(scale, L->scale_dev.p, sizeof(float) * t->tilenum, cudaMemcpyDeviceToHost));
    return MF_OK;
}

int mf_tiles_set_precisions(mf_tiles *t, const unsigned char *prec) {
    if (!t || !prec) return MF_ERR_ARG;
    std::vector<uint8_t> p(prec, prec + t->tilenum);
    for (auto &v : p)
        if (v > MF_PREC_FP8) return MF_ERR_ARG;
    int rc = build_layout(t, t->Lmix[0], p, 0);
    if (rc) return rc;
    for (int l = 1; l < MF_NLEVELS; ++l) t->Lmix[l].built = false;
    t->Lbicg.built = false;
    t->nlevels = 1;
    t->level_switch[0] = 0.0;
    t->mixed_ready = true;
    return MF_OK;
}

// ------------------------------------------------------------------ SpMV
static int prepare_x(mf_tiles *t, int level, const double *x, const void **xs, cudaStream_t st = 0) {
    // the x stage reads whole 16-entry segments: use x directly when it is
    // 16-byte aligned and covers every segment, else a padded copy
    const size_t need = (size_t)t->tilen * 16;
    if (level >= 0 && level < MF_NLEVELS && t->mixed_ready && t->Lmix[level].x32) {
        // the layout stages x in FP32: a rounded, zero-padded copy
        if (t->x32buf.n < need && t->x32buf.alloc(need)) return MF_ERR_NOMEM;
        int rc = launch_to_f32(t->colA, x, t->x32buf.p, need, st);
        if (rc) return rc;
        *xs = t->x32buf.p;
        return MF_OK;
    }
    if (((uintptr_t)x & 15u) == 0 && (size_t)t->colA == need) {
        *xs = x;
        return MF_OK;
    }
    if (t->xpad.n < need && t->xpad.alloc(need)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->xpad.p, 0, need * sizeof(double), st));
    MF_CUDA_TRY(cudaMemcpyAsync(t->xpad.p, x, (size_t)t->colA * sizeof(double), cudaMemcpyDeviceToDevice, st));
    *xs = t->xpad.p;
    return MF_OK;
}

int mf_spmv(const mf_tiles *tc, const double *x, double *y, void *stream) {
    mf_tiles *t = const_cast<mf_tiles *>(tc);
    if (!t || !x || !y) return MF_ERR_ARG;
    const void *xs;
    int rc = prepare_x(t, -1, x, &xs, (cudaStream_t)stream);
    if (rc) return rc;
    rc = launch_spmv(t, -1, xs, y, 1, (cudaStream_t)stream);
    if (rc) return rc;
    MF_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return MF_OK;
}

int mf_spmv_level(const mf_tiles *tc, int level, const double *x, double *y) {
    mf_tiles *t = const_cast<mf_tiles *>(tc);
    if (!t || !x || !y) return MF_ERR_ARG;
    const void *xs;
    int rc = prepare_x(t, level, x, &xs);
    if (rc) return rc;
    rc = launch_spmv(t, level, xs, y, 1, 0);
    if (rc) return rc;
    MF_CUDA_TRY(cudaDeviceSynchronize());
    return MF_OK;
}

int mf_spmv_host(const mf_tiles *t, const double *x, double *y) {
    if (!t || !x || !y) return MF_ERR_ARG;
    DevArray<double> dx, dy;
    if (dx.alloc((size_t)t->tilen * 16) || dy.alloc((size_t)t->tilem * 16)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemset(dx.p, 0, sizeof(double) * t->tilen * 16));
    MF_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(double) * t->colA, cudaMemcpyHostToDevice));
    int rc = mf_spmv(t, dx.p, dy.p, nullptr);
    if (rc) return rc;
    MF_CUDA_TRY(cudaMemcpy(y, dy.p, sizeof(double) * t->rowA, cudaMemcpyDeviceToHost));
    return MF_OK;
}

int mf_spmv_bench_level(const mf_tiles *tc, int level, const double *x, double *y, int reps, double *ms,
                        double *alg_bytes) {
    mf_tiles *t = const_cast<mf_tiles *>(tc);
    if (!t || !x || !y || reps <= 0) return MF_ERR_ARG;
    const void *xs;
    int rc = prepare_x(t, level, x, &xs);  // outside the timed launches
    if (rc) return rc;
    // warm-up
    if ((rc = launch_spmv(t, level, xs, y, 1, 0))) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps; ++i)
        if ((rc = launch_spmv(t, level, xs, y, 1, 0))) return rc;
    cudaEventRecord(e1, 0);
    MF_CUDA_TRY(cudaEventSynchronize(e1));
    float f = 0;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = f / reps;
    if (alg_bytes) *alg_bytes = level >= 0 ? t->Lmix[level].alg_bytes : t->L64.alg_bytes;
    return MF_OK;
}

int mf_spmv_bench(const mf_tiles *t, const double *x, double *y, int reps, double *ms, double *alg_bytes) {
    return mf_spmv_bench_level(t, -1, x, y, reps, ms, alg_bytes);
}

// --------------------------------------------------------------- solvers
static int ensure_workspace(mf_tiles *t) {
    const size_t n16 = (size_t)t->tilem * 16;
    const size_t need = 9 * n16 + 2 * 4 * (size_t)t->G + 64;  // 8 vectors + the FP32 pair
    if (t->ws.n < need) {
        if (t->ws.alloc(need)) return MF_ERR_NOMEM;
    }
    const size_t sw = sync_words(t->G) + sizeof(DevResult) / 4 + 8;
    if (t->sync.n < sw) {
        if (t->sync.alloc(sw)) return MF_ERR_NOMEM;
    }
    return MF_OK;
}

struct WsView {
    double *b, *x, *r, *d, *q, *s, *t, *rh, *partial;
    float *p32, *s32;  // FP32 SpMV inputs of the mixed BiCGSTAB
    DevResult *res;
};

static WsView ws_view(mf_tiles *t) {
    const size_t n16 = (size_t)t->tilem * 16;
    WsView v;
    double *w = t->ws.p;
    v.b = w;
    v.x = w + n16;
    v.r = w + 2 * n16;
    v.d = w + 3 * n16;
    v.q = w + 4 * n16;
    v.s = w + 5 * n16;
    v.t = w + 6 * n16;
    v.rh = w + 7 * n16;
    v.p32 = reinterpret_cast<float *>(w + 8 * n16);
    v.s32 = v.p32 + n16;
    v.partial = w + 9 * n16;
    v.res = reinterpret_cast<DevResult *>(t->sync.p + sync_words(t->G));
    return v;
}

static int true_residual_ws(mf_tiles *t, const double *b, const double *x, double *rel) {
    // ax into the q slot of the workspace, norms into the partial area tail
    WsView v = ws_view(t);
    int rc = launch_spmv(t, -1, x, v.q, 1, 0);
    if (rc) return rc;
    double *out = v.partial + 2 * 4 * t->G;
    if ((rc = launch_residual_norms(t->rowA, b, v.q, out, 0))) return rc;
    double h[2];
    MF_CUDA_TRY(cudaMemcpy(h, out, sizeof h, cudaMemcpyDeviceToHost));
    *rel = h[1] > 0 ? std::sqrt(h[0]) / std::sqrt(h[1]) : std::sqrt(h[0]);
    return MF_OK;
}

// kind 0 = CG, 1 = BiCGSTAB, 2 = Jacobi-preconditioned CG (FP64 layout).
// b_dev / x_dev: n entries (device). x in: x0.
static int solve_dev_once(mf_tiles *t, int kind, const double *b_dev, double *x_dev, double tol, int maxiter,
                          const mf_options *opt_in, mf_result *res) {
    if (!t || !b_dev || !x_dev) return MF_ERR_ARG;
    if (t->rowA != t->colA) {
        set_last_error("the solvers need a square matrix");
        return MF_ERR_UNSUPPORTED;
    }
    mf_options opt = opt_in ? *opt_in : t->opt;
    int rc = ensure_workspace(t);
    if (rc) return rc;
    WsView v = ws_view(t);
    const size_t n16 = (size_t)t->tilem * 16;
    const int n = t->rowA;
    MF_CUDA_TRY(cudaMemsetAsync(t->ws.p, 0, sizeof(double) * 9 * n16));
    MF_CUDA_TRY(cudaMemcpyAsync(v.b, b_dev, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    MF_CUDA_TRY(cudaMemcpyAsync(v.x, x_dev, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    MF_CUDA_TRY(cudaMemsetAsync(t->sync.p, 0, sizeof(uint32_t) * t->sync.n));
    KParams P;
    base_params(t, P);
    if (opt.timeout_s > 0) P.limit_ns = (uint64_t)(opt.timeout_s * 1e9);
    P.sync = t->sync.p;
    P.partial = v.partial;
    P.b = v.b;
    P.x = v.x;
    P.r = v.r;
    P.d = v.d;
    P.q = v.q;
    P.s = v.s;
    P.t = v.t;
    P.rh = v.rh;
    P.p32 = v.p32;
    P.s32 = v.s32;
    P.tol = tol;
    P.maxiter = maxiter;
    P.fixed_iterations = opt.fixed_iterations;
    P.replace_every = opt.replace_every;
    P.res = v.res;
    P.inject_wait = opt.reserved[0] == 0x5741 ? 1 : 0;
    P.prefetch = opt.reserved[3] == 1 ? 1 : 0;
    if (opt.reserved[1] > 0) {
        const int ti = opt.reserved[1] > 4096 ? 4096 : opt.reserved[1];
        if (t->trace.n < (size_t)ti * 8 && t->trace.alloc((size_t)ti * 8)) return MF_ERR_NOMEM;
        MF_CUDA_TRY(cudaMemsetAsync(t->trace.p, 0, sizeof(uint64_t) * ti * 8));
        P.trace = t->trace.p;
        P.trace_iters = ti;
        t->trace_iters = ti;
    }
    // A mixed solve whose levels hold no tile below FP64 (every row block
    // oversize, for example) gains nothing from the low-precision kernels
    // and runs the FP64 solver: the single-reduction CG keeps its search
    // directions in FP32, which only pays with a low-precision operator.
    bool any_low = false;
    for (int l = 0; l < MF_NLEVELS; ++l)
        if (t->Lmix[l].built && t->Lmix[l].kind != LAYOUT_FP64) any_low = true;
    const bool mixed =
        (kind == 0 || kind == 1) && opt.precision_mode != MF_MODE_FP64 && t->mixed_ready && any_low;
    const Layout *lv[MF_NLEVELS] = {nullptr, nullptr, nullptr};  // the mixed levels this solve runs
    if (mixed) {
        int nl = 1;
        auto add_level = [&](const Layout &L, double rel) {
            lv[nl - 1] = &L;
            LayoutArgs &a = P.lay[nl];
            a.slabs = L.slabs.p;
            a.head = L.head.p;
            a.cta_slab = L.cta_slab.p;
            a.cta_rb = L.cta_rb.p;
            a.cta_dep = L.cta_dep.p;
            a.kind = L.kind;
            a.x32 = L.x32 ? 1 : 0;
            P.level_rel[nl] = rel;
            ++nl;
        };
        bool below32 = false;
        for (int l = 0; l < t->nlevels && t->Lmix[l].built; ++l)
            for (auto p : t->Lmix[l].prec) below32 = below32 || p > MF_PREC_FP32;
        if (kind == 1 && below32) {
            if (!t->Lbicg.built) {
                std::vector<uint8_t> p32(t->Lmix[0].prec);
                for (auto &p : p32)
                    if (p > MF_PREC_FP32) p = MF_PREC_FP32;
                if ((rc = build_layout(t, t->Lbicg, p32, 0)) != MF_OK) return rc;
            }
            add_level(t->Lbicg, 0.0);
        } else {
            for (int l = 0; l < t->nlevels; ++l) {
                if (!t->Lmix[l].built) break;
                add_level(t->Lmix[l], t->level_switch[l]);
            }
        }
        P.nlay = nl;
        P.start_layout = 1;
        P.true_check = 1;
        if (P.replace_every <= 0) P.replace_every = 50;
    } else {
        P.replace_every = 0;  // the FP64 recurrence of the reference never replaces
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    // mixed layouts run the single-reduction CG unless the classic
    // recurrence is asked for (mf_options.reserved[2] == 1)
    if (kind == 2) {
        int rj = launch_jacobi_inv(n, (int)n16, t->diag.p, v.s, 0);
        if (rj) return rj;
    }
    int launch_kind = kind == 2 ? 4 : (mixed && kind == 0 && opt.reserved[2] != 1) ? 2 : kind;
    // x and r stay in tensor memory when every CTA's rows fit it, the ring
    // holds the vector passes' copies, and one CTA runs per SM (each CTA
    // allocates all of the SM's tensor memory)
    if ((launch_kind == 2 || launch_kind == 4 || (launch_kind == 0 && !mixed)) && opt.reserved[5] != 1 &&
        t->G == t->nsm) {
        int rows_max = 0;
        for (size_t g = 0; g + 1 < t->h_cta_rb.size(); ++g)
            rows_max = std::max(rows_max, 16 * (t->h_cta_rb[g + 1] - t->h_cta_rb[g]));
        const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
        if (rows_max <= TMEM_ROWS_MAX && tm_vectors_fit(rows_max, slab_max))
            launch_kind = launch_kind == 2 ? 3 : launch_kind == 4 ? 6 : 5;
    }
    if (launch_kind == 6) {
        // the tensor-memory PCG applies 1/a_ii from an FP32 copy: only when
        // every 1/a_ii is an FP32 normal number (checked once per handle)
        if (t->minv_f32_ok < 0) {
            double lo = 0.0, hi = 0.0;
            if ((rc = abs_range(v.s, (long long)n16, &lo, &hi, 0)) != MF_OK) return rc;
            t->minv_f32_ok = (lo == 0.0 || lo >= 1.2e-38) && hi <= 3.0e38 ? 1 : 0;
        }
        if (!t->minv_f32_ok) launch_kind = 4;
    }
    if (launch_kind == 6) {  // the FP32 copy of 1/a_ii that the ring copies carry
        int rj = launch_to_f32((int)n16, v.s, v.p32, n16, 0);
        if (rj) return rj;
    }
    rc = launch_solver(t, launch_kind, P, 0);
    cudaEventRecord(e1, 0);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (ce != cudaSuccess) {
        set_last_error(cudaGetErrorString(ce));
        return MF_ERR_CUDA;
    }
    DevResult dr;
    uint32_t err[2];
    MF_CUDA_TRY(cudaMemcpy(&dr, v.res, sizeof dr, cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(err, t->sync.p + SYNC_ERROR, sizeof err, cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(x_dev, v.x, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    int status = err[0] ? (int)err[0] : dr.status;
    mf_result R;
    std::memset(&R, 0, sizeof R);
    R.status = status;
    R.iterations = err[0] ? -1 : dr.iterations;
    R.replacements = dr.replacements;
    R.level_switches = dr.level_switches;
    R.error_site = (int)err[1];
    R.rel_residual_rec = dr.bb > 0 ? std::sqrt(dr.rr) / std::sqrt(dr.bb) : std::sqrt(dr.rr);
    R.time_ms = ms;
    R.spmv_bytes_fp64 = t->L64.alg_bytes;
    const Layout *Lf = &t->L64;
    if (mixed && dr.final_layout >= 1 && dr.final_layout <= MF_NLEVELS && lv[dr.final_layout - 1])
        Lf = lv[dr.final_layout - 1];
    R.spmv_bytes = Lf->alg_bytes;
    for (int p = 0; p < 4; ++p) R.tile_frac[p] = Lf->tile_frac[p];
    R.iters_fp64 = dr.it_layout[0];
    R.fell_back_fp64 = kind <= 1 ? dr.pad : 0;
    for (int l = 0; l < 3; ++l) {
        R.iters_level[l] = dr.it_layout[l + 1];
        R.spmv_bytes_level[l] = (mixed && lv[l]) ? lv[l]->alg_bytes : 0.0;
    }
    {
        // per iteration: the SpMVs' algorithmic bytes + the vector bytes the
        // launched kernel moves per row (the SpMVs count their own x and y):
        // BiCGSTAB (two SpMVs) FP64 112 (r^ in both SpMV epilogues and s in
        // the second; s pass: r, v in, s out; x, r, p pass: s, x, p, t, v
        // in, x, r, p out), mixed 136 (s from global memory, three vector
        // passes, FP32 copies of s and p out); CG with
        // vectors in global memory 56 (x, r, d, q; single-reduction CG
        // likewise), Jacobi PCG 72 (+ 1/a_ii); with x and r in tensor memory:
        // single-reduction CG 28 (p, s, w in; p, s and the FP32 copy of r
        // out; w from the SpMV), FP64 CG 32 (q, d in; q, d out), Jacobi PCG
        // 40 (q, d and the FP32 1/a_ii twice in; q, d out)
        const double vpr = kind == 1 ? (P.nlay > 1 ? 136.0 : 112.0)
                           : launch_kind == 3 ? 28.0
                           : launch_kind == 5 ? 32.0
                           : launch_kind == 6 ? 40.0
                           : launch_kind == 4 ? 72.0
                                              : 56.0;
        const double vec = vpr * (double)n;
        const double nsp = kind == 1 ? 2.0 : 1.0;
        double tb = (double)(1 + dr.replacements) * (t->L64.alg_bytes + 16.0 * n);  // initial + replacements
        tb += (double)dr.it_layout[0] * (nsp * t->L64.alg_bytes + vec);
        for (int l = 0; l < 3; ++l) tb += (double)dr.it_layout[l + 1] * (nsp * R.spmv_bytes_level[l] + vec);
        R.total_bytes = tb;
    }
    R.rel_residual_true = NAN;
    if (!err[0] && opt.check_true_residual) {
        double rel = 0;
        int rc2 = true_residual_ws(t, v.b, v.x, &rel);
        if (rc2) return rc2;
        R.rel_residual_true = rel;
    }
    if (res) *res = R;
    return status;
}

// With the learned selector's layouts, a CG solve that misses the tolerance,
// falls back to the FP64 layout, or runs more than 10% over the reference
// iteration count (mf_options.reserved[6]) is solved again from the same x0
// with layouts from the magnitude rule, which this handle keeps afterwards.
static int solve_dev(mf_tiles *t, int kind, const double *b_dev, double *x_dev, double tol, int maxiter,
                     const mf_options *opt_in, mf_result *res) {
    if (!t || !b_dev || !x_dev) return MF_ERR_ARG;
    const mf_options opt = opt_in ? *opt_in : t->opt;
    const bool mlp = kind == 0 && t->mixed_ready && t->opt.precision_mode == MF_MODE_MIXED_MLP &&
                     opt.precision_mode != MF_MODE_FP64;
    if (!mlp) return solve_dev_once(t, kind, b_dev, x_dev, tol, maxiter, opt_in, res);
    DevArray<double> x0;
    if (x0.alloc((size_t)t->rowA)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpy(x0.p, x_dev, sizeof(double) * t->rowA, cudaMemcpyDeviceToDevice));
    mf_result R;
    std::memset(&R, 0, sizeof R);
    int rc = solve_dev_once(t, kind, b_dev, x_dev, tol, maxiter, opt_in, &R);
    const int ref = opt.reserved[6];
    const bool solved = rc == MF_OK || rc == MF_ERR_NOT_CONVERGED || rc == MF_ERR_BREAKDOWN;
    const bool bad = rc == MF_ERR_NOT_CONVERGED || rc == MF_ERR_BREAKDOWN || R.fell_back_fp64 ||
                     (ref > 0 && R.iterations > 1.1 * ref);
    if (solved && bad) {
        t->opt.precision_mode = MF_MODE_MIXED_RULE;
        if ((rc = build_mixed_levels(t, 0)) != MF_OK) return rc;
        MF_CUDA_TRY(cudaMemcpy(x_dev, x0.p, sizeof(double) * t->rowA, cudaMemcpyDeviceToDevice));
        mf_options o2 = opt;
        o2.precision_mode = MF_MODE_MIXED_RULE;
        const double first_ms = R.time_ms;
        std::memset(&R, 0, sizeof R);
        rc = solve_dev_once(t, kind, b_dev, x_dev, tol, maxiter, &o2, &R);
        R.selector_fallback = 1;
        R.time_ms += first_ms;  // both solves
    }
    if (res) *res = R;
    return rc;
}

// Re-plans the handle's layouts (FP64 and, when present, the mixed levels)
// with the candidate slab geometry and returns the time of the SpMV the
// solvers run (the mixed level 0 when present, else FP64), averaged over
// reps launches.
static int tune_candidate(mf_tiles *t, int slab_bytes, int rbps, int reps, double *ms) {
    t->opt.slab_bytes = slab_bytes;
    t->opt.rb_per_slab = rbps;
    int G = 0, rc;
    if ((rc = kernel_config(t, &G)) != MF_OK) return rc;
    std::vector<uint8_t> prec(t->tilenum, MF_PREC_FP64);
    if ((rc = build_layout(t, t->L64, prec, 0)) != MF_OK) return rc;
    const bool mixed = t->opt.precision_mode != MF_MODE_FP64;
    if (mixed && (rc = build_mixed_levels(t, 0)) != MF_OK) return rc;
    const int level = (mixed && t->mixed_ready) ? 0 : -1;
    if ((rc = ensure_workspace(t)) != MF_OK) return rc;
    WsView v = ws_view(t);
    const size_t n16 = (size_t)t->tilen * 16;
    MF_CUDA_TRY(cudaMemsetAsync(v.x, 0, sizeof(double) * n16));
    const void *xs;
    if ((rc = prepare_x(t, level, v.x, &xs)) != MF_OK) return rc;
    if ((rc = launch_spmv(t, level, xs, v.q, 1, 0)) != MF_OK) return rc;  // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps && rc == MF_OK; ++i) rc = launch_spmv(t, level, xs, v.q, 1, 0);
    cudaEventRecord(e1, 0);
    cudaError_t ce = cudaEventSynchronize(e1);
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (ce != cudaSuccess) {
        set_last_error(cudaGetErrorString(ce));
        return MF_ERR_CUDA;
    }
    *ms = f / reps;
    return MF_OK;
}

int mf_tiles_autotune(mf_tiles *t, int reps, mf_tune_result *out) {
    if (!t || !out) return MF_ERR_ARG;
    if (reps <= 0) reps = 20;
    MF_CUDA_TRY(cudaSetDevice(t->opt.device));
    std::memset(out, 0, sizeof *out);
    static const int kSlab[] = {24576, 32768, 40960};
    static const int kRb[] = {16, 30, 60, 120};
    double best = 1e30;
    int bsb = 0, brb = 0;
    for (int sb : kSlab)
        for (int rb : kRb) {
            double ms = 0;
            const int rc = tune_candidate(t, sb, rb, reps, &ms);
            if (rc == MF_ERR_ARG) continue;  // does not fit shared memory
            if (rc) return rc;
            const int k = out->candidates++;
            out->cand_slab_bytes[k] = sb;
            out->cand_rb_per_slab[k] = rb;
            out->cand_ms[k] = ms;
            if (sb == SLAB_MAX_DEFAULT && rb == (t->opt.precision_mode != MF_MODE_FP64 ? RB_PER_SLAB_X32
                                                                                        : RB_PER_SLAB_X64))
                out->ms_default = ms;
            if (ms < best) {
                best = ms;
                bsb = sb;
                brb = rb;
            }
        }
    if (out->candidates == 0) return MF_ERR_RESIDENCY;
    double ms = 0;
    int rc = tune_candidate(t, bsb, brb, reps, &ms);  // leave the handle on the choice
    if (rc) return rc;
    out->slab_bytes = bsb;
    out->rb_per_slab = brb;
    out->ms_best = best;
    return MF_OK;
}

int mf_solve_cg_dev(mf_tiles *t, const double *b, double *x, double tol, int maxiter, const mf_options *opt,
                    mf_result *res) {
    return solve_dev(t, 0, b, x, tol, maxiter, opt, res);
}
int mf_solve_pcg_dev(mf_tiles *t, const double *b, double *x, double tol, int maxiter, const mf_options *opt,
                     mf_result *res) {
    return solve_dev(t, 2, b, x, tol, maxiter, opt, res);
}
int mf_solve_bicgstab_dev(mf_tiles *t, const double *b, double *x, double tol, int maxiter,
                          const mf_options *opt, mf_result *res) {
    return solve_dev(t, 1, b, x, tol, maxiter, opt, res);
}

static int solve_host(mf_tiles *t, int kind, const double *b, double *x, double tol, int maxiter,
                      const mf_options *opt, mf_result *res) {
    if (!t || !b || !x) return MF_ERR_ARG;
    DevArray<double> db, dx;
    if (db.alloc(t->rowA) || dx.alloc(t->rowA)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpy(db.p, b, sizeof(double) * t->rowA, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(double) * t->rowA, cudaMemcpyHostToDevice));
    int rc = solve_dev(t, kind, db.p, dx.p, tol, maxiter, opt, res);
    if (rc == MF_OK || rc == MF_ERR_NOT_CONVERGED || rc == MF_ERR_BREAKDOWN)
        MF_CUDA_TRY(cudaMemcpy(x, dx.p, sizeof(double) * t->rowA, cudaMemcpyDeviceToHost));
    return rc;
}

int mf_solve_cg(mf_tiles *t, const double *b, double *x, double tol, int maxiter, const mf_options *opt,
                mf_result *res) {
    return solve_host(t, 0, b, x, tol, maxiter, opt, res);
}
int mf_solve_pcg(mf_tiles *t, const double *b, double *x, double tol, int maxiter, const mf_options *opt,
                 mf_result *res) {
    return solve_host(t, 2, b, x, tol, maxiter, opt, res);
}
int mf_solve_bicgstab(mf_tiles *t, const double *b, double *x, double tol, int maxiter, const mf_options *opt,
                      mf_result *res) {
    return solve_host(t, 1, b, x, tol, maxiter, opt, res);
}

int mf_trace(const mf_tiles *t, unsigned long long *out, int max_iters) {
    if (!t || !out || max_iters <= 0) return MF_ERR_ARG;
    const int n = std::min(max_iters, t->trace_iters);
    if (n <= 0) return 0;
    MF_CUDA_TRY(cudaMemcpy(out, t->trace.p, sizeof(uint64_t) * 8 * n, cudaMemcpyDeviceToHost));
    return n;
}

int mf_true_residual(mf_tiles *t, const double *b, const double *x, double *rel) {
    if (!t || !b || !x || !rel) return MF_ERR_ARG;
    int rc = ensure_workspace(t);
    if (rc) return rc;
    WsView v = ws_view(t);
    const size_t n16 = (size_t)t->tilem * 16;
    MF_CUDA_TRY(cudaMemset(v.x, 0, sizeof(double) * n16));
    MF_CUDA_TRY(cudaMemcpy(v.x, x, sizeof(double) * t->rowA, cudaMemcpyDeviceToDevice));
    return true_residual_ws(t, b, v.x, rel);
}

}  // extern "C"
