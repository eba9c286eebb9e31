// GPU csr2block: encodes a CSR matrix into the 16x16 tile arrays of
// Tile_create (Performance-Comparison/csr2block.h:267-422), bit-exact, plus the
// row-compression arrays of the CG driver (Mille-feuille_CG_NVIDIA.cu:4154-4213).
//
// Per row block (16 rows) the entries are sorted by (tile column, CSR
// position). Because CSR order is row-major, that order is exactly the
// reference's value order: tiles in ascending column, rows inside a tile in
// order, entries of a row in CSR order. Row block rb's values therefore
// occupy [row_ptr[16 rb], row_ptr[16 rb + 16]) of Blockcsr_Val, so no value
// offsets need a scan; only the tile counts do.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "tiles.h"

namespace mf {

namespace {

constexpr int ENC_THREADS = 256;
constexpr int ENC_CAP = 2048;  // entries of a row block sorted in shared memory

// ---- exclusive scan (int32, in place) ------------------------------------
constexpr int SCAN_T = 256, SCAN_PER = 4, SCAN_CHUNK = SCAN_T * SCAN_PER;

__device__ int block_excl_scan(int v, int *sh, int &total) {
    // sh: SCAN_T ints
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < (SCAN_T / 32) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_T / 32) sh[lane] = s;
    }
    __syncthreads();
    const int base = w > 0 ? sh[w - 1] : 0;
    total = sh[SCAN_T / 32 - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void scan_block_sums(const int *d, long long n, int *sums) {
    __shared__ int sh[SCAN_T];
    const long long base = (long long)blockIdx.x * SCAN_CHUNK;
    int s = 0;
    for (int k = 0; k < SCAN_PER; ++k) {
        long long i = base + (long long)threadIdx.x * SCAN_PER + k;
        if (i < n) s += d[i];
    }
    int total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_sums_serial(int *sums, long long nb) {
    __shared__ int sh[SCAN_T];
    int carry = 0;
    for (long long c = 0; c < nb; c += SCAN_T) {
        long long i = c + threadIdx.x;
        int v = i < nb ? sums[i] : 0;
        int total;
        int ex = block_excl_scan(v, sh, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void scan_apply(int *d, long long n, const int *sums) {
    __shared__ int sh[SCAN_T];
    const long long base = (long long)blockIdx.x * SCAN_CHUNK + (long long)threadIdx.x * SCAN_PER;
    int v[SCAN_PER];
    int s = 0;
    for (int k = 0; k < SCAN_PER; ++k) {
        v[k] = (base + k < n) ? d[base + k] : 0;
        s += v[k];
    }
    int total;
    int ex = block_excl_scan(s, sh, total) + sums[blockIdx.x];
    for (int k = 0; k < SCAN_PER; ++k) {
        if (base + k < n) d[base + k] = ex;
        ex += v[k];
    }
}

// ---- encoder ------------------------------------------------------------------
__device__ __forceinline__ int rb_end_row(int rb, int tilem, int rowA) {
    return rb == tilem - 1 ? rowA : (rb + 1) * 16;
}

// Bitonic sort of P (power of two) 64-bit keys by one CTA.
__device__ void bitonic_sort(unsigned long long *key, int P) {
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = key[i], b = key[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        key[i] = b;
                        key[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
}

// Pass 1: sort the row block's entries by (tile column, local position) and
// count its distinct tile columns (csr2block.h:6-41).
__global__ void __launch_bounds__(ENC_THREADS) enc_sort_count(int rowA, int tilem, const int *__restrict__ rp,
                                                              const int *__restrict__ ci, int *__restrict__ perm,
                                                              int *__restrict__ tile_count,
                                                              unsigned long long *__restrict__ gkeys,
                                                              long long gkeys_cap, int big_only, int rb_base) {
    __shared__ unsigned long long skey[ENC_CAP];
    __shared__ int sred[ENC_THREADS / 32];
    const int rb = rb_base + blockIdx.x;
    if (rb >= tilem) return;
    const int start = rp[rb * 16];
    const int m = rp[rb_end_row(rb, tilem, rowA)] - start;
    const bool big = m > ENC_CAP;
    if (big != (big_only != 0)) return;
    int P = 1;
    while (P < m) P <<= 1;
    unsigned long long *key = skey;
    if (big) {
        if ((long long)P > gkeys_cap) return;  // host sized gkeys for the largest row block
        key = gkeys;
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x)
        key[i] = i < m ? (((unsigned long long)(unsigned)(ci[start + i] >> 4)) << 32) | (unsigned)i
                       : ~0ull;
    __syncthreads();
    bitonic_sort(key, P);
    int cnt = 0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        perm[start + i] = (int)(key[i] & 0xffffffffu);
        if (i == 0 || (key[i] >> 32) != (key[i - 1] >> 32)) ++cnt;
    }
    // block sum of cnt
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < ENC_THREADS / 32; ++w) s += sred[w];
        tile_count[rb] = s;
    }
}

// Pass 2: scatter values / columns / row pointers of every tile
// (csr2block.h:43-107 and :152-265) using the sorted order of pass 1.
__global__ void __launch_bounds__(ENC_THREADS) enc_emit(int rowA, int tilem, const int *__restrict__ rp,
                                                        const int *__restrict__ ci, const double *__restrict__ val,
                                                        const int *__restrict__ perm, const int *__restrict__ tile_ptr,
                                                        int *__restrict__ tile_col, int *__restrict__ tile_cnt,
                                                        unsigned char *__restrict__ blknnznnz,
                                                        double *__restrict__ bval, float *__restrict__ bval_low,
                                                        unsigned char *__restrict__ bcol,
                                                        unsigned char *__restrict__ bptr, int *__restrict__ gfirst,
                                                        unsigned char *__restrict__ grow, int big_only,
                                                        int rb_base) {
    __shared__ int sfirst[ENC_CAP + 1];
    __shared__ unsigned char srow[ENC_CAP];
    __shared__ int srp[17];
    __shared__ int sh[SCAN_T];
    const int rb = rb_base + blockIdx.x;
    if (rb >= tilem) return;
    const int r0 = rb * 16;
    const int r1 = rb_end_row(rb, tilem, rowA);
    const int rowlen = r1 - r0;
    const int start = rp[r0];
    const int m = rp[r1] - start;
    const bool big = m > ENC_CAP;
    if (big != (big_only != 0)) return;
    int *first = big ? gfirst : sfirst;
    unsigned char *rowof = big ? grow : srow;
    if (threadIdx.x <= rowlen) srp[threadIdx.x] = rp[r0 + threadIdx.x] - start;
    __syncthreads();
    const int tp0 = tile_ptr[rb];
    const int ntile = tile_ptr[rb + 1] - tp0;
    const int tp_last = tile_ptr[tilem - 1];
    const int rowlen_last = rowA - (tilem - 1) * 16;
    // tile index of each sorted entry by a chunked block scan of "new tile" flags
    int carry = 0;
    for (int c = 0; c < m; c += ENC_THREADS) {
        const int i = c + threadIdx.x;
        int e = 0, tc = -1, flag = 0;
        if (i < m) {
            const int k = perm[start + i];
            e = start + k;
            tc = ci[e] >> 4;
            if (i == 0) flag = 1;
            else flag = (ci[start + perm[start + i - 1]] >> 4) != tc;
            // row of local position k
            int lo = 0, hi = rowlen - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (srp[mid] <= k) lo = mid; else hi = mid - 1;
            }
            rowof[i] = (unsigned char)lo;
            const double v = val[e];
            bval[start + i] = v;
            bval_low[start + i] = __double2float_rn(v);
            bcol[start + i] = (unsigned char)(ci[e] & 15);
        }
        int total;
        const int ex = block_excl_scan(flag, sh, total);
        if (i < m && flag) {
            const int j = carry + ex;
            tile_col[tp0 + j] = tc;
            first[j] = i;
        }
        carry += total;
    }
    if (threadIdx.x == 0) first[ntile] = m;
    __syncthreads();
    // per tile: nnz count and the row pointers (exclusive scan of row counts)
    for (int j = threadIdx.x; j < ntile; j += blockDim.x) {
        const int c = first[j + 1] - first[j];
        tile_cnt[tp0 + j] = c;
        blknnznnz[tp0 + j] = (unsigned char)c;
    }
    for (int p = threadIdx.x; p < ntile * rowlen; p += blockDim.x) {
        const int j = p / rowlen, r = p - j * rowlen;
        int lo = first[j], hi = first[j + 1];
        while (lo < hi) {  // first entry of the tile whose row >= r
            const int mid = (lo + hi) >> 1;
            if (rowof[mid] < r) lo = mid + 1; else hi = mid;
        }
        const int t = tp0 + j;
        const long long off = t < tp_last ? 16ll * t : 16ll * tp_last + (long long)rowlen_last * (t - tp_last);
        bptr[off + r] = (unsigned char)(lo - first[j]);
    }
}

__global__ void enc_rowblock_sizes(int rowA, int tilem, const int *rp, int *maxm) {
    const int rb = blockIdx.x * blockDim.x + threadIdx.x;
    if (rb >= tilem) return;
    const int m = rp[rb_end_row(rb, tilem, rowA)] - rp[rb * 16];
    atomicMax(maxm, m);
}

__global__ void enc_csrptr_offsets(int tilenum, int tilem, int rowA, const int *tile_ptr, int *csrptr_off) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t > tilenum) return;
    const int tp_last = tile_ptr[tilem - 1];
    const int rl = rowA - (tilem - 1) * 16;
    csrptr_off[t] = t <= tp_last ? (int)(16 * t) : (int)(16 * tp_last + rl * (t - tp_last));
}

// Row compression: count of non-empty rows + 1 per tile. With quirk1, the
// last row block of a 1-row tail uses the pointers Tile_create leaves there
// (exclusive_scan_char skips length 1, so ptr[0] holds the row count).
__device__ __forceinline__ void tile_row_range(int t, int ri, int rl, const int *tile_off, const int *csrptr_off,
                                               const unsigned char *bptr, int &st, int &sp) {
    const int cc = csrptr_off[t];
    const int nk = tile_off[t + 1] - tile_off[t];
    if (rl == 1) {
        st = nk;  // Tile_create keeps the unscanned count for a 1-row tail
        sp = nk;
        return;
    }
    st = bptr[cc + ri];
    sp = ri == rl - 1 ? nk : bptr[cc + ri + 1];
}

__global__ void enc_rowcomp_count(int tilenum, int tilem, int rowA, const int *tile_ptr, const int *tile_off,
                                  const int *csrptr_off, const unsigned char *bptr, int *nonzero_row_new,
                                  int *tile_rowidx) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tilenum) return;
    int lo = 0, hi = tilem - 1;  // row block of tile t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_ptr[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int rb = lo;
    const int rl = rb == tilem - 1 ? rowA - (tilem - 1) * 16 : 16;
    int c = 1;
    for (int ri = 0; ri < rl; ++ri) {
        int st, sp;
        tile_row_range(t, ri, rl, tile_off, csrptr_off, bptr, st, sp);
        if (sp != st) ++c;
    }
    nonzero_row_new[t] = c;
    tile_rowidx[t] = rb;
}

__global__ void enc_rowcomp_fill(int tilenum, int tilem, int rowA, const int *tile_off, const int *csrptr_off,
                                 const unsigned char *bptr, const int *nonzero_row_new, const int *tile_rowidx,
                                 unsigned char *rid, unsigned char *rpn) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tilenum) return;
    const int rb = tile_rowidx[t];
    const int rl = rb == tilem - 1 ? rowA - (tilem - 1) * 16 : 16;
    int base = nonzero_row_new[t], fl = 0;
    for (int ri = 0; ri < rl; ++ri) {
        int st, sp;
        tile_row_range(t, ri, rl, tile_off, csrptr_off, bptr, st, sp);
        if (ri == 0) {
            rid[base + fl] = 0;
            rpn[base + fl] = 0;
            ++fl;
        }
        if (sp != st) {
            rid[base + fl] = (unsigned char)ri;
            rpn[base + fl] = (unsigned char)sp;
            ++fl;
        }
    }
}

__global__ void enc_block_signal(int tilem, const int *tile_ptr, int *block_signal) {
    const int rb = blockIdx.x * blockDim.x + threadIdx.x;
    if (rb > tilem) return;
    block_signal[rb] = rb < tilem ? tile_ptr[rb + 1] - tile_ptr[rb] : 0;
}

__global__ void enc_diag(int rowA, const int *rp, const int *ci, const double *val, double *diag) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rowA) return;
    double d = 0.0;
    for (int p = rp[r]; p < rp[r + 1]; ++p)
        if (ci[p] == r) d += val[p];
    diag[r] = d;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

int exclusive_scan_int(int *d, long long n, cudaStream_t s) {
    if (n <= 0) return MF_OK;
    const long long nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    DevArray<int> sums;
    if (sums.alloc((size_t)nb)) return MF_ERR_NOMEM;
    scan_block_sums<<<(unsigned)nb, SCAN_T, 0, s>>>(d, n, sums.p);
    scan_sums_serial<<<1, SCAN_T, 0, s>>>(sums.p, nb);
    scan_apply<<<(unsigned)nb, SCAN_T, 0, s>>>(d, n, sums.p);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_OK;
}

// Encodes rows [0, n) of a device CSR whose columns lie in [0, ncols).
// The CSR checks every encode needs before any kernel indexes by it:
// row_ptr starts at 0, ends at nnz and never decreases; 0 <= col_idx < ncols.
__global__ void enc_validate(int n, int ncols, int nnz, const int *__restrict__ rp, const int *__restrict__ ci,
                             int *bad) {
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int b = 0;
    for (long long i = tid; i < nnz; i += stride) {
        const int c = ci[i];
        b |= (c < 0) | (c >= ncols);
    }
    for (long long i = tid; i < n; i += stride) b |= rp[i] > rp[i + 1];
    if (tid == 0) b |= (rp[0] != 0) | (rp[n] != nnz);
    if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}

int encode_device(mf_tiles *t, int n, int ncols, int nnz, const int *rp, const int *ci, const double *val,
                  cudaStream_t s) {
    const int rowA = n, colA = ncols;
    t->rowA = rowA;
    t->colA = colA;
    t->tilem = (rowA + 15) / 16;
    t->tilen = (colA + 15) / 16;
    const int tilem = t->tilem;
    t->csrsize = nnz;
    if (tilem == 0) return MF_ERR_ARG;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);

    DevArray<int> perm, maxm;
    if (perm.alloc(nnz) || maxm.alloc(2)) return MF_ERR_NOMEM;  // [0] max entries of a row block, [1] invalid CSR
    if (t->tile_ptr.alloc(tilem + 1)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->tile_ptr.p, 0, sizeof(int) * (tilem + 1), s));
    MF_CUDA_TRY(cudaMemsetAsync(maxm.p, 0, 2 * sizeof(int), s));
    enc_validate<<<592, 256, 0, s>>>(rowA, colA, nnz, rp, ci, maxm.p + 1);
    enc_rowblock_sizes<<<nblk(tilem, 256), 256, 0, s>>>(rowA, tilem, rp, maxm.p);
    int hmv[2] = {0, 0};
    MF_CUDA_TRY(cudaMemcpyAsync(hmv, maxm.p, sizeof hmv, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (hmv[1]) {
        set_last_error("invalid CSR: row_ptr must run from 0 to nnz without decreasing, col_idx within [0, ncols)");
        return MF_ERR_ARG;
    }
    const int hmax = hmv[0];
    long long cap = 1;
    while (cap < hmax) cap <<= 1;
    const bool any_big = hmax > ENC_CAP;
    DevArray<unsigned long long> gkeys;
    DevArray<int> gfirst;
    DevArray<unsigned char> grow;
    if (any_big) {
        if (gkeys.alloc((size_t)cap) || gfirst.alloc((size_t)hmax + 1) || grow.alloc((size_t)hmax))
            return MF_ERR_NOMEM;
    }
    enc_sort_count<<<tilem, ENC_THREADS, 0, s>>>(rowA, tilem, rp, ci, perm.p, t->tile_ptr.p, gkeys.p,
                                                 any_big ? cap : 0, 0, 0);
    // Row blocks with more than ENC_CAP entries share one global scratch and
    // are processed one launch each, in order.
    std::vector<int> big_rbs;
    if (any_big) {
        std::vector<int> rows(rowA + 1);
        MF_CUDA_TRY(cudaMemcpyAsync(rows.data(), rp, sizeof(int) * (rowA + 1), cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaStreamSynchronize(s));
        for (int rb = 0; rb < tilem; ++rb)
            if (rows[rb == tilem - 1 ? rowA : (rb + 1) * 16] - rows[rb * 16] > ENC_CAP) big_rbs.push_back(rb);
        for (int rb : big_rbs)
            enc_sort_count<<<1, ENC_THREADS, 0, s>>>(rowA, tilem, rp, ci, perm.p, t->tile_ptr.p, gkeys.p, cap, 1, rb);
    }
    MF_CUDA_TRY(cudaGetLastError());
    int rc = exclusive_scan_int(t->tile_ptr.p, tilem + 1, s);
    if (rc) return rc;
    int tilenum = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&tilenum, t->tile_ptr.p + tilem, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    t->tilenum = tilenum;
    const int rowlen_last = rowA - (tilem - 1) * 16;
    int tp_last = 0;
    MF_CUDA_TRY(cudaMemcpy(&tp_last, t->tile_ptr.p + tilem - 1, sizeof(int), cudaMemcpyDeviceToHost));
    t->csrptrlen = 16 * tp_last + rowlen_last * (tilenum - tp_last);

    if (t->tile_col.alloc(tilenum) || t->tile_off.alloc(tilenum + 1) || t->csrptr_off.alloc(tilenum + 1) ||
        t->val.alloc(nnz) || t->val_low.alloc(nnz) || t->col.alloc(nnz) || t->ptr.alloc(t->csrptrlen) ||
        t->blknnznnz.alloc(tilenum + 1))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->tile_off.p, 0, sizeof(int) * (tilenum + 1), s));
    MF_CUDA_TRY(cudaMemsetAsync(t->blknnznnz.p, 0, tilenum + 1, s));
    enc_emit<<<tilem, ENC_THREADS, 0, s>>>(rowA, tilem, rp, ci, val, perm.p, t->tile_ptr.p, t->tile_col.p,
                                           t->tile_off.p, t->blknnznnz.p, t->val.p, t->val_low.p, t->col.p,
                                           t->ptr.p, gfirst.p, grow.p, 0, 0);
    for (int rb : big_rbs)
        enc_emit<<<1, ENC_THREADS, 0, s>>>(rowA, tilem, rp, ci, val, perm.p, t->tile_ptr.p, t->tile_col.p,
                                           t->tile_off.p, t->blknnznnz.p, t->val.p, t->val_low.p, t->col.p,
                                           t->ptr.p, gfirst.p, grow.p, 1, rb);
    MF_CUDA_TRY(cudaGetLastError());
    rc = exclusive_scan_int(t->tile_off.p, tilenum + 1, s);
    if (rc) return rc;
    enc_csrptr_offsets<<<nblk(tilenum + 1, 256), 256, 0, s>>>(tilenum, tilem, rowA, t->tile_ptr.p,
                                                              t->csrptr_off.p);
    // row compression
    if (t->nonzero_row_new.alloc(tilenum + 1) || t->tile_rowidx.alloc(tilenum) ||
        t->block_signal.alloc(tilem + 1))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->nonzero_row_new.p, 0, sizeof(int) * (tilenum + 1), s));
    if (tilenum > 0)
        enc_rowcomp_count<<<nblk(tilenum, 256), 256, 0, s>>>(tilenum, tilem, rowA, t->tile_ptr.p, t->tile_off.p,
                                                             t->csrptr_off.p, t->ptr.p, t->nonzero_row_new.p,
                                                             t->tile_rowidx.p);
    rc = exclusive_scan_int(t->nonzero_row_new.p, tilenum + 1, s);
    if (rc) return rc;
    MF_CUDA_TRY(cudaMemcpyAsync(&t->cnt_non_new, t->nonzero_row_new.p + tilenum, sizeof(int),
                                cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (t->blockrowid_new.alloc(t->cnt_non_new + 1) || t->blockcsr_ptr_new.alloc(t->cnt_non_new + 1))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->blockrowid_new.p, 0, t->cnt_non_new + 1, s));
    MF_CUDA_TRY(cudaMemsetAsync(t->blockcsr_ptr_new.p, 0, t->cnt_non_new + 1, s));
    if (tilenum > 0)
        enc_rowcomp_fill<<<nblk(tilenum, 256), 256, 0, s>>>(tilenum, tilem, rowA, t->tile_off.p, t->csrptr_off.p,
                                                            t->ptr.p, t->nonzero_row_new.p, t->tile_rowidx.p,
                                                            t->blockrowid_new.p, t->blockcsr_ptr_new.p);
    enc_block_signal<<<nblk(tilem + 1, 256), 256, 0, s>>>(tilem, t->tile_ptr.p, t->block_signal.p);
    if (t->diag.alloc((size_t)tilem * 16)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(t->diag.p, 0, sizeof(double) * tilem * 16, s));
    enc_diag<<<nblk(rowA, 256), 256, 0, s>>>(rowA, rp, ci, val, t->diag.p);
    MF_CUDA_TRY(cudaGetLastError());
    cudaEventRecord(e1, s);
    MF_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    t->encode_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MF_OK;
}

}  // namespace mf
