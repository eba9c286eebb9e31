// CG on k <= 16 right-hand sides at once (the block-CG workload of the
// benchmark configs: k = 16 on the 128^3 Poisson). The k recurrences are the
// reference's CG, each with its own alpha and beta, sharing every
// matrix-panel product Q = A P: the matrix is read once per iteration for
// all k columns.
//
// Panels (B, X, R, P, Q) are n x 16 row-major (the right-hand sides of a row
// are one line). Two panel precisions:
//
// MF_PANEL_FP32 (default, k_mr_fused): P and Q in FP32, x, r, dots and
// scalars FP64, true-residual replacement; one cooperative persistent
// launch for the whole solve (its comment below has the details).
//
// MF_PANEL_FP64 (exact): every panel FP64, and column j of Q is bit for bit
// the single-right-hand-side SpMV of column j of P, so each column is the
// FP64 CG. The SpMM gives a half-warp to a row and a lane to a right-hand
// side: the matrix entry is broadcast, the panel row load is coalesced, and
// each column keeps blockspmv_cpu's order (per 16-column tile in CSR order,
// then added to the row total tile by tile). One iteration is five launches
// with fixed grids (every reduction sums per-block partials in a fixed
// order, so the scalars are deterministic):
//   spmm (Q = A P, partial d.q)  ->  alpha_j  ->  r -= alpha q (partial r.r)
//   ->  beta_j, convergence  ->  x += alpha p, p = r + beta p
// A right-hand side that has converged gets alpha = beta = 0 and p = 0 from
// then on. Blocks of iterations are captured in a CUDA graph and replayed
// until every right-hand side has converged or maxiter is reached.
//
// Both read the matrix as a copy padded to a multiple of 8 entries a row
// (padding: the row's last column, value 0), so a lane issues the panel
// loads of 8 entries at once instead of one dependent load after another; a
// padding entry adds 0 * p, which leaves a sum that starts at +0 bit for bit
// unchanged. Rows longer than MR_PAD_MAX, or padding that would more than
// double the stored entries, keep the CSR loop.
//
// The product runs on CUDA cores: the 7-point tiles hold ~17 of 256 entries,
// so a tensor-core tile x panel product would stream or expand dense 16 x 16
// tiles for 6.5 % useful products, while the iteration is bound by the
// panel passes over x, r, p and q, not by the product.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "mf_internal.h"
#include "tiles.h"

namespace mf {
namespace {

constexpr int KW = 16;           // panel width
constexpr int MR_BLOCKS = 1184;  // fixed grid of the row kernels (8 per SM)
constexpr int MR_THREADS = 256;
constexpr int MR_GRAPH_ITERS = 25;
constexpr int MR_CH = 8;        // padded entries a half-warp loads at once
constexpr int MR_PAD_MAX = 64;  // longest row the padded copy takes

struct MrState {
    double rr[KW], dq[KW], alpha[KW], beta[KW], bb[KW];
    int done[KW], iters[KW];
    int it, k;
};

__device__ __forceinline__ double mr_dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double mr_dadd(double a, double b) { return __dadd_rn(a, b); }

// Block reduction of 16 per-lane values (lane & 15 = right-hand side) into
// out[16], in a fixed order.
__device__ void block_sum16(double v, double (*sred)[KW], double *out) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    if (lane < KW) sred[w][lane] = v;
    __syncthreads();
    if (threadIdx.x < KW) {
        double a = 0.0;
        for (int q = 0; q < MR_THREADS / 32; ++q) a += sred[q][threadIdx.x];
        out[threadIdx.x] = a;
    }
    __syncthreads();
}

// Q = A P for the rows of this block (grid-stride over rows, half-warp per
// row); partial[blockIdx.x][j] = sum over its rows of P[row][j] * Q[row][j].
__global__ void __launch_bounds__(MR_THREADS) k_mr_spmm(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                      const double *__restrict__ val, const double *__restrict__ P,
                                                      double *__restrict__ Q, double *part) {
    __shared__ double sred[MR_THREADS / 32][KW];
    const int j = threadIdx.x & 15;
    const int hw = (blockIdx.x * MR_THREADS + threadIdx.x) >> 4, nhw = (gridDim.x * MR_THREADS) >> 4;
    double dq = 0.0;
    for (int row = hw; row < n; row += nhw) {
        const int s = rp[row], e = rp[row + 1];
        double acc = 0.0, sum = 0.0;
        int tile = s < e ? ci[s] >> 4 : 0;
        for (int q = s; q < e; ++q) {
            const int c = ci[q];
            if ((c >> 4) != tile) {  // next 16-column tile: add the finished tile sum
                acc = mr_dadd(acc, sum);
                sum = 0.0;
                tile = c >> 4;
            }
            sum = mr_dadd(sum, mr_dmul(__ldg(P + (size_t)c * KW + j), val[q]));
        }
        acc = mr_dadd(acc, sum);
        Q[(size_t)row * KW + j] = acc;
        dq += P[(size_t)row * KW + j] * acc;
    }
    __shared__ double bres[KW];
    block_sum16(dq, sred, bres);
    if (threadIdx.x < KW) part[(size_t)blockIdx.x * KW + threadIdx.x] = bres[threadIdx.x];
}

// The same product over the padded copy: W (a multiple of MR_CH) entries per
// row, row-major, 32-byte aligned rows of columns and 64-byte rows of values.
__global__ void __launch_bounds__(MR_THREADS) k_mr_spmm_pad(int n, int W, const int *__restrict__ ec,
                                                          const double *__restrict__ ev, const double *__restrict__ P,
                                                          double *__restrict__ Q, double *part) {
    __shared__ double sred[MR_THREADS / 32][KW];
    const int j = threadIdx.x & 15;
    const int hw = (blockIdx.x * MR_THREADS + threadIdx.x) >> 4, nhw = (gridDim.x * MR_THREADS) >> 4;
    double dq = 0.0;
    for (int row = hw; row < n; row += nhw) {
        const int *rc = ec + (size_t)row * W;
        const double *rv = ev + (size_t)row * W;
        double acc = 0.0, sum = 0.0;
        int tile = __ldg(rc) >> 4;
        for (int k0 = 0; k0 < W; k0 += MR_CH) {
            int c[MR_CH];
            double a[MR_CH], p[MR_CH];
            const int4 c0 = __ldg(reinterpret_cast<const int4 *>(rc + k0));
            const int4 c1 = __ldg(reinterpret_cast<const int4 *>(rc + k0 + 4));
            c[0] = c0.x, c[1] = c0.y, c[2] = c0.z, c[3] = c0.w;
            c[4] = c1.x, c[5] = c1.y, c[6] = c1.z, c[7] = c1.w;
#pragma unroll
            for (int i = 0; i < MR_CH; ++i) p[i] = __ldg(P + (size_t)c[i] * KW + j);
#pragma unroll
            for (int i = 0; i < MR_CH; i += 2) {
                const double2 v = __ldg(reinterpret_cast<const double2 *>(rv + k0 + i));
                a[i] = v.x;
                a[i + 1] = v.y;
            }
#pragma unroll
            for (int i = 0; i < MR_CH; ++i) {
                const int t = c[i] >> 4;
                if (t != tile) {  // next 16-column tile: add the finished tile sum
                    acc = mr_dadd(acc, sum);
                    sum = 0.0;
                    tile = t;
                }
                sum = mr_dadd(sum, mr_dmul(p[i], a[i]));
            }
        }
        acc = mr_dadd(acc, sum);
        Q[(size_t)row * KW + j] = acc;
        dq += P[(size_t)row * KW + j] * acc;
    }
    __shared__ double bres[KW];
    block_sum16(dq, sred, bres);
    if (threadIdx.x < KW) part[(size_t)blockIdx.x * KW + threadIdx.x] = bres[threadIdx.x];
}

// Checks of a device CSR before any column index is used: flags[1] |= 1 when
// rp[0] != 0 or a row pointer decreases (reads rp only).
__global__ void k_mr_check_rp(int n, const int *rp, int *flags) {
    int bad = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        if (rp[r + 1] < rp[r] || (r == 0 && rp[0] != 0)) bad = 1;
    if (bad) atomicOr(flags + 1, bad);
}
// flags[1] |= 2 for a column outside [0, n), 4 for columns that do not
// ascend within a row; flags[0] = the longest row.
__global__ void k_mr_check_ci(int n, const int *rp, const int *ci, int *flags) {
    __shared__ int smax, sbad;
    if (threadIdx.x == 0) smax = 0, sbad = 0;
    __syncthreads();
    int mx = 0, bad = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int s = rp[r], e = rp[r + 1];
        for (int q = s; q < e; ++q) {
            const int c = ci[q];
            if (c < 0 || c >= n) bad |= 2;
            if (q > s && c <= ci[q - 1]) bad |= 4;
        }
        mx = max(mx, e - s);
    }
    atomicMax(&smax, mx);
    if (bad) atomicOr(&sbad, bad);
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicMax(flags, smax);
        if (sbad) atomicOr(flags + 1, sbad);
    }
}

// Padded copy: entry k < len of row r is the CSR entry, the rest repeat the
// row's last column (column r for an empty row) with value 0.
__global__ void k_mr_pad(int n, int W, const int *rp, const int *ci, const double *val, int *ec, double *ev) {
    const long long tot = (long long)n * W;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(e / W), k = (int)(e % W);
        const int s = rp[row], len = rp[row + 1] - s;
        if (k < len) {
            ec[e] = ci[s + k];
            ev[e] = val[s + k];
        } else {
            ec[e] = len > 0 ? ci[s + len - 1] : row;
            ev[e] = 0.0;
        }
    }
}

// Sums the partials of every right-hand side in block order; mode 0: d.q ->
// alpha, mode 1: r.r -> beta, convergence, iteration counts.
__global__ void k_mr_scalars(const double *part, int nb, MrState *st, int mode, double tol, int maxiter) {
    __shared__ double tot[KW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < KW) {
        double a = 0.0;
        for (int b = lane; b < nb; b += 32) a += part[(size_t)b * KW + w];
        for (int d = 16; d > 0; d >>= 1) a += __shfl_xor_sync(0xffffffffu, a, d);
        if (lane == 0) tot[w] = a;
    }
    __syncthreads();
    const int j = threadIdx.x;
    if (j >= KW) return;
    if (mode == 0) {
        const bool live = j < st->k && !st->done[j];
        st->dq[j] = tot[j];
        st->alpha[j] = (live && tot[j] != 0.0) ? st->rr[j] / tot[j] : 0.0;
    } else {
        if (j < st->k && !st->done[j]) {
            const double rrn = tot[j];
            st->beta[j] = st->rr[j] != 0.0 ? rrn / st->rr[j] : 0.0;
            st->rr[j] = rrn;
            st->iters[j] += 1;
            const double rel = st->bb[j] > 0 ? sqrt(rrn / st->bb[j]) : sqrt(rrn);
            if (!(rel > tol) || st->iters[j] >= maxiter || !isfinite(rrn)) {
                st->done[j] = 1;
                st->beta[j] = 0.0;
            }
        } else {
            st->beta[j] = 0.0;
        }
        if (j == 0) st->it += 1;
    }
}

// r -= alpha q over the panel; partial r.r.
__global__ void __launch_bounds__(MR_THREADS) k_mr_update_r(long long nel, double *R, const double *Q,
                                                          const MrState *st, double *part) {
    __shared__ double sred[MR_THREADS / 32][KW];
    __shared__ double bres[KW];
    const int j = threadIdx.x & 15;  // the block stride is a multiple of 16
    const double a = st->alpha[j];
    double rr = 0.0;
    for (long long e = blockIdx.x * (long long)MR_THREADS + threadIdx.x; e < nel; e += (long long)gridDim.x * MR_THREADS) {
        const double r = R[e] - a * Q[e];
        R[e] = r;
        rr += r * r;
    }
    block_sum16(rr, sred, bres);
    if (threadIdx.x < KW) part[(size_t)blockIdx.x * KW + threadIdx.x] = bres[threadIdx.x];
}

// x += alpha p, p = r + beta p (p = 0 once the right-hand side has converged).
__global__ void __launch_bounds__(MR_THREADS) k_mr_update_xp(long long nel, double *X, double *P, const double *R,
                                                           const MrState *st) {
    const int j = threadIdx.x & 15;
    const double a = st->alpha[j], bt = st->beta[j];
    const bool done = st->done[j] != 0;
    for (long long e = blockIdx.x * (long long)MR_THREADS + threadIdx.x; e < nel; e += (long long)gridDim.x * MR_THREADS) {
        const double p = P[e];
        X[e] += a * p;
        P[e] = done ? 0.0 : R[e] + bt * p;
    }
}

// Initial state: R = B - A X (Q holds A X), P = R, rr_j, bb_j.
__global__ void __launch_bounds__(MR_THREADS) k_mr_init(long long nel, const double *B, const double *Q, double *R,
                                                      double *P, double *part) {
    __shared__ double sred[MR_THREADS / 32][KW];
    __shared__ double bres[KW];
    double rr = 0.0, bb = 0.0;
    for (long long e = blockIdx.x * (long long)MR_THREADS + threadIdx.x; e < nel; e += (long long)gridDim.x * MR_THREADS) {
        const double r = B[e] - Q[e];
        R[e] = r;
        P[e] = r;
        rr += r * r;
        bb += B[e] * B[e];
    }
    block_sum16(rr, sred, bres);
    if (threadIdx.x < KW) part[(size_t)blockIdx.x * 2 * KW + threadIdx.x] = bres[threadIdx.x];
    block_sum16(bb, sred, bres);
    if (threadIdx.x < KW) part[(size_t)blockIdx.x * 2 * KW + KW + threadIdx.x] = bres[threadIdx.x];
}

__global__ void k_mr_init_state(const double *part, int nb, MrState *st, int k, double tol) {
    const int j = threadIdx.x;
    if (j >= KW) return;
    double rr = 0.0, bb = 0.0;
    for (int b = 0; b < nb; ++b) {
        rr += part[(size_t)b * 2 * KW + j];
        bb += part[(size_t)b * 2 * KW + KW + j];
    }
    st->rr[j] = rr;
    st->bb[j] = bb;
    st->alpha[j] = st->beta[j] = st->dq[j] = 0.0;
    st->iters[j] = 0;
    const double rel = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
    st->done[j] = (j >= k || !(rel > tol)) ? 1 : 0;
    if (j == 0) {
        st->it = 0;
        st->k = k;
    }
}

// column j of the n x k column-major matrix <-> column j of the panel
__global__ void k_mr_pack(int n, int k, const double *cm, double *panel) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * KW;
         e += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(e / KW), j = (int)(e % KW);
        panel[e] = j < k ? cm[(size_t)j * n + row] : 0.0;
    }
}
__global__ void k_mr_unpack(int n, int k, const double *panel, double *cm) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * k;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / n), row = (int)(e % n);
        cm[e] = panel[(size_t)row * KW + j];
    }
}


// ---- FP32-direction panels in one persistent launch -----------------------
//
// The k <= 16 recurrences of the FP64 path with the search directions P and
// the products Q = A P stored in FP32 (x, r, the dots and the scalars stay
// FP64): p = fl32(r + beta p), q = fl32(A p) with the product summed in FP64
// in blockspmv_cpu's order. FP32 directions need the true residual: after
// the r update, r = b - A x replaces it every MRF_REPLACE iterations and
// whenever a column's recursive residual reaches tol; a column converges only
// on that true residual, and a replacement whose true residual norm exceeds
// twice the recursive one restarts that column's recurrence (beta = 0). Each
// column then runs the recurrence of mfo_cg_dir32 (oracle), independently of
// the others.
//
// One cooperative launch runs the whole solve. Every CTA owns a contiguous
// range of rows; per iteration
//   S  : Q = fl32(A P) on its rows (P rows of the CTAs its columns reach,
//        waited for by epoch flags), partial p.q          -> grid sum -> alpha
//   U1 : r -= alpha q, partial r.r                        -> grid sum
//   (replacement: x += alpha p, publish, r = b - A x for the columns that
//    replace, partial r.r                                 -> grid sum)
//   U2 : x += alpha p (unless done above), p = fl32(r + beta p), publish.
// A thread owns four right-hand sides of a row (a quarter-warp per row: one
// 16-byte FP32 or two 16-byte FP64 accesses per panel row), so every panel
// access is a full 64- or 128-byte line per row and the column partials
// reduce across the lanes with equal lane & 3. Grid sums: per-CTA partials
// in a fixed order, a release/acquire arrival counter, every CTA summing the
// same partials in the same order (all CTAs hold identical scalars, so every
// decision is uniform). Every wait is bounded (MF_ERR_TIMEOUT).
constexpr int MRF_THREADS = 512;
constexpr int MRF_WARPS = MRF_THREADS / 32;
constexpr int MRF_ROWS = MRF_THREADS / 4;  // rows a CTA covers per step
constexpr int MRF_REPLACE = 50;
constexpr int MRF_STAGES = 3;            // bulk-copy ring of the vector passes
constexpr int MRF_STAGE_BYTES = 24576;   // rows of one chunk, every array of the pass
// per-thread landing slots of the product's panel gathers: two units
// (8 entries each) of 16 bytes a thread
constexpr int MRF_GATHER_BYTES = 2 * MR_CH * MRF_THREADS * 16;
constexpr int MRF_DYN_SMEM = MRF_STAGES * MRF_STAGE_BYTES + MRF_GATHER_BYTES;
// Window blocks (matrices of at most 8 entries a row): 128-row blocks whose
// columns fall in at most MRF_WIN_SEGS 16-row panel segments in at most
// MRF_WIN_RUNS contiguous runs get those panel rows staged by bulk copies.
constexpr int MRF_BLK = MRF_ROWS;
constexpr int MRF_WIN_SEGS = 40;
constexpr int MRF_WIN_RUNS = 8;
constexpr int MRF_WOFF_EL = MRF_BLK * 8 * 8;                 // values [8][128] FP64, then
constexpr int MRF_WOFF_EC = MRF_WOFF_EL + MRF_BLK * 8 * 2;   // slots [8][128] u16, then
constexpr int MRF_WOFF_WIN = MRF_WOFF_EC + MRF_BLK * 8 * 4;  // columns [8][128] (unstaged blocks), then
constexpr int MRF_WSTAGE_BYTES = MRF_WOFF_WIN + MRF_WIN_SEGS * 1024;  // the window (1 KB a segment)
enum { MRF_MODE_CSR = 0, MRF_MODE_PAD = 1, MRF_MODE_WIN = 2 };

struct MrfRun {
    int seg0;               // first 16-row panel segment
    uint16_t nseg, slot0;   // segments, first window segment
};
struct MrfPlan {
    int staged, nruns, own_slot, nseg;  // own_slot: window row of the block's first row
    MrfRun run[MRF_WIN_RUNS];
};
static_assert(MRF_THREADS == 512, "the grid sum stages 32 chunks of 16 columns");
constexpr int MRF_FLAG_STRIDE = 8;  // one 32-byte sector per CTA flag
enum { MRF_ARRIVE = 0, MRF_ERROR = 32, MRF_SITE = 33, MRF_FLAGS = 64 };

struct MrfOut {
    double rr[KW], bb[KW];
    int iters[KW], conv[KW];
    int it, pad;
};

struct MrfParams {
    int n, W, G, rows_per_cta, padded;
    int nblk, stage_bytes;
    const double *evT;     // window mode: values [block][8][128]
    const uint16_t *elT;   // window slot | 0x8000 at the first entry of a 16-column tile
    const int *ecT;        // columns [block][8][128]
    const MrfPlan *plan;   // [block]
    const int *ec;
    const double *ev;
    const int *rp, *ci;
    const double *val;
    const double *B;
    double *X, *R;
    float *P, *Q;
    uint32_t *sync;
    double *partial;  // [2][G][16]
    const int *dep;   // [G][2]: first and last CTA whose rows this CTA's columns reach
    double tol;
    int maxiter, replace_every;
    uint64_t limit_ns;
    MrfOut *out;
};

struct MrfShared {
    double red[MRF_WARPS][KW];
    double chunk[32][KW];
    double bres[KW];
    double rr[KW], bb[KW], alpha[KW], beta[KW];
    int live[KW], rep[KW], iters[KW], conv[KW], restart[KW];
    int any_rep, n_live, abort;
    uint64_t full[MRF_STAGES];
};

// A thread's first row of a pass, made opaque to the compiler so that the
// pass's address arithmetic is not hoisted out of the iteration loop (where
// it would hold registers across every other pass).
__device__ __forceinline__ int mrf_first_row(int r0) {
    int v = r0 + (int)(threadIdx.x >> 2);
    asm volatile("" : "+r"(v));
    return v;
}

__device__ __forceinline__ void mrf_error(uint32_t *sync, uint32_t code, uint32_t site) {
    if (atomicCAS(sync + MRF_ERROR, 0u, code) == 0u) atomicExch(sync + MRF_SITE, site);
}

// Grid-wide sum of 16 column partials; v[m] is this thread's partial of
// column 4 (lane & 3) + m. Result in S.bres (every CTA the same bits).
__device__ bool mrf_gsum(const MrfParams &P, MrfShared &S, double (&v)[4], uint32_t &phase) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        v[m] += __shfl_xor_sync(0xffffffffu, v[m], 4);
        v[m] += __shfl_xor_sync(0xffffffffu, v[m], 8);
        v[m] += __shfl_xor_sync(0xffffffffu, v[m], 16);
    }
    if (lane < 4)
#pragma unroll
        for (int m = 0; m < 4; ++m) S.red[w][lane * 4 + m] = v[m];
    __syncthreads();
    const int G = P.G, slot = phase & 1;
    if (tid < KW) {
        double a = 0.0;
        for (int q = 0; q < MRF_WARPS; ++q) a += S.red[q][tid];
        P.partial[((size_t)slot * G + blockIdx.x) * KW + tid] = a;
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        red_release_add(P.sync + MRF_ARRIVE, 1u);
        const uint32_t target = (phase + 1) * (uint32_t)G;
        if (ld_acquire(P.sync + MRF_ARRIVE) < target) {
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(P.sync + MRF_ARRIVE) >= target) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(P.sync + MRF_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > P.limit_ns) {
                        mrf_error(P.sync, (uint32_t)MF_ERR_TIMEOUT, 1);
                        S.abort = 1;
                        break;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (S.abort) return false;
    {
        const int j = tid & 15, c = tid >> 4;  // 32 chunks of CTAs per column
        double a = 0.0;
        for (int g = c; g < G; g += 32) a += __ldcg(&P.partial[((size_t)slot * G + g) * KW + j]);
        S.chunk[c][j] = a;
    }
    __syncthreads();
    if (tid < KW) {
        double a = 0.0;
        for (int c = 0; c < 32; ++c) a += S.chunk[c][tid];
        S.bres[tid] = a;
    }
    __syncthreads();
    ++phase;
    return true;
}

__device__ void mrf_publish(const MrfParams &P, uint32_t ep) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(P.sync + MRF_FLAGS + blockIdx.x * MRF_FLAG_STRIDE, ep);
    }
}

// Wait until the CTAs whose rows this CTA's columns reach have published `ep`.
__device__ bool mrf_wait(const MrfParams &P, MrfShared &S, uint32_t ep) {
    if (threadIdx.x < 32) {
        const int lo = P.dep[2 * blockIdx.x], hi = P.dep[2 * blockIdx.x + 1];
        for (int c = lo + (int)threadIdx.x; c <= hi; c += 32) {
            const uint32_t *f = P.sync + MRF_FLAGS + c * MRF_FLAG_STRIDE;
            if (ld_acquire(f) >= ep) continue;
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(f) >= ep) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(P.sync + MRF_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > P.limit_ns) {
                        mrf_error(P.sync, (uint32_t)MF_ERR_TIMEOUT, 2);
                        S.abort = 1;
                        break;
                    }
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    return S.abort == 0;
}

__device__ __forceinline__ void ld_d4(const double *p, double (&v)[4]) {
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p + 2));
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
// Gathered panel rows: plain loads, cached in L1 within a phase. They are
// written by other CTAs between phases; the epoch wait's acquire (gpu scope)
// orders these loads after those writes, so no stale line is read.
__device__ __forceinline__ void ld_d4_l1(const double *p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const double2 b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
// 16-byte asynchronous copy global -> shared through L1 (per thread; the
// thread waits for its own groups and reads only its own slots).
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The same with an L2 eviction policy (the streamed FP64 panels X and R).
__device__ __forceinline__ void st_d4_pol(double *p, const double (&v)[4], uint64_t pol) {
    st2_hint(p, make_double2(v[0], v[1]), pol);
    st2_hint(p + 2, make_double2(v[2], v[3]), pol);
}
__device__ __forceinline__ void st_d4(double *p, const double (&v)[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

// Four columns of one entry: sum += a * v (the FP64 products of the tile sum).
__device__ __forceinline__ void mrf_fma4(double (&sum)[4], double a, const double (&v)[4]) {
#pragma unroll
    for (int m = 0; m < 4; ++m) sum[m] = dadd(sum[m], dmul(v[m], a));
}

// acc = row `row` of A times columns 4 cg .. 4 cg + 3 of the panel V (FP32
// P or FP64 X), in blockspmv_cpu's order: per 16-column tile in CSR order,
// the tile sums added to the row total tile by tile.
template <bool PAD, bool X64>
__device__ __forceinline__ void mrf_row(const MrfParams &P, int row, int cg, double (&acc)[4]) {
    double sum[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0, sum[m] = 0.0;
    if (PAD) {
        const int *rc = P.ec + (size_t)row * P.W;
        const double *rv = P.ev + (size_t)row * P.W;
        int tile = __ldg(rc) >> 4;
        for (int k0 = 0; k0 < P.W; k0 += MR_CH) {
            int c[MR_CH];
            double a[MR_CH];
            const int4 c0 = __ldg(reinterpret_cast<const int4 *>(rc + k0));
            const int4 c1 = __ldg(reinterpret_cast<const int4 *>(rc + k0 + 4));
            c[0] = c0.x, c[1] = c0.y, c[2] = c0.z, c[3] = c0.w;
            c[4] = c1.x, c[5] = c1.y, c[6] = c1.z, c[7] = c1.w;
#pragma unroll
            for (int i = 0; i < MR_CH; i += 2) {
                const double2 d = __ldg(reinterpret_cast<const double2 *>(rv + k0 + i));
                a[i] = d.x;
                a[i + 1] = d.y;
            }
            if (X64) {
                // FP64 panel rows (the replacement residual): two groups of 4
#pragma unroll
                for (int h = 0; h < MR_CH; h += 4) {
                    double v[4][4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) ld_d4_l1(P.X + (size_t)c[h + i] * KW + 4 * cg, v[i]);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int t = c[h + i] >> 4;
                        if (t != tile) {
#pragma unroll
                            for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                            tile = t;
                        }
                        mrf_fma4(sum, a[h + i], v[i]);
                    }
                }
            } else {
                float4 f[MR_CH];
#pragma unroll
                for (int i = 0; i < MR_CH; ++i) f[i] = *reinterpret_cast<const float4 *>(P.P + (size_t)c[i] * KW + 4 * cg);
#pragma unroll
                for (int i = 0; i < MR_CH; ++i) {
                    const int t = c[i] >> 4;
                    if (t != tile) {
#pragma unroll
                        for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                        tile = t;
                    }
                    const double v[4] = {(double)f[i].x, (double)f[i].y, (double)f[i].z, (double)f[i].w};
                    mrf_fma4(sum, a[i], v);
                }
            }
        }
    } else {
        const int s = P.rp[row], e = P.rp[row + 1];
        int tile = s < e ? P.ci[s] >> 4 : 0;
        for (int q = s; q < e; ++q) {
            const int c = P.ci[q];
            double v[4];
            if (X64) {
                ld_d4_l1(P.X + (size_t)c * KW + 4 * cg, v);
            } else {
                const float4 f = *reinterpret_cast<const float4 *>(P.P + (size_t)c * KW + 4 * cg);
                v[0] = f.x, v[1] = f.y, v[2] = f.z, v[3] = f.w;
            }
            if ((c >> 4) != tile) {
#pragma unroll
                for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                tile = c >> 4;
            }
            mrf_fma4(sum, P.val[q], v);
        }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]);
}

// r = b - A x for the columns with rep set (all at set-up); partial r.r of
// the resulting r (and b.b when bb is given).
// acc = row `row` of A times columns 4 cg .. 4 cg + 3 of the FP64 panel X,
// from the window mode's transposed arrays ([block][entry][row]: the loads
// of a warp's 8 rows are consecutive); blockspmv_cpu's order.
__device__ __forceinline__ void mrf_row_t(const MrfParams &P, int row, int cg, double (&acc)[4]) {
    double sum[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0, sum[m] = 0.0;
    const size_t base = (size_t)(row / MRF_BLK) * 8 * MRF_BLK + (row % MRF_BLK);
    int c[8];
    double a[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) c[e] = __ldg(P.ecT + base + (size_t)e * MRF_BLK), a[e] = __ldg(P.evT + base + (size_t)e * MRF_BLK);
    int tile = c[0] >> 4;
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
        double v[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i) ld_d4_l1(P.X + (size_t)c[h + i] * KW + 4 * cg, v[i]);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int t = c[h + i] >> 4;
            if (t != tile) {
#pragma unroll
                for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                tile = t;
            }
            mrf_fma4(sum, a[h + i], v[i]);
        }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]);
}

template <int MODE>
__device__ void mrf_residual(const MrfParams &P, const MrfShared &S, int r0, int r1, double (&rr)[4],
                             double (*bb)[4]) {
    const int cg = threadIdx.x & 3;
    bool rep[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) rep[m] = S.rep[4 * cg + m] != 0, rr[m] = 0.0;
#pragma unroll 1
    for (int row = mrf_first_row(r0); row < r1; row += MRF_ROWS) {
        double ax[4], b[4], r[4];
        if (MODE == MRF_MODE_WIN)
            mrf_row_t(P, row, cg, ax);
        else
            mrf_row<MODE == MRF_MODE_PAD, true>(P, row, cg, ax);
        ld_d4(P.B + (size_t)row * KW + 4 * cg, b);
        ld_d4(P.R + (size_t)row * KW + 4 * cg, r);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (rep[m]) r[m] = __dsub_rn(b[m], ax[m]);
            rr[m] += r[m] * r[m];
            if (bb) (*bb)[m] += b[m] * b[m];
        }
        st_d4(P.R + (size_t)row * KW + 4 * cg, r);
    }
}

// The bulk-copy ring of the vector passes: a pass walks this CTA's rows in
// chunks; thread 0 stages every array a chunk needs with cp.async.bulk (the
// rows of a CTA are contiguous, so each array of a chunk is one copy) up to
// MRF_STAGES chunks ahead, and the whole CTA computes from shared memory and
// stores its results to global memory. `par` holds the parity of each
// stage's next wait (uniform across the CTA). L2 policies: the streamed
// arrays (matrix, X, R, B, Q) evict first; the search directions P, which
// the product pass reads again through the windows of several blocks, evict
// last.
struct MrfRing {
    uint8_t *buf;
    int sb;  // bytes a stage
    uint32_t par;
    uint64_t pol;  // evict first
    uint64_t pl;   // evict last (P)
};

__device__ __forceinline__ void mrf_wait_full(const MrfParams &P, MrfShared &S, MrfRing &R, int k) {
    const uint32_t ph = (R.par >> k) & 1u;
    R.par ^= 1u << k;
    if (mbar_try_wait(&S.full[k], ph)) return;
    const uint64_t t0 = globaltimer();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(&S.full[k], ph)) return;
        if ((spin & 15u) == 0 && globaltimer() - t0 > P.limit_ns) {
            // reported to the host; the pass runs on (the copy lands in this
            // CTA's own shared memory whenever it completes)
            mrf_error(P.sync, (uint32_t)MF_ERR_TIMEOUT, 3);
            return;
        }
    }
}

// One pass over this CTA's rows [r0, r1) in chunks of C rows: issue(chunk,
// stage) is called by thread 0 only (expect_tx, then the copies), body(chunk
// first row, rows in chunk, stage) by every thread.
template <class Issue, class Body>
__device__ __forceinline__ void mrf_pass(const MrfParams &P, MrfShared &S, MrfRing &R, int r0, int r1, int C,
                                         Issue issue, Body body) {
    const int nch = (r1 - r0 + C - 1) / C;
    if (threadIdx.x == 0)
        for (int c = 0; c < nch && c < MRF_STAGES; ++c) issue(r0 + c * C, min(C, r1 - r0 - c * C), c);
#pragma unroll 1
    for (int i = 0; i < nch; ++i) {
        const int k = i % MRF_STAGES;
        const int rb = r0 + i * C, rn = min(C, r1 - rb);
        mrf_wait_full(P, S, R, k);
        body(rb, rn, R.buf + (size_t)k * R.sb);
        __syncthreads();  // every thread is done with stage k
        const int nx = i + MRF_STAGES;
        if (threadIdx.x == 0 && nx < nch) issue(r0 + nx * C, min(C, r1 - r0 - nx * C), k);
    }
    fence_proxy_async_global();  // this thread's global stores before later bulk reads of them
}

// The product pass over the padded matrix: q = fl32(A p) on this CTA's rows,
// partial p.q. The ring stages each chunk's column indices, values and own
// p rows (bulk copies); a thread owns one row of a chunk and walks it in
// units of 8 entries. The 8 panel-row gathers of a unit go into the
// thread's own shared-memory slots by cp.async while the thread computes
// the previous unit (software pipeline across units and chunks; the unit's
// values, tiles and own p travel in registers, so a ring stage is released
// as soon as its units are issued). Same sums, same order as mrf_row.
__device__ __forceinline__ void mrf_spmm_pad(const MrfParams &P, MrfShared &S, MrfRing &R, int r0, int r1, int cs,
                                             double (&pq)[4]) {
    const int tid = threadIdx.x, cg = tid & 3, rs = tid >> 2, W = P.W;
    float4 *gb = reinterpret_cast<float4 *>(R.buf + (size_t)MRF_STAGES * R.sb);  // [2][8][threads]
    // the unit in flight (issued, not yet computed)
    double pa[MR_CH];
    int pt[MR_CH];
    float4 pown = make_float4(0.f, 0.f, 0.f, 0.f);
    int prow = -1, pbuf = 0;
    bool plast = false, have = false;
    double acc[4], sum[4];
    int tile = 0;
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0, sum[m] = 0.0;
    auto compute_prev = [&]() {
        const float4 *g = gb + (size_t)pbuf * MR_CH * MRF_THREADS + tid;
#pragma unroll
        for (int i = 0; i < MR_CH; ++i) {
            if (pt[i] != tile) {
#pragma unroll
                for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                tile = pt[i];
            }
            const float4 f = g[(size_t)i * MRF_THREADS];
            const double v[4] = {(double)f.x, (double)f.y, (double)f.z, (double)f.w};
            mrf_fma4(sum, pa[i], v);
        }
        if (plast) {
            float4 q;
            q.x = __double2float_rn(dadd(acc[0], sum[0]));
            q.y = __double2float_rn(dadd(acc[1], sum[1]));
            q.z = __double2float_rn(dadd(acc[2], sum[2]));
            q.w = __double2float_rn(dadd(acc[3], sum[3]));
            *reinterpret_cast<float4 *>(P.Q + (size_t)prow * KW + 4 * cg) = q;
            pq[0] += (double)pown.x * (double)q.x;
            pq[1] += (double)pown.y * (double)q.y;
            pq[2] += (double)pown.z * (double)q.z;
            pq[3] += (double)pown.w * (double)q.w;
#pragma unroll
            for (int m = 0; m < 4; ++m) acc[m] = 0.0, sum[m] = 0.0;
        }
    };
    const int nch = (r1 - r0 + cs - 1) / cs;
    auto issue = [&](int rb, int rn, int k) {
        uint8_t *st = R.buf + (size_t)k * R.sb;
        const uint32_t bc = (uint32_t)rn * W * 4, bv = (uint32_t)rn * W * 8, bp = (uint32_t)rn * 64;
        mbar_arrive_expect_tx(&S.full[k], bc + bv + bp);
        bulk_g2s(st, P.ec + (size_t)rb * W, bc, &S.full[k], R.pol);
        bulk_g2s(st + (size_t)cs * W * 4, P.ev + (size_t)rb * W, bv, &S.full[k], R.pol);
        bulk_g2s(st + (size_t)cs * W * 12, P.P + (size_t)rb * KW, bp, &S.full[k], R.pol);
    };
    if (tid == 0)
        for (int c = 0; c < nch && c < MRF_STAGES; ++c) issue(r0 + c * cs, min(cs, r1 - r0 - c * cs), c);
#pragma unroll 1
    for (int i = 0; i < nch; ++i) {
        const int k = i % MRF_STAGES;
        const int rb = r0 + i * cs, rn = min(cs, r1 - rb);
        mrf_wait_full(P, S, R, k);
        const uint8_t *st = R.buf + (size_t)k * R.sb;
        if (rs < rn) {
            const int *rc = reinterpret_cast<const int *>(st) + (size_t)rs * W;
            const double *rv = reinterpret_cast<const double *>(st + (size_t)cs * W * 4) + (size_t)rs * W;
            const float4 own = reinterpret_cast<const float4 *>(st + (size_t)cs * W * 12)[rs * 4 + cg];
#pragma unroll 1
            for (int k0 = 0; k0 < W; k0 += MR_CH) {
                int c[MR_CH];
                const int4 c0 = reinterpret_cast<const int4 *>(rc + k0)[0];
                const int4 c1 = reinterpret_cast<const int4 *>(rc + k0)[1];
                c[0] = c0.x, c[1] = c0.y, c[2] = c0.z, c[3] = c0.w;
                c[4] = c1.x, c[5] = c1.y, c[6] = c1.z, c[7] = c1.w;
                const int b = have ? pbuf ^ 1 : 0;
                float4 *g = gb + (size_t)b * MR_CH * MRF_THREADS + tid;
#pragma unroll
                for (int e = 0; e < MR_CH; ++e) cp_async16(g + (size_t)e * MRF_THREADS, P.P + (size_t)c[e] * KW + 4 * cg);
                cp_async_commit();
                if (have) {
                    cp_async_wait<1>();
                    compute_prev();
                }
                if (k0 == 0 && !have) tile = c[0] >> 4;
#pragma unroll
                for (int e = 0; e < MR_CH; ++e) pa[e] = rv[k0 + e], pt[e] = c[e] >> 4;
                if (k0 == 0 && have && plast) tile = c[0] >> 4;
                pown = own;
                prow = rb + rs;
                plast = k0 + MR_CH >= W;
                pbuf = b;
                have = true;
            }
        }
        __syncthreads();  // every thread has read stage k
        const int nx = i + MRF_STAGES;
        if (tid == 0 && nx < nch) issue(r0 + nx * cs, min(cs, r1 - r0 - nx * cs), k);
    }
    if (have) {
        cp_async_wait<0>();
        compute_prev();
    }
    fence_proxy_async_global();
}

// The product pass of the window mode: one 128-row block a chunk. The
// stage holds the block's values and window slots ([entry][row], so a
// warp's 8 rows read consecutive words) and either its panel window (the
// runs of 16-row segments its columns and its own rows fall in, one bulk
// copy a run) or, for an unstaged block, its column indices (the panel rows
// are then loaded from global memory). Same sums, same order as mrf_row.
__device__ __forceinline__ void mrf_spmm_win(const MrfParams &P, MrfShared &S, MrfRing &R, int r0, int r1,
                                             const MrfPlan *plans, double (&pq)[4]) {
    const int tid = threadIdx.x, cg = tid & 3, rs = tid >> 2;
    const int b0 = r0 / MRF_BLK;
    const int nch = (r1 - r0 + MRF_BLK - 1) / MRF_BLK;
    auto issue = [&](int i, int k) {
        uint8_t *st = R.buf + (size_t)k * R.sb;
        const MrfPlan &pl = plans[i];
        const size_t blk = (size_t)(b0 + i);
        uint32_t bytes = MRF_WOFF_EC;
        if (pl.staged) bytes += (uint32_t)pl.nseg * 1024;
        else bytes += MRF_BLK * 8 * 4;
        mbar_arrive_expect_tx(&S.full[k], bytes);
        bulk_g2s(st, P.evT + blk * 8 * MRF_BLK, MRF_BLK * 8 * 8, &S.full[k], R.pol);
        bulk_g2s(st + MRF_WOFF_EL, P.elT + blk * 8 * MRF_BLK, MRF_BLK * 8 * 2, &S.full[k], R.pol);
        if (pl.staged) {
            for (int j = 0; j < pl.nruns; ++j) {
                const MrfRun ru = pl.run[j];
                bulk_g2s(st + MRF_WOFF_WIN + (size_t)ru.slot0 * 1024, P.P + (size_t)ru.seg0 * 16 * KW,
                         (uint32_t)ru.nseg * 1024, &S.full[k], R.pl);
            }
        } else {
            bulk_g2s(st + MRF_WOFF_EC, P.ecT + blk * 8 * MRF_BLK, MRF_BLK * 8 * 4, &S.full[k], R.pol);
        }
    };
    if (tid == 0)
        for (int c = 0; c < nch && c < MRF_STAGES; ++c) issue(c, c);
#pragma unroll 1
    for (int i = 0; i < nch; ++i) {
        const int k = i % MRF_STAGES;
        const int rb = r0 + i * MRF_BLK, rn = min(MRF_BLK, r1 - rb);
        mrf_wait_full(P, S, R, k);
        const uint8_t *st = R.buf + (size_t)k * R.sb;
        if (rs < rn) {
            const double *ev = reinterpret_cast<const double *>(st);
            const uint16_t *el = reinterpret_cast<const uint16_t *>(st + MRF_WOFF_EL);
            const float4 *win = reinterpret_cast<const float4 *>(st + MRF_WOFF_WIN);
            const MrfPlan &pl = plans[i];
            double acc[4], sum[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) acc[m] = 0.0, sum[m] = 0.0;
            float4 own;
            if (pl.staged) {
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const uint32_t l = el[e * MRF_BLK + rs];
                    if (e > 0 && (l & 0x8000u)) {  // next 16-column tile: add the finished tile sum
#pragma unroll
                        for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                    }
                    const float4 f = win[(l & 0x7fffu) * 4 + cg];
                    const double v[4] = {(double)f.x, (double)f.y, (double)f.z, (double)f.w};
                    mrf_fma4(sum, ev[e * MRF_BLK + rs], v);
                }
                own = win[(pl.own_slot + rs) * 4 + cg];
            } else {
                const int *ec = reinterpret_cast<const int *>(st + MRF_WOFF_EC);
                float4 f[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    f[e] = *reinterpret_cast<const float4 *>(P.P + (size_t)ec[e * MRF_BLK + rs] * KW + 4 * cg);
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    if (e > 0 && (el[e * MRF_BLK + rs] & 0x8000u)) {
#pragma unroll
                        for (int m = 0; m < 4; ++m) acc[m] = dadd(acc[m], sum[m]), sum[m] = 0.0;
                    }
                    const double v[4] = {(double)f[e].x, (double)f[e].y, (double)f[e].z, (double)f[e].w};
                    mrf_fma4(sum, ev[e * MRF_BLK + rs], v);
                }
                own = __ldcg(reinterpret_cast<const float4 *>(P.P + (size_t)(rb + rs) * KW + 4 * cg));
            }
            float4 q;
            q.x = __double2float_rn(dadd(acc[0], sum[0]));
            q.y = __double2float_rn(dadd(acc[1], sum[1]));
            q.z = __double2float_rn(dadd(acc[2], sum[2]));
            q.w = __double2float_rn(dadd(acc[3], sum[3]));
            *reinterpret_cast<float4 *>(P.Q + (size_t)(rb + rs) * KW + 4 * cg) = q;
            pq[0] += (double)own.x * (double)q.x;
            pq[1] += (double)own.y * (double)q.y;
            pq[2] += (double)own.z * (double)q.z;
            pq[3] += (double)own.w * (double)q.w;
        }
        __syncthreads();  // every thread is done with stage k
        const int nx = i + MRF_STAGES;
        if (tid == 0 && nx < nch) issue(nx, k);
    }
    fence_proxy_async_global();
}

template <int MODE>
__global__ void __launch_bounds__(MRF_THREADS, 1) k_mr_fused(MrfParams P) {
    __shared__ MrfShared S;
    extern __shared__ __align__(128) uint8_t mrf_dyn[];
    const int tid = threadIdx.x, cg = tid & 3, rs = tid >> 2;
    const int r0 = min(P.n, blockIdx.x * P.rows_per_cta), r1 = min(P.n, r0 + P.rows_per_cta);
    MrfRing ring;
    ring.buf = mrf_dyn;
    ring.sb = P.stage_bytes;
    ring.par = 0;
    ring.pol = policy_evict_first();
    ring.pl = policy_evict_last();
    if (tid == 0) {
        S.abort = 0, S.any_rep = 0;
        for (int k = 0; k < MRF_STAGES; ++k) mbar_init(&S.full[k], 1);
        mbar_fence_init();
    }
    if (tid < KW) {
        S.rep[tid] = 1;
        S.iters[tid] = 0;
        S.conv[tid] = 0;
        S.restart[tid] = 0;
    }
    // window mode: this CTA's block plans, after the ring (they never change)
    MrfPlan *plans = reinterpret_cast<MrfPlan *>(mrf_dyn + (size_t)MRF_STAGES * P.stage_bytes);
    if (MODE == MRF_MODE_WIN) {
        const int b0 = r0 / MRF_BLK, nb = (r1 - r0 + MRF_BLK - 1) / MRF_BLK;
        const int *src = reinterpret_cast<const int *>(P.plan + b0);
        int *dst = reinterpret_cast<int *>(plans);
        for (int w = tid; w < nb * (int)(sizeof(MrfPlan) / 4); w += MRF_THREADS) dst[w] = __ldg(src + w);
    }
    __syncthreads();
    // chunk rows of the padded product pass: column indices, values and own p
    const int cs = MODE == MRF_MODE_PAD ? min(MRF_ROWS, MRF_STAGE_BYTES / (12 * P.W + 64)) : 0;
    uint32_t phase = 0, ep = 0;
    // set-up: r = b - A x0, r.r, b.b, p = fl32(r)
    {
        double rr[4], bb[4] = {0.0, 0.0, 0.0, 0.0};
        mrf_residual<MODE>(P, S, r0, r1, rr, &bb);
        if (!mrf_gsum(P, S, rr, phase)) return;
        if (tid < KW) S.rr[tid] = S.bres[tid];
        if (!mrf_gsum(P, S, bb, phase)) return;
        if (tid < KW) {
            const double b2 = S.bres[tid], r2 = S.rr[tid];
            S.bb[tid] = b2;
            const double rel = b2 > 0 ? sqrt(r2 / b2) : sqrt(r2);
            S.live[tid] = rel > P.tol ? 1 : 0;  // NaN: not live, not converged
            S.conv[tid] = rel <= P.tol ? 1 : 0;
        }
        __syncthreads();
        bool live[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) live[m] = S.live[4 * cg + m] != 0;
#pragma unroll 1
        for (int row = mrf_first_row(r0); row < r1; row += MRF_ROWS) {
            double r[4];
            ld_d4(P.R + (size_t)row * KW + 4 * cg, r);
            float4 p;
            p.x = live[0] ? __double2float_rn(r[0]) : 0.f;
            p.y = live[1] ? __double2float_rn(r[1]) : 0.f;
            p.z = live[2] ? __double2float_rn(r[2]) : 0.f;
            p.w = live[3] ? __double2float_rn(r[3]) : 0.f;
            *reinterpret_cast<float4 *>(P.P + (size_t)row * KW + 4 * cg) = p;
        }
        fence_proxy_async_global();
        mrf_publish(P, ++ep);
    }
    int it = 0;
    for (;;) {
        if (tid == 0) {
            int nl = 0;
            for (int j = 0; j < KW; ++j) nl += S.live[j];
            S.n_live = nl;
        }
        __syncthreads();
        if (S.n_live == 0 || it >= P.maxiter) break;
        ++it;
        // S: q = fl32(A p), partial p.q
        if (!mrf_wait(P, S, ep)) return;
        {
            double pq[4] = {0.0, 0.0, 0.0, 0.0};
            if (MODE == MRF_MODE_WIN) {
                mrf_spmm_win(P, S, ring, r0, r1, plans, pq);
            } else if (MODE == MRF_MODE_PAD) {
                mrf_spmm_pad(P, S, ring, r0, r1, cs, pq);
            } else {
#pragma unroll 1
                for (int row = mrf_first_row(r0); row < r1; row += MRF_ROWS) {
                    double acc[4];
                    mrf_row<false, false>(P, row, cg, acc);
                    float4 q;
                    q.x = __double2float_rn(acc[0]);
                    q.y = __double2float_rn(acc[1]);
                    q.z = __double2float_rn(acc[2]);
                    q.w = __double2float_rn(acc[3]);
                    *reinterpret_cast<float4 *>(P.Q + (size_t)row * KW + 4 * cg) = q;
                    const float4 p = __ldcg(reinterpret_cast<const float4 *>(P.P + (size_t)row * KW + 4 * cg));
                    pq[0] += (double)p.x * (double)q.x;
                    pq[1] += (double)p.y * (double)q.y;
                    pq[2] += (double)p.z * (double)q.z;
                    pq[3] += (double)p.w * (double)q.w;
                }
                fence_proxy_async_global();
            }
            if (!mrf_gsum(P, S, pq, phase)) return;
        }
        if (tid < KW) {
            const double dq = S.bres[tid];
            double a = 0.0;
            if (S.live[tid]) {
                if (dq > 0.0 && isfinite(dq)) {
                    a = S.rr[tid] / dq;
                } else {
                    S.live[tid] = 0;  // breakdown: stops, not converged
                    S.iters[tid] = it;
                }
            }
            S.alpha[tid] = a;
        }
        __syncthreads();
        double al[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) al[m] = S.alpha[4 * cg + m];
        // U1: r -= alpha q, partial r.r
        {
            double rr[4] = {0.0, 0.0, 0.0, 0.0};
            auto issue = [&](int rb, int rn, int k) {
                uint8_t *st = ring.buf + (size_t)k * ring.sb;
                mbar_arrive_expect_tx(&S.full[k], (uint32_t)rn * 192);
                bulk_g2s(st, P.R + (size_t)rb * KW, (uint32_t)rn * 128, &S.full[k], ring.pol);
                bulk_g2s(st + MRF_ROWS * 128, P.Q + (size_t)rb * KW, (uint32_t)rn * 64, &S.full[k], ring.pol);
            };
            auto body = [&](int rb, int rn, const uint8_t *st) {
                if (rs >= rn) return;
                const int row = rb + rs;
                double r[4];
                const double2 r01 = reinterpret_cast<const double2 *>(st)[rs * 8 + cg * 2];
                const double2 r23 = reinterpret_cast<const double2 *>(st)[rs * 8 + cg * 2 + 1];
                const float4 q = reinterpret_cast<const float4 *>(st + MRF_ROWS * 128)[rs * 4 + cg];
                r[0] = __dsub_rn(r01.x, dmul(al[0], (double)q.x));
                r[1] = __dsub_rn(r01.y, dmul(al[1], (double)q.y));
                r[2] = __dsub_rn(r23.x, dmul(al[2], (double)q.z));
                r[3] = __dsub_rn(r23.y, dmul(al[3], (double)q.w));
#pragma unroll
                for (int m = 0; m < 4; ++m) rr[m] += r[m] * r[m];
                st_d4_pol(P.R + (size_t)row * KW + 4 * cg, r, ring.pol);
            };
            mrf_pass(P, S, ring, r0, r1, MRF_ROWS, issue, body);
            if (!mrf_gsum(P, S, rr, phase)) return;
        }
        if (tid < KW) {
            const double rrn = S.bres[tid], b2 = S.bb[tid];
            const double rel = b2 > 0 ? sqrt(rrn / b2) : sqrt(rrn);
            S.rep[tid] = S.live[tid] && ((P.replace_every > 0 && it % P.replace_every == 0) || !(rel > P.tol));
            S.beta[tid] = rrn;  // r.r of the recursive residual, until replaced
            S.restart[tid] = 0;
        }
        __syncthreads();
        if (tid == 0) {
            int any = 0;
            for (int j = 0; j < KW; ++j) any |= S.rep[j];
            S.any_rep = any;
        }
        __syncthreads();
        const bool replaced = S.any_rep != 0;
        if (replaced) {
            // x += alpha p (every column), publish x, r = b - A x where rep
            auto issue = [&](int rb, int rn, int k) {
                uint8_t *st = ring.buf + (size_t)k * ring.sb;
                mbar_arrive_expect_tx(&S.full[k], (uint32_t)rn * 192);
                bulk_g2s(st, P.X + (size_t)rb * KW, (uint32_t)rn * 128, &S.full[k], ring.pol);
                bulk_g2s(st + MRF_ROWS * 128, P.P + (size_t)rb * KW, (uint32_t)rn * 64, &S.full[k], ring.pl);
            };
            auto body = [&](int rb, int rn, const uint8_t *st) {
                if (rs >= rn) return;
                const int row = rb + rs;
                double x[4];
                const double2 x01 = reinterpret_cast<const double2 *>(st)[rs * 8 + cg * 2];
                const double2 x23 = reinterpret_cast<const double2 *>(st)[rs * 8 + cg * 2 + 1];
                const float4 p = reinterpret_cast<const float4 *>(st + MRF_ROWS * 128)[rs * 4 + cg];
                x[0] = dadd(x01.x, dmul(al[0], (double)p.x));
                x[1] = dadd(x01.y, dmul(al[1], (double)p.y));
                x[2] = dadd(x23.x, dmul(al[2], (double)p.z));
                x[3] = dadd(x23.y, dmul(al[3], (double)p.w));
                st_d4_pol(P.X + (size_t)row * KW + 4 * cg, x, ring.pol);
            };
            mrf_pass(P, S, ring, r0, r1, MRF_ROWS, issue, body);
            mrf_publish(P, ++ep);
            if (!mrf_wait(P, S, ep)) return;
            double rr[4];
            mrf_residual<MODE>(P, S, r0, r1, rr, nullptr);
            fence_proxy_async_global();
            if (!mrf_gsum(P, S, rr, phase)) return;
            if (tid < KW) {
                const double rrn = S.bres[tid], b2 = S.bb[tid];
                if (S.rep[tid]) {
                    // a true residual norm more than twice the recursive one:
                    // the FP32 products let the recursive residual drift below
                    // it, and beta from the two would break the directions'
                    // conjugacy; restart from the true residual (p = r)
                    S.restart[tid] = rrn > 4.0 * S.beta[tid];
                    S.beta[tid] = rrn;
                    const double rel = b2 > 0 ? sqrt(rrn / b2) : sqrt(rrn);
                    if (!(rel > P.tol)) {  // converged on the true residual
                        S.live[tid] = 0;
                        S.conv[tid] = 1;
                        S.iters[tid] = it;
                        S.rr[tid] = rrn;
                    }
                }
            }
        }
        if (tid < KW) {
            const double rrn = S.beta[tid];
            if (S.live[tid]) {
                S.beta[tid] = S.restart[tid] ? 0.0 : rrn / S.rr[tid];
                S.rr[tid] = rrn;
                S.iters[tid] = it;
                if (!isfinite(rrn)) S.live[tid] = 0;
            } else {
                S.beta[tid] = 0.0;
            }
        }
        __syncthreads();
        // U2: x += alpha p (unless done above), p = fl32(r + beta p)
        {
            double bt[4];
            bool live[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) bt[m] = S.beta[4 * cg + m], live[m] = S.live[4 * cg + m] != 0;
            constexpr int C2 = MRF_ROWS / 2;  // 320 bytes a row: P, R, X
            auto issue = [&](int rb, int rn, int k) {
                uint8_t *st = ring.buf + (size_t)k * ring.sb;
                mbar_arrive_expect_tx(&S.full[k], (uint32_t)rn * (replaced ? 192 : 320));
                bulk_g2s(st, P.P + (size_t)rb * KW, (uint32_t)rn * 64, &S.full[k], ring.pl);
                bulk_g2s(st + C2 * 64, P.R + (size_t)rb * KW, (uint32_t)rn * 128, &S.full[k], ring.pol);
                if (!replaced)
                    bulk_g2s(st + C2 * 192, P.X + (size_t)rb * KW, (uint32_t)rn * 128, &S.full[k], ring.pol);
            };
            auto body = [&](int rb, int rn, const uint8_t *st) {
                // two threads a row-quarter: the pass's chunk is half as many rows
                if (rs >= rn) return;
                const int row = rb + rs;
                const float4 p = reinterpret_cast<const float4 *>(st)[rs * 4 + cg];
                const double2 r01 = reinterpret_cast<const double2 *>(st + C2 * 64)[rs * 8 + cg * 2];
                const double2 r23 = reinterpret_cast<const double2 *>(st + C2 * 64)[rs * 8 + cg * 2 + 1];
                if (!replaced) {
                    const double2 x01 = reinterpret_cast<const double2 *>(st + C2 * 192)[rs * 8 + cg * 2];
                    const double2 x23 = reinterpret_cast<const double2 *>(st + C2 * 192)[rs * 8 + cg * 2 + 1];
                    double x[4];
                    x[0] = dadd(x01.x, dmul(al[0], (double)p.x));
                    x[1] = dadd(x01.y, dmul(al[1], (double)p.y));
                    x[2] = dadd(x23.x, dmul(al[2], (double)p.z));
                    x[3] = dadd(x23.y, dmul(al[3], (double)p.w));
                    st_d4_pol(P.X + (size_t)row * KW + 4 * cg, x, ring.pol);
                }
                float4 np;
                np.x = live[0] ? __double2float_rn(dadd(r01.x, dmul(bt[0], (double)p.x))) : 0.f;
                np.y = live[1] ? __double2float_rn(dadd(r01.y, dmul(bt[1], (double)p.y))) : 0.f;
                np.z = live[2] ? __double2float_rn(dadd(r23.x, dmul(bt[2], (double)p.z))) : 0.f;
                np.w = live[3] ? __double2float_rn(dadd(r23.y, dmul(bt[3], (double)p.w))) : 0.f;
                stf4_hint(P.P + (size_t)row * KW + 4 * cg, np, ring.pl);
            };
            mrf_pass(P, S, ring, r0, r1, C2, issue, body);
        }
        mrf_publish(P, ++ep);
    }
    if (blockIdx.x == 0 && tid < KW) {
        P.out->rr[tid] = S.rr[tid];
        P.out->bb[tid] = S.bb[tid];
        P.out->iters[tid] = S.iters[tid];
        P.out->conv[tid] = S.conv[tid];
        if (tid == 0) P.out->it = it;
    }
}

// Window layout of a matrix of at most 8 entries a row, one 128-thread CTA
// per 128-row block (a thread per row): entries padded to 8 as k_mr_pad
// does, stored [block][entry][row]; the block's distinct 16-row panel
// segments (its columns' and its own rows') sorted, as runs; an entry's
// window slot = its segment's rank * 16 + column % 16, with 0x8000 set where
// the entry starts a new 16-column tile. Blocks with more than MRF_WIN_SEGS
// segments or MRF_WIN_RUNS runs are left unstaged (slots 0).
__global__ void __launch_bounds__(MRF_BLK) k_mrf_layout(int n, const int *rp, const int *ci, const double *val,
                                                       double *evT, uint16_t *elT, int *ecT, MrfPlan *plan) {
    constexpr int NS = 2048;  // 8 * 128 entry segments + 8 own segments, padded to a power of two
    __shared__ int sg[NS];
    __shared__ int uq[NS];
    __shared__ int scnt[MRF_BLK];
    __shared__ int stot, sstaged;
    const int blk = blockIdx.x, r = threadIdx.x, row = blk * MRF_BLK + r;
    int c[8];
    double v[8];
    int s0 = 0, len = 0;
    if (row < n) s0 = rp[row], len = rp[row + 1] - s0;  // len <= 8 (checked by the host)
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        if (e < len) {
            c[e] = ci[s0 + e];
            v[e] = val[s0 + e];
        } else {
            c[e] = len > 0 ? ci[s0 + len - 1] : min(row, n - 1);
            v[e] = 0.0;
        }
    }
    const size_t base = (size_t)blk * 8 * MRF_BLK + r;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        evT[base + (size_t)e * MRF_BLK] = v[e];
        ecT[base + (size_t)e * MRF_BLK] = c[e];
        sg[e * MRF_BLK + r] = c[e] >> 4;
    }
    for (int i = 8 * MRF_BLK + r; i < NS; i += MRF_BLK)
        sg[i] = i < 8 * MRF_BLK + 8 ? blk * 8 + (i - 8 * MRF_BLK) : INT_MAX;
    __syncthreads();
    for (int kk = 2; kk <= NS; kk <<= 1) {  // bitonic sort, ascending
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = r; i < NS; i += MRF_BLK) {
                const int pi = i ^ j;
                if (pi > i) {
                    const int a = sg[i], b = sg[pi];
                    if ((a > b) == ((i & kk) == 0)) sg[i] = b, sg[pi] = a;
                }
            }
            __syncthreads();
        }
    }
    constexpr int PER = NS / MRF_BLK;
    int cnt = 0;
    for (int i = r * PER; i < r * PER + PER; ++i) cnt += sg[i] != INT_MAX && (i == 0 || sg[i] != sg[i - 1]);
    scnt[r] = cnt;
    __syncthreads();
    if (r == 0) {
        int a = 0;
        for (int t = 0; t < MRF_BLK; ++t) {
            const int x = scnt[t];
            scnt[t] = a;
            a += x;
        }
        stot = a;
    }
    __syncthreads();
    int pos = scnt[r];
    for (int i = r * PER; i < r * PER + PER; ++i)
        if (sg[i] != INT_MAX && (i == 0 || sg[i] != sg[i - 1])) uq[pos++] = sg[i];
    __syncthreads();
    const int U = stot;
    if (r == 0) {
        MrfPlan pl;
        memset(&pl, 0, sizeof pl);
        bool ok = U <= MRF_WIN_SEGS;
        int nr = 0;
        for (int q = 0; ok && q < U; ++q) {
            if (q == 0 || uq[q] != uq[q - 1] + 1) {
                if (nr == MRF_WIN_RUNS) {
                    ok = false;
                    break;
                }
                pl.run[nr].seg0 = uq[q];
                pl.run[nr].slot0 = (uint16_t)q;
                pl.run[nr].nseg = 0;
                ++nr;
            }
            pl.run[nr - 1].nseg++;
        }
        if (ok) {
            pl.staged = 1;
            pl.nruns = nr;
            pl.nseg = U;
            for (int q = 0; q < U; ++q)
                if (uq[q] == blk * 8) pl.own_slot = q * 16;
        } else {
            memset(&pl, 0, sizeof pl);
        }
        plan[blk] = pl;
        sstaged = ok ? 1 : 0;
    }
    __syncthreads();
    const bool staged = sstaged != 0;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        uint32_t slot = 0;
        if (staged) {
            const int sgv = c[e] >> 4;
            int lo = 0, hi = U - 1;
            while (lo < hi) {  // the segment is in uq[0..U)
                const int mid = (lo + hi) >> 1;
                if (uq[mid] < sgv) lo = mid + 1;
                else hi = mid;
            }
            slot = (uint32_t)lo * 16 + (uint32_t)(c[e] & 15);
        }
        const bool first = e > 0 && (c[e] >> 4) != (c[e - 1] >> 4);
        elT[base + (size_t)e * MRF_BLK] = (uint16_t)(slot | (first ? 0x8000u : 0u));
    }
}

// dep[2c], dep[2c+1] = the first and last CTA owning a column that the rows
// of CTA c reach (one block per CTA).
__global__ void k_mrf_deps(int n, int rows_per_cta, const int *rp, const int *ci, int *dep) {
    __shared__ int smin, smax;
    const int c = blockIdx.x;
    const int r0 = min(n, c * rows_per_cta), r1 = min(n, r0 + rows_per_cta);
    if (threadIdx.x == 0) smin = r0 < r1 ? r0 : 0, smax = r0 < r1 ? r1 - 1 : 0;
    __syncthreads();
    int lo = INT_MAX, hi = -1;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const int s = rp[r], e = rp[r + 1];
        if (s < e) lo = min(lo, ci[s]), hi = max(hi, ci[e - 1]);  // columns ascend within a row
    }
    if (hi >= 0) {
        atomicMin(&smin, lo);
        atomicMax(&smax, hi);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dep[2 * c] = smin / rows_per_cta;
        dep[2 * c + 1] = smax / rows_per_cta;
    }
}
}  // namespace
}  // namespace mf

using namespace mf;

namespace {

struct StreamGuard {
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    ~StreamGuard() {
        if (ge) cudaGraphExecDestroy(ge);
        if (g) cudaGraphDestroy(g);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    }
};

// The FP64 panel path: five launches per iteration, replayed as a graph.
int multi_fp64(int n, const int *rp, const int *ci, const double *val, int k, const double *B, double *X,
               double tol, int maxiter, bool padded, int W, cudaStream_t s, MrState &h) {
    const long long nel = (long long)n * KW;
    const int pk = 592;
    // the padded copy of the matrix (CSR loop when it does not fit)
    DevArray<int> pec;
    DevArray<double> pev;
    if (padded && (pec.alloc((size_t)n * W) || pev.alloc((size_t)n * W))) {
        padded = false;
        pec.release();
        pev.release();
        (void)cudaGetLastError();
    }
    if (padded) k_mr_pad<<<pk, 256, 0, s>>>(n, W, rp, ci, val, pec.p, pev.p);
    const int *ec = pec.p;
    const double *ev = pev.p;
    DevArray<double> pb, px, pr, pp, pq, part;
    DevArray<MrState> st;
    if (pb.alloc(nel) || px.alloc(nel) || pr.alloc(nel) || pp.alloc(nel) || pq.alloc(nel) ||
        part.alloc((size_t)MR_BLOCKS * 2 * KW) || st.alloc(1))
        return MF_ERR_NOMEM;
    int sp_blocks = MR_BLOCKS;
    if (padded) {
        int dev = 0, nsm = 0, occ = 0;
        MF_CUDA_TRY(cudaGetDevice(&dev));
        MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mr_spmm_pad, MR_THREADS, 0));
        if (occ > 0 && nsm > 0) sp_blocks = std::min(MR_BLOCKS, occ * nsm);  // one resident wave
    }
    auto spmm = [&](const double *Pin, double *Qout) {
        if (padded)
            k_mr_spmm_pad<<<sp_blocks, MR_THREADS, 0, s>>>(n, W, ec, ev, Pin, Qout, part.p);
        else
            k_mr_spmm<<<MR_BLOCKS, MR_THREADS, 0, s>>>(n, rp, ci, val, Pin, Qout, part.p);
    };
    k_mr_pack<<<pk, 256, 0, s>>>(n, k, B, pb.p);
    k_mr_pack<<<pk, 256, 0, s>>>(n, k, X, px.p);
    spmm(px.p, pq.p);
    k_mr_init<<<MR_BLOCKS, MR_THREADS, 0, s>>>(nel, pb.p, pq.p, pr.p, pp.p, part.p);
    k_mr_init_state<<<1, 32, 0, s>>>(part.p, MR_BLOCKS, st.p, k, tol);
    MF_CUDA_TRY(cudaGetLastError());
    // one block of iterations, captured once and replayed
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    MF_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < MR_GRAPH_ITERS; ++i) {
        spmm(pp.p, pq.p);
        k_mr_scalars<<<1, 32 * KW, 0, s>>>(part.p, padded ? sp_blocks : MR_BLOCKS, st.p, 0, tol, maxiter);
        k_mr_update_r<<<MR_BLOCKS, MR_THREADS, 0, s>>>(nel, pr.p, pq.p, st.p, part.p);
        k_mr_scalars<<<1, 32 * KW, 0, s>>>(part.p, MR_BLOCKS, st.p, 1, tol, maxiter);
        k_mr_update_xp<<<MR_BLOCKS, MR_THREADS, 0, s>>>(nel, px.p, pp.p, pr.p, st.p);
    }
    MF_CUDA_TRY(cudaStreamEndCapture(s, &g));
    const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    MF_CUDA_TRY(ei);
    struct ExecGuard {
        cudaGraphExec_t e;
        ~ExecGuard() { cudaGraphExecDestroy(e); }
    } eg{ge};
    for (int blocks = 0;; ++blocks) {
        MF_CUDA_TRY(cudaMemcpyAsync(&h, st.p, sizeof h, cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaStreamSynchronize(s));
        bool all = true;
        for (int j = 0; j < k; ++j) all = all && h.done[j];
        if (all || (long long)blocks * MR_GRAPH_ITERS >= maxiter) break;
        MF_CUDA_TRY(cudaGraphLaunch(ge, s));
    }
    k_mr_unpack<<<pk, 256, 0, s>>>(n, k, px.p, X);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

// The FP32 panel path: one cooperative persistent launch (k_mr_fused).
// Window mode for matrices of at most 8 entries a row whose block plans fit
// in shared memory; the padded-gather mode for other padded matrices; the
// CSR loop otherwise.
int multi_fp32(int n, const int *rp, const int *ci, const double *val, int k, const double *B, double *X,
               double tol, int maxiter, bool padded, int W, cudaStream_t s, MrState &h) {
    const int pk = 592;
    int dev = 0, nsm = 0, coop = 0, smax = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (!coop || nsm < 1) {
        set_last_error("mf_solve_cg_multi: the device cannot run the persistent panel kernel");
        return MF_ERR_UNSUPPORTED;
    }
    const int nblk = (n + MRF_BLK - 1) / MRF_BLK;
    int mode = !padded ? MRF_MODE_CSR : W == 8 ? MRF_MODE_WIN : MRF_MODE_PAD;
    int G = 0, rows_per_cta = 0, stage_bytes = MRF_STAGE_BYTES;
    size_t dyn = 0;
    const void *kfn = nullptr;
    for (;;) {
        kfn = mode == MRF_MODE_WIN   ? (const void *)k_mr_fused<MRF_MODE_WIN>
              : mode == MRF_MODE_PAD ? (const void *)k_mr_fused<MRF_MODE_PAD>
                                     : (const void *)k_mr_fused<MRF_MODE_CSR>;
        cudaFuncAttributes fa;
        MF_CUDA_TRY(cudaFuncGetAttributes(&fa, kfn));
        if (mode == MRF_MODE_WIN) {
            stage_bytes = MRF_WSTAGE_BYTES;
            const int bpc = (nblk + nsm - 1) / nsm;  // one CTA an SM: the ring takes most of shared memory
            dyn = (size_t)MRF_STAGES * stage_bytes + (size_t)bpc * sizeof(MrfPlan);
            if (dyn + fa.sharedSizeBytes > (size_t)smax) {
                mode = MRF_MODE_PAD;  // too many blocks a CTA for the plans
                continue;
            }
            G = nsm;
            rows_per_cta = bpc * MRF_BLK;
        } else {
            stage_bytes = MRF_STAGE_BYTES;
            dyn = mode == MRF_MODE_PAD ? (size_t)MRF_DYN_SMEM : (size_t)MRF_STAGES * MRF_STAGE_BYTES;
        }
        MF_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        int occ = 0;
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, MRF_THREADS, dyn));
        if (occ < 1) {
            set_last_error("mf_solve_cg_multi: the persistent panel kernel does not fit an SM");
            return MF_ERR_UNSUPPORTED;
        }
        if (mode != MRF_MODE_WIN) {
            G = std::min(occ, 2) * nsm;
            rows_per_cta = (n + G - 1) / G;
        }
        break;
    }
    // panels hold whole 128-row blocks (zero past n): window copies read them
    const size_t npad = (size_t)nblk * MRF_BLK, nel = npad * KW;
    DevArray<double> pb, px, pr, part, pev;
    DevArray<float> pp, pq;
    DevArray<int> dep, pec;
    DevArray<uint16_t> pel;
    DevArray<MrfPlan> plan;
    DevArray<uint32_t> sync;
    DevArray<MrfOut> out;
    const size_t sync_words = (size_t)MRF_FLAGS + (size_t)G * MRF_FLAG_STRIDE;
    if (pb.alloc(nel) || px.alloc(nel) || pr.alloc(nel) || pp.alloc(nel) || pq.alloc(nel) ||
        part.alloc((size_t)2 * G * KW) || dep.alloc((size_t)2 * G) || sync.alloc(sync_words) || out.alloc(1))
        return MF_ERR_NOMEM;
    if (mode == MRF_MODE_WIN) {
        if (pev.alloc(npad * 8) || pec.alloc(npad * 8) || pel.alloc(npad * 8) || plan.alloc(nblk))
            return MF_ERR_NOMEM;
        k_mrf_layout<<<nblk, MRF_BLK, 0, s>>>(n, rp, ci, val, pev.p, pel.p, pec.p, plan.p);
    } else if (mode == MRF_MODE_PAD) {
        if (pec.alloc((size_t)n * W) || pev.alloc((size_t)n * W)) return MF_ERR_NOMEM;
        k_mr_pad<<<pk, 256, 0, s>>>(n, W, rp, ci, val, pec.p, pev.p);
    }
    MF_CUDA_TRY(cudaMemsetAsync(sync.p, 0, sync_words * sizeof(uint32_t), s));
    MF_CUDA_TRY(cudaMemsetAsync(pb.p, 0, nel * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(px.p, 0, nel * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(pr.p, 0, nel * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(pp.p, 0, nel * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(pq.p, 0, nel * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(out.p, 0, sizeof(MrfOut), s));
    k_mr_pack<<<pk, 256, 0, s>>>(n, k, B, pb.p);
    k_mr_pack<<<pk, 256, 0, s>>>(n, k, X, px.p);
    k_mrf_deps<<<G, 256, 0, s>>>(n, rows_per_cta, rp, ci, dep.p);
    MF_CUDA_TRY(cudaGetLastError());
    MrfParams P;
    std::memset(&P, 0, sizeof P);
    P.n = n;
    P.W = W;
    P.G = G;
    P.rows_per_cta = rows_per_cta;
    P.padded = mode != MRF_MODE_CSR ? 1 : 0;
    P.nblk = nblk;
    P.stage_bytes = stage_bytes;
    P.ec = mode == MRF_MODE_PAD ? pec.p : nullptr;
    P.ev = mode == MRF_MODE_PAD ? pev.p : nullptr;
    P.evT = mode == MRF_MODE_WIN ? pev.p : nullptr;
    P.elT = pel.p;
    P.ecT = mode == MRF_MODE_WIN ? pec.p : nullptr;
    P.plan = plan.p;
    P.rp = rp;
    P.ci = ci;
    P.val = val;
    P.B = pb.p;
    P.X = px.p;
    P.R = pr.p;
    P.P = pp.p;
    P.Q = pq.p;
    P.sync = sync.p;
    P.partial = part.p;
    P.dep = dep.p;
    P.tol = tol;
    P.maxiter = maxiter;
    P.replace_every = MRF_REPLACE;
    P.limit_ns = 30ull * 1000000000ull;  // a wait this long means a fault, not a slow CTA
    P.out = out.p;
    void *args[] = {&P};
    MF_CUDA_TRY(cudaLaunchCooperativeKernel(kfn, dim3(G), dim3(MRF_THREADS), args, dyn, s));
    MF_CUDA_TRY(cudaGetLastError());
    MrfOut ho;
    uint32_t err[2];
    MF_CUDA_TRY(cudaMemcpyAsync(&ho, out.p, sizeof ho, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(err, sync.p + MRF_ERROR, sizeof err, cudaMemcpyDeviceToHost, s));
    k_mr_unpack<<<pk, 256, 0, s>>>(n, k, px.p, X);
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (err[0]) {
        set_last_error("mf_solve_cg_multi: a bounded wait of the panel kernel ran out (site " +
                       std::to_string(err[1]) + ")");
        return (int)err[0];
    }
    std::memset(&h, 0, sizeof h);
    for (int j = 0; j < KW; ++j) {
        h.rr[j] = ho.rr[j];
        h.bb[j] = ho.bb[j];
        h.iters[j] = ho.iters[j];
        h.done[j] = ho.conv[j];
    }
    h.it = ho.it;
    h.k = k;
    return MF_OK;
}

}  // namespace

extern "C" int mf_solve_cg_multi_dev_ex(int panel, int n, const int *rp, const int *ci, const double *val, int k,
                                        const double *B, double *X, double tol, int maxiter, int *iterations,
                                        double *rel_residual, double *time_ms) {
    if (n <= 0 || !rp || !ci || !val || !B || !X || k < 1 || k > KW || maxiter < 0 ||
        (panel != MF_PANEL_FP64 && panel != MF_PANEL_FP32)) {
        set_last_error("mf_solve_cg_multi_dev: bad arguments (1 <= k <= 16, panel MF_PANEL_FP64 / MF_PANEL_FP32)");
        return MF_ERR_ARG;
    }
    DevArray<int> flags;
    if (flags.alloc(2)) return MF_ERR_NOMEM;
    StreamGuard guard;
    MF_CUDA_TRY(cudaStreamCreateWithFlags(&guard.s, cudaStreamNonBlocking));
    MF_CUDA_TRY(cudaEventCreate(&guard.e0));
    MF_CUDA_TRY(cudaEventCreate(&guard.e1));
    cudaStream_t s = guard.s;
    cudaEvent_t e0 = guard.e0, e1 = guard.e1;
    MF_CUDA_TRY(cudaEventRecord(e0, s));
    const int pk = 592;
    // the CSR checks: row pointers first, then (reading only entries the row
    // pointers cover) the columns and the longest row
    int hf[2] = {0, 0}, nnz = 0;
    MF_CUDA_TRY(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), s));
    k_mr_check_rp<<<pk, 256, 0, s>>>(n, rp, flags.p);
    MF_CUDA_TRY(cudaMemcpyAsync(hf, flags.p, sizeof hf, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&nnz, rp + n, sizeof nnz, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (hf[1]) {
        set_last_error("mf_solve_cg_multi_dev: invalid CSR: row_ptr[0] != 0 or row_ptr decreasing");
        return MF_ERR_ARG;
    }
    k_mr_check_ci<<<pk, 256, 0, s>>>(n, rp, ci, flags.p);
    MF_CUDA_TRY(cudaMemcpyAsync(hf, flags.p, sizeof hf, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (hf[1] & 2) {
        set_last_error("mf_solve_cg_multi_dev: invalid CSR: column index outside [0, n)");
        return MF_ERR_ARG;
    }
    if (hf[1] & 4) {
        set_last_error("mf_solve_cg_multi_dev: columns must ascend within each row");
        return MF_ERR_ARG;
    }
    // rows padded to a multiple of 8 entries for the product (the CSR loop
    // when the padding does not pay)
    const int W = (hf[0] + MR_CH - 1) / MR_CH * MR_CH;
    const bool padded = W >= MR_CH && W <= MR_PAD_MAX && (long long)n * W <= 2LL * std::max(nnz, n);
    MrState h;
    std::memset(&h, 0, sizeof h);
    const int rc = panel == MF_PANEL_FP32 ? multi_fp32(n, rp, ci, val, k, B, X, tol, maxiter, padded, W, s, h)
                                          : multi_fp64(n, rp, ci, val, k, B, X, tol, maxiter, padded, W, s, h);
    if (rc) return rc;
    MF_CUDA_TRY(cudaEventRecord(e1, s));
    MF_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (time_ms) *time_ms = ms;
    int status = MF_OK;
    for (int j = 0; j < k; ++j) {
        const double rel = h.bb[j] > 0 ? std::sqrt(h.rr[j] / h.bb[j]) : std::sqrt(h.rr[j]);
        if (iterations) iterations[j] = h.iters[j];
        if (rel_residual) rel_residual[j] = rel;
        if (!(rel <= tol)) status = MF_ERR_NOT_CONVERGED;
    }
    return status;
}

extern "C" int mf_solve_cg_multi_dev(int n, const int *rp, const int *ci, const double *val, int k, const double *B,
                                     double *X, double tol, int maxiter, int *iterations, double *rel_residual,
                                     double *time_ms) {
    return mf_solve_cg_multi_dev_ex(MF_PANEL_FP32, n, rp, ci, val, k, B, X, tol, maxiter, iterations, rel_residual,
                                    time_ms);
}

extern "C" int mf_solve_cg_multi_ex(int panel, const mf_csr *A, int k, const double *B, double *X, double tol,
                                    int maxiter, int *iterations, double *rel_residual, double *time_ms) {
    if (!A || !B || !X || A->n <= 0 || A->n != A->ncols || k < 1 || k > KW) return MF_ERR_ARG;
    const int n = A->n;
    for (int i = 0; i < n; ++i)
        for (int q = A->row_ptr[i] + 1; q < A->row_ptr[i + 1]; ++q)
            if (A->col_idx[q] <= A->col_idx[q - 1]) {
                set_last_error("mf_solve_cg_multi: columns must ascend within each row");
                return MF_ERR_ARG;
            }
    DevArray<int> rp, ci;
    DevArray<double> v, b, x;
    if (rp.alloc(n + 1) || ci.alloc(std::max(1, A->nnz)) || v.alloc(std::max(1, A->nnz)) ||
        b.alloc((size_t)n * k) || x.alloc((size_t)n * k))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpy(rp.p, A->row_ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(ci.p, A->col_idx, sizeof(int) * A->nnz, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(v.p, A->val, sizeof(double) * A->nnz, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(b.p, B, sizeof(double) * n * k, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(x.p, X, sizeof(double) * n * k, cudaMemcpyHostToDevice));
    const int rc = mf_solve_cg_multi_dev_ex(panel, n, rp.p, ci.p, v.p, k, b.p, x.p, tol, maxiter, iterations,
                                            rel_residual, time_ms);
    if (rc == MF_OK || rc == MF_ERR_NOT_CONVERGED)
        MF_CUDA_TRY(cudaMemcpy(X, x.p, sizeof(double) * n * k, cudaMemcpyDeviceToHost));
    return rc;
}

extern "C" int mf_solve_cg_multi(const mf_csr *A, int k, const double *B, double *X, double tol, int maxiter,
                                 int *iterations, double *rel_residual, double *time_ms) {
    return mf_solve_cg_multi_ex(MF_PANEL_FP32, A, k, B, X, tol, maxiter, iterations, rel_residual, time_ms);
}
