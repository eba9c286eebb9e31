// CG on k <= 16 right-hand sides at once (the block-CG workload of the
// benchmark configs: k = 16 on the 128^3 Poisson). The k recurrences are the
// reference's CG, each with its own alpha and beta, sharing every
// matrix-panel product Q = A P: the matrix is read once per iteration for
// all k columns.
//
// Panels (B, X, R, P, Q) are n x 16 row-major (the right-hand sides of a row
// are one 128-byte line). The SpMM gives a half-warp to a row and a lane to a
// right-hand side: the matrix entry is broadcast, the panel row load is
// coalesced, and each column keeps blockspmv_cpu's order (per 16-column
// tile in CSR order, then added to the row total tile by tile), so column j
// of Q is bit for bit the single-right-hand-side SpMV of column j of P.
// The matrix is first copied into rows padded to a multiple of 8 entries
// (padding: the row's last column, value 0), so a half-warp issues the
// panel loads of 8 entries at once instead of one dependent load after
// another; a padding entry adds 0 * p, which leaves a sum that starts at +0
// bit for bit unchanged. Rows longer than MR_PAD_MAX, or padding that would
// more than double the stored entries, keep the CSR loop.
// The panel product stays FP64: a BF16 / FP16 tile-times-panel product on
// tensor cores would perturb the 128^3 variable-coefficient operator (scaled
// condition ~1e10) past definiteness, as the FP16 tiles of the mixed layouts
// already do, and the solve could not reach a 1e-10 FP64 residual.
//
// One iteration is five launches with fixed grids (every reduction sums
// per-block partials in a fixed order, so the scalars are deterministic):
//   spmm (Q = A P, partial d.q)  ->  alpha_j  ->  r -= alpha q (partial r.r)
//   ->  beta_j, convergence  ->  x += alpha p, p = r + beta p
// A right-hand side that has converged gets alpha = beta = 0 and p = 0 from
// then on. Blocks of iterations are captured in a CUDA graph and replayed
// until every right-hand side has converged or maxiter is reached.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

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

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" int mf_solve_cg_multi_dev(int n, const int *rp, const int *ci, const double *val, int k, const double *B,
                                     double *X, double tol, int maxiter, int *iterations, double *rel_residual,
                                     double *time_ms) {
    if (n <= 0 || !rp || !ci || !val || !B || !X || k < 1 || k > KW || maxiter < 0) {
        set_last_error("mf_solve_cg_multi_dev: bad arguments (1 <= k <= 16)");
        return MF_ERR_ARG;
    }
    const long long nel = (long long)n * KW;
    DevArray<double> pb, px, pr, pp, pq, part;
    DevArray<MrState> st;
    DevArray<int> flags;
    if (pb.alloc(nel) || px.alloc(nel) || pr.alloc(nel) || pp.alloc(nel) || pq.alloc(nel) ||
        part.alloc((size_t)MR_BLOCKS * 2 * KW) || st.alloc(1) || flags.alloc(2))
        return MF_ERR_NOMEM;
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
    } guard;
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
    // the padded copy of the matrix for the SpMM (CSR loop when it does not pay)
    const int W = (hf[0] + MR_CH - 1) / MR_CH * MR_CH;
    DevArray<int> ec;
    DevArray<double> ev;
    bool padded = W >= MR_CH && W <= MR_PAD_MAX && (long long)n * W <= 2LL * std::max(nnz, n);
    if (padded && (ec.alloc((size_t)n * W) || ev.alloc((size_t)n * W))) {
        padded = false;  // not enough memory for the copy: CSR loop
        ec.release();
        ev.release();
        (void)cudaGetLastError();
    }
    int sp_blocks = MR_BLOCKS;
    if (padded) {
        int dev = 0, nsm = 0, occ = 0;
        MF_CUDA_TRY(cudaGetDevice(&dev));
        MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mr_spmm_pad, MR_THREADS, 0));
        if (occ > 0 && nsm > 0) sp_blocks = std::min(MR_BLOCKS, occ * nsm);  // one resident wave
        k_mr_pad<<<pk, 256, 0, s>>>(n, W, rp, ci, val, ec.p, ev.p);
    }
    auto spmm = [&](const double *Pin, double *Qout) {
        if (padded)
            k_mr_spmm_pad<<<sp_blocks, MR_THREADS, 0, s>>>(n, W, ec.p, ev.p, Pin, Qout, part.p);
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
    MF_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < MR_GRAPH_ITERS; ++i) {
        spmm(pp.p, pq.p);
        k_mr_scalars<<<1, 32 * KW, 0, s>>>(part.p, padded ? sp_blocks : MR_BLOCKS, st.p, 0, tol, maxiter);
        k_mr_update_r<<<MR_BLOCKS, MR_THREADS, 0, s>>>(nel, pr.p, pq.p, st.p, part.p);
        k_mr_scalars<<<1, 32 * KW, 0, s>>>(part.p, MR_BLOCKS, st.p, 1, tol, maxiter);
        k_mr_update_xp<<<MR_BLOCKS, MR_THREADS, 0, s>>>(nel, px.p, pp.p, pr.p, st.p);
    }
    MF_CUDA_TRY(cudaStreamEndCapture(s, &guard.g));
    MF_CUDA_TRY(cudaGraphInstantiate(&guard.ge, guard.g, 0));
    MrState h;
    for (int blocks = 0;; ++blocks) {
        MF_CUDA_TRY(cudaMemcpyAsync(&h, st.p, sizeof h, cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaStreamSynchronize(s));
        bool all = true;
        for (int j = 0; j < k; ++j) all = all && h.done[j];
        if (all || (long long)blocks * MR_GRAPH_ITERS >= maxiter) break;
        MF_CUDA_TRY(cudaGraphLaunch(guard.ge, s));
    }
    k_mr_unpack<<<pk, 256, 0, s>>>(n, k, px.p, X);
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

extern "C" int mf_solve_cg_multi(const mf_csr *A, int k, const double *B, double *X, double tol, int maxiter,
                                 int *iterations, double *rel_residual, double *time_ms) {
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
    const int rc = mf_solve_cg_multi_dev(n, rp.p, ci.p, v.p, k, b.p, x.p, tol, maxiter, iterations, rel_residual,
                                         time_ms);
    if (rc == MF_OK || rc == MF_ERR_NOT_CONVERGED)
        MF_CUDA_TRY(cudaMemcpy(X, x.p, sizeof(double) * n * k, cudaMemcpyDeviceToHost));
    return rc;
}
