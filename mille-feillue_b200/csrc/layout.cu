// Slab layout of the persistent solver (row-sliced planes, see tiles.h).
//
// The row blocks are split into G contiguous CTA ranges of equal cost (slab
// bytes + per-row vector work), and each range into slabs: consecutive row
// blocks whose encoded bytes fit one shared-memory stage and whose distinct
// x segments (16-entry pieces of the input vector) fit the x stage as at
// most MAXRUNS contiguous runs. Row-block sizes and plane precisions are
// computed on the GPU from the encoder's tile arrays; the host plans the
// slabs over those sizes and the tile columns; the slab bytes are written on
// the GPU.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>

#include "common.cuh"
#include "tiles.h"

namespace mf {

namespace {

struct SlabPlan {
    int rb0, nrb, ntiles, mode;
    uint32_t bytes, off16;
    int seg_off, nseg;  // unique sorted x segments (staged mode)
    int run_off, nruns;
};

struct TileArgs {
    const int *tile_ptr, *tile_col, *tile_off, *csrptr_off;
    const unsigned char *bptr;
    const double *val;
    const unsigned char *col;
    const unsigned char *prec;
    const float *scale;
    int tilem, rowA;
};

// Walks the entries of row r of row block rb in the reference's order
// (tiles ascending, CSR order inside the tile).
struct RowCursor {
    int t, t1;   // current tile, end tile
    int q, qe;   // current entry index, end (absolute in val/col)
    int r, rl;
};

__device__ __forceinline__ void row_range(const TileArgs &A, int t, int r, int rl, int &s, int &e) {
    const int base = A.tile_off[t];
    const int nk = A.tile_off[t + 1] - base;
    const int cc = A.csrptr_off[t];
    s = base + A.bptr[cc + r];
    e = base + (r + 1 < rl ? (int)A.bptr[cc + r + 1] : nk);
}

__device__ __forceinline__ void cursor_skip_empty(const TileArgs &A, RowCursor &c) {
    while (c.q >= c.qe && c.t < c.t1) {
        ++c.t;
        if (c.t < c.t1) row_range(A, c.t, c.r, c.rl, c.q, c.qe);
    }
}

__device__ __forceinline__ void cursor_init(const TileArgs &A, RowCursor &c, int rb, int r) {
    c.r = r;
    c.rl = rb == A.tilem - 1 ? A.rowA - (A.tilem - 1) * 16 : 16;
    c.t = A.tile_ptr[rb];
    c.t1 = A.tile_ptr[rb + 1];
    c.q = c.qe = 0;
    if (r < c.rl && c.t < c.t1) {
        row_range(A, c.t, r, c.rl, c.q, c.qe);
        cursor_skip_empty(A, c);
    } else {
        c.t = c.t1;
    }
}

__device__ __forceinline__ bool cursor_valid(const RowCursor &c) { return c.t < c.t1 && c.q < c.qe; }

__device__ __forceinline__ void cursor_next(const TileArgs &A, RowCursor &c) {
    ++c.q;
    cursor_skip_empty(A, c);
}


// ---- mixed layouts: entry classes, compensation, plane formats -----------
// Entry class: the tile's precision, except that a diagonal entry (column ==
// row) of an FP16 / FP8 tile is FP32. A row block's planes are grouped by
// class (FP64, FP32, FP16, FP8 planes in that order); plane j of a group
// holds the j-th entry of that class of each of the 16 rows, in the
// reference's order.
__device__ __forceinline__ int entry_class(const TileArgs &A, int t, bool is_diag) {
    const int p = A.prec[t];
    return (is_diag && p > MF_PREC_FP32) ? MF_PREC_FP32 : p;
}

__device__ __forceinline__ bool entry_is_diag(const TileArgs &A, const RowCursor &c, int row) {
    return A.tile_col[c.t] * 16 + (int)A.col[c.q] == row;
}

// Dequantized value of entry q of tile t (FP64 tiles: the value itself).
__device__ __forceinline__ double dequant(const TileArgs &A, int t, int q) {
    const int p = A.prec[t];
    const double v = A.val[q];
    if (p == MF_PREC_FP64) return v;
    if (p == MF_PREC_FP32) return (double)__double2float_rn(v);
    const double s = (double)A.scale[t];
    const double inv = 1.0 / s;
    if (p == MF_PREC_FP16) return (double)__half2float(__double2half(v * inv)) * s;
    const __nv_fp8_storage_t b = __nv_cvt_double_to_fp8(v * inv, __NV_SATFINITE, __NV_E4M3);
    return (double)__half2float(__half(__nv_cvt_fp8_to_halfraw(b, __NV_E4M3))) * s;
}

// Value of an entry at its class (a promoted diagonal keeps FP32).
__device__ __forceinline__ double entry_value(const TileArgs &A, int t, int q, bool is_diag) {
    if (is_diag && A.prec[t] > MF_PREC_FP32) return (double)__double2float_rn(A.val[q]);
    return dequant(A, t, q);
}

__device__ __forceinline__ double class_round(int cls, double v) {
    return cls == MF_PREC_FP64 ? v : (double)__double2float_rn(v);
}

// Moves the cursor to the row's next entry of class `cls` (or past the end).
__device__ __forceinline__ void cursor_seek_class(const TileArgs &A, RowCursor &c, int cls, int row) {
    while (cursor_valid(c) && entry_class(A, c.t, entry_is_diag(A, c, row)) != cls) cursor_next(A, c);
}

// Row-sum-preserving compensation of a row (one lane per row): a row with
// exactly one diagonal entry a_ii > 0, every other entry <= 0 and a diagonal
// of class FP64 / FP32 stores its diagonal as the class value of
// a_ii - delta, delta = sum over the other entries in the reference's order
// of (dequantized - a_ij) in FP64. Writing A as a sum of edge terms
// (-a_ij)(e_i - e_j)(e_i - e_j)^T plus the diagonal of row sums, the rounding
// then only moves edge weights, each by at most u_p relative, so that for a
// symmetric diagonally dominant Z-matrix (1 - u) A <= A~ <= (1 + u) A: the
// low-precision operator stays positive definite with A's conditioning.
// Returns true and the diagonal's stored value when the row qualifies.
__device__ bool row_compensation(const TileArgs &A, RowCursor c, int row, double &diag_value) {
    int nd = 0;
    bool z = true;
    double delta = 0.0, aii = 0.0;
    int dcls = MF_PREC_FP64;
    for (; cursor_valid(c); cursor_next(A, c)) {
        const double a = A.val[c.q];
        if (entry_is_diag(A, c, row)) {
            ++nd;
            aii = a;
            dcls = entry_class(A, c.t, true);
        } else {
            if (!(a <= 0.0)) z = false;
            delta += entry_value(A, c.t, c.q, false) - a;
        }
    }
    if (nd != 1 || !z || !(aii > 0.0) || dcls > MF_PREC_FP32) return false;
    diag_value = class_round(dcls, aii - delta);
    return true;
}

// Storage format of one plane of class `cls` (warp-wide; lanes without an
// entry pass has = false). FP64 / FP32 classes store their own type. An
// FP16 (FP8) class plane is stored as FP16 (FP8) values times a common
// power-of-two 2^k when every nonzero value / 2^k is an exact normal number
// of that type, else in the next wider type that holds them exactly (the
// values carry at most 11 (4) significant bits).
__device__ void plane_format(int cls, bool has, double v, int &pprec, int &pexp) {
    const unsigned full = 0xffffffffu;
    pexp = 0;
    if (cls <= MF_PREC_FP32) {
        pprec = cls;
        return;
    }
    const bool nz = has && v != 0.0;
    const int e = nz ? ilogb(v) : 0;
    // the largest value's significand (for the FP8 maximum 448 = 1.75 * 2^8)
    const int emax = (int)__reduce_max_sync(full, nz ? (unsigned)(e + 4096) : 0u) - 4096;
    const int emin = (int)__reduce_min_sync(full, nz ? (unsigned)(e + 4096) : 0xffffffffu) - 4096;
    const bool anynz = __any_sync(full, nz);
    if (!anynz) {
        pprec = cls;
        return;
    }
    // scale 1 when the values fit as they are (the SpMV then skips the
    // multiply), else the largest value at the top of the type's range
    if (cls == MF_PREC_FP8) {
        const bool big = __any_sync(full, nz && e == emax && fabs(v) > 1.75 * ldexp(1.0, e));
        const int top = big ? 7 : 8;
        const int k = (emax <= top && emin >= -6) ? 0 : emax - top;
        if (emin - k >= -6 && k >= -126 && k <= 127) {
            pprec = MF_PREC_FP8;
            pexp = k;
            return;
        }
    }
    const int k = (emax <= 15 && emin >= -14) ? 0 : emax - 15;
    if (emin - k >= -14 && k >= -126 && k <= 127) {
        pprec = MF_PREC_FP16;
        pexp = k;
        return;
    }
    pprec = MF_PREC_FP32;
}

// Power-of-two scale of every FP16 / FP8 tile (1 for the others).
__global__ void k_tile_scales(int tilenum, const int *tile_off, const double *val, const unsigned char *prec,
                              float *scale) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= tilenum) return;
    const int vo = tile_off[t], nk = tile_off[t + 1] - vo;
    double mx = 0.0;
    for (int k = lane; k < nk; k += 32) mx = fmax(mx, fabs(val[vo + k]));
    for (int d = 16; d > 0; d >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    if (lane) return;
    const int p = prec[t];
    double s = 1.0;
    if (p >= MF_PREC_FP16 && mx > 0.0) {
        int e;
        frexp(mx, &e);
        if (p == MF_PREC_FP16) {
            s = ldexp(1.0, e - 15);
        } else {
            const double ratio = mx / 448.0;
            int k2;
            frexp(ratio, &k2);
            if (ldexp(1.0, k2 - 1) == ratio) k2 -= 1;
            s = ldexp(1.0, k2);
        }
    }
    scale[t] = (float)s;
}

// Per row block: plane count W and value bytes of the row-sliced block; in
// mixed layouts also the bytes of promoted diagonal entries beyond their
// tile's width (for the algorithmic byte count).
__global__ void k_rb_info(TileArgs A, bool mixed, int *rbW, unsigned *rbvb, unsigned *rbprom, uint8_t *rbaff) {
    const int lane = threadIdx.x & 31;
    const int rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (rb >= A.tilem) return;
    const int row = rb * 16 + lane;
    RowCursor c;
    cursor_init(A, c, rb, lane < 16 ? lane : 99);
    int cnt[4] = {0, 0, 0, 0};
    unsigned prom = 0;
    {
        RowCursor d = c;
        while (lane < 16 && cursor_valid(d)) {
            const bool dg = entry_is_diag(A, d, row);
            const int cl = mixed ? entry_class(A, d.t, dg) : MF_PREC_FP64;
            ++cnt[cl];
            if (mixed && dg && A.prec[d.t] > MF_PREC_FP32) prom += 4u - prec_width(A.prec[d.t]);
            cursor_next(A, d);
        }
    }
    int W = 0;
    unsigned vb = 0;
    bool aff = mixed && c.rl == 16;  // affine: see tiles.h
    for (int cl = 0; cl < 4; ++cl) {
        const int ncl = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt[cl]);
        W += ncl;
        if (!mixed) {
            vb += 128u * ncl;
            continue;
        }
        if (cl == MF_PREC_FP64 && ncl > 0) aff = false;
        RowCursor d = c;
        for (int j = 0; j < ncl; ++j) {
            if (lane < 16) cursor_seek_class(A, d, cl, row);
            const bool has = lane < 16 && cursor_valid(d);
            const double v = has ? entry_value(A, d.t, d.q, entry_is_diag(A, d, row)) : 0.0;
            int pp, pe;
            plane_format(cl, has, v, pp, pe);
            vb += 16u * prec_width(pp);
            // every row has an entry here, at the same offset from its row
            const int off = has ? A.tile_col[d.t] * 16 + (int)A.col[d.q] - row : 0;
            const unsigned full = 0xffffffffu;
            const bool all16 = __popc(__ballot_sync(full, has)) == 16;
            const int omin = (int)__reduce_min_sync(full, lane < 16 ? (unsigned)(off + (1 << 30)) : 0xffffffffu);
            const int omax = (int)__reduce_max_sync(full, lane < 16 ? (unsigned)(off + (1 << 30)) : 0u);
            if (!all16 || omin != omax) aff = false;
            if (has) cursor_next(A, d);
        }
    }
    prom = __reduce_add_sync(0xffffffffu, prom);
    if (lane == 0) {
        rbW[rb] = W;
        rbvb[rb] = vb;
        rbprom[rb] = prom;
        rbaff[rb] = aff ? 1 : 0;
    }
}

constexpr int FILL_THREADS = 256;

__global__ void __launch_bounds__(FILL_THREADS) k_fill_slabs(const SlabPlan *__restrict__ plans,
                                                             const int *__restrict__ slab_cta,
                                                             const int *__restrict__ cta_slab,
                                                             const int *__restrict__ segs,
                                                             const XRun *__restrict__ runs, TileArgs A,
                                                             const int *__restrict__ rbW,
                                                             const unsigned *__restrict__ rbvb,
                                                             const uint8_t *__restrict__ rbaff, bool mixed,
                                                             uint32_t segbytes, uint32_t zpos, uint8_t *slabs) {
    __shared__ uint32_t s_off[RB_PER_SLAB_MAX + 1];
    const int s = blockIdx.x;
    const SlabPlan P = plans[s];
    uint8_t *base = slabs + (size_t)P.off16 * 16;
    const bool gather = P.mode == SLAB_GATHER;
    for (uint32_t i = threadIdx.x * 16; i < P.bytes; i += FILL_THREADS * 16)
        *reinterpret_cast<uint4 *>(base + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
        SlabHeader h;
        memset(&h, 0, sizeof h);
        h.rb0 = P.rb0;
        h.nrb = (uint16_t)P.nrb;
        h.ntiles = (uint16_t)min(P.ntiles, 65535);
        h.nxseg = (uint16_t)P.nseg;
        h.mode = (uint16_t)P.mode;
        h.mixed = mixed ? 1 : 0;
        h.bytes = P.bytes;
        const int g = slab_cta[s];
        const int nx = s + STAGES;
        if (nx < cta_slab[g + 1]) {
            const SlabPlan Q = plans[nx];
            h.next_off16 = Q.off16;
            h.next_bytes = Q.bytes;
            h.next_xbytes = Q.mode == SLAB_STAGED ? (uint32_t)Q.nseg * segbytes : 0u;
            h.next_nruns = Q.mode == SLAB_STAGED ? (uint16_t)Q.nruns : 0;
            XRun *dst = reinterpret_cast<XRun *>(base + SLAB_HDR);
            for (int k = 0; k < h.next_nruns; ++k) dst[k] = runs[Q.run_off + k];
        }
        const int pf = s + 2 * STAGES;
        if (pf < cta_slab[g + 1]) {
            h.pf_off16 = plans[pf].off16;
            h.pf_bytes = plans[pf].bytes;
        }
        *reinterpret_cast<SlabHeader *>(base) = h;
        uint32_t off = slab_blocks_off(P.mode == SLAB_OVERSIZE ? 0 : P.nrb);
        RbDir *dir = reinterpret_cast<RbDir *>(base + slab_rbdir_off());
        if (P.mode != SLAB_OVERSIZE) {
            for (int j = 0; j < P.nrb; ++j) {
                s_off[j] = off;
                const int W = rbW[P.rb0 + j];
                dir[j].off = off;
                uint32_t dslot = 0;  // own column segment in the staged x window
                if (P.mode == SLAB_STAGED) {
                    const int *sg = segs + P.seg_off;
                    int lo = 0, hi = P.nseg;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (sg[mid] < P.rb0 + j) lo = mid + 1;
                        else hi = mid;
                    }
                    if (lo < P.nseg && sg[lo] == P.rb0 + j) dslot = (uint32_t)lo + 1u;
                }
                dir[j].W = (uint32_t)W | (dslot << 16);
                off += rb_block_bytes(W, mixed, gather, rbvb[P.rb0 + j], rbaff[P.rb0 + j] != 0);
            }
            dir[P.nrb].off = off;
            dir[P.nrb].W = 0;
        }
    }
    __syncthreads();
    if (P.mode == SLAB_OVERSIZE) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = warp; j < P.nrb; j += FILL_THREADS / 32) {
        const int rb = P.rb0 + j;
        const int W = rbW[rb];
        const int row = rb * 16 + lane;
        uint8_t *blk = base + s_off[j];
        RowCursor c;
        cursor_init(A, c, rb, lane < 16 ? lane : 99);
        // row lengths, class counts, compensation
        int len = 0, cnt[4] = {0, 0, 0, 0};
        {
            RowCursor d = c;
            while (lane < 16 && cursor_valid(d)) {
                ++len;
                ++cnt[mixed ? entry_class(A, d.t, entry_is_diag(A, d, row)) : MF_PREC_FP64];
                cursor_next(A, d);
            }
        }
        double diag_v = 0.0;
        const bool comp = mixed && lane < 16 && row_compensation(A, c, row, diag_v);
        const bool aff = mixed && !gather && rbaff[rb] != 0;
        if (!mixed && lane < 16) blk[lane] = (uint8_t)len;
        uint64_t pbits = 0;
        bool fast = true, unscaled = true;
        int8_t *sexp = reinterpret_cast<int8_t *>(blk + rbm_sexp_off());
        uint16_t *bases = reinterpret_cast<uint16_t *>(blk + rbm_base_off(W));
        uint8_t *idxb = blk + (mixed ? rbm_idx_off(W, aff) : rb_idx_off());
        uint8_t *vals = blk + (mixed ? rbm_vals_off(W, gather, aff) : rb_vals_off(W, gather));
        uint32_t voff = 0;
        int k = 0;
        for (int cl = 0; cl < 4; ++cl) {
            const int ncl = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt[cl]);
            if (mixed && lane == 0) blk[cl] = (uint8_t)ncl;
            RowCursor d = c;
            int prev_t = -1;  // previous entry's tile among this class (FP64 tile starts)
            for (int jj = 0; jj < ncl; ++jj, ++k) {
                if (mixed && lane < 16) cursor_seek_class(A, d, cl, row);
                const bool has = lane < 16 && cursor_valid(d);
                const bool dg = has && entry_is_diag(A, d, row);
                double v = 0.0;
                if (has) v = mixed ? (dg && comp ? diag_v : entry_value(A, d.t, d.q, dg)) : A.val[d.q];
                int pp = MF_PREC_FP64, pe = 0;
                if (mixed) {
                    plane_format(cl, has, v, pp, pe);
                    pbits |= (uint64_t)pp << (2 * k);
                    if (lane == 0) sexp[k] = (int8_t)pe;
                    if (pp != cl) fast = false;
                    if (pe != 0) unscaled = false;
                }
                if (has) {
                    const int t = d.t;
                    const bool start = t != prev_t;
                    prev_t = t;
                    const int colx = A.tile_col[t];
                    const int cin = A.col[d.q];
                    if (gather) {
                        uint32_t id = (uint32_t)(colx * 16 + cin);
                        if (start && cl == MF_PREC_FP64) id |= IDX32_START;
                        reinterpret_cast<uint32_t *>(idxb)[k * 16 + lane] = id;
                    } else {
                        int a = 0, b = P.nseg - 1;
                        while (a < b) {
                            const int mid = (a + b) >> 1;
                            if (segs[P.seg_off + mid] < colx) a = mid + 1; else b = mid;
                        }
                        uint32_t id = (uint32_t)(a * 16 + cin);
                        if (aff) {
                            if (lane == 0) bases[k] = (uint16_t)id;  // entry of row r at bases[k] + r
                        } else {
                            if (start && cl == MF_PREC_FP64) id |= IDX16_START;
                            reinterpret_cast<uint16_t *>(idxb)[k * 16 + lane] = (uint16_t)id;
                        }
                    }
                    uint8_t *pv = vals + voff;
                    const double sv = ldexp(v, -pe);  // exact: a power-of-two rescaling
                    if (pp == MF_PREC_FP64) {
                        reinterpret_cast<double *>(pv)[lane] = v;
                    } else if (pp == MF_PREC_FP32) {
                        reinterpret_cast<float *>(pv)[lane] = (float)v;  // exact: v is a class value
                    } else if (pp == MF_PREC_FP16) {
                        reinterpret_cast<__half *>(pv)[lane] = __double2half(sv);  // exact
                    } else {
                        pv[lane] = (uint8_t)__nv_cvt_double_to_fp8(sv, __NV_SATFINITE, __NV_E4M3);  // exact
                    }
                    cursor_next(A, d);
                } else if (lane < 16) {
                    // padding entry, value 0 (the zeroed slab): staged rows
                    // index the zero slot, gather rows carry the padding flag
                    if (gather) reinterpret_cast<uint32_t *>(idxb)[k * 16 + lane] = IDX32_PAD;
                    else reinterpret_cast<uint16_t *>(idxb)[k * 16 + lane] = (uint16_t)zpos;
                }
                voff += 16u * prec_width(pp);
            }
        }
        if (mixed && lane == 0) {
            *reinterpret_cast<uint64_t *>(blk + 8) = pbits;
            blk[4] = (uint8_t)((fast ? RBF_FAST : 0) | (aff ? RBF_AFFINE : 0) | (fast && unscaled ? RBF_UNSCALED : 0));
        }
    }
}


// ---- GPU slab planner ---------------------------------------------------------
// Plans every CTA's slabs on the device with the same greedy rules as the
// host planner (check_plans): one warp per CTA range. The lanes first copy
// the range's row-block data and tile columns into shared memory (when they
// fit; else they are read from global memory), then walk the row blocks
// together: a row block's tile columns enter the slab's x-segment set (a
// linear-probing hash set in shared memory) 32 at a time, a row block that
// does not fit is taken out again as a whole (removals are always of the
// latest inserts, so emptying their slots keeps the set consistent), and the
// warp sorts each staged slab's segments to form its runs. The plans, segments and runs go
// to CTA-local scratch (at most one slab per row block, one segment and one
// run per tile), with per-CTA counts; k_plan_compact then places them.
struct PlanArgs {
    const int *tile_ptr, *tile_col, *cta_rb, *rbW;
    const unsigned *rbvb;
    const uint8_t *rbaff;
    int tilen, mixed, xseg_max, slab_lim, rbps, maxw;
};
struct PlanCounts {  // per CTA
    int nslabs, nsegs, nruns, ngather, nover, pad;
    unsigned long long bytes;
    int cmin, cmax;  // smallest / largest tile column of the range (-1 when it has no tiles)
};
struct PlanScratch {  // CTA g: plans from cta_rb[g], segments and runs from tile_ptr[cta_rb[g]]
    SlabPlan *plans;  // off16 holds the CTA-local byte offset; seg_off / run_off are CTA-local
    int *segs;
    XRun *runs;
    uint8_t *over_rb;
};

constexpr int PLAN_HASH = 1024;    // > 2 * (the largest x window in segments + 1)
constexpr int PLAN_MEM = 512;      // members kept: fewer than xseg_max + 33 (a batch of 32 past it at most)
constexpr int PLAN_PRE_RB = 2048;  // row blocks of a CTA range prefetched into shared memory
constexpr int PLAN_PRE_T = 6144;   // tile columns prefetched
constexpr size_t PLAN_DYN_SMEM = (size_t)(PLAN_PRE_RB + 1) * 4 + (size_t)PLAN_PRE_RB * 9 + (size_t)PLAN_PRE_T * 4;

__global__ void __launch_bounds__(32) k_plan(PlanArgs A, PlanCounts *cnt, PlanScratch O) {
    extern __shared__ __align__(16) uint8_t pdyn[];
    __shared__ int hkey[PLAN_HASH];
    __shared__ int mem[PLAN_MEM], mslot[PLAN_MEM], sorted[PLAN_MEM];
    const unsigned full = 0xffffffffu;
    const int g = blockIdx.x, lane = threadIdx.x;
    for (int i = lane; i < PLAN_HASH; i += 32) hkey[i] = -1;
    const int lo = A.cta_rb[g], hi = A.cta_rb[g + 1];
    const int t0 = A.tile_ptr[lo], t1 = A.tile_ptr[hi];
    // the range's data in shared memory when it fits
    const bool pre_rb = hi - lo <= PLAN_PRE_RB, pre_t = t1 - t0 <= PLAN_PRE_T;
    int *s_tp = reinterpret_cast<int *>(pdyn);
    int *s_w = s_tp + PLAN_PRE_RB + 1;
    unsigned *s_vb = reinterpret_cast<unsigned *>(s_w + PLAN_PRE_RB);
    int *s_tc = reinterpret_cast<int *>(s_vb + PLAN_PRE_RB);
    uint8_t *s_aff = reinterpret_cast<uint8_t *>(s_tc + PLAN_PRE_T);
    if (pre_rb) {
        for (int i = lane; i <= hi - lo; i += 32) s_tp[i] = A.tile_ptr[lo + i];
        for (int i = lane; i < hi - lo; i += 32) {
            s_w[i] = A.rbW[lo + i];
            s_vb[i] = A.rbvb[lo + i];
            s_aff[i] = A.rbaff[lo + i];
        }
    }
    if (pre_t)
        for (int i = lane; i < t1 - t0; i += 32) s_tc[i] = A.tile_col[t0 + i];
    __syncwarp();
    auto TP = [&](int rb) { return pre_rb ? s_tp[rb - lo] : A.tile_ptr[rb]; };
    auto TC = [&](int k) { return pre_t ? s_tc[k - t0] : A.tile_col[k]; };
    auto RW = [&](int rb) { return pre_rb ? s_w[rb - lo] : A.rbW[rb]; };
    const bool mixed = A.mixed != 0;
    auto rb_bytes = [&](int rb, bool gather) {
        const unsigned vb = pre_rb ? s_vb[rb - lo] : A.rbvb[rb];
        const bool af = (pre_rb ? s_aff[rb - lo] : A.rbaff[rb]) != 0;
        return rb_block_bytes(RW(rb), mixed, gather, vb, af);
    };
    auto find = [&](int key) -> bool {
        if (key < 0 || key >= A.tilen) return false;
        for (uint32_t h = ((uint32_t)key * 2654435761u) & (PLAN_HASH - 1);; h = (h + 1) & (PLAN_HASH - 1)) {
            const int v = hkey[h];
            if (v == key) return true;
            if (v < 0) return false;
        }
    };
    // The slab's segment set: n members (mem[0..n), in batches) and its run
    // count, both uniform across the warp. add_rb adds a row block's tile
    // columns 32 at a time: with S the members before the batch and N its new
    // keys, runs grows by sum over N of 1 - [k-1 in S or N] - [k+1 in S].
    // Past xseg_max members the set stops growing (the slab cannot be staged:
    // only that fact is used, as by the host planner).
    int n = 0, runs = 0;
    auto add_rb = [&](int rb) {
        const int k0 = TP(rb), k1 = TP(rb + 1);
        for (int base = k0; base < k1 && n <= A.xseg_max; base += 32) {
            const int k = base + lane;
            const bool has = k < k1;
            const int key = has ? TC(k) : -1;
            const bool isnew = has && !find(key);
            const bool left_s = isnew && find(key - 1), right_s = isnew && find(key + 1);
            // tile columns ascend within a row block (Tile_create's order), so
            // among the batch's new keys only the previous lane's can be key - 1
            const int nk = isnew ? key : -2;
            const int nk_prev = __shfl_up_sync(full, nk, 1);
            const bool left_n = isnew && lane > 0 && nk_prev == key - 1;
            const int d = isnew ? 1 - ((left_s || left_n) ? 1 : 0) - (right_s ? 1 : 0) : 0;
            const unsigned bal = __ballot_sync(full, isnew);
            if (isnew) {
                uint32_t h = ((uint32_t)key * 2654435761u) & (PLAN_HASH - 1);
                while (atomicCAS(&hkey[h], -1, key) != -1) h = (h + 1) & (PLAN_HASH - 1);
                const int pos = n + __popc(bal & ((1u << lane) - 1u));
                mem[pos] = key;
                mslot[pos] = (int)h;
            }
            int dsum = d;
            for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(full, dsum, o);
            n += __popc(bal);
            runs += dsum;
            __syncwarp();
        }
    };
    auto clear_to = [&](int n0) {  // removes the members past n0 (whole batches)
        for (int i = n0 + lane; i < n; i += 32) hkey[mslot[i]] = -1;
        __syncwarp();
        n = n0;
    };
    SlabPlan *plans = O.plans + lo;
    int *segs = O.segs + t0;
    XRun *rout = O.runs + t0;
    int slab = 0, segpos = 0, runpos = 0, ngather = 0, nover = 0;
    unsigned long long bytepos = 0;
    int rb = lo;
    while (rb < hi) {
        const int rb0 = rb;
        int nrb = 1, mode;
        const int ntiles0 = TP(rb + 1) - TP(rb);
        int ntiles = ntiles0;
        uint32_t bytes;
        add_rb(rb);
        const bool staged0 = n <= A.xseg_max && runs <= MAXRUNS;
        const uint32_t tot0 = slab_blocks_off(1) + rb_bytes(rb, !staged0);
        bool staged = false;
        if (tot0 > (uint32_t)A.slab_lim || RW(rb) > A.maxw) {
            mode = SLAB_OVERSIZE;
            bytes = slab_blocks_off(0);
            ++nover;
            if (lane == 0) O.over_rb[rb] = 1;
        } else {
            staged = staged0;
            mode = staged ? SLAB_STAGED : SLAB_GATHER;
            uint32_t body = rb_bytes(rb, !staged);
            int nx = rb + 1;
            while (nx < hi && nrb < A.rbps) {
                if (RW(nx) > A.maxw) break;
                const uint32_t bx = rb_bytes(nx, !staged);
                if (slab_blocks_off(nrb + 1) + body + bx > (uint32_t)A.slab_lim) break;
                if (staged) {
                    const int n0 = n, r0 = runs;
                    add_rb(nx);
                    if (n > A.xseg_max || runs > MAXRUNS) {
                        clear_to(n0);
                        runs = r0;
                        break;
                    }
                }
                nrb += 1;
                ntiles += TP(nx + 1) - TP(nx);
                body += bx;
                ++nx;
            }
            bytes = slab_blocks_off(nrb) + body;
            if (!staged) ++ngather;
        }
        // ---- staged slabs: sort the segments (bitonic), write them and their runs
        int nseg = 0, nruns = 0;
        if (staged) {
            int m = 1;
            while (m < n) m <<= 1;
            for (int i = lane; i < m; i += 32) sorted[i] = i < n ? mem[i] : 0x7fffffff;
            __syncwarp();
            for (int k = 2; k <= m; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < m; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int a = sorted[i], b = sorted[l];
                            if ((a > b) == ((i & k) == 0)) {
                                sorted[i] = b;
                                sorted[l] = a;
                            }
                        }
                    }
                    __syncwarp();
                }
            nseg = n;
            for (int i = lane; i < n; i += 32) segs[segpos + i] = sorted[i];
            if (lane == 0) {
                for (int i = 0; i < n; ++i) {
                    if (i == 0 || sorted[i] != sorted[i - 1] + 1) rout[runpos + nruns++] = XRun{sorted[i], 0, (uint16_t)i};
                    rout[runpos + nruns - 1].nseg++;
                }
            }
            nruns = __shfl_sync(full, nruns, 0);
        }
        if (lane == 0) {
            SlabPlan P;
            P.rb0 = rb0;
            P.nrb = nrb;
            P.ntiles = ntiles;
            P.mode = mode;
            P.bytes = bytes;
            P.off16 = (uint32_t)bytepos;  // CTA-local byte offset until compaction
            P.seg_off = staged ? segpos : 0;
            P.nseg = nseg;
            P.run_off = staged ? runpos : 0;
            P.nruns = nruns;
            plans[slab] = P;
        }
        bytepos += bytes;
        rb = rb0 + nrb;
        clear_to(0);
        runs = 0;
        segpos += nseg;
        runpos += nruns;
        ++slab;
    }
    // the range's smallest / largest tile column (its x dependencies)
    int cmin = 0x7fffffff, cmax = -1;
    for (int k = t0 + lane; k < t1; k += 32) {
        const int c = TC(k);
        cmin = min(cmin, c);
        cmax = max(cmax, c);
    }
    for (int o = 16; o > 0; o >>= 1) {
        cmin = min(cmin, __shfl_xor_sync(full, cmin, o));
        cmax = max(cmax, __shfl_xor_sync(full, cmax, o));
    }
    if (lane == 0) {
        PlanCounts c;
        c.nslabs = slab;
        c.nsegs = segpos;
        c.nruns = runpos;
        c.ngather = ngather;
        c.nover = nover;
        c.pad = 0;
        c.bytes = bytepos;
        c.cmin = cmax < 0 ? -1 : cmin;
        c.cmax = cmax;
        cnt[g] = c;
    }
}

// Layout tallies over the tiles, one thread per row block: tiles per
// precision, algorithmic bytes (integers, so the sum is exact and
// deterministic), and whether a row block outside the oversize ones holds an
// FP64 tile. out: [0..3] tile counts, [4] bytes, [5] any FP64 tile.
__global__ void k_layout_tally(const int *tile_ptr, const int *tile_off, const uint8_t *prec, const uint8_t *over_rb,
                               const unsigned *rbprom, int tilem, int mixed, unsigned long long *out) {
    const int rb = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long c[4] = {0, 0, 0, 0}, bytes = 0, any64 = 0;
    if (rb < tilem) {
        const bool ov = over_rb[rb] != 0;
        for (int k = tile_ptr[rb]; k < tile_ptr[rb + 1]; ++k) {
            const int p = prec[k];
            const unsigned long long nnz = (unsigned long long)(tile_off[k + 1] - tile_off[k]);
            ++c[p];
            bytes += nnz * (prec_width(p) + 1u) + 8u + (p == MF_PREC_FP8 ? 4u : 0u);
            if (!ov && p == MF_PREC_FP64) any64 = 1;
        }
        if (mixed && !ov) bytes += rbprom[rb];
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int q = 0; q < 4; ++q) c[q] += __shfl_xor_sync(0xffffffffu, c[q], o);
        bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        any64 |= __shfl_xor_sync(0xffffffffu, any64, o);
    }
    if ((threadIdx.x & 31) == 0) {
        for (int q = 0; q < 4; ++q)
            if (c[q]) atomicAdd(&out[q], c[q]);
        if (bytes) atomicAdd(&out[4], bytes);
        if (any64) atomicOr(&out[5], 1ull);
    }
}

// Places CTA g's plans, segments and runs at the offsets of the counts'
// prefix sums (slab_base, seg_base, run_base, byte_base per CTA).
__global__ void k_plan_compact(const int *cta_rb, const int *tile_ptr, const PlanCounts *cnt, PlanScratch S,
                               const int *slab_base, const int *seg_base, const int *run_base,
                               const unsigned long long *byte_base, SlabPlan *plans, int *segs, XRun *runs,
                               int *slab_cta) {
    const int g = blockIdx.x;
    const int lo = cta_rb[g], t0 = tile_ptr[lo];
    const PlanCounts c = cnt[g];
    for (int i = threadIdx.x; i < c.nslabs; i += blockDim.x) {
        SlabPlan P = S.plans[lo + i];
        P.off16 = (uint32_t)((byte_base[g] + P.off16) / 16);
        if (P.mode == SLAB_STAGED) {
            P.seg_off += seg_base[g];
            P.run_off += run_base[g];
        }
        plans[slab_base[g] + i] = P;
        slab_cta[slab_base[g] + i] = g;
    }
    for (int i = threadIdx.x; i < c.nsegs; i += blockDim.x) segs[seg_base[g] + i] = S.segs[t0 + i];
    for (int i = threadIdx.x; i < c.nruns; i += blockDim.x) runs[run_base[g] + i] = S.runs[t0 + i];
}

// Issue records of the first STAGES slabs of every CTA (one thread per record).
__global__ void k_heads(const SlabPlan *__restrict__ plans, const XRun *__restrict__ runs, const int *cta_slab,
                        int G, uint32_t segbytes, uint8_t *head) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= G * STAGES) return;
    const int g = q / STAGES, k = q % STAGES;
    uint32_t *rec = reinterpret_cast<uint32_t *>(head + (size_t)q * ISSUE_REC);
    for (int i = 0; i < ISSUE_REC / 4; ++i) rec[i] = 0;
    const int s = cta_slab[g] + k;
    if (s >= cta_slab[g + 1]) return;
    const SlabPlan P = plans[s];
    rec[0] = P.off16;
    rec[1] = P.bytes;
    rec[2] = P.mode == SLAB_STAGED ? (uint32_t)P.nseg * segbytes : 0u;
    rec[3] = P.mode == SLAB_STAGED ? (uint32_t)P.nruns : 0u;
    if (P.mode == SLAB_STAGED) {
        XRun *dst = reinterpret_cast<XRun *>(rec + 4);
        for (int i = 0; i < P.nruns; ++i) dst[i] = runs[P.run_off + i];
    }
}

}  // namespace

// ---- planner check ------------------------------------------------------------
// The host planner (the reference for the GPU planner k_plan): the same
// greedy rules, one CTA range after another. Used only when the planner
// check is on, to compare every plan, segment and run with the GPU's.
static bool g_planner_check = false;
static long long g_planner_checked = 0, g_planner_mismatch = 0;
bool planner_check_on() { return g_planner_check; }

int check_plans(mf_tiles *t, int G, const std::vector<int> &cta_rb, const std::vector<int> &rbW,
                const std::vector<unsigned> &rbvb, const std::vector<uint8_t> &rbaff, bool mixed, bool x32,
                int xseg_max, int slab_lim, int rbps, int maxw, const std::vector<int> &cta_slab_gpu, int ns,
                int nsegs, int nruns, const DevArray<SlabPlan> &d_plans, const DevArray<int> &d_slab_cta,
                const DevArray<int> &d_segs, const DevArray<XRun> &d_runs, cudaStream_t st) {
    if (int rc = ensure_host_tiles(t)) return rc;
    const auto &tp = t->h_tile_ptr;
    const auto &tc = t->h_tile_col;
    auto rb_bytes = [&](int rb, bool gather) {
        return rb_block_bytes(rbW[rb], mixed, gather, rbvb[rb], rbaff[rb] != 0);
    };
    std::vector<SlabPlan> plans;
    std::vector<int> segs, slab_cta, cta_slab(G + 1, 0);
    std::vector<XRun> runs;
    std::vector<uint8_t> inseg((size_t)t->tilen + 2, 0);
    std::vector<int> members, cur;
    int seg_runs = 0;
    auto seg_add = [&](int s) {
        if (inseg[s + 1]) return;
        inseg[s + 1] = 1;
        members.push_back(s);
        seg_runs += 1 - inseg[s] - inseg[s + 2];
    };
    auto seg_drop_to = [&](size_t n) {
        while (members.size() > n) {
            const int s = members.back();
            members.pop_back();
            inseg[s + 1] = 0;
            seg_runs -= 1 - inseg[s] - inseg[s + 2];
        }
    };
    uint64_t off = 0;
    for (int g = 0; g < G; ++g) {
        cta_slab[g] = (int)plans.size();
        int rb = cta_rb[g];
        while (rb < cta_rb[g + 1]) {
            SlabPlan P;
            std::memset(&P, 0, sizeof P);
            P.rb0 = rb;
            for (int k = tp[rb]; k < tp[rb + 1]; ++k) seg_add(tc[k]);
            const bool staged0 = (int)members.size() <= xseg_max && seg_runs <= MAXRUNS;
            const uint32_t tot0 = slab_blocks_off(1) + rb_bytes(rb, !staged0);
            if (tot0 > (uint32_t)slab_lim || rbW[rb] > maxw) {
                P.mode = SLAB_OVERSIZE;
                P.nrb = 1;
                P.ntiles = tp[rb + 1] - tp[rb];
                P.bytes = slab_blocks_off(0);
                rb += 1;
            } else {
                const bool staged = staged0;
                P.mode = staged ? SLAB_STAGED : SLAB_GATHER;
                P.nrb = 1;
                P.ntiles = tp[rb + 1] - tp[rb];
                uint32_t body = rb_bytes(rb, !staged);
                int nx = rb + 1;
                while (nx < cta_rb[g + 1] && P.nrb < rbps) {
                    if (rbW[nx] > maxw) break;
                    const uint32_t bx = rb_bytes(nx, !staged);
                    if (slab_blocks_off(P.nrb + 1) + body + bx > (uint32_t)slab_lim) break;
                    if (staged) {
                        const size_t n0 = members.size();
                        for (int k = tp[nx]; k < tp[nx + 1]; ++k) seg_add(tc[k]);
                        if ((int)members.size() > xseg_max || seg_runs > MAXRUNS) {
                            seg_drop_to(n0);
                            break;
                        }
                    }
                    P.nrb += 1;
                    P.ntiles += tp[nx + 1] - tp[nx];
                    body += bx;
                    ++nx;
                }
                P.bytes = slab_blocks_off(P.nrb) + body;
                rb = nx;
            }
            if (P.mode == SLAB_STAGED) {
                cur.assign(members.begin(), members.end());
                std::sort(cur.begin(), cur.end());
                P.seg_off = (int)segs.size();
                P.nseg = (int)cur.size();
                segs.insert(segs.end(), cur.begin(), cur.end());
                P.run_off = (int)runs.size();
                for (size_t i = 0; i < cur.size(); ++i) {
                    if (i == 0 || cur[i] != cur[i - 1] + 1) runs.push_back(XRun{cur[i], 0, (uint16_t)i});
                    runs.back().nseg++;
                }
                P.nruns = (int)runs.size() - P.run_off;
            }
            P.off16 = (uint32_t)(off / 16);
            off += P.bytes;
            seg_drop_to(0);
            plans.push_back(P);
            slab_cta.push_back(g);
        }
    }
    cta_slab[G] = (int)plans.size();
    long long bad = 0;
    if ((int)plans.size() != ns || (int)segs.size() != nsegs || (int)runs.size() != nruns || cta_slab != cta_slab_gpu) {
        bad = 1;
    } else {
        std::vector<SlabPlan> gp(ns);
        std::vector<int> gs(nsegs), gsc(ns);
        std::vector<XRun> gr(nruns);
        if (ns) MF_CUDA_TRY(cudaMemcpyAsync(gp.data(), d_plans.p, sizeof(SlabPlan) * ns, cudaMemcpyDeviceToHost, st));
        if (ns) MF_CUDA_TRY(cudaMemcpyAsync(gsc.data(), d_slab_cta.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, st));
        if (nsegs) MF_CUDA_TRY(cudaMemcpyAsync(gs.data(), d_segs.p, sizeof(int) * nsegs, cudaMemcpyDeviceToHost, st));
        if (nruns) MF_CUDA_TRY(cudaMemcpyAsync(gr.data(), d_runs.p, sizeof(XRun) * nruns, cudaMemcpyDeviceToHost, st));
        MF_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < ns; ++i) {
            const SlabPlan &a = plans[i], &b = gp[i];
            if (a.rb0 != b.rb0 || a.nrb != b.nrb || a.ntiles != b.ntiles || a.mode != b.mode || a.bytes != b.bytes ||
                a.off16 != b.off16 || a.nseg != b.nseg || a.nruns != b.nruns ||
                (a.mode == SLAB_STAGED && (a.seg_off != b.seg_off || a.run_off != b.run_off)))
                ++bad;
        }
        if (gsc != slab_cta || gs != segs) ++bad;
        for (int i = 0; i < nruns; ++i)
            if (gr[i].seg0 != runs[i].seg0 || gr[i].nseg != runs[i].nseg || gr[i].slot0 != runs[i].slot0) ++bad;
    }
    (void)x32;
    ++g_planner_checked;
    g_planner_mismatch += bad;
    return MF_OK;
}

int build_layout(mf_tiles *t, Layout &L, const std::vector<uint8_t> &prec_in, cudaStream_t st) {
    auto t_start = std::chrono::steady_clock::now();
    const int tilem = t->tilem, tilenum = t->tilenum;
    const int G = t->G;
    const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
    const int slab_area = (slab_max + 127) & ~127;  // the solver kernels' slab area (solver.h)
    int slab_lim = slab_max;                         // largest slab of this layout
    const auto &tp = t->h_tile_ptr;
    std::vector<uint8_t> prec(prec_in);
    if ((int)prec.size() != tilenum) prec.assign(tilenum, MF_PREC_FP64);
    bool mixed = false;
    for (auto p : prec)
        if (p != MF_PREC_FP64) {
            mixed = true;
            break;
        }

    // device: tile scales, row-block plane counts and value bytes
    if (L.prec_dev.alloc(tilenum) || L.scale_dev.alloc(tilenum)) return MF_ERR_NOMEM;
    DevArray<int> d_rbW;
    DevArray<unsigned> d_rbvb, d_rbprom;
    DevArray<uint8_t> d_rbaff;
    if (d_rbW.alloc(tilem) || d_rbvb.alloc(tilem) || d_rbprom.alloc(tilem) || d_rbaff.alloc(tilem))
        return MF_ERR_NOMEM;
    if (tilenum > 0) {
        MF_CUDA_TRY(cudaMemcpyAsync(L.prec_dev.p, prec.data(), tilenum, cudaMemcpyHostToDevice, st));
        k_tile_scales<<<(tilenum + 7) / 8, 256, 0, st>>>(tilenum, t->tile_off.p, t->val.p, L.prec_dev.p,
                                                        L.scale_dev.p);
    }
    TileArgs A{t->tile_ptr.p, t->tile_col.p, t->tile_off.p, t->csrptr_off.p, t->ptr.p, t->val.p, t->col.p,
               L.prec_dev.p, L.scale_dev.p, tilem, t->rowA};
    k_rb_info<<<(tilem + 7) / 8, 256, 0, st>>>(A, mixed, d_rbW.p, d_rbvb.p, d_rbprom.p, d_rbaff.p);
    MF_CUDA_TRY(cudaGetLastError());
    std::vector<int> rbW(tilem);
    std::vector<unsigned> rbvb(tilem);
    std::vector<uint8_t> rbaff(tilem);
    MF_CUDA_TRY(cudaMemcpyAsync(rbW.data(), d_rbW.p, sizeof(int) * tilem, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaMemcpyAsync(rbvb.data(), d_rbvb.p, sizeof(unsigned) * tilem, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaMemcpyAsync(rbaff.data(), d_rbaff.p, tilem, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaStreamSynchronize(st));

    auto rb_bytes = [&](int rb, bool gather) {
        return rb_block_bytes(rbW[rb], mixed, gather, rbvb[rb], rbaff[rb] != 0);
    };
    const int maxw = mixed ? MAXW_MIXED : MAXW;
    // CTA ranges of equal cost, computed once per matrix and shared by every
    // layout so that all layouts give each CTA the same rows
    if ((int)t->h_cta_rb.size() != G + 1) {
        std::vector<double> pref(tilem + 1, 0.0);
        for (int rb = 0; rb < tilem; ++rb) pref[rb + 1] = pref[rb] + (double)rb_bytes(rb, false) + 16.0 * 72.0;
        std::vector<int> part(G + 1, tilem);
        part[0] = 0;
        int rb = 0;
        for (int g = 1; g < G; ++g) {
            const double target = pref[tilem] * g / G;
            while (rb < tilem && pref[rb] < target) ++rb;
            part[g] = rb;
        }
        part[G] = tilem;
        t->h_cta_rb.swap(part);
    }
    const std::vector<int> &cta_rb = t->h_cta_rb;
    // Layouts whose tiles are all below FP64 stage x in FP32 (64-byte
    // segments): twice the x window per stage, so slabs may hold twice the
    // row blocks. An oversize row block turns its tiles FP64, and then the
    // layout is planned again with FP64 x.
    bool x32 = mixed;
    for (size_t k = 0; k < prec.size() && x32; ++k) x32 = prec[k] != MF_PREC_FP64;
    // slabs: planned on the GPU (k_plan into CTA-local scratch, counts,
    // k_plan_compact). With the planner check on (mf_check_planner), the host
    // planner plans the same layout and every plan, segment and run is
    // compared.
    int n_gather = 0, n_over = 0, xseg_max = XSEG_MAX, rbps = RB_PER_SLAB_X64;
    uint32_t segbytes = 128u;
    DevArray<int> d_cta_rb, d_sb, d_gb, d_rbase;
    DevArray<unsigned long long> d_bb;
    DevArray<PlanCounts> d_cnt;
    DevArray<SlabPlan> d_plans, sc_plans;
    DevArray<int> d_slab_cta, d_segs, sc_segs;
    DevArray<XRun> d_runs, sc_runs;
    DevArray<uint8_t> d_over;
    if (d_cta_rb.alloc(G + 1) || d_cnt.alloc(G) || d_sb.alloc(G) || d_gb.alloc(G) || d_rbase.alloc(G) ||
        d_bb.alloc(G) || d_over.alloc(tilem) || sc_plans.alloc(tilem) || sc_segs.alloc(tilenum) ||
        sc_runs.alloc(tilenum))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpyAsync(d_cta_rb.p, cta_rb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    static bool plan_smem_set = false;
    if (!plan_smem_set) {
        MF_CUDA_TRY(cudaFuncSetAttribute(k_plan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PLAN_DYN_SMEM));
        plan_smem_set = true;
    }
    std::vector<int> cta_slab(G + 1, 0);
    std::vector<PlanCounts> hcnt;
    uint64_t off = 0;
    int ns = 0, nsegs = 0, nruns = 0;
    for (;;) {
        xseg_max = x32 ? xseg_max32(slab_area) : XSEG_MAX;
        segbytes = x32 ? 64u : 128u;
        rbps = t->opt.rb_per_slab > 0 ? std::min(t->opt.rb_per_slab, RB_PER_SLAB_MAX)
                                      : (x32 ? RB_PER_SLAB_X32 : RB_PER_SLAB_X64);
        slab_lim = x32 ? x_off_of(slab_area, true) : slab_max;
        const PlanArgs pa{t->tile_ptr.p, t->tile_col.p, d_cta_rb.p, d_rbW.p, d_rbvb.p, d_rbaff.p, t->tilen,
                          mixed ? 1 : 0, xseg_max, slab_lim, rbps, maxw};
        MF_CUDA_TRY(cudaMemsetAsync(d_over.p, 0, tilem, st));
        k_plan<<<G, 32, PLAN_DYN_SMEM, st>>>(pa, d_cnt.p, PlanScratch{sc_plans.p, sc_segs.p, sc_runs.p, d_over.p});
        MF_CUDA_TRY(cudaGetLastError());
        hcnt.assign(G, PlanCounts{});
        std::vector<PlanCounts> &hc = hcnt;
        MF_CUDA_TRY(cudaMemcpyAsync(hc.data(), d_cnt.p, sizeof(PlanCounts) * G, cudaMemcpyDeviceToHost, st));
        MF_CUDA_TRY(cudaStreamSynchronize(st));
        std::vector<int> sb(G), gb(G), rbase(G);
        std::vector<unsigned long long> bb(G);
        ns = nsegs = nruns = 0;
        off = 0;
        n_gather = n_over = 0;
        for (int g = 0; g < G; ++g) {
            cta_slab[g] = sb[g] = ns;
            gb[g] = nsegs;
            rbase[g] = nruns;
            bb[g] = off;
            ns += hc[g].nslabs;
            nsegs += hc[g].nsegs;
            nruns += hc[g].nruns;
            off += hc[g].bytes;
            n_gather += hc[g].ngather;
            n_over += hc[g].nover;
        }
        cta_slab[G] = ns;
        if (x32 && n_over > 0) {  // planned again with FP64 x
            x32 = false;
            continue;
        }
        if (d_plans.alloc(ns) || d_slab_cta.alloc(ns) || d_segs.alloc(nsegs) || d_runs.alloc(nruns))
            return MF_ERR_NOMEM;
        MF_CUDA_TRY(cudaMemcpyAsync(d_sb.p, sb.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
        MF_CUDA_TRY(cudaMemcpyAsync(d_gb.p, gb.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
        MF_CUDA_TRY(cudaMemcpyAsync(d_rbase.p, rbase.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
        MF_CUDA_TRY(cudaMemcpyAsync(d_bb.p, bb.data(), sizeof(unsigned long long) * G, cudaMemcpyHostToDevice, st));
        k_plan_compact<<<G, 128, 0, st>>>(d_cta_rb.p, t->tile_ptr.p, d_cnt.p,
                                           PlanScratch{sc_plans.p, sc_segs.p, sc_runs.p, d_over.p}, d_sb.p, d_gb.p,
                                           d_rbase.p, d_bb.p, d_plans.p, d_segs.p, d_runs.p, d_slab_cta.p);
        MF_CUDA_TRY(cudaGetLastError());
        break;
    }
    if (off / 16 > 0xffffffffull) {
        set_last_error("slab layout exceeds 64 GiB");
        return MF_ERR_UNSUPPORTED;
    }
    // oversize row blocks are computed in FP64 from the tile arrays
    std::vector<uint8_t> over(tilem, 0);
    if (n_over > 0) {
        if (int rc = ensure_host_tiles(t)) return rc;
        MF_CUDA_TRY(cudaMemcpyAsync(over.data(), d_over.p, tilem, cudaMemcpyDeviceToHost, st));
        MF_CUDA_TRY(cudaStreamSynchronize(st));
        for (int rb = 0; rb < tilem; ++rb)
            if (over[rb])
                for (int k = tp[rb]; k < tp[rb + 1]; ++k) prec[k] = MF_PREC_FP64;
        if (tilenum > 0) {
            MF_CUDA_TRY(cudaMemcpyAsync(L.prec_dev.p, prec.data(), tilenum, cudaMemcpyHostToDevice, st));
            k_tile_scales<<<(tilenum + 7) / 8, 256, 0, st>>>(tilenum, t->tile_off.p, t->val.p, L.prec_dev.p,
                                                            L.scale_dev.p);
        }
    }
    if (planner_check_on()) {
        const int rc = check_plans(t, G, cta_rb, rbW, rbvb, rbaff, mixed, x32, xseg_max, slab_lim, rbps, maxw,
                                   cta_slab, ns, nsegs, nruns, d_plans, d_slab_cta, d_segs, d_runs, st);
        if (rc) return rc;
    }
    // issue records of the first STAGES slabs of every CTA
    if (L.head.alloc((size_t)G * STAGES * ISSUE_REC) || L.cta_slab.alloc(G + 1)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_slab.p, cta_slab.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    k_heads<<<(G * STAGES + 127) / 128, 128, 0, st>>>(d_plans.p, d_runs.p, L.cta_slab.p, G, segbytes, L.head.p);
    MF_CUDA_TRY(cudaGetLastError());
    // dependency ranges: CTAs owning the x segments a CTA reads (each
    // range's smallest / largest tile column comes with the plan counts)
    std::vector<int> dep(2 * G);
    for (int g = 0; g < G; ++g) {
        int cmin = hcnt[g].cmin, cmax = hcnt[g].cmax;
        if (cmax < 0) {
            dep[2 * g] = g;
            dep[2 * g + 1] = g - 1;  // empty range
            continue;
        }
        cmin = std::min(cmin, tilem - 1);
        cmax = std::min(cmax, tilem - 1);
        auto owner = [&](int c) {
            return (int)(std::upper_bound(cta_rb.begin(), cta_rb.end(), c) - cta_rb.begin()) - 1;
        };
        dep[2 * g] = owner(cmin);
        dep[2 * g + 1] = owner(cmax);
    }
    // tiles per precision, algorithmic bytes and the layout kind (oversize
    // row blocks run in FP64 from the tile arrays and do not count)
    DevArray<unsigned long long> d_tally;
    if (d_tally.alloc(6)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemsetAsync(d_tally.p, 0, sizeof(unsigned long long) * 6, st));
    if (tilem > 0)
        k_layout_tally<<<(tilem + 255) / 256, 256, 0, st>>>(t->tile_ptr.p, t->tile_off.p, L.prec_dev.p, d_over.p,
                                                            d_rbprom.p, tilem, mixed ? 1 : 0, d_tally.p);
    MF_CUDA_TRY(cudaGetLastError());
    unsigned long long tally[6];
    MF_CUDA_TRY(cudaMemcpyAsync(tally, d_tally.p, sizeof tally, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaStreamSynchronize(st));
    int kind = LAYOUT_FP64;
    if (mixed) {
        kind = tally[5] ? LAYOUT_ANY : LAYOUT_LOW;
        // the LOW row path reads FP32 x: a layout planned with FP64 x (after
        // an oversize row block) takes the general path, which rounds x per
        // entry to the same FP32 value
        if (kind == LAYOUT_LOW && !x32) kind = LAYOUT_ANY;
    }
    const double alg = 16.0 * (double)t->rowA + (double)tally[4];
    double cnt[4];
    for (int q = 0; q < 4; ++q) cnt[q] = (double)tally[q];
    // fill
    if (L.slabs.alloc(off + 16) || L.cta_rb.alloc(G + 1) || L.cta_dep.alloc(2 * G)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_rb.p, cta_rb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_dep.p, dep.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
    if (ns > 0)
        k_fill_slabs<<<ns, FILL_THREADS, 0, st>>>(d_plans.p, d_slab_cta.p, L.cta_slab.p, d_segs.p, d_runs.p, A,
                                                 d_rbW.p, d_rbvb.p, d_rbaff.p, mixed, segbytes,
                                                 zero_pos_of(slab_area, x32), L.slabs.p);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaStreamSynchronize(st));
    L.prec.swap(prec);
    L.G = G;
    L.nslabs = ns;
    L.n_gather = n_gather;
    L.n_oversize = n_over;
    L.slab_max = slab_max;
    L.rb_per_slab = rbps;
    L.mixed = mixed;
    L.kind = kind;
    L.x32 = x32;
    L.bytes = off;
    L.alg_bytes = alg;
    for (int p = 0; p < 4; ++p) L.tile_frac[p] = tilenum > 0 ? cnt[p] / tilenum : 0.0;
    L.built = true;
    t->layout_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return MF_OK;
}

}  // namespace mf

extern "C" int mf_check_planner(int on, long long *checked, long long *mismatches) {
    const int prev = mf::g_planner_check ? 1 : 0;
    if (on >= 0) {
        mf::g_planner_check = on != 0;
        mf::g_planner_checked = mf::g_planner_mismatch = 0;
    }
    if (checked) *checked = mf::g_planner_checked;
    if (mismatches) *mismatches = mf::g_planner_mismatch;
    return prev;
}
