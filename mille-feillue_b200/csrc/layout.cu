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

}  // namespace

int build_layout(mf_tiles *t, Layout &L, const std::vector<uint8_t> &prec_in, cudaStream_t st) {
    auto t_start = std::chrono::steady_clock::now();
    const int tilem = t->tilem, tilenum = t->tilenum;
    const int G = t->G;
    const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
    const int slab_area = (slab_max + 127) & ~127;  // the solver kernels' slab area (solver.h)
    int slab_lim = slab_max;                         // largest slab of this layout
    const auto &tp = t->h_tile_ptr;
    const auto &tc = t->h_tile_col;
    const auto &tn = t->h_tile_nnz;
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
    std::vector<unsigned> rbvb(tilem), rbprom(tilem);
    std::vector<uint8_t> rbaff(tilem);
    MF_CUDA_TRY(cudaMemcpyAsync(rbW.data(), d_rbW.p, sizeof(int) * tilem, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaMemcpyAsync(rbvb.data(), d_rbvb.p, sizeof(unsigned) * tilem, cudaMemcpyDeviceToHost, st));
    MF_CUDA_TRY(cudaMemcpyAsync(rbprom.data(), d_rbprom.p, sizeof(unsigned) * tilem, cudaMemcpyDeviceToHost, st));
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
    // slabs: the CTAs' row-block ranges are planned independently (on up to
    // 16 host threads for large matrices) and concatenated in CTA order
    std::vector<SlabPlan> plans;
    std::vector<int> seg_all;
    std::vector<XRun> run_all;
    std::vector<int> slab_cta;
    std::vector<int> cta_slab(G + 1, 0);
    struct Part {  // one thread's CTAs
        std::vector<SlabPlan> plans;
        std::vector<int> segs, nslab;
        std::vector<XRun> runs;
        int n_gather = 0, n_over = 0;
    };
    int n_gather = 0, n_over = 0, xseg_max = XSEG_MAX, rbps = RB_PER_SLAB_X64;
    uint32_t segbytes = 128u;
    auto plan_ctas = [&](int g0, int g1, Part &out) {
        // x segments (tile columns) of the slab being planned, kept
        // incrementally since a row block adds only a few: membership (offset
        // by one so that s - 1 and s + 1 are always addressable), the members
        // in insertion order, and the number of runs of consecutive segments
        std::vector<uint8_t> inseg((size_t)t->tilen + 2, 0);
        std::vector<int> members, cur;
        int seg_runs = 0;
        auto seg_add = [&](int s) {
            if (inseg[s + 1]) return;
            inseg[s + 1] = 1;
            members.push_back(s);
            seg_runs += 1 - inseg[s] - inseg[s + 2];
        };
        auto seg_drop_to = [&](size_t n) {  // undo the adds past the first n, newest first
            while (members.size() > n) {
                const int s = members.back();
                members.pop_back();
                inseg[s + 1] = 0;
                seg_runs -= 1 - inseg[s] - inseg[s + 2];
            }
        };
        for (int g = g0; g < g1; ++g) {
            const size_t first = out.plans.size();
            int rb = cta_rb[g];
            while (rb < cta_rb[g + 1]) {
                SlabPlan P{};
                P.rb0 = rb;
                for (int k = tp[rb]; k < tp[rb + 1]; ++k) seg_add(tc[k]);
                const bool staged0 = (int)members.size() <= xseg_max && seg_runs <= MAXRUNS;
                const uint32_t tot0 = slab_blocks_off(1) + rb_bytes(rb, !staged0);
                if (tot0 > (uint32_t)slab_lim || rbW[rb] > maxw) {
                    P.mode = SLAB_OVERSIZE;
                    P.nrb = 1;
                    P.ntiles = tp[rb + 1] - tp[rb];
                    P.bytes = slab_blocks_off(0);
                    for (int k = tp[rb]; k < tp[rb + 1]; ++k) prec[k] = MF_PREC_FP64;  // this CTA's tiles only
                    ++out.n_over;
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
                    if (!staged) ++out.n_gather;
                    rb = nx;
                }
                if (P.mode == SLAB_STAGED) {
                    cur.assign(members.begin(), members.end());
                    std::sort(cur.begin(), cur.end());
                    P.seg_off = (int)out.segs.size();  // within this part; offset at the merge
                    P.nseg = (int)cur.size();
                    out.segs.insert(out.segs.end(), cur.begin(), cur.end());
                    P.run_off = (int)out.runs.size();
                    for (size_t i = 0; i < cur.size(); ++i) {
                        if (i == 0 || cur[i] != cur[i - 1] + 1) out.runs.push_back(XRun{cur[i], 0, (uint16_t)i});
                        out.runs.back().nseg++;
                    }
                    P.nruns = (int)out.runs.size() - P.run_off;
                }
                seg_drop_to(0);
                out.plans.push_back(P);
            }
            out.nslab.push_back((int)(out.plans.size() - first));
        }
    };
    for (;;) {
        xseg_max = x32 ? xseg_max32(slab_area) : XSEG_MAX;
        slab_lim = x32 ? x_off_of(slab_area, true) : slab_max;
        segbytes = x32 ? 64u : 128u;
        rbps = t->opt.rb_per_slab > 0 ? std::min(t->opt.rb_per_slab, RB_PER_SLAB_MAX)
                                      : (x32 ? RB_PER_SLAB_X32 : RB_PER_SLAB_X64);
        const unsigned hw = std::thread::hardware_concurrency();
        const int nth = tilem >= 16384 ? std::max(1, std::min({16, (int)(hw ? hw : 1), G})) : 1;
        std::vector<Part> parts(nth);
        if (nth == 1) {
            plan_ctas(0, G, parts[0]);
        } else {
            std::vector<std::thread> th;
            for (int i = 0; i < nth; ++i)
                th.emplace_back(plan_ctas, (int)((long long)G * i / nth), (int)((long long)G * (i + 1) / nth),
                                std::ref(parts[i]));
            for (auto &x : th) x.join();
        }
        plans.clear();
        seg_all.clear();
        run_all.clear();
        slab_cta.clear();
        cta_slab.assign(G + 1, 0);
        n_gather = n_over = 0;
        int g = 0;
        for (auto &pt : parts) {
            const int soff = (int)seg_all.size(), roff = (int)run_all.size();
            size_t k = 0;
            for (int cnt : pt.nslab) {
                cta_slab[g] = (int)plans.size();
                for (int j = 0; j < cnt; ++j, ++k) {
                    SlabPlan P = pt.plans[k];
                    if (P.mode == SLAB_STAGED) {
                        P.seg_off += soff;
                        P.run_off += roff;
                    }
                    plans.push_back(P);
                    slab_cta.push_back(g);
                }
                ++g;
            }
            seg_all.insert(seg_all.end(), pt.segs.begin(), pt.segs.end());
            run_all.insert(run_all.end(), pt.runs.begin(), pt.runs.end());
            n_gather += pt.n_gather;
            n_over += pt.n_over;
        }
        cta_slab[G] = (int)plans.size();
        if (x32 && n_over > 0) {
            x32 = false;
            prec = prec_in;
            if ((int)prec.size() != tilenum) prec.assign(tilenum, MF_PREC_FP64);
            continue;
        }
        break;
    }
    const int ns = (int)plans.size();
    uint64_t off = 0;
    for (auto &P : plans) {
        P.off16 = (uint32_t)(off / 16);
        off += P.bytes;
    }
    if (off / 16 > 0xffffffffull) {
        set_last_error("slab layout exceeds 64 GiB");
        return MF_ERR_UNSUPPORTED;
    }
    // oversize row blocks are computed in FP64 from the tile arrays
    if (n_over > 0 && tilenum > 0) {
        MF_CUDA_TRY(cudaMemcpyAsync(L.prec_dev.p, prec.data(), tilenum, cudaMemcpyHostToDevice, st));
        k_tile_scales<<<(tilenum + 7) / 8, 256, 0, st>>>(tilenum, t->tile_off.p, t->val.p, L.prec_dev.p,
                                                        L.scale_dev.p);
    }
    // issue records of the first STAGES slabs of every CTA
    std::vector<uint8_t> head((size_t)G * STAGES * ISSUE_REC, 0);
    for (int g = 0; g < G; ++g)
        for (int k = 0; k < STAGES; ++k) {
            const int s = cta_slab[g] + k;
            uint32_t *rec = reinterpret_cast<uint32_t *>(&head[((size_t)g * STAGES + k) * ISSUE_REC]);
            if (s >= cta_slab[g + 1]) continue;
            const SlabPlan &P = plans[s];
            rec[0] = P.off16;
            rec[1] = P.bytes;
            rec[2] = P.mode == SLAB_STAGED ? (uint32_t)P.nseg * segbytes : 0u;
            rec[3] = P.mode == SLAB_STAGED ? (uint32_t)P.nruns : 0u;
            if (P.mode == SLAB_STAGED) std::memcpy(&rec[4], &run_all[P.run_off], sizeof(XRun) * P.nruns);
        }
    // dependency ranges: CTAs owning the x segments a CTA reads
    std::vector<int> dep(2 * G);
    for (int g = 0; g < G; ++g) {
        int cmin = INT32_MAX, cmax = -1;
        for (int k = tp[cta_rb[g]]; k < tp[cta_rb[g + 1]]; ++k) {
            cmin = std::min(cmin, tc[k]);
            cmax = std::max(cmax, tc[k]);
        }
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
    // layout kind (oversize row blocks run in FP64 from the tile arrays and
    // do not count)
    int kind = LAYOUT_FP64;
    if (mixed) {
        bool any64 = false;
        for (const auto &P : plans)
            if (P.mode != SLAB_OVERSIZE)
                for (int k = tp[P.rb0]; k < tp[P.rb0 + P.nrb] && !any64; ++k) any64 = prec[k] == MF_PREC_FP64;
        kind = any64 ? LAYOUT_ANY : LAYOUT_LOW;
        // the LOW row path reads FP32 x: a layout planned with FP64 x (after
        // an oversize row block) takes the general path, which rounds x per
        // entry to the same FP32 value
        if (kind == LAYOUT_LOW && !x32) kind = LAYOUT_ANY;
    }
    // algorithmic bytes and precision fractions
    double alg = 16.0 * (double)t->rowA;
    double cnt[4] = {0, 0, 0, 0};
    for (int k = 0; k < tilenum; ++k) {
        alg += tile_alg_bytes(prec[k], tn[k]);
        cnt[prec[k]] += 1;
    }
    // diagonal entries of FP16 / FP8 tiles are stored in FP32 (oversize row
    // blocks hold FP64 tiles only)
    if (mixed)
        for (const auto &P : plans)
            if (P.mode != SLAB_OVERSIZE)
                for (int rb = P.rb0; rb < P.rb0 + P.nrb; ++rb) alg += (double)rbprom[rb];
    // upload and fill
    DevArray<SlabPlan> d_plans;
    DevArray<int> d_slab_cta, d_segs;
    DevArray<XRun> d_runs;
    if (L.slabs.alloc(off + 16) || L.head.alloc(head.size()) || L.cta_slab.alloc(G + 1) ||
        L.cta_rb.alloc(G + 1) || L.cta_dep.alloc(2 * G) || d_plans.alloc(ns) || d_slab_cta.alloc(ns) ||
        d_segs.alloc(seg_all.size()) || d_runs.alloc(run_all.size()))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpyAsync(L.head.p, head.data(), head.size(), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_slab.p, cta_slab.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_rb.p, cta_rb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_dep.p, dep.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
    if (ns > 0) {
        MF_CUDA_TRY(cudaMemcpyAsync(d_plans.p, plans.data(), sizeof(SlabPlan) * ns, cudaMemcpyHostToDevice, st));
        MF_CUDA_TRY(cudaMemcpyAsync(d_slab_cta.p, slab_cta.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    }
    if (!seg_all.empty())
        MF_CUDA_TRY(cudaMemcpyAsync(d_segs.p, seg_all.data(), sizeof(int) * seg_all.size(), cudaMemcpyHostToDevice, st));
    if (!run_all.empty())
        MF_CUDA_TRY(cudaMemcpyAsync(d_runs.p, run_all.data(), sizeof(XRun) * run_all.size(), cudaMemcpyHostToDevice, st));
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
