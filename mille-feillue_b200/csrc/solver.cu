// Persistent single-kernel solvers and the tiled SpMV for sm_100a.
//
// One CTA per SM (or more, from the occupancy query) owns a contiguous range
// of row blocks for the whole solve. Its matrix slabs stream from HBM into a
// STAGES-deep shared-memory ring with 1D bulk copies (cp.async.bulk, mbarrier
// completion, L2 evict_first); the x segments each slab needs are staged by
// the same mechanism as contiguous runs. One thread per matrix row sums the
// row in the order of blockspmv_cpu (Performance-Comparison/blockspmv_cpu.h:
// 85-112): per tile in ascending column, sum = 0, sum += x*v in stored order,
// then y += sum; FP64 tiles use non-fused multiply/add, so the result is
// bit-identical to that loop.
//
// Grid-wide dot products: each CTA reduces its partial in a fixed order,
// stores it in a double-buffered slot, then arrives on a monotonic counter
// with a release add; every CTA waits with acquire loads until all G CTAs
// arrived, then sums the G partials in the same fixed order, so all CTAs
// hold the identical value (no grid.sync, no kernel boundary). Vector halos
// between iterations use per-CTA epoch flags (st.release / ld.acquire) that
// only the CTAs whose rows a CTA reads are waited on. Every wait is bounded
// by %globaltimer; on expiry the kernel records MF_ERR_TIMEOUT and returns.
//
// The recurrences follow Mille-feuille_CG_NVIDIA.cu:722-804 (CG) and
// Mille-feuille_BiCGSTAB_NVIDIA.cu:787-1061 (BiCGSTAB), run to a tolerance
// instead of a fixed iteration count. The FP64 BiCGSTAB computes the same
// iterates with two grid reductions an iteration instead of three
// (r^.r_new = r^.s - omega r^.t): equal in exact arithmetic, rounded
// differently.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "solver.h"
#include "tiles.h"

namespace mf {

// ---------------------------------------------------------------- smem
struct __align__(16) Smem {
    uint64_t full[STAGES];   // slab + x runs landed (producer arrive + tx bytes)
    uint64_t empty[STAGES];  // every consumer warp is done with the stage
    uint64_t upd;            // bulk copies of the own rows' vectors (vector pass)
    uint32_t abort;
    uint8_t res_tag[STAGES];  // 1 + layout whose slab (index = stage) the stage holds; 0: none
    int slab0[KMAX_LAYOUTS], slab1[KMAX_LAYOUTS];
    double red[NWARPS + 1][4];
    double bres[4];
    uint8_t head[KMAX_LAYOUTS][STAGES][ISSUE_REC];
};

__device__ __forceinline__ uint8_t *stage_ptr(uint8_t *dyn, int k, int stride) { return dyn + (size_t)k * stride; }

// The standalone SpMV launch has no sync block (sync == nullptr): a timeout
// there only aborts the CTA.
__device__ void set_error_w(uint32_t *sync, uint32_t code, uint32_t site) {
    if (sync && atomicCAS(sync + SYNC_ERROR, 0u, code) == 0u) atomicExch(sync + SYNC_SITE, site);
}
__device__ void set_error(const KParams &P, uint32_t code, uint32_t site) { set_error_w(P.sync, code, site); }

// Thread 0: issue the bulk copies of one slab (x runs first, slab last: the
// issue record may live inside the stage the slab overwrites).
// An x segment is 16 entries: 128 bytes of FP64 x, 64 bytes of FP32 x.
__device__ void issue_slab(Smem &S, uint8_t *stage, int xoff, int k, uint32_t off16, uint32_t bytes,
                           uint32_t xbytes, int nruns, const XRun *runs, const uint8_t *slabs,
                           const uint8_t *xv, uint32_t segb, uint64_t pol_m, uint64_t pol_v) {
    mbar_arrive_expect_tx(&S.full[k], bytes + xbytes);
    uint8_t *xarea = stage + xoff;
    for (int q = 0; q < nruns; ++q) {
        const XRun r = runs[q];
        bulk_g2s(xarea + (size_t)r.slot0 * segb, xv + (size_t)r.seg0 * segb, (uint32_t)r.nseg * segb, &S.full[k],
                 pol_v);
    }
    bulk_g2s(stage, slabs + (size_t)off16 * 16, bytes, &S.full[k], pol_m);
}

// Pipeline state kept in registers across SpMV calls: consumer parity of
// each stage's full barrier, producer parity of each stage's empty barrier,
// and the stages filled at least once (whose refill must wait for empty).
struct Pipe {
    uint32_t fph = 0, eph = 0, filled = 0;
};

__device__ bool wait_bar(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((spin & 15u) == 0 && globaltimer() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ float to_f32(double v) { return __double2float_rn(v); }
__device__ __forceinline__ float to_f32(float v) { return v; }

__device__ __forceinline__ float exp2_int(int e) { return __int_as_float((e + 127) << 23); }  // e in [-126, 127]
__device__ __forceinline__ float fp8_to_float(uint8_t b) {
    return __half2float(__half(__nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)b, __NV_E4M3)));
}

// x-window position source of a staged mixed row block, one instruction
// stream for both kinds: plane k of lane r sits at (p[k * stride] & POS) +
// add, with p = base, stride 1, add = r for affine blocks and p = idx + r,
// stride 16, add 0 otherwise (two half-warps of a warp may hold one of each
// without diverging).
struct PosSrc {
    const uint16_t *p;
    uint32_t stride, add;
    __device__ __forceinline__ uint32_t operator()(int k) const {
        return ((uint32_t)p[(uint32_t)k * stride] & IDX16_POS) + add;
    }
};
__device__ __forceinline__ PosSrc pos_src(const uint8_t *blk, int W, int r, uint32_t flags) {
    PosSrc s;
    if (flags & RBF_AFFINE) {
        s.p = reinterpret_cast<const uint16_t *>(blk + rbm_base_off(W));
        s.stride = 1u;
        s.add = (uint32_t)r;
    } else {
        s.p = reinterpret_cast<const uint16_t *>(blk + rbm_idx_off(W, false)) + r;
        s.stride = 16u;
        s.add = 0u;
    }
    return s;
}

// Class-group loops of a mixed row block (FP32, FP16, FP8 classes, each
// plane stored in its class type): sumf = fmaf((float)x, v, sumf) plane by
// plane from plane k on. UNSC: every scale is 1.
template <bool UNSC, typename XT>
__device__ __forceinline__ float low_groups(const uint8_t *vals, int k, int n32, int n16, int n8, int r,
                                            const int8_t *sexp, const XT *xs, const PosSrc &pos, float sumf) {
    const float *v32 = reinterpret_cast<const float *>(vals) + r;
#pragma unroll 4
    for (int j = 0; j < n32; ++j) sumf = __fmaf_rn(to_f32(xs[pos(k + j)]), v32[j * 16], sumf);
    k += n32;
    const __half *h = reinterpret_cast<const __half *>(vals + 64u * n32) + r;
#pragma unroll 4
    for (int j = 0; j < n16; ++j) {
        const float v = __half2float(h[j * 16]);
        sumf = __fmaf_rn(to_f32(xs[pos(k + j)]), UNSC ? v : v * exp2_int(sexp[k + j]), sumf);
    }
    k += n16;
    const uint8_t *b8 = vals + 64u * n32 + 32u * n16 + r;
    for (int j = 0; j < n8; ++j) {
        const float v = fp8_to_float(b8[j * 16]);
        sumf = __fmaf_rn(to_f32(xs[pos(k + j)]), UNSC ? v : v * exp2_int(sexp[k + j]), sumf);
    }
    return sumf;
}

// Two staged row blocks, each with one FP32-class and N16 FP16-class planes
// (all stored in their class type), fully unrolled so that a lane issues
// all position, x and value loads of both rows before the first FMA: the row
// sums of mixed_row, in the same order. UNSC: every scale is 1.
template <int N16, bool UNSC>
__device__ __forceinline__ void rows2_fixed(const uint8_t *b1, const uint8_t *b2, uint32_t f1, uint32_t f2, int r,
                                            const float *xs, float &s1, float &s2) {
    constexpr int NW = 1 + N16;
    const PosSrc p1 = pos_src(b1, NW, r, f1), p2 = pos_src(b2, NW, r, f2);
    const uint8_t *v1 = b1 + rbm_vals_off(NW, false, (f1 & RBF_AFFINE) != 0);
    const uint8_t *v2 = b2 + rbm_vals_off(NW, false, (f2 & RBF_AFFINE) != 0);
    const int8_t *e1 = reinterpret_cast<const int8_t *>(b1 + rbm_sexp_off());
    const int8_t *e2 = reinterpret_cast<const int8_t *>(b2 + rbm_sexp_off());
    float x1[NW], x2[NW], w1[NW], w2[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        x1[k] = xs[p1(k)];
        x2[k] = xs[p2(k)];
    }
    w1[0] = reinterpret_cast<const float *>(v1)[r];
    w2[0] = reinterpret_cast<const float *>(v2)[r];
#pragma unroll
    for (int j = 0; j < N16; ++j) {
        const float h1 = __half2float(reinterpret_cast<const __half *>(v1 + 64u)[j * 16 + r]);
        const float h2 = __half2float(reinterpret_cast<const __half *>(v2 + 64u)[j * 16 + r]);
        w1[1 + j] = UNSC ? h1 : h1 * exp2_int(e1[1 + j]);
        w2[1 + j] = UNSC ? h2 : h2 * exp2_int(e2[1 + j]);
    }
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        s1 = __fmaf_rn(x1[k], w1[k], s1);
        s2 = __fmaf_rn(x2[k], w2[k], s2);
    }
}

// Row r of a mixed-layout row block (planes grouped by entry class, see
// tiles.h). FP64-class entries: sum = 0, sum += x*v, acc += sum at each tile
// start, exactly blockspmv_cpu's order. The FP32-, FP16- and FP8-class
// entries: one FP32 accumulator, sumf = fmaf((float)x, v, sumf), group by
// group in plane order. Returns acc + (double)sumf. Staged rows loop over all
// planes (padding entries index the zero slot with value 0); gather rows
// skip the x load of padding entries (PAD flag, value 0).
template <bool GATHER, typename XT>
__device__ __forceinline__ double mixed_row(const uint8_t *blk, int W, int r, const XT *xs,
                                            const XT *__restrict__ xg) {
    const uint32_t cnt = *reinterpret_cast<const uint32_t *>(blk);
    const uint32_t flags = blk[4];
    const int n64 = cnt & 0xffu, n32 = (cnt >> 8) & 0xffu, n16 = (cnt >> 16) & 0xffu, n8 = cnt >> 24;
    const int8_t *sexp = reinterpret_cast<const int8_t *>(blk + rbm_sexp_off());
    const bool aff = !GATHER && (flags & RBF_AFFINE);
    const uint8_t *idxb = blk + rbm_idx_off(W, aff);
    const uint8_t *vals = blk + rbm_vals_off(W, GATHER, aff);
    const uint16_t *base = reinterpret_cast<const uint16_t *>(blk + rbm_base_off(W));
    auto ld_x = [&](int k, uint32_t &id) -> XT {
        if constexpr (GATHER) {
            id = reinterpret_cast<const uint32_t *>(idxb)[k * 16 + r];
            return (id & IDX32_PAD) ? XT(0) : __ldcg(xg + (id & IDX32_POS));
        } else {
            if (aff) {
                id = (uint32_t)base[k] + (uint32_t)r;
                return xs[id];
            }
            id = reinterpret_cast<const uint16_t *>(idxb)[k * 16 + r];
            return xs[id & IDX16_POS];
        }
    };
    double acc = 0.0;
    uint32_t voff = 0;
    int k = 0;
    if (n64 > 0) {
        const double *v = reinterpret_cast<const double *>(vals) + r;
        double sum = 0.0;
        for (; k < n64; ++k) {
            uint32_t id;
            const double x = (double)ld_x(k, id);
            if (id & (GATHER ? IDX32_START : IDX16_START)) {
                acc = dadd(acc, sum);
                sum = 0.0;
            }
            sum = dadd(sum, dmul(x, v[k * 16]));
        }
        acc = dadd(acc, sum);
        voff = 128u * n64;
    }
    float sumf = 0.0f;
    if (flags & RBF_FAST) {
        if constexpr (GATHER) {
            // gather rows: x from L2; padding entries (PAD) read as 0
            const float *v32 = reinterpret_cast<const float *>(vals + voff) + r;
            for (int j = 0; j < n32; ++j) {
                uint32_t id;
                const XT x = ld_x(k + j, id);
                sumf = __fmaf_rn(to_f32(x), v32[j * 16], sumf);
            }
            k += n32;
            voff += 64u * n32;
            const __half *h = reinterpret_cast<const __half *>(vals + voff) + r;
            for (int j = 0; j < n16; ++j) {
                uint32_t id;
                const XT x = ld_x(k + j, id);
                sumf = __fmaf_rn(to_f32(x), __half2float(h[j * 16]) * exp2_int(sexp[k + j]), sumf);
            }
            k += n16;
            voff += 32u * n16;
            for (int j = 0; j < n8; ++j) {
                uint32_t id;
                const XT x = ld_x(k + j, id);
                sumf = __fmaf_rn(to_f32(x), fp8_to_float(vals[voff + j * 16 + r]) * exp2_int(sexp[k + j]), sumf);
            }
        } else {
            const PosSrc pos = pos_src(blk, W, r, flags);
            sumf = (flags & RBF_UNSCALED) ? low_groups<true>(vals + voff, k, n32, n16, n8, r, sexp, xs, pos, sumf)
                                          : low_groups<false>(vals + voff, k, n32, n16, n8, r, sexp, xs, pos, sumf);
        }
    } else {
        // some FP16 / FP8 class plane stored wider: decode plane by plane
        const uint64_t pbits = *reinterpret_cast<const uint64_t *>(blk + 8);
        for (; k < W; ++k) {
            const uint32_t pr = (uint32_t)(pbits >> (2 * k)) & 3u;
            uint32_t id;
            const XT x = ld_x(k, id);
            const float sc = exp2_int(sexp[k]);
            float v;
            if (pr == MF_PREC_FP32) v = reinterpret_cast<const float *>(vals + voff)[r];
            else if (pr == MF_PREC_FP16) v = __half2float(reinterpret_cast<const __half *>(vals + voff)[r]) * sc;
            else v = fp8_to_float(vals[voff + r]) * sc;
            sumf = __fmaf_rn(to_f32(x), v, sumf);
            voff += 128u >> pr;
        }
    }
    return dadd(acc, (double)sumf);
}

// Sum of row r of row block j of a staged / gather slab (row-sliced planes).
// FP64 layouts: sum = 0, sum += x*v in order, acc += sum at each tile start,
// exactly blockspmv_cpu's order. Mixed layouts: mixed_row.
// GB > 1: FP64 gather rows issue GB x loads from L2 before using the first
// (more gathers in flight, more registers: for kernels with registers to
// spare; the solver kernels with 128 live registers take GB = 1).
template <int KIND, int GB, typename XT>
__device__ __forceinline__ double slab_row(const uint8_t *st, const SlabHeader &h, int j, int r, const XT *xstage,
                                           const XT *__restrict__ xg) {
    const RbDir d = reinterpret_cast<const RbDir *>(st + slab_rbdir_off())[j];
    const uint8_t *blk = st + d.off;
    const int W = (int)(d.W & 0xffffu);
    const int len = blk[r];
    const bool gather = h.mode == SLAB_GATHER;
    double acc = 0.0, sum = 0.0;
    if (KIND == LAYOUT_FP64) {
        const double *vals = reinterpret_cast<const double *>(blk + rb_vals_off(W, gather));
        if (!gather) {
            // all W planes: padding entries add x(zero slot) * 0 = +0 to a sum
            // that is never -0, which leaves it unchanged; the trip count is
            // the same for the 16 lanes of the row block
            const uint16_t *idx = reinterpret_cast<const uint16_t *>(blk + rb_idx_off());
#pragma unroll 4
            for (int k = 0; k < W; ++k) {
                const uint32_t id = idx[k * 16 + r];
                const double v = vals[k * 16 + r];
                const XT x = xstage[id & IDX16_POS];
                if (id & IDX16_START) {
                    acc = dadd(acc, sum);
                    sum = 0.0;
                }
                sum = dadd(sum, dmul(x, v));
            }
        } else if (GB == 1) {
            const uint32_t *idx = reinterpret_cast<const uint32_t *>(blk + rb_idx_off());
#pragma unroll 4
            for (int k = 0; k < len; ++k) {
                const uint32_t id = idx[k * 16 + r];
                const double v = vals[k * 16 + r];
                const XT x = __ldcg(xg + (id & IDX32_POS));
                if (id & IDX32_START) {
                    acc = dadd(acc, sum);
                    sum = 0.0;
                }
                sum = dadd(sum, dmul(x, v));
            }
        } else {
            // x comes from L2 entry by entry: issue GB loads before the
            // first is used so that a lane keeps GB gathers in flight
            const uint32_t *idx = reinterpret_cast<const uint32_t *>(blk + rb_idx_off());
            for (int k0 = 0; k0 < len; k0 += GB) {
                uint32_t id[GB];
                double v[GB];
                XT x[GB];
#pragma unroll
                for (int u = 0; u < GB; ++u) {
                    const bool on = k0 + u < len;
                    id[u] = on ? idx[(k0 + u) * 16 + r] : 0u;
                    v[u] = on ? vals[(k0 + u) * 16 + r] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < GB; ++u) x[u] = k0 + u < len ? __ldcg(xg + (id[u] & IDX32_POS)) : XT(0);
#pragma unroll
                for (int u = 0; u < GB; ++u) {
                    if (k0 + u < len) {
                        if (id[u] & IDX32_START) {
                            acc = dadd(acc, sum);
                            sum = 0.0;
                        }
                        sum = dadd(sum, dmul(x[u], v[u]));
                    }
                }
            }
        }
        return dadd(acc, sum);
    }
    return gather ? mixed_row<true>(blk, W, r, xstage, xg) : mixed_row<false>(blk, W, r, xstage, xg);
}

// Two staged row blocks of one half-warp without FP64-class planes, all
// planes stored in their class type, with equal class groups and scale
// flags, interleaved in one loop: two independent load and accumulate chains
// per lane, each in the order of mixed_row (identical results). Returns false
// (nothing computed) when the pair does not qualify.
template <bool UNSC>
__device__ __forceinline__ void pair_groups(const uint8_t *b1, const uint8_t *b2, int W, uint32_t f1, uint32_t f2,
                                            int n32, int n16, int n8, int r, const float *xs, float &s1, float &s2) {
    const PosSrc p1 = pos_src(b1, W, r, f1), p2 = pos_src(b2, W, r, f2);
    const int8_t *e1 = reinterpret_cast<const int8_t *>(b1 + rbm_sexp_off());
    const int8_t *e2 = reinterpret_cast<const int8_t *>(b2 + rbm_sexp_off());
    const uint8_t *v1 = b1 + rbm_vals_off(W, false, f1 & RBF_AFFINE), *v2 = b2 + rbm_vals_off(W, false, f2 & RBF_AFFINE);
    {
        const float *w1 = reinterpret_cast<const float *>(v1) + r, *w2 = reinterpret_cast<const float *>(v2) + r;
#pragma unroll 2
        for (int k = 0; k < n32; ++k) {
            s1 = __fmaf_rn(xs[p1(k)], w1[k * 16], s1);
            s2 = __fmaf_rn(xs[p2(k)], w2[k * 16], s2);
        }
    }
    const int k0 = n32;
    const __half *h1 = reinterpret_cast<const __half *>(v1 + 64u * n32) + r;
    const __half *h2 = reinterpret_cast<const __half *>(v2 + 64u * n32) + r;
#pragma unroll 2
    for (int j = 0; j < n16; ++j) {
        const int k = k0 + j;
        const float a1 = __half2float(h1[j * 16]), a2 = __half2float(h2[j * 16]);
        s1 = __fmaf_rn(xs[p1(k)], UNSC ? a1 : a1 * exp2_int(e1[k]), s1);
        s2 = __fmaf_rn(xs[p2(k)], UNSC ? a2 : a2 * exp2_int(e2[k]), s2);
    }
    const int k1 = n32 + n16;
    const uint32_t o8 = 64u * n32 + 32u * n16 + r;
    for (int j = 0; j < n8; ++j) {
        const int k = k1 + j;
        const float a1 = fp8_to_float(v1[o8 + j * 16]), a2 = fp8_to_float(v2[o8 + j * 16]);
        s1 = __fmaf_rn(xs[p1(k)], UNSC ? a1 : a1 * exp2_int(e1[k]), s1);
        s2 = __fmaf_rn(xs[p2(k)], UNSC ? a2 : a2 * exp2_int(e2[k]), s2);
    }
}

__device__ __forceinline__ bool pair_mixed(const uint8_t *st, int j1, int j2, int r, const float *xs, double &a1,
                                           double &a2) {
    const RbDir *dir = reinterpret_cast<const RbDir *>(st + slab_rbdir_off());
    const RbDir d1 = dir[j1], d2 = dir[j2];
    const int W = (int)(d1.W & 0xffffu);
    const uint8_t *b1 = st + d1.off, *b2 = st + d2.off;
    const uint32_t c1 = *reinterpret_cast<const uint32_t *>(b1), c2 = *reinterpret_cast<const uint32_t *>(b2);
    const uint32_t f1 = b1[4], f2 = b2[4];
    if (c1 != c2 || (c1 & 0xffu) != 0u || ((f1 ^ f2) & RBF_UNSCALED) || !(f1 & f2 & RBF_FAST)) return false;
    const int n32 = (c1 >> 8) & 0xffu, n16 = (c1 >> 16) & 0xffu, n8 = c1 >> 24;
    float s1 = 0.0f, s2 = 0.0f;
    if (n8 == 0 && n32 == 1 && n16 >= 3 && n16 <= 6) {
        // the 3D 7-point / 2D 5-point stencil shapes and their boundary
        // faces (a plane of the domain lacks one neighbour: the first and
        // last planes of the 3D stencil have 5), fully unrolled
        const bool u = (f1 & RBF_UNSCALED) != 0;
        switch (n16) {
            case 6:
                if (u) rows2_fixed<6, true>(b1, b2, f1, f2, r, xs, s1, s2);
                else rows2_fixed<6, false>(b1, b2, f1, f2, r, xs, s1, s2);
                break;
            case 5:
                if (u) rows2_fixed<5, true>(b1, b2, f1, f2, r, xs, s1, s2);
                else rows2_fixed<5, false>(b1, b2, f1, f2, r, xs, s1, s2);
                break;
            case 4:
                if (u) rows2_fixed<4, true>(b1, b2, f1, f2, r, xs, s1, s2);
                else rows2_fixed<4, false>(b1, b2, f1, f2, r, xs, s1, s2);
                break;
            default:
                if (u) rows2_fixed<3, true>(b1, b2, f1, f2, r, xs, s1, s2);
                else rows2_fixed<3, false>(b1, b2, f1, f2, r, xs, s1, s2);
                break;
        }
        a1 = (double)s1;
        a2 = (double)s2;
        return true;
    }
    if (f1 & RBF_UNSCALED) pair_groups<true>(b1, b2, W, f1, f2, n32, n16, n8, r, xs, s1, s2);
    else pair_groups<false>(b1, b2, W, f1, f2, n32, n16, n8, r, xs, s1, s2);
    a1 = (double)s1;
    a2 = (double)s2;
    return true;
}

// Global tile arrays (the oversize path) and the source of one SpMV.
struct SpmvSrc {
    const uint8_t *slabs;
    const uint8_t *head;  // STAGES issue records (shared memory)
    int ns, kind, site;
    int resident_ok;      // slabs may stay in the ring between SpMVs (site = layout index)
    int x32;              // x staged in FP32 (the input vector is FP32)
    GTiles gt;
};
struct PipeCfg {
    int stage_stride, slab_area;
    uint64_t limit_ns;
    uint32_t *sync;
    int prefetch;  // L2 bulk prefetch of the slab 2*STAGES ahead (off by default: it slowed the ring)
};
__device__ __forceinline__ GTiles gtiles_of(const KParams &P) {
    return GTiles{P.tile_ptr, P.tile_col, P.tile_off, P.csrptr_off, P.ptr, P.val, P.col, P.tilem, P.rowA};
}

// Row sum of an oversize row block straight from the global tile arrays.
__device__ double global_row(const GTiles &P, int rb, int r, const double *__restrict__ xg) {
    const int rl = rb == P.tilem - 1 ? P.rowA - (P.tilem - 1) * 16 : 16;
    if (r >= rl) return 0.0;
    double acc = 0.0;
    for (int t = P.tile_ptr[rb]; t < P.tile_ptr[rb + 1]; ++t) {
        const int xo = P.tile_col[t] * 16;
        const int vo = P.tile_off[t];
        const int nk = P.tile_off[t + 1] - vo;
        const int cc = P.csrptr_off[t];
        const int s = P.ptr[cc + r];
        const int e = r + 1 < rl ? P.ptr[cc + r + 1] : nk;
        double sum = 0.0;
        for (int q = s; q < e; ++q) sum = dadd(sum, dmul(__ldcg(xg + xo + P.col[vo + q]), P.val[vo + q]));
        acc = dadd(acc, sum);
    }
    return acc;
}

// Tiled SpMV of this CTA's row range with layout `lay` and input vector xv.
// Warp PRODUCER_WARP (one lane) streams the CTA's slabs into the STAGES-deep
// ring: it waits until the consumers released a stage, then issues the x
// runs and the slab of the next slab with 1D bulk copies. The NWARPS
// consumer warps wait for a stage's full barrier, compute their row blocks
// (one half-warp per row block, one lane per row) and release the stage.
// For every row < rowA: v = epi.pre(row) (any type) is loaded before the row's
// entries, then epi(row, acc, v) runs with the row sum. Returns false on
// abort.
template <bool MIXED, class Epi, int GB = 1>
__device__ bool cta_spmv_src(const SpmvSrc &L, const PipeCfg &C, const void *xv, Smem &S, uint8_t *dyn,
                             Pipe &pp, Epi &epi) {
    const int ns = L.ns;
    const int stride = C.stage_stride;
    const int xoff = x_off_of(C.slab_area, L.x32 != 0);  // the layout's x window in a stage
    const int tid = threadIdx.x;
    const int w = tid >> 5, lane = tid & 31;
    const int half = lane >> 4, r = lane & 15;
    if (w == PRODUCER_WARP) {
        if (lane == 0) {
            const uint64_t pm = policy_evict_first(), pv = policy_evict_last();
            fence_proxy_async_global();
            for (int i = 0; i < ns; ++i) {
                const int k = i % STAGES;
                uint8_t *st = stage_ptr(dyn, k, stride);
                if ((pp.filled >> k) & 1u) {
                    if (!wait_bar(&S.empty[k], (pp.eph >> k) & 1u, C.limit_ns)) {
                        set_error_w(C.sync, (uint32_t)MF_ERR_TIMEOUT, 110 + L.site);
                        S.abort = 1;
                        break;
                    }
                    pp.eph ^= 1u << k;
                }
                pp.filled |= 1u << k;
                uint32_t off16, bytes, xbytes;
                int nruns;
                const XRun *runs;
                if (i < STAGES) {
                    const uint32_t *rec = reinterpret_cast<const uint32_t *>(L.head + i * ISSUE_REC);
                    off16 = rec[0];
                    bytes = rec[1];
                    xbytes = rec[2];
                    nruns = (int)rec[3];
                    runs = reinterpret_cast<const XRun *>(rec + 4);
                } else {
                    // the slab consumed from this stage carries the record of slab i
                    const SlabHeader *h = reinterpret_cast<const SlabHeader *>(st);
                    off16 = h->next_off16;
                    bytes = h->next_bytes;
                    xbytes = h->next_xbytes;
                    nruns = h->next_nruns;
                    runs = reinterpret_cast<const XRun *>(st + SLAB_HDR);
                    if (C.prefetch && h->pf_bytes) bulk_prefetch_l2(L.slabs + (size_t)h->pf_off16 * 16, h->pf_bytes);
                }
                fence_proxy_async_smem();
                // a CTA with at most STAGES slabs puts slab i in stage i on
                // every SpMV: when the stage still holds it (same layout,
                // nothing else written into the ring since), only its x
                // window is copied
                const bool keep = L.resident_ok && ns <= STAGES;
                if (keep && S.res_tag[k] == (uint8_t)(L.site + 1)) {
                    mbar_arrive_expect_tx(&S.full[k], xbytes);
                    const uint32_t segb = L.x32 ? 64u : 128u;
                    for (int q = 0; q < nruns; ++q) {
                        const XRun rr = runs[q];
                        bulk_g2s(st + xoff + (size_t)rr.slot0 * segb,
                                 static_cast<const uint8_t *>(xv) + (size_t)rr.seg0 * segb, (uint32_t)rr.nseg * segb,
                                 &S.full[k], pv);
                    }
                } else {
                    issue_slab(S, st, xoff, k, off16, bytes, xbytes, nruns, runs, L.slabs,
                               static_cast<const uint8_t *>(xv), L.x32 ? 64u : 128u, pm, pv);
                    S.res_tag[k] = keep ? (uint8_t)(L.site + 1) : (uint8_t)0;
                }
            }
        }
        __syncwarp();
    } else {
        // half-warp that takes the first row block of the slab: advancing it
        // by each slab's row-block count spreads slabs of few row blocks
        // (gather mode) over all half-warps, so that consecutive slabs are
        // computed at once instead of queueing on the first few warps
        int base = 0;
        for (int i = 0; i < ns; ++i) {
            const int k = i % STAGES;
            uint8_t *st = stage_ptr(dyn, k, stride);
            if (!wait_bar(&S.full[k], (pp.fph >> k) & 1u, C.limit_ns)) {
                set_error_w(C.sync, (uint32_t)MF_ERR_TIMEOUT, 100 + L.site);
                S.abort = 1;
                break;
            }
            pp.fph ^= 1u << k;
            const SlabHeader h = *reinterpret_cast<const SlabHeader *>(st);
            if (h.mode == SLAB_OVERSIZE) {
                if (w == 0 && half == 0) {
                    const int row = h.rb0 * 16 + r;
                    using PV = decltype(epi.pre(0));
                    const PV pv = row < L.gt.rowA ? epi.pre(row) : PV(0);
                    const double acc = global_row(L.gt, h.rb0, r, static_cast<const double *>(xv));
                    if (row < L.gt.rowA) epi(row, acc, pv);
                }
            } else {
                int j0 = 2 * w + half - base;
                if (j0 < 0) j0 += 2 * NWARPS;
                base = (base + h.nrb) % (2 * NWARPS);
                const double *xsg = reinterpret_cast<const double *>(st + xoff);
                using PV = decltype(epi.pre(0));
                // the pre-loaded value keeps its own type until the epilogue:
                // a conversion here would wait for the load before the row's
                // arithmetic instead of overlapping it
                auto pre_of = [&](int jj, int row, bool live) -> PV {
                    if constexpr (Epi::kUsesX) {
                        // the row's own x value from the stage (rows this CTA
                        // wrote just before load slowly from global memory);
                        // an FP64 value is not taken from an FP32 stage
                        const uint32_t ds = reinterpret_cast<const RbDir *>(st + slab_rbdir_off())[jj].W >> 16;
                        if (ds == 0u || !live || (L.x32 && sizeof(PV) == 8)) return live ? epi.pre(row) : PV(0);
                        if (L.x32) return PV(reinterpret_cast<const float *>(xsg)[(ds - 1u) * 16u + r]);
                        return PV(xsg[(ds - 1u) * 16u + r]);
                    } else {
                        return live ? epi.pre(row) : PV(0);
                    }
                };
                int jstart = j0;
                if (MIXED && L.kind == LAYOUT_LOW && h.mode == SLAB_STAGED) {
                    // row blocks j and j + 2 NWARPS of this half-warp computed
                    // together; a pair that does not qualify (or a lone last
                    // row block) goes to the loop below
                    const float *xs = reinterpret_cast<const float *>(st + xoff);
                    for (; jstart + 2 * NWARPS < h.nrb; jstart += 4 * NWARPS) {
                        const int j2 = jstart + 2 * NWARPS;
                        const int row1 = (h.rb0 + jstart) * 16 + r, row2 = (h.rb0 + j2) * 16 + r;
                        const bool live1 = row1 < L.gt.rowA, live2 = row2 < L.gt.rowA;
                        const PV pv1 = pre_of(jstart, row1, live1), pv2 = pre_of(j2, row2, live2);
                        double a1, a2;
                        if (!pair_mixed(st, jstart, j2, r, xs, a1, a2)) {
                            a1 = slab_row<LAYOUT_LOW, GB>(st, h, jstart, r, xs, static_cast<const float *>(xv));
                            a2 = slab_row<LAYOUT_LOW, GB>(st, h, j2, r, xs, static_cast<const float *>(xv));
                        }
                        if (live1) epi(row1, a1, pv1);
                        if (live2) epi(row2, a2, pv2);
                    }
                }
                for (int j = jstart; j < h.nrb; j += 2 * NWARPS) {
                    const int row = (h.rb0 + j) * 16 + r;
                    const bool live = row < L.gt.rowA;
                    const PV pv = pre_of(j, row, live);
                    const double *xg = static_cast<const double *>(xv);
                    double acc;
                    if (!MIXED || L.kind == LAYOUT_FP64) acc = slab_row<LAYOUT_FP64, GB>(st, h, j, r, xsg, xg);
                    else if (L.kind == LAYOUT_LOW)  // always FP32 x
                        acc = slab_row<LAYOUT_LOW, GB>(st, h, j, r, reinterpret_cast<const float *>(xsg),
                                                       static_cast<const float *>(xv));
                    else acc = slab_row<LAYOUT_ANY, GB>(st, h, j, r, xsg, xg);
                    if (live) epi(row, acc, pv);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&S.empty[k]);
        }
    }
    __syncthreads();
    return S.abort == 0;
}


// Grid-kernel form: layout `lay` of the kernel parameters, this CTA's slabs.
// xv: FP64 vector, or FP32 when the layout stages x in FP32.
template <bool MIXED, class Epi, int GB = 1>
__device__ bool cta_spmv(const KParams &P, int lay, const void *xv, Smem &S, uint8_t *dyn, Pipe &pp, Epi &epi) {
    SpmvSrc L;
    L.slabs = P.lay[lay].slabs;
    L.head = &S.head[lay][0][0];
    L.ns = S.slab1[lay] - S.slab0[lay];
    L.kind = P.lay[lay].kind;
    L.x32 = P.lay[lay].x32;
    L.site = lay;
    L.resident_ok = 1;
    L.gt = gtiles_of(P);
    const PipeCfg C{P.stage_stride, P.slab_area, P.limit_ns, P.sync, P.prefetch};
    return cta_spmv_src<MIXED, Epi, GB>(L, C, xv, S, dyn, pp, epi);
}

// Block reduction of NV partials in a fixed order, then the grid-wide sum.
// A group of G CTAs that synchronize with each other (the whole grid for the
// single-system kernels, a slice of it for the batched one).
struct Ctx {
    uint32_t *sync;
    double *partial;
    int G, rank;
    uint64_t limit_ns;
};

template <int NV>
__device__ bool group_sum(const Ctx &X, Smem &S, const double (&v)[NV], double (&out)[NV], uint32_t &phase) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    double t[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        t[k] = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) S.red[w][k] = t[k];
    __syncthreads();
    const int G = X.G;
    const int slot = phase & 1;
    if (tid == 0) {
        double p[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            p[k] = 0.0;
            for (int q = 0; q <= NWARPS; ++q) p[k] += S.red[q][k];
            X.partial[((size_t)slot * G + X.rank) * 4 + k] = p[k];
        }
        red_release_add(X.sync + SYNC_ARRIVE, 1u);
        const uint32_t target = (phase + 1) * (uint32_t)G;
        if (ld_acquire(X.sync + SYNC_ARRIVE) < target) {
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(X.sync + SYNC_ARRIVE) >= target) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(X.sync + SYNC_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > X.limit_ns) {
                        set_error_w(X.sync, (uint32_t)MF_ERR_TIMEOUT, 10);
                        S.abort = 1;
                        break;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (S.abort) return false;
    if (w == 0) {
        double a[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) a[k] = 0.0;
        for (int c = lane; c < G; c += 32)
#pragma unroll
            for (int k = 0; k < NV; ++k) a[k] += __ldcg(&X.partial[((size_t)slot * G + c) * 4 + k]);
#pragma unroll
        for (int k = 0; k < NV; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < NV; ++k) S.bres[k] = a[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = S.bres[k];
    ++phase;
    return true;
}

__device__ __forceinline__ Ctx ctx_of(const KParams &P) {
    return Ctx{P.sync, P.partial, (int)gridDim.x, (int)blockIdx.x, P.limit_ns};
}
template <int NV>
__device__ bool grid_sum(const KParams &P, Smem &S, const double (&v)[NV], double (&out)[NV], uint32_t &phase) {
    return group_sum<NV>(ctx_of(P), S, v, out, phase);
}

// Publish this CTA's rows of the halo vectors under epoch `ep`.
__device__ void publish_x(const Ctx &X, uint32_t ep) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        fence_proxy_async_global();
        st_release(X.sync + SYNC_FLAGS + X.rank * FLAG_STRIDE, ep);
    }
}
__device__ void publish(const KParams &P, uint32_t ep) { publish_x(ctx_of(P), ep); }

// Wait until the group's CTAs lo..hi (whose rows this CTA reads) have
// published epoch `ep`.
__device__ bool wait_deps_x(const Ctx &X, Smem &S, int lo, int hi, uint32_t ep) {
    if (threadIdx.x < 32) {
        for (int c = lo + (int)threadIdx.x; c <= hi; c += 32) {
            const uint32_t *f = X.sync + SYNC_FLAGS + c * FLAG_STRIDE;
            if (ld_acquire(f) >= ep) continue;
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(f) >= ep) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(X.sync + SYNC_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > X.limit_ns) {
                        set_error_w(X.sync, (uint32_t)MF_ERR_TIMEOUT, 20);
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
__device__ bool wait_deps(const KParams &P, Smem &S, int lay, uint32_t ep) {
    return wait_deps_x(ctx_of(P), S, P.lay[lay].cta_dep[2 * blockIdx.x], P.lay[lay].cta_dep[2 * blockIdx.x + 1], ep);
}

// The zero slot of every stage (XZERO_OFF): written at set-up, and again
// after a vector pass whose bulk copies went through the ring (the caller
// has a barrier between the pass's last reads of the ring and this).
__device__ __forceinline__ void zero_slots(uint8_t *dyn, int stage_stride, int slab_area) {
    if (threadIdx.x < STAGES)
        *reinterpret_cast<uint4 *>(dyn + (size_t)threadIdx.x * stage_stride + slab_area + XZERO_OFF) =
            make_uint4(0u, 0u, 0u, 0u);
}

__device__ void kernel_setup(const KParams &P, Smem &S, int nlay) {
    extern __shared__ __align__(128) uint8_t dyn[];
    const int tid = threadIdx.x;
    zero_slots(dyn, P.stage_stride, P.slab_area);
    if (tid == 0) {
        for (int k = 0; k < STAGES; ++k) {
            mbar_init(&S.full[k], 1);
            mbar_init(&S.empty[k], NWARPS);
        }
        mbar_init(&S.upd, 1);
        mbar_fence_init();
        S.abort = 0;
        for (int k = 0; k < STAGES; ++k) S.res_tag[k] = 0;
    }
    for (int l = 0; l < nlay; ++l) {
        const uint8_t *src = P.lay[l].head + (size_t)blockIdx.x * STAGES * ISSUE_REC;
        for (int i = tid; i < STAGES * ISSUE_REC; i += blockDim.x) (&S.head[l][0][0])[i] = src[i];
        if (tid == 0) {
            S.slab0[l] = P.lay[l].cta_slab[blockIdx.x];
            S.slab1[l] = P.lay[l].cta_slab[blockIdx.x + 1];
        }
    }
    __syncthreads();
}

// Vector passes run over the CTA's own row blocks [lo, hi) (16-row aligned,
// zero padded past rowA) in pairs of rows with 16-byte loads, VB pairs per
// thread per batch so that all loads of a batch are in flight together.
#define MF_PAIRS(VB, lo, hi, ...)                                                     \
    for (int _b = ((lo) >> 1) + threadIdx.x; _b < ((hi) >> 1); _b += NTHREADS * (VB)) { \
        constexpr int _vb = (VB);                                                     \
        __VA_ARGS__                                                                   \
    }
#define MF_FOR_VB for (int u = 0; u < _vb; ++u)
#define MF_PI(u) (_b + (u) * NTHREADS)
#define MF_LIVE(u, hi) (MF_PI(u) < ((hi) >> 1))

// ------------------------------------------------------------------ SpMV
struct EpiStore {
    static constexpr bool kUsesX = false;
    double *y;
    __device__ double pre(int) const { return 0.0; }
    __device__ void operator()(int row, double acc, double) const { y[row] = acc; }
};

// Launched with programmatic stream serialization: the next SpMV in the
// stream may be scheduled as soon as this one starts (it occupies an SM only
// once this grid's CTA there has exited), does its set-up (barriers, issue
// records of the constant layout), and waits for this grid to complete
// before it reads x or writes y. Without that launch attribute both
// instructions do nothing.
template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1) k_spmv(KParams P, const void *x, double *y, int lay, int reps) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    asm volatile("griddepcontrol.launch_dependents;");
    kernel_setup(P, S, lay + 1);
    asm volatile("griddepcontrol.wait;" ::: "memory");
    Pipe pp;
    EpiStore epi{y};
    for (int it = 0; it < reps; ++it) {
        if (!cta_spmv<MIXED, EpiStore, 8>(P, lay, x, S, dyn, pp, epi)) return;
    }
}

// -------------------------------------------------------------------- CG
// The solver's vectors are read and written with an L2 evict_last policy
// so they stay resident in L2 while the matrix streams with evict_first.
struct EpiResidual {  // r = b - A x, rr += r*r
    static constexpr bool kUsesX = false;
    const double *b;
    double *r;
    double rr;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(b + row, pol); }
    __device__ void operator()(int row, double acc, double bv) {
        const double v = bv - acc;
        st_hint(r + row, v, pol);
        rr += v * v;
    }
};
struct EpiResidual32 {  // r = b - A x and its FP32 copy, rr += r*r
    static constexpr bool kUsesX = false;
    const double *b;
    double *r;
    float *r32;
    double rr;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(b + row, pol); }
    __device__ void operator()(int row, double acc, double bv) {
        const double v = bv - acc;
        st_hint(r + row, v, pol);
        stf_hint(r32 + row, __double2float_rn(v), pol);
        rr += v * v;
    }
};
struct EpiQ {  // q = A d, dq += d*q
    static constexpr bool kUsesX = true;  // d is the SpMV input
    const double *d;
    double *q;
    double dq;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(d + row, pol); }
    __device__ void operator()(int row, double acc, double dv) {
        st_hint(q + row, acc, pol);
        dq += dv * acc;
    }
};

// Phase trace: CTA 0 thread 0 writes %globaltimer at slot s of iteration it.
#define MF_TRACE(it, s)                                                                   \
    do {                                                                                  \
        if (P.trace && blockIdx.x == 0 && threadIdx.x == 0 && (it) < P.trace_iters)       \
            P.trace[(size_t)(it) * 8 + (s)] = globaltimer();                              \
    } while (0)

template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1) k_cg(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, P.nlay);
    const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0;
    const uint64_t vpol = policy_evict_last();
    const int lay64 = 0;
    int lay = P.start_layout;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int vlo = rb_lo * 16, vhi = rb_hi * 16;  // own rows, zero padded past rowA
    double *x = P.x, *r = P.r, *d = P.d, *q = P.q;
    float *d32 = MIXED ? reinterpret_cast<float *>(P.t) : nullptr;  // FP32 d for FP32-x layouts
    const double *b = P.b;
    if (P.inject_wait) {
        // test hook: a dependency epoch no CTA ever publishes; the bounded
        // wait must end the solve with MF_ERR_TIMEOUT
        if (!wait_deps(P, S, 0, 0xffffffffu)) return;
    }
    // r = b - A x0, d = r; (rr, bb)
    EpiResidual er{b, r, 0.0, vpol};
    if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, er)) return;
    __syncthreads();
    double bbp = 0.0;
    MF_PAIRS(4, vlo, vhi, {
        double2 rv[_vb], bv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
        }
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            st2_hint(d + 2 * MF_PI(u), rv[u], vpol);
            if (MIXED)
                stf2_hint(d32 + 2 * MF_PI(u), make_float2(__double2float_rn(rv[u].x), __double2float_rn(rv[u].y)),
                          vpol);
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
        }
    })
    double v2[2] = {er.rr, bbp}, o2[2];
    if (!grid_sum<2>(P, S, v2, o2, phase)) return;
    double rr = o2[0];
    const double bb = o2[1];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK, repl = 0, switches = 0;
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    // With true_check, a recursive residual under tol is confirmed with the
    // FP64 true residual b - A x before the solve stops (mixed layouts).
    bool pending = false;
    int it_lay[KMAX_LAYOUTS] = {0, 0, 0, 0};
    double rr_best = rr;
    int fellback = 0;
    while (it < maxit && (fixed || rel > tol || pending)) {
        // true-residual replacement r = b - A x (FP64 layout): periodic, or
        // to confirm convergence
        if (pending || (P.replace_every > 0 && it > 0 && it % P.replace_every == 0)) {
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiResidual e2{b, r, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, e2)) return;
            double v1[1] = {e2.rr}, o1[1];
            if (!grid_sum<1>(P, S, v1, o1, phase)) return;
            const double rr_rec = rr;
            rr = o1[0];
            ++repl;
            if (pending) {
                pending = false;
                rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
                if (rel <= tol) break;
            }
            // a true residual norm more than twice the recursive one (a
            // low-precision operator's iterate drifted from A's): restart
            // the directions from the true residual, d = r
            if (rr > 4.0 * rr_rec) {
                MF_PAIRS(4, vlo, vhi, {
                    double2 rv[_vb];
#pragma unroll
                    MF_FOR_VB if (MF_LIVE(u, vhi)) rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
#pragma unroll
                    MF_FOR_VB if (MF_LIVE(u, vhi)) {
                        st2_hint(d + 2 * MF_PI(u), rv[u], vpol);
                        if (MIXED)
                            stf2_hint(d32 + 2 * MF_PI(u),
                                      make_float2(__double2float_rn(rv[u].x), __double2float_rn(rv[u].y)), vpol);
                    }
                })
                ++ep;
                publish(P, ep);
            }
            // a low-precision operator that lets the true residual grow
            // 100x above the best seen falls back to the FP64 layout
            if (MIXED && lay != lay64) {
                if (rr < rr_best) rr_best = rr;
                if (!(rr <= 1e4 * rr_best)) {
                    lay = lay64;
                    fellback = 1;
                }
            }
            // tighten the precision level as the true residual falls
            if (MIXED) {
                const double relt = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
                while (lay != lay64 && lay < P.nlay - 1 && relt < P.level_rel[lay]) {
                    ++lay;
                    ++switches;
                }
            }
        }
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, lay, ep)) return;
        MF_TRACE(it, 1);
        ++it_lay[lay];
        EpiQ eq{d, q, 0.0, vpol};
        bool ok;
        if (MIXED && lay != lay64) ok = cta_spmv<true>(P, lay, P.lay[lay].x32 ? (const void *)d32 : d, S, dyn, pp, eq);
        else ok = cta_spmv<false>(P, lay64, d, S, dyn, pp, eq);
        if (!ok) return;
        MF_TRACE(it, 2);
        double v1[1] = {eq.dq}, o1[1];
        if (!grid_sum<1>(P, S, v1, o1, phase)) return;
        MF_TRACE(it, 3);
        const double dq = o1[0];
        if (!(dq != 0.0) || !isfinite(dq)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rr / dq;
        double rrp = 0.0;
        MF_PAIRS(4, vlo, vhi, {
            double2 rv[_vb], qv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                qv[u] = ld2_hint(q + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 o;
                o.x = rv[u].x - alpha * qv[u].x;
                o.y = rv[u].y - alpha * qv[u].y;
                st2_hint(r + 2 * MF_PI(u), o, vpol);
                rrp += o.x * o.x + o.y * o.y;
            }
        })
        MF_TRACE(it, 4);
        double w1[1] = {rrp}, u1[1];
        if (!grid_sum<1>(P, S, w1, u1, phase)) return;
        MF_TRACE(it, 5);
        const double rrn = u1[0];
        ++it;
        rel = bnorm > 0 ? sqrt(rrn) / bnorm : 0.0;
        const double beta = rrn / rr;
        const bool done = !fixed && rel <= tol && !P.true_check;
        if (!fixed && rel <= tol && P.true_check) pending = true;
        MF_PAIRS(4, vlo, vhi, {
            double2 dv[_vb], xv[_vb], rv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                dv[u] = ld2_hint(d + 2 * MF_PI(u), vpol);
                xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 xo, dn;
                xo.x = xv[u].x + alpha * dv[u].x;
                xo.y = xv[u].y + alpha * dv[u].y;
                st2_hint(x + 2 * MF_PI(u), xo, vpol);
                if (!done) {
                    dn.x = rv[u].x + beta * dv[u].x;
                    dn.y = rv[u].y + beta * dv[u].y;
                    st2_hint(d + 2 * MF_PI(u), dn, vpol);
                    if (MIXED)
                        stf2_hint(d32 + 2 * MF_PI(u), make_float2(__double2float_rn(dn.x), __double2float_rn(dn.y)),
                                  vpol);
                }
            }
        })
        rr = rrn;
        ++ep;
        publish(P, ep);
        MF_TRACE(it - 1, 6);
        if (!isfinite(rrn)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
    }
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = repl;
        P.res->level_switches = switches;
        P.res->rr = rr;
        P.res->bb = bb;
        P.res->final_layout = lay;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = it_lay[l];
        P.res->pad = fellback;
    }
    (void)G;
}

// ----------------------------------------------- Jacobi-preconditioned CG
// PCG with M = diag(A) (KSPCG + PCJACOBI, the "jpcg" runs of the reference's
// PETSc comparison) on the FP64 layout, in one persistent kernel like k_cg:
//   z = M^-1 r;  d = z;  rz = r.z
//   q = A d;  alpha = rz / d.q;  x += alpha d;  r -= alpha q;  z = M^-1 r
//   beta = (r.z)_new / rz;  d = z + beta d
// M^-1 is applied on the fly from 1/a_ii (P.s, filled by the host); z is
// never stored. The stop test is the unpreconditioned ||r|| / ||b||, as for
// CG; r.z and r.r share one grid reduction.
__global__ void __launch_bounds__(NTHREADS, 1) k_pcg(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, 1);
    const int g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0;
    const uint64_t vpol = policy_evict_last();
    const int vlo = P.lay[0].cta_rb[g] * 16, vhi = P.lay[0].cta_rb[g + 1] * 16;
    double *x = P.x, *r = P.r, *d = P.d, *q = P.q;
    const double *minv = P.s, *b = P.b;
    // r = b - A x0;  d = z = M^-1 r
    EpiResidual er{b, r, 0.0, vpol};
    if (!cta_spmv<false>(P, 0, x, S, dyn, pp, er)) return;
    double rzp = 0.0, bbp = 0.0;
    MF_PAIRS(2, vlo, vhi, {
        double2 rv[_vb], bv[_vb], mv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
            mv[u] = ld2_hint(minv + 2 * MF_PI(u), vpol);
        }
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            double2 z;
            z.x = mv[u].x * rv[u].x;
            z.y = mv[u].y * rv[u].y;
            st2_hint(d + 2 * MF_PI(u), z, vpol);
            rzp += rv[u].x * z.x + rv[u].y * z.y;
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
        }
    })
    double v3[3] = {er.rr, rzp, bbp}, o3[3];
    if (!grid_sum<3>(P, S, v3, o3, phase)) return;
    double rr = o3[0], rz = o3[1];
    const double bb = o3[2];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK;
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    while (it < maxit && (fixed || rel > tol)) {
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, 0, ep)) return;
        MF_TRACE(it, 1);
        EpiQ eq{d, q, 0.0, vpol};
        if (!cta_spmv<false>(P, 0, d, S, dyn, pp, eq)) return;
        MF_TRACE(it, 2);
        double v1[1] = {eq.dq}, o1[1];
        if (!grid_sum<1>(P, S, v1, o1, phase)) return;
        MF_TRACE(it, 3);
        const double dq = o1[0];
        if (!(dq != 0.0) || !isfinite(dq)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rz / dq;
        double rzn = 0.0, rrn = 0.0;
        MF_PAIRS(2, vlo, vhi, {
            double2 rv[_vb], qv[_vb], mv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                qv[u] = ld2_hint(q + 2 * MF_PI(u), vpol);
                mv[u] = ld2_hint(minv + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 o;
                o.x = rv[u].x - alpha * qv[u].x;
                o.y = rv[u].y - alpha * qv[u].y;
                st2_hint(r + 2 * MF_PI(u), o, vpol);
                rzn += o.x * (mv[u].x * o.x) + o.y * (mv[u].y * o.y);
                rrn += o.x * o.x + o.y * o.y;
            }
        })
        MF_TRACE(it, 4);
        double w2[2] = {rzn, rrn}, u2[2];
        if (!grid_sum<2>(P, S, w2, u2, phase)) return;
        MF_TRACE(it, 5);
        rr = u2[1];
        ++it;
        rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        const double beta = u2[0] / rz;
        rz = u2[0];
        const bool done = !fixed && rel <= tol;
        MF_PAIRS(2, vlo, vhi, {
            double2 dv[_vb], xv[_vb], rv[_vb], mv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                dv[u] = ld2_hint(d + 2 * MF_PI(u), vpol);
                xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                if (!done) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    mv[u] = ld2_hint(minv + 2 * MF_PI(u), vpol);
                }
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 xo, dn;
                xo.x = xv[u].x + alpha * dv[u].x;
                xo.y = xv[u].y + alpha * dv[u].y;
                st2_hint(x + 2 * MF_PI(u), xo, vpol);
                if (!done) {
                    dn.x = mv[u].x * rv[u].x + beta * dv[u].x;
                    dn.y = mv[u].y * rv[u].y + beta * dv[u].y;
                    st2_hint(d + 2 * MF_PI(u), dn, vpol);
                }
            }
        })
        ++ep;
        publish(P, ep);
        MF_TRACE(it - 1, 6);
        if (!isfinite(rr)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
    }
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = 0;
        P.res->level_switches = 0;
        P.res->rr = rr;
        P.res->bb = bb;
        P.res->final_layout = 0;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = l == 0 ? it : 0;
        P.res->pad = 0;
    }
}

// 1/a_ii for the Jacobi preconditioner (rows with a zero diagonal and the
// padding rows keep 1 / 0 so that they pass r through / stay zero).
__global__ void k_jacobi_inv(int n, int npad, const double *diag, double *minv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x)
        minv[i] = i < n ? (diag[i] != 0.0 ? 1.0 / diag[i] : 1.0) : 0.0;
}

int launch_jacobi_inv(int n, int npad, const double *diag, double *minv, cudaStream_t s) {
    int blocks = (npad + 255) / 256;
    blocks = blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks);
    k_jacobi_inv<<<blocks, 256, 0, s>>>(n, npad, diag, minv);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

// ------------------------------------------------- CG, single reduction
// Chronopoulos-Gear form of CG for the mixed-precision layouts: one grid
// reduction and one fused vector pass per iteration. w = A r comes from the
// low-precision SpMV; the directions p and s = A p, and w, are stored in
// FP32; x and r (and the dots and scalars) stay FP64; r is replaced by the
// FP64 true residual b - A x every replace_every iterations and before the
// solve stops.
//   p = r + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;
//   w = A r;  gamma = r.r;  delta = w.r;
//   beta = gamma / gamma_old;  alpha = gamma / (delta + 2 beta r.s + beta^2 p.s)
// with r.s and p.s (the previous s and p) summed in the vector pass (or, for
// r.s, after a replacement) and reduced with gamma and delta: the textbook
// delta - beta gamma / alpha_old assumes r orthogonal to the previous
// direction, which each replacement breaks by the low-precision operator's
// gap to A.
struct EpiW {  // w = A r (FP32), gamma += r*r, delta += w*r
    static constexpr bool kUsesX = false;
    const double *r;
    float *w;
    double g, dl;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(r + row, pol); }
    __device__ void operator()(int row, double acc, double rv) {
        const float wf = __double2float_rn(acc);
        stf_hint(w + row, wf, pol);
        g += rv * rv;
        dl += (double)wf * rv;
    }
};

__global__ void __launch_bounds__(NTHREADS, 1) k_cgcg(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    __shared__ double s_wpart[2][NWARPS + 1];  // the warps' shares of r.s and p.s
    kernel_setup(P, S, P.nlay);
    const int g = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    Pipe pp;
    uint32_t phase = 0;
    const uint64_t vpol = policy_evict_last();
    const int lay64 = 0;
    int lay = P.start_layout;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int vlo = rb_lo * 16, vhi = rb_hi * 16;
    double *x = P.x, *r = P.r;
    float *pv32 = reinterpret_cast<float *>(P.d), *sv32 = reinterpret_cast<float *>(P.q),
          *wv32 = reinterpret_cast<float *>(P.s);
    float *r32 = reinterpret_cast<float *>(P.t);  // FP32 r: the input of FP32-x layouts
    const double *b = P.b;
    // r = b - A x0; p = s = 0
    EpiResidual32 er{b, r, r32, 0.0, vpol};
    if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, er)) return;
    double bbp = 0.0;
    MF_PAIRS(2, vlo, vhi, {
        double2 bv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
            stf2_hint(pv32 + 2 * MF_PI(u), make_float2(0.f, 0.f), vpol);
            stf2_hint(sv32 + 2 * MF_PI(u), make_float2(0.f, 0.f), vpol);
        }
    })
    if (lane == 0) s_wpart[0][wid] = s_wpart[1][wid] = 0.0;
    double v1[1] = {bbp}, o1[1];
    if (!grid_sum<1>(P, S, v1, o1, phase)) return;
    const double bb = o1[0];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK, repl = 0, switches = 0, fellback = 0;
    int it_lay[KMAX_LAYOUTS] = {0, 0, 0, 0};
    double gamma_old = 0.0, rel = 1.0, rr_best = 1e300, gam = 0.0;
    bool first = true, pending = false;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    while (true) {
        const bool repl_now = pending || (P.replace_every > 0 && it > 0 && it % P.replace_every == 0);
        if (repl_now) {
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiResidual32 e2{b, r, r32, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, e2)) return;
            // r.s of the replaced r with the current s (p.s is unchanged)
            double rsl = 0.0;
            MF_PAIRS(2, vlo, vhi, {
                double2 rv[_vb];
                float2 sw[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    sw[u] = ldf2_hint(sv32 + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) rsl += rv[u].x * (double)sw[u].x + rv[u].y * (double)sw[u].y;
            })
            for (int o = 16; o > 0; o >>= 1) rsl += __shfl_xor_sync(0xffffffffu, rsl, o);
            if (lane == 0) s_wpart[0][wid] = rsl;
            double a1[1] = {e2.rr}, c1[1];
            if (!grid_sum<1>(P, S, a1, c1, phase)) return;
            ++repl;
            ++ep;
            publish(P, ep);
            const double relt = bnorm > 0 ? sqrt(c1[0]) / bnorm : 0.0;
            if (pending) {
                pending = false;
                rel = relt;
                if (rel <= tol) break;
            }
            // a true residual norm more than twice the recursive one (the
            // low-precision operator's iterate has drifted from A's):
            // beta = gamma_true / gamma_old would break the directions'
            // conjugacy, so the next step restarts from the true residual
            // (beta = 0: p = r, s = w)
            if (c1[0] > 4.0 * gam) first = true;
            if (lay != lay64) {
                if (c1[0] < rr_best) rr_best = c1[0];
                if (!(c1[0] <= 1e4 * rr_best)) {
                    lay = lay64;
                    fellback = 1;
                }
                while (lay != lay64 && lay < P.nlay - 1 && relt < P.level_rel[lay]) {
                    ++lay;
                    ++switches;
                }
            }
        }
        if (it >= maxit) break;
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, lay, ep)) return;
        MF_TRACE(it, 1);
        ++it_lay[lay];
        EpiW ew{r, wv32, 0.0, 0.0, vpol};
        bool ok;
        if (lay != lay64) ok = cta_spmv<true>(P, lay, P.lay[lay].x32 ? (const void *)r32 : r, S, dyn, pp, ew);
        else ok = cta_spmv<false>(P, lay64, r, S, dyn, pp, ew);
        if (!ok) return;
        MF_TRACE(it, 2);
        double a2[4] = {ew.g, ew.dl, lane == 0 ? s_wpart[0][wid] : 0.0, lane == 0 ? s_wpart[1][wid] : 0.0}, c2[4];
        if (!grid_sum<4>(P, S, a2, c2, phase)) return;
        MF_TRACE(it, 3);
        gam = c2[0];
        const double delta = c2[1], rs_old = c2[2], ps_old = c2[3];
        rel = bnorm > 0 ? sqrt(gam) / bnorm : 0.0;
        if (!fixed && rel <= tol) {
            pending = true;  // confirm with the FP64 true residual
            continue;
        }
        double alpha, beta;
        if (first) {
            beta = 0.0;
            alpha = gam / delta;
            first = false;
        } else {
            beta = gam / gamma_old;
            alpha = gam / (delta + beta * (2.0 * rs_old + beta * ps_old));  // p.A p, as in cgcg_tm_body
        }
        if (!isfinite(alpha) || !isfinite(beta) || alpha == 0.0) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        double rsn = 0.0, psn = 0.0;
        MF_PAIRS(4, vlo, vhi, {
            double2 rv[_vb], xv[_vb];
            float2 pw[_vb], sw[_vb], ww[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                pw[u] = ldf2_hint(pv32 + 2 * MF_PI(u), vpol);
                sw[u] = ldf2_hint(sv32 + 2 * MF_PI(u), vpol);
                ww[u] = ldf2_hint(wv32 + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                const double px = rv[u].x + beta * (double)pw[u].x, py = rv[u].y + beta * (double)pw[u].y;
                const double sx = (double)ww[u].x + beta * (double)sw[u].x,
                             sy = (double)ww[u].y + beta * (double)sw[u].y;
                const float2 pf = make_float2(__double2float_rn(px), __double2float_rn(py));
                const float2 sf = make_float2(__double2float_rn(sx), __double2float_rn(sy));
                stf2_hint(pv32 + 2 * MF_PI(u), pf, vpol);
                stf2_hint(sv32 + 2 * MF_PI(u), sf, vpol);
                double2 xo, ro;
                xo.x = xv[u].x + alpha * (double)pf.x;
                xo.y = xv[u].y + alpha * (double)pf.y;
                ro.x = rv[u].x - alpha * (double)sf.x;
                ro.y = rv[u].y - alpha * (double)sf.y;
                st2_hint(x + 2 * MF_PI(u), xo, vpol);
                st2_hint(r + 2 * MF_PI(u), ro, vpol);
                stf2_hint(r32 + 2 * MF_PI(u), make_float2(__double2float_rn(ro.x), __double2float_rn(ro.y)), vpol);
                rsn += ro.x * (double)sf.x + ro.y * (double)sf.y;
                psn += (double)pf.x * (double)sf.x + (double)pf.y * (double)sf.y;
            }
        })
        for (int o = 16; o > 0; o >>= 1) {
            rsn += __shfl_xor_sync(0xffffffffu, rsn, o);
            psn += __shfl_xor_sync(0xffffffffu, psn, o);
        }
        if (lane == 0) {
            s_wpart[0][wid] = rsn;
            s_wpart[1][wid] = psn;
        }
        gamma_old = gam;
        MF_TRACE(it, 4);
        MF_TRACE(it, 5);
        ++it;
        ++ep;
        publish(P, ep);
        MF_TRACE(it - 1, 6);
    }
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = repl;
        P.res->level_switches = switches;
        P.res->rr = bnorm > 0 ? rel * rel * bb : gam;
        P.res->bb = bb;
        P.res->final_layout = lay;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = it_lay[l];
        P.res->pad = fellback;
    }
}

// ------------------------------------- CG, single reduction, x and r in TMEM
// The recurrence of k_cgcg with x and r of the CTA's own rows resident in
// tensor memory across iterations (16 bytes a row, at most 16384 rows a CTA),
// so the fused vector pass reads and writes only the FP32 vectors p, s, w and
// the FP32 copy r32 of r (the SpMV input and the halo) in global memory.
// Own rows come in blocks of 512: in block k, rows 4L .. 4L+3 belong to TMEM
// lane L (thread L % 32 of warp L / 32 of a warpgroup), columns 16k + 4j ..
// +3 holding (x low, x high, r low, r high) of row 4L + j; warp w serves the
// blocks k = w/4, w/4 + 4, ... One 16-column TMEM load and 16-byte loads of
// p, s, w cover a thread's four rows. gamma = r.r is summed where r is
// produced, delta = w.r32 in the SpMV epilogue (w itself comes from the FP32
// operator applied to r32). x goes to global memory for the FP64
// true-residual replacement and at the end; r also while the FP64 layout is
// active.
struct EpiW32 {  // w = A r (FP32), delta += w * r (r in FP32)
    // r(row) is the SpMV input: taken from the x stage when the row block's
    // own segment is staged there, else loaded
    static constexpr bool kUsesX = true;
    const float *r32;
    float *w;
    double dl;
    uint64_t pol;
    __device__ float pre(int row) const { return ldf_hint(r32 + row, pol); }
    __device__ void operator()(int row, double acc, float rv) {
        const float wf = __double2float_rn(acc);
        stf_hint(w + row, wf, pol);
        dl += (double)wf * (double)rv;
    }
};

constexpr int TM_CB = 2;  // 512-row blocks in flight per warp

struct TmemRows {
    uint32_t base;  // TMEM address of lane 32*q, column 0
    int q, k0, nblk, nrows, vlo;
    __device__ uint32_t addr(int k) const { return base + 16u * (uint32_t)k; }
    // first of the thread's four rows in block k (own-row index)
    __device__ int row_of(int k) const { return k * 512 + 4 * (32 * q + (int)(threadIdx.x & 31)); }
};
// Built inside each pass from the TMEM base (shared memory) and the CTA's
// row range, so that none of it stays live across the SpMV, which needs
// every register it can get.
__device__ __forceinline__ TmemRows tm_rows(const KParams &P, const volatile uint32_t *s_tmem) {
    const int g = blockIdx.x, w = threadIdx.x >> 5;
    TmemRows T;
    T.vlo = P.lay[0].cta_rb[g] * 16;
    T.nrows = P.lay[0].cta_rb[g + 1] * 16 - T.vlo;
    T.q = w & 3;
    T.k0 = w >> 2;
    T.nblk = (T.nrows + 511) / 512;
    T.base = *s_tmem + ((uint32_t)(32 * T.q) << 16);
    return T;
}

__device__ __forceinline__ double tm_x(const uint32_t (&t)[16], int j) {
    return __hiloint2double((int)t[4 * j + 1], (int)t[4 * j]);
}
__device__ __forceinline__ double tm_r(const uint32_t (&t)[16], int j) {
    return __hiloint2double((int)t[4 * j + 3], (int)t[4 * j + 2]);
}
__device__ __forceinline__ void tm_set(uint32_t (&t)[16], int j, double x, double r) {
    t[4 * j] = (uint32_t)__double2loint(x);
    t[4 * j + 1] = (uint32_t)__double2hiint(x);
    t[4 * j + 2] = (uint32_t)__double2loint(r);
    t[4 * j + 3] = (uint32_t)__double2hiint(r);
}

// x (when xg) and r of the own rows from global memory into TMEM; returns the
// thread's share of r.r. xg == nullptr keeps x in TMEM. Own rows are a
// multiple of 16, so a thread's four rows are all live or all past the end.
__device__ double tm_load(const TmemRows &T, const double *xg, const double *rg, uint64_t pol) {
    double rr = 0.0;
    for (int k = T.k0; k < T.nblk; k += 4) {
        const int i = T.row_of(k);
        const bool live = i < T.nrows;
        uint32_t t[16];
        __syncwarp();  // tcgen05 ops are warp-collective
        if (!xg) tmem_ld16(T.addr(k), t);
        double2 r01 = make_double2(0.0, 0.0), r23 = r01, x01 = r01, x23 = r01;
        if (live) {
            r01 = ld2_hint(rg + T.vlo + i, pol);
            r23 = ld2_hint(rg + T.vlo + i + 2, pol);
            if (xg) {
                x01 = ld2_hint(xg + T.vlo + i, pol);
                x23 = ld2_hint(xg + T.vlo + i + 2, pol);
            }
        }
        if (!xg) {
            tmem_wait_ld16(t);
            x01 = make_double2(tm_x(t, 0), tm_x(t, 1));
            x23 = make_double2(tm_x(t, 2), tm_x(t, 3));
        }
        tm_set(t, 0, x01.x, r01.x);
        tm_set(t, 1, x01.y, r01.y);
        tm_set(t, 2, x23.x, r23.x);
        tm_set(t, 3, x23.y, r23.y);
        tmem_st16_wait(T.addr(k), t);
        rr += r01.x * r01.x + r01.y * r01.y + r23.x * r23.x + r23.y * r23.y;
    }
    return rr;
}

// x (and r when rg) of the own rows from TMEM to global memory.
__device__ void tm_store(const TmemRows &T, double *xg, double *rg, uint64_t pol) {
    for (int k = T.k0; k < T.nblk; k += 4) {
        uint32_t t[16];
        __syncwarp();
        tmem_ld16(T.addr(k), t);
        tmem_wait_ld16(t);
        const int i = T.row_of(k);
        if (i < T.nrows) {
            st2_hint(xg + T.vlo + i, make_double2(tm_x(t, 0), tm_x(t, 1)), pol);
            st2_hint(xg + T.vlo + i + 2, make_double2(tm_x(t, 2), tm_x(t, 3)), pol);
            if (rg) {
                st2_hint(rg + T.vlo + i, make_double2(tm_r(t, 0), tm_r(t, 1)), pol);
                st2_hint(rg + T.vlo + i + 2, make_double2(tm_r(t, 2), tm_r(t, 3)), pol);
            }
        }
    }
}

// The vector pass of k_cgcg on TMEM-resident x, r:
//   p = r + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;  r32 = r
// p and s are stored in FP32, so they are formed by FP32 fused multiply-adds
// (p = fma(beta, p, float(r)), s = fma(beta, s, w)); x and r stay FP64. That
// is four FP32 <-> FP64 conversions a row instead of eight: conversions run
// on a narrow pipe and bounded this pass. The own rows' p, s, w
// (FP32) come into the copy ring, idle between two SpMVs, by three bulk
// copies issued while the reduction runs: one 12-byte-per-row transfer
// instead of per-thread loads waiting on L2. The host launches this kernel
// only when 12 bytes per own row fit the ring (tm_vectors_fit).
// Thread 0, after every thread's writes of p, s, w were fenced for the async
// proxy and a barrier: the copies complete on S.upd.
__device__ void tm_upd_issue(Smem &S, uint8_t *dyn, const float *pv, const float *sv, const float *wv, int vlo,
                             int nrows, uint64_t pol) {
    const uint32_t bytes = 4u * (uint32_t)nrows;  // nrows is a multiple of 16: 64-byte multiples
    fence_proxy_async_smem();  // the ring was last read by generic loads
    for (int k = 0; k < STAGES; ++k) S.res_tag[k] = 0;  // the copies overwrite the slabs
    mbar_arrive_expect_tx(&S.upd, 3u * bytes);
    bulk_g2s(dyn, pv + vlo, bytes, &S.upd, pol);
    bulk_g2s(dyn + bytes, sv + vlo, bytes, &S.upd, pol);
    bulk_g2s(dyn + 2u * bytes, wv + vlo, bytes, &S.upd, pol);
}
// The pass itself, with p, s, w read from the ring copy (sp, ss, sw: own-row
// index); p, s, r32 (and r when rg) go to global memory. Returns the
// thread's share of the new r.r.
__device__ double tm_update_smem(const TmemRows &T, double alpha, double beta, const float *sp,
                                              const float *ss, const float *sw, float *pv, float *sv, float *r32,
                                              double *rg, uint64_t pol, double &rs_out, double &ps_out) {
    double rr = 0.0, rs = 0.0, ps = 0.0;
    const float bf = (float)beta;
    for (int k = T.k0; k < T.nblk; k += 4 * TM_CB) {
        uint32_t t[TM_CB][16];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < TM_CB; ++u)
            if (k + 4 * u < T.nblk) tmem_ld16(T.addr(k + 4 * u), t[u]);
#pragma unroll
        for (int u = 0; u < TM_CB; ++u) {
            const int kk = k + 4 * u;
            __syncwarp();
            if (kk < T.nblk) {
                tmem_wait_ld16(t[u]);
                const int i = T.row_of(kk);
                const bool live = i < T.nrows;
                float4 pf = make_float4(0.f, 0.f, 0.f, 0.f), sf = pf, wf = pf;
                if (live) {
                    pf = *reinterpret_cast<const float4 *>(sp + i);
                    sf = *reinterpret_cast<const float4 *>(ss + i);
                    wf = *reinterpret_cast<const float4 *>(sw + i);
                }
                const float pin[4] = {pf.x, pf.y, pf.z, pf.w};
                const float sin_[4] = {sf.x, sf.y, sf.z, sf.w};
                const float win[4] = {wf.x, wf.y, wf.z, wf.w};
                float pn[4], sn[4], rn[4];
                double rsq = 0.0, rsd = 0.0, psd = 0.0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    double xv = tm_x(t[u], j), rv = tm_r(t[u], j);
                    pn[j] = __fmaf_rn(bf, pin[j], __double2float_rn(rv));
                    sn[j] = __fmaf_rn(bf, sin_[j], win[j]);
                    xv = fma(alpha, (double)pn[j], xv);
                    rv = fma(-alpha, (double)sn[j], rv);
                    tm_set(t[u], j, xv, rv);
                    rn[j] = __double2float_rn(rv);
                    rsq += rv * rv;
                    rsd += rv * (double)sn[j];
                    psd += (double)pn[j] * (double)sn[j];
                }
                tmem_st16_wait(T.addr(kk), t[u]);
                if (live) {
                    const int row = T.vlo + i;
                    stf4_hint(pv + row, make_float4(pn[0], pn[1], pn[2], pn[3]), pol);
                    stf4_hint(sv + row, make_float4(sn[0], sn[1], sn[2], sn[3]), pol);
                    stf4_hint(r32 + row, make_float4(rn[0], rn[1], rn[2], rn[3]), pol);
                    if (rg) {
                        st2_hint(rg + row, make_double2(tm_r(t[u], 0), tm_r(t[u], 1)), pol);
                        st2_hint(rg + row + 2, make_double2(tm_r(t[u], 2), tm_r(t[u], 3)), pol);
                    }
                    rr += rsq;
                    rs += rsd;
                    ps += psd;
                }
            }
        }
    }
    rs_out = rs;
    ps_out = ps;
    return rr;
}

__device__ __forceinline__ void cgcg_tm_body(const KParams &P, Smem &S, uint8_t *dyn, const volatile uint32_t *s_tmem,
                                             volatile double *s_gpart, volatile double (*s_wpart)[NWARPS + 1]) {
    const int g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0;
    const uint64_t vpol = policy_evict_last();
    const int lay64 = 0;
    int lay = P.start_layout;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int vlo = rb_lo * 16, vhi = rb_hi * 16;
    if (12ll * (vhi - vlo) > (long long)STAGES * P.stage_stride) {  // the host checks this first
        set_error(P, (uint32_t)MF_ERR_UNSUPPORTED, 31);
        return;
    }
    double *x = P.x, *r = P.r;
    float *pv32 = reinterpret_cast<float *>(P.d), *sv32 = reinterpret_cast<float *>(P.q),
          *wv32 = reinterpret_cast<float *>(P.s);
    float *r32 = reinterpret_cast<float *>(P.t);
    const double *b = P.b;
    // r = b - A x0 (global r and r32); p = s = 0; x, r into TMEM
    EpiResidual32 er{b, r, r32, 0.0, vpol};
    if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, er)) return;
    double bbp = 0.0;
    MF_PAIRS(2, vlo, vhi, {
        double2 bv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
            stf2_hint(pv32 + 2 * MF_PI(u), make_float2(0.f, 0.f), vpol);
            stf2_hint(sv32 + 2 * MF_PI(u), make_float2(0.f, 0.f), vpol);
        }
    })
    // this thread's share of r.r, carried to the next reduction in shared
    // memory (not in a register across the SpMV); the warps' shares of r.s
    // and p.s (p = s = 0 before the first iteration) likewise
    s_gpart[tid] = tm_load(tm_rows(P, s_tmem), x, r, vpol);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) s_wpart[0][wid] = s_wpart[1][wid] = 0.0;
    double v1[1] = {bbp}, o1[1];
    if (!grid_sum<1>(P, S, v1, o1, phase)) return;
    const double bb = o1[0];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK, repl = 0, switches = 0, fellback = 0;
    int it_lay[KMAX_LAYOUTS] = {0, 0, 0, 0};
    double gamma_old = 0.0, rel = 1.0, rr_best = 1e300, gam = 0.0;
    bool first = true, pending = false;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    uint32_t uph = 0;
    while (true) {
        const bool repl_now = pending || (P.replace_every > 0 && it > 0 && it % P.replace_every == 0);
        if (repl_now) {
            // x to global memory for the FP64 SpMV, then r = b - A x into TMEM
            tm_store(tm_rows(P, s_tmem), x, nullptr, vpol);
            ++ep;
            publish(P, ep);
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiResidual32 e2{b, r, r32, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, e2)) return;
            const double gl = tm_load(tm_rows(P, s_tmem), nullptr, r, vpol);
            s_gpart[tid] = gl;
            // r.s of the replaced r with the current s (the next step's
            // p.A p needs it; p.s is unchanged)
            double rsl = 0.0;
            MF_PAIRS(2, vlo, vhi, {
                double2 rv[_vb];
                float2 sv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    sv[u] = *reinterpret_cast<const float2 *>(sv32 + 2 * MF_PI(u));
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) rsl += rv[u].x * (double)sv[u].x + rv[u].y * (double)sv[u].y;
            })
            for (int o = 16; o > 0; o >>= 1) rsl += __shfl_xor_sync(0xffffffffu, rsl, o);
            if (lane == 0) s_wpart[0][wid] = rsl;
            double a1[1] = {gl}, c1[1];
            if (!grid_sum<1>(P, S, a1, c1, phase)) return;
            ++repl;
            ++ep;
            publish(P, ep);
            const double relt = bnorm > 0 ? sqrt(c1[0]) / bnorm : 0.0;
            if (pending) {
                pending = false;
                rel = relt;
                if (rel <= tol) break;
            }
            // a true residual norm more than twice the recursive one (the
            // low-precision operator's iterate has drifted from A's):
            // beta = gamma_true / gamma_old would break the directions'
            // conjugacy, so the next step restarts from the true residual
            // (beta = 0: p = r, s = w)
            if (c1[0] > 4.0 * gam) first = true;
            if (lay != lay64) {
                if (c1[0] < rr_best) rr_best = c1[0];
                if (!(c1[0] <= 1e4 * rr_best)) {
                    lay = lay64;
                    fellback = 1;
                }
                while (lay != lay64 && lay < P.nlay - 1 && relt < P.level_rel[lay]) {
                    ++lay;
                    ++switches;
                }
            }
        }
        if (it >= maxit) break;
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, lay, ep)) return;
        MF_TRACE(it, 1);
        ++it_lay[lay];
        EpiW32 ew{r32, wv32, 0.0, vpol};
        bool ok;
        if (lay != lay64) ok = cta_spmv<true>(P, lay, P.lay[lay].x32 ? (const void *)r32 : r, S, dyn, pp, ew);
        else ok = cta_spmv<false>(P, lay64, r, S, dyn, pp, ew);
        if (!ok) return;
        MF_TRACE(it, 2);
        // the ring is idle until the next SpMV: p, s, w of the own rows come
        // into it while the reduction runs (every writer fences its stores
        // for the async proxy before the barrier)
        fence_proxy_async_global();
        __syncthreads();
        if (tid == 0) tm_upd_issue(S, dyn, pv32, sv32, wv32, vlo, vhi - vlo, vpol);
        double a2[4] = {s_gpart[tid], ew.dl, lane == 0 ? s_wpart[0][wid] : 0.0, lane == 0 ? s_wpart[1][wid] : 0.0},
               c2[4];
        const bool red_ok = grid_sum<4>(P, S, a2, c2, phase);
        // no path leaves with the copies in flight
        if (!wait_bar(&S.upd, uph, P.limit_ns)) {
            set_error(P, (uint32_t)MF_ERR_TIMEOUT, 30);
            return;
        }
        uph ^= 1u;
        if (!red_ok) return;
        MF_TRACE(it, 3);
        gam = c2[0];
        const double delta = c2[1], rs_old = c2[2], ps_old = c2[3];
        rel = bnorm > 0 ? sqrt(gam) / bnorm : 0.0;
        if (!fixed && rel <= tol) {
            pending = true;  // confirm with the FP64 true residual
            zero_slots(dyn, P.stage_stride, P.slab_area);  // the copies overwrote them
            continue;
        }
        // p = r + beta p_old, s = w + beta s_old: p.A p = p.s = r.w + 2 beta
        // r.s_old + beta^2 p_old.s_old (A symmetric). Summed from its parts
        // rather than taken as delta - beta gamma / alpha_old, which assumes
        // the orthogonality of r to the previous direction: a true-residual
        // replacement breaks that by the gap between the low-precision
        // operator and A.
        double alpha, beta;
        if (first) {
            beta = 0.0;
            alpha = gam / delta;
            first = false;
        } else {
            beta = gam / gamma_old;
            alpha = gam / (delta + beta * (2.0 * rs_old + beta * ps_old));
        }
        if (!isfinite(alpha) || !isfinite(beta) || alpha == 0.0) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const float *sp = reinterpret_cast<const float *>(dyn);
        double rsn, psn;
        // the next SpMV reads r from global memory unless its layout stages
        // x in FP32 (then it reads r32): the FP64 layout, and mixed layouts
        // with FP64 tiles, need r written back from tensor memory
        const bool r_global = lay == lay64 || !P.lay[lay].x32;
        s_gpart[tid] = tm_update_smem(tm_rows(P, s_tmem), alpha, beta, sp, sp + (vhi - vlo), sp + 2 * (vhi - vlo),
                                      pv32, sv32, r32, r_global ? r : nullptr, vpol, rsn, psn);
        for (int o = 16; o > 0; o >>= 1) {
            rsn += __shfl_xor_sync(0xffffffffu, rsn, o);
            psn += __shfl_xor_sync(0xffffffffu, psn, o);
        }
        if (lane == 0) {
            s_wpart[0][wid] = rsn;
            s_wpart[1][wid] = psn;
        }
        gamma_old = gam;
        MF_TRACE(it, 4);
        MF_TRACE(it, 5);
        ++it;
        ++ep;
        publish(P, ep);
        // the copies overwrote the zero slots: restored after publish's
        // barrier (the pass is done reading the ring) and before the next
        // SpMV (the halo wait ends with a barrier)
        zero_slots(dyn, P.stage_stride, P.slab_area);
        MF_TRACE(it - 1, 6);
    }
    tm_store(tm_rows(P, s_tmem), x, r, vpol);
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = repl;
        P.res->level_switches = switches;
        P.res->rr = bnorm > 0 ? rel * rel * bb : gam;
        P.res->bb = bb;
        P.res->final_layout = lay;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = it_lay[l];
        P.res->pad = fellback;
    }
}

// One CTA per SM holds all 512 TMEM columns for the whole solve; every exit
// of the body (including aborts) comes back here to release them.
__global__ void __launch_bounds__(NTHREADS, 1) k_cgcg_tm(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    __shared__ uint32_t s_tmem;
    __shared__ double s_gpart[NTHREADS];
    __shared__ double s_wpart[2][NWARPS + 1];
    kernel_setup(P, S, P.nlay);
    const int w = threadIdx.x >> 5;
    if (w == 0) tmem_alloc512(&s_tmem);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    cgcg_tm_body(P, S, dyn, &s_tmem, s_gpart, s_wpart);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    if (w == 0) tmem_dealloc512(s_tmem);
}

// ------------------------------------------------------- FP64 CG with TMEM
// The reference's CG recurrence (as k_cg<false>) with x and r of the own
// rows resident in tensor memory for the whole solve; d (the SpMV input,
// read by the neighbours' x windows) and q stay in global memory. Each of
// the two vector passes reads its global vector from a bulk copy into the
// idle ring, issued before the grid reduction that precedes the pass:
//   r -= alpha q            (q copied while d.q is reduced)
//   x += alpha d; d = r + beta d   (d copied while r.r is reduced)
// Global traffic per row and iteration: q 8 + d 16 bytes instead of 64.

// r -= alpha q over the TMEM rows, q from the ring copy (own-row index);
// returns the thread's share of the new r.r.
__device__ double tm_cg_r(const TmemRows &T, double alpha, const double *sq) {
    double rr = 0.0;
    for (int k = T.k0; k < T.nblk; k += 4 * TM_CB) {
        uint32_t t[TM_CB][16];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < TM_CB; ++u)
            if (k + 4 * u < T.nblk) tmem_ld16(T.addr(k + 4 * u), t[u]);
#pragma unroll
        for (int u = 0; u < TM_CB; ++u) {
            const int kk = k + 4 * u;
            __syncwarp();
            if (kk < T.nblk) {
                tmem_wait_ld16(t[u]);
                const int i = T.row_of(kk);
                if (i < T.nrows) {
                    const double2 q01 = *reinterpret_cast<const double2 *>(sq + i);
                    const double2 q23 = *reinterpret_cast<const double2 *>(sq + i + 2);
                    const double qv[4] = {q01.x, q01.y, q23.x, q23.y};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const double rv = tm_r(t[u], j) - alpha * qv[j];
                        tm_set(t[u], j, tm_x(t[u], j), rv);
                        rr += rv * rv;
                    }
                }
                tmem_st16_wait(T.addr(kk), t[u]);
            }
        }
    }
    return rr;
}
// x += alpha d and (unless done) d = r + beta d to global memory, d from the
// ring copy.
__device__ void tm_cg_xd(const TmemRows &T, double alpha, double beta, bool done, const double *sd, double *dg,
                         uint64_t pol) {
    for (int k = T.k0; k < T.nblk; k += 4 * TM_CB) {
        uint32_t t[TM_CB][16];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < TM_CB; ++u)
            if (k + 4 * u < T.nblk) tmem_ld16(T.addr(k + 4 * u), t[u]);
#pragma unroll
        for (int u = 0; u < TM_CB; ++u) {
            const int kk = k + 4 * u;
            __syncwarp();
            if (kk < T.nblk) {
                tmem_wait_ld16(t[u]);
                const int i = T.row_of(kk);
                if (i < T.nrows) {
                    const double2 d01 = *reinterpret_cast<const double2 *>(sd + i);
                    const double2 d23 = *reinterpret_cast<const double2 *>(sd + i + 2);
                    const double dv[4] = {d01.x, d01.y, d23.x, d23.y};
                    double dn[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const double rv = tm_r(t[u], j);
                        tm_set(t[u], j, tm_x(t[u], j) + alpha * dv[j], rv);
                        dn[j] = rv + beta * dv[j];
                    }
                    if (!done) {
                        st2_hint(dg + T.vlo + i, make_double2(dn[0], dn[1]), pol);
                        st2_hint(dg + T.vlo + i + 2, make_double2(dn[2], dn[3]), pol);
                    }
                }
                tmem_st16_wait(T.addr(kk), t[u]);
            }
        }
    }
}
// Thread 0: one bulk copy of the own rows of an FP64 vector into the ring.
__device__ void tm_vec_issue(Smem &S, uint8_t *dyn, const double *v, int vlo, int nrows, uint64_t pol) {
    const uint32_t bytes = 8u * (uint32_t)nrows;  // nrows is a multiple of 16
    fence_proxy_async_smem();  // the ring was last read by generic loads
    for (int k = 0; k < STAGES; ++k) S.res_tag[k] = 0;  // the copy overwrites the slabs
    mbar_arrive_expect_tx(&S.upd, bytes);
    bulk_g2s(dyn, v + vlo, bytes, &S.upd, pol);
}

__device__ __forceinline__ void cg_tm_body(const KParams &P, Smem &S, uint8_t *dyn, const volatile uint32_t *s_tmem) {
    const int g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0, uph = 0;
    const uint64_t vpol = policy_evict_last();
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int vlo = rb_lo * 16, vhi = rb_hi * 16;
    if (8ll * (vhi - vlo) > (long long)STAGES * P.stage_stride) {  // the host checks this first
        set_error(P, (uint32_t)MF_ERR_UNSUPPORTED, 32);
        return;
    }
    double *x = P.x, *r = P.r, *d = P.d, *q = P.q;
    const double *b = P.b;
    const double *sv = reinterpret_cast<const double *>(dyn);
    if (P.inject_wait) {
        // test hook (as in k_cg): an epoch no CTA publishes; the bounded wait
        // must end the solve with MF_ERR_TIMEOUT
        if (!wait_deps(P, S, 0, 0xffffffffu)) return;
    }
    // the bulk copy of the own rows of v (written by this CTA's threads
    // before: each fences its stores for the async proxy, then the barrier)
    auto copy_own = [&](const double *v) {
        fence_proxy_async_global();
        __syncthreads();
        if (tid == 0) tm_vec_issue(S, dyn, v, vlo, vhi - vlo, vpol);
    };
    auto copy_wait = [&]() -> bool {
        if (!wait_bar(&S.upd, uph, P.limit_ns)) {
            set_error(P, (uint32_t)MF_ERR_TIMEOUT, 33);
            return false;
        }
        uph ^= 1u;
        return true;
    };
    // r = b - A x0 (global), d = r; x, r into TMEM; (rr, bb)
    EpiResidual er{b, r, 0.0, vpol};
    if (!cta_spmv<false>(P, 0, x, S, dyn, pp, er)) return;
    __syncthreads();
    double bbp = 0.0;
    MF_PAIRS(4, vlo, vhi, {
        double2 rv[_vb], bv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
        }
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            st2_hint(d + 2 * MF_PI(u), rv[u], vpol);
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
        }
    })
    __syncthreads();
    tm_load(tm_rows(P, s_tmem), x, r, vpol);
    double v2[2] = {er.rr, bbp}, o2[2];
    if (!grid_sum<2>(P, S, v2, o2, phase)) return;
    double rr = o2[0];
    const double bb = o2[1];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK;
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    while (it < maxit && (fixed || rel > tol)) {
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, 0, ep)) return;
        MF_TRACE(it, 1);
        EpiQ eq{d, q, 0.0, vpol};
        if (!cta_spmv<false>(P, 0, d, S, dyn, pp, eq)) return;
        MF_TRACE(it, 2);
        copy_own(q);
        double v1[1] = {eq.dq}, o1[1];
        const bool ok1 = grid_sum<1>(P, S, v1, o1, phase);
        if (!copy_wait() || !ok1) return;  // no path leaves with the copy in flight
        MF_TRACE(it, 3);
        const double dq = o1[0];
        if (!(dq != 0.0) || !isfinite(dq)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rr / dq;
        const double rrp = tm_cg_r(tm_rows(P, s_tmem), alpha, sv);
        MF_TRACE(it, 4);
        // every thread is done reading q from the ring before d lands there
        __syncthreads();
        copy_own(d);
        double w1[1] = {rrp}, u1[1];
        const bool ok2 = grid_sum<1>(P, S, w1, u1, phase);
        if (!copy_wait() || !ok2) return;
        MF_TRACE(it, 5);
        const double rrn = u1[0];
        ++it;
        rel = bnorm > 0 ? sqrt(rrn) / bnorm : 0.0;
        const double beta = rrn / rr;
        const bool done = !fixed && rel <= tol;
        tm_cg_xd(tm_rows(P, s_tmem), alpha, beta, done, sv, d, vpol);
        rr = rrn;
        ++ep;
        publish(P, ep);
        zero_slots(dyn, P.stage_stride, P.slab_area);  // as in k_cgcg_tm
        MF_TRACE(it - 1, 6);
        if (!isfinite(rrn)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
    }
    __syncthreads();
    tm_store(tm_rows(P, s_tmem), x, r, vpol);
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = 0;
        P.res->level_switches = 0;
        P.res->rr = rr;
        P.res->bb = bb;
        P.res->final_layout = 0;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = l == 0 ? it : 0;
        P.res->pad = 0;
    }
}

// One CTA per SM holds all 512 TMEM columns for the whole solve; every exit
// of the body (including aborts) comes back here to release them.
__global__ void __launch_bounds__(NTHREADS, 1) k_cg_tm(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    __shared__ uint32_t s_tmem;
    kernel_setup(P, S, 1);
    const int w = threadIdx.x >> 5;
    if (w == 0) tmem_alloc512(&s_tmem);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    cg_tm_body(P, S, dyn, &s_tmem);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    if (w == 0) tmem_dealloc512(s_tmem);
}

// ------------------------------------------- Jacobi PCG with TMEM (k_pcg_tm)
// k_pcg's recurrence with x and r in tensor memory (as k_cg_tm); d and q in
// global memory. The Jacobi scaling 1/a_ii is applied from an FP32 copy that
// rides with q (r pass) and with d (x/d pass) in the ring: 12 bytes a row.

// Thread 0: q (or d) and the FP32 scaling of the own rows into the ring.
__device__ void tm_vec2_issue(Smem &S, uint8_t *dyn, const double *v, const float *m32, int vlo, int nrows,
                              uint64_t pol) {
    const uint32_t b8 = 8u * (uint32_t)nrows, b4 = 4u * (uint32_t)nrows;  // nrows is a multiple of 16
    fence_proxy_async_smem();  // the ring was last read by generic loads
    for (int k = 0; k < STAGES; ++k) S.res_tag[k] = 0;  // the copies overwrite the slabs
    mbar_arrive_expect_tx(&S.upd, b8 + b4);
    bulk_g2s(dyn, v + vlo, b8, &S.upd, pol);
    bulk_g2s(dyn + b8, m32 + vlo, b4, &S.upd, pol);
}
// r -= alpha q, z = m r; returns the thread's shares of r.z (rz) and r.r.
__device__ double tm_pcg_r(const TmemRows &T, double alpha, const double *sq, const float *sm, double &rz) {
    double rr = 0.0;
    rz = 0.0;
    for (int k = T.k0; k < T.nblk; k += 4 * TM_CB) {
        uint32_t t[TM_CB][16];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < TM_CB; ++u)
            if (k + 4 * u < T.nblk) tmem_ld16(T.addr(k + 4 * u), t[u]);
#pragma unroll
        for (int u = 0; u < TM_CB; ++u) {
            const int kk = k + 4 * u;
            __syncwarp();
            if (kk < T.nblk) {
                tmem_wait_ld16(t[u]);
                const int i = T.row_of(kk);
                if (i < T.nrows) {
                    const double2 q01 = *reinterpret_cast<const double2 *>(sq + i);
                    const double2 q23 = *reinterpret_cast<const double2 *>(sq + i + 2);
                    const float4 m4 = *reinterpret_cast<const float4 *>(sm + i);
                    const double qv[4] = {q01.x, q01.y, q23.x, q23.y};
                    const double mv[4] = {(double)m4.x, (double)m4.y, (double)m4.z, (double)m4.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const double rv = tm_r(t[u], j) - alpha * qv[j];
                        tm_set(t[u], j, tm_x(t[u], j), rv);
                        rz += rv * (mv[j] * rv);
                        rr += rv * rv;
                    }
                }
                tmem_st16_wait(T.addr(kk), t[u]);
            }
        }
    }
    return rr;
}
// x += alpha d and (unless done) d = m r + beta d to global memory.
__device__ void tm_pcg_xd(const TmemRows &T, double alpha, double beta, bool done, const double *sd, const float *sm,
                          double *dg, uint64_t pol) {
    for (int k = T.k0; k < T.nblk; k += 4 * TM_CB) {
        uint32_t t[TM_CB][16];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < TM_CB; ++u)
            if (k + 4 * u < T.nblk) tmem_ld16(T.addr(k + 4 * u), t[u]);
#pragma unroll
        for (int u = 0; u < TM_CB; ++u) {
            const int kk = k + 4 * u;
            __syncwarp();
            if (kk < T.nblk) {
                tmem_wait_ld16(t[u]);
                const int i = T.row_of(kk);
                if (i < T.nrows) {
                    const double2 d01 = *reinterpret_cast<const double2 *>(sd + i);
                    const double2 d23 = *reinterpret_cast<const double2 *>(sd + i + 2);
                    const float4 m4 = *reinterpret_cast<const float4 *>(sm + i);
                    const double dv[4] = {d01.x, d01.y, d23.x, d23.y};
                    const double mv[4] = {(double)m4.x, (double)m4.y, (double)m4.z, (double)m4.w};
                    double dn[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const double rv = tm_r(t[u], j);
                        tm_set(t[u], j, tm_x(t[u], j) + alpha * dv[j], rv);
                        dn[j] = mv[j] * rv + beta * dv[j];
                    }
                    if (!done) {
                        st2_hint(dg + T.vlo + i, make_double2(dn[0], dn[1]), pol);
                        st2_hint(dg + T.vlo + i + 2, make_double2(dn[2], dn[3]), pol);
                    }
                }
                tmem_st16_wait(T.addr(kk), t[u]);
            }
        }
    }
}

__device__ __forceinline__ void pcg_tm_body(const KParams &P, Smem &S, uint8_t *dyn, const volatile uint32_t *s_tmem) {
    const int g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0, uph = 0;
    const uint64_t vpol = policy_evict_last();
    const int vlo = P.lay[0].cta_rb[g] * 16, vhi = P.lay[0].cta_rb[g + 1] * 16;
    const int nrows = vhi - vlo;
    if (12ll * nrows > (long long)STAGES * P.stage_stride) {  // the host checks this first
        set_error(P, (uint32_t)MF_ERR_UNSUPPORTED, 34);
        return;
    }
    double *x = P.x, *r = P.r, *d = P.d, *q = P.q;
    const float *m32 = P.p32;  // FP32 1/a_ii
    const double *b = P.b;
    const double *sv = reinterpret_cast<const double *>(dyn);
    const float *sm = reinterpret_cast<const float *>(dyn + 8 * (size_t)nrows);
    auto copy_own = [&](const double *v) {
        fence_proxy_async_global();
        __syncthreads();
        if (tid == 0) tm_vec2_issue(S, dyn, v, m32, vlo, nrows, vpol);
    };
    auto copy_wait = [&]() -> bool {
        if (!wait_bar(&S.upd, uph, P.limit_ns)) {
            set_error(P, (uint32_t)MF_ERR_TIMEOUT, 35);
            return false;
        }
        uph ^= 1u;
        return true;
    };
    // r = b - A x0 (global); d = z = m r; x, r into TMEM; (rr, rz, bb)
    EpiResidual er{b, r, 0.0, vpol};
    if (!cta_spmv<false>(P, 0, x, S, dyn, pp, er)) return;
    __syncthreads();
    double rzp = 0.0, bbp = 0.0;
    MF_PAIRS(2, vlo, vhi, {
        double2 rv[_vb], bv[_vb];
        float2 mv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
            mv[u] = *reinterpret_cast<const float2 *>(m32 + 2 * MF_PI(u));
        }
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            double2 z;
            z.x = (double)mv[u].x * rv[u].x;
            z.y = (double)mv[u].y * rv[u].y;
            st2_hint(d + 2 * MF_PI(u), z, vpol);
            rzp += rv[u].x * z.x + rv[u].y * z.y;
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
        }
    })
    __syncthreads();
    tm_load(tm_rows(P, s_tmem), x, r, vpol);
    double v3[3] = {er.rr, rzp, bbp}, o3[3];
    if (!grid_sum<3>(P, S, v3, o3, phase)) return;
    double rr = o3[0], rz = o3[1];
    const double bb = o3[2];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK;
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    while (it < maxit && (fixed || rel > tol)) {
        MF_TRACE(it, 0);
        if (!wait_deps(P, S, 0, ep)) return;
        MF_TRACE(it, 1);
        EpiQ eq{d, q, 0.0, vpol};
        if (!cta_spmv<false>(P, 0, d, S, dyn, pp, eq)) return;
        MF_TRACE(it, 2);
        copy_own(q);
        double v1[1] = {eq.dq}, o1[1];
        const bool ok1 = grid_sum<1>(P, S, v1, o1, phase);
        if (!copy_wait() || !ok1) return;  // no path leaves with the copies in flight
        MF_TRACE(it, 3);
        const double dq = o1[0];
        if (!(dq != 0.0) || !isfinite(dq)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rz / dq;
        double rzn;
        const double rrn_p = tm_pcg_r(tm_rows(P, s_tmem), alpha, sv, sm, rzn);
        MF_TRACE(it, 4);
        __syncthreads();  // every thread is done reading q before d lands there
        copy_own(d);
        double w2[2] = {rzn, rrn_p}, u2[2];
        const bool ok2 = grid_sum<2>(P, S, w2, u2, phase);
        if (!copy_wait() || !ok2) return;
        MF_TRACE(it, 5);
        rr = u2[1];
        ++it;
        rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        const double beta = u2[0] / rz;
        rz = u2[0];
        const bool done = !fixed && rel <= tol;
        tm_pcg_xd(tm_rows(P, s_tmem), alpha, beta, done, sv, sm, d, vpol);
        ++ep;
        publish(P, ep);
        zero_slots(dyn, P.stage_stride, P.slab_area);  // as in k_cgcg_tm
        MF_TRACE(it - 1, 6);
        if (!isfinite(rr)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
    }
    __syncthreads();
    tm_store(tm_rows(P, s_tmem), x, r, vpol);
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = 0;
        P.res->level_switches = 0;
        P.res->rr = rr;
        P.res->bb = bb;
        P.res->final_layout = 0;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = l == 0 ? it : 0;
        P.res->pad = 0;
    }
}

__global__ void __launch_bounds__(NTHREADS, 1) k_pcg_tm(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    __shared__ uint32_t s_tmem;
    kernel_setup(P, S, 1);
    const int w = threadIdx.x >> 5;
    if (w == 0) tmem_alloc512(&s_tmem);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    pcg_tm_body(P, S, dyn, &s_tmem);
    tcgen05_fence_before_sync();
    __syncthreads();
    tcgen05_fence_after_sync();
    if (w == 0) tmem_dealloc512(s_tmem);
}

// -------------------------------------------------------------- BiCGSTAB
struct EpiDot {  // y = A p, dot += z*y
    static constexpr bool kUsesX = false;
    const double *z;
    double *y;
    double dot;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(z + row, pol); }
    __device__ void operator()(int row, double acc, double zv) {
        st_hint(y + row, acc, pol);
        dot += zv * acc;
    }
};
struct EpiDot2 {  // t = A s, ts += t*s, tt += t*t
    static constexpr bool kUsesX = true;  // s is the SpMV input
    const double *s;
    double *t;
    double ts, tt;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(s + row, pol); }
    __device__ void operator()(int row, double acc, double sv) {
        st_hint(t + row, acc, pol);
        ts += acc * sv;
        tt += acc * acc;
    }
};
struct EpiDot4 {  // t = A s; ts += t*s, tt += t*t, hs += r^*s, ht += r^*t
    static constexpr bool kUsesX = true;  // s is the SpMV input
    const double *s, *rh;
    double *t;
    double ts, tt, hs, ht;
    uint64_t pol;
    __device__ double pre(int row) const { return ld_hint(s + row, pol); }
    __device__ void operator()(int row, double acc, double sv) {
        st_hint(t + row, acc, pol);
        const double hv = ld_hint(rh + row, pol);
        ts += acc * sv;
        tt += acc * acc;
        hs += hv * sv;
        ht += hv * acc;
    }
};

// MIXED: both SpMVs run on the low-precision layouts (FP32 copies of p and
// s are their input on FP32-x layouts); x, r, p, s, t, v, the dots and the
// scalars stay FP64. r is replaced by the FP64 true residual b - A x every
// replace_every iterations and before the solve stops, rho = r^.r is
// recomputed from it, and the levels and the FP64 fallback follow k_cg.
template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1) k_bicgstab(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, P.nlay);
    const int g = blockIdx.x, tid = threadIdx.x;
    Pipe pp;
    uint32_t phase = 0;
    const uint64_t vpol = policy_evict_last();
    const int lay64 = 0;
    int lay = MIXED ? P.start_layout : 0;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int vlo = rb_lo * 16, vhi = rb_hi * 16;  // own rows, zero padded past rowA
    double *x = P.x, *r = P.r, *p = P.d, *v = P.q, *s = P.s, *t = P.t, *rh = P.rh;
    float *p32 = P.p32, *s32 = P.s32;
    const double *b = P.b;
    EpiResidual er{b, r, 0.0, vpol};
    if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, er)) return;
    __syncthreads();
    double bbp = 0.0, rhop = 0.0;
    MF_PAIRS(4, vlo, vhi, {
        double2 rv[_vb], bv[_vb];
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
            bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
        }
#pragma unroll
        MF_FOR_VB if (MF_LIVE(u, vhi)) {
            st2_hint(rh + 2 * MF_PI(u), rv[u], vpol);
            st2_hint(p + 2 * MF_PI(u), rv[u], vpol);
            if (MIXED)
                stf2_hint(p32 + 2 * MF_PI(u), make_float2(__double2float_rn(rv[u].x), __double2float_rn(rv[u].y)),
                          vpol);
            bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
            rhop += rv[u].x * rv[u].x + rv[u].y * rv[u].y;
        }
    })
    double v3[3] = {er.rr, bbp, rhop}, o3[3];
    if (!grid_sum<3>(P, S, v3, o3, phase)) return;
    double rr = o3[0];
    const double bb = o3[1];
    double rho = o3[2];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK, repl = 0, switches = 0, fellback = 0;
    int it_lay[KMAX_LAYOUTS] = {0, 0, 0, 0};
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    double rr_best = rr;
    bool pending = false;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    if constexpr (!MIXED) {
        // FP64: two grid reductions and two vector passes an iteration.
        // rho' = r^.r_new = r^.s - omega r^.t joins the t.s, t.t reduction;
        // the x, r and p updates share one pass; that pass's r.r is reduced
        // with the next iteration's r^.v, so the stop test sees it after the
        // next SpMV, with x already final (that SpMV's v goes unused).
        double rrp = 0.0;
        bool carry = false;  // rrp holds the r.r of an update not yet reduced
        while (carry || (it < maxit && (fixed || rel > tol))) {
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiDot ev{rh, v, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, p, S, dyn, pp, ev)) return;
            double a1[2] = {ev.dot, rrp}, b1[2];
            if (!grid_sum<2>(P, S, a1, b1, phase)) return;
            if (carry) {
                carry = false;
                rr = b1[1];
                rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
                if (!isfinite(rr)) {
                    status = MF_ERR_BREAKDOWN;
                    break;
                }
                if (it >= maxit || (!fixed && rel <= tol)) break;
            }
            if (!(b1[0] != 0.0) || !isfinite(b1[0])) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
            const double alpha = rho / b1[0];
            MF_PAIRS(4, vlo, vhi, {
                double2 rv[_vb], vv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    vv[u] = ld2_hint(v + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    double2 o;
                    o.x = rv[u].x - alpha * vv[u].x;
                    o.y = rv[u].y - alpha * vv[u].y;
                    st2_hint(s + 2 * MF_PI(u), o, vpol);
                }
            })
            ++ep;
            publish(P, ep);
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiDot4 et{s, rh, t, 0.0, 0.0, 0.0, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, s, S, dyn, pp, et)) return;
            double a2[4] = {et.ts, et.tt, et.hs, et.ht}, b2[4];
            if (!grid_sum<4>(P, S, a2, b2, phase)) return;
            if (!(b2[1] != 0.0) || !isfinite(b2[1])) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
            const double omega = b2[0] / b2[1];
            const double rho1 = b2[2] - omega * b2[3];
            const double beta = omega != 0.0 ? (rho1 * alpha) / (rho * omega) : 0.0;
            rrp = 0.0;
            MF_PAIRS(2, vlo, vhi, {
                double2 sv[_vb], xv[_vb], pv[_vb], tv[_vb], vv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    sv[u] = ld2_hint(s + 2 * MF_PI(u), vpol);
                    xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                    pv[u] = ld2_hint(p + 2 * MF_PI(u), vpol);
                    tv[u] = ld2_hint(t + 2 * MF_PI(u), vpol);
                    vv[u] = ld2_hint(v + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    double2 xo, ro, po;
                    xo.x = xv[u].x + alpha * pv[u].x + omega * sv[u].x;
                    xo.y = xv[u].y + alpha * pv[u].y + omega * sv[u].y;
                    st2_hint(x + 2 * MF_PI(u), xo, vpol);
                    ro.x = sv[u].x - omega * tv[u].x;
                    ro.y = sv[u].y - omega * tv[u].y;
                    st2_hint(r + 2 * MF_PI(u), ro, vpol);
                    po.x = ro.x + beta * (pv[u].x - omega * vv[u].x);
                    po.y = ro.y + beta * (pv[u].y - omega * vv[u].y);
                    st2_hint(p + 2 * MF_PI(u), po, vpol);
                    rrp += ro.x * ro.x + ro.y * ro.y;
                }
            })
            rho = rho1;
            ++it;
            carry = true;
            ++ep;
            publish(P, ep);
            if (omega == 0.0) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
        }
        if (carry) {  // a breakdown left the last update's r.r unreduced
            double a1[1] = {rrp}, b1[1];
            if (!grid_sum<1>(P, S, a1, b1, phase)) return;
            rr = b1[0];
            rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        }
    } else {
    while (it < maxit && (fixed || rel > tol || pending)) {
        if (MIXED && (pending || (P.replace_every > 0 && it > 0 && it % P.replace_every == 0))) {
            // r = b - A x on the FP64 layout, rho = r^.r from it
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiResidual e2{b, r, 0.0, vpol};
            if (!cta_spmv<false>(P, lay64, x, S, dyn, pp, e2)) return;
            double rhr = 0.0;
            MF_PAIRS(4, vlo, vhi, {
                double2 rv[_vb], hv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    hv[u] = ld2_hint(rh + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) rhr += rv[u].x * hv[u].x + rv[u].y * hv[u].y;
            })
            double c2[2] = {e2.rr, rhr}, d2[2];
            if (!grid_sum<2>(P, S, c2, d2, phase)) return;
            rr = d2[0];
            rho = d2[1];
            ++repl;
            rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
            if (pending) {
                pending = false;
                if (rel <= tol) break;
            }
            if (lay != lay64) {
                if (rr < rr_best) rr_best = rr;
                if (!(rr <= 1e4 * rr_best)) {
                    lay = lay64;
                    fellback = 1;
                }
                while (lay != lay64 && lay < P.nlay - 1 && rel < P.level_rel[lay]) {
                    ++lay;
                    ++switches;
                }
            }
        }
        if (it >= maxit) break;
        ++it_lay[lay];
        if (!wait_deps(P, S, lay, ep)) return;
        EpiDot ev{rh, v, 0.0, vpol};
        bool ok;
        if (MIXED && lay != lay64) ok = cta_spmv<true>(P, lay, P.lay[lay].x32 ? (const void *)p32 : p, S, dyn, pp, ev);
        else ok = cta_spmv<false>(P, lay64, p, S, dyn, pp, ev);
        if (!ok) return;
        double a1[1] = {ev.dot}, b1[1];
        if (!grid_sum<1>(P, S, a1, b1, phase)) return;
        if (!(b1[0] != 0.0) || !isfinite(b1[0])) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rho / b1[0];
        MF_PAIRS(4, vlo, vhi, {
            double2 rv[_vb], vv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                vv[u] = ld2_hint(v + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 o;
                o.x = rv[u].x - alpha * vv[u].x;
                o.y = rv[u].y - alpha * vv[u].y;
                st2_hint(s + 2 * MF_PI(u), o, vpol);
                if (MIXED)
                    stf2_hint(s32 + 2 * MF_PI(u), make_float2(__double2float_rn(o.x), __double2float_rn(o.y)), vpol);
            }
        })
        ++ep;
        publish(P, ep);
        if (!wait_deps(P, S, lay, ep)) return;
        EpiDot2 et{s, t, 0.0, 0.0, vpol};
        if (MIXED && lay != lay64) ok = cta_spmv<true>(P, lay, P.lay[lay].x32 ? (const void *)s32 : s, S, dyn, pp, et);
        else ok = cta_spmv<false>(P, lay64, s, S, dyn, pp, et);
        if (!ok) return;
        double a2[2] = {et.ts, et.tt}, b2[2];
        if (!grid_sum<2>(P, S, a2, b2, phase)) return;
        if (!(b2[1] != 0.0) || !isfinite(b2[1])) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double omega = b2[0] / b2[1];
        double rrp = 0.0, rhp = 0.0;
        MF_PAIRS(2, vlo, vhi, {
            double2 sv[_vb], xv[_vb], pv[_vb], tv[_vb], hv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                sv[u] = ld2_hint(s + 2 * MF_PI(u), vpol);
                xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                pv[u] = ld2_hint(p + 2 * MF_PI(u), vpol);
                tv[u] = ld2_hint(t + 2 * MF_PI(u), vpol);
                hv[u] = ld2_hint(rh + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 xo, ro;
                xo.x = xv[u].x + alpha * pv[u].x + omega * sv[u].x;
                xo.y = xv[u].y + alpha * pv[u].y + omega * sv[u].y;
                st2_hint(x + 2 * MF_PI(u), xo, vpol);
                ro.x = sv[u].x - omega * tv[u].x;
                ro.y = sv[u].y - omega * tv[u].y;
                st2_hint(r + 2 * MF_PI(u), ro, vpol);
                rrp += ro.x * ro.x + ro.y * ro.y;
                rhp += ro.x * hv[u].x + ro.y * hv[u].y;
            }
        })
        double a3[2] = {rhp, rrp}, b3[2];
        if (!grid_sum<2>(P, S, a3, b3, phase)) return;
        const double rho1 = b3[0];
        rr = b3[1];
        ++it;
        rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        if (!isfinite(rr) || omega == 0.0) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const bool stop = !fixed && rel <= tol;
        if (stop && !(MIXED && P.true_check)) break;
        if (stop) pending = true;  // confirm with the FP64 true residual (p still advances)
        const double beta = (rho1 * alpha) / (rho * omega);
        MF_PAIRS(4, vlo, vhi, {
            double2 rv[_vb], pv[_vb], vv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                pv[u] = ld2_hint(p + 2 * MF_PI(u), vpol);
                vv[u] = ld2_hint(v + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                double2 o;
                o.x = rv[u].x + beta * (pv[u].x - omega * vv[u].x);
                o.y = rv[u].y + beta * (pv[u].y - omega * vv[u].y);
                st2_hint(p + 2 * MF_PI(u), o, vpol);
                if (MIXED)
                    stf2_hint(p32 + 2 * MF_PI(u), make_float2(__double2float_rn(o.x), __double2float_rn(o.y)), vpol);
            }
        })
        rho = rho1;
        ++ep;
        publish(P, ep);
    }
    }
    if (g == 0 && tid == 0) {
        if (status == MF_OK && !fixed && rel > tol) status = MF_ERR_NOT_CONVERGED;
        P.res->iterations = it;
        P.res->status = status;
        P.res->replacements = repl;
        P.res->level_switches = switches;
        P.res->rr = rr;
        P.res->bb = bb;
        P.res->final_layout = lay;
        for (int l = 0; l < KMAX_LAYOUTS; ++l) P.res->it_layout[l] = MIXED ? it_lay[l] : (l == 0 ? it : 0);
        P.res->pad = fellback;
    }
}

// ---------------------------------------------------------------- norms
__global__ void k_residual_norms(int n, const double *b, const double *ax, double *out) {
    // out[0] += sum (b - ax)^2, out[1] += sum b^2 (atomic, used for checks only)
    double s0 = 0.0, s1 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double e = b[i] - ax[i];
        s0 += e * e;
        s1 += b[i] * b[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, s0);
        atomicAdd(out + 1, s1);
    }
}

// ------------------------------------------------------------ batched CG
// The grid is split into groups of B.gs CTAs. Rank 0 of a group takes the
// next system from a device queue (largest first) and a group reduction
// hands it to the other ranks; the group then runs the FP64 CG recurrence of
// the single-system kernel on it with the system's gs-CTA slab layout:
// reductions and halo flags stay inside the group, so groups never wait for
// each other and many systems are in flight at once.
__global__ void __launch_bounds__(NTHREADS, 1) k_batch_cg(BatchParams B) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    __shared__ unsigned s_q;
    __shared__ int s_rng[4];
    KParams P0;  // only the fields kernel_setup reads
    P0.nlay = 0;
    P0.stage_stride = B.stage_stride;
    P0.slab_area = B.slab_area;
    kernel_setup(P0, S, 0);
    const int tid = threadIdx.x;
    const int grp = blockIdx.x / B.gs, rank = blockIdx.x % B.gs;
    const Ctx X{B.gsync + (size_t)grp * B.gsync_words, B.gpartial + (size_t)grp * 8 * B.gs, B.gs, rank,
                B.limit_ns};
    Pipe pp;
    uint32_t phase = 0, ep = 0;
    const uint64_t vpol = policy_evict_last();
    const PipeCfg C{B.stage_stride, B.slab_area, B.limit_ns, X.sync, 0};
    const bool fixed = B.fixed_iterations > 0;
    const int maxit = fixed ? B.fixed_iterations : B.maxiter;
    while (true) {
        if (rank == 0 && tid == 0) s_q = atomicAdd(B.queue, 1u);
        __syncthreads();
        double v0[1] = {(rank == 0 && tid == 0) ? (double)s_q : 0.0}, o0[1];
        if (!group_sum<1>(X, S, v0, o0, phase)) return;
        const unsigned qi = (unsigned)o0[0];
        if (qi >= (unsigned)B.count) break;
        const int sys = B.order[qi];
        const SysDesc D = B.sys[sys];
        const uint8_t *hsrc = D.head + (size_t)rank * STAGES * ISSUE_REC;
        for (int i = tid; i < STAGES * ISSUE_REC; i += NTHREADS) (&S.head[0][0][0])[i] = hsrc[i];
        if (tid == 0) {
            s_rng[0] = D.cta_slab[rank + 1] - D.cta_slab[rank];
            s_rng[1] = D.cta_rb[rank];
            s_rng[2] = D.cta_rb[rank + 1];
            s_rng[3] = 0;
            // the ring holds the previous system's slabs
            for (int k = 0; k < STAGES; ++k) S.res_tag[k] = 0;
        }
        __syncthreads();
        const int dep_lo = D.cta_dep[2 * rank], dep_hi = D.cta_dep[2 * rank + 1];
        SpmvSrc L;
        L.slabs = D.slabs;
        L.head = &S.head[0][0][0];
        L.ns = s_rng[0];
        L.kind = D.kind;
        L.site = 40;
        L.resident_ok = 1;  // within this system's solve
        L.x32 = 0;  // FP64 layouts
        L.gt = D.gt;
        const int vlo = s_rng[1] * 16, vhi = s_rng[2] * 16;
        __syncthreads();  // s_rng read by all before the next system overwrites it
        double *x = D.x, *r = D.r, *d = D.d, *q = D.q;
        const double *b = D.b;
        // r = b - A x0, d = r (x0 is written before the launch: no halo wait)
        EpiResidual er{b, r, 0.0, vpol};
        if (!cta_spmv_src<false, EpiResidual, 8>(L, C, x, S, dyn, pp, er)) return;
        double bbp = 0.0;
        MF_PAIRS(4, vlo, vhi, {
            double2 rv[_vb], bv[_vb];
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                bv[u] = ld2_hint(b + 2 * MF_PI(u), vpol);
            }
#pragma unroll
            MF_FOR_VB if (MF_LIVE(u, vhi)) {
                st2_hint(d + 2 * MF_PI(u), rv[u], vpol);
                bbp += bv[u].x * bv[u].x + bv[u].y * bv[u].y;
            }
        })
        double v2[2] = {er.rr, bbp}, o2[2];
        if (!group_sum<2>(X, S, v2, o2, phase)) return;
        publish_x(X, ++ep);
        double rr = o2[0];
        const double bb = o2[1];
        const double bnorm = sqrt(bb);
        double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        int it = 0, status = MF_OK;
        while (it < maxit && (fixed || rel > B.tol)) {
            if (!wait_deps_x(X, S, dep_lo, dep_hi, ep)) return;
            EpiQ eq{d, q, 0.0, vpol};
            if (!cta_spmv_src<false, EpiQ, 8>(L, C, d, S, dyn, pp, eq)) return;
            double v1[1] = {eq.dq}, o1[1];
            if (!group_sum<1>(X, S, v1, o1, phase)) return;
            const double dq = o1[0];
            if (!(dq != 0.0) || !isfinite(dq)) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
            const double alpha = rr / dq;
            double rrp = 0.0;
            MF_PAIRS(4, vlo, vhi, {
                double2 rv[_vb], qv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                    qv[u] = ld2_hint(q + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    double2 o;
                    o.x = rv[u].x - alpha * qv[u].x;
                    o.y = rv[u].y - alpha * qv[u].y;
                    st2_hint(r + 2 * MF_PI(u), o, vpol);
                    rrp += o.x * o.x + o.y * o.y;
                }
            })
            double w1[1] = {rrp}, u1[1];
            if (!group_sum<1>(X, S, w1, u1, phase)) return;
            const double rrn = u1[0];
            ++it;
            rel = bnorm > 0 ? sqrt(rrn) / bnorm : 0.0;
            const double beta = rrn / rr;
            const bool done = !fixed && rel <= B.tol;
            MF_PAIRS(4, vlo, vhi, {
                double2 dv[_vb], xv[_vb], rv[_vb];
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    dv[u] = ld2_hint(d + 2 * MF_PI(u), vpol);
                    xv[u] = ld2_hint(x + 2 * MF_PI(u), vpol);
                    rv[u] = ld2_hint(r + 2 * MF_PI(u), vpol);
                }
#pragma unroll
                MF_FOR_VB if (MF_LIVE(u, vhi)) {
                    double2 xo, dn;
                    xo.x = xv[u].x + alpha * dv[u].x;
                    xo.y = xv[u].y + alpha * dv[u].y;
                    st2_hint(x + 2 * MF_PI(u), xo, vpol);
                    if (!done) {
                        dn.x = rv[u].x + beta * dv[u].x;
                        dn.y = rv[u].y + beta * dv[u].y;
                        st2_hint(d + 2 * MF_PI(u), dn, vpol);
                    }
                }
            })
            rr = rrn;
            publish_x(X, ++ep);  // d complete before any rank's next SpMV stages it
            if (!isfinite(rrn)) {
                status = MF_ERR_BREAKDOWN;
                break;
            }
        }
        if (rank == 0 && tid == 0) {
            if (status == MF_OK && !fixed && rel > B.tol) status = MF_ERR_NOT_CONVERGED;
            BatchResult R;
            R.iterations = it;
            R.status = status;
            R.rr = rr;
            R.bb = bb;
            B.res[sys] = R;
        }
        __syncthreads();
    }
}

// ================================================================= host side
static int dyn_smem(int slab_max) { return STAGES * stage_stride_of(slab_max); }

int kernel_config(mf_tiles *t, int *G_out) {
    const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
    const int dyn = dyn_smem(slab_max);
    int optin = 0;
    MF_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, t->device));
    // static shared memory: Smem, plus the TMEM kernel's per-thread partials
    if (dyn + (int)sizeof(Smem) + NTHREADS * 8 + 64 > optin) {
        set_last_error("slab_bytes too large: the stage ring does not fit shared memory");
        return MF_ERR_ARG;
    }
    const void *kerns[] = {(const void *)k_cg<false>, (const void *)k_cg<true>, (const void *)k_bicgstab<false>,
                           (const void *)k_bicgstab<true>,
                           (const void *)k_spmv<false>, (const void *)k_spmv<true>, (const void *)k_cgcg,
                           (const void *)k_batch_cg, (const void *)k_cgcg_tm, (const void *)k_pcg,
                           (const void *)k_cg_tm, (const void *)k_pcg_tm};
    int occ_min = 1 << 30;
    for (const void *k : kerns) {
        MF_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
        int occ = 0;
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, NTHREADS, dyn));
        occ_min = occ < occ_min ? occ : occ_min;
    }
    if (occ_min < 1) {
        set_last_error("persistent kernel does not fit one SM");
        return MF_ERR_RESIDENCY;
    }
    int per_sm = t->opt.ctas_per_sm > 0 ? t->opt.ctas_per_sm : 1;
    if (per_sm > occ_min) per_sm = occ_min;
    *G_out = t->nsm * per_sm;
    return MF_OK;
}

static void fill_layout_args(LayoutArgs &a, const Layout &L) {
    a.kind = L.kind;
    a.x32 = L.x32 ? 1 : 0;
    a.slabs = L.slabs.p;
    a.head = L.head.p;
    a.cta_slab = L.cta_slab.p;
    a.cta_rb = L.cta_rb.p;
    a.cta_dep = L.cta_dep.p;
}

void base_params(mf_tiles *t, KParams &P) {
    std::memset(&P, 0, sizeof P);
    const int slab_max = t->L64.slab_max;
    P.stage_stride = stage_stride_of(slab_max);
    P.slab_area = slab_area_of(slab_max);
    P.rowA = t->rowA;
    P.tilem = t->tilem;
    P.tile_ptr = t->tile_ptr.p;
    P.tile_col = t->tile_col.p;
    P.tile_off = t->tile_off.p;
    P.csrptr_off = t->csrptr_off.p;
    P.ptr = t->ptr.p;
    P.val = t->val.p;
    P.col = t->col.p;
    const double lim = t->opt.timeout_s > 0 ? t->opt.timeout_s : 2.0;
    P.limit_ns = (uint64_t)(lim * 1e9);
    P.prefetch = t->opt.reserved[3] == 1 ? 1 : 0;
    fill_layout_args(P.lay[0], t->L64);
    P.nlay = 1;
}

__global__ void k_to_f32(int n, const double *__restrict__ src, float *__restrict__ dst, size_t npad) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npad; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = i < (size_t)n ? __double2float_rn(src[i]) : 0.0f;
}

int launch_to_f32(int n, const double *src, float *dst, size_t npad, cudaStream_t s) {
    size_t blocks = (npad + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    k_to_f32<<<(unsigned)blocks, 256, 0, s>>>(n, src, dst, npad);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

int launch_spmv(mf_tiles *t, int level, const void *x, double *y, int reps, cudaStream_t s) {
    KParams P;
    base_params(t, P);
    int lay = 0;
    bool mixed = false;
    if (level >= 0) {
        if (!t->mixed_ready || level >= MF_NLEVELS) return MF_ERR_ARG;
        fill_layout_args(P.lay[1], t->Lmix[level]);
        P.nlay = 2;
        lay = 1;
        mixed = true;
    }
    const int dyn = dyn_smem(t->L64.slab_max);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(t->G);
    cfg.blockDim = dim3(NTHREADS);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (mixed) MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_spmv<true>, P, x, y, lay, reps));
    else MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_spmv<false>, P, x, y, lay, reps));
    return MF_OK;
}

int launch_solver(mf_tiles *t, int kind, KParams &P, cudaStream_t s) {
    const int dyn = dyn_smem(t->L64.slab_max);
    void *args[] = {&P};
    const void *k = kind == 0   ? (P.nlay > 1 ? (const void *)k_cg<true> : (const void *)k_cg<false>)
                    : kind == 2 ? (const void *)k_cgcg
                    : kind == 3 ? (const void *)k_cgcg_tm
                    : kind == 4 ? (const void *)k_pcg
                    : kind == 5 ? (const void *)k_cg_tm
                    : kind == 6 ? (const void *)k_pcg_tm
                                : (P.nlay > 1 ? (const void *)k_bicgstab<true> : (const void *)k_bicgstab<false>);
    MF_CUDA_TRY(cudaLaunchCooperativeKernel(k, dim3(t->G), dim3(NTHREADS), args, dyn, s));
    return MF_OK;
}

int launch_batch(const BatchParams &B, int grid, cudaStream_t s) {
    // cooperative: the CTAs of a group wait on each other, so all must be
    // resident at once (the launch fails instead of deadlocking)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NTHREADS);
    cfg.dynamicSmemBytes = STAGES * (size_t)B.stage_stride;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch_cg, B));
    return MF_OK;
}

int launch_residual_norms(int n, const double *b, const double *ax, double *out, cudaStream_t s) {
    MF_CUDA_TRY(cudaMemsetAsync(out, 0, 2 * sizeof(double), s));
    int blocks = (n + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    k_residual_norms<<<blocks, 256, 0, s>>>(n, b, ax, out);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

}  // namespace mf
