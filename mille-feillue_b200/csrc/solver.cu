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
// instead of a fixed iteration count.
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
    uint64_t full[STAGES];
    uint32_t abort;
    uint32_t pad;
    int slab0[KMAX_LAYOUTS], slab1[KMAX_LAYOUTS];
    double red[NWARPS][4];
    double bres[4];
    uint8_t head[KMAX_LAYOUTS][STAGES][ISSUE_REC];
};

__device__ __forceinline__ uint8_t *stage_ptr(uint8_t *dyn, int k, int stride) { return dyn + (size_t)k * stride; }

__device__ void set_error(const KParams &P, uint32_t code, uint32_t site) {
    if (atomicCAS(P.sync + SYNC_ERROR, 0u, code) == 0u) atomicExch(P.sync + SYNC_SITE, site);
}

// Thread 0: issue the bulk copies of one slab (x runs first, slab last: the
// issue record may live inside the stage the slab overwrites).
__device__ void issue_slab(Smem &S, uint8_t *stage, int slab_area, int k, uint32_t off16, uint32_t bytes,
                           uint32_t xbytes, int nruns, const XRun *runs, const uint8_t *slabs,
                           const double *xv, uint64_t pol_m, uint64_t pol_v) {
    mbar_arrive_expect_tx(&S.full[k], bytes + xbytes);
    uint8_t *xarea = stage + slab_area;
    for (int q = 0; q < nruns; ++q) {
        const XRun r = runs[q];
        bulk_g2s(xarea + (size_t)r.slot0 * 128, xv + (size_t)r.seg0 * 16, (uint32_t)r.nseg * 128u, &S.full[k], pol_v);
    }
    bulk_g2s(stage, slabs + (size_t)off16 * 16, bytes, &S.full[k], pol_m);
}

__device__ bool wait_full(Smem &S, int k, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(&S.full[k], parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(&S.full[k], parity)) return true;
        if ((spin & 15u) == 0 && globaltimer() - t0 > limit_ns) return false;
    }
}

// Sum of one row over the tiles [t0, t1) of a staged / gather slab.
template <bool MIXED>
__device__ __forceinline__ double slab_row(const uint8_t *st, const SlabHeader &h, int j, int r, const double *xstage,
                                           const double *__restrict__ xg) {
    const SlabOffsets o = slab_offsets(h.nrb, h.ntiles, 0, 0);
    const RbDir *rbd = reinterpret_cast<const RbDir *>(st + o.rbdir);
    const uint32_t *slot = reinterpret_cast<const uint32_t *>(st + o.slot);
    const uint8_t *rowend = st + o.rowend;
    const uint8_t *vals = st + o.vals;
    const uint8_t *cols = st + (uint32_t)h.cols16 * 16u;
    const RbDir d0 = rbd[j], d1 = rbd[j + 1];
    uint32_t coff = d0.col0, voff = d0.val_off;
    const bool staged = h.mode == SLAB_STAGED;
    double acc = 0.0;
    for (int t = d0.tile0; t < d1.tile0; ++t) {
        const uint32_t sw = slot[t];
        const uint8_t *re = rowend + 16 * t;
        const int e15 = re[15];
        const int nk = e15 ? e15 : 256;
        const int s = r ? re[r - 1] : 0;
        const int e = r == 15 ? nk : re[r];
        const uint32_t idx = sw & 0x3fffffffu;
        const int prec = MIXED ? (int)(sw >> 30) : 0;
        const uint8_t *cb = cols + coff;
        if (prec == MF_PREC_FP64) {
            const double *vb = reinterpret_cast<const double *>(vals + voff);
            double sum = 0.0;
            if (staged) {
                const double *xs = xstage + idx * 16;
                for (int q = s; q < e; ++q) sum = dadd(sum, dmul(xs[cb[q]], vb[q]));
            } else {
                const double *xs = xg + (size_t)idx * 16;
                for (int q = s; q < e; ++q) sum = dadd(sum, dmul(__ldcg(xs + cb[q]), vb[q]));
            }
            acc = dadd(acc, sum);
            voff += 8u * nk;
        } else {
            const double *xs = staged ? xstage + idx * 16 : xg + (size_t)idx * 16;
            float sum = 0.0f;
            float scale = 1.0f;
            if (prec == MF_PREC_FP32) {
                const float *vb = reinterpret_cast<const float *>(vals + voff);
                for (int q = s; q < e; ++q) {
                    const double xv = staged ? xs[cb[q]] : __ldcg(xs + cb[q]);
                    sum = __fmaf_rn(__double2float_rn(xv), vb[q], sum);
                }
                voff += align8u(4u * nk);
            } else if (prec == MF_PREC_FP16) {
                scale = *reinterpret_cast<const float *>(vals + voff);
                const __half *vb = reinterpret_cast<const __half *>(vals + voff + 4);
                for (int q = s; q < e; ++q) {
                    const double xv = staged ? xs[cb[q]] : __ldcg(xs + cb[q]);
                    sum = __fmaf_rn(__double2float_rn(xv), __half2float(vb[q]), sum);
                }
                voff += align8u(4u + 2u * nk);
            } else {
                scale = *reinterpret_cast<const float *>(vals + voff);
                const uint8_t *vb = vals + voff + 4;
                for (int q = s; q < e; ++q) {
                    const double xv = staged ? xs[cb[q]] : __ldcg(xs + cb[q]);
                    const __half_raw hr = __nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)vb[q], __NV_E4M3);
                    sum = __fmaf_rn(__double2float_rn(xv), __half2float(__half(hr)), sum);
                }
                voff += align8u(4u + (uint32_t)nk);
            }
            acc = dadd(acc, dmul((double)sum, (double)scale));
        }
        coff += nk;
    }
    return acc;
}

// Row sum of an oversize row block straight from the global tile arrays.
__device__ double global_row(const KParams &P, int rb, int r, const double *__restrict__ xg) {
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
// For every row < rowA: v = epi.pre(row) is loaded before the row's tiles,
// then epi(row, acc, v) runs with the row sum. Returns false on abort.
template <bool MIXED, class Epi>
__device__ bool cta_spmv(const KParams &P, int lay, const double *xv, Smem &S, uint8_t *dyn, uint32_t &ph,
                         Epi &epi) {
    const int ns = S.slab1[lay] - S.slab0[lay];
    const int stride = P.stage_stride;
    const int slab_area = P.slab_area;
    const LayoutArgs &L = P.lay[lay];
    const int tid = threadIdx.x;
    const int w = tid >> 5, lane = tid & 31;
    const int half = lane >> 4, r = lane & 15;
    if (tid == 0) {
        const uint64_t pm = policy_evict_first(), pv = policy_evict_last();
        fence_proxy_async_global();
        for (int k = 0; k < STAGES && k < ns; ++k) {
            const uint32_t *rec = reinterpret_cast<const uint32_t *>(S.head[lay][k]);
            issue_slab(S, stage_ptr(dyn, k, stride), slab_area, k, rec[0], rec[1], rec[2], (int)rec[3],
                       reinterpret_cast<const XRun *>(rec + 4), L.slabs, xv, pm, pv);
        }
    }
    for (int i = 0; i < ns; ++i) {
        const int k = i % STAGES;
        uint8_t *st = stage_ptr(dyn, k, stride);
        if (!wait_full(S, k, (ph >> k) & 1u, P.limit_ns)) {
            set_error(P, (uint32_t)MF_ERR_TIMEOUT, 100 + lay);
            return false;
        }
        ph ^= 1u << k;
        const SlabHeader h = *reinterpret_cast<const SlabHeader *>(st);
        if (h.mode == SLAB_OVERSIZE) {
            if (w == 0 && half == 0) {
                const int row = h.rb0 * 16 + r;
                const double pv = row < P.rowA ? epi.pre(row) : 0.0;
                const double acc = global_row(P, h.rb0, r, xv);
                if (row < P.rowA) epi(row, acc, pv);
            }
        } else {
            for (int j = 2 * w + half; j < h.nrb; j += 2 * NWARPS) {
                const int row = (h.rb0 + j) * 16 + r;
                const bool live = row < P.rowA;
                const double pv = live ? epi.pre(row) : 0.0;
                const double acc =
                    slab_row<MIXED>(st, h, j, r, reinterpret_cast<const double *>(st + slab_area), xv);
                if (live) epi(row, acc, pv);
            }
        }
        __syncthreads();
        if (tid == 0 && h.next_bytes != 0u) {
            const uint64_t pm = policy_evict_first(), pv = policy_evict_last();
            fence_proxy_async_smem();
            issue_slab(S, st, slab_area, k, h.next_off16, h.next_bytes, h.next_xbytes, h.next_nruns,
                       reinterpret_cast<const XRun *>(st + 32), L.slabs, xv, pm, pv);
        }
    }
    return true;
}

// Block reduction of NV partials in a fixed order, then the grid-wide sum.
template <int NV>
__device__ bool grid_sum(const KParams &P, Smem &S, const double (&v)[NV], double (&out)[NV], uint32_t &phase) {
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
    const int G = gridDim.x;
    const int slot = phase & 1;
    if (tid == 0) {
        double p[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            p[k] = 0.0;
            for (int q = 0; q < NWARPS; ++q) p[k] += S.red[q][k];
            P.partial[((size_t)slot * G + blockIdx.x) * 4 + k] = p[k];
        }
        red_release_add(P.sync + SYNC_ARRIVE, 1u);
        const uint32_t target = (phase + 1) * (uint32_t)G;
        if (ld_acquire(P.sync + SYNC_ARRIVE) < target) {
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(P.sync + SYNC_ARRIVE) >= target) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(P.sync + SYNC_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > P.limit_ns) {
                        set_error(P, (uint32_t)MF_ERR_TIMEOUT, 10);
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
            for (int k = 0; k < NV; ++k) a[k] += __ldcg(&P.partial[((size_t)slot * G + c) * 4 + k]);
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

// Publish this CTA's rows of the halo vectors under epoch `ep`.
__device__ void publish(const KParams &P, uint32_t ep) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        fence_proxy_async_global();
        st_release(P.sync + SYNC_FLAGS + blockIdx.x * FLAG_STRIDE, ep);
    }
}

// Wait until every CTA whose rows this CTA reads has published epoch `ep`.
__device__ bool wait_deps(const KParams &P, Smem &S, int lay, uint32_t ep) {
    const int lo = P.lay[lay].cta_dep[2 * blockIdx.x], hi = P.lay[lay].cta_dep[2 * blockIdx.x + 1];
    if (threadIdx.x < 32) {
        for (int c = lo + (int)threadIdx.x; c <= hi; c += 32) {
            const uint32_t *f = P.sync + SYNC_FLAGS + c * FLAG_STRIDE;
            if (ld_acquire(f) >= ep) continue;
            const uint64_t t0 = globaltimer();
            for (uint32_t spin = 1;; ++spin) {
                if (ld_acquire(f) >= ep) break;
                if ((spin & 63u) == 0) {
                    if (ld_relaxed(P.sync + SYNC_ERROR) != 0u) {
                        S.abort = 1;
                        break;
                    }
                    if (globaltimer() - t0 > P.limit_ns) {
                        set_error(P, (uint32_t)MF_ERR_TIMEOUT, 20);
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

__device__ void kernel_setup(const KParams &P, Smem &S, int nlay) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int k = 0; k < STAGES; ++k) mbar_init(&S.full[k], 1);
        mbar_fence_init();
        S.abort = 0;
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

// ------------------------------------------------------------------ SpMV
struct EpiStore {
    double *y;
    __device__ double pre(int) const { return 0.0; }
    __device__ void operator()(int row, double acc, double) const { y[row] = acc; }
};

template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1) k_spmv(KParams P, const double *x, double *y, int lay, int reps) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, lay + 1);
    uint32_t ph = 0;
    EpiStore epi{y};
    for (int it = 0; it < reps; ++it) {
        if (!cta_spmv<MIXED>(P, lay, x, S, dyn, ph, epi)) return;
    }
}

// -------------------------------------------------------------------- CG
struct EpiResidual {  // r = b - A x, rr += r*r
    const double *b;
    double *r;
    double rr;
    __device__ double pre(int row) const { return __ldcg(b + row); }
    __device__ void operator()(int row, double acc, double bv) {
        const double v = bv - acc;
        r[row] = v;
        rr += v * v;
    }
};
struct EpiQ {  // q = A d, dq += d*q
    const double *d;
    double *q;
    double dq;
    __device__ double pre(int row) const { return __ldcg(d + row); }
    __device__ void operator()(int row, double acc, double dv) {
        q[row] = acc;
        dq += dv * acc;
    }
};

template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1) k_cg(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, P.nlay);
    const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x;
    uint32_t ph = 0, phase = 0;
    const int lay64 = 0;
    int lay = P.start_layout;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int row_lo = rb_lo * 16, row_hi = min(rb_hi * 16, P.rowA);
    double *x = P.x, *r = P.r, *d = P.d, *q = P.q;
    const double *b = P.b;
    if (P.inject_wait) {
        // test hook: a dependency epoch no CTA ever publishes; the bounded
        // wait must end the solve with MF_ERR_TIMEOUT
        if (!wait_deps(P, S, 0, 0xffffffffu)) return;
    }
    // r = b - A x0, d = r; (rr, bb)
    EpiResidual er{b, r, 0.0};
    if (!cta_spmv<false>(P, lay64, x, S, dyn, ph, er)) return;
    __syncthreads();
    double bbp = 0.0;
    for (int i = row_lo + tid; i < row_hi; i += NTHREADS) {
        d[i] = r[i];
        bbp += b[i] * b[i];
    }
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
    while (it < maxit && (fixed || rel > tol)) {
        // periodic true-residual replacement r = b - A x (FP64 layout)
        if (P.replace_every > 0 && it > 0 && it % P.replace_every == 0) {
            if (!wait_deps(P, S, lay64, ep)) return;
            EpiResidual e2{b, r, 0.0};
            if (!cta_spmv<false>(P, lay64, x, S, dyn, ph, e2)) return;
            double v1[1] = {e2.rr}, o1[1];
            if (!grid_sum<1>(P, S, v1, o1, phase)) return;
            rr = o1[0];
            ++repl;
            // tighten the precision level as the true residual falls
            if (MIXED) {
                const double relt = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
                while (lay < P.nlay - 1 && relt < P.level_rel[lay]) {
                    ++lay;
                    ++switches;
                }
            }
        }
        if (!wait_deps(P, S, lay, ep)) return;
        EpiQ eq{d, q, 0.0};
        bool ok;
        if (MIXED && lay != lay64) ok = cta_spmv<true>(P, lay, d, S, dyn, ph, eq);
        else ok = cta_spmv<false>(P, lay64, d, S, dyn, ph, eq);
        if (!ok) return;
        double v1[1] = {eq.dq}, o1[1];
        if (!grid_sum<1>(P, S, v1, o1, phase)) return;
        const double dq = o1[0];
        if (!(dq != 0.0) || !isfinite(dq)) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rr / dq;
        double rrp = 0.0;
        for (int i = row_lo + tid; i < row_hi; i += NTHREADS) {
            const double ri = r[i] - alpha * q[i];
            r[i] = ri;
            rrp += ri * ri;
        }
        double w1[1] = {rrp}, u1[1];
        if (!grid_sum<1>(P, S, w1, u1, phase)) return;
        const double rrn = u1[0];
        ++it;
        rel = bnorm > 0 ? sqrt(rrn) / bnorm : 0.0;
        const double beta = rrn / rr;
        const bool done = !fixed && rel <= tol;
        for (int i = row_lo + tid; i < row_hi; i += NTHREADS) {
            const double di = d[i];
            x[i] += alpha * di;
            if (!done) d[i] = r[i] + beta * di;
        }
        rr = rrn;
        ++ep;
        publish(P, ep);
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
    }
    (void)G;
}

// -------------------------------------------------------------- BiCGSTAB
struct EpiDot {  // y = A p, dot += z*y
    const double *z;
    double *y;
    double dot;
    __device__ double pre(int row) const { return __ldcg(z + row); }
    __device__ void operator()(int row, double acc, double zv) {
        y[row] = acc;
        dot += zv * acc;
    }
};
struct EpiDot2 {  // t = A s, ts += t*s, tt += t*t
    const double *s;
    double *t;
    double ts, tt;
    __device__ double pre(int row) const { return __ldcg(s + row); }
    __device__ void operator()(int row, double acc, double sv) {
        t[row] = acc;
        ts += acc * sv;
        tt += acc * acc;
    }
};

__global__ void __launch_bounds__(NTHREADS, 1) k_bicgstab(KParams P) {
    extern __shared__ __align__(128) uint8_t dyn[];
    __shared__ Smem S;
    kernel_setup(P, S, 1);
    const int g = blockIdx.x, tid = threadIdx.x;
    uint32_t ph = 0, phase = 0;
    const int rb_lo = P.lay[0].cta_rb[g], rb_hi = P.lay[0].cta_rb[g + 1];
    const int row_lo = rb_lo * 16, row_hi = min(rb_hi * 16, P.rowA);
    double *x = P.x, *r = P.r, *p = P.d, *v = P.q, *s = P.s, *t = P.t, *rh = P.rh;
    const double *b = P.b;
    EpiResidual er{b, r, 0.0};
    if (!cta_spmv<false>(P, 0, x, S, dyn, ph, er)) return;
    __syncthreads();
    double bbp = 0.0, rhop = 0.0;
    for (int i = row_lo + tid; i < row_hi; i += NTHREADS) {
        const double ri = r[i];
        rh[i] = ri;
        p[i] = ri;
        bbp += b[i] * b[i];
        rhop += ri * ri;
    }
    double v3[3] = {er.rr, bbp, rhop}, o3[3];
    if (!grid_sum<3>(P, S, v3, o3, phase)) return;
    double rr = o3[0];
    const double bb = o3[1];
    double rho = o3[2];
    const double bnorm = sqrt(bb);
    const double tol = P.tol;
    uint32_t ep = 1;
    publish(P, ep);
    int it = 0, status = MF_OK;
    double rel = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
    const bool fixed = P.fixed_iterations > 0;
    const int maxit = fixed ? P.fixed_iterations : P.maxiter;
    while (it < maxit && (fixed || rel > tol)) {
        if (!wait_deps(P, S, 0, ep)) return;
        EpiDot ev{rh, v, 0.0};
        if (!cta_spmv<false>(P, 0, p, S, dyn, ph, ev)) return;
        double a1[1] = {ev.dot}, b1[1];
        if (!grid_sum<1>(P, S, a1, b1, phase)) return;
        if (!(b1[0] != 0.0) || !isfinite(b1[0])) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rho / b1[0];
        for (int i = row_lo + tid; i < row_hi; i += NTHREADS) s[i] = r[i] - alpha * v[i];
        ++ep;
        publish(P, ep);
        if (!wait_deps(P, S, 0, ep)) return;
        EpiDot2 et{s, t, 0.0, 0.0};
        if (!cta_spmv<false>(P, 0, s, S, dyn, ph, et)) return;
        double a2[2] = {et.ts, et.tt}, b2[2];
        if (!grid_sum<2>(P, S, a2, b2, phase)) return;
        if (!(b2[1] != 0.0) || !isfinite(b2[1])) {
            status = MF_ERR_BREAKDOWN;
            break;
        }
        const double omega = b2[0] / b2[1];
        double rrp = 0.0, rhp = 0.0;
        for (int i = row_lo + tid; i < row_hi; i += NTHREADS) {
            const double si = s[i];
            x[i] = x[i] + alpha * p[i] + omega * si;
            const double ri = si - omega * t[i];
            r[i] = ri;
            rrp += ri * ri;
            rhp += ri * rh[i];
        }
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
        if (!fixed && rel <= tol) break;
        const double beta = (rho1 * alpha) / (rho * omega);
        for (int i = row_lo + tid; i < row_hi; i += NTHREADS) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        rho = rho1;
        ++ep;
        publish(P, ep);
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

// ================================================================= host side
static int dyn_smem(int slab_max) { return STAGES * stage_stride_of(slab_max); }

int kernel_config(mf_tiles *t, int *G_out) {
    const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
    const int dyn = dyn_smem(slab_max);
    const void *kerns[] = {(const void *)k_cg<false>, (const void *)k_cg<true>, (const void *)k_bicgstab,
                           (const void *)k_spmv<false>, (const void *)k_spmv<true>};
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
    fill_layout_args(P.lay[0], t->L64);
    P.nlay = 1;
}

int launch_spmv(mf_tiles *t, int level, const double *x, double *y, int reps, cudaStream_t s) {
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
    if (mixed)
        k_spmv<true><<<t->G, NTHREADS, dyn, s>>>(P, x, y, lay, reps);
    else
        k_spmv<false><<<t->G, NTHREADS, dyn, s>>>(P, x, y, lay, reps);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

int launch_solver(mf_tiles *t, int kind, KParams &P, cudaStream_t s) {
    const int dyn = dyn_smem(t->L64.slab_max);
    void *args[] = {&P};
    const void *k = kind == 0 ? (P.nlay > 1 ? (const void *)k_cg<true> : (const void *)k_cg<false>)
                              : (const void *)k_bicgstab;
    MF_CUDA_TRY(cudaLaunchCooperativeKernel(k, dim3(t->G), dim3(NTHREADS), args, dyn, s));
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
