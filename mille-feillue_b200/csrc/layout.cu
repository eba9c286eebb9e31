// Slab layout of the persistent solver.
//
// The row blocks are split into G contiguous CTA ranges of equal cost (slab
// bytes + per-row vector work), and each range into slabs: consecutive row
// blocks whose encoded bytes fit one shared-memory stage and whose distinct
// x segments (16-entry pieces of the input vector) fit the x stage as at
// most MAXRUNS contiguous runs. The planner runs on the host over the tile
// column indices; the slab bytes themselves are written on the GPU from the
// encoder's tile arrays.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "tiles.h"

namespace mf {

namespace {

struct SlabPlan {
    int rb0, nrb, ntiles, t0, nnz, mode;
    uint32_t valbytes, bytes, off16;
    int seg_off, nseg;  // unique sorted x segments (staged mode)
    int run_off, nruns;
};

constexpr int FILL_THREADS = 256;

// Device: one CTA writes one slab.
__global__ void __launch_bounds__(FILL_THREADS) fill_slabs(
    const SlabPlan *__restrict__ plans, const int *__restrict__ slab_cta, const int *__restrict__ cta_slab,
    const int *__restrict__ segs, const XRun *__restrict__ runs, const int *__restrict__ tile_ptr,
    const int *__restrict__ tile_col, const int *__restrict__ tile_off, const int *__restrict__ csrptr_off,
    const unsigned char *__restrict__ bptr, const double *__restrict__ val, const unsigned char *__restrict__ col,
    const unsigned char *__restrict__ prec, float *__restrict__ scale_out, int tilem, int rowA, uint8_t *slabs) {
    __shared__ uint32_t s_voff[MAXT + 1];
    __shared__ uint32_t s_coff[MAXT + 1];
    __shared__ int sh[FILL_THREADS / 32];
    const int s = blockIdx.x;
    const SlabPlan P = plans[s];
    uint8_t *base = slabs + (size_t)P.off16 * 16;
    const SlabOffsets o = slab_offsets(P.nrb, P.ntiles, P.valbytes, P.nnz);
    // zero the slab (padding bytes deterministic)
    for (uint32_t i = threadIdx.x * 16; i < P.bytes; i += FILL_THREADS * 16)
        *reinterpret_cast<uint4 *>(base + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
        SlabHeader h;
        memset(&h, 0, sizeof h);
        h.rb0 = P.rb0;
        h.nrb = (uint16_t)P.nrb;
        h.ntiles = (uint16_t)P.ntiles;
        h.nxseg = (uint16_t)P.nseg;
        h.mode = (uint16_t)P.mode;
        h.bytes = P.bytes;
        h.cols16 = (uint16_t)(o.cols / 16);
        const int g = slab_cta[s];
        const int nx = s + STAGES;
        if (nx < cta_slab[g + 1]) {
            const SlabPlan Q = plans[nx];
            h.next_off16 = Q.off16;
            h.next_bytes = Q.bytes;
            h.next_xbytes = Q.mode == SLAB_STAGED ? (uint32_t)Q.nseg * 128u : 0u;
            h.next_nruns = Q.mode == SLAB_STAGED ? (uint16_t)Q.nruns : 0;
            XRun *dst = reinterpret_cast<XRun *>(base + o.runs);
            for (int k = 0; k < h.next_nruns; ++k) dst[k] = runs[Q.run_off + k];
        }
        *reinterpret_cast<SlabHeader *>(base) = h;
    }
    if (P.mode == SLAB_OVERSIZE) return;
    // per-tile value / column offsets (block scan over the slab's tiles)
    const int nt = P.ntiles;
    const int per = (nt + FILL_THREADS - 1) / FILL_THREADS;
    uint32_t vsum = 0, csum = 0;
    for (int k = 0; k < per; ++k) {
        const int j = threadIdx.x * per + k;
        if (j < nt) {
            const int t = P.t0 + j;
            const int nk = tile_off[t + 1] - tile_off[t];
            vsum += tile_val_bytes(prec[t], nk);
            csum += (uint32_t)nk;
        }
    }
    // exclusive block scan of (vsum, csum): both fit 32 bits; do two scans
    for (int pass = 0; pass < 2; ++pass) {
        uint32_t v = pass == 0 ? vsum : csum;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        uint32_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) sh[w] = (int)x;
        __syncthreads();
        uint32_t wb = 0;
        for (int q = 0; q < w; ++q) wb += (uint32_t)sh[q];
        uint32_t ex = wb + x - v;
        __syncthreads();
        uint32_t *dst = pass == 0 ? s_voff : s_coff;
        for (int k = 0; k < per; ++k) {
            const int j = threadIdx.x * per + k;
            if (j < nt) {
                dst[j] = ex;
                const int t = P.t0 + j;
                const int nk = tile_off[t + 1] - tile_off[t];
                ex += pass == 0 ? tile_val_bytes(prec[t], nk) : (uint32_t)nk;
            }
        }
        if (threadIdx.x == FILL_THREADS - 1) dst[nt] = ex;
        __syncthreads();
    }
    // row-block directory
    RbDir *rbd = reinterpret_cast<RbDir *>(base + o.rbdir);
    for (int j = threadIdx.x; j <= P.nrb; j += FILL_THREADS) {
        const int tj = (j < P.nrb ? tile_ptr[P.rb0 + j] : tile_ptr[P.rb0 + P.nrb]) - P.t0;
        RbDir d;
        d.tile0 = (uint16_t)tj;
        d.val_off = s_voff[tj];
        d.col0 = (uint16_t)s_coff[tj];
        rbd[j] = d;
    }
    uint32_t *slot = reinterpret_cast<uint32_t *>(base + o.slot);
    uint8_t *rowend = base + o.rowend;
    uint8_t *vals = base + o.vals;
    uint8_t *cols = base + o.cols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // one warp per tile
    for (int j = warp; j < nt; j += FILL_THREADS / 32) {
        const int t = P.t0 + j;
        const int p = prec[t];
        const int vo = tile_off[t];
        const int nk = tile_off[t + 1] - vo;
        // row block of tile t and its row length
        int lo = P.rb0, hi = P.rb0 + P.nrb - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_ptr[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const int rl = lo == tilem - 1 ? rowA - (tilem - 1) * 16 : 16;
        if (lane == 0) {
            uint32_t sv;
            if (P.mode == SLAB_STAGED) {
                // slot = position of the tile column in the sorted unique list
                const int c = tile_col[t];
                int a = 0, b = P.nseg - 1;
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    if (segs[P.seg_off + mid] < c) a = mid + 1; else b = mid;
                }
                sv = (uint32_t)a;
            } else {
                sv = (uint32_t)tile_col[t];
            }
            slot[j] = sv | ((uint32_t)p << 30);
        }
        if (lane < 16) {
            const int r = lane;
            const int cc = csrptr_off[t];
            int e;
            if (r + 1 < rl) e = bptr[cc + r + 1];
            else e = nk;
            rowend[16 * j + r] = (uint8_t)(e & 255);
        }
        // values: maximum magnitude for the scale of FP16 / FP8 tiles
        double mx = 0.0;
        for (int k = lane; k < nk; k += 32) mx = fmax(mx, fabs(val[vo + k]));
        for (int d = 16; d > 0; d >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        double scale = 1.0;
        if (p >= MF_PREC_FP16 && mx > 0.0) {
            int e;
            frexp(mx, &e);
            if (p == MF_PREC_FP16) {
                scale = ldexp(1.0, e - 15);
            } else {
                const double ratio = mx / 448.0;
                int k2;
                frexp(ratio, &k2);
                if (ldexp(1.0, k2 - 1) == ratio) k2 -= 1;
                scale = ldexp(1.0, k2);
            }
        }
        if (lane == 0) scale_out[t] = (float)scale;
        uint8_t *vb = vals + s_voff[j];
        const double inv = 1.0 / scale;  // exact: power of two
        if (p == MF_PREC_FP64) {
            for (int k = lane; k < nk; k += 32) reinterpret_cast<double *>(vb)[k] = val[vo + k];
        } else if (p == MF_PREC_FP32) {
            for (int k = lane; k < nk; k += 32) reinterpret_cast<float *>(vb)[k] = __double2float_rn(val[vo + k]);
        } else if (p == MF_PREC_FP16) {
            if (lane == 0) *reinterpret_cast<float *>(vb) = (float)scale;
            for (int k = lane; k < nk; k += 32)
                reinterpret_cast<__half *>(vb + 4)[k] = __double2half(val[vo + k] * inv);
        } else {
            if (lane == 0) *reinterpret_cast<float *>(vb) = (float)scale;
            for (int k = lane; k < nk; k += 32)
                vb[4 + k] = (uint8_t)__nv_cvt_double_to_fp8(val[vo + k] * inv, __NV_SATFINITE, __NV_E4M3);
        }
        for (int k = lane; k < nk; k += 32) cols[s_coff[j] + k] = col[vo + k];
    }
}

}  // namespace

int build_layout(mf_tiles *t, Layout &L, const std::vector<uint8_t> &prec_in, cudaStream_t st) {
    auto t_start = std::chrono::steady_clock::now();
    const int tilem = t->tilem, tilenum = t->tilenum;
    const int G = t->G;
    const int slab_max = t->opt.slab_bytes > 0 ? t->opt.slab_bytes : SLAB_MAX_DEFAULT;
    const int rbps = t->opt.rb_per_slab > 0 ? std::min(t->opt.rb_per_slab, RB_PER_SLAB_MAX) : RB_PER_SLAB_MAX;
    const auto &tp = t->h_tile_ptr;
    const auto &tc = t->h_tile_col;
    const auto &tn = t->h_tile_nnz;
    std::vector<uint8_t> prec(prec_in);
    if ((int)prec.size() != tilenum) prec.assign(tilenum, MF_PREC_FP64);

    // per row block: encoded bytes (without the slab header) and cost
    std::vector<uint32_t> rbbytes(tilem);
    std::vector<double> pref(tilem + 1, 0.0);
    for (int rb = 0; rb < tilem; ++rb) {
        uint64_t b = 8;
        for (int k = tp[rb]; k < tp[rb + 1]; ++k) b += 4 + 16 + tile_val_bytes(prec[k], tn[k]) + tn[k];
        rbbytes[rb] = (uint32_t)std::min<uint64_t>(b, 0xffffffffu);
        pref[rb + 1] = pref[rb] + (double)b + 16.0 * 72.0;
    }
    // CTA ranges of equal cost, computed once per matrix and shared by every
    // layout so that all layouts give each CTA the same rows
    if ((int)t->h_cta_rb.size() != G + 1) {
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
    // slabs
    std::vector<SlabPlan> plans;
    std::vector<int> seg_all;
    std::vector<XRun> run_all;
    std::vector<int> slab_cta;
    std::vector<int> cta_slab(G + 1, 0);
    std::vector<int> cur, merged, rbsegs;
    auto count_runs = [](const std::vector<int> &v) {
        int r = 0;
        for (size_t i = 0; i < v.size(); ++i)
            if (i == 0 || v[i] != v[i - 1] + 1) ++r;
        return r;
    };
    int n_gather = 0, n_over = 0;
    for (int g = 0; g < G; ++g) {
        cta_slab[g] = (int)plans.size();
        int rb = cta_rb[g];
        while (rb < cta_rb[g + 1]) {
            SlabPlan P{};
            P.rb0 = rb;
            P.t0 = tp[rb];
            cur.clear();
            // first row block decides the mode
            const int ntl = tp[rb + 1] - tp[rb];
            int nnz0 = 0;
            uint32_t vb0 = 0;
            for (int k = tp[rb]; k < tp[rb + 1]; ++k) {
                nnz0 += tn[k];
                vb0 += tile_val_bytes(prec[k], tn[k]);
            }
            const uint32_t tot0 = slab_offsets(1, ntl, vb0, nnz0).total;
            rbsegs.assign(tc.begin() + tp[rb], tc.begin() + tp[rb + 1]);  // ascending already
            if (tot0 > (uint32_t)slab_max || ntl > MAXT) {
                P.mode = SLAB_OVERSIZE;
                P.nrb = 1;
                P.ntiles = 0;
                P.nnz = 0;
                P.valbytes = 0;
                P.bytes = slab_offsets(1, 0, 0, 0).total;
                for (int k = tp[rb]; k < tp[rb + 1]; ++k) prec[k] = MF_PREC_FP64;
                ++n_over;
                rb += 1;
            } else {
                const bool staged = (int)rbsegs.size() <= XSEG_MAX && count_runs(rbsegs) <= MAXRUNS;
                P.mode = staged ? SLAB_STAGED : SLAB_GATHER;
                if (staged) cur = rbsegs;
                P.nrb = 1;
                P.ntiles = ntl;
                P.nnz = nnz0;
                P.valbytes = vb0;
                int nx = rb + 1;
                while (nx < cta_rb[g + 1] && P.nrb < rbps) {
                    const int ntx = tp[nx + 1] - tp[nx];
                    int nnzx = 0;
                    uint32_t vbx = 0;
                    for (int k = tp[nx]; k < tp[nx + 1]; ++k) {
                        nnzx += tn[k];
                        vbx += tile_val_bytes(prec[k], tn[k]);
                    }
                    if (P.ntiles + ntx > MAXT) break;
                    const uint32_t tot = slab_offsets(P.nrb + 1, P.ntiles + ntx, P.valbytes + vbx, P.nnz + nnzx).total;
                    if (tot > (uint32_t)slab_max) break;
                    if (staged) {
                        merged.clear();
                        std::set_union(cur.begin(), cur.end(), tc.begin() + tp[nx], tc.begin() + tp[nx + 1],
                                       std::back_inserter(merged));
                        if ((int)merged.size() > XSEG_MAX || count_runs(merged) > MAXRUNS) break;
                        cur.swap(merged);
                    }
                    P.nrb += 1;
                    P.ntiles += ntx;
                    P.nnz += nnzx;
                    P.valbytes += vbx;
                    ++nx;
                }
                P.bytes = slab_offsets(P.nrb, P.ntiles, P.valbytes, P.nnz).total;
                if (!staged) ++n_gather;
                rb = nx;
            }
            if (P.mode == SLAB_STAGED) {
                P.seg_off = (int)seg_all.size();
                P.nseg = (int)cur.size();
                seg_all.insert(seg_all.end(), cur.begin(), cur.end());
                P.run_off = (int)run_all.size();
                for (size_t i = 0; i < cur.size(); ++i) {
                    if (i == 0 || cur[i] != cur[i - 1] + 1) run_all.push_back(XRun{cur[i], 0, (uint16_t)i});
                    run_all.back().nseg++;
                }
                P.nruns = (int)run_all.size() - P.run_off;
            }
            plans.push_back(P);
            slab_cta.push_back(g);
        }
    }
    cta_slab[G] = (int)plans.size();
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
            rec[2] = P.mode == SLAB_STAGED ? (uint32_t)P.nseg * 128u : 0u;
            rec[3] = P.mode == SLAB_STAGED ? (uint32_t)P.nruns : 0u;
            if (P.mode == SLAB_STAGED)
                std::memcpy(&rec[4], &run_all[P.run_off], sizeof(XRun) * P.nruns);
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
    // algorithmic bytes and precision fractions
    double alg = 16.0 * (double)t->rowA;
    double cnt[4] = {0, 0, 0, 0};
    for (int k = 0; k < tilenum; ++k) {
        alg += tile_alg_bytes(prec[k], tn[k]);
        cnt[prec[k]] += 1;
    }
    // upload
    DevArray<SlabPlan> d_plans;
    DevArray<int> d_slab_cta, d_segs;
    DevArray<XRun> d_runs;
    if (L.slabs.alloc(off + 16) || L.head.alloc(head.size()) || L.cta_slab.alloc(G + 1) ||
        L.cta_rb.alloc(G + 1) || L.cta_dep.alloc(2 * G) || L.prec_dev.alloc(tilenum) ||
        L.scale_dev.alloc(tilenum) || d_plans.alloc(ns) || d_slab_cta.alloc(ns) ||
        d_segs.alloc(seg_all.size()) || d_runs.alloc(run_all.size()))
        return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemcpyAsync(L.head.p, head.data(), head.size(), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_slab.p, cta_slab.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_rb.p, cta_rb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemcpyAsync(L.cta_dep.p, dep.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
    if (tilenum > 0)
        MF_CUDA_TRY(cudaMemcpyAsync(L.prec_dev.p, prec.data(), tilenum, cudaMemcpyHostToDevice, st));
    MF_CUDA_TRY(cudaMemsetAsync(L.scale_dev.p, 0, sizeof(float) * std::max(tilenum, 1), st));
    if (ns > 0) {
        MF_CUDA_TRY(cudaMemcpyAsync(d_plans.p, plans.data(), sizeof(SlabPlan) * ns, cudaMemcpyHostToDevice, st));
        MF_CUDA_TRY(cudaMemcpyAsync(d_slab_cta.p, slab_cta.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    }
    if (!seg_all.empty())
        MF_CUDA_TRY(cudaMemcpyAsync(d_segs.p, seg_all.data(), sizeof(int) * seg_all.size(), cudaMemcpyHostToDevice, st));
    if (!run_all.empty())
        MF_CUDA_TRY(cudaMemcpyAsync(d_runs.p, run_all.data(), sizeof(XRun) * run_all.size(), cudaMemcpyHostToDevice, st));
    if (ns > 0)
        fill_slabs<<<ns, FILL_THREADS, 0, st>>>(d_plans.p, d_slab_cta.p, L.cta_slab.p, d_segs.p, d_runs.p,
                                               t->tile_ptr.p, t->tile_col.p, t->tile_off.p, t->csrptr_off.p,
                                               t->ptr.p, t->val.p, t->col.p, L.prec_dev.p, L.scale_dev.p, tilem,
                                               t->rowA, L.slabs.p);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaStreamSynchronize(st));
    L.prec.swap(prec);
    L.G = G;
    L.nslabs = ns;
    L.n_gather = n_gather;
    L.n_oversize = n_over;
    L.slab_max = slab_max;
    L.rb_per_slab = rbps;
    L.bytes = off;
    L.alg_bytes = alg;
    for (int p = 0; p < 4; ++p) L.tile_frac[p] = tilenum > 0 ? cnt[p] / tilenum : 0.0;
    L.built = true;
    t->layout_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return MF_OK;
}

}  // namespace mf
