// Per-tile precision selection for the mixed-precision layouts.
//
// Features (one warp per tile, from the encoder's tile arrays and the
// diagonal): f0 = log10 of the tile's scaled magnitude
// m_t = max |a_ij| / sqrt(|a_ii a_jj|), f1 = log10 of the tile's dynamic
// range max|a| / min|a|, f2 = nnz / 256, f3 = 1 for a diagonal tile,
// f4 = log10 max|a| relative to the matrix maximum, f5 = log10 of the
// relative residual at which the precision is used (filled per level).
//
// Magnitude rule: at level l with tolerance tau_l a tile takes the lowest of
// FP8, FP16, FP32 whose unit roundoff u_p satisfies u_p * m_t <= tau_l and
// whose range holds the tile (FP8 also needs a dynamic range <= 2^12);
// diagonal tiles never go below FP32; otherwise FP64. The levels tighten as
// the true residual falls (the solver switches at replacement points).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "tiles.h"

namespace mf {

namespace {

__global__ void k_tile_features(int tilenum, int tilem, const int *tile_ptr, const int *tile_col,
                                const int *tile_off, const int *csrptr_off, const unsigned char *bptr,
                                const unsigned char *col, const double *val, const double *diag, int rowA,
                                float *feat) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= tilenum) return;
    int lo = 0, hi = tilem - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_ptr[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int rb = lo;
    const int rl = rb == tilem - 1 ? rowA - (tilem - 1) * 16 : 16;
    const int vo = tile_off[t], nk = tile_off[t + 1] - vo;
    const int cc = csrptr_off[t];
    const int c0 = tile_col[t] * 16;
    double smax = 0.0, amax = 0.0, amin = INFINITY;
    for (int k = lane; k < nk; k += 32) {
        // row of entry k: last r with ptr[r] <= k
        int r = 0;
        for (int q = 1; q < rl; ++q)
            if (bptr[cc + q] <= k) r = q;
        const int i = rb * 16 + r, j = c0 + col[vo + k];
        const double a = fabs(val[vo + k]);
        const double di = fabs(diag[i]), dj = j < rowA ? fabs(diag[j]) : 0.0;
        const double s = (di > 0 && dj > 0) ? a / sqrt(di * dj) : INFINITY;
        smax = fmax(smax, s);
        amax = fmax(amax, a);
        if (a > 0) amin = fmin(amin, a);
    }
    for (int d = 16; d > 0; d >>= 1) {
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, d));
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, d));
        amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, d));
    }
    if (lane == 0) {
        float *f = feat + (size_t)t * 6;
        f[0] = (float)log10(fmax(smax, 1e-300));
        f[1] = amax > 0 && amin < INFINITY ? (float)log10(amax / amin) : 0.0f;
        f[2] = nk / 256.0f;
        f[3] = tile_col[t] == rb ? 1.0f : 0.0f;
        f[4] = (float)log10(fmax(amax, 1e-300));  // made relative on the host
        f[5] = 0.0f;
    }
}

}  // namespace

int tile_features(mf_tiles *t, std::vector<float> &feat, cudaStream_t s) {
    const int tn = t->tilenum;
    feat.assign((size_t)tn * 6, 0.0f);
    if (tn == 0) return MF_OK;
    DevArray<float> d;
    if (d.alloc((size_t)tn * 6)) return MF_ERR_NOMEM;
    k_tile_features<<<(tn + 7) / 8, 256, 0, s>>>(tn, t->tilem, t->tile_ptr.p, t->tile_col.p, t->tile_off.p,
                                                 t->csrptr_off.p, t->ptr.p, t->col.p, t->val.p, t->diag.p, t->rowA,
                                                 d.p);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaMemcpyAsync(feat.data(), d.p, sizeof(float) * feat.size(), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    float gmax = -1e30f;
    for (int k = 0; k < tn; ++k) gmax = std::max(gmax, feat[(size_t)k * 6 + 4]);
    for (int k = 0; k < tn; ++k) feat[(size_t)k * 6 + 4] -= gmax;
    return MF_OK;
}

// Unit roundoffs of FP8-E4M3, FP16, FP32.
static const double kU[4] = {0x1p-53, 0x1p-24, 0x1p-11, 0x1p-4};

uint8_t rule_precision(const float *f, double tau) {
    const double m = std::pow(10.0, (double)f[0]);
    const bool diag = f[3] > 0.5f;
    const double range = std::pow(10.0, (double)f[1]);
    if (!std::isfinite(m)) return MF_PREC_FP64;
    if (!diag && kU[MF_PREC_FP8] * m <= tau && range <= 4096.0) return MF_PREC_FP8;
    if (!diag && kU[MF_PREC_FP16] * m <= tau && range <= 1e8) return MF_PREC_FP16;
    if (kU[MF_PREC_FP32] * m <= tau) return MF_PREC_FP32;
    return MF_PREC_FP64;
}

// Row blocks whose tiles are mostly FP32 keep every low-precision tile in
// FP32: a row block whose planes all hold FP32 runs the lean FP32 loop, and
// the few FP16 / FP8 tiles would save only a few bytes.
void promote_minority(const mf_tiles *t, std::vector<uint8_t> &p) {
    for (int rb = 0; rb < t->tilem; ++rb) {
        const int t0 = t->h_tile_ptr[rb], t1 = t->h_tile_ptr[rb + 1];
        int n32 = 0, nsub = 0;
        for (int k = t0; k < t1; ++k) {
            n32 += p[k] == MF_PREC_FP32;
            nsub += p[k] == MF_PREC_FP16 || p[k] == MF_PREC_FP8;
        }
        if (nsub > 0 && 2 * nsub < n32 + nsub)
            for (int k = t0; k < t1; ++k)
                if (p[k] == MF_PREC_FP16 || p[k] == MF_PREC_FP8) p[k] = MF_PREC_FP32;
    }
}

// Level tolerances of the magnitude rule and the relative true residual
// below which the solver moves to the next level. The tolerance bounds the
// entry perturbation relative to the Jacobi scale sqrt(a_ii a_jj); it must
// stay below the smallest eigenvalue of the Jacobi-scaled matrix or the
// perturbed operator can lose definiteness (a 128^3 variable-coefficient
// Poisson diverges with FP16 off-diagonal tiles, tau ~ 5e-4).
const double kLevelTau[MF_NLEVELS] = {2e-7, 1e-7, 1e-7};
const double kLevelSwitch[MF_NLEVELS] = {1e-6, 0.0, 0.0};

int build_mixed_levels(mf_tiles *t, cudaStream_t s) {
    const int mode = t->opt.precision_mode;
    for (int l = 0; l < MF_NLEVELS; ++l) t->Lmix[l].built = false;
    if (mode == MF_MODE_FIXED) {
        if (t->opt.fixed_precision < MF_PREC_FP64 || t->opt.fixed_precision > MF_PREC_FP8) return MF_ERR_ARG;
        std::vector<uint8_t> p(t->tilenum, (uint8_t)t->opt.fixed_precision);
        int rc = build_layout(t, t->Lmix[0], p, s);
        if (rc) return rc;
        t->nlevels = 1;
        t->mixed_ready = true;
        return MF_OK;
    }
    if (mode != MF_MODE_MIXED_RULE) {
        set_last_error("precision mode not available");
        return MF_ERR_UNSUPPORTED;
    }
    std::vector<float> feat;
    int rc = tile_features(t, feat, s);
    if (rc) return rc;
    const double scale = t->opt.mixed_tau > 0 ? t->opt.mixed_tau : 1.0;
    int nl = 0;
    std::vector<uint8_t> prev;
    for (int l = 0; l < MF_NLEVELS; ++l) {
        std::vector<uint8_t> p(t->tilenum);
        for (int k = 0; k < t->tilenum; ++k) p[k] = rule_precision(&feat[(size_t)k * 6], kLevelTau[l] * scale);
        promote_minority(t, p);
        if (l > 0 && p == prev) break;  // identical to the previous level
        rc = build_layout(t, t->Lmix[l], p, s);
        if (rc) return rc;
        t->level_switch[l] = kLevelSwitch[l];
        prev.swap(p);
        ++nl;
    }
    t->nlevels = nl;
    t->mixed_ready = true;
    return MF_OK;
}

}  // namespace mf
