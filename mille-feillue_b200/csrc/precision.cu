// Per-tile precision selection for the mixed-precision layouts (features:
// features.cuh).
//
// Magnitude rule: at level l with tolerance tau_l a tile takes the lowest of
// FP8, FP16, FP32 whose unit roundoff u_p satisfies u_p * m_t <= tau_l and
// whose range holds the tile (FP8 also needs a dynamic range <= 2^12);
// diagonal tiles never go below FP32; otherwise FP64. The levels tighten as
// the true residual falls (the solver switches at replacement points).
//
// Row blocks whose rows are all diagonally dominant Z-rows (one diagonal
// entry a_ii > 0, every other entry <= 0, row sum >= 0 up to rounding) are
// stored with row-sum-preserving compensation (layout.cu): there the
// rounding of an entry moves only an
// edge weight of the operator, by at most u_p relative, so its tiles take
// the lowest precision with u_p <= kCompTau whatever their magnitude (FP16
// within its range; the diagonal entries themselves stay FP32).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "features.cuh"
#include "tiles.h"

namespace mf {

int mlp_select(mf_tiles *t, int nlev, const double *rel_res, std::vector<uint8_t> &prec, cudaStream_t s);  // mlp.cu

TileFeatArgs tile_feat_args(const mf_tiles *t) {
    TileFeatArgs A;
    A.tilenum = t->tilenum;
    A.tilem = t->tilem;
    A.rowA = t->rowA;
    A.lognnz = 0.0f;
    A.logrange = 0.0f;
    A.tile_ptr = t->tile_ptr.p;
    A.tile_col = t->tile_col.p;
    A.tile_off = t->tile_off.p;
    A.csrptr_off = t->csrptr_off.p;
    A.bptr = t->ptr.p;
    A.col = t->col.p;
    A.val = t->val.p;
    A.diag = t->diag.p;
    return A;
}

namespace {

__global__ void k_tile_features(TileFeatArgs A, float *feat) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= A.tilenum) return;
    float f[5];
    warp_tile_features(A, t, f);
    if ((threadIdx.x & 31) == 0) {
        float *o = feat + (size_t)t * 6;
        for (int k = 0; k < 5; ++k) o[k] = f[k];
        o[5] = 0.0f;
    }
}

// Positive doubles order like their bit patterns: the min / max of |a| over
// the nonzeros by integer atomics (the caller sets mn to ~0 and mx to 0).
__global__ void k_absminmax(const double *v, long long n, unsigned long long *mn, unsigned long long *mx) {
    unsigned long long lo = ~0ull, hi = 0ull;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v[i]));
        if (b != 0ull) lo = b < lo ? b : lo;
        hi = b > hi ? b : hi;
    }
    for (int d = 16; d > 0; d >>= 1) {
        const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, lo, d), h2 = __shfl_xor_sync(0xffffffffu, hi, d);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mn, lo);
        atomicMax(mx, hi);
    }
}

}  // namespace

// Smallest nonzero and largest |v[i]| over n device values (lo = hi = 0 when
// every value is zero).
int abs_range(const double *v, long long n, double *lo, double *hi, cudaStream_t s) {
    *lo = *hi = 0.0;
    if (n <= 0) return MF_OK;
    DevArray<unsigned long long> d;
    if (d.alloc(2)) return MF_ERR_NOMEM;
    const unsigned long long init[2] = {~0ull, 0ull};
    MF_CUDA_TRY(cudaMemcpyAsync(d.p, init, sizeof init, cudaMemcpyHostToDevice, s));
    k_absminmax<<<592, 256, 0, s>>>(v, n, d.p, d.p + 1);
    MF_CUDA_TRY(cudaGetLastError());
    unsigned long long h[2];
    MF_CUDA_TRY(cudaMemcpyAsync(h, d.p, sizeof h, cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[0] == ~0ull || h[1] == 0ull) return MF_OK;
    std::memcpy(lo, &h[0], sizeof *lo);
    std::memcpy(hi, &h[1], sizeof *hi);
    return MF_OK;
}

// The whole-matrix features f2 and f4 (a device reduction over the values).
int matrix_features(const mf_tiles *t, float *lognnz, float *logrange, cudaStream_t s) {
    *lognnz = (float)std::log10(std::max(1.0, (double)t->csrsize));
    *logrange = 0.0f;
    double lo = 0.0, hi = 0.0;
    const int rc = abs_range(t->val.p, (long long)t->csrsize, &lo, &hi, s);
    if (rc) return rc;
    if (lo > 0.0) *logrange = (float)std::log10(hi / lo);
    return MF_OK;
}

// Features f0..f5 of every tile, on the device (f5 = 0).
int tile_features_dev(mf_tiles *t, DevArray<float> &d, cudaStream_t s) {
    const int tn = t->tilenum;
    if (d.alloc((size_t)(tn > 0 ? tn : 1) * 6)) return MF_ERR_NOMEM;
    if (tn == 0) return MF_OK;
    TileFeatArgs A = tile_feat_args(t);
    int rc = matrix_features(t, &A.lognnz, &A.logrange, s);
    if (rc) return rc;
    k_tile_features<<<(tn + 7) / 8, 256, 0, s>>>(A, d.p);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

int tile_features(mf_tiles *t, std::vector<float> &feat, cudaStream_t s) {
    const int tn = t->tilenum;
    feat.assign((size_t)tn * 6, 0.0f);
    if (tn == 0) return MF_OK;
    DevArray<float> d;
    int rc = tile_features_dev(t, d, s);
    if (rc) return rc;
    MF_CUDA_TRY(cudaMemcpyAsync(feat.data(), d.p, sizeof(float) * feat.size(), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_OK;
}

// Unit roundoffs of FP8-E4M3, FP16, FP32.
static const double kU[4] = {0x1p-53, 0x1p-24, 0x1p-11, 0x1p-4};

// Largest relative edge-weight perturbation accepted for compensated row
// blocks (the operator then lies within (1 +- u) A): FP16 (u = 4.9e-4)
// passes, FP8 (u = 6.25e-2) does not (CG with true-residual replacement
// stalls on the 128^3 variable-coefficient Poisson with every off-diagonal
// entry in FP8).
static const double kCompTau = 1e-3;

namespace {
// 1 for a row block whose rows are all diagonally dominant Z-rows: exactly
// one diagonal entry, positive, every other entry <= 0, and a row sum of at
// least -1e-12 a_ii (zero up to the rounding of the sum: the compensated
// operator keeps the row sums, and its perturbation is bounded relative to
// the matrix only where they are non-negative). One warp per row block, a
// lane per row.
__global__ void k_rb_zrows(TileFeatArgs A, uint8_t *zflag) {
    const int lane = threadIdx.x & 31;
    const int rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (rb >= A.tilem) return;
    const int rl = rb == A.tilem - 1 ? A.rowA - (A.tilem - 1) * 16 : 16;
    bool ok = true;
    if (lane < rl) {
        const int row = rb * 16 + lane;
        int nd = 0;
        bool z = true, pos = false;
        double diag = 0.0, sum = 0.0;
        for (int t = A.tile_ptr[rb]; t < A.tile_ptr[rb + 1]; ++t) {
            const int vo = A.tile_off[t], nk = A.tile_off[t + 1] - vo;
            const int cc = A.csrptr_off[t];
            const int q0 = A.bptr[cc + lane], q1 = lane + 1 < rl ? (int)A.bptr[cc + lane + 1] : nk;
            for (int q = q0; q < q1; ++q) {
                const double a = A.val[vo + q];
                sum += a;
                if (A.tile_col[t] * 16 + (int)A.col[vo + q] == row) {
                    ++nd;
                    pos = a > 0.0;
                    diag = a;
                } else if (!(a <= 0.0)) {
                    z = false;
                }
            }
        }
        ok = nd == 1 && z && pos && sum >= -1e-12 * diag;
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) zflag[rb] = ok ? 1 : 0;
}
}  // namespace

// Per row block: all rows diagonally dominant Z-rows (device flags).
int rb_zrows_dev(const mf_tiles *t, DevArray<uint8_t> &d, cudaStream_t s) {
    if (d.alloc(t->tilem > 0 ? t->tilem : 1)) return MF_ERR_NOMEM;
    if (t->tilem == 0) return MF_OK;
    k_rb_zrows<<<(t->tilem + 7) / 8, 256, 0, s>>>(tile_feat_args(t), d.p);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

struct RuleThresholds {
    float mag[4];           // largest log10 tile magnitude that passes, per precision
    float range16, range8;  // largest log10 tile range allowed for FP16 / FP8
};

// The magnitude rule for a tile with features f (f0 = log10 of its scaled
// magnitude m, f1 = log10 of its value range, f3 = diagonal tile): the lowest
// precision p with u_p * m <= tau, FP8 only for an off-diagonal tile of range
// <= 4096, FP16 only for one of range <= 1e8, FP32 before FP64. Each test
// (u_p * 10^f0 <= tau, 10^f1 <= R, evaluated in double) increases with f, so
// it holds exactly for the floats up to the largest one that passes it,
// found once per level by bisection over the ordered float values; a tile
// then needs float comparisons only (NaN features fail every test: FP64).
namespace {
int32_t fkey(float f) {
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b >= 0 ? b : -(b & 0x7fffffff);
}
float fval(int32_t k) {
    const int32_t b = k >= 0 ? k : (int32_t)((uint32_t)(-k) | 0x80000000u);
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
template <class Pred>
float largest_passing(Pred pass) {  // pass holds on (-inf, x] for some float x
    int64_t lo = fkey(-INFINITY), hi = fkey(INFINITY);  // the span exceeds int32
    if (!pass(fval((int32_t)lo))) return NAN;  // nothing passes
    if (pass(fval((int32_t)hi))) return INFINITY;
    while (hi - lo > 1) {  // pass(lo), !pass(hi)
        const int64_t mid = lo + (hi - lo) / 2;
        if (pass(fval((int32_t)mid))) lo = mid;
        else hi = mid;
    }
    return fval((int32_t)lo);
}
}  // namespace

RuleThresholds rule_thresholds(double tau) {
    RuleThresholds r;
    for (int p = MF_PREC_FP32; p <= MF_PREC_FP8; ++p)
        r.mag[p] = largest_passing([&](float f) { return kU[p] * std::pow(10.0, (double)f) <= tau; });
    r.range16 = largest_passing([](float f) { return std::pow(10.0, (double)f) <= 1e8; });
    r.range8 = largest_passing([](float f) { return std::pow(10.0, (double)f) <= 4096.0; });
    return r;
}

__host__ __device__ uint8_t rule_precision_fast(const float *f, const RuleThresholds &r) {
    const float f0 = f[0], f1 = f[1];
    const bool diag = f[3] > 0.5f;
    if (!diag && f0 <= r.mag[MF_PREC_FP8] && f1 <= r.range8) return MF_PREC_FP8;
    if (!diag && f0 <= r.mag[MF_PREC_FP16] && f1 <= r.range16) return MF_PREC_FP16;
    if (f0 <= r.mag[MF_PREC_FP32]) return MF_PREC_FP32;
    return MF_PREC_FP64;
}


// The rule for every tile at one level (one thread per row block):
// compensated row blocks (zrb) take the lowest precision allowed by
// kCompTau within its range (comp8 / comp16 / comp32 say which are), the
// others the magnitude rule with thresholds thr.
__global__ void k_rule(const int *tile_ptr, const float *feat, const uint8_t *zrb, RuleThresholds thr,
                       RuleThresholds any, int comp8, int comp16, int comp32, int tilem, uint8_t *prec) {
    const int rb = blockIdx.x * blockDim.x + threadIdx.x;
    if (rb >= tilem) return;
    for (int k = tile_ptr[rb]; k < tile_ptr[rb + 1]; ++k) {
        const float *f = feat + (size_t)k * 6;
        uint8_t p;
        if (zrb[rb]) {
            const float f1 = f[1];
            p = (comp8 && f1 <= any.range8) ? MF_PREC_FP8
                : (comp16 && f1 <= any.range16) ? MF_PREC_FP16
                : comp32 ? MF_PREC_FP32 : rule_precision_fast(f, thr);
        } else {
            p = rule_precision_fast(f, thr);
        }
        prec[k] = p;
    }
}

// Level tolerances of the magnitude rule and the relative true residual
// below which the solver moves to the next level. The tolerance bounds the
// entry perturbation relative to the Jacobi scale sqrt(a_ii a_jj); it must
// stay below the smallest eigenvalue of the Jacobi-scaled matrix or the
// perturbed operator can lose definiteness (a 128^3 variable-coefficient
// Poisson diverges with uncompensated FP16 off-diagonal tiles, tau ~ 5e-4).
// Compensated row blocks do not use these levels.
const double kLevelTau[MF_NLEVELS] = {2e-7, 1e-7, 1e-7};
const double kLevelSwitch[MF_NLEVELS] = {1e-6, 0.0, 0.0};

int build_mixed_levels(mf_tiles *t, cudaStream_t s) {
    const int mode = t->opt.precision_mode;
    for (int l = 0; l < MF_NLEVELS; ++l) t->Lmix[l].built = false;
    t->Lbicg.built = false;
    if (mode == MF_MODE_FIXED) {
        if (t->opt.fixed_precision < MF_PREC_FP64 || t->opt.fixed_precision > MF_PREC_FP8) return MF_ERR_ARG;
        std::vector<uint8_t> p(t->tilenum, (uint8_t)t->opt.fixed_precision);
        int rc = build_layout(t, t->Lmix[0], p, s);
        if (rc) return rc;
        t->nlevels = 1;
        t->mixed_ready = true;
        return MF_OK;
    }
    if (mode == MF_MODE_MIXED_MLP) {
        // the learned selector: one class per tile and level, with the
        // level's starting relative residual as the sixth feature
        double res[MF_NLEVELS];
        int nlev = 0;
        for (int l = 0; l < MF_NLEVELS; ++l) {
            res[l] = l == 0 ? 1.0 : kLevelSwitch[l - 1];
            ++nlev;
            if (kLevelSwitch[l] <= 0.0) break;  // the last level used
        }
        std::vector<uint8_t> pm;
        int rc = mlp_select(t, nlev, res, pm, s);
        if (rc) return rc;
        int nl = 0;
        std::vector<uint8_t> prev;
        for (int l = 0; l < nlev; ++l) {
            std::vector<uint8_t> p(pm.begin() + (size_t)l * t->tilenum, pm.begin() + (size_t)(l + 1) * t->tilenum);
            if (l > 0 && p == prev) break;
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
    if (mode != MF_MODE_MIXED_RULE) {
        set_last_error("precision mode not available");
        return MF_ERR_UNSUPPORTED;
    }
    DevArray<float> feat;
    int rc = tile_features_dev(t, feat, s);
    if (rc) return rc;
    DevArray<uint8_t> zrb, dprec;
    if ((rc = rb_zrows_dev(t, zrb, s))) return rc;
    if (dprec.alloc(t->tilenum > 0 ? t->tilenum : 1)) return MF_ERR_NOMEM;
    const double scale = t->opt.mixed_tau > 0 ? t->opt.mixed_tau : 1.0;
    // compensated row blocks: the lowest precision with u_p <= kCompTau
    // (scaled like the level tolerances) whose range holds the tile
    const RuleThresholds any = rule_thresholds(INFINITY);
    const bool comp16 = kU[MF_PREC_FP16] <= kCompTau * scale, comp8 = kU[MF_PREC_FP8] <= kCompTau * scale;
    const bool comp32 = kU[MF_PREC_FP32] <= kCompTau * scale;
    int nl = 0;
    std::vector<uint8_t> prev;
    for (int l = 0; l < MF_NLEVELS; ++l) {
        std::vector<uint8_t> p(t->tilenum);
        const RuleThresholds thr = rule_thresholds(kLevelTau[l] * scale);
        if (t->tilem > 0)
            k_rule<<<(t->tilem + 255) / 256, 256, 0, s>>>(t->tile_ptr.p, feat.p, zrb.p, thr, any, comp8 ? 1 : 0,
                                                          comp16 ? 1 : 0, comp32 ? 1 : 0, t->tilem, dprec.p);
        MF_CUDA_TRY(cudaGetLastError());
        if (t->tilenum > 0)
            MF_CUDA_TRY(cudaMemcpyAsync(p.data(), dprec.p, t->tilenum, cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaStreamSynchronize(s));
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
