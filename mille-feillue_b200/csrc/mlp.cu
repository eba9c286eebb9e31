// Learned per-tile precision selector: an MLP 6 -> 64 -> 64 -> 4 (ReLU) over
// the tile features of features.cuh; class c is the tile's storage precision
// (0 FP64, 1 FP32, 2 FP16, 3 FP8). Weights are laid out W1[64][6], b1[64],
// W2[64][64], b2[64], W3[4][64], b3[4] (4868 floats).
//
// Training runs on the GPU: a forward/backward kernel with one warp per
// sample (lane i owns hidden units 2i, 2i+1) whose per-block gradient sums
// are added in a fixed order (the gradient is deterministic), and an Adam
// step. Inference is fused into the feature pass: the warp that computed a
// tile's features evaluates the network with the weights rounded to BF16 and
// FP32 accumulation, once per precision level.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "features.cuh"
#include "mf_internal.h"
#include "tiles.h"

namespace mf {

TileFeatArgs tile_feat_args(const mf_tiles *t);  // precision.cu
int matrix_features(const mf_tiles *t, float *lognnz, float *logrange, cudaStream_t s);
int tile_features(mf_tiles *t, std::vector<float> &feat, cudaStream_t s);

namespace {

constexpr int H = 64;
constexpr int OW1 = 0, OB1 = 384, OW2 = 448, OB2 = 4544, OW3 = 4608, OB3 = 4864, NW = 4868;
constexpr int GRAD_WARPS = 4;
// forward weights in shared memory: W1T[6][64], b1, W2T[64][64], b2, W3[4][64],
// b3 (the W1 / W2 blocks transposed so that a lane's two units are adjacent)
constexpr int FW_FLOATS = NW;
// the backward pass also needs W2 itself
constexpr int GW_FLOATS = NW + H * H;

// Weights into shared memory (transposed forward blocks; W2 row-major copy
// at w2 when given). bf16: round every weight to BF16 first.
__device__ void load_weights(const float *w, float *sw, float *w2, bool bf16) {
    for (int i = threadIdx.x; i < NW; i += blockDim.x) {
        float v = w[i];
        if (bf16) v = __bfloat162float(__float2bfloat16_rn(v));
        int dst = i;
        if (i < OB1) {
            const int u = i / 6, k = i % 6;
            dst = OW1 + k * H + u;
        } else if (i >= OW2 && i < OB2) {
            const int j = i - OW2, u = j / H, k = j % H;
            dst = OW2 + k * H + u;
            if (w2) w2[j] = v;
        }
        sw[dst] = v;
    }
}

struct Fwd {
    float h0, h1;  // layer-1 units 2*lane, 2*lane+1
    float g0, g1;  // layer-2 units
    float o[4];    // logits (every lane)
};

// Forward pass of one sample by a warp.
__device__ __forceinline__ Fwd warp_forward(const float *sw, const float (&x)[6]) {
    const int lane = threadIdx.x & 31, u0 = 2 * lane;
    Fwd F;
    float a0 = sw[OB1 + u0], a1 = sw[OB1 + u0 + 1];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float2 wt = *reinterpret_cast<const float2 *>(&sw[OW1 + k * H + u0]);
        a0 = fmaf(wt.x, x[k], a0);
        a1 = fmaf(wt.y, x[k], a1);
    }
    F.h0 = fmaxf(a0, 0.f);
    F.h1 = fmaxf(a1, 0.f);
    float z0 = sw[OB2 + u0], z1 = sw[OB2 + u0 + 1];
#pragma unroll 8
    for (int kk = 0; kk < 32; ++kk) {
        const float ha = __shfl_sync(0xffffffffu, F.h0, kk), hb = __shfl_sync(0xffffffffu, F.h1, kk);
        const float2 wa = *reinterpret_cast<const float2 *>(&sw[OW2 + (2 * kk) * H + u0]);
        const float2 wb = *reinterpret_cast<const float2 *>(&sw[OW2 + (2 * kk + 1) * H + u0]);
        z0 = fmaf(wa.x, ha, fmaf(wb.x, hb, z0));
        z1 = fmaf(wa.y, ha, fmaf(wb.y, hb, z1));
    }
    F.g0 = fmaxf(z0, 0.f);
    F.g1 = fmaxf(z1, 0.f);
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        const float2 w3 = *reinterpret_cast<const float2 *>(&sw[OW3 + o * H + u0]);
        float p = fmaf(w3.x, F.g0, w3.y * F.g1);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) p += __shfl_xor_sync(0xffffffffu, p, d);
        F.o[o] = p + sw[OB3 + o];
    }
    return F;
}

// Gradient of the mean softmax cross-entropy over the samples of the
// block's chunk; scale = 1 / (samples of the whole batch). The block's sum
// goes to part[blockIdx.x][NW] (standard layout), its loss to part_loss.
__global__ void __launch_bounds__(GRAD_WARPS * 32) k_mlp_grad(const float *__restrict__ w, const float *__restrict__ x,
                                                           const int *__restrict__ y, int n, int chunk, float scale,
                                                           float *part, float *part_loss) {
    extern __shared__ float smem[];
    float *sw = smem;            // FW_FLOATS
    float *w2 = sw + FW_FLOATS;  // W2 row-major
    float *G = w2 + H * H;       // GRAD_WARPS x NW (W1 / W2 blocks transposed)
    __shared__ float s_loss[GRAD_WARPS];
    load_weights(w, sw, w2, false);
    for (int i = threadIdx.x; i < GRAD_WARPS * NW; i += blockDim.x) G[i] = 0.f;
    __syncthreads();
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, u0 = 2 * lane;
    float *Gw = G + wid * NW;
    const int s0 = blockIdx.x * chunk, s1 = min(n, s0 + chunk);
    float lsum = 0.f;
    for (int s = s0 + wid; s < s1; s += GRAD_WARPS) {
        float xs[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) xs[k] = x[(size_t)s * 6 + k];
        const int lab = y[s];
        const Fwd F = warp_forward(sw, xs);
        float mx = F.o[0];
#pragma unroll
        for (int o = 1; o < 4; ++o) mx = fmaxf(mx, F.o[o]);
        float p[4], z = 0.f;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            p[o] = expf(F.o[o] - mx);
            z += p[o];
        }
        float d3[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            p[o] /= z;
            d3[o] = (p[o] - (o == lab ? 1.f : 0.f)) * scale;
        }
        lsum += -logf(p[lab] + 1e-30f);
        // layer 3
        float e0 = 0.f, e1 = 0.f;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            float2 *g3 = reinterpret_cast<float2 *>(&Gw[OW3 + o * H + u0]);
            float2 v = *g3;
            v.x = fmaf(d3[o], F.g0, v.x);
            v.y = fmaf(d3[o], F.g1, v.y);
            *g3 = v;
            const float2 w3 = *reinterpret_cast<const float2 *>(&sw[OW3 + o * H + u0]);
            e0 = fmaf(w3.x, d3[o], e0);
            e1 = fmaf(w3.y, d3[o], e1);
        }
        if (lane == 0)
#pragma unroll
            for (int o = 0; o < 4; ++o) Gw[OB3 + o] += d3[o];
        // layer 2: d2 = (W3^T d3) masked; gW2[u][k] += d2[u] h1[k] (stored at k*H + u)
        const float d20 = F.g0 > 0.f ? e0 : 0.f, d21 = F.g1 > 0.f ? e1 : 0.f;
        Gw[OB2 + u0] += d20;
        Gw[OB2 + u0 + 1] += d21;
        float c0 = 0.f, c1 = 0.f;
#pragma unroll 4
        for (int kk = 0; kk < 32; ++kk) {
            const float ha = __shfl_sync(0xffffffffu, F.h0, kk), hb = __shfl_sync(0xffffffffu, F.h1, kk);
            float2 *ga = reinterpret_cast<float2 *>(&Gw[OW2 + (2 * kk) * H + u0]);
            float2 *gb = reinterpret_cast<float2 *>(&Gw[OW2 + (2 * kk + 1) * H + u0]);
            float2 va = *ga, vb = *gb;
            va.x = fmaf(d20, ha, va.x);
            va.y = fmaf(d21, ha, va.y);
            vb.x = fmaf(d20, hb, vb.x);
            vb.y = fmaf(d21, hb, vb.y);
            *ga = va;
            *gb = vb;
            // d1[u] = sum_o W2[o][u] d2[o]
            const float da = __shfl_sync(0xffffffffu, d20, kk), db = __shfl_sync(0xffffffffu, d21, kk);
            const float2 wa = *reinterpret_cast<const float2 *>(&w2[(2 * kk) * H + u0]);
            const float2 wb = *reinterpret_cast<const float2 *>(&w2[(2 * kk + 1) * H + u0]);
            c0 = fmaf(wa.x, da, fmaf(wb.x, db, c0));
            c1 = fmaf(wa.y, da, fmaf(wb.y, db, c1));
        }
        // layer 1
        const float d10 = F.h0 > 0.f ? c0 : 0.f, d11 = F.h1 > 0.f ? c1 : 0.f;
        Gw[OB1 + u0] += d10;
        Gw[OB1 + u0 + 1] += d11;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float2 *g1 = reinterpret_cast<float2 *>(&Gw[OW1 + k * H + u0]);
            float2 v = *g1;
            v.x = fmaf(d10, xs[k], v.x);
            v.y = fmaf(d11, xs[k], v.y);
            *g1 = v;
        }
        __syncwarp();
    }
    if (lane == 0) s_loss[wid] = lsum;
    __syncthreads();
    for (int i = threadIdx.x; i < NW; i += blockDim.x) {
        int src = i;
        if (i < OB1) src = OW1 + (i % 6) * H + i / 6;
        else if (i >= OW2 && i < OB2) src = OW2 + ((i - OW2) % H) * H + (i - OW2) / H;
        float a = 0.f;
        for (int q = 0; q < GRAD_WARPS; ++q) a += G[q * NW + src];
        part[(size_t)blockIdx.x * NW + i] = a;
    }
    if (threadIdx.x == 0) {
        float a = 0.f;
        for (int q = 0; q < GRAD_WARPS; ++q) a += s_loss[q];
        part_loss[blockIdx.x] = a;
    }
}

// out[i] = sum over blocks b of part[b][i], in block order.
__global__ void k_mlp_reduce(const float *part, int nb, float *out, const float *part_loss, float *loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < NW) {
        float a = 0.f;
        for (int b = 0; b < nb; ++b) a += part[(size_t)b * NW + i];
        out[i] = a;
    }
    if (i == 0 && loss) {
        float a = 0.f;
        for (int b = 0; b < nb; ++b) a += part_loss[b];
        *loss = a;
    }
}

__global__ void k_mlp_adam(float *w, float *m, float *v, const float *g, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NW) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

__global__ void __launch_bounds__(256) k_mlp_forward(const float *w, const float *x, int n, int bf16, float *logits) {
    __shared__ __align__(16) float sw[FW_FLOATS];
    load_weights(w, sw, nullptr, bf16 != 0);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int s = blockIdx.x * warps + (threadIdx.x >> 5); s < n; s += gridDim.x * warps) {
        float xs[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) xs[k] = x[(size_t)s * 6 + k];
        const Fwd F = warp_forward(sw, xs);
        if (lane < 4) logits[(size_t)s * 4 + lane] = F.o[lane];
    }
}

// Features + network for every tile, one warp per tile: precision class of
// tile t at level l -> prec[l * tilenum + t], with f5 = logres[l]. Hard limits
// on the network's choice: FP8 needs a tile dynamic range <= 2^12 and FP16
// <= 1e8, and a tile whose scaled magnitude is not finite stays FP64. (The
// diagonal entries of an FP16 / FP8 tile are stored in FP32 by the layout
// whatever the class, so diagonal tiles need no limit of their own.)
__global__ void __launch_bounds__(256) k_tile_select_mlp(TileFeatArgs A, const float *w, int nlev,
                                                          const float *logres, uint8_t *prec) {
    __shared__ __align__(16) float sw[FW_FLOATS];
    load_weights(w, sw, nullptr, true);
    __syncthreads();
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= A.tilenum) return;
    float f[5];
    warp_tile_features(A, t, f);
    float xs[6] = {f[0], f[1], f[2], f[3], f[4], 0.f};
    for (int l = 0; l < nlev; ++l) {
        xs[5] = logres[l];
        const Fwd F = warp_forward(sw, xs);
        int c = 0;
#pragma unroll
        for (int o = 1; o < 4; ++o)
            if (F.o[o] > F.o[c]) c = o;
        if (c == MF_PREC_FP8 && xs[1] > 3.6124f) c = MF_PREC_FP16;  // log10(4096)
        if (c == MF_PREC_FP16 && xs[1] > 8.0f) c = MF_PREC_FP32;
        if (!isfinite(xs[0]) || xs[0] > 300.f) c = MF_PREC_FP64;
        if ((threadIdx.x & 31) == 0) prec[(size_t)l * A.tilenum + t] = (uint8_t)c;
    }
}

std::mutex g_w_mu;
std::vector<float> g_weights;  // process-wide selector weights (host)

int grad_launch(const float *w, const float *x, const int *y, int n, float scale, DevArray<float> &part,
                DevArray<float> &ploss, float *g, float *loss_dev, cudaStream_t s) {
    const int chunk = 512;
    const int nb = std::max(1, (n + chunk - 1) / chunk);
    if (part.n < (size_t)nb * NW && part.alloc((size_t)nb * NW)) return MF_ERR_NOMEM;
    if (ploss.n < (size_t)nb && ploss.alloc((size_t)nb)) return MF_ERR_NOMEM;
    const size_t smem = sizeof(float) * (GW_FLOATS + (size_t)GRAD_WARPS * NW);
    MF_CUDA_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mlp_grad<<<nb, GRAD_WARPS * 32, smem, s>>>(w, x, y, n, chunk, scale, part.p, ploss.p);
    MF_CUDA_TRY(cudaGetLastError());
    k_mlp_reduce<<<(NW + 255) / 256, 256, 0, s>>>(part.p, nb, g, ploss.p, loss_dev);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_OK;
}

}  // namespace

// Precision classes of every tile at nlev levels with the process-wide
// weights (host output prec[l * tilenum + t]).
int mlp_select(mf_tiles *t, int nlev, const double *rel_res, std::vector<uint8_t> &prec, cudaStream_t s) {
    std::vector<float> w;
    {
        std::lock_guard<std::mutex> lk(g_w_mu);
        w = g_weights;
    }
    if ((int)w.size() != NW) {
        set_last_error("no selector weights loaded (mf_mlp_set_weights)");
        return MF_ERR_ARG;
    }
    const int tn = t->tilenum;
    prec.assign((size_t)nlev * tn, (uint8_t)MF_PREC_FP64);
    if (tn == 0 || nlev <= 0) return MF_OK;
    DevArray<float> dw, dres;
    DevArray<uint8_t> dp;
    if (dw.alloc(NW) || dres.alloc(nlev) || dp.alloc((size_t)nlev * tn)) return MF_ERR_NOMEM;
    std::vector<float> lr(nlev);
    for (int l = 0; l < nlev; ++l) lr[l] = (float)std::log10(std::max(rel_res[l], 1e-300));
    MF_CUDA_TRY(cudaMemcpyAsync(dw.p, w.data(), sizeof(float) * NW, cudaMemcpyHostToDevice, s));
    MF_CUDA_TRY(cudaMemcpyAsync(dres.p, lr.data(), sizeof(float) * nlev, cudaMemcpyHostToDevice, s));
    TileFeatArgs A = tile_feat_args(t);
    int rc = matrix_features(t, &A.lognnz, &A.logrange, s);
    if (rc) return rc;
    k_tile_select_mlp<<<(tn + 7) / 8, 256, 0, s>>>(A, dw.p, nlev, dres.p, dp.p);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaMemcpyAsync(prec.data(), dp.p, prec.size(), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_OK;
}

}  // namespace mf

using namespace mf;

extern "C" {

int mf_mlp_set_weights(const float *w) {
    std::lock_guard<std::mutex> lk(g_w_mu);
    if (!w) {
        g_weights.clear();
        return MF_OK;
    }
    for (int i = 0; i < NW; ++i)
        if (!std::isfinite(w[i])) {
            set_last_error("selector weights are not finite");
            return MF_ERR_ARG;
        }
    g_weights.assign(w, w + NW);
    return MF_OK;
}

int mf_mlp_get_weights(float *w) {
    std::lock_guard<std::mutex> lk(g_w_mu);
    if ((int)g_weights.size() != NW) return MF_ERR_ARG;
    if (w) std::memcpy(w, g_weights.data(), sizeof(float) * NW);
    return MF_OK;
}

int mf_mlp_forward_dev(const float *w, const float *x, int n, int bf16, float *logits) {
    if (!w || !x || !logits || n < 0) return MF_ERR_ARG;
    if (n == 0) return MF_OK;
    const int blocks = std::min(1184, (n + 7) / 8);
    k_mlp_forward<<<blocks, 256>>>(w, x, n, bf16, logits);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaDeviceSynchronize());
    return MF_OK;
}

int mf_mlp_grad_dev(const float *w, const float *x, const int *labels, int n, float *g, float *loss) {
    if (!w || !x || !labels || !g || n <= 0) return MF_ERR_ARG;
    DevArray<float> part, ploss, dl;
    if (dl.alloc(1)) return MF_ERR_NOMEM;
    int rc = grad_launch(w, x, labels, n, 1.f / (float)n, part, ploss, g, dl.p, 0);
    if (rc) return rc;
    float h = 0.f;
    MF_CUDA_TRY(cudaMemcpy(&h, dl.p, sizeof h, cudaMemcpyDeviceToHost));
    if (loss) *loss = h / (float)n;
    return MF_OK;
}

int mf_mlp_train_dev(float *w, const float *x, const int *labels, int n, int steps, int batch, float lr,
                     float *loss) {
    if (!w || !x || !labels || n <= 0 || steps < 0 || batch <= 0 || !(lr > 0.f)) return MF_ERR_ARG;
    batch = std::min(batch, n);
    DevArray<float> m, v, g, part, ploss, dl;
    if (m.alloc(NW) || v.alloc(NW) || g.alloc(NW) || dl.alloc(1)) return MF_ERR_NOMEM;
    MF_CUDA_TRY(cudaMemset(m.p, 0, sizeof(float) * NW));
    MF_CUDA_TRY(cudaMemset(v.p, 0, sizeof(float) * NW));
    double p1 = 1.0, p2 = 1.0;
    for (int it = 0; it < steps; ++it) {
        // mini-batch it covers samples [it*batch mod n, +batch) (the caller
        // shuffles the samples); a batch running past n stops at n
        const int off = (int)(((long long)it * batch) % n);
        const int cnt = std::min(batch, n - off);
        int rc = grad_launch(w, x + (size_t)off * 6, labels + off, cnt, 1.f / (float)cnt, part, ploss, g.p, dl.p, 0);
        if (rc) return rc;
        p1 *= 0.9;
        p2 *= 0.999;
        k_mlp_adam<<<(NW + 255) / 256, 256>>>(w, m.p, v.p, g.p, lr, (float)(1.0 / (1.0 - p1)),
                                              (float)(1.0 / (1.0 - p2)));
        MF_CUDA_TRY(cudaGetLastError());
        if (loss && it == steps - 1) {
            float h = 0.f;
            MF_CUDA_TRY(cudaMemcpy(&h, dl.p, sizeof h, cudaMemcpyDeviceToHost));
            *loss = h / (float)cnt;
        }
    }
    MF_CUDA_TRY(cudaDeviceSynchronize());
    return MF_OK;
}

int mf_tiles_features(const mf_tiles *tc, float *feat) {
    mf_tiles *t = const_cast<mf_tiles *>(tc);
    if (!t || !feat) return MF_ERR_ARG;
    MF_CUDA_TRY(cudaSetDevice(t->opt.device));
    std::vector<float> f;
    int rc = tile_features(t, f, 0);
    if (rc) return rc;
    std::memcpy(feat, f.data(), sizeof(float) * f.size());
    return MF_OK;
}

int mf_tiles_select_mlp(const mf_tiles *tc, int nlev, const double *rel_res, unsigned char *prec) {
    mf_tiles *t = const_cast<mf_tiles *>(tc);
    if (!t || !rel_res || !prec || nlev <= 0) return MF_ERR_ARG;
    MF_CUDA_TRY(cudaSetDevice(t->opt.device));
    std::vector<uint8_t> p;
    int rc = mlp_select(t, nlev, rel_res, p, 0);
    if (rc) return rc;
    std::memcpy(prec, p.data(), p.size());
    return MF_OK;
}

}  // extern "C"
