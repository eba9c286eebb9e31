// mf_solve_cg_dev_noalloc: the FP64 persistent CG solve with all of its
// device scratch in a file-scope static __device__ array, so the call itself
// allocates no device memory.
//
// Who needs it: callers that cannot allocate at solve time. A serving process
// whose own allocator (a caching allocator, a memory pool sized at start-up)
// already holds all free HBM would see mf_solve_cg_dev's first-call
// cudaMalloc of its workspace fail. A latency-sensitive caller can't afford
// the implicit device-wide synchronization of cudaMalloc / cudaFree either.
// The matrix itself is still encoded (and allocated) up front by mf_encode.
//
// Limits: n rounded up to a multiple of 16 must be <= MF_NOALLOC_MAX_ROWS
// (131072) and the solver grid must have <= 1024 CTAs; larger systems return
// MF_ERR_ARG with a message and are left to mf_solve_cg_dev. The scratch costs
// about 5.1 MiB of device memory per device, taken when the module loads.
//
// Set-up: the first call on each device (with that device current) looks up
// the scratch address with cudaGetSymbolAddress. Make that first call before
// any stream capture begins. The address is cached for the life of the
// process: a cudaDeviceReset on that device invalidates it, and calls after
// such a reset are not supported.
//
// Concurrency: there is one scratch per device, so calls in flight at the same
// time on one device (from two threads, or on two streams) race on it. Callers
// must serialize them.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "mf_internal.h"
#include "solver.h"

namespace mf {
namespace {

constexpr int NA_MAX_G = 1024;
constexpr size_t NA_VEC_WORDS = 5 * (size_t)MF_NOALLOC_MAX_ROWS;  // b, x, r, d, q
constexpr size_t NA_PART_WORDS = 2 * 4 * (size_t)NA_MAX_G + 64;   // reduction slots + norms
constexpr size_t NA_SYNC_U32 =
    (size_t)SYNC_FLAGS + (size_t)NA_MAX_G * FLAG_STRIDE + 32 + sizeof(DevResult) / 4 + 8;
constexpr size_t NA_WORDS = NA_VEC_WORDS + NA_PART_WORDS + (NA_SYNC_U32 + 1) / 2;
constexpr int NA_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[NA_WORDS];

std::mutex g_na_mu;
double *g_na_ptr[NA_MAX_DEVICES];

// Address of this device's scratch (the current device must be `dev`).
int scratch_of(int dev, double **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        set_last_error("mf_solve_cg_dev_noalloc: device ordinal out of range");
        return MF_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("mf_solve_cg_dev_noalloc: cudaGetSymbolAddress: ") +
                           cudaGetErrorString(e));
            return MF_ERR_CUDA;
        }
        g_na_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_na_ptr[dev];
    return MF_OK;
}

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" int mf_solve_cg_dev_noalloc(mf_tiles *t, const double *b_dev, double *x_dev, double tol,
                                       int maxiter, const mf_options *opt_in, mf_result *res) {
    if (!t || !b_dev || !x_dev) return MF_ERR_ARG;
    if (t->rowA != t->colA) {
        set_last_error("the solvers need a square matrix");
        return MF_ERR_UNSUPPORTED;
    }
    const size_t n16 = (size_t)t->tilem * 16;
    if (n16 > (size_t)MF_NOALLOC_MAX_ROWS) {
        set_last_error("mf_solve_cg_dev_noalloc: " + std::to_string(t->rowA) +
                       " rows exceed the static scratch limit of " + std::to_string(MF_NOALLOC_MAX_ROWS) +
                       " (use mf_solve_cg_dev)");
        return MF_ERR_ARG;
    }
    if (t->G > NA_MAX_G) {
        set_last_error("mf_solve_cg_dev_noalloc: the solver grid exceeds 1024 CTAs");
        return MF_ERR_ARG;
    }
    const mf_options opt = opt_in ? *opt_in : t->opt;
    MF_CUDA_TRY(cudaSetDevice(t->opt.device));
    double *w = nullptr;
    int rc = scratch_of(t->opt.device, &w);
    if (rc) return rc;

    const int n = t->rowA;
    double *vb = w, *vx = w + n16, *vr = w + 2 * n16, *vd = w + 3 * n16, *vq = w + 4 * n16;
    double *partial = w + NA_VEC_WORDS;
    uint32_t *sync = reinterpret_cast<uint32_t *>(w + NA_VEC_WORDS + NA_PART_WORDS);
    DevResult *dres = reinterpret_cast<DevResult *>(sync + sync_words(t->G));

    // Must start at zero: the vectors (their padding rows past n are read by
    // the SpMV and the dot products), the grid-sync counters, the CTA epoch
    // flags, the error word and the result record.
    MF_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(double) * 5 * n16));
    MF_CUDA_TRY(cudaMemsetAsync(sync, 0, sizeof(uint32_t) * (sync_words(t->G) + sizeof(DevResult) / 4 + 8)));
    MF_CUDA_TRY(cudaMemcpyAsync(vb, b_dev, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    MF_CUDA_TRY(cudaMemcpyAsync(vx, x_dev, sizeof(double) * n, cudaMemcpyDeviceToDevice));

    KParams P;
    base_params(t, P);
    if (opt.timeout_s > 0) P.limit_ns = (uint64_t)(opt.timeout_s * 1e9);
    P.sync = sync;
    P.partial = partial;
    P.b = vb;
    P.x = vx;
    P.r = vr;
    P.d = vd;
    P.q = vq;
    P.tol = tol;
    P.maxiter = maxiter;
    P.fixed_iterations = opt.fixed_iterations;
    P.replace_every = 0;
    P.res = dres;
    P.prefetch = opt.reserved[3] == 1 ? 1 : 0;
    rc = launch_solver(t, 0, P, 0);  // nlay == 1: the FP64 kernel
    if (rc) return rc;

    DevResult dr;
    uint32_t err[2];
    MF_CUDA_TRY(cudaMemcpy(&dr, dres, sizeof dr, cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(err, sync + SYNC_ERROR, sizeof err, cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(x_dev, vx, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    const int status = err[0] ? (int)err[0] : dr.status;
    mf_result R;
    std::memset(&R, 0, sizeof R);
    R.status = status;
    R.iterations = err[0] ? -1 : dr.iterations;
    R.error_site = (int)err[1];
    R.rel_residual_rec = dr.bb > 0 ? std::sqrt(dr.rr) / std::sqrt(dr.bb) : std::sqrt(dr.rr);
    R.time_ms = 0;  // not timed: timing would need events
    R.spmv_bytes = R.spmv_bytes_fp64 = t->L64.alg_bytes;
    R.tile_frac[0] = 1.0;
    R.iters_fp64 = dr.it_layout[0];
    R.total_bytes = (double)dr.it_layout[0] * (t->L64.alg_bytes + 56.0 * n) + t->L64.alg_bytes + 16.0 * n;
    R.rel_residual_true = NAN;
    if (!err[0] && opt.check_true_residual) {
        // A x into the q slot, the two norms into the tail of the partials
        double *out = partial + 2 * 4 * (size_t)t->G;
        if ((rc = launch_spmv(t, -1, vx, vq, 1, 0))) return rc;
        if ((rc = launch_residual_norms(n, vb, vq, out, 0))) return rc;
        double h[2];
        MF_CUDA_TRY(cudaMemcpy(h, out, sizeof h, cudaMemcpyDeviceToHost));
        R.rel_residual_true = h[1] > 0 ? std::sqrt(h[0]) / std::sqrt(h[1]) : std::sqrt(h[0]);
    }
    if (res) *res = R;
    return status;
}
