// Batched solve of many independent systems of uneven size in one
// persistent launch. The grid is split into groups of gs CTAs; every system
// gets a gs-CTA slab layout, each group takes systems from a device queue in
// decreasing nnz order (longest-processing-time first) and runs the FP64 CG
// recurrence of the single-system kernel on them, with reductions and halo
// flags local to the group. The whole solve (queue reset, scatter of b,
// vector reset, the persistent launch, gather of x) is captured once in a
// CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "solver.h"
#include "tiles.h"

namespace mf {
int encode_dev_impl(int n, int ncols, int nnz, const int *rp, const int *ci, const double *val,
                    const mf_options *opt, int G_force, mf_tiles **out);
}

using namespace mf;

struct mf_batch {
    int count = 0, device = 0, grid = 0, gs = 1, ngroups = 0;
    std::vector<mf_tiles *> one;   // gs-CTA layouts (batched launch)
    std::vector<mf_tiles *> full;  // whole-GPU layouts (one launch per system)
    std::vector<int> n;
    std::vector<long long> nnz;
    std::vector<long long> voff, poff;  // workspace (16-padded) / packed offsets
    long long total_rows = 0, total_nnz = 0, ws_rows = 0;
    DevArray<SysDesc> d_desc;
    DevArray<int> d_order, d_n;
    DevArray<long long> d_voff, d_poff;
    DevArray<unsigned> d_queue;
    DevArray<BatchResult> d_res;
    DevArray<uint32_t> d_sync;    // per group sync words
    DevArray<double> d_partial;   // per group reduction partials
    DevArray<double> ws;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    const double *g_b = nullptr;
    double *g_x = nullptr;
    double g_tol = 0;
    int g_maxiter = 0;
    BatchParams params;
    ~mf_batch() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
        for (auto *t : one) mf_free(t);
        for (auto *t : full) mf_free(t);
    }
};

namespace {

constexpr int kBatchGroupDefault = 4;  // CTAs per system group (fastest of 4, 8, 16 on the 512-system set)
// group sync words: arrive counter, error word, rank flags (32-byte aligned)
size_t group_sync_words(int gs) { return (sync_words(gs) + 7) & ~(size_t)7; }

// packed[poff_s + i] <-> ws vector of system s, row i (i < n_s)
__global__ void k_scatter(const double *packed, double *ws, const long long *voff, const long long *poff,
                          const int *n, int count, long long ws_rows, int which) {
    for (int s = blockIdx.x; s < count; s += gridDim.x) {
        double *dst = ws + (long long)which * ws_rows + voff[s];
        const double *src = packed + poff[s];
        for (int i = threadIdx.x; i < n[s]; i += blockDim.x) dst[i] = src[i];
    }
}
__global__ void k_gather(double *packed, const double *ws, const long long *voff, const long long *poff,
                         const int *n, int count, long long ws_rows, int which) {
    for (int s = blockIdx.x; s < count; s += gridDim.x) {
        const double *src = ws + (long long)which * ws_rows + voff[s];
        double *dst = packed + poff[s];
        for (int i = threadIdx.x; i < n[s]; i += blockDim.x) dst[i] = src[i];
    }
}

}  // namespace

extern "C" {

int mf_batch_create(int count, const mf_csr *systems, const mf_options *opt_in, int with_baseline,
                    mf_batch **out) {
    if (count <= 0 || !systems || !out) return MF_ERR_ARG;
    mf_options opt;
    if (opt_in) opt = *opt_in;
    else mf_options_default(&opt);
    opt.precision_mode = MF_MODE_FP64;
    auto *B = new mf_batch;
    B->count = count;
    B->device = opt.device;
    MF_CUDA_TRY(cudaSetDevice(opt.device));
    B->n.resize(count);
    B->nnz.resize(count);
    B->voff.resize(count);
    B->poff.resize(count);
    long long vo = 0, po = 0;
    for (int s = 0; s < count; ++s) {
        const mf_csr &A = systems[s];
        if (A.n <= 0 || A.n != A.ncols) {
            delete B;
            return MF_ERR_ARG;
        }
        B->n[s] = A.n;
        B->nnz[s] = A.nnz;
        B->voff[s] = vo;
        B->poff[s] = po;
        vo += ((long long)(A.n + 15) / 16) * 16;
        po += A.n;
        B->total_nnz += A.nnz;
    }
    B->total_rows = po;
    B->ws_rows = vo;
    {
        int nsm = 0;
        MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opt.device));
        int gs = opt.reserved[4] > 0 ? opt.reserved[4] : kBatchGroupDefault;
        if (gs > nsm) gs = nsm;
        B->gs = gs;
        B->ngroups = nsm / gs;
        B->grid = B->ngroups * gs;
    }
    // per-system encodes: single-CTA layouts (and whole-GPU ones for the
    // one-launch-per-system comparison)
    for (int s = 0; s < count; ++s) {
        const mf_csr &A = systems[s];
        DevArray<int> rp, ci;
        DevArray<double> v;
        if (rp.alloc(A.n + 1) || ci.alloc(A.nnz) || v.alloc(A.nnz)) {
            delete B;
            return MF_ERR_NOMEM;
        }
        MF_CUDA_TRY(cudaMemcpy(rp.p, A.row_ptr, sizeof(int) * (A.n + 1), cudaMemcpyHostToDevice));
        MF_CUDA_TRY(cudaMemcpy(ci.p, A.col_idx, sizeof(int) * A.nnz, cudaMemcpyHostToDevice));
        MF_CUDA_TRY(cudaMemcpy(v.p, A.val, sizeof(double) * A.nnz, cudaMemcpyHostToDevice));
        mf_tiles *t1 = nullptr;
        int rc = encode_dev_impl(A.n, A.n, A.nnz, rp.p, ci.p, v.p, &opt, B->gs, &t1);
        if (rc) {
            delete B;
            return rc;
        }
        B->one.push_back(t1);
        if (with_baseline) {
            mf_tiles *tg = nullptr;
            rc = encode_dev_impl(A.n, A.n, A.nnz, rp.p, ci.p, v.p, &opt, 0, &tg);
            if (rc) {
                delete B;
                return rc;
            }
            B->full.push_back(tg);
        }
    }
    // device descriptors
    if (B->ws.alloc((size_t)5 * B->ws_rows) || B->d_desc.alloc(count) || B->d_order.alloc(count) ||
        B->d_n.alloc(count) || B->d_voff.alloc(count) || B->d_poff.alloc(count) || B->d_queue.alloc(1) ||
        B->d_res.alloc(count) || B->d_sync.alloc((size_t)B->ngroups * group_sync_words(B->gs)) ||
        B->d_partial.alloc((size_t)B->ngroups * 8 * B->gs)) {
        delete B;
        return MF_ERR_NOMEM;
    }
    std::vector<SysDesc> desc(count);
    for (int s = 0; s < count; ++s) {
        mf_tiles *t = B->one[s];
        SysDesc &D = desc[s];
        std::memset(&D, 0, sizeof D);
        D.slabs = t->L64.slabs.p;
        D.head = t->L64.head.p;
        D.cta_slab = t->L64.cta_slab.p;
        D.cta_rb = t->L64.cta_rb.p;
        D.cta_dep = t->L64.cta_dep.p;
        D.ns = t->L64.nslabs;
        D.kind = t->L64.kind;
        D.gt = GTiles{t->tile_ptr.p, t->tile_col.p, t->tile_off.p, t->csrptr_off.p, t->ptr.p, t->val.p,
                      t->col.p, t->tilem, t->rowA};
        double *w = B->ws.p + B->voff[s];
        D.b = w;
        D.x = w + B->ws_rows;
        D.r = w + 2 * B->ws_rows;
        D.d = w + 3 * B->ws_rows;
        D.q = w + 4 * B->ws_rows;
        D.n16 = t->tilem * 16;
    }
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B->nnz[a] > B->nnz[b]; });
    MF_CUDA_TRY(cudaMemcpy(B->d_desc.p, desc.data(), sizeof(SysDesc) * count, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(B->d_order.p, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(B->d_n.p, B->n.data(), sizeof(int) * count, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(B->d_voff.p, B->voff.data(), sizeof(long long) * count, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaMemcpy(B->d_poff.p, B->poff.data(), sizeof(long long) * count, cudaMemcpyHostToDevice));
    MF_CUDA_TRY(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    BatchParams &P = B->params;
    std::memset(&P, 0, sizeof P);
    P.sys = B->d_desc.p;
    P.order = B->d_order.p;
    P.count = count;
    P.queue = B->d_queue.p;
    P.stage_stride = stage_stride_of(B->one[0]->L64.slab_max);
    P.slab_area = slab_area_of(B->one[0]->L64.slab_max);
    P.limit_ns = (uint64_t)((opt.timeout_s > 0 ? opt.timeout_s : 2.0) * 1e9);
    P.gs = B->gs;
    P.gsync_words = (int)group_sync_words(B->gs);
    P.gsync = B->d_sync.p;
    P.gpartial = B->d_partial.p;
    P.res = B->d_res.p;
    *out = B;
    return MF_OK;
}

int mf_batch_solve_cg_dev(mf_batch *B, const double *b, double *x, double tol, int maxiter, double *ms) {
    if (!B || !b || !x) return MF_ERR_ARG;
    MF_CUDA_TRY(cudaSetDevice(B->device));
    const bool same = B->gexec && B->g_b == b && B->g_x == x && B->g_tol == tol && B->g_maxiter == maxiter;
    if (!same) {
        if (B->gexec) cudaGraphExecDestroy(B->gexec);
        if (B->graph) cudaGraphDestroy(B->graph);
        B->gexec = nullptr;
        B->graph = nullptr;
        BatchParams P = B->params;
        P.tol = tol;
        P.maxiter = maxiter;
        cudaStream_t s = B->stream;
        MF_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaMemsetAsync(B->d_queue.p, 0, sizeof(unsigned), s);
        cudaMemsetAsync(B->d_sync.p, 0, sizeof(uint32_t) * B->d_sync.n, s);
        cudaMemsetAsync(B->ws.p, 0, sizeof(double) * 5 * B->ws_rows, s);
        k_scatter<<<std::min(B->count, 1024), 256, 0, s>>>(b, B->ws.p, B->d_voff.p, B->d_poff.p, B->d_n.p,
                                                          B->count, B->ws_rows, 0);
        const int lrc = launch_batch(P, B->grid, s);
        if (lrc) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);  // leave the stream usable
            if (g) cudaGraphDestroy(g);
            return lrc;
        }
        k_gather<<<std::min(B->count, 1024), 256, 0, s>>>(x, B->ws.p, B->d_voff.p, B->d_poff.p, B->d_n.p,
                                                         B->count, B->ws_rows, 1);
        MF_CUDA_TRY(cudaStreamEndCapture(s, &B->graph));
        MF_CUDA_TRY(cudaGraphInstantiate(&B->gexec, B->graph, 0));
        B->g_b = b;
        B->g_x = x;
        B->g_tol = tol;
        B->g_maxiter = maxiter;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, B->stream);
    MF_CUDA_TRY(cudaGraphLaunch(B->gexec, B->stream));
    cudaEventRecord(e1, B->stream);
    MF_CUDA_TRY(cudaEventSynchronize(e1));
    float f = 0;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = f;
    std::vector<uint32_t> gw((size_t)B->ngroups * group_sync_words(B->gs));
    MF_CUDA_TRY(cudaMemcpy(gw.data(), B->d_sync.p, sizeof(uint32_t) * gw.size(), cudaMemcpyDeviceToHost));
    for (int g = 0; g < B->ngroups; ++g) {
        const uint32_t err = gw[(size_t)g * group_sync_words(B->gs) + SYNC_ERROR];
        if (err) return (int)err;
    }
    return MF_OK;
}

int mf_batch_solve_cg_each_dev(mf_batch *B, const double *b, double *x, double tol, int maxiter, double *ms) {
    if (!B || !b || !x) return MF_ERR_ARG;
    if ((int)B->full.size() != B->count) {
        set_last_error("batch created without the per-system layouts");
        return MF_ERR_ARG;
    }
    MF_CUDA_TRY(cudaSetDevice(B->device));
    mf_options opt;
    mf_options_default(&opt);
    opt.check_true_residual = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    // x0 = 0, as in the batched solve
    MF_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * B->total_rows, 0));
    std::vector<BatchResult> res(B->count);
    for (int s = 0; s < B->count; ++s) {
        mf_result R;
        const int rc = mf_solve_cg_dev(B->full[s], b + B->poff[s], x + B->poff[s], tol, maxiter, &opt, &R);
        if (rc != MF_OK && rc != MF_ERR_NOT_CONVERGED) return rc;
        res[s].iterations = R.iterations;
        res[s].status = R.status;
        res[s].rr = R.rel_residual_rec * R.rel_residual_rec;
        res[s].bb = 1.0;
    }
    cudaEventRecord(e1, 0);
    MF_CUDA_TRY(cudaEventSynchronize(e1));
    float f = 0;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = f;
    MF_CUDA_TRY(cudaMemcpy(B->d_res.p, res.data(), sizeof(BatchResult) * B->count, cudaMemcpyHostToDevice));
    return MF_OK;
}

int mf_batch_results(const mf_batch *B, int *iterations, int *status, double *rel_residual) {
    if (!B) return MF_ERR_ARG;
    std::vector<BatchResult> res(B->count);
    MF_CUDA_TRY(cudaMemcpy(res.data(), B->d_res.p, sizeof(BatchResult) * B->count, cudaMemcpyDeviceToHost));
    for (int s = 0; s < B->count; ++s) {
        if (iterations) iterations[s] = res[s].iterations;
        if (status) status[s] = res[s].status;
        if (rel_residual) rel_residual[s] = res[s].bb > 0 ? std::sqrt(res[s].rr / res[s].bb) : std::sqrt(res[s].rr);
    }
    return MF_OK;
}

int mf_batch_info(const mf_batch *B, long long *total_rows, long long *total_nnz, int *grid) {
    if (!B) return MF_ERR_ARG;
    if (total_rows) *total_rows = B->total_rows;
    if (total_nnz) *total_nnz = B->total_nnz;
    if (grid) *grid = B->grid;
    return MF_OK;
}

void mf_batch_free(mf_batch *B) { delete B; }

}  // extern "C"
