// Kernel parameter block and host launch entry points of the persistent
// solver kernels (solver.cu). Host-includable (no device code).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "tiles.h"

namespace mf {

constexpr int NWARPS = 15;                 // consumer warps per CTA (2 row blocks each)
constexpr int PRODUCER_WARP = NWARPS;      // one more warp issues the bulk copies
constexpr int NTHREADS = (NWARPS + 1) * 32;
constexpr int KMAX_LAYOUTS = 1 + MF_NLEVELS;
constexpr int FLAG_STRIDE = 8;             // one 32-byte sector per CTA flag
enum { SYNC_ARRIVE = 0, SYNC_ERROR = 32, SYNC_SITE = 33, SYNC_FLAGS = 64 };
inline size_t sync_words(int G) { return (size_t)SYNC_FLAGS + (size_t)G * FLAG_STRIDE + 32; }

inline int slab_area_of(int slab_max) { return (slab_max + 127) & ~127; }
// slab | x window (XSEG_MAX 128-byte segments) | 128 bytes holding the zero slot
inline int stage_stride_of(int slab_max) { return slab_area_of(slab_max) + XSEG_MAX * 128 + 128; }

struct LayoutArgs {
    const uint8_t *slabs;
    const uint8_t *head;
    const int *cta_slab, *cta_rb, *cta_dep;
    int kind;  // LAYOUT_*
    int x32;   // x staged in FP32: the SpMV input is an FP32 vector
};

struct DevResult {
    int iterations, status, replacements, level_switches, final_layout, pad;
    double rr, bb;
    int it_layout[KMAX_LAYOUTS];  // iterations run with each layout
};

struct KParams {
    LayoutArgs lay[KMAX_LAYOUTS];
    int nlay, start_layout;
    int stage_stride, slab_area;
    int rowA, tilem;
    const int *tile_ptr, *tile_col, *tile_off, *csrptr_off;
    const uint8_t *ptr;
    const double *val;
    const uint8_t *col;
    uint64_t limit_ns;
    uint32_t *sync;
    double *partial;
    double *x, *r, *d, *q, *s, *t, *rh;
    float *p32, *s32;  // FP32 copies of the mixed BiCGSTAB's SpMV inputs
    const double *b;
    double tol;
    int maxiter, fixed_iterations, replace_every;
    int inject_wait;  // test hook: wait once on a flag that nothing sets
    int true_check;   // confirm convergence with the FP64 true residual
    int trace_iters;  // CTA 0 records %globaltimer at each phase boundary
    int prefetch;     // L2 bulk prefetch of slabs ahead of the ring
    uint64_t *trace;  // [trace_iters][8]
    double level_rel[KMAX_LAYOUTS];
    DevResult *res;
};

// ---- batched solve: groups of CTAs, one system per group at a time, from a device queue
struct GTiles {
    const int *tile_ptr, *tile_col, *tile_off, *csrptr_off;
    const uint8_t *ptr;
    const double *val;
    const uint8_t *col;
    int tilem, rowA;
};
struct SysDesc {
    const uint8_t *slabs;  // slab layout of the system for one group of gs CTAs
    const uint8_t *head;   // STAGES issue records per CTA of the group
    const int *cta_slab, *cta_rb, *cta_dep;  // per-rank slab / row-block ranges, halo ranks
    int ns, kind;
    GTiles gt;             // tile arrays (oversize row blocks)
    double *b, *x, *r, *d, *q;  // 16*tilem entries each
    int n16, pad;
};
struct BatchResult {
    int iterations, status;
    double rr, bb;
};
struct BatchParams {
    const SysDesc *sys;
    const int *order;  // systems, largest first
    int count, maxiter, fixed_iterations, pad;
    unsigned *queue;
    double tol;
    int stage_stride, slab_area;
    uint64_t limit_ns;
    int gs, gsync_words;  // CTAs per group; sync words per group
    uint32_t *gsync;      // per group: arrive counter, error word, rank flags
    double *gpartial;     // per group: 2 slots x gs x 4 partial sums
    BatchResult *res;
};
int launch_batch(const BatchParams &B, int grid, cudaStream_t s);

int kernel_config(mf_tiles *t, int *G_out);
void base_params(mf_tiles *t, KParams &P);
// x: FP64, or FP32 (16*tilen entries) when the level's layout stages FP32 x.
int launch_spmv(mf_tiles *t, int level, const void *x, double *y, int reps, cudaStream_t s);
// dst[0..n) = (float)src[0..n), dst[n..npad) = 0.
int launch_to_f32(int n, const double *src, float *dst, size_t npad, cudaStream_t s);
// kind 0 CG, 1 BiCGSTAB, 2 single-reduction CG, 3 the same with x and r in
// TMEM (every CTA's rows <= TMEM_ROWS_MAX), 4 Jacobi-preconditioned CG.
constexpr int TMEM_ROWS_MAX = 128 * 128;
// The TMEM kernel's vector pass copies 12 bytes per own row into the ring.
inline bool tm_vectors_fit(int rows_max, int slab_max) {
    return 12ll * rows_max <= (long long)STAGES * stage_stride_of(slab_max);
}
int launch_solver(mf_tiles *t, int kind, KParams &P, cudaStream_t s);
int launch_residual_norms(int n, const double *b, const double *ax, double *out, cudaStream_t s);
// minv[i] = 1 / diag[i] for i < n (1 where diag is 0), 0 up to npad.
int launch_jacobi_inv(int n, int npad, const double *diag, double *minv, cudaStream_t s);

}  // namespace mf
