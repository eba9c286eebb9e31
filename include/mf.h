/*
 * mf.h -- C ABI of the B200-native tiled CG / BiCGSTAB solver (libmf.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an int status (MF_OK = 0, negative = error, see mf_status_str).
 * Host pointers are named *_host, device pointers *_dev.
 *
 * Reference interfaces replaced (paths are inside the Mille-feuille tree):
 *   cg_solve_inc(...)        Performance-Comparison/Mille-feuille_CG_NVIDIA.cu:3979
 *   bicgstab(...)            Performance-Comparison/Mille-feuille_BiCGSTAB_NVIDIA.cu:1476
 *   Tile_create(...)         Performance-Comparison/csr2block.h:267
 *   blockspmv_cpu(...)       Performance-Comparison/blockspmv_cpu.h:2   (SpMV part)
 *   read_Dmatrix_32(...)     Performance-Comparison/biio2.0/src/biio.h:153
 *   binary_read_csr / binary_write_csr   biio2.0/src/biio.h:22 / :74
 *   row compression          Mille-feuille_CG_NVIDIA.cu:4154-4213
 *   two-pointer balance      Mille-feuille_CG_NVIDIA.cu:4216-4484
 */
#ifndef MF_H_
#define MF_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
    MF_OK = 0,
    MF_ERR_ARG = -1,           /* invalid argument / precondition           */
    MF_ERR_CUDA = -2,          /* a CUDA runtime call failed                */
    MF_ERR_TIMEOUT = -3,       /* a bounded device wait ran out             */
    MF_ERR_NOT_CONVERGED = -4, /* maxiter reached above tolerance           */
    MF_ERR_BREAKDOWN = -5,     /* zero/NaN denominator in the recurrence    */
    MF_ERR_IO = -6,            /* file could not be read / parsed           */
    MF_ERR_NOMEM = -7,         /* host or device allocation failed          */
    MF_ERR_RESIDENCY = -8,     /* persistent grid cannot be co-resident     */
    MF_ERR_UNSUPPORTED = -9    /* feature not available for this input      */
};
const char *mf_status_str(int status);
/* Text of the last error recorded by the library (thread-unsafe, for logs). */
const char *mf_last_error(void);

/* ---- precision ------------------------------------------------------- */
enum { MF_PREC_FP64 = 0, MF_PREC_FP32 = 1, MF_PREC_FP16 = 2, MF_PREC_FP8 = 3 };
/* Mixed modes apply to mf_solve_cg* and mf_solve_bicgstab*. A mixed layout
 * whose levels hold no tile below FP64 (every row block oversize, for
 * example) is solved by the FP64 kernels.                                   */
enum {
    MF_MODE_FP64 = 0,        /* every tile FP64, exact blockspmv order          */
    MF_MODE_MIXED_RULE = 1,  /* per-tile precision from the precision rule:     */
                             /* FP16 with row-sum compensation on diagonally    */
                             /* dominant Z-row blocks, the magnitude rule else  */
    MF_MODE_MIXED_MLP = 2,   /* per-tile precision from the learned selector    */
    MF_MODE_FIXED = 3        /* every tile at options.fixed_precision           */
};

/* ---- host CSR matrix (0-based, int32) -------------------------------- */
typedef struct {
    int n;              /* rows                                  */
    int ncols;          /* columns                               */
    int nnz;            /* row_ptr[n]                            */
    const int *row_ptr; /* n+1, row_ptr[0] == 0                  */
    const int *col_idx; /* nnz                                   */
    const double *val;  /* nnz                                   */
} mf_csr;

/* ---- options ---------------------------------------------------------- */
typedef struct {
    int precision_mode;      /* MF_MODE_*                                      */
    int fixed_precision;     /* MF_PREC_* used by MF_MODE_FIXED                */
    int replace_every;       /* true-residual replacement period of the mixed
                                precision modes (FP64 mode never replaces)    */
    int ctas_per_sm;         /* persistent CTAs per SM, 0 = autotune           */
    int rb_per_slab;         /* row blocks per slab, 0 = default (60 at most)  */
    int slab_bytes;          /* max bytes of one streamed slab, 0 = default    */
    double timeout_s;        /* limit of every device spin-wait, 0 = 2 s       */
    int check_true_residual; /* confirm convergence with b - A x (default 1)   */
    int fixed_iterations;    /* >0: run exactly this many iterations           */
    double mixed_tau;        /* magnitude-rule tolerance scale, 0 = default    */
    int device;              /* CUDA device ordinal                            */
    int reserved[7];         /* reserved[0] == 0x5741: test hook, the CG kernel
                                first waits on a flag nothing sets, so the
                                bounded wait must end it with MF_ERR_TIMEOUT;
                                reserved[1] = N > 0: trace the first N CG
                                iterations (see mf_trace); reserved[2] = 1:
                                mixed layouts use the classic two-reduction
                                CG instead of the single-reduction
                                (Chronopoulos-Gear) form; reserved[3] = 1:
                                L2 prefetch of slabs 2*STAGES ahead of the
                                copy ring (off by default: on B200 it cost
                                2-10 us per SpMV; read at encode for
                                mf_spmv, at solve for the solvers);
                                reserved[4] = CTAs per system group of
                                mf_batch_create (0 = 4); reserved[5] = 1:
                                the CG kernels (FP64 and single-reduction
                                mixed) keep x and r in global memory
                                instead of tensor memory;
                                reserved[6] = N > 0: reference iteration
                                count for the learned selector's fallback   */
} mf_options;
void mf_options_default(mf_options *opt);

/* ---- solve result ----------------------------------------------------- */
typedef struct {
    int status;              /* MF_OK or MF_ERR_*                              */
    int iterations;          /* iterations executed                            */
    int replacements;        /* true-residual replacements performed           */
    int level_switches;      /* precision tightenings performed                */
    double rel_residual_true;/* ||b - A x|| / ||b|| recomputed in FP64         */
    double rel_residual_rec; /* recursive residual ||r_k|| / ||b||             */
    double time_ms;          /* device time of the solve launch                */
    double spmv_bytes;       /* algorithmic bytes of one SpMV (current layout) */
    double spmv_bytes_fp64;  /* algorithmic bytes of one FP64 SpMV             */
    double tile_frac[4];     /* fraction of tiles per MF_PREC_* at the end     */
    int error_site;          /* device error site code (0 = none)              */
    int iters_fp64;          /* iterations whose SpMV used the FP64 layout     */
    int iters_level[3];      /* iterations per mixed-precision level           */
    double spmv_bytes_level[3]; /* algorithmic bytes of one SpMV per level     */
    double total_bytes;      /* algorithmic bytes of the whole solve: every
                                SpMV (replacements included) + the vector
                                bytes the launched kernel moves per row and
                                iteration (56 with vectors in global memory;
                                28 mixed and 32 FP64 CG, 40 Jacobi PCG with
                                x and r in tensor memory; 88 BiCGSTAB)        */
    int fell_back_fp64;      /* 1 if a low-precision level let the true
                                residual grow and the solve finished on the
                                FP64 layout                                   */
    int selector_fallback;   /* MF_MODE_MIXED_MLP: 1 if the learned selector's
                                solve missed the tolerance, fell back to FP64
                                or ran > 10% over mf_options.reserved[6]
                                iterations, and the magnitude rule solved it  */
} mf_result;

/* ---- opaque handles --------------------------------------------------- */
typedef struct mf_matrix mf_matrix; /* host CSR (+ optional vectors)          */
typedef struct mf_tiles mf_tiles;   /* device tile matrix + solver layout     */

/* ---- host matrices: generators, readers, writers ---------------------- */
/* 2D 5-point Laplacian on an N x N grid, b = A * ones.                       */
int mf_gen_poisson2d(int N, mf_matrix **out);
/* 3D 7-point upwind convection-diffusion, D = 1, h = 1, v = (vx,vy,vz),
 * b ~ U[-1,1] drawn from seed.                                               */
int mf_gen_convdiff3d(int N, double vx, double vy, double vz, uint64_t seed,
                      mf_matrix **out);
/* 3D 7-point variable-coefficient Poisson, face coefficients log-uniform in
 * [klo, khi], x* ~ U[0,1] (same stream), b = A x*.                           */
int mf_gen_varpoisson3d(int N, double klo, double khi, uint64_t seed,
                        mf_matrix **out);
/* Random sparse SPD system (4..12 off-diagonals per row, U[-1,0], symmetrised,
 * diagonal = row sum of |off| + 0.01), b ~ U[-1,1].                          */
int mf_gen_spd_random(int n, uint64_t seed, mf_matrix **out);
/* Sizes of a batch: count values log-uniform in [lo, hi].                    */
int mf_gen_batch_sizes(int count, int lo, int hi, uint64_t seed, int *sizes_host);
/* Matrix Market reader with read_Dmatrix_32 semantics (0-based, symmetric
 * and hermitian expanded, file order kept within rows).                      */
int mf_read_mtx(const char *path, mf_matrix **out);
/* .cbd binary CSR (int rows, int cols, int64 nnz, int64 row_ptr[rows+1],
 * int col_idx[nnz], double val[nnz]).                                        */
int mf_read_cbd(const char *path, mf_matrix **out);
int mf_write_cbd(const mf_matrix *m, const char *path);
int mf_matrix_from_csr(int n, int ncols, int nnz, const int *row_ptr,
                       const int *col_idx, const double *val, mf_matrix **out);
int mf_matrix_info(const mf_matrix *m, int *n, int *ncols, int *nnz,
                   int *has_b, int *has_xstar);
int mf_matrix_csr(const mf_matrix *m, mf_csr *csr);      /* borrowed views */
const double *mf_matrix_b(const mf_matrix *m);            /* NULL if none   */
const double *mf_matrix_xstar(const mf_matrix *m);        /* NULL if none   */
int mf_matrix_set_b(mf_matrix *m, const double *b_host);
void mf_matrix_free(mf_matrix *m);

/* ---- tile encoder (GPU csr2block) ------------------------------------- */
/* Upload a host CSR and encode it on the GPU into 16x16 tiles (the
 * Tile_create layout) plus the solver's slab layout.                         */
int mf_encode(const mf_csr *A, const mf_options *opt, mf_tiles **out);
/* Same, from CSR arrays already on the device (no host copies).              */
int mf_encode_dev(int n, int ncols, int nnz, const int *row_ptr_dev,
                  const int *col_idx_dev, const double *val_dev,
                  const mf_options *opt, mf_tiles **out);
void mf_free(mf_tiles *t);

typedef struct {
    int rowA, colA, tilem, tilen, tilenum, csrsize, csrptrlen;
    int cnt_non_new;       /* nonzero_row_new[tilenum] (row compression)     */
    int nslabs, nctas;     /* solver layout                                  */
    long long layout_bytes;/* bytes of the slab layout (current level)       */
    double encode_ms;      /* device time of the encoder                     */
    double layout_ms;      /* host + device time of the slab layout build    */
} mf_tile_info;
int mf_tiles_info(const mf_tiles *t, mf_tile_info *info);

/* Host copies of the Tile_create arrays (caller allocates, NULL = skip).
 * Sizes: tile_ptr tilem+1; tile_columnidx tilenum; tile_nnz, blknnz,
 * csr_offset, csrptr_offset tilenum+1; Format tilenum; blknnznnz tilenum+1;
 * Blockcsr_Val, Blockcsr_Val_Low, Tile_csr_Col csrsize; Blockcsr_Ptr
 * csrptrlen; csr_compressedIdx ceil(csrsize/2) (always zero, as in the
 * reference). Derived arrays: ptroffset1, ptroffset2, tile_rowidx tilenum;
 * nonzero_row_new tilenum+1; blockrowid_new, blockcsr_ptr_new
 * cnt_non_new+1; block_signal tilem+1.                                       */
typedef struct {
    int *tile_ptr, *tile_columnidx, *tile_nnz, *blknnz, *csr_offset,
        *csrptr_offset;
    char *Format;
    unsigned char *blknnznnz;
    double *Blockcsr_Val;
    float *Blockcsr_Val_Low;
    unsigned char *Tile_csr_Col, *Blockcsr_Ptr, *csr_compressedIdx;
    int *ptroffset1, *ptroffset2, *tile_rowidx, *nonzero_row_new, *block_signal;
    unsigned char *blockrowid_new, *blockcsr_ptr_new;
} mf_tile_arrays;
int mf_tiles_export(const mf_tiles *t, mf_tile_arrays *host);

/* Per-tile precision codes (MF_PREC_*) and scales of the current layout.    */
int mf_tiles_precisions(const mf_tiles *t, unsigned char *prec_host,
                        float *scale_host);
/* Re-encode the solver layout with explicit per-tile precisions.            */
int mf_tiles_set_precisions(mf_tiles *t, const unsigned char *prec_host);

/* Two-pointer warp work split of the reference driver (compatibility
 * export; the solver itself uses an nnz-balanced contiguous partition).
 * Returns the number of warp units in *index; arrays sized tilenum+1 and
 * index+1 (call once with NULL arrays to get *index).                       */
int mf_balance_twopointer(const mf_tiles *t, int block_nnz, int block_per_warp,
                          int *index, int *balance_tile_ptr_new,
                          int *index_each_block_new, int *row_each_block_new,
                          int *non_each_block_new);

/* ---- SpMV ------------------------------------------------------------- */
/* y = A x with the tiled kernel. x_dev has ncols entries, y_dev rowA.
 * FP64 layout: bit-identical to blockspmv_cpu's summation order.
 * stream: a cudaStream_t (NULL = default stream).                           */
int mf_spmv(const mf_tiles *t, const double *x_dev, double *y_dev, void *stream);
/* Same with host buffers (copies included).                                 */
int mf_spmv_host(const mf_tiles *t, const double *x_host, double *y_host);
/* Device time (ms) of `reps` back-to-back tiled SpMVs on the given vectors. */
int mf_spmv_bench(const mf_tiles *t, const double *x_dev, double *y_dev,
                  int reps, double *ms_per_spmv, double *alg_bytes);
/* Same two calls on mixed-precision layout `level` (-1 = FP64 layout).      */
int mf_spmv_level(const mf_tiles *t, int level, const double *x_dev, double *y_dev);
int mf_spmv_bench_level(const mf_tiles *t, int level, const double *x_dev,
                        double *y_dev, int reps, double *ms_per_spmv,
                        double *alg_bytes);

/* ---- solvers ---------------------------------------------------------- */
/* Single persistent-kernel CG. b and x (x0 in, solution out) on the host.  */
int mf_solve_cg(mf_tiles *t, const double *b_host, double *x_host, double tol,
                int maxiter, const mf_options *opt, mf_result *res);
/* Same with device vectors (n entries each).                                */
int mf_solve_cg_dev(mf_tiles *t, const double *b_dev, double *x_dev, double tol,
                    int maxiter, const mf_options *opt, mf_result *res);
/* Jacobi-preconditioned CG (M = diag(A), the "jpcg" runs of the reference's
 * PETSc comparison: KSPCG + PCJACOBI, PC/PETSc/src/ksp/ksp/impls/cg/cg.c),
 * FP64 layout, one persistent kernel; stops on the unpreconditioned
 * ||b - A x|| / ||b|| <= tol like mf_solve_cg. precision_mode is ignored.   */
int mf_solve_pcg(mf_tiles *t, const double *b_host, double *x_host, double tol,
                 int maxiter, const mf_options *opt, mf_result *res);
int mf_solve_pcg_dev(mf_tiles *t, const double *b_dev, double *x_dev,
                     double tol, int maxiter, const mf_options *opt,
                     mf_result *res);
/* Single persistent-kernel BiCGSTAB.                                         */
int mf_solve_bicgstab(mf_tiles *t, const double *b_host, double *x_host,
                      double tol, int maxiter, const mf_options *opt,
                      mf_result *res);
int mf_solve_bicgstab_dev(mf_tiles *t, const double *b_dev, double *x_dev,
                          double tol, int maxiter, const mf_options *opt,
                          mf_result *res);
/* mf_solve_cg_dev without device allocation (no counterpart in the
 * reference): the FP64 CG with all of its scratch in a static device array,
 * for callers that cannot allocate at solve time (their allocator holds the
 * free HBM, or they can't afford cudaMalloc's device-wide synchronization).
 * Limit: n rounded up to 16 <= MF_NOALLOC_MAX_ROWS, else MF_ERR_ARG.
 * Always FP64 (mixed layouts unused); time_ms is 0; reserved[1] is ignored.
 * The first call on a device sets up (looks up the scratch address): make it
 * before any stream capture. The address is kept for the life of the
 * process, so cudaDeviceReset on that device makes later calls invalid.
 * One scratch per device: overlapping calls on one device race and must be
 * serialized by the caller.                                                */
#define MF_NOALLOC_MAX_ROWS 131072
int mf_solve_cg_dev_noalloc(mf_tiles *t, const double *b_dev, double *x_dev,
                            double tol, int maxiter, const mf_options *opt,
                            mf_result *res);
/* Self-check of the slab planner (no counterpart in the reference; the
 * reference's two-pointer split, Mille-feuille_CG_NVIDIA.cu:4216-4484, is
 * host code). Layouts are planned on the GPU; while the check is on (on = 1;
 * on = -1 only reads the counters), every layout built is planned again by
 * the host planner and each plan, segment and run is compared. Returns the
 * previous setting; *checked = layouts compared, *mismatches = differences
 * found since the check was last switched. Process-wide, not thread-safe. */
int mf_check_planner(int on, long long *checked, long long *mismatches);
/* Phase timestamps (ns, %globaltimer of CTA 0) of the last traced CG solve:
 * out[8*i + s] for iteration i, slot s = 0 iteration start, 1 halo ready,
 * 2 SpMV done, 3 alpha known, 4 r updated, 5 beta known, 6 x / d published.
 * Returns the number of iterations written.                                 */
int mf_trace(const mf_tiles *t, unsigned long long *out, int max_iters);
/* ||b - A x|| / ||b|| with the FP64 tiled SpMV (device vectors).             */
int mf_true_residual(mf_tiles *t, const double *b_dev, const double *x_dev,
                     double *rel);

/* ---- CG on up to 16 right-hand sides at once (no reference counterpart) -- */
/* k <= 16 independent CG recurrences (each its own alpha, beta and stop
 * test, the reference's CG) sharing every matrix-panel product, so the
 * matrix streams once per iteration for all of them. B, X: n x k column-major
 * (column j = right-hand side j; X holds x0 on entry). The SpMM keeps
 * blockspmv_cpu's order per column; the CSR columns must ascend within each
 * row. The _dev variant checks the CSR on the GPU before use (row_ptr[0]
 * == 0, row_ptr non-decreasing, columns in [0, n) and ascending) and returns
 * MF_ERR_ARG otherwise; it reads row_ptr[n] entries of col_idx_dev/val_dev.
 * Per right-hand side: iterations and final relative residual;
 * *time_ms = device time of the whole call. MF_ERR_NOT_CONVERGED if any
 * column missed tol within maxiter.                                          */
int mf_solve_cg_multi(const mf_csr *A, int k, const double *B_host,
                      double *X_host, double tol, int maxiter,
                      int *iterations, double *rel_residual, double *time_ms);
int mf_solve_cg_multi_dev(int n, const int *row_ptr_dev, const int *col_idx_dev,
                          const double *val_dev, int k, const double *B_dev,
                          double *X_dev, double tol, int maxiter,
                          int *iterations, double *rel_residual,
                          double *time_ms);
/* Panel precision of the multi-right-hand-side CG. MF_PANEL_FP32 (what the
 * two calls above use): search directions P and products Q = A P stored in
 * FP32 (the product summed in FP64, then rounded), x, r, dots and scalars
 * FP64, r replaced by b - A x every 50 iterations and whenever a column's
 * recursive residual reaches tol; a column converges on that true residual
 * (rel_residual is then the true one), and a replacement whose true residual
 * norm exceeds twice the recursive one restarts that column (p = r). One persistent launch per solve.
 * MF_PANEL_FP64: every panel FP64; each column is exactly the single
 * right-hand-side FP64 CG (recursive residual), five launches an iteration. */
#define MF_PANEL_FP64 0
#define MF_PANEL_FP32 1
int mf_solve_cg_multi_ex(int panel, const mf_csr *A, int k,
                         const double *B_host, double *X_host, double tol,
                         int maxiter, int *iterations, double *rel_residual,
                         double *time_ms);
int mf_solve_cg_multi_dev_ex(int panel, int n, const int *row_ptr_dev,
                             const int *col_idx_dev, const double *val_dev,
                             int k, const double *B_dev, double *X_dev,
                             double tol, int maxiter, int *iterations,
                             double *rel_residual, double *time_ms);

/* ---- autotuner (no reference counterpart) ------------------------------- */
/* The tile shape is the reference's 16x16 (the bit-exact contract); what is
 * tuned is the slab geometry of the solver layouts: bytes per slab (24, 32,
 * 40 KB: the copy-ring stage) x row blocks per slab (16, 30, 60). Every
 * candidate re-plans the handle's FP64 and mixed layouts (no re-encode) and
 * times the SpMV the solvers run (the mixed level 0 when present, else
 * FP64) over `reps` launches; the handle keeps the fastest. Results do not
 * depend on the choice (the SpMV is bit-exact for every geometry).           */
typedef struct {
    int slab_bytes, rb_per_slab;   /* the choice (now in the handle)           */
    double ms_best, ms_default;    /* SpMV time of the choice / of the default */
    int candidates;
    int cand_slab_bytes[16], cand_rb_per_slab[16];
    double cand_ms[16];
} mf_tune_result;
int mf_tiles_autotune(mf_tiles *t, int reps, mf_tune_result *out);

/* ---- memory-cost report (Memory-Cost/memory_Mille_feillue.cu:659-921) ---- */
typedef struct {
    double csr_bytes;            /* CSR as the cuSPARSE study counts it:
                                    (n+1)*4 + nnz*(4 + 8)                      */
    double tile_index_bytes;     /* the reference tally of the tile metadata,
                                    row compression and column bytes          */
    double tile_value_bytes[4];  /* value bytes per precision MF_PREC_* of the
                                    level-0 mix (all FP64 without a mixed
                                    layout)                                    */
    double tile_total_bytes;     /* index + value bytes (the study's memory_MB
                                    x 2^20)                                    */
    double slab_bytes_fp64;      /* this library's FP64 slab layout           */
    double slab_bytes_mixed;     /* its mixed layouts, all levels             */
    double workspace_bytes;      /* solver workspace currently held           */
    double device_bytes;         /* every device allocation of the handle     */
} mf_memory_cost;
int mf_memory_report(const mf_tiles *t, mf_memory_cost *out);

/* ---- learned precision selector (MF_MODE_MIXED_MLP) --------------------- */
/* An MLP 6 -> 64 -> 64 -> 4 (ReLU) over per-tile features; its classes are
 * the tile precisions MF_PREC_*. Features: f0 = log10 max|a_ij|/sqrt(a_ii
 * a_jj) over the tile, f1 = log10 max|a|/min|a| over the tile, f2 = log10
 * of the matrix nnz, f3 = diagonal tile, f4 = log10 max|a|/min|a| over the
 * matrix, f5 = log10 of the relative residual at which the precision is
 * used. Weights (MF_MLP_WEIGHTS floats): W1[64][6], b1[64], W2[64][64],
 * b2[64], W3[4][64], b3[4]. Inference rounds them to BF16 and accumulates in
 * FP32. The reference has no counterpart (it stores every tile in FP64).   */
#define MF_MLP_WEIGHTS 4868
int mf_mlp_set_weights(const float *w_host);  /* process-wide; NULL clears   */
int mf_mlp_get_weights(float *w_host);        /* MF_ERR_ARG when none set    */
/* Features f0..f4 of every tile, feat[6*t + k] (f5 = 0).                     */
int mf_tiles_features(const mf_tiles *t, float *feat_host);
/* Selector classes at nlev residual levels: prec[l*tilenum + t].            */
int mf_tiles_select_mlp(const mf_tiles *t, int nlev, const double *rel_res,
                        unsigned char *prec_host);
/* The training kernels (device pointers): logits[4n] of n samples x[6n];
 * gradient g of the mean softmax cross-entropy (*loss on the host); `steps`
 * Adam steps, step i on the samples [i*batch mod n, +batch).                */
int mf_mlp_forward_dev(const float *w, const float *x, int n, int bf16,
                       float *logits);
int mf_mlp_grad_dev(const float *w, const float *x, const int *labels, int n,
                    float *g, float *loss);
int mf_mlp_train_dev(float *w, const float *x, const int *labels, int n,
                     int steps, int batch, float lr, float *loss);

/* ---- batched solve of many independent systems ------------------------- */
/* Encodes `count` square systems (host CSR) for one persistent launch. The
 * grid is split into groups of opt->reserved[4] CTAs (0 = 4); each group
 * solves whole systems taken from a device queue, largest first, with
 * reductions local to the group. with_baseline != 0 also builds whole-GPU
 * layouts for mf_batch_solve_cg_each_dev (one launch per system).          */
typedef struct mf_batch mf_batch;
int mf_batch_create(int count, const mf_csr *systems, const mf_options *opt,
                    int with_baseline, mf_batch **out);
/* FP64 CG on every system. b / x: device arrays holding the systems' vectors
 * back to back in creation order (x0 = 0). The solve is captured in a CUDA
 * graph on first use and replayed; *ms = device time of the replay.         */
int mf_batch_solve_cg_dev(mf_batch *B, const double *b_dev, double *x_dev,
                          double tol, int maxiter, double *ms);
/* The same systems with one single-system solver launch each (x0 = 0).      */
int mf_batch_solve_cg_each_dev(mf_batch *B, const double *b_dev, double *x_dev,
                               double tol, int maxiter, double *ms);
/* Per-system iterations, status and recursive relative residual.            */
int mf_batch_results(const mf_batch *B, int *iterations, int *status,
                     double *rel_residual);
/* Totals, and the grid (groups x CTAs per group) of the batched launch.    */
int mf_batch_info(const mf_batch *B, long long *total_rows,
                  long long *total_nnz, int *grid);
void mf_batch_free(mf_batch *B);

/* ---- drop-in replacements of the reference entry points --------------- */
/* Same signature as the reference. n is truncated to a multiple of 16 as
 * the reference's callers do; columns beyond the truncated n are dropped.
 * x is zeroed and overwritten with the solution; *iter receives the
 * iteration count (the reference leaves it untouched). maxiter and
 * threshold (relative residual) are honoured; filename, ori and block_nnz
 * are accepted for signature compatibility.                                 */
void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low,
                  double *x, double *b, int n, int *iter, int maxiter,
                  double threshold, char *filename, int nnzR, int ori,
                  int block_nnz);
/* Returns 0 on convergence, 1 otherwise (reference: 1 when itr >= maxits).
 * rhs is overwritten with A * ones and solved from x = 0, as the reference
 * does; tolerance 1e-10 relative, at most 10000 iterations.                 */
int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x,
             int nnzR, char *filename, int n, int block_nnz);

/* ---- version ------------------------------------------------------------ */
const char *mf_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MF_H_ */
