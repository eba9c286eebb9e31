/*
 * mf_oracle.h -- CPU oracle of the tiled CG / BiCGSTAB path.
 *
 * TEST INFRASTRUCTURE ONLY. This library checks the CUDA path: only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py
 * may load it. The product path (libmf.so) never links or calls it.
 *
 * Each function restates an algorithm of the Mille-feuille reference in
 * plain C; the file:line it follows is given beside it. The restatement is
 * pinned against the reference's own headers compiled unmodified
 * (oracle/ref_harness.cpp -> oracle/_ref/libmfref.so) and against the
 * golden fixtures in tests/golden/ that harness produced.
 */
#ifndef MF_ORACLE_H_
#define MF_ORACLE_H_
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int rowA, colA, tilem, tilen, tilenum, csrsize, csrptrlen;
    int *tile_ptr, *tile_columnidx, *tile_nnz, *blknnz, *csr_offset, *csrptr_offset;
    char *Format;
    unsigned char *blknnznnz;
    double *Blockcsr_Val;
    float *Blockcsr_Val_Low;
    unsigned char *Tile_csr_Col, *Blockcsr_Ptr, *csr_compressedIdx;
} mfo_tiles;

/* csr2block.h:267-422 (Tile_create, steps 1-4 and the scans). */
int mfo_tile_create(int rowA, int colA, const int *rp, const int *ci, const double *val,
                    mfo_tiles *t);
void mfo_tiles_free(mfo_tiles *t);

/* blockspmv_cpu.h:2-112, with the intra-tile column taken from Tile_csr_Col
 * (the reference decodes csr_compressedIdx, which Tile_create leaves zero).
 * Writes y[0..rowA), ptroffset1/2[tilenum] and *rowblkblock. */
void mfo_blockspmv(const mfo_tiles *t, const double *x, double *y, int *ptroffset1,
                   int *ptroffset2, int *rowblkblock);

/* Row compression, Mille-feuille_CG_NVIDIA.cu:4154-4213. Sizes:
 * nonzero_row_new tilenum+1, tile_rowidx tilenum, block_signal tilem+1;
 * blockrowid_new / blockcsr_ptr_new are allocated (cnt+1) and returned. */
int mfo_row_compress(const mfo_tiles *t, int *nonzero_row_new, int *tile_rowidx,
                     int *block_signal, unsigned char **blockrowid_new,
                     unsigned char **blockcsr_ptr_new);

/* Two-pointer warp work split, Mille-feuille_CG_NVIDIA.cu:4216-4484.
 * Returns index (number of warp units). Arrays may be NULL (count only). */
int mfo_balance_twopointer(const mfo_tiles *t, int block_nnz, int block_per_warp,
                           int *balance_tile_ptr_new, int *index_each_block_new,
                           int *row_each_block_new, int *non_each_block_new);

/* Plain CSR SpMV in CSR order (FP64). */
void mfo_csr_spmv(int n, const int *rp, const int *ci, const double *v, const double *x,
                  double *y);

/* Deterministic dot product: 64 fixed chunks summed in order. */
double mfo_dot(int n, const double *a, const double *b);

/* CG of Mille-feuille_CG_NVIDIA.cu:722-804 (alpha = snew/(d.q), x += alpha d,
 * r -= alpha q, snew = r.r, beta = snew/sold, d = r + beta d) run to
 * ||r||/||b|| <= tol with the tiled SpMV. x holds x0 on entry.
 * Returns iterations; *rel_res = final recursive relative residual. */
int mfo_cg(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter,
           double *rel_res);

/* One column of the FP32-direction multi-right-hand-side CG: d and q = A d
 * rounded to FP32, x, r, dots and scalars FP64, r replaced by b - A x every
 * `replace` iterations and when the recursive residual reaches tol (the stop
 * test uses that true residual); a replacement whose true residual norm is
 * more than twice the recursive one restarts the recurrence (d = r). */
int mfo_cg_dir32(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter, int replace,
                 double *rel_res);

/* Jacobi-preconditioned CG (KSPCG + PCJACOBI, PETSc/src/ksp/ksp/impls/cg/cg.c:112-380);
 * diag[i] = a_ii. Stops on the unpreconditioned ||r|| / ||b|| <= tol. */
int mfo_pcg_jacobi(const mfo_tiles *t, const double *diag, const double *b, double *x, double tol,
                   int maxiter, double *rel_res);

/* BiCGSTAB of Mille-feuille_BiCGSTAB_NVIDIA.cu:787-1061 / cuSPARSE_BiCGSTAB.cu:579-666. */
int mfo_bicgstab(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter,
                 double *rel_res);

/* OCP FP8 E4M3 (bias 7, max 448, no inf, NaN = S.1111.111), round to nearest
 * even, saturating to +-448. */
uint8_t mfo_fp8_e4m3_encode(double v);
double mfo_fp8_e4m3_decode(uint8_t b);
/* IEEE binary16, round to nearest even (overflow -> inf). */
uint16_t mfo_fp16_encode(double v);
double mfo_fp16_decode(uint16_t h);

/* Per-tile power-of-two scale used for FP16 / FP8 tiles (1 for others). */
double mfo_tile_scale(int prec, double maxabs);

/* Mixed-precision tiled SpMV: tile t stored at prec[t] (0 fp64, 1 fp32,
 * 2 fp16, 3 fp8) with a power-of-two scale for fp16 / fp8; diagonal entries
 * never below fp32; the diagonal of a diagonally dominant Z-row absorbs its
 * row's rounding (row sums preserved); FP64-class entries summed per tile in
 * FP64, the others in one FP32 accumulator by class (fp32, fp16, fp8). The
 * full definition is in mf_oracle.c. */
void mfo_mixed_spmv(const mfo_tiles *t, const unsigned char *prec, const double *x,
                    double *y);

/* MLP 6->64->64->4 (ReLU), FP32: forward logits, and one SGD step of the
 * softmax cross-entropy loss (mean over the batch). Weights row-major
 * W1[64][6], b1[64], W2[64][64], b2[64], W3[4][64], b3[4]. Gradients are
 * written to g* (same layout). Returns the loss. */
float mfo_mlp_forward(const float *W1, const float *b1, const float *W2, const float *b2,
                      const float *W3, const float *b3, const float *x, int batch,
                      float *logits);
float mfo_mlp_grad(const float *W1, const float *b1, const float *W2, const float *b2,
                   const float *W3, const float *b3, const float *x, const int *labels,
                   int batch, float *gW1, float *gb1, float *gW2, float *gb2, float *gW3,
                   float *gb3);

/* A generated system: 0-based CSR (columns ascending), right-hand side b and,
 * where the workload defines one, the exact solution x* (else NULL). All
 * arrays are malloc'ed; mfo_system_free releases them. */
typedef struct {
    int n, nnz;
    int *row_ptr, *col_idx;
    double *val, *b, *xstar;
} mfo_system;

/* The synthetic workloads (oracle/workloads.c). Return 0, or -1 on bad
 * arguments / allocation failure. */
int mfo_gen_poisson2d(int N, mfo_system *m);
int mfo_gen_convdiff3d(int N, double vx, double vy, double vz, uint64_t seed, mfo_system *m);
int mfo_gen_varpoisson3d(int N, double klo, double khi, uint64_t seed, mfo_system *m);
void mfo_system_free(mfo_system *m);

/* OpenMP threads of the calling thread's later parallel regions (n > 0;
 * n <= 0 leaves them); returns the count now in effect. A launcher such as
 * torchrun sets OMP_NUM_THREADS=1 per process, which a timed CPU baseline
 * overrides here to use every host core it may run on. */
int mfo_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
