/*
 * mf_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see mf_oracle.h).
 *
 * Restatements of the Mille-feuille reference's CPU-side algorithms in plain
 * C. Paths are relative to the reference tree; PC/ = Performance-Comparison/.
 */
#include "mf_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define T16 16

static int rowlen_of(const mfo_tiles *t, int rb) {
    /* csr2block.h:74 -- the last row block may be shorter */
    return rb == t->tilem - 1 ? t->rowA - (t->tilem - 1) * T16 : T16;
}

static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* PC/csr2block.h:267-422. Step 1 counts distinct tile columns per row
 * block, step 2 lists them in ascending order with per-tile nnz and per-row
 * counts, step 3 sets Format = 0 (CSR) and the offsets, step 4 scatters the
 * values row-major inside each tile, CSR order inside each row. The result
 * here is computed with a per-row-block sort instead of tilen-sized flag
 * arrays; the arrays are identical. */
int mfo_tile_create(int rowA, int colA, const int *rp, const int *ci, const double *val,
                    mfo_tiles *t) {
    memset(t, 0, sizeof *t);
    t->rowA = rowA;
    t->colA = colA;
    t->tilem = rowA % T16 == 0 ? rowA / T16 : rowA / T16 + 1;
    t->tilen = colA % T16 == 0 ? colA / T16 : colA / T16 + 1;
    const int tilem = t->tilem;
    t->tile_ptr = (int *)calloc((size_t)tilem + 1, sizeof(int));
    if (!t->tile_ptr) return -1;

    /* step 1: distinct tile columns per row block (csr2block.h:6-41) */
    int maxrb = 0;
    for (int rb = 0; rb < tilem; ++rb) {
        int s = rp[rb * T16], e = rp[rb == tilem - 1 ? rowA : (rb + 1) * T16];
        if (e - s > maxrb) maxrb = e - s;
    }
    int *tcs = (int *)malloc(sizeof(int) * (size_t)(maxrb > 0 ? maxrb : 1));
    for (int rb = 0; rb < tilem; ++rb) {
        int s = rp[rb * T16], e = rp[rb == tilem - 1 ? rowA : (rb + 1) * T16];
        int m = e - s, u = 0;
        for (int k = 0; k < m; ++k) tcs[k] = ci[s + k] / T16;
        qsort(tcs, (size_t)m, sizeof(int), cmp_int);
        for (int k = 0; k < m; ++k)
            if (k == 0 || tcs[k] != tcs[k - 1]) ++u;
        t->tile_ptr[rb] = u;
    }
    /* exclusive scan (utils.h:34-49) */
    {
        int run = 0;
        for (int rb = 0; rb <= tilem; ++rb) {
            int c = t->tile_ptr[rb];
            t->tile_ptr[rb] = run;
            run += c;
        }
    }
    const int tilenum = t->tile_ptr[tilem];
    t->tilenum = tilenum;
    t->tile_columnidx = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    t->tile_nnz = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    unsigned char *tile_csr_ptr = (unsigned char *)calloc((size_t)tilenum * T16 + 1, 1);

    /* step 2 (csr2block.h:43-107) */
    for (int rb = 0; rb < tilem; ++rb) {
        int s = rp[rb * T16], e = rp[rb == tilem - 1 ? rowA : (rb + 1) * T16];
        int m = e - s, u = 0;
        for (int k = 0; k < m; ++k) tcs[k] = ci[s + k] / T16;
        qsort(tcs, (size_t)m, sizeof(int), cmp_int);
        for (int k = 0; k < m; ++k)
            if (k == 0 || tcs[k] != tcs[k - 1]) t->tile_columnidx[t->tile_ptr[rb] + u++] = tcs[k];
        int rl = rowlen_of(t, rb);
        for (int ri = 0; ri < rl; ++ri) {
            int r = rb * T16 + ri;
            for (int p = rp[r]; p < rp[r + 1]; ++p) {
                int jc = ci[p] / T16;
                /* binary search the tile of column block jc */
                int lo = t->tile_ptr[rb], hi = t->tile_ptr[rb + 1] - 1;
                while (lo < hi) {
                    int mid = (lo + hi) / 2;
                    if (t->tile_columnidx[mid] < jc) lo = mid + 1; else hi = mid;
                }
                t->tile_nnz[lo]++;
                tile_csr_ptr[(size_t)lo * T16 + ri]++;
            }
        }
    }
    free(tcs);
    {
        int run = 0;
        for (int k = 0; k <= tilenum; ++k) {
            int c = t->tile_nnz[k];
            t->tile_nnz[k] = run;
            run += c;
        }
    }

    /* step 3 (csr2block.h:109-150) */
    t->Format = (char *)calloc((size_t)tilenum + 1, 1);
    t->blknnz = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    t->blknnznnz = (unsigned char *)calloc((size_t)tilenum + 1, 1);
    t->csr_offset = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    t->csrptr_offset = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    for (int rb = 0; rb < tilem; ++rb)
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            int c = t->tile_nnz[k + 1] - t->tile_nnz[k];
            t->blknnz[k] = c;
            t->csr_offset[k] = c;
            t->csrptr_offset[k] = rowlen_of(t, rb);
        }
    int csrsize = 0, csrptrlen = 0;
    for (int rb = 0; rb < tilem; ++rb)
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            csrsize += t->blknnz[k];
            csrptrlen += rowlen_of(t, rb);
        }
    t->csrsize = csrsize;
    t->csrptrlen = csrptrlen;
    for (int k = 0; k <= tilenum; ++k) t->blknnznnz[k] = (unsigned char)t->blknnz[k];
    int *scans[3] = {t->csr_offset, t->csrptr_offset, t->blknnz};
    for (int a = 0; a < 3; ++a) {
        if (tilenum + 1 <= 1) continue; /* utils.h:36: length 0/1 untouched */
        int run = 0;
        for (int k = 0; k <= tilenum; ++k) {
            int c = scans[a][k];
            scans[a][k] = run;
            run += c;
        }
    }

    /* step 4 (csr2block.h:152-265) */
    t->Blockcsr_Val = (double *)calloc((size_t)csrsize + 1, sizeof(double));
    t->Blockcsr_Val_Low = (float *)calloc((size_t)csrsize + 1, sizeof(float));
    t->Tile_csr_Col = (unsigned char *)calloc((size_t)csrsize + 1, 1);
    t->Blockcsr_Ptr = (unsigned char *)calloc((size_t)csrptrlen + 1, 1);
    t->csr_compressedIdx = (unsigned char *)calloc((size_t)csrsize / 2 + 2, 1);
    int *fillc = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    for (int rb = 0; rb < tilem; ++rb) {
        int rl = rowlen_of(t, rb);
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            unsigned char *p = tile_csr_ptr + (size_t)k * T16;
            /* exclusive_scan_char (utils.h:50-65) leaves length <= 1 alone */
            if (rl > 1) {
                unsigned char run = 0;
                for (int ri = 0; ri < rl; ++ri) {
                    unsigned char c = p[ri];
                    p[ri] = run;
                    run = (unsigned char)(run + c);
                }
            }
            for (int ri = 0; ri < rl; ++ri) t->Blockcsr_Ptr[t->csrptr_offset[k] + ri] = p[ri];
        }
        /* rows in order, entries in CSR order: tile t receives its entries in
         * CSR order; each row's run starts at the row pointer of that tile */
        if (rl == 1) continue; /* csr2block.h:239-251 copies nothing then */
        for (int ri = 0; ri < rl; ++ri) {
            int r = rb * T16 + ri;
            for (int q = rp[r]; q < rp[r + 1]; ++q) {
                int jc = ci[q] / T16;
                int lo = t->tile_ptr[rb], hi = t->tile_ptr[rb + 1] - 1;
                while (lo < hi) {
                    int mid = (lo + hi) / 2;
                    if (t->tile_columnidx[mid] < jc) lo = mid + 1; else hi = mid;
                }
                int pos = t->csr_offset[lo] + fillc[lo]++;
                t->Blockcsr_Val[pos] = val[q];
                t->Blockcsr_Val_Low[pos] = (float)val[q];
                t->Tile_csr_Col[pos] = (unsigned char)(ci[q] - jc * T16);
            }
        }
    }
    free(fillc);
    free(tile_csr_ptr);
    return 0;
}

void mfo_tiles_free(mfo_tiles *t) {
    free(t->tile_ptr); free(t->tile_columnidx); free(t->tile_nnz); free(t->blknnz);
    free(t->csr_offset); free(t->csrptr_offset); free(t->Format); free(t->blknnznnz);
    free(t->Blockcsr_Val); free(t->Blockcsr_Val_Low); free(t->Tile_csr_Col);
    free(t->Blockcsr_Ptr); free(t->csr_compressedIdx);
    memset(t, 0, sizeof *t);
}

/* PC/blockspmv_cpu.h:2-112. Per row block: y = 0; per tile in ascending
 * tile-column order: per row, sum = 0; sum += x * v over the row's entries
 * in stored order; y += sum. ptroffset1/2 are the running value / row
 * pointer offsets (:96-97); rowblkblock counts PREFETCH_SMEM_TH=4 splits
 * (:34-45). */
void mfo_blockspmv(const mfo_tiles *t, const double *x, double *y, int *ptroffset1,
                   int *ptroffset2, int *rowblkblock) {
    if (rowblkblock) {
        int cnt = 0;
        for (int rb = 0; rb < t->tilem; ++rb) {
            int nb = t->tile_ptr[rb + 1] - t->tile_ptr[rb];
            cnt += nb <= 4 ? 1 : (int)ceil((double)nb / 4.0);
        }
        *rowblkblock = cnt;
    }
    if (ptroffset1 || ptroffset2) {
        int csroffset = 0, csrcount = 0;
        for (int rb = 0; rb < t->tilem; ++rb) {
            int rl = rowlen_of(t, rb);
            for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
                if (ptroffset1) ptroffset1[k] = csroffset;
                if (ptroffset2) ptroffset2[k] = csrcount;
                csroffset += t->blknnz[k + 1] - t->blknnz[k];
                csrcount += rl;
            }
        }
    }
    if (!x || !y) return;
#pragma omp parallel for schedule(static)
    for (int rb = 0; rb < t->tilem; ++rb) {
        int rl = rowlen_of(t, rb);
        double acc[T16];
        for (int ri = 0; ri < T16; ++ri) acc[ri] = 0.0;
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            const int xo = t->tile_columnidx[k] * T16;
            const int vo = t->blknnz[k];
            const int nk = t->blknnz[k + 1] - t->blknnz[k];
            const unsigned char *bp = t->Blockcsr_Ptr + t->csrptr_offset[k];
            for (int ri = 0; ri < rl; ++ri) {
                int st = bp[ri];
                int sp = ri == rl - 1 ? nk : bp[ri + 1];
                double sum = 0.0;
                for (int q = st; q < sp; ++q) {
                    sum += x[xo + t->Tile_csr_Col[vo + q]] * t->Blockcsr_Val[vo + q];
                }
                acc[ri] += sum;
            }
        }
        for (int ri = 0; ri < rl; ++ri) y[rb * T16 + ri] = acc[ri];
    }
}

/* PC/Mille-feuille_CG_NVIDIA.cu:4154-4213 */
int mfo_row_compress(const mfo_tiles *t, int *nonzero_row_new, int *tile_rowidx,
                     int *block_signal, unsigned char **blockrowid_new,
                     unsigned char **blockcsr_ptr_new) {
    const int tilenum = t->tilenum, tilem = t->tilem;
    int *po2 = (int *)malloc(sizeof(int) * (size_t)(tilenum + 1));
    mfo_blockspmv(t, NULL, NULL, NULL, po2, NULL);
    memset(nonzero_row_new, 0, sizeof(int) * (size_t)(tilenum + 1));
    for (int rb = 0; rb < tilem; ++rb) {
        int rl = rowlen_of(t, rb);
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            int cc = po2[k];
            tile_rowidx[k] = rb;
            for (int ri = 0; ri < rl; ++ri) {
                int stop = ri == rl - 1 ? (t->blknnz[k + 1] - t->blknnz[k]) : t->Blockcsr_Ptr[ri + 1 + cc];
                if (stop != t->Blockcsr_Ptr[cc + ri]) nonzero_row_new[k] += 1;
            }
            nonzero_row_new[k] += 1;
        }
    }
    {
        int run = 0;
        for (int k = 0; k <= tilenum; ++k) {
            int c = nonzero_row_new[k];
            nonzero_row_new[k] = run;
            run += c;
        }
    }
    const int cnt = nonzero_row_new[tilenum];
    unsigned char *rid = (unsigned char *)calloc((size_t)cnt + 1, 1);
    unsigned char *rpn = (unsigned char *)calloc((size_t)cnt + 1, 1);
    memset(block_signal, 0, sizeof(int) * (size_t)(tilem + 1));
    for (int rb = 0; rb < tilem; ++rb) {
        int rl = rowlen_of(t, rb);
        block_signal[rb] = t->tile_ptr[rb + 1] - t->tile_ptr[rb];
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            int cc = po2[k], base = nonzero_row_new[k], fl = 0;
            for (int ri = 0; ri < rl; ++ri) {
                int stop = ri == rl - 1 ? (t->blknnz[k + 1] - t->blknnz[k]) : t->Blockcsr_Ptr[ri + 1 + cc];
                if (ri == 0) {
                    rid[base + fl] = (unsigned char)ri;
                    rpn[base + fl] = 0;
                    fl++;
                }
                if (stop != t->Blockcsr_Ptr[cc + ri]) {
                    rid[base + fl] = (unsigned char)ri;
                    rpn[base + fl] = (unsigned char)stop;
                    fl++;
                }
            }
        }
    }
    free(po2);
    *blockrowid_new = rid;
    *blockcsr_ptr_new = rpn;
    return cnt;
}

/* PC/Mille-feuille_CG_NVIDIA.cu:4216-4484: tiles are taken alternately
 * from the front (i) and the back (j); a unit closes when adding the next
 * tile would reach block_nnz nnz or block_per_warp tiles. */
int mfo_balance_twopointer(const mfo_tiles *t, int block_nnz, int block_per_warp,
                           int *bptr, int *idx_new, int *row_new, int *non_new) {
    const int tilenum = t->tilenum;
    int *non = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    int *row = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    for (int rb = 0; rb < t->tilem; ++rb)
        for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
            non[k] = t->blknnz[k + 1] - t->blknnz[k];
            row[k] = rb;
        }
    const int fill = bptr != NULL;
    int i = 0, j = tilenum - 1, cnt = 0, units = 1, step = 0, nblk = 0;
#define TAKE(src)                                                             \
    do {                                                                      \
        if (fill) {                                                           \
            idx_new[step] = (src); row_new[step] = row[src]; non_new[step] = non[src]; \
        }                                                                     \
    } while (0)
    if (fill) {
        memset(bptr, 0, sizeof(int));
    }
    while (i < j) {
        if (non[i] + cnt < block_nnz && nblk + 1 < block_per_warp) {
            cnt += non[i]; TAKE(i); ++i; ++step; ++nblk;
        } else {
            TAKE(i); ++i; ++step;
            if (fill) bptr[units] = step;
            ++units; cnt = 0; nblk = 0;
        }
        if (non[j] + cnt < block_nnz && nblk + 1 < block_per_warp) {
            cnt += non[j]; TAKE(j); --j; ++step; ++nblk;
        } else {
            TAKE(j); --j; ++step;
            if (fill) bptr[units] = step;
            ++units; cnt = 0; nblk = 0;
        }
        if (i == j) {
            TAKE(j); ++step;
            if (fill) bptr[units] = step;
        }
        if (i > j) {
            TAKE(j);
            if (fill) bptr[units] = step;
        }
    }
#undef TAKE
    free(non);
    free(row);
    return units;
}

void mfo_csr_spmv(int n, const int *rp, const int *ci, const double *v, const double *x,
                  double *y) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
        double s = 0.0;
        for (int p = rp[r]; p < rp[r + 1]; ++p) s += v[p] * x[ci[p]];
        y[r] = s;
    }
}

double mfo_dot(int n, const double *a, const double *b) {
    double part[64];
    const int nc = 64;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; ++c) {
        long long lo = (long long)n * c / nc, hi = (long long)n * (c + 1) / nc;
        double s = 0.0;
        for (long long k = lo; k < hi; ++k) s += a[k] * b[k];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < nc; ++c) s += part[c];
    return s;
}

int mfo_cg(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter,
           double *rel_res) {
    const int n = t->rowA;
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *d = (double *)malloc(sizeof(double) * (size_t)n);
    double *q = (double *)malloc(sizeof(double) * (size_t)n);
    mfo_blockspmv(t, x, q, NULL, NULL, NULL);
    for (int i = 0; i < n; ++i) { r[i] = b[i] - q[i]; d[i] = r[i]; }
    const double bn = sqrt(mfo_dot(n, b, b));
    double snew = mfo_dot(n, r, r);
    int it = 0;
    double rel = bn > 0 ? sqrt(snew) / bn : 0.0;
    while (it < maxiter && rel > tol) {
        mfo_blockspmv(t, d, q, NULL, NULL, NULL);
        const double alpha = snew / mfo_dot(n, d, q);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) { x[i] += alpha * d[i]; r[i] -= alpha * q[i]; }
        const double sold = snew;
        snew = mfo_dot(n, r, r);
        ++it;
        rel = sqrt(snew) / bn;
        if (rel <= tol) break;
        const double beta = snew / sold;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
    }
    if (rel_res) *rel_res = rel;
    free(r); free(d); free(q);
    return it;
}

/* One column of the 16-right-hand-side CG with FP32 search directions
 * (csrc/multi.cu, panel FP32): the reference recurrence
 * (Mille-feuille_CG_NVIDIA.cu:722-804) with d stored in FP32 (d = fl32(r +
 * beta d)) and q = fl32(A d) (the tiled SpMV in the reference's order on the
 * FP32 values); x, r, the dots and the scalars stay FP64. After the r update,
 * r is replaced by the true residual b - A x (FP64) every `replace`
 * iterations and whenever the recursive residual reaches tol; convergence is
 * decided on that true residual only. */
int mfo_cg_dir32(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter, int replace,
                 double *rel_res) {
    const int n = t->rowA;
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *d = (double *)malloc(sizeof(double) * (size_t)n);
    double *q = (double *)malloc(sizeof(double) * (size_t)n);
    mfo_blockspmv(t, x, q, NULL, NULL, NULL);
    for (int i = 0; i < n; ++i) { r[i] = b[i] - q[i]; d[i] = (double)(float)r[i]; }
    const double bb = mfo_dot(n, b, b);
    double rr = mfo_dot(n, r, r);
    double rel = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
    int it = 0;
    while (it < maxiter && rel > tol) {
        ++it;
        mfo_blockspmv(t, d, q, NULL, NULL, NULL);
        for (int i = 0; i < n; ++i) q[i] = (double)(float)q[i];
        const double dq = mfo_dot(n, d, q);
        if (!(dq > 0.0) || !isfinite(dq)) break; /* breakdown: not converged */
        const double alpha = rr / dq;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) { x[i] += alpha * d[i]; r[i] -= alpha * q[i]; }
        double rrn = mfo_dot(n, r, r);
        double relr = bb > 0 ? sqrt(rrn / bb) : sqrt(rrn);
        int restart = 0;
        if ((replace > 0 && it % replace == 0) || !(relr > tol)) {
            const double rec = rrn;
            mfo_blockspmv(t, x, q, NULL, NULL, NULL);
            for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
            rrn = mfo_dot(n, r, r);
            relr = bb > 0 ? sqrt(rrn / bb) : sqrt(rrn);
            rel = relr;
            if (!(relr > tol)) { rr = rrn; break; }
            /* a true residual norm more than twice the recursive one: the
             * directions no longer match r; restart from it (d = r) */
            restart = rrn > 4.0 * rec;
        }
        rel = relr;
        const double beta = restart ? 0.0 : rrn / rr;
        rr = rrn;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) d[i] = (double)(float)(r[i] + beta * d[i]);
    }
    if (rel_res) *rel_res = rel;
    free(r); free(d); free(q);
    return it;
}

/* Jacobi-preconditioned CG: KSPCG with PCJACOBI as in the "jpcg" runs of the
 * reference's PETSc comparison (PC/PETSc/src/ksp/ksp/impls/cg/cg.c:112-380,
 * unpreconditioned-norm stop test as test_a100.sh asks): z = r / a_ii,
 * alpha = (r.z) / (d.q), beta = (r.z)_new / (r.z)_old, d = z + beta d, stop on
 * ||r|| / ||b|| <= tol. diag[i] = a_ii (0 leaves the row unscaled). */
int mfo_pcg_jacobi(const mfo_tiles *t, const double *diag, const double *b, double *x, double tol,
                   int maxiter, double *rel_res) {
    const int n = t->rowA;
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *z = (double *)malloc(sizeof(double) * (size_t)n);
    double *d = (double *)malloc(sizeof(double) * (size_t)n);
    double *q = (double *)malloc(sizeof(double) * (size_t)n);
    double *minv = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) minv[i] = diag[i] != 0.0 ? 1.0 / diag[i] : 1.0;
    mfo_blockspmv(t, x, q, NULL, NULL, NULL);
    for (int i = 0; i < n; ++i) { r[i] = b[i] - q[i]; z[i] = minv[i] * r[i]; d[i] = z[i]; }
    const double bn = sqrt(mfo_dot(n, b, b));
    double rz = mfo_dot(n, r, z);
    double rel = bn > 0 ? sqrt(mfo_dot(n, r, r)) / bn : 0.0;
    int it = 0;
    while (it < maxiter && rel > tol) {
        mfo_blockspmv(t, d, q, NULL, NULL, NULL);
        const double alpha = rz / mfo_dot(n, d, q);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) { x[i] += alpha * d[i]; r[i] -= alpha * q[i]; z[i] = minv[i] * r[i]; }
        const double rzold = rz;
        rz = mfo_dot(n, r, z);
        ++it;
        rel = sqrt(mfo_dot(n, r, r)) / bn;
        if (rel <= tol) break;
        const double beta = rz / rzold;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) d[i] = z[i] + beta * d[i];
    }
    if (rel_res) *rel_res = rel;
    free(r); free(z); free(d); free(q); free(minv);
    return it;
}

int mfo_bicgstab(const mfo_tiles *t, const double *b, double *x, double tol, int maxiter,
                 double *rel_res) {
    const int n = t->rowA;
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *rh = (double *)malloc(sizeof(double) * (size_t)n);
    double *p = (double *)malloc(sizeof(double) * (size_t)n);
    double *v = (double *)malloc(sizeof(double) * (size_t)n);
    double *s = (double *)malloc(sizeof(double) * (size_t)n);
    double *tt = (double *)malloc(sizeof(double) * (size_t)n);
    mfo_blockspmv(t, x, v, NULL, NULL, NULL);
    for (int i = 0; i < n; ++i) { r[i] = b[i] - v[i]; rh[i] = r[i]; p[i] = r[i]; }
    const double bn = sqrt(mfo_dot(n, b, b));
    double rho = mfo_dot(n, r, rh);
    double rel = bn > 0 ? sqrt(mfo_dot(n, r, r)) / bn : 0.0;
    int it = 0;
    while (it < maxiter && rel > tol) {
        mfo_blockspmv(t, p, v, NULL, NULL, NULL);
        const double alpha = rho / mfo_dot(n, rh, v);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        mfo_blockspmv(t, s, tt, NULL, NULL, NULL);
        const double omega = mfo_dot(n, tt, s) / mfo_dot(n, tt, tt);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * p[i] + omega * s[i];
            r[i] = s[i] - omega * tt[i];
        }
        const double rho1 = mfo_dot(n, r, rh);
        ++it;
        rel = sqrt(mfo_dot(n, r, r)) / bn;
        if (rel <= tol) break;
        const double beta = (rho1 * alpha) / (rho * omega);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        rho = rho1;
    }
    if (rel_res) *rel_res = rel;
    free(r); free(rh); free(p); free(v); free(s); free(tt);
    return it;
}

/* ---- low-precision formats (OCP 8-bit FP spec v1.0; IEEE 754 binary16) ---- */

/* Round |v| (finite, >= 0) to a float with `mbits` explicit mantissa bits,
 * minimum normal exponent emin and subnormal quantum 2^(emin - mbits), ties
 * to even. Returns the rounded magnitude. */
static double round_mag(double a, int mbits, int emin) {
    if (a == 0.0) return 0.0;
    int e;
    frexp(a, &e);            /* a = f * 2^e, f in [0.5, 1) */
    int ex = e - 1;          /* a in [2^ex, 2^(ex+1)) */
    if (ex < emin) ex = emin;
    double q = ldexp(1.0, ex - mbits);   /* quantum */
    double m = a / q;                    /* exact: power-of-two scaling */
    double fl = floor(m);
    double rem = m - fl;
    if (rem > 0.5 || (rem == 0.5 && fmod(fl, 2.0) != 0.0)) fl += 1.0;
    return fl * q;
}

uint8_t mfo_fp8_e4m3_encode(double v) {
    if (isnan(v)) return 0x7F;
    uint8_t sgn = signbit(v) ? 0x80 : 0;
    double a = fabs(v);
    double r = round_mag(a, 3, -6);
    if (r > 448.0) r = 448.0; /* saturate (SATFINITE) */
    if (r == 0.0) return sgn;
    int e;
    frexp(r, &e);
    int ex = e - 1;
    if (ex < -6) { /* subnormal: 0.mmm * 2^-6 */
        int m = (int)(r / ldexp(1.0, -9));
        return (uint8_t)(sgn | m);
    }
    int m = (int)((r / ldexp(1.0, ex) - 1.0) * 8.0);
    return (uint8_t)(sgn | ((ex + 7) << 3) | m);
}

double mfo_fp8_e4m3_decode(uint8_t b) {
    int s = b >> 7, E = (b >> 3) & 15, m = b & 7;
    double v;
    if (E == 15 && m == 7) return NAN;
    if (E == 0) v = ldexp((double)m, -9);
    else v = ldexp(1.0 + m / 8.0, E - 7);
    return s ? -v : v;
}

uint16_t mfo_fp16_encode(double v) {
    if (isnan(v)) return 0x7E00;
    uint16_t sgn = signbit(v) ? 0x8000 : 0;
    double a = fabs(v);
    double r = round_mag(a, 10, -14);
    if (r >= 65520.0 || isinf(a)) return (uint16_t)(sgn | 0x7C00);
    if (r > 65504.0) r = 65504.0;
    if (r == 0.0) return sgn;
    int e;
    frexp(r, &e);
    int ex = e - 1;
    if (ex < -14) {
        int m = (int)(r / ldexp(1.0, -24));
        return (uint16_t)(sgn | m);
    }
    int m = (int)((r / ldexp(1.0, ex) - 1.0) * 1024.0);
    return (uint16_t)(sgn | ((ex + 15) << 10) | m);
}

double mfo_fp16_decode(uint16_t h) {
    int s = h >> 15, E = (h >> 10) & 31, m = h & 1023;
    double v;
    if (E == 31) v = m ? NAN : INFINITY;
    else if (E == 0) v = ldexp((double)m, -24);
    else v = ldexp(1.0 + m / 1024.0, E - 15);
    return s ? -v : v;
}

double mfo_tile_scale(int prec, double maxabs) {
    /* power-of-two scale s.t. maxabs / scale lands in (2^14, 2^15] (fp16) or
     * (224, 448] (fp8); 1 for fp64/fp32 and for all-zero tiles */
    if (maxabs <= 0.0 || prec < 2) return 1.0;
    int e;
    frexp(maxabs, &e); /* maxabs in [2^(e-1), 2^e) */
    if (prec == 2) return ldexp(1.0, e - 15);
    /* fp8: want maxabs/2^k <= 448 -> k = smallest with 2^k >= maxabs/448 */
    double ratio = maxabs / 448.0;
    int k;
    frexp(ratio, &k); /* ratio in [2^(k-1), 2^k) */
    if (ldexp(1.0, k - 1) == ratio) k -= 1;
    return ldexp(1.0, k);
}

/* Dequantized value of v stored in a tile of precision p with scale s. */
static double deq_value(int p, double v, double s) {
    if (p == 0) return v;
    if (p == 1) return (double)(float)v;
    if (p == 2) return mfo_fp16_decode(mfo_fp16_encode(v / s)) * s;
    return mfo_fp8_e4m3_decode(mfo_fp8_e4m3_encode(v / s)) * s;
}

/* One entry of a row in the reference's order (tiles ascending, CSR order
 * inside a tile). */
typedef struct {
    int col, cls, is_diag;
    double a, deq;
} mx_entry;

void mfo_mixed_spmv(const mfo_tiles *t, const unsigned char *prec, const double *x,
                    double *y) {
    /* The mixed-precision operator (no reference counterpart; the reference's
     * own mixed path keeps per-tile-column FP32 / FP16 / int8 copies,
     * MP/Mille-feuille_CG.cu:452-530).
     *
     * Entry class: the tile's precision p_t, except that a diagonal entry
     * (column == row) of an FP16 / FP8 tile is FP32. Dequantized value:
     * FP64 v; FP32 (float)v; FP16 / FP8 decode(encode(v / s_t)) * s_t with
     * the tile's power-of-two scale s_t (mfo_tile_scale of its max |v|).
     *
     * Row-sum-preserving compensation: a row with exactly one diagonal entry,
     * a_ii > 0, every other entry <= 0 and a diagonal of class FP64 or FP32
     * stores its diagonal as the class value of a_ii - delta_i, where delta_i
     * = sum over the row's other entries (reference order, FP64) of
     * (dequantized - a_ij). Writing A = sum_{i<j} (-a_ij) (e_i - e_j)(e_i -
     * e_j)^T + diag(row sums), the rounding then moves only the edge weights,
     * each by at most u_p relative, and for a symmetric diagonally dominant
     * Z-matrix (1 - u) A <= A~ <= (1 + u) A: the operator stays positive
     * definite with the same conditioning, however small its eigenvalues.
     *
     * Row sum: acc = sum over the FP64-class tiles in ascending order of
     * (sum = 0; sum += x * v in CSR order); sumf = fmaf((float)x, (float)v,
     * sumf) over the FP32-class entries in reference order, then the
     * FP16-class ones, then the FP8-class ones; y = acc + (double)sumf. */
    double *scale = (double *)malloc(sizeof(double) * (size_t)(t->tilenum > 0 ? t->tilenum : 1));
    for (int k = 0; k < t->tilenum; ++k) {
        double mx = 0.0;
        for (int q = t->blknnz[k]; q < t->blknnz[k + 1]; ++q)
            if (fabs(t->Blockcsr_Val[q]) > mx) mx = fabs(t->Blockcsr_Val[q]);
        scale[k] = mfo_tile_scale(prec[k], mx);
    }
#pragma omp parallel
    {
        mx_entry *row = NULL;
        int cap = 0;
#pragma omp for schedule(static)
        for (int rb = 0; rb < t->tilem; ++rb) {
            const int rl = rowlen_of(t, rb);
            for (int ri = 0; ri < rl; ++ri) {
                const int grow = rb * T16 + ri;
                int n = 0;
                for (int k = t->tile_ptr[rb]; k < t->tile_ptr[rb + 1]; ++k) {
                    const int vo = t->blknnz[k], nk = t->blknnz[k + 1] - vo;
                    const unsigned char *bp = t->Blockcsr_Ptr + t->csrptr_offset[k];
                    const int st = bp[ri], sp = ri == rl - 1 ? nk : bp[ri + 1];
                    for (int q = st; q < sp; ++q) {
                        if (n == cap) {
                            cap = cap ? 2 * cap : 64;
                            row = (mx_entry *)realloc(row, sizeof(mx_entry) * (size_t)cap);
                        }
                        mx_entry *e = &row[n++];
                        e->col = t->tile_columnidx[k] * T16 + t->Tile_csr_Col[vo + q];
                        e->a = t->Blockcsr_Val[vo + q];
                        e->is_diag = e->col == grow;
                        e->cls = prec[k];
                        if (e->is_diag && e->cls > 1) e->cls = 1;
                        e->deq = deq_value(prec[k], e->a, scale[k]);
                        if (e->is_diag && prec[k] > 1) e->deq = (double)(float)e->a;
                    }
                }
                /* compensation */
                int nd = 0, zrow = 1, di = -1;
                for (int q = 0; q < n; ++q) {
                    if (row[q].is_diag) { ++nd; di = q; }
                    else if (!(row[q].a <= 0.0)) zrow = 0;
                }
                if (nd == 1 && zrow && row[di].a > 0.0) {
                    double delta = 0.0;
                    for (int q = 0; q < n; ++q)
                        if (!row[q].is_diag) delta += row[q].deq - row[q].a;
                    const double dv = row[di].a - delta;
                    row[di].deq = row[di].cls == 0 ? dv : (double)(float)dv;
                }
                /* FP64 class: per-tile sums in tile order (entries of one tile
                 * are contiguous in reference order) */
                double acc = 0.0, sum = 0.0;
                int cur_tile_col = -1;
                for (int q = 0; q < n; ++q) {
                    if (row[q].cls != 0) continue;
                    const int tcol = row[q].col / T16;
                    if (tcol != cur_tile_col) {
                        if (cur_tile_col >= 0) acc += sum;
                        sum = 0.0;
                        cur_tile_col = tcol;
                    }
                    sum += x[row[q].col] * row[q].deq;
                }
                if (cur_tile_col >= 0) acc += sum;
                float sumf = 0.0f;
                for (int c = 1; c <= 3; ++c)
                    for (int q = 0; q < n; ++q)
                        if (row[q].cls == c) sumf = fmaf((float)x[row[q].col], (float)row[q].deq, sumf);
                y[grow] = acc + (double)sumf;
            }
        }
        free(row);
    }
    free(scale);
}

/* ---- MLP oracle (6 -> 64 -> 64 -> 4, ReLU, softmax cross-entropy) ---- */
static void mlp_layers(const float *W1, const float *b1, const float *W2, const float *b2,
                       const float *W3, const float *b3, const float *x, float *h1, float *h2,
                       float *out) {
    for (int o = 0; o < 64; ++o) {
        float s = b1[o];
        for (int i = 0; i < 6; ++i) s += W1[o * 6 + i] * x[i];
        h1[o] = s > 0 ? s : 0;
    }
    for (int o = 0; o < 64; ++o) {
        float s = b2[o];
        for (int i = 0; i < 64; ++i) s += W2[o * 64 + i] * h1[i];
        h2[o] = s > 0 ? s : 0;
    }
    for (int o = 0; o < 4; ++o) {
        float s = b3[o];
        for (int i = 0; i < 64; ++i) s += W3[o * 64 + i] * h2[i];
        out[o] = s;
    }
}

float mfo_mlp_forward(const float *W1, const float *b1, const float *W2, const float *b2,
                      const float *W3, const float *b3, const float *x, int batch,
                      float *logits) {
    float h1[64], h2[64];
    for (int s = 0; s < batch; ++s)
        mlp_layers(W1, b1, W2, b2, W3, b3, x + 6 * s, h1, h2, logits + 4 * s);
    return 0.0f;
}

float mfo_mlp_grad(const float *W1, const float *b1, const float *W2, const float *b2,
                   const float *W3, const float *b3, const float *x, const int *labels,
                   int batch, float *gW1, float *gb1, float *gW2, float *gb2, float *gW3,
                   float *gb3) {
    memset(gW1, 0, sizeof(float) * 64 * 6); memset(gb1, 0, sizeof(float) * 64);
    memset(gW2, 0, sizeof(float) * 64 * 64); memset(gb2, 0, sizeof(float) * 64);
    memset(gW3, 0, sizeof(float) * 4 * 64); memset(gb3, 0, sizeof(float) * 4);
    double loss = 0.0;
    const float inv = 1.0f / (float)batch;
    for (int s = 0; s < batch; ++s) {
        float h1[64], h2[64], out[4], p[4], d3[4], d2[64], d1[64];
        const float *xs = x + 6 * s;
        mlp_layers(W1, b1, W2, b2, W3, b3, xs, h1, h2, out);
        float mx = out[0];
        for (int o = 1; o < 4; ++o) if (out[o] > mx) mx = out[o];
        float z = 0;
        for (int o = 0; o < 4; ++o) { p[o] = expf(out[o] - mx); z += p[o]; }
        for (int o = 0; o < 4; ++o) p[o] /= z;
        loss += -log((double)p[labels[s]] + 1e-30);
        for (int o = 0; o < 4; ++o) d3[o] = (p[o] - (o == labels[s] ? 1.0f : 0.0f)) * inv;
        for (int o = 0; o < 4; ++o) {
            gb3[o] += d3[o];
            for (int i = 0; i < 64; ++i) gW3[o * 64 + i] += d3[o] * h2[i];
        }
        for (int i = 0; i < 64; ++i) {
            float g = 0;
            for (int o = 0; o < 4; ++o) g += W3[o * 64 + i] * d3[o];
            d2[i] = h2[i] > 0 ? g : 0;
        }
        for (int o = 0; o < 64; ++o) {
            gb2[o] += d2[o];
            for (int i = 0; i < 64; ++i) gW2[o * 64 + i] += d2[o] * h1[i];
        }
        for (int i = 0; i < 64; ++i) {
            float g = 0;
            for (int o = 0; o < 64; ++o) g += W2[o * 64 + i] * d2[o];
            d1[i] = h1[i] > 0 ? g : 0;
        }
        for (int o = 0; o < 64; ++o) {
            gb1[o] += d1[o];
            for (int i = 0; i < 6; ++i) gW1[o * 6 + i] += d1[o] * xs[i];
        }
    }
    return (float)(loss / batch);
}

int mfo_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}
