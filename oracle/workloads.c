/*
 * workloads.c -- the synthetic test matrices, generated on the CPU by the
 * oracle (TEST INFRASTRUCTURE ONLY; see mf_oracle.h).
 *
 * The reference measures on SuiteSparse matrices that are not part of its
 * tree; the solver is measured instead on seeded synthetic systems whose
 * definitions are restated here from the workload descriptions (2D 5-point
 * Poisson, 3D upwind convection-diffusion, 3D variable-coefficient Poisson).
 * The CPU baseline builds its matrices here, so that timing the reference
 * algorithm never loads the product library; a CPU test checks that these
 * arrays equal the product's generators entry for entry.
 *
 * Random draws come from MT19937-64 (Matsumoto & Nishimura; the 64-bit
 * variant of Nishimura, ACM TOMACS 10(4), 2000), restated below from the
 * published algorithm: a 53-bit uniform is (next >> 11) * 2^-53.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "mf_oracle.h"

/* ------------------------------------------------------------ MT19937-64 */
enum { MT_N = 312, MT_M = 156 };

typedef struct {
    uint64_t s[MT_N];
    int i;
} mt64;

static void mt64_seed(mt64 *g, uint64_t seed) {
    g->s[0] = seed;
    for (int k = 1; k < MT_N; ++k)
        g->s[k] = 6364136223846793005ULL * (g->s[k - 1] ^ (g->s[k - 1] >> 62)) + (uint64_t)k;
    g->i = MT_N;
}

static uint64_t mt64_next(mt64 *g) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    const uint64_t a = 0xB5026F5AA96619E9ULL;
    if (g->i >= MT_N) {
        for (int k = 0; k < MT_N; ++k) {
            const uint64_t y = (g->s[k] & upper) | (g->s[(k + 1) % MT_N] & lower);
            g->s[k] = g->s[(k + MT_M) % MT_N] ^ (y >> 1) ^ ((y & 1ULL) ? a : 0ULL);
        }
        g->i = 0;
    }
    uint64_t x = g->s[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

static double mt64_u01(mt64 *g) { return (double)(mt64_next(g) >> 11) * 0x1.0p-53; }

static double mt64_logu(mt64 *g, double lo, double hi) {
    const double a = log(lo), b = log(hi);
    return exp(a + mt64_u01(g) * (b - a));
}

/* --------------------------------------------------------------- output */
static int alloc_out(mfo_system *m, long long n, long long cap, int with_xstar) {
    m->n = (int)n;
    m->nnz = 0;
    m->row_ptr = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    m->col_idx = (int *)malloc(sizeof(int) * (size_t)cap);
    m->val = (double *)malloc(sizeof(double) * (size_t)cap);
    m->b = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    m->xstar = with_xstar ? (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1)) : NULL;
    if (!m->row_ptr || !m->col_idx || !m->val || !m->b || (with_xstar && !m->xstar)) {
        mfo_system_free(m);
        return -1;
    }
    m->row_ptr[0] = 0;
    return 0;
}

static inline void put(mfo_system *m, long long c, double v) {
    m->col_idx[m->nnz] = (int)c;
    m->val[m->nnz] = v;
    m->nnz++;
}

void mfo_system_free(mfo_system *m) {
    free(m->row_ptr);
    free(m->col_idx);
    free(m->val);
    free(m->b);
    free(m->xstar);
    m->row_ptr = m->col_idx = NULL;
    m->val = m->b = m->xstar = NULL;
}

/* b[r] = sum_p val[p] * w[col[p]] over row r in CSR order (w = NULL: ones). */
static void row_products(mfo_system *m, const double *w) {
    for (int r = 0; r < m->n; ++r) {
        double s = 0.0;
        for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p)
            s += w ? m->val[p] * w[m->col_idx[p]] : m->val[p];
        m->b[r] = s;
    }
}

/* 2D 5-point Laplacian on an N x N grid, row r = i + N j, diagonal 4 and
 * -1 to the grid neighbours, columns ascending; b = A * ones. */
int mfo_gen_poisson2d(int N, mfo_system *m) {
    if (N <= 0 || (long long)N * N > (1LL << 30)) return -1;
    const long long n = (long long)N * N;
    if (alloc_out(m, n, 5 * n, 0)) return -1;
    for (long long j = 0; j < N; ++j)
        for (long long i = 0; i < N; ++i) {
            const long long r = i + (long long)N * j;
            if (j > 0) put(m, r - N, -1.0);
            if (i > 0) put(m, r - 1, -1.0);
            put(m, r, 4.0);
            if (i + 1 < N) put(m, r + 1, -1.0);
            if (j + 1 < N) put(m, r + N, -1.0);
            m->row_ptr[r + 1] = m->nnz;
        }
    row_products(m, NULL);
    return 0;
}

/* 3D 7-point upwind convection-diffusion on an N^3 grid, D = 1, h = 1,
 * velocity v: per axis the neighbour upstream of the flow carries
 * -(1 + |v_d|) and the one downstream -1; the diagonal is 6 + sum |v_d|;
 * neighbours outside the grid are dropped (Dirichlet). Row r = i + N j +
 * N^2 k, columns ascending. b[r] = 2u - 1 (u uniform, seed). */
int mfo_gen_convdiff3d(int N, double vx, double vy, double vz, uint64_t seed, mfo_system *m) {
    if (N <= 0 || (long long)N * N * N > (1LL << 30)) return -1;
    const long long n = (long long)N * N * N, s1 = N, s2 = (long long)N * N;
    if (alloc_out(m, n, 7 * n, 0)) return -1;
    const double v[3] = {vx, vy, vz};
    double minus[3], plus[3];
    for (int d = 0; d < 3; ++d) {
        minus[d] = v[d] >= 0 ? -1.0 - v[d] : -1.0; /* flow from the minus side */
        plus[d] = v[d] >= 0 ? -1.0 : -1.0 + v[d];
    }
    const double diag = 6.0 + fabs(vx) + fabs(vy) + fabs(vz);
    for (long long k = 0; k < N; ++k)
        for (long long j = 0; j < N; ++j)
            for (long long i = 0; i < N; ++i) {
                const long long r = i + s1 * j + s2 * k;
                if (k > 0) put(m, r - s2, minus[2]);
                if (j > 0) put(m, r - s1, minus[1]);
                if (i > 0) put(m, r - 1, minus[0]);
                put(m, r, diag);
                if (i + 1 < N) put(m, r + 1, plus[0]);
                if (j + 1 < N) put(m, r + s1, plus[1]);
                if (k + 1 < N) put(m, r + s2, plus[2]);
                m->row_ptr[r + 1] = m->nnz;
            }
    mt64 g;
    mt64_seed(&g, seed);
    for (long long r = 0; r < n; ++r) m->b[r] = 2.0 * mt64_u01(&g) - 1.0;
    return 0;
}

/* 3D 7-point variable-coefficient Poisson on an N^3 grid. Every cell face
 * carries k_f ~ logU[klo, khi], drawn in this order: the faces normal to x
 * (index (k, j, i), i = 0..N), then those normal to y ((k, j, i), j = 0..N),
 * then those normal to z ((k, j, i), k = 0..N), each in row-major order.
 * A_rr = sum of the cell's six faces (faces on the boundary included:
 * Dirichlet), A_rc = -k_f of the shared face. x* ~ U[0,1] continues the same
 * stream; b = A x* in CSR order. */
int mfo_gen_varpoisson3d(int N, double klo, double khi, uint64_t seed, mfo_system *m) {
    if (N <= 0 || !(klo > 0) || !(khi >= klo) || (long long)N * N * N > (1LL << 30)) return -1;
    const long long n = (long long)N * N * N, s1 = N, s2 = (long long)N * N, N1 = N + 1;
    double *fx = (double *)malloc(sizeof(double) * (size_t)(N * s1 * N1));
    double *fy = (double *)malloc(sizeof(double) * (size_t)(N * N1 * N));
    double *fz = (double *)malloc(sizeof(double) * (size_t)(N1 * s2));
    if (!fx || !fy || !fz || alloc_out(m, n, 7 * n, 1)) {
        free(fx); free(fy); free(fz);
        return -1;
    }
    mt64 g;
    mt64_seed(&g, seed);
    for (long long q = 0; q < N * s1 * N1; ++q) fx[q] = mt64_logu(&g, klo, khi);
    for (long long q = 0; q < N * N1 * N; ++q) fy[q] = mt64_logu(&g, klo, khi);
    for (long long q = 0; q < N1 * s2; ++q) fz[q] = mt64_logu(&g, klo, khi);
#define FX(k, j, i) fx[((k) * N + (j)) * N1 + (i)]
#define FY(k, j, i) fy[((k) * N1 + (j)) * N + (i)]
#define FZ(k, j, i) fz[((k) * N + (j)) * N + (i)]
    for (long long k = 0; k < N; ++k)
        for (long long j = 0; j < N; ++j)
            for (long long i = 0; i < N; ++i) {
                const long long r = i + s1 * j + s2 * k;
                const double w = FX(k, j, i), e = FX(k, j, i + 1);
                const double s = FY(k, j, i), nn = FY(k, j + 1, i);
                const double lo = FZ(k, j, i), hi = FZ(k + 1, j, i);
                if (k > 0) put(m, r - s2, -lo);
                if (j > 0) put(m, r - s1, -s);
                if (i > 0) put(m, r - 1, -w);
                put(m, r, w + e + s + nn + lo + hi);
                if (i + 1 < N) put(m, r + 1, -e);
                if (j + 1 < N) put(m, r + s1, -nn);
                if (k + 1 < N) put(m, r + s2, -hi);
                m->row_ptr[r + 1] = m->nnz;
            }
#undef FX
#undef FY
#undef FZ
    free(fx); free(fy); free(fz);
    for (long long r = 0; r < n; ++r) m->xstar[r] = mt64_u01(&g);
    row_products(m, m->xstar);
    return 0;
}
