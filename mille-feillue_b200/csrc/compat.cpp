// Drop-in replacements of the reference's C entry points
// (Performance-Comparison/Mille-feuille_CG_NVIDIA.cu:3979 cg_solve_inc and
// Mille-feuille_BiCGSTAB_NVIDIA.cu:1476 bicgstab) on top of the C ABI, and
// the reference driver's two-pointer warp work split as a compatibility
// export (Mille-feuille_CG_NVIDIA.cu:4216-4484).
#include <cstdio>
#include <cstring>
#include <vector>

#include "tiles.h"

extern "C" {

// Keeps the rows [0, nt) and the columns [0, nt) of a CSR matrix.
static void truncate_csr(const int *rp, const int *ci, const double *v, int nt, std::vector<int> &R,
                         std::vector<int> &C, std::vector<double> &V) {
    R.assign(nt + 1, 0);
    C.clear();
    V.clear();
    for (int r = 0; r < nt; ++r) {
        for (int p = rp[r]; p < rp[r + 1]; ++p)
            if (ci[p] < nt) {
                C.push_back(ci[p]);
                V.push_back(v[p]);
            }
        R[r + 1] = (int)C.size();
    }
}

void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n, int *iter,
                  int maxiter, double threshold, char *filename, int nnzR, int ori, int block_nnz) {
    (void)Val_Low; (void)filename; (void)nnzR; (void)ori; (void)block_nnz;
    const int nt = (n / 16) * 16;
    if (nt <= 0) return;
    std::vector<int> R, C;
    std::vector<double> V;
    truncate_csr(RowPtr, ColIdx, Val, nt, R, C, V);
    mf_csr A{nt, nt, (int)C.size(), R.data(), C.data(), V.data()};
    mf_options opt;
    mf_options_default(&opt);
    mf_tiles *t = nullptr;
    if (mf_encode(&A, &opt, &t) != MF_OK) return;
    std::memset(x, 0, sizeof(double) * n);
    mf_result res;
    const double tol = threshold > 0 ? threshold : 1e-10;
    const int mi = maxiter > 0 ? maxiter : 10000;
    mf_solve_cg(t, b, x, tol, mi, &opt, &res);
    if (iter) *iter = res.iterations;
    std::printf("iter=%d,time_cg=%lf ms,rel_residual=%e,true_rel_residual=%e\n", res.iterations, res.time_ms,
                res.rel_residual_rec, res.rel_residual_true);
    mf_free(t);
}

int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename, int n,
             int block_nnz) {
    (void)filename; (void)nnzR; (void)block_nnz;
    const int nt = (n / 16) * 16;
    if (nt <= 0) return 1;
    // rhs = A * ones over the full rows (Mille-feuille_BiCGSTAB_NVIDIA.cu:1982-1989)
    for (int i = 0; i < nt; ++i) {
        rhs[i] = 0;
        for (int j = RowPtr[i]; j < RowPtr[i + 1]; ++j) rhs[i] += Val[j];
    }
    std::vector<int> R, C;
    std::vector<double> V;
    truncate_csr(RowPtr, ColIdx, Val, nt, R, C, V);
    mf_csr A{nt, nt, (int)C.size(), R.data(), C.data(), V.data()};
    mf_options opt;
    mf_options_default(&opt);
    mf_tiles *t = nullptr;
    if (mf_encode(&A, &opt, &t) != MF_OK) return 1;
    std::memset(x, 0, sizeof(double) * n);
    mf_result res;
    const int rc = mf_solve_bicgstab(t, rhs, x, 1e-10, 10000, &opt, &res);
    std::printf("iter=%d,time_bicg=%lf ms,rel_residual=%e,true_rel_residual=%e\n", res.iterations, res.time_ms,
                res.rel_residual_rec, res.rel_residual_true);
    mf_free(t);
    return rc == MF_OK ? 0 : 1;
}

int mf_balance_twopointer(const mf_tiles *t, int block_nnz, int block_per_warp, int *index, int *bptr,
                          int *idx_new, int *row_new, int *non_new) {
    if (!t || !index || block_nnz <= 0 || block_per_warp <= 0) return MF_ERR_ARG;
    if (int rc = mf::ensure_host_tiles(t)) return rc;
    const int tilenum = t->tilenum;
    std::vector<int> non(tilenum + 1, 0), row(tilenum + 1, 0);
    for (int rb = 0; rb < t->tilem; ++rb)
        for (int k = t->h_tile_ptr[rb]; k < t->h_tile_ptr[rb + 1]; ++k) {
            non[k] = t->h_tile_nnz[k];
            row[k] = rb;
        }
    const bool fill = bptr && idx_new && row_new && non_new;
    // Tiles are taken alternately from the front (i) and the back (j) of the
    // tile list; a warp unit closes when the next tile would bring it to
    // block_nnz nonzeros or block_per_warp tiles.
    int i = 0, j = tilenum - 1, cnt = 0, units = 1, step = 0, nblk = 0;
    auto take = [&](int src) {
        if (fill) {
            idx_new[step] = src;
            row_new[step] = row[src];
            non_new[step] = non[src];
        }
    };
    if (fill) bptr[0] = 0;
    while (i < j) {
        if (non[i] + cnt < block_nnz && nblk + 1 < block_per_warp) {
            cnt += non[i];
            take(i);
            ++i;
            ++step;
            ++nblk;
        } else {
            take(i);
            ++i;
            ++step;
            if (fill) bptr[units] = step;
            ++units;
            cnt = 0;
            nblk = 0;
        }
        if (non[j] + cnt < block_nnz && nblk + 1 < block_per_warp) {
            cnt += non[j];
            take(j);
            --j;
            ++step;
            ++nblk;
        } else {
            take(j);
            --j;
            ++step;
            if (fill) bptr[units] = step;
            ++units;
            cnt = 0;
            nblk = 0;
        }
        if (i == j) {
            take(j);
            ++step;
            if (fill) bptr[units] = step;
        } else if (i > j) {
            take(j);
            if (fill) bptr[units] = step;
        }
    }
    *index = units;
    return MF_OK;
}

}  // extern "C"
