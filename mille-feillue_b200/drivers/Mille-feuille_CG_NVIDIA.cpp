// Drop-in for the reference's Mille-feuille_CG_NVIDIA driver
// (Performance-Comparison/Mille-feuille_CG_NVIDIA.cu:4937-5001): same argv
// (matrix.mtx [block_nnz]); reads the matrix with read_Dmatrix_32 semantics,
// sets x = 1, b = A x and calls cg_solve_inc.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "mf.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s matrix.mtx [block_nnz]\n", argv[0]);
        return 1;
    }
    const int block_nnz = argc > 2 ? std::atoi(argv[2]) : 0;
    mf_matrix *m = nullptr;
    int rc = mf_read_mtx(argv[1], &m);
    if (rc != MF_OK) {
        std::fprintf(stderr, "cannot read %s: %s\n", argv[1], mf_status_str(rc));
        return 1;
    }
    mf_csr A;
    mf_matrix_csr(m, &A);
    if (A.n != A.ncols) {
        std::printf("unequal\n");
        return 0;
    }
    std::vector<float> low(A.nnz);
    for (int i = 0; i < A.nnz; ++i) low[i] = (float)A.val[i];
    const int ori = A.n;
    const int n = (A.n / 16) * 16;
    std::vector<double> X(n, 1.0), Y(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = A.row_ptr[i]; j < A.row_ptr[i + 1]; ++j) Y[i] += A.val[j] * X[A.col_idx[j]];
    int iter = 0;
    cg_solve_inc(const_cast<int *>(A.row_ptr), const_cast<int *>(A.col_idx), const_cast<double *>(A.val),
                 low.data(), X.data(), Y.data(), n, &iter, 10000, 1e-10, argv[1], A.nnz, ori, block_nnz);
    mf_matrix_free(m);
    return 0;
}
