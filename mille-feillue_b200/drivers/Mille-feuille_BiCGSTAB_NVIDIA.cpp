// Drop-in for the reference's Mille-feuille_BiCGSTAB_NVIDIA driver
// (Performance-Comparison/Mille-feuille_BiCGSTAB_NVIDIA.cu:2278-2304): same
// argv (matrix.mtx [block_nnz]); x = 0, rhs = A * ones, calls bicgstab.
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
    std::vector<double> x(A.n, 0.0), rhs(A.n, 1.0);
    const int ret = bicgstab(const_cast<int *>(A.row_ptr), const_cast<int *>(A.col_idx),
                             const_cast<double *>(A.val), rhs.data(), x.data(), A.nnz, argv[1], A.n, block_nnz);
    mf_matrix_free(m);
    return ret;
}
