// Library baseline for the solver benchmarks: CG and BiCGSTAB built from
// cuSPARSE (CSR SpMV, CUSPARSE_SPMV_ALG_DEFAULT) and cuBLAS level-1 calls
// with host-side scalars, one library call per vector operation, the way a
// caller assembles the solvers from the vendor libraries. The reference
// compares its synchronisation-free kernels against such a loop
// (Performance-Comparison/cuSPARSE_CG.cu, cuSPARSE_BiCGSTAB.cu: cuSPARSE SpMV
// plus cuBLAS dot / axpy with the scalars returned to the host every
// iteration); this file is an independent implementation of the textbook
// recurrences for timing on the same GPU, not part of libmf.
//
// C ABI (host CSR and vectors; the matrix, b and x are uploaded before the
// timed loop):
//   int cusp_cg(n, nnz, row_ptr, col_idx, val, b, x, tol, maxiter,
//               &iterations, &ms, &rel_residual)
//   int cusp_bicgstab(...same...)
// ms is the device time of the iteration loop (CUDA events around it);
// the stop test is ||r||/||b|| <= tol on the recursive residual, checked every
// iteration; tol <= 0 runs exactly maxiter iterations.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>

#include <cmath>
#include <cstdio>

namespace {

struct Ctx {
    cusparseHandle_t sp = nullptr;
    cublasHandle_t bl = nullptr;
    cusparseSpMatDescr_t A = nullptr;
    int *rp = nullptr, *ci = nullptr;
    double *val = nullptr;
    void *buf = nullptr;
    ~Ctx() {
        if (A) cusparseDestroySpMat(A);
        if (sp) cusparseDestroy(sp);
        if (bl) cublasDestroy(bl);
        cudaFree(rp);
        cudaFree(ci);
        cudaFree(val);
        cudaFree(buf);
    }
};

#define CK(x)                   \
    do {                        \
        if ((x) != 0) return -2; \
    } while (0)

int setup(Ctx &c, int n, int nnz, const int *rp, const int *ci, const double *val) {
    CK(cudaMalloc((void **)&c.rp, sizeof(int) * (n + 1)));
    CK(cudaMalloc((void **)&c.ci, sizeof(int) * (nnz > 0 ? nnz : 1)));
    CK(cudaMalloc((void **)&c.val, sizeof(double) * (nnz > 0 ? nnz : 1)));
    CK(cudaMemcpy(c.rp, rp, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    if (nnz > 0) {
        CK(cudaMemcpy(c.ci, ci, sizeof(int) * nnz, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c.val, val, sizeof(double) * nnz, cudaMemcpyHostToDevice));
    }
    CK(cusparseCreate(&c.sp));
    CK(cublasCreate(&c.bl));
    CK(cublasSetPointerMode(c.bl, CUBLAS_POINTER_MODE_HOST));
    CK(cusparseCreateCsr(&c.A, n, n, nnz, c.rp, c.ci, c.val, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                         CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F));
    return 0;
}

// y = A x through dense-vector descriptors made once per vector.
struct Vec {
    double *p = nullptr;
    cusparseDnVecDescr_t d = nullptr;
    ~Vec() {
        if (d) cusparseDestroyDnVec(d);
        cudaFree(p);
    }
    int make(int n) {
        if (cudaMalloc((void **)&p, sizeof(double) * n) != cudaSuccess) return -2;
        if (cudaMemset(p, 0, sizeof(double) * n) != cudaSuccess) return -2;
        return cusparseCreateDnVec(&d, n, p, CUDA_R_64F) == CUSPARSE_STATUS_SUCCESS ? 0 : -2;
    }
};

int spmv_buffer(Ctx &c, Vec &x, Vec &y) {
    const double one = 1.0, zero = 0.0;
    size_t bytes = 0;
    CK(cusparseSpMV_bufferSize(c.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, c.A, x.d, &zero, y.d, CUDA_R_64F,
                               CUSPARSE_SPMV_ALG_DEFAULT, &bytes));
    CK(cudaMalloc(&c.buf, bytes > 0 ? bytes : 8));
    return 0;
}

int spmv(Ctx &c, Vec &x, Vec &y) {
    const double one = 1.0, zero = 0.0;
    CK(cusparseSpMV(c.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, c.A, x.d, &zero, y.d, CUDA_R_64F,
                    CUSPARSE_SPMV_ALG_DEFAULT, c.buf));
    return 0;
}

}  // namespace

extern "C" {

int cusp_cg(int n, int nnz, const int *rp, const int *ci, const double *val, const double *b, double *x, double tol,
            int maxiter, int *iterations, double *ms, double *rel_residual) {
    Ctx c;
    if (setup(c, n, nnz, rp, ci, val)) return -2;
    Vec vb, vx, vr, vp, vq;
    if (vb.make(n) || vx.make(n) || vr.make(n) || vp.make(n) || vq.make(n)) return -2;
    CK(cudaMemcpy(vb.p, b, sizeof(double) * n, cudaMemcpyHostToDevice));
    if (spmv_buffer(c, vp, vq)) return -2;
    // x0 = 0: r = b, p = r
    CK(cudaMemcpy(vr.p, vb.p, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(vp.p, vb.p, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    double bnorm = 0.0, rr = 0.0;
    CK(cublasDnrm2(c.bl, n, vb.p, 1, &bnorm));
    CK(cublasDdot(c.bl, n, vr.p, 1, vr.p, 1, &rr));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    int it = 0;
    double rel = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
    while (it < maxiter && (tol <= 0.0 || rel > tol)) {
        if (spmv(c, vp, vq)) return -2;
        double pq = 0.0;
        CK(cublasDdot(c.bl, n, vp.p, 1, vq.p, 1, &pq));
        if (!(pq != 0.0) || !std::isfinite(pq)) break;
        const double alpha = rr / pq, malpha = -alpha;
        CK(cublasDaxpy(c.bl, n, &alpha, vp.p, 1, vx.p, 1));
        CK(cublasDaxpy(c.bl, n, &malpha, vq.p, 1, vr.p, 1));
        double rrn = 0.0;
        CK(cublasDdot(c.bl, n, vr.p, 1, vr.p, 1, &rrn));
        ++it;
        rel = bnorm > 0 ? std::sqrt(rrn) / bnorm : 0.0;
        const double beta = rrn / rr, one = 1.0;
        CK(cublasDscal(c.bl, n, &beta, vp.p, 1));
        CK(cublasDaxpy(c.bl, n, &one, vr.p, 1, vp.p, 1));
        rr = rrn;
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaMemcpy(x, vx.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    *iterations = it;
    *ms = f;
    *rel_residual = rel;
    return 0;
}

int cusp_bicgstab(int n, int nnz, const int *rp, const int *ci, const double *val, const double *b, double *x,
                  double tol, int maxiter, int *iterations, double *ms, double *rel_residual) {
    Ctx c;
    if (setup(c, n, nnz, rp, ci, val)) return -2;
    Vec vb, vx, vr, vrh, vp, vv, vs, vt;
    if (vb.make(n) || vx.make(n) || vr.make(n) || vrh.make(n) || vp.make(n) || vv.make(n) || vs.make(n) ||
        vt.make(n))
        return -2;
    CK(cudaMemcpy(vb.p, b, sizeof(double) * n, cudaMemcpyHostToDevice));
    if (spmv_buffer(c, vp, vv)) return -2;
    // x0 = 0: r = r^ = p = b
    CK(cudaMemcpy(vr.p, vb.p, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(vrh.p, vb.p, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(vp.p, vb.p, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    double bnorm = 0.0, rho = 0.0;
    CK(cublasDnrm2(c.bl, n, vb.p, 1, &bnorm));
    CK(cublasDdot(c.bl, n, vrh.p, 1, vr.p, 1, &rho));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    int it = 0;
    double rel = bnorm > 0 ? std::sqrt(rho) / bnorm : 0.0;
    while (it < maxiter && (tol <= 0.0 || rel > tol)) {
        if (spmv(c, vp, vv)) return -2;  // v = A p
        double rv = 0.0;
        CK(cublasDdot(c.bl, n, vrh.p, 1, vv.p, 1, &rv));
        if (!(rv != 0.0) || !std::isfinite(rv)) break;
        const double alpha = rho / rv, malpha = -alpha, one = 1.0;
        // s = r - alpha v
        CK(cudaMemcpyAsync(vs.p, vr.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, 0));
        CK(cublasDaxpy(c.bl, n, &malpha, vv.p, 1, vs.p, 1));
        if (spmv(c, vs, vt)) return -2;  // t = A s
        double ts = 0.0, tt = 0.0;
        CK(cublasDdot(c.bl, n, vt.p, 1, vs.p, 1, &ts));
        CK(cublasDdot(c.bl, n, vt.p, 1, vt.p, 1, &tt));
        if (!(tt != 0.0) || !std::isfinite(tt)) break;
        const double omega = ts / tt, momega = -omega;
        // x += alpha p + omega s;  r = s - omega t
        CK(cublasDaxpy(c.bl, n, &alpha, vp.p, 1, vx.p, 1));
        CK(cublasDaxpy(c.bl, n, &omega, vs.p, 1, vx.p, 1));
        CK(cudaMemcpyAsync(vr.p, vs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, 0));
        CK(cublasDaxpy(c.bl, n, &momega, vt.p, 1, vr.p, 1));
        double rho1 = 0.0, rr = 0.0;
        CK(cublasDdot(c.bl, n, vrh.p, 1, vr.p, 1, &rho1));
        CK(cublasDdot(c.bl, n, vr.p, 1, vr.p, 1, &rr));
        ++it;
        rel = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
        if (omega == 0.0 || !std::isfinite(rr)) break;
        // p = r + beta (p - omega v)
        const double beta = (rho1 * alpha) / (rho * omega);
        CK(cublasDaxpy(c.bl, n, &momega, vv.p, 1, vp.p, 1));
        CK(cublasDscal(c.bl, n, &beta, vp.p, 1));
        CK(cublasDaxpy(c.bl, n, &one, vr.p, 1, vp.p, 1));
        rho = rho1;
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaMemcpy(x, vx.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    *iterations = it;
    *ms = f;
    *rel_residual = rel;
    return 0;
}

}  // extern "C"
