// Features of the precision selectors for one tile, computed by one warp
// from the encoder's tile arrays and the matrix diagonal:
//   f0 = log10 of the scaled magnitude m_t = max |a_ij| / sqrt(|a_ii a_jj|)
//   f1 = log10 of the tile's dynamic range max|a| / min|a| (0 when empty)
//   f2 = log10 of the matrix's nnz                       (whole matrix)
//   f3 = 1 for a diagonal tile (tile column == row block), else 0
//   f4 = log10 of the matrix's dynamic range max|a|/min|a| (whole matrix)
//   f5 = log10 of the relative residual at which the precision is used
// The two whole-matrix features tell a per-tile model how small the
// operator's smallest scaled eigenvalue may be (it falls with the size and
// the coefficient contrast), which bounds the safe rounding.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace mf {

struct TileFeatArgs {
    int tilenum, tilem, rowA;
    float lognnz, logrange;  // f2, f4
    const int *tile_ptr, *tile_col, *tile_off, *csrptr_off;
    const unsigned char *bptr, *col;
    const double *val, *diag;
};

// Every lane of the warp returns the features f0..f4 of tile t.
__device__ __forceinline__ void warp_tile_features(const TileFeatArgs &A, int t, float (&f)[5]) {
    const int lane = threadIdx.x & 31;
    int lo = 0, hi = A.tilem - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (A.tile_ptr[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const int rb = lo;
    const int rl = rb == A.tilem - 1 ? A.rowA - (A.tilem - 1) * 16 : 16;
    const int vo = A.tile_off[t], nk = A.tile_off[t + 1] - vo;
    const int cc = A.csrptr_off[t];
    const int c0 = A.tile_col[t] * 16;
    double smax = 0.0, amax = 0.0, amin = INFINITY;
    for (int k = lane; k < nk; k += 32) {
        // row of entry k: last r with ptr[r] <= k
        int r = 0;
        for (int q = 1; q < rl; ++q)
            if (A.bptr[cc + q] <= k) r = q;
        const int i = rb * 16 + r, j = c0 + A.col[vo + k];
        const double a = fabs(A.val[vo + k]);
        const double di = fabs(A.diag[i]), dj = j < A.rowA ? fabs(A.diag[j]) : 0.0;
        const double s = (di > 0 && dj > 0) ? a / sqrt(di * dj) : INFINITY;
        smax = fmax(smax, s);
        amax = fmax(amax, a);
        if (a > 0) amin = fmin(amin, a);
    }
    for (int d = 16; d > 0; d >>= 1) {
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, d));
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, d));
        amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, d));
    }
    f[0] = (float)log10(fmax(smax, 1e-300));
    f[1] = amax > 0 && amin < INFINITY ? (float)log10(amax / amin) : 0.0f;
    f[2] = A.lognnz;
    f[3] = A.tile_col[t] == rb ? 1.0f : 0.0f;
    f[4] = A.logrange;
}

}  // namespace mf
