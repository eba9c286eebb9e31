// Internal device-side structures of libmf: the tile matrix produced by the
// GPU encoder (the Tile_create arrays of Performance-Comparison/csr2block.h)
// and the streamed slab layout the persistent kernels consume.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "mf_internal.h"

#define MF_CUDA_TRY(expr)                                                            \
    do {                                                                             \
        cudaError_t _e = (expr);                                                     \
        if (_e != cudaSuccess) {                                                     \
            mf::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
            return MF_ERR_CUDA;                                                      \
        }                                                                            \
    } while (0)

namespace mf {

template <class T>
struct DevArray {
    T *p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { release(); }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        if (cudaMalloc((void **)&p, count * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            set_last_error("cudaMalloc failed");
            return MF_ERR_NOMEM;
        }
        n = count;
        return MF_OK;
    }
    int zero(cudaStream_t s = 0) { return cudaMemsetAsync(p, 0, n * sizeof(T), s) == cudaSuccess ? MF_OK : MF_ERR_CUDA; }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// ---- slab layout ------------------------------------------------------------
// A slab is a run of consecutive row blocks of one CTA's range, stored as one
// 16-byte aligned byte range so that one bulk copy brings it into shared
// memory. Byte layout (every section 16-byte aligned):
//   SlabHeader (32 B)
//   runs[MAXRUNS]           x-segment runs to stage for the slab that the
//                           CTA consumes STAGES slabs later (issue record)
//   rbdir[nrb + 1]          per row block: value byte offset, first tile,
//                           first column byte
//   slot[ntiles]  (u32)     staged x-segment slot (or, in gather mode, the
//                           tile column) | precision << 30
//   rowend[ntiles][16] (u8) inclusive end of each row inside the tile
//                           (row 15's end 256 stored as 0)
//   vals                    per tile: FP64 8n | FP32 4n | FP16 4+2n | FP8 4+n
//                           bytes, each block 8-byte aligned, FP16/FP8 blocks
//                           start with a float power-of-two scale
//   cols[nnz]     (u8)      intra-tile column (Tile_csr_Col)
constexpr int STAGES = 3;
constexpr int MAXRUNS = 24;
constexpr int XSEG_MAX = 128;      // staged x segments per slab (16 KB)
constexpr int MAXT = 2048;         // tiles per slab
constexpr int SLAB_MAX_DEFAULT = 40960;
constexpr int RB_PER_SLAB_MAX = 32;
constexpr int ISSUE_REC = 16 + MAXRUNS * 8;

enum { SLAB_STAGED = 0, SLAB_GATHER = 1, SLAB_OVERSIZE = 2 };

struct SlabHeader {
    int32_t rb0;
    uint16_t nrb, ntiles;
    uint16_t nxseg, mode;
    uint16_t next_nruns, cols16;  // cols16: byte offset of cols / 16
    uint32_t next_off16;  // issue record of the slab consumed STAGES later
    uint32_t next_bytes;  // 0 = none
    uint32_t next_xbytes;
    uint32_t bytes;
};
static_assert(sizeof(SlabHeader) == 32, "slab header is 32 bytes");

struct XRun {
    int32_t seg0;
    uint16_t nseg, slot0;
};

struct RbDir {
    uint32_t val_off;
    uint16_t tile0, col0;
};

struct SlabOffsets {
    uint32_t runs, rbdir, slot, rowend, vals, cols, total;
};

__host__ __device__ inline uint32_t align16u(uint32_t v) { return (v + 15u) & ~15u; }
__host__ __device__ inline uint32_t align8u(uint32_t v) { return (v + 7u) & ~7u; }

__host__ __device__ inline SlabOffsets slab_offsets(int nrb, int ntiles, uint32_t valbytes, int nnz) {
    SlabOffsets o;
    o.runs = 32;
    o.rbdir = align16u(o.runs + 8u * MAXRUNS);
    o.slot = align16u(o.rbdir + 8u * (uint32_t)(nrb + 1));
    o.rowend = align16u(o.slot + 4u * (uint32_t)ntiles);
    o.vals = o.rowend + 16u * (uint32_t)ntiles;
    o.cols = align16u(o.vals + valbytes);
    o.total = align16u(o.cols + (uint32_t)nnz);
    return o;
}

// Bytes of one tile's value block in the slab layout.
__host__ __device__ inline uint32_t tile_val_bytes(int prec, int nnz) {
    switch (prec) {
        case MF_PREC_FP64: return 8u * nnz;
        case MF_PREC_FP32: return align8u(4u * nnz);
        case MF_PREC_FP16: return align8u(4u + 2u * nnz);
        default: return align8u(4u + (uint32_t)nnz);
    }
}

// Algorithmic bytes of one tile (value bytes + 1 column byte per nnz + 8 per
// tile + 4 for an FP8 scale): the per-unit figure the roofline uses.
__host__ __device__ inline double tile_alg_bytes(int prec, int nnz) {
    const int s = prec == MF_PREC_FP64 ? 8 : prec == MF_PREC_FP32 ? 4 : prec == MF_PREC_FP16 ? 2 : 1;
    return (double)nnz * (s + 1) + 8.0 + (prec == MF_PREC_FP8 ? 4.0 : 0.0);
}

struct Layout {
    DevArray<uint8_t> slabs;     // all slab bytes
    DevArray<uint8_t> head;      // G x STAGES issue records
    DevArray<int> cta_slab;      // G+1: slab range of each CTA
    DevArray<int> cta_rb;        // G+1: row-block range of each CTA
    DevArray<int> cta_dep;       // 2G: CTA range whose vector entries a CTA reads
    DevArray<uint8_t> prec_dev;  // per tile precision
    DevArray<float> scale_dev;   // per tile scale (FP16 / FP8)
    std::vector<uint8_t> prec;   // host copy of the precisions
    int G = 0, nslabs = 0, n_gather = 0, n_oversize = 0;
    int slab_max = 0, rb_per_slab = 0;  // stage size / row blocks the planner used
    size_t bytes = 0;
    double alg_bytes = 0;        // algorithmic bytes of one SpMV
    double tile_frac[4] = {0, 0, 0, 0};
    bool built = false;
};

}  // namespace mf

constexpr int MF_NLEVELS = 3;

struct mf_tiles {
    int rowA = 0, colA = 0, tilem = 0, tilen = 0, tilenum = 0, csrsize = 0, csrptrlen = 0;
    int cnt_non_new = 0;
    int device = 0, nsm = 0;
    int G = 0;  // persistent CTAs
    mf_options opt;
    // Tile_create arrays (device); tile_off is tile_nnz == blknnz == csr_offset
    mf::DevArray<int> tile_ptr, tile_col, tile_off, csrptr_off;
    mf::DevArray<double> val;
    mf::DevArray<float> val_low;
    mf::DevArray<uint8_t> col, ptr, blknnznnz;
    // row compression (Mille-feuille_CG_NVIDIA.cu:4154-4213)
    mf::DevArray<int> nonzero_row_new, tile_rowidx, block_signal;
    mf::DevArray<uint8_t> blockrowid_new, blockcsr_ptr_new;
    // per-row diagonal (precision rule features)
    mf::DevArray<double> diag;
    // solver layouts
    mf::Layout L64;
    mf::Layout Lmix[MF_NLEVELS];
    bool mixed_ready = false;
    double encode_ms = 0, layout_ms = 0;
    // host copies used by the layout planner; h_cta_rb is the CTA row-block
    // partition shared by every layout of this matrix
    std::vector<int> h_tile_ptr, h_tile_col, h_tile_nnz, h_cta_rb;
    // solver workspace
    mf::DevArray<double> ws;
    mf::DevArray<uint32_t> sync;
    mf::DevArray<double> xpad;  // padded copy of a user x for mf_spmv
};

namespace mf {
int encode_device(mf_tiles *t, int n, int ncols, int nnz, const int *rp, const int *ci,
                  const double *val, cudaStream_t s);
int build_layout(mf_tiles *t, Layout &L, const std::vector<uint8_t> &prec, cudaStream_t s);
int exclusive_scan_int(int *d, long long n, cudaStream_t s);  // in place, n elements
}  // namespace mf
