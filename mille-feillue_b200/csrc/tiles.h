// Internal device-side structures of libmf: the tile matrix produced by the
// GPU encoder (the Tile_create arrays of Performance-Comparison/csr2block.h)
// and the streamed slab layout the persistent kernels consume.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
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

// Device buffers come from the current device's stream-ordered memory pool,
// kept warm (its release threshold is raised once per device): a handle
// encoded, solved and freed again and again reuses the same memory instead
// of mapping and unmapping hundreds of MB per call. Each allocation is made
// usable by every stream before it returns, and each free first waits for
// the device, as a plain cudaFree would, because the batched and multi-RHS
// solvers run on streams of their own.
inline bool pool_ready(int dev) {
    static bool ready[64] = {};
    if (dev < 0 || dev >= 64) return false;
    if (!ready[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return false;
        uint64_t keep = UINT64_MAX;
        if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) return false;
        ready[dev] = true;
    }
    return true;
}

template <class T>
struct DevArray {
    T *p = nullptr;
    size_t n = 0;
    bool pooled = false;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { release(); }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        int dev = 0;
        cudaGetDevice(&dev);
        pooled = pool_ready(dev);
        const cudaError_t e = pooled ? cudaMallocAsync((void **)&p, count * sizeof(T), 0)
                                     : cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess || (pooled && cudaStreamSynchronize(0) != cudaSuccess)) {
            if (e == cudaSuccess) release();
            p = nullptr;
            set_last_error("device allocation failed");
            return MF_ERR_NOMEM;
        }
        n = count;
        return MF_OK;
    }
    int zero(cudaStream_t s = 0) { return cudaMemsetAsync(p, 0, n * sizeof(T), s) == cudaSuccess ? MF_OK : MF_ERR_CUDA; }
    void release() {
        if (p) {
            if (pooled) {
                cudaDeviceSynchronize();
                cudaFreeAsync(p, 0);
            } else {
                cudaFree(p);
            }
        }
        p = nullptr;
        n = 0;
        pooled = false;
    }
};

// ---- slab layout ------------------------------------------------------------
// A slab is a run of consecutive row blocks of one CTA's range, stored as one
// 16-byte aligned byte range so that one bulk copy brings it into shared
// memory. Byte layout (every section 16-byte aligned):
//   SlabHeader (48 B)
//   runs[MAXRUNS]       x-segment runs to stage for the slab that the CTA
//                       consumes STAGES slabs later (issue record)
//   rbdir[nrb + 1]      per row block: byte offset of its block, plane count
//   row-block blocks    one per row block, "row-sliced planes".
//   FP64 layouts:
//     rowlen[16]  (u8)  entries of each of the 16 rows
//     idx[W][16]        u16 x-window position (staged) or u32 column
//                       (gather) of entry k of row r, with the flag
//                       TILE_START (first entry of a new tile in this row)
//     vals[W][16]       FP64; plane k holds entry k of the 16 rows, in the
//                       reference's order (tiles in ascending column,
//                       entries of the row inside a tile in CSR order)
//   Mixed layouts (W <= 32): the planes are grouped by entry class (the
//   tile's precision; a diagonal entry of an FP16 / FP8 tile is FP32) in the
//   order FP64, FP32, FP16, FP8; plane j of a group holds the j-th entry of
//   that class of each row, in the reference's order.
//     head (16 B)       u8 plane counts of the four groups, u8 flags
//                       (RBF_*), 3 B pad, u64 storage precision of each
//                       plane (2 bits per plane)
//     sexp[W]           int8 exponent k of each plane's storage scale 2^k
//                       (padded to 16 B)
//     base[W]           (affine blocks in staged slabs only) u16 x-window
//                       position of row 0's entry of each plane: entry k of
//                       row r sits at base[k] + r, and no idx is stored
//     idx[W][16]        (other blocks) as in FP64 layouts; TILE_START only
//                       in FP64-class planes; padding entries index the
//                       stage's zero slot (staged) or carry PAD (gather)
//     vals              FP64/FP32/FP16/FP8 planes of 16 x width bytes
// A row block is affine when it has 16 rows, no FP64-class entry, and in
// every plane the column of row r's entry is (its row + a constant): its x
// positions then follow from the plane's base in any staged slab (the
// segments of those columns are consecutive, hence in consecutive slots).
constexpr int STAGES = 4;
constexpr int MAXRUNS = 24;
constexpr int XSEG_MAX = 112;      // staged x segments per slab (14 KB of FP64 x)
// Byte offset, inside a stage's x window, of 16 zero bytes that no copy
// writes. The padding entries of staged planes (plane k >= the row's length)
// index it with value 0, so a loop over all W planes of a row block adds
// 0 * 0 for them whatever x holds.
constexpr uint32_t XZERO_OFF = XSEG_MAX * 128;
// Layouts staging FP32 x (every tile below FP64) move XEXTRA32 bytes of each
// stage from the slab area to the x window, when the slab area is large
// enough: their slabs are small (FP16 values), and the wider window lets a
// slab hold twice the row blocks of an FP64-x layout. The window then ends
// at the same zero slot. (Measured on the 128^3 Poisson: 6 KB with 60 row
// blocks a slab is faster than 12 KB / 90 or 16 KB / 120.)
constexpr int XEXTRA32 = 6144;
__host__ __device__ inline int x32_extra(int slab_area) { return slab_area >= 4 * XEXTRA32 ? XEXTRA32 : 0; }
// Start of the x window in a stage, and the x-window position of the zero
// slot (the index of padding entries), for a layout staging FP32 or FP64 x.
__host__ __device__ inline int x_off_of(int slab_area, bool x32) {
    return x32 ? slab_area - x32_extra(slab_area) : slab_area;
}
__host__ __device__ inline uint32_t zero_pos_of(int slab_area, bool x32) {
    return x32 ? (XZERO_OFF + (uint32_t)x32_extra(slab_area)) / 4u : XZERO_OFF / 8u;
}
// Staged x segments per slab of an FP32-x layout (64-byte segments).
__host__ __device__ inline int xseg_max32(int slab_area) { return (int)(XZERO_OFF + x32_extra(slab_area)) / 64; }
constexpr int MAXW = 255;          // planes per row block (rowlen is u8)
constexpr int MAXW_MIXED = 32;     // planes per row block in mixed layouts
constexpr int SLAB_MAX_DEFAULT = 40960;
constexpr int RB_PER_SLAB_MAX = 120;  // four per consumer half-warp (a tuner candidate)
constexpr int RB_PER_SLAB_X32 = 60;   // default for layouts staging FP32 x
constexpr int RB_PER_SLAB_X64 = 30;  // default for layouts staging FP64 x
constexpr int ISSUE_REC = 16 + MAXRUNS * 8;
constexpr uint32_t IDX16_START = 0x8000u, IDX16_POS = 0x3fffu;
constexpr uint32_t IDX32_START = 0x80000000u, IDX32_PAD = 0x40000000u, IDX32_POS = 0x3fffffffu;

enum { SLAB_STAGED = 0, SLAB_GATHER = 1, SLAB_OVERSIZE = 2 };

struct SlabHeader {
    int32_t rb0;
    uint16_t nrb, ntiles;
    uint16_t nxseg, mode;
    uint16_t next_nruns, mixed;
    uint32_t next_off16;  // issue record of the slab consumed STAGES later
    uint32_t next_bytes;  // 0 = none
    uint32_t next_xbytes;
    uint32_t bytes;
    uint32_t pf_off16;  // slab consumed 2*STAGES later: prefetched into L2
    uint32_t pf_bytes;  // 0 = none
    uint32_t pad1, pad2;
};
static_assert(sizeof(SlabHeader) == 48, "slab header is 48 bytes");
constexpr uint32_t SLAB_HDR = 48;

struct XRun {
    int32_t seg0;
    uint16_t nseg, slot0;
};

struct RbDir {
    uint32_t off;  // byte offset of the row-block block from the slab start
    uint32_t W;    // planes (low 16 bits); high 16 bits: 1 + the x-stage slot of
                   // the row block's own column segment (0: not staged)
};

// Layout kinds: every tile FP64 / every tile below FP64 / both.
enum { LAYOUT_FP64 = 0, LAYOUT_LOW = 1, LAYOUT_ANY = 2 };

__host__ __device__ inline uint32_t align16u(uint32_t v) { return (v + 15u) & ~15u; }
__host__ __device__ inline uint32_t align8u(uint32_t v) { return (v + 7u) & ~7u; }

__host__ __device__ inline uint32_t slab_rbdir_off() { return align16u(SLAB_HDR + 8u * MAXRUNS); }
__host__ __device__ inline uint32_t slab_blocks_off(int nrb) { return align16u(slab_rbdir_off() + 8u * (nrb + 1)); }

// Offsets inside one FP64 row-block block.
__host__ __device__ inline uint32_t rb_idx_off() { return 16u; }
__host__ __device__ inline uint32_t rb_vals_off(int W, bool gather) {
    return align16u(rb_idx_off() + (uint32_t)W * 16u * (gather ? 4u : 2u));
}
// Offsets inside one mixed row-block block (aff: stored affine, which needs
// a staged slab).
enum { RBF_FAST = 1, RBF_AFFINE = 2, RBF_UNSCALED = 4 };
// RBF_FAST: every FP16-class plane stored as FP16 and every FP8-class one
// as FP8; RBF_UNSCALED: besides, every such plane's scale is 1.
__host__ __device__ inline uint32_t rbm_sexp_off() { return 16u; }
__host__ __device__ inline uint32_t rbm_base_off(int W) { return 16u + align16u((uint32_t)W); }
__host__ __device__ inline uint32_t rbm_idx_off(int W, bool aff) {
    return rbm_base_off(W) + (aff ? align16u(2u * (uint32_t)W) : 0u);
}
__host__ __device__ inline uint32_t rbm_vals_off(int W, bool gather, bool aff) {
    const bool a = aff && !gather;
    return align16u(rbm_idx_off(W, a) + (a ? 0u : (uint32_t)W * 16u * (gather ? 4u : 2u)));
}
__host__ __device__ inline uint32_t rb_block_bytes(int W, bool mixed, bool gather, uint32_t valbytes,
                                                   bool aff = false) {
    return mixed ? align16u(rbm_vals_off(W, gather, aff) + valbytes) : align16u(rb_vals_off(W, gather) + valbytes);
}
__host__ __device__ inline uint32_t prec_width(int prec) {
    return prec == MF_PREC_FP64 ? 8u : prec == MF_PREC_FP32 ? 4u : prec == MF_PREC_FP16 ? 2u : 1u;
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
    bool mixed = false;                  // plane precision info present
    int kind = 0;                        // LAYOUT_*
    bool x32 = false;                    // x staged in FP32: the SpMV input is an FP32 vector
                                         // (every LAYOUT_LOW layout)
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
    // BiCGSTAB's mixed layout, built on its first mixed solve when the
    // levels hold FP16 / FP8 tiles: those tiles raised to FP32 (the
    // replacement-window argument that makes compensated FP16 safe for CG
    // does not carry over to BiCGSTAB, whose iterations then grow ~2x)
    mf::Layout Lbicg;
    bool mixed_ready = false;
    int nlevels = 0;                        // mixed levels built
    double level_switch[MF_NLEVELS] = {0};  // relative residual to leave level l
    double encode_ms = 0, layout_ms = 0;
    // host copies of tile_ptr, tile_col and the per-tile nnz, fetched on
    // first use (mf::ensure_host_tiles: oversize row blocks, the planner
    // check, the memory report, the two-pointer export), not per encode
    mutable std::vector<int> h_tile_ptr, h_tile_col, h_tile_nnz;
    mutable bool host_tiles = false;
    mutable std::mutex host_tiles_mu;  // const entry points may fetch them concurrently
    // the CTA row-block partition shared by every layout of this matrix
    std::vector<int> h_cta_rb;
    // solver workspace
    mf::DevArray<double> ws;
    mf::DevArray<uint32_t> sync;
    mf::DevArray<double> xpad;  // padded copy of a user x for mf_spmv
    mf::DevArray<float> x32buf;  // FP32 copy of x for layouts staging FP32 x
    mf::DevArray<uint64_t> trace;  // phase timestamps of the last traced solve
    int trace_iters = 0;
    int minv_f32_ok = -1;  // every 1/a_ii fits FP32 (-1: not checked yet)
};

namespace mf {
int encode_device(mf_tiles *t, int n, int ncols, int nnz, const int *rp, const int *ci,
                  const double *val, cudaStream_t s);
int build_layout(mf_tiles *t, Layout &L, const std::vector<uint8_t> &prec, cudaStream_t s);
int ensure_host_tiles(const mf_tiles *t);  // fills h_tile_ptr, h_tile_col, h_tile_nnz once
int exclusive_scan_int(int *d, long long n, cudaStream_t s);  // in place, n elements
}  // namespace mf
