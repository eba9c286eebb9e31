// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own CPU code, unmodified, from the reference
// tree at build time (oracle/Makefile passes -I<reference>/Performance-Comparison)
// and exposes it through a small C ABI so the oracle restatement and the GPU
// encoder can be checked against it:
//   Tile_create        Performance-Comparison/csr2block.h:267
//   blockspmv_cpu      Performance-Comparison/blockspmv_cpu.h:2
//   encode             Performance-Comparison/encode.h:29  (fills the nibble
//                      column array that Tile_create leaves zero, so that
//                      blockspmv_cpu decodes the real intra-tile columns)
//   read_Dmatrix_32    Performance-Comparison/biio2.0/src/biio.h:153
// The output is written only to oracle/_ref/.
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "csr2block.h"
#include "blockspmv_cpu.h"
#include "biio2.0/src/biio.h"

extern "C" {

struct ref_handle {
    Tile_matrix m;
    int rowA, colA;
    bool compressed;
};

void *ref_tile_create(int rowA, int colA, int nnz, int *rp, int *ci, double *val) {
    ref_handle *h = (ref_handle *)calloc(1, sizeof(ref_handle));
    float *low = (float *)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
    for (int i = 0; i < nnz; ++i) low[i] = (float)val[i];
    h->rowA = rowA;
    h->colA = colA;
    Tile_create(&h->m, rowA, colA, nnz, rp, ci, val, low);
    free(low);
    return h;
}

void ref_tile_sizes(void *hp, int *out7) {
    ref_handle *h = (ref_handle *)hp;
    out7[0] = h->m.tilem;
    out7[1] = h->m.tilen;
    out7[2] = h->m.tilenum;
    out7[3] = h->m.csrsize;
    out7[4] = h->m.csrptrlen;
    out7[5] = h->rowA;
    out7[6] = h->colA;
}

// Copies one array by name into dst (caller sized).
int ref_tile_array(void *hp, const char *name, void *dst) {
    ref_handle *h = (ref_handle *)hp;
    Tile_matrix &m = h->m;
    const size_t tn = (size_t)m.tilenum;
#define CP(field, count, type)                                   \
    if (!strcmp(name, #field)) {                                 \
        memcpy(dst, m.field, (count) * sizeof(type));            \
        return 0;                                                \
    }
    CP(tile_ptr, (size_t)m.tilem + 1, int)
    CP(tile_columnidx, tn, int)
    CP(tile_nnz, tn + 1, int)
    CP(blknnz, tn + 1, int)
    CP(csr_offset, tn + 1, int)
    CP(csrptr_offset, tn + 1, int)
    CP(Format, tn, char)
    CP(blknnznnz, tn + 1, unsigned char)
    CP(Blockcsr_Val, (size_t)m.csrsize, double)
    CP(Blockcsr_Val_Low, (size_t)m.csrsize, float)
    CP(Tile_csr_Col, (size_t)m.csrsize, unsigned char)
    CP(Blockcsr_Ptr, (size_t)m.csrptrlen, unsigned char)
    CP(csr_compressedIdx, (size_t)(m.csrsize % 2 == 0 ? m.csrsize / 2 : m.csrsize / 2 + 1),
       unsigned char)
#undef CP
    return -1;
}

// blockspmv_cpu with the nibble column array filled by the reference's own
// encode(); fill_compressed = 0 runs it exactly as the drivers do (all
// intra-tile columns decode as 0).
void ref_blockspmv(void *hp, double *x, double *y, int *ptroffset1, int *ptroffset2,
                   int *rowblkblock, int fill_compressed) {
    ref_handle *h = (ref_handle *)hp;
    Tile_matrix &m = h->m;
    if (fill_compressed && !h->compressed && m.csrsize > 0) {
        encode(m.Tile_csr_Col, m.csr_compressedIdx, m.csrsize, 0);
        h->compressed = true;
    }
    unsigned int *a = nullptr;
    int *b = nullptr, *c = nullptr;
    blockspmv_cpu(&m, ptroffset1, ptroffset2, rowblkblock, &a, &b, &c, h->rowA, h->colA, 0,
                  nullptr, nullptr, nullptr, x, y, nullptr);
    free(a);
    free(b);
    free(c);
}

void ref_tile_free(void *hp) {
    ref_handle *h = (ref_handle *)hp;
    if (!h) return;
    Tile_matrix &m = h->m;
    free(m.tile_ptr); free(m.tile_columnidx); free(m.tile_nnz); free(m.Format);
    free(m.blknnz); free(m.blknnznnz); free(m.tilewidth); free(m.csr_offset);
    free(m.csrptr_offset); free(m.Blockcsr_Val); free(m.Blockcsr_Val_Low);
    free(m.Blockcsr_Ptr); free(m.csr_compressedIdx); free(m.Tile_csr_Col);
    free(h);
}

// read_Dmatrix_32 into caller-visible malloc'd arrays (free with ref_free).
int ref_read_mtx(const char *path, int *m, int *n, int *nnz, int **rp, int **ci, double **val) {
    int sym = 0;
    read_Dmatrix_32(m, n, nnz, rp, ci, val, &sym, (char *)path);
    return sym;
}

// binary_read_csr (biio.h:22-72): the .cbd file into malloc'd arrays (row
// pointers are 64-bit there). Returns its status (0 ok, -1 failure).
int ref_read_cbd(const char *path, int *m, int *n, int64_t *nnz, int64_t **rp, int **ci, double **val) {
    return binary_read_csr(m, n, nnz, rp, ci, val, (char *)path);
}

// binary_write_csr (biio.h:74-97).
void ref_write_cbd(const char *path, int m, int n, int64_t nnz, int64_t *rp, int *ci, double *val) {
    binary_write_csr(m, n, nnz, rp, ci, val, (char *)path);
}

void ref_free(void *p) { free(p); }

}  // extern "C"
