// Host-side CSR matrices: seeded synthetic generators for the solver's
// workloads, the Matrix Market reader and the .cbd binary CSR reader/writer.
//
// Reader semantics follow Performance-Comparison/biio2.0/src/biio.h:153-194
// (read_Dmatrix_32) and biio2.0/src/mmio_highlevel.h:151-321 (mmio_data):
// 1-based -> 0-based, symmetric/hermitian files expanded to both triangles,
// entries kept in file order within each row (no sort), pattern -> 1.0,
// complex -> real part. The .cbd layout is biio.h:22-97.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>

#include "mf_internal.h"

namespace mf {
static std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
const std::string &last_error() { return g_last_error; }

struct Rng {
    std::mt19937_64 eng;
    explicit Rng(uint64_t seed) : eng(seed) {}
    // 53-bit uniform in [0,1).
    double u() { return (double)(eng() >> 11) * 0x1.0p-53; }
    double loguniform(double lo, double hi) {
        return std::exp(std::log(lo) + u() * (std::log(hi) - std::log(lo)));
    }
    uint64_t next() { return eng(); }
};
}  // namespace mf

using mf::Rng;

static int finish(mf_matrix *m, mf_matrix **out) {
    *out = m;
    return MF_OK;
}

extern "C" {

int mf_gen_poisson2d(int N, mf_matrix **out) {
    if (N <= 0 || !out) return MF_ERR_ARG;
    if ((long long)N * N > (1LL << 30)) return MF_ERR_ARG;
    auto *m = new mf_matrix;
    const int n = N * N;
    m->n = m->ncols = n;
    m->row_ptr.resize(n + 1);
    m->col_idx.reserve((size_t)5 * n);
    m->val.reserve((size_t)5 * n);
    m->b.assign(n, 0.0);
    m->row_ptr[0] = 0;
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            const int r = i + N * j;
            auto put = [&](int c, double v) {
                m->col_idx.push_back(c);
                m->val.push_back(v);
            };
            if (j > 0) put(r - N, -1.0);
            if (i > 0) put(r - 1, -1.0);
            put(r, 4.0);
            if (i < N - 1) put(r + 1, -1.0);
            if (j < N - 1) put(r + N, -1.0);
            m->row_ptr[r + 1] = (int)m->col_idx.size();
        }
    // b = A * ones, summed in CSR order.
    for (int r = 0; r < n; ++r) {
        double s = 0.0;
        for (int k = m->row_ptr[r]; k < m->row_ptr[r + 1]; ++k) s += m->val[k];
        m->b[r] = s;
    }
    return finish(m, out);
}

int mf_gen_convdiff3d(int N, double vx, double vy, double vz, uint64_t seed,
                      mf_matrix **out) {
    if (N <= 0 || !out) return MF_ERR_ARG;
    if ((long long)N * N * N > (1LL << 30)) return MF_ERR_ARG;
    // Upwind finite differences with D = 1, h = 1 (cell Peclet |v|/2):
    //   upwind neighbour  -(1 + |v_d|), downwind neighbour -1,
    //   diagonal 6 + |vx| + |vy| + |vz|; Dirichlet boundaries drop neighbours.
    auto *m = new mf_matrix;
    const long long n = (long long)N * N * N;
    m->n = m->ncols = (int)n;
    m->row_ptr.resize(n + 1);
    m->col_idx.reserve((size_t)7 * n);
    m->val.reserve((size_t)7 * n);
    const double v[3] = {vx, vy, vz};
    double lo[3], hi[3];  // coefficient of the minus / plus neighbour per axis
    for (int d = 0; d < 3; ++d) {
        lo[d] = v[d] >= 0 ? -(1.0 + v[d]) : -1.0;
        hi[d] = v[d] >= 0 ? -1.0 : -(1.0 - v[d]);
    }
    const double diag = 6.0 + std::fabs(vx) + std::fabs(vy) + std::fabs(vz);
    const long long sx = 1, sy = N, sz = (long long)N * N;
    m->row_ptr[0] = 0;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                const long long r = i + sy * j + sz * k;
                auto put = [&](long long c, double val) {
                    m->col_idx.push_back((int)c);
                    m->val.push_back(val);
                };
                if (k > 0) put(r - sz, lo[2]);
                if (j > 0) put(r - sy, lo[1]);
                if (i > 0) put(r - sx, lo[0]);
                put(r, diag);
                if (i < N - 1) put(r + sx, hi[0]);
                if (j < N - 1) put(r + sy, hi[1]);
                if (k < N - 1) put(r + sz, hi[2]);
                m->row_ptr[r + 1] = (int)m->col_idx.size();
            }
    Rng rng(seed);
    m->b.resize(n);
    for (long long r = 0; r < n; ++r) m->b[r] = 2.0 * rng.u() - 1.0;
    return finish(m, out);
}

int mf_gen_varpoisson3d(int N, double klo, double khi, uint64_t seed,
                        mf_matrix **out) {
    if (N <= 0 || !out || !(klo > 0) || !(khi >= klo)) return MF_ERR_ARG;
    if ((long long)N * N * N > (1LL << 30)) return MF_ERR_ARG;
    // Face coefficients k_f ~ logU[klo, khi]. Draw order: x-faces
    // (k, j, i = 0..N), then y-faces (k, j = 0..N, i), then z-faces
    // (k = 0..N, j, i). A_ii = sum of the cell's six faces (boundary faces
    // included: Dirichlet), A_ij = -k_f. x* ~ U[0,1] follows on the same
    // stream; b = A x* summed in CSR order.
    Rng rng(seed);
    const long long Np = N + 1;
    std::vector<double> kx((size_t)N * N * Np), ky((size_t)N * Np * N),
        kz((size_t)Np * N * N);
    for (auto &f : kx) f = rng.loguniform(klo, khi);
    for (auto &f : ky) f = rng.loguniform(klo, khi);
    for (auto &f : kz) f = rng.loguniform(klo, khi);
    auto KX = [&](long long k, long long j, long long i) { return kx[(k * N + j) * Np + i]; };
    auto KY = [&](long long k, long long j, long long i) { return ky[(k * Np + j) * N + i]; };
    auto KZ = [&](long long k, long long j, long long i) { return kz[(k * N + j) * N + i]; };
    auto *m = new mf_matrix;
    const long long n = (long long)N * N * N;
    m->n = m->ncols = (int)n;
    m->row_ptr.resize(n + 1);
    m->col_idx.reserve((size_t)7 * n);
    m->val.reserve((size_t)7 * n);
    const long long sy = N, sz = (long long)N * N;
    m->row_ptr[0] = 0;
    for (long long k = 0; k < N; ++k)
        for (long long j = 0; j < N; ++j)
            for (long long i = 0; i < N; ++i) {
                const long long r = i + sy * j + sz * k;
                const double fxm = KX(k, j, i), fxp = KX(k, j, i + 1);
                const double fym = KY(k, j, i), fyp = KY(k, j + 1, i);
                const double fzm = KZ(k, j, i), fzp = KZ(k + 1, j, i);
                const double diag = fxm + fxp + fym + fyp + fzm + fzp;
                auto put = [&](long long c, double val) {
                    m->col_idx.push_back((int)c);
                    m->val.push_back(val);
                };
                if (k > 0) put(r - sz, -fzm);
                if (j > 0) put(r - sy, -fym);
                if (i > 0) put(r - 1, -fxm);
                put(r, diag);
                if (i < N - 1) put(r + 1, -fxp);
                if (j < N - 1) put(r + sy, -fyp);
                if (k < N - 1) put(r + sz, -fzp);
                m->row_ptr[r + 1] = (int)m->col_idx.size();
            }
    m->xstar.resize(n);
    for (long long r = 0; r < n; ++r) m->xstar[r] = rng.u();
    m->b.resize(n);
    for (long long r = 0; r < n; ++r) {
        double s = 0.0;
        for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p)
            s += m->val[p] * m->xstar[m->col_idx[p]];
        m->b[r] = s;
    }
    return finish(m, out);
}

int mf_gen_spd_random(int n, uint64_t seed, mf_matrix **out) {
    if (n < 2 || !out) return MF_ERR_ARG;
    // Row i draws m_i = 4 + (next % 9) off-diagonal columns j != i uniformly
    // (j = next % (n-1), shifted past i) with weight w = -u, u ~ U[0,1).
    // The matrix is symmetrised as (B + B^T) / 2 over the union pattern
    // (duplicates summed), the diagonal is sum_j |A_ij| + 0.01, b ~ U[-1,1].
    Rng rng(seed);
    struct E { int r, c; double v; };
    std::vector<E> coo;
    coo.reserve((size_t)n * 16);
    for (int i = 0; i < n; ++i) {
        const int mcount = 4 + (int)(rng.next() % 9ull);
        for (int t = 0; t < mcount; ++t) {
            int j = (int)(rng.next() % (uint64_t)(n - 1));
            if (j >= i) ++j;
            const double w = -rng.u();
            coo.push_back({i, j, 0.5 * w});
            coo.push_back({j, i, 0.5 * w});
        }
    }
    std::sort(coo.begin(), coo.end(), [](const E &a, const E &b) {
        return a.r != b.r ? a.r < b.r : a.c < b.c;
    });
    auto *m = new mf_matrix;
    m->n = m->ncols = n;
    m->row_ptr.assign(n + 1, 0);
    m->col_idx.reserve(coo.size() + n);
    m->val.reserve(coo.size() + n);
    size_t p = 0;
    for (int i = 0; i < n; ++i) {
        // merge duplicates of row i
        std::vector<std::pair<int, double>> row;
        while (p < coo.size() && coo[p].r == i) {
            if (!row.empty() && row.back().first == coo[p].c)
                row.back().second += coo[p].v;
            else
                row.push_back({coo[p].c, coo[p].v});
            ++p;
        }
        double dsum = 0.0;
        for (auto &e : row) dsum += std::fabs(e.second);
        bool placed = false;
        for (auto &e : row) {
            if (!placed && e.first > i) {
                m->col_idx.push_back(i);
                m->val.push_back(dsum + 0.01);
                placed = true;
            }
            m->col_idx.push_back(e.first);
            m->val.push_back(e.second);
        }
        if (!placed) {
            m->col_idx.push_back(i);
            m->val.push_back(dsum + 0.01);
        }
        m->row_ptr[i + 1] = (int)m->col_idx.size();
    }
    m->b.resize(n);
    for (int i = 0; i < n; ++i) m->b[i] = 2.0 * rng.u() - 1.0;
    return finish(m, out);
}

int mf_gen_batch_sizes(int count, int lo, int hi, uint64_t seed, int *sizes) {
    if (count < 0 || lo <= 0 || hi < lo || (count > 0 && !sizes)) return MF_ERR_ARG;
    Rng rng(seed);
    for (int s = 0; s < count; ++s)
        sizes[s] = (int)std::llround(rng.loguniform((double)lo, (double)hi));
    return MF_OK;
}

// ---------------------------------------------------------------- readers

int mf_read_mtx(const char *path, mf_matrix **out) {
    if (!path || !out) return MF_ERR_ARG;
    FILE *f = std::fopen(path, "r");
    if (!f) { mf::set_last_error(std::string("cannot open ") + path); return MF_ERR_IO; }
    char line[4096];
    if (!std::fgets(line, sizeof line, f)) { std::fclose(f); return MF_ERR_IO; }
    std::string banner(line);
    for (auto &ch : banner) ch = (char)std::tolower((unsigned char)ch);
    if (banner.rfind("%%matrixmarket", 0) != 0 || banner.find("coordinate") == std::string::npos) {
        std::fclose(f);
        mf::set_last_error("not a coordinate Matrix Market file");
        return MF_ERR_IO;
    }
    const bool pattern = banner.find("pattern") != std::string::npos;
    const bool complex_ = banner.find("complex") != std::string::npos;
    const bool integer = banner.find("integer") != std::string::npos;
    // symmetric and hermitian are expanded; skew-symmetric is read as
    // general, exactly as mmio_highlevel.h:193-201 does.
    const bool symmetric = banner.find(" symmetric") != std::string::npos ||
                           banner.find("hermitian") != std::string::npos;
    (void)integer;
    long long rows = 0, cols = 0, nnz_file = 0;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        if (std::sscanf(line, "%lld %lld %lld", &rows, &cols, &nnz_file) == 3) break;
    }
    if (rows <= 0 || cols <= 0 || nnz_file < 0 || rows > INT32_MAX || cols > INT32_MAX) {
        std::fclose(f);
        return MF_ERR_IO;
    }
    std::vector<int> ri(nnz_file), ci(nnz_file);
    std::vector<double> vv(nnz_file);
    std::vector<long long> cnt(rows + 1, 0);
    for (long long e = 0; e < nnz_file; ++e) {
        long long a, b;
        double x = 1.0, y = 0.0;
        int got;
        if (pattern)
            got = std::fscanf(f, "%lld %lld", &a, &b) == 2;
        else if (complex_)
            got = std::fscanf(f, "%lld %lld %lg %lg", &a, &b, &x, &y) == 4;
        else
            got = std::fscanf(f, "%lld %lld %lg", &a, &b, &x) == 3;
        if (!got || a < 1 || b < 1 || a > rows || b > cols) {
            std::fclose(f);
            mf::set_last_error("malformed Matrix Market entry");
            return MF_ERR_IO;
        }
        ri[e] = (int)(a - 1);
        ci[e] = (int)(b - 1);
        vv[e] = x;
        cnt[ri[e]]++;
        if (symmetric && ri[e] != ci[e]) cnt[ci[e]]++;
    }
    std::fclose(f);
    // exclusive scan of the row counts
    long long run = 0;
    for (long long r = 0; r <= rows; ++r) {
        long long c = cnt[r];
        cnt[r] = run;
        run += c;
    }
    if (run > INT32_MAX) { mf::set_last_error("nnz exceeds int32"); return MF_ERR_UNSUPPORTED; }
    auto *m = new mf_matrix;
    m->n = (int)rows;
    m->ncols = (int)cols;
    m->row_ptr.resize(rows + 1);
    for (long long r = 0; r <= rows; ++r) m->row_ptr[r] = (int)cnt[r];
    m->col_idx.resize(run);
    m->val.resize(run);
    std::vector<long long> fill(rows, 0);
    for (long long e = 0; e < nnz_file; ++e) {
        const int a = ri[e], b = ci[e];
        long long o = m->row_ptr[a] + fill[a]++;
        m->col_idx[o] = b;
        m->val[o] = vv[e];
        if (symmetric && a != b) {
            o = m->row_ptr[b] + fill[b]++;
            m->col_idx[o] = a;
            m->val[o] = vv[e];
        }
    }
    return finish(m, out);
}

int mf_read_cbd(const char *path, mf_matrix **out) {
    if (!path || !out) return MF_ERR_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return MF_ERR_IO;
    int rows = 0, cols = 0;
    int64_t nnz = 0;
    bool ok = std::fread(&rows, sizeof(int), 1, f) == 1 && std::fread(&cols, sizeof(int), 1, f) == 1 &&
              std::fread(&nnz, sizeof(int64_t), 1, f) == 1;
    if (!ok || rows < 0 || cols < 0 || nnz < 0 || nnz > INT32_MAX) { std::fclose(f); return MF_ERR_IO; }
    std::vector<int64_t> rp(rows + 1);
    auto *m = new mf_matrix;
    m->n = rows;
    m->ncols = cols;
    m->col_idx.resize(nnz);
    m->val.resize(nnz);
    ok = std::fread(rp.data(), sizeof(int64_t), rows + 1, f) == (size_t)(rows + 1) &&
         std::fread(m->col_idx.data(), sizeof(int), nnz, f) == (size_t)nnz &&
         std::fread(m->val.data(), sizeof(double), nnz, f) == (size_t)nnz;
    std::fclose(f);
    if (!ok) { delete m; return MF_ERR_IO; }
    m->row_ptr.resize(rows + 1);
    for (int r = 0; r <= rows; ++r) m->row_ptr[r] = (int)rp[r];
    return finish(m, out);
}

int mf_write_cbd(const mf_matrix *m, const char *path) {
    if (!m || !path) return MF_ERR_ARG;
    FILE *f = std::fopen(path, "wb");
    if (!f) return MF_ERR_IO;
    const int rows = m->n, cols = m->ncols;
    const int64_t nnz = (int64_t)m->col_idx.size();
    std::vector<int64_t> rp(m->row_ptr.begin(), m->row_ptr.end());
    bool ok = std::fwrite(&rows, sizeof(int), 1, f) == 1 && std::fwrite(&cols, sizeof(int), 1, f) == 1 &&
              std::fwrite(&nnz, sizeof(int64_t), 1, f) == 1 &&
              std::fwrite(rp.data(), sizeof(int64_t), rows + 1, f) == (size_t)(rows + 1) &&
              std::fwrite(m->col_idx.data(), sizeof(int), nnz, f) == (size_t)nnz &&
              std::fwrite(m->val.data(), sizeof(double), nnz, f) == (size_t)nnz;
    std::fclose(f);
    return ok ? MF_OK : MF_ERR_IO;
}

int mf_matrix_from_csr(int n, int ncols, int nnz, const int *row_ptr, const int *col_idx,
                       const double *val, mf_matrix **out) {
    if (n < 0 || ncols < 0 || nnz < 0 || !row_ptr || !out || (nnz > 0 && (!col_idx || !val)))
        return MF_ERR_ARG;
    if (row_ptr[0] != 0 || row_ptr[n] != nnz) return MF_ERR_ARG;
    auto *m = new mf_matrix;
    m->n = n;
    m->ncols = ncols;
    m->row_ptr.assign(row_ptr, row_ptr + n + 1);
    m->col_idx.assign(col_idx, col_idx + nnz);
    m->val.assign(val, val + nnz);
    return finish(m, out);
}

int mf_matrix_info(const mf_matrix *m, int *n, int *ncols, int *nnz, int *has_b, int *has_xstar) {
    if (!m) return MF_ERR_ARG;
    if (n) *n = m->n;
    if (ncols) *ncols = m->ncols;
    if (nnz) *nnz = (int)m->col_idx.size();
    if (has_b) *has_b = !m->b.empty();
    if (has_xstar) *has_xstar = !m->xstar.empty();
    return MF_OK;
}

int mf_matrix_csr(const mf_matrix *m, mf_csr *csr) {
    if (!m || !csr) return MF_ERR_ARG;
    csr->n = m->n;
    csr->ncols = m->ncols;
    csr->nnz = (int)m->col_idx.size();
    csr->row_ptr = m->row_ptr.data();
    csr->col_idx = m->col_idx.data();
    csr->val = m->val.data();
    return MF_OK;
}

const double *mf_matrix_b(const mf_matrix *m) { return (m && !m->b.empty()) ? m->b.data() : nullptr; }
const double *mf_matrix_xstar(const mf_matrix *m) {
    return (m && !m->xstar.empty()) ? m->xstar.data() : nullptr;
}
int mf_matrix_set_b(mf_matrix *m, const double *b) {
    if (!m || !b) return MF_ERR_ARG;
    m->b.assign(b, b + m->n);
    return MF_OK;
}
void mf_matrix_free(mf_matrix *m) { delete m; }

}  // extern "C"
