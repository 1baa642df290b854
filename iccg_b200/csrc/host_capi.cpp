// host_capi.cpp -- extern "C" wrappers of the host-side routines (iccg.h).
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "host.hpp"
#include "../../include/iccg.h"

struct iccg_crs {
    iccg::CRS A;
};

namespace iccg {
thread_local std::string g_host_err;

template <class F>
int guarded(F&& f)
{
    try {
        f();
        return ICCG_OK;
    } catch (const Error& e) {
        g_host_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_host_err = "out of host memory";
        return ICCG_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return ICCG_ERR_ARG;
    }
}

// the argument checks of wrap() without its copy
void check_crs(int n, const int* rowptr, const int* colind, const double* val, bool need_val)
{
    if (n < 0 || !rowptr) throw Error(ICCG_ERR_ARG, "bad CRS arguments");
    const int nnz = rowptr[n];
    if (nnz < 0 || rowptr[0] != 0) throw Error(ICCG_ERR_ARG, "bad rowptr");
    // every row range inside [0, nnz]: the routines below read colind[k] for
    // k in [rowptr[i], rowptr[i+1])
    for (int i = 0; i < n; ++i)
        if (rowptr[i + 1] < rowptr[i] || rowptr[i + 1] > nnz)
            throw Error(ICCG_ERR_ARG, "rowptr must be nondecreasing and end at nnz");
    if (nnz > 0 && (!colind || (need_val && !val))) throw Error(ICCG_ERR_ARG, "null colind/val");
}

// a result matrix into the caller's arrays, on host threads
void copy_out(const CRS& B, int* rowptr, int* colind, double* val)
{
    const int T = host_threads(B.nnz());
    parallel_copy(rowptr, B.rowptr.data(), sizeof(int) * B.rowptr.size(), T);
    parallel_copy(colind, B.colind.data(), sizeof(int) * B.colind.size(), T);
    parallel_copy(val, B.val.data(), sizeof(double) * B.val.size(), T);
}

static CRS wrap(int n, const int* rowptr, const int* colind, const double* val)
{
    if (n < 0 || !rowptr) throw Error(ICCG_ERR_ARG, "bad CRS arguments");
    CRS A;
    A.n = n;
    A.rowptr.assign(rowptr, rowptr + n + 1);
    const int nnz = rowptr[n];
    if (nnz < 0 || rowptr[0] != 0) throw Error(ICCG_ERR_ARG, "bad rowptr");
    if (nnz > 0 && (!colind || !val)) throw Error(ICCG_ERR_ARG, "null colind/val");
    A.colind.assign(colind, colind + nnz);
    A.val.assign(val, val + nnz);
    return A;
}
}  // namespace iccg

using iccg::guarded;

extern "C" {

const char* iccg_last_error(void) { return iccg::g_host_err.c_str(); }

int iccg_mm_read(const char* path, iccg_crs** out)
{
    return guarded([&] {
        if (!path || !out) throw iccg::Error(ICCG_ERR_ARG, "null argument");
        auto* h = new iccg_crs;
        try {
            h->A = iccg::read_matrix_market_crs(path);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int iccg_mm_write(const char* path, int n, const int* rowptr, const int* colind, const double* val,
                  int symmetric)
{
    return guarded([&] { iccg::write_matrix_market(path, iccg::wrap(n, rowptr, colind, val), symmetric != 0); });
}

int iccg_crs_create(int n, const int* rowptr, const int* colind, const double* val, iccg_crs** out)
{
    return guarded([&] {
        auto* h = new iccg_crs;
        h->A = iccg::wrap(n, rowptr, colind, val);
        *out = h;
    });
}

int iccg_crs_dims(const iccg_crs* a, int* n, int* nnz)
{
    if (!a) return ICCG_ERR_ARG;
    if (n) *n = a->A.n;
    if (nnz) *nnz = a->A.nnz();
    return ICCG_OK;
}

int iccg_crs_copy(const iccg_crs* a, int* rowptr, int* colind, double* val)
{
    if (!a) return ICCG_ERR_ARG;
    if (rowptr) std::memcpy(rowptr, a->A.rowptr.data(), sizeof(int) * a->A.rowptr.size());
    if (colind) std::memcpy(colind, a->A.colind.data(), sizeof(int) * a->A.colind.size());
    if (val) std::memcpy(val, a->A.val.data(), sizeof(double) * a->A.val.size());
    return ICCG_OK;
}

void iccg_crs_free(iccg_crs* a) { delete a; }

int iccg_read_assignment(int kind, const char* path, int n_expected, int* out, int* k_out)
{
    return guarded([&] {
        int k = 0;
        auto v = iccg::read_assignment_1based(kind, path, n_expected, k);
        std::memcpy(out, v.data(), sizeof(int) * v.size());
        *k_out = k;
    });
}

int iccg_write_assignment(const char* path, int n, const int* values0, int k)
{
    return guarded([&] { iccg::write_assignment_1based(path, values0, n, k); });
}

int iccg_perm_by_color(int n, const int* color, int* new_of_old)
{
    return guarded([&] {
        std::vector<int> c(color, color + n);
        auto p = iccg::build_permutation_by_color(c);
        std::memcpy(new_of_old, p.data(), sizeof(int) * (size_t)n);
    });
}

int iccg_perm_by_block_color(int n, int nb, const int* block_of_old, const int* block_color,
                             int* new_of_old)
{
    return guarded([&] {
        for (int i = 0; i < n; ++i)
            if (block_of_old[i] < 0 || block_of_old[i] >= nb) throw iccg::Error(ICCG_ERR_ARG, "block id out of range");
        std::vector<int> b(block_of_old, block_of_old + n), c(block_color, block_color + nb);
        auto p = iccg::build_permutation_by_block_color(b, c);
        std::memcpy(new_of_old, p.data(), sizeof(int) * (size_t)n);
    });
}

int iccg_ptap_lower(int n, const int* rowptr, const int* colind, const double* val,
                    const int* new_of_old, int cap, int* out_rowptr, int* out_colind,
                    double* out_val, int* out_nnz)
{
    return guarded([&] {
        iccg::check_crs(n, rowptr, colind, val);
        if (n > 0 && !new_of_old) throw iccg::Error(ICCG_ERR_ARG, "null new_of_old");
        iccg::CRS B = iccg::permute_ptap_lower(n, rowptr, colind, val, new_of_old);
        if (B.nnz() > cap) throw iccg::Error(ICCG_ERR_ARG, "output capacity too small");
        iccg::copy_out(B, out_rowptr, out_colind, out_val);
        *out_nnz = B.nnz();
    });
}

int iccg_expand_lower_nnz(int n, const int* rowptr, const int* colind, int* out_nnz)
{
    return guarded([&] {
        if (!out_nnz) throw iccg::Error(ICCG_ERR_ARG, "null out_nnz");
        iccg::check_crs(n, rowptr, colind, nullptr, false);
        long long nz = 0;
        for (int i = 0; i < n; ++i)
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) nz += (colind[k] == i) ? 1 : 2;
        if (nz > 2147483647LL) throw iccg::Error(ICCG_ERR_ARG, "expanded matrix exceeds int32 nnz");
        *out_nnz = (int)nz;
    });
}

int iccg_expand_lower_to_full(int n, const int* rowptr, const int* colind, const double* val,
                              int* out_rowptr, int* out_colind, double* out_val)
{
    return guarded([&] {
        iccg::check_crs(n, rowptr, colind, val);
        iccg::copy_out(iccg::expand_lower_to_full(n, rowptr, colind, val), out_rowptr, out_colind, out_val);
    });
}

int iccg_color_schedule(int n, const int* color, int nc, const int* new_of_old, int* color_ptr,
                        int* rows_of_color)
{
    return guarded([&] {
        std::vector<int> c(color, color + n), p(new_of_old, new_of_old + n), cp, rc;
        iccg::build_color_schedule(c, nc, p, cp, rc);
        std::memcpy(color_ptr, cp.data(), sizeof(int) * cp.size());
        std::memcpy(rows_of_color, rc.data(), sizeof(int) * rc.size());
    });
}

int iccg_abmc_schedule(int n, const int* new_of_old, const int* block_of_old, const int* block_color,
                       int nb, int nc, int* color_ptr_blk, int* blocks_of_color, int* block_ptr,
                       int* rows_of_block)
{
    return guarded([&] {
        std::vector<int> p(new_of_old, new_of_old + n), b(block_of_old, block_of_old + n),
            c(block_color, block_color + nb), cpb, boc, bp, rob;
        iccg::build_abmc_schedule(p, b, c, nb, nc, cpb, boc, bp, rob);
        std::memcpy(color_ptr_blk, cpb.data(), sizeof(int) * cpb.size());
        std::memcpy(blocks_of_color, boc.data(), sizeof(int) * boc.size());
        std::memcpy(block_ptr, bp.data(), sizeof(int) * bp.size());
        std::memcpy(rows_of_block, rob.data(), sizeof(int) * rob.size());
    });
}

// DebugCheck_InterBlockSameColorEdges (cg_crs.cpp:171-224), as counts.
long long iccg_check_interblock_same_color(int n, const int* rowptr, const int* colind,
                                           const int* block_of_old, const int* block_color,
                                           int nb, int nc, long long* by_color)
{
    if (by_color) for (int c = 0; c < nc; ++c) by_color[c] = 0;
    long long total = 0;
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int j = colind[k];
            if (j <= i) continue;
            const int bi = block_of_old[i], bj = block_of_old[j];
            if (bi < 0 || bi >= nb || bj < 0 || bj >= nb) return ICCG_ERR_ARG;
            if (bi == bj) continue;
            const int ci = block_color[bi], cj = block_color[bj];
            if (ci < 0 || ci >= nc || cj < 0 || cj >= nc) return ICCG_ERR_ARG;
            if (ci == cj) { ++total; if (by_color) by_color[ci]++; }
        }
    return total;
}

// DebugCheck_ScheduleHazards_OnLower (cg_crs.cpp:259-336), as counts.
long long iccg_check_schedule_hazards(int n, const int* rowptr, const int* colind,
                                      const int* new_of_old, const int* color_old,
                                      const int* block_of_old, long long* same_block,
                                      long long* cross_block)
{
    std::vector<int> old_of_new((size_t)n, -1);
    for (int o = 0; o < n; ++o) {
        const int id = new_of_old[o];
        if (id < 0 || id >= n) return ICCG_ERR_ARG;
        old_of_new[(size_t)id] = o;
    }
    long long total = 0, sb = 0, xb = 0;
    for (int i = 0; i < n; ++i) {
        const int oi = old_of_new[(size_t)i];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int j = colind[k];
            if (j > i) continue;
            if (j == i) break;
            const int oj = old_of_new[(size_t)j];
            if (color_old[oj] == color_old[oi]) {
                ++total;
                if (block_of_old) (block_of_old[oi] == block_of_old[oj] ? sb : xb)++;
            }
        }
    }
    if (same_block) *same_block = sb;
    if (cross_block) *cross_block = xb;
    return total;
}

int iccg_gen_stencil(int kind, int nx, int ny, int nz, double wx, double wy, double wz, iccg_crs** out)
{
    return guarded([&] {
        auto* h = new iccg_crs;
        try { h->A = iccg::gen_stencil(kind, nx, ny, nz, wx, wy, wz); } catch (...) { delete h; throw; }
        *out = h;
    });
}

int iccg_gen_diffusion27(int nx, int ny, int nz, double contrast, unsigned long long seed, iccg_crs** out)
{
    return guarded([&] {
        auto* h = new iccg_crs;
        try { h->A = iccg::gen_diffusion27(nx, ny, nz, contrast, seed); } catch (...) { delete h; throw; }
        *out = h;
    });
}

int iccg_gen_knn_laplacian(int npts, int k, double diag_shift, unsigned long long seed, iccg_crs** out)
{
    return guarded([&] {
        auto* h = new iccg_crs;
        try { h->A = iccg::gen_knn_laplacian(npts, k, diag_shift, seed); } catch (...) { delete h; throw; }
        *out = h;
    });
}

// y = A x on the host with the reference's rounding (cg_crs.cpp:68-77:
// products and sums rounded separately, in CSR order).
int iccg_host_spmv(int n, const int* rowptr, const int* colind, const double* val, const double* x, double* y)
{
    return guarded([&] {
        if (n < 0 || !rowptr || !x || !y) throw iccg::Error(ICCG_ERR_ARG, "bad arguments");
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s = s + val[k] * x[colind[k]];
            y[i] = s;
        }
    });
}

int iccg_gen_uniform(int n, unsigned long long seed, double* out)
{
    return guarded([&] {
        if (n < 0 || (n > 0 && !out)) throw iccg::Error(ICCG_ERR_ARG, "bad arguments");
        iccg::gen_uniform(n, seed, out);
    });
}

int iccg_color_greedy(int n, const int* rowptr, const int* colind, int* color, int* nc)
{
    return guarded([&] { *nc = iccg::color_greedy(n, rowptr, colind, color); });
}

int iccg_block_partition(int n, const int* rowptr, const int* colind, int block_size, int method,
                         int* block_of_old, int* nb)
{
    return guarded([&] { *nb = iccg::block_partition(n, rowptr, colind, block_size, method, block_of_old); });
}

int iccg_color_blocks(int n, const int* rowptr, const int* colind, const int* block_of_old, int nb,
                      int* block_color, int* nc)
{
    return guarded([&] { *nc = iccg::color_blocks(n, rowptr, colind, block_of_old, nb, block_color); });
}

}  // extern "C"
