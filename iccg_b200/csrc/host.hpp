// host.hpp -- host-side data structures and set-up routines of iccg_b200.
//
// The CRS container and ColorSchedule view keep the reference's layout
// (crs_io.hpp:10-49, color.hpp:9-22).  Every ordering routine here is a new
// implementation that reproduces the reference's output bit for bit; the
// file:line of the reference function each one stands in for is given at
// its definition.
#pragma once
#include <sys/mman.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace iccg {

struct CRS {
    int n = 0;
    std::vector<int> rowptr;   // n+1
    std::vector<int> colind;   // nnz
    std::vector<double> val;   // nnz
    int nnz() const { return (int)colind.size(); }
};

struct ColorSchedule {
    int nc = 0;
    const int* color_ptr = nullptr;
    const int* rows_of_color = nullptr;
    enum Mode { MC_NODE, ABMC_BLOCK } mode = MC_NODE;
    int nb = 0;
    const int* color_ptr_blk = nullptr;
    const int* blocks_of_color = nullptr;
    const int* block_ptr = nullptr;
    const int* rows_of_block = nullptr;
};

// Error carrying an iccg.h status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---- formats ----
CRS read_matrix_market_crs(const std::string& path);
void write_matrix_market(const std::string& path, const CRS& A, bool symmetric_lower);
std::vector<int> read_assignment_1based(int kind, const std::string& path, int n_expected,
                                        int& k_out);
void write_assignment_1based(const std::string& path, const int* v0, int n, int k);

// ---- orderings / schedules ----
std::vector<int> build_permutation_by_color(const std::vector<int>& color);
std::vector<int> build_permutation_by_block_color(const std::vector<int>& block_of_old,
                                                  const std::vector<int>& block_color);
CRS permute_ptap_lower(const CRS& A, const std::vector<int>& new_of_old);
CRS permute_ptap_lower(int n, const int* rowptr, const int* colind, const double* val, const int* new_of_old);
CRS expand_lower_to_full(const CRS& L);
CRS expand_lower_to_full(int n, const int* rowptr, const int* colind, const double* val);
// C ABI argument checks of a CRS (rowptr nondecreasing, inside [0, nnz]) and
// the copy of a result into caller arrays (host_capi.cpp)
void check_crs(int n, const int* rowptr, const int* colind, const double* val, bool need_val = true);
void copy_out(const CRS& B, int* rowptr, int* colind, double* val);
void build_color_schedule(const std::vector<int>& color, int nc,
                          const std::vector<int>& new_of_old, std::vector<int>& color_ptr,
                          std::vector<int>& rows_of_color);
void build_abmc_schedule(const std::vector<int>& new_of_old, const std::vector<int>& block_of_old,
                         const std::vector<int>& block_color, int nb, int nc,
                         std::vector<int>& color_ptr_blk, std::vector<int>& blocks_of_color,
                         std::vector<int>& block_ptr, std::vector<int>& rows_of_block);

// ---- generators ----
CRS gen_stencil(int kind, int nx, int ny, int nz, double wx, double wy, double wz);
CRS gen_diffusion27(int nx, int ny, int nz, double contrast, uint64_t seed);
CRS gen_knn_laplacian(int npts, int k, double diag_shift, uint64_t seed);
void gen_uniform(int n, uint64_t seed, double* out);
int color_greedy(int n, const int* rowptr, const int* colind, int* color);
int block_partition(int n, const int* rowptr, const int* colind, int B, int method,
                    int* block_of_old);
int color_blocks(int n, const int* rowptr, const int* colind, const int* block_of_old, int nb,
                 int* block_color);

// ---- host threads ----
// Threads worth using for a host pass over `work` matrix entries: 1 below
// about a million, else up to 16.  ICCG_HOST_THREADS in the environment
// sets the count instead (results never depend on it).
inline int host_threads(long long work)
{
    if (const char* e = std::getenv("ICCG_HOST_THREADS")) {
        const int t = std::atoi(e);
        if (t > 0) return std::min(t, 256);
    }
    if (work < (1ll << 20)) return 1;
    const long long hw = std::max(1u, std::thread::hardware_concurrency());
    return (int)std::min({hw, 16ll, work >> 18});
}

// fn(t) for t = 0..T-1 on T threads (the caller's is one).  Parts whose
// thread cannot be started run on the caller's thread.  fn must not throw.
template <class Fn>
void run_parts(int T, const Fn& fn)
{
    if (T <= 1) {
        fn(0);
        return;
    }
    std::vector<std::thread> th;
    th.reserve((size_t)T - 1);
    int started = 1;
    try {
        for (; started < T; ++started) th.emplace_back(fn, started);
    } catch (...) {
    }
    fn(0);
    for (int t = started; t < T; ++t) fn(t);
    for (auto& x : th) x.join();
}

// s[1..T] holds per-part sums; makes s[t] the sum of the parts before t
inline void scan_parts(std::vector<long long>& s)
{
    for (size_t t = 1; t < s.size(); ++t) s[t] += s[t - 1];
}

// T + 1 row boundaries splitting rows [0, n) into parts with about equal
// numbers of entries of rowptr
inline std::vector<int> row_parts(int n, const int* rowptr, int T)
{
    std::vector<int> rb((size_t)T + 1, 0);
    const long long nnz = n > 0 ? rowptr[n] : 0;
    for (int t = 1; t <= T; ++t) {
        rb[(size_t)t] = t == T ? n : (int)(std::lower_bound(rowptr, rowptr + n, (int)(nnz * t / T)) - rowptr);
        rb[(size_t)t] = std::max(rb[(size_t)t], rb[(size_t)t - 1]);
    }
    return rb;
}

// memcpy split over T threads (a fresh destination faults its pages in
// parallel)
void parallel_copy(void* dst, const void* src, size_t bytes, int T);

// Sizes v to `count` elements for a caller that then writes all of them.
// A vector that must grow is reallocated without copying its old contents,
// and its range is advised for transparent huge pages before the first
// touch: on a large system the set-up is bound by faults on fresh host
// pages, and a 2 MB page is one fault instead of 512.
template <class T>
void size_for_fill(std::vector<T>& v, size_t count)
{
    if (v.capacity() < count) {
        std::vector<T>().swap(v);
        v.reserve(count);
        const uintptr_t huge = (uintptr_t)2 << 20, a = (uintptr_t)v.data();
        const uintptr_t b = (a + huge - 1) & ~(huge - 1), e = (a + count * sizeof(T)) & ~(huge - 1);
        if (e > b) (void)madvise((void*)b, e - b, MADV_HUGEPAGE);
    }
    v.resize(count);
}

// ---- IC(0) layout ----
// The sparsity layout of IC(0) on A's lower triangle: L's rows (Lp, Li) and
// diagonal places (dpos), its columns (Up, Ui, ut_src = each column entry's
// index into Li), the strictly lower part of L's rows (Sp, Si, s_src) and
// the strictly upper part of L^T's rows (Tp, Ti, t_src).
struct Ic0Layout {
    std::vector<int> Lp, Li, dpos, Up, Ui, ut_src, Sp, Si, s_src, Tp, Ti, t_src;
};
// Builds L's layout and its initial values Lx0 (A's lower entries) on
// `threads` host threads; the result is the same for every thread count.
// Throws Error(ICCG_ERR_DIAG) naming the first row without a diagonal entry.
void build_ic0_layout(int n, const int* rowptr, const int* colind, const double* val, Ic0Layout& out,
                      std::vector<double>& Lx0, int threads);

// ---- SELL-32 layout ----
// The row order of a lane-interleaved matrix: Q row q holds CRS row q2r[q]
// (r2q is its inverse), of unit unit_of[r] at step step_of[r] of the unit.
struct SellOrder {
    int nq = 0;
    const int* q2r = nullptr;
    const int* r2q = nullptr;
    const int* unit_of = nullptr;
    const int* step_of = nullptr;
};
// Host arrays of a SELL-32 matrix.  Slice s (32 Q rows) occupies slots
// [h_ptr[s], h_ptr[s+1]); entry j of the slice's lane l sits at slot
// h_ptr[s] + 32 j + l.  h_col is a Q column, or -(step + 1) for an entry of
// the row's own unit in an encoded matrix; src is the entry's CRS value
// index (-1 on padding); h_len[q] = row length | in-unit entries << 16.
struct SellLayout {
    long long slots = 0;
    int max_nin = 0;           // most in-unit entries of a row (encoded matrices)
    std::vector<int> h_ptr;    // slices + 1
    std::vector<int> h_col;    // slots
    std::vector<int> h_len;    // Q rows
    std::vector<int> src;      // slots
    // encoded matrices, per Q row: 1 when the row has at most one in-unit
    // entry and that entry is the unit's row one step before it in the
    // sweep's order
    std::vector<unsigned char> prev_only;
    std::vector<unsigned char> unit_only;  // encoded: 1 when every entry of the row is in-unit
};
// Fills M for the rows of `slices` ((first Q row, rows) pairs) of the CRS
// pattern (rp, ci); src_map, when given, maps a CRS entry to its value
// index.  encode 1 (forward) or 2 (backward) marks in-unit entries, which
// must come last (1) or first (2) in every row; otherwise it returns false
// and leaves M as it was.  Throws Error(ICCG_ERR_ARG) when the slots
// overflow int32 or a row is longer than 65535 entries.
bool build_sell_layout(const std::vector<std::pair<int, int>>& slices, const int* rp, const int* ci,
                       const int* src_map, const SellOrder& order, int encode, SellLayout& M, int threads);

// splitmix64 step
inline uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double u01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * 0x1.0p-53; }

}  // namespace iccg
