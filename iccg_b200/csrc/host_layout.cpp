// host_layout.cpp -- the host-side layouts of the device matrices, built on
// host threads: the IC(0) sparsity layout of a CRS matrix and the SELL-32
// slot layout of a matrix in lane-interleaved row order.
//
// One pass of counts, an exclusive scan and one pass of fills per array, so
// every array is sized exactly once: on a large system the set-up is bound
// by first touches of fresh host pages, not by arithmetic.  Row passes split
// the rows into chunks with about equal numbers of A's entries; column and
// slice passes split the columns or slices into equal ranges.  Each thread
// writes only its own rows', columns' or slices' slots, with the values a
// single thread would write, so the result does not depend on the number of
// threads.
#include <algorithm>
#include <cstring>

#include "host.hpp"
#include "../../include/iccg.h"

namespace iccg {

// extract_lower_with_diag (ic0.cpp:14-38), diag_pos (ic0.cpp:47-54) and
// build_csc_from_crs (ic0.cpp:118-151) of the reference, plus the strict
// lower / strict upper split the substitutions run on.
void build_ic0_layout(int n, const int* rp, const int* ci, const double* val, Ic0Layout& L,
                      std::vector<double>& Lx0, int threads)
{
    const int T = std::max(1, std::min(threads, n));
    // row parts: about nnz / T of A's entries each; column parts: n / T columns
    const std::vector<int> rb = row_parts(n, rp, T);
    std::vector<int> cb((size_t)T + 1, 0);
    for (int t = 1; t <= T; ++t) cb[(size_t)t] = (int)((long long)n * t / T);

    // rows: entries of L (columns <= i), the strictly lower ones before the
    // first diagonal entry, and that entry's place in the row
    size_for_fill(L.Lp, (size_t)n + 1);
    size_for_fill(L.Sp, (size_t)n + 1);
    size_for_fill(L.dpos, (size_t)n);
    std::vector<long long> sl((size_t)T + 1, 0), ss((size_t)T + 1, 0);
    std::vector<int> missing((size_t)T, -1);
    run_parts(T, [&](int t) {
        long long a = 0, b = 0;
        for (int i = rb[(size_t)t]; i < rb[(size_t)t + 1]; ++i) {
            int cl = 0, cs = 0;
            bool diag = false;
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (j > i) continue;
                if (!diag) {
                    if (j == i) diag = true;
                    else ++cs;
                }
                ++cl;
            }
            L.Lp[(size_t)i] = cl;
            L.Sp[(size_t)i] = cs;
            L.dpos[(size_t)i] = diag ? cs : -1;
            if (!diag && missing[(size_t)t] < 0) missing[(size_t)t] = i;
            a += cl;
            b += cs;
        }
        sl[(size_t)t + 1] = a;
        ss[(size_t)t + 1] = b;
    });
    for (int t = 0; t < T; ++t)
        if (missing[(size_t)t] >= 0)
            throw Error(ICCG_ERR_DIAG, "IC(0): diagonal missing at row " + std::to_string(missing[(size_t)t]));
    scan_parts(sl);
    scan_parts(ss);
    const int nnzL = (int)sl[(size_t)T], nnzS = (int)ss[(size_t)T];
    run_parts(T, [&](int t) {
        int a = (int)sl[(size_t)t], b = (int)ss[(size_t)t];
        for (int i = rb[(size_t)t]; i < rb[(size_t)t + 1]; ++i) {
            const int cl = L.Lp[(size_t)i], cs = L.Sp[(size_t)i];
            L.Lp[(size_t)i] = a;
            L.Sp[(size_t)i] = b;
            L.dpos[(size_t)i] += a;
            a += cl;
            b += cs;
        }
    });
    L.Lp[(size_t)n] = nnzL;
    L.Sp[(size_t)n] = nnzS;

    size_for_fill(L.Li, (size_t)nnzL);
    size_for_fill(Lx0, (size_t)nnzL);
    size_for_fill(L.Si, (size_t)nnzS);
    size_for_fill(L.s_src, (size_t)nnzS);
    run_parts(T, [&](int t) {
        for (int i = rb[(size_t)t]; i < rb[(size_t)t + 1]; ++i) {
            const int l0 = L.Lp[(size_t)i], s0 = L.Sp[(size_t)i], cs = L.Sp[(size_t)i + 1] - s0;
            int p = l0;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (ci[k] <= i) {
                    L.Li[(size_t)p] = ci[k];
                    Lx0[(size_t)p] = val[k];
                    ++p;
                }
            for (int m = 0; m < cs; ++m) {
                L.Si[(size_t)s0 + m] = L.Li[(size_t)l0 + m];
                L.s_src[(size_t)s0 + m] = l0 + m;
            }
        }
    });

    // columns of L (its CSC), by row parts: part u counts, per column, the
    // entries of its rows; a column's entries from part u follow those of
    // the parts before it, so every column lists its rows in ascending order,
    // as a single scan of the rows would.  Each part holds n counters, so the
    // parts are capped at about twice the entries per column.
    size_for_fill(L.Up, (size_t)n + 1);
    size_for_fill(L.Tp, (size_t)n + 1);
    const int TU = (int)std::max(1ll, std::min<long long>(T, 2ll * nnzL / std::max(1, n)));
    const std::vector<int> ub = row_parts(n, L.Lp.data(), TU);
    std::vector<std::vector<int>> at((size_t)TU);
    run_parts(TU, [&](int u) {
        std::vector<int>& c = at[(size_t)u];
        c.assign((size_t)n, 0);
        for (int k = L.Lp[(size_t)ub[(size_t)u]]; k < L.Lp[(size_t)ub[(size_t)u + 1]]; ++k) ++c[(size_t)L.Li[(size_t)k]];
    });
    std::vector<long long> su((size_t)T + 1, 0), st((size_t)T + 1, 0);
    run_parts(T, [&](int t) {
        long long s = 0;
        for (int j = cb[(size_t)t]; j < cb[(size_t)t + 1]; ++j)
            for (int u = 0; u < TU; ++u) s += at[(size_t)u][(size_t)j];
        su[(size_t)t + 1] = s;
    });
    scan_parts(su);
    // each part's count becomes the slot of its first entry in the column
    run_parts(T, [&](int t) {
        int a = (int)su[(size_t)t];
        for (int j = cb[(size_t)t]; j < cb[(size_t)t + 1]; ++j) {
            L.Up[(size_t)j] = a;
            for (int u = 0; u < TU; ++u) {
                const int c = at[(size_t)u][(size_t)j];
                at[(size_t)u][(size_t)j] = a;
                a += c;
            }
        }
    });
    L.Up[(size_t)n] = nnzL;
    size_for_fill(L.Ui, (size_t)nnzL);
    size_for_fill(L.ut_src, (size_t)nnzL);
    run_parts(TU, [&](int u) {
        std::vector<int>& next = at[(size_t)u];
        for (int i = ub[(size_t)u]; i < ub[(size_t)u + 1]; ++i)
            for (int k = L.Lp[(size_t)i]; k < L.Lp[(size_t)i + 1]; ++k) {
                const int p = next[(size_t)L.Li[(size_t)k]]++;
                L.Ui[(size_t)p] = i;
                L.ut_src[(size_t)p] = k;
            }
    });
    std::vector<std::vector<int>>().swap(at);
    run_parts(T, [&](int t) {
        const int c0 = cb[(size_t)t], c1 = cb[(size_t)t + 1];
        if (c0 >= c1) return;
        // rows of L^T: the strictly upper entries of each column
        long long s = 0;
        for (int j = c0; j < c1; ++j) {
            int c = 0;
            for (int k = L.Up[(size_t)j]; k < L.Up[(size_t)j + 1]; ++k) c += L.Ui[(size_t)k] > j;
            L.Tp[(size_t)j] = c;
            s += c;
        }
        st[(size_t)t + 1] = s;
    });
    scan_parts(st);
    const int nnzT = (int)st[(size_t)T];
    size_for_fill(L.Ti, (size_t)nnzT);
    size_for_fill(L.t_src, (size_t)nnzT);
    run_parts(T, [&](int t) {
        int a = (int)st[(size_t)t];
        for (int j = cb[(size_t)t]; j < cb[(size_t)t + 1]; ++j) {
            L.Tp[(size_t)j] = a;
            for (int k = L.Up[(size_t)j]; k < L.Up[(size_t)j + 1]; ++k)
                if (L.Ui[(size_t)k] > j) {
                    L.Ti[(size_t)a] = L.Ui[(size_t)k];
                    L.t_src[(size_t)a] = L.ut_src[(size_t)k];
                    ++a;
                }
        }
    });
    L.Tp[(size_t)n] = nnzT;
}


bool build_sell_layout(const std::vector<std::pair<int, int>>& slices, const int* rp, const int* ci,
                       const int* src_map, const SellOrder& o, int encode, SellLayout& M, int threads)
{
    const int ns = (int)slices.size();
    const int T = std::max(1, std::min(threads, ns));
    std::vector<int> sb((size_t)T + 1, 0);
    for (int t = 1; t <= T; ++t) sb[(size_t)t] = (int)((long long)ns * t / T);
    auto in_unit = [&](int r, int cj) { return o.unit_of[cj] == o.unit_of[r]; };

    // an encoded matrix needs the in-unit entries of each row last (forward)
    // or first (backward)
    if (encode) {
        std::vector<unsigned char> ok((size_t)T, 1);
        run_parts(T, [&](int t) {
            for (int s = sb[(size_t)t]; s < sb[(size_t)t + 1] && ok[(size_t)t]; ++s)
                for (int l = 0; l < slices[(size_t)s].second; ++l) {
                    const int r = o.q2r[slices[(size_t)s].first + l];
                    bool seen_in = false, seen_out = false;
                    for (int k = rp[r]; k < rp[r + 1]; ++k) {
                        const bool inside = in_unit(r, ci[k]);
                        if ((encode == 1 && seen_in && !inside) || (encode == 2 && seen_out && inside)) {
                            ok[(size_t)t] = 0;
                            break;
                        }
                        seen_in |= inside;
                        seen_out |= !inside;
                    }
                }
        });
        for (int t = 0; t < T; ++t)
            if (!ok[(size_t)t]) return false;
    }

    // slice widths (longest row), then the slot offsets
    size_for_fill(M.h_ptr, (size_t)ns + 1);
    std::vector<unsigned char> too_long((size_t)T, 0);
    run_parts(T, [&](int t) {
        for (int s = sb[(size_t)t]; s < sb[(size_t)t + 1]; ++s) {
            int w = 0;
            for (int l = 0; l < slices[(size_t)s].second; ++l) {
                const int r = o.q2r[slices[(size_t)s].first + l];
                w = std::max(w, rp[r + 1] - rp[r]);
            }
            M.h_ptr[(size_t)s] = w;
            if (w > 0xffff) too_long[(size_t)t] = 1;
        }
    });
    long long slot = 0;
    for (int s = 0; s < ns; ++s) slot += 32LL * M.h_ptr[(size_t)s];
    if (slot > 2147483647LL) throw Error(ICCG_ERR_ARG, "matrix too large for int32 SELL slots");
    for (int t = 0; t < T; ++t)
        if (too_long[(size_t)t]) throw Error(ICCG_ERR_ARG, "row longer than 65535 entries");
    slot = 0;
    for (int s = 0; s < ns; ++s) {
        const int w = M.h_ptr[(size_t)s];
        M.h_ptr[(size_t)s] = (int)slot;
        slot += 32LL * w;
    }
    M.h_ptr[(size_t)ns] = (int)slot;
    M.slots = slot;

    // slots: lane l of slice s holds entry j of its row at ptr[s] + 32 j + l;
    // padding has column 0 and source -1
    size_for_fill(M.h_col, (size_t)slot);
    size_for_fill(M.src, (size_t)slot);
    size_for_fill(M.h_len, (size_t)o.nq);
    size_for_fill(M.prev_only, encode ? (size_t)o.nq : 0);
    size_for_fill(M.unit_only, encode ? (size_t)o.nq : 0);
    std::vector<int> nin_max((size_t)T, 0);
    run_parts(T, [&](int t) {
        int most = 0;
        for (int s = sb[(size_t)t]; s < sb[(size_t)t + 1]; ++s) {
            const int p0 = M.h_ptr[(size_t)s], p1 = M.h_ptr[(size_t)s + 1];
            std::fill(M.h_col.begin() + p0, M.h_col.begin() + p1, 0);
            std::fill(M.src.begin() + p0, M.src.begin() + p1, -1);
            for (int l = 0; l < slices[(size_t)s].second; ++l) {
                const int q = slices[(size_t)s].first + l;
                const int r = o.q2r[q];
                const int b = rp[r], L = rp[r + 1] - b;
                int nin = 0;
                bool prev = true;
                for (int j = 0; j < L; ++j) {
                    const size_t pos = (size_t)p0 + 32 * (size_t)j + (size_t)l;
                    const int cj = ci[b + j];
                    if (encode && in_unit(r, cj)) {
                        M.h_col[pos] = -(o.step_of[cj] + 1);
                        ++nin;
                        prev = prev && o.step_of[cj] == o.step_of[r] + (encode == 1 ? -1 : 1);
                    } else {
                        M.h_col[pos] = o.r2q[cj];
                    }
                    M.src[pos] = src_map ? src_map[b + j] : b + j;
                }
                M.h_len[(size_t)q] = L | (nin << 16);
                most = std::max(most, nin);
                if (encode) {
                    M.prev_only[(size_t)q] = (unsigned char)(prev && nin <= 1);
                    M.unit_only[(size_t)q] = (unsigned char)(nin == L);
                }
            }
        }
        nin_max[(size_t)t] = most;
    });
    M.max_nin = *std::max_element(nin_max.begin(), nin_max.end());
    return true;
}

void parallel_copy(void* dst, const void* src, size_t bytes, int T)
{
    T = std::max(1, T);
    run_parts(T, [&](int t) {
        const size_t b0 = bytes * (size_t)t / (size_t)T, b1 = bytes * (size_t)(t + 1) / (size_t)T;
        if (b1 > b0) std::memcpy((char*)dst + b0, (const char*)src + b0, b1 - b0);
    });
}

}  // namespace iccg
