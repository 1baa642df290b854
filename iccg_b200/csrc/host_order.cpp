// host_order.cpp -- file formats, permutations, P^T A P and schedules.
//
// New implementations (counting sorts, flat buckets) that reproduce the
// reference's results bit for bit; each function cites the reference
// routine whose output it must equal.
#include <algorithm>
#include <charconv>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>

#include "host.hpp"
#include "../../include/iccg.h"

namespace iccg {

namespace {

// whole-file reader
std::string slurp(const std::string& path)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(ICCG_ERR_IO, "Failed to open: " + path);
    std::string s;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz > 0) {
        s.resize((size_t)sz);
        size_t got = std::fread(&s[0], 1, (size_t)sz, f);
        s.resize(got);
    }
    std::fclose(f);
    return s;
}

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// Sequential line cursor over a buffer (getline semantics: the last line may
// lack a newline; a trailing newline does not produce an extra empty line).
struct Lines {
    const char* p;
    const char* end;
    bool next(const char*& b, const char*& e)
    {
        if (p >= end) return false;
        b = p;
        const char* nl = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        e = nl ? nl : end;
        p = nl ? nl + 1 : end;
        return true;
    }
};

// token reader within [p, e)
bool next_token(const char*& p, const char* e, std::string& tok)
{
    while (p < e && is_ws(*p)) ++p;
    if (p >= e) return false;
    const char* s = p;
    while (p < e && !is_ws(*p)) ++p;
    tok.assign(s, p);
    return true;
}

bool parse_ll(const char*& p, const char* e, long long& v)
{
    while (p < e && is_ws(*p)) ++p;
    if (p >= e) return false;
    {
        // plain decimal digits of up to 18 places end at whitespace or the
        // line's end: read directly (strtoll gives the same value); anything
        // else goes through strtoll below
        const char* q = p;
        long long x = 0;
        while (q < e && q - p < 18 && *q >= '0' && *q <= '9') x = x * 10 + (*q++ - '0');
        if (q > p && (q == e || is_ws(*q))) {
            v = x;
            p = q;
            return true;
        }
    }
    char buf[64];
    size_t len = 0;
    while (p + len < e && !is_ws(p[len]) && len < 63) { buf[len] = p[len]; ++len; }
    buf[len] = 0;
    char* q;
    errno = 0;
    v = std::strtoll(buf, &q, 10);
    if (q == buf) return false;
    p += (q - buf);
    return true;
}

bool parse_double(const char*& p, const char* e, double& v)
{
    while (p < e && is_ws(*p)) ++p;
    if (p >= e) return false;
    {
        // decimal forms: std::from_chars, correctly rounded like strtod, so
        // the same double; a token it does not take whole (a leading '+',
        // hexadecimal, inf / nan) goes through strtod below
        double x;
        const auto r = std::from_chars(p, e, x);
        if (r.ec == std::errc() && (r.ptr == e || is_ws(*r.ptr))) {
            v = x;
            p = r.ptr;
            return true;
        }
    }
    char buf[128];
    size_t len = 0;
    while (p + len < e && !is_ws(p[len]) && len < 127) { buf[len] = p[len]; ++len; }
    buf[len] = 0;
    char* q;
    v = std::strtod(buf, &q);
    if (q == buf) return false;
    p += (q - buf);
    return true;
}

std::string lower(std::string s)
{
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// true if some (row, column) occurs three or more times in the entry list
bool has_triple_entry(int nrows, const std::vector<int>& I, const std::vector<int>& J)
{
    const size_t m = I.size();
    std::vector<int> cnt((size_t)nrows + 1, 0);
    for (size_t t = 0; t < m; ++t) cnt[(size_t)I[t] + 1]++;
    for (int r = 0; r < nrows; ++r) cnt[(size_t)r + 1] += cnt[(size_t)r];
    std::vector<int> cols(m);
    {
        std::vector<int> cur(cnt.begin(), cnt.end() - 1);
        for (size_t t = 0; t < m; ++t) cols[(size_t)cur[(size_t)I[t]]++] = J[t];
    }
    for (int r = 0; r < nrows; ++r) {
        int* s = cols.data() + cnt[(size_t)r];
        int* e = cols.data() + cnt[(size_t)r + 1];
        if (e - s < 3) continue;
        std::sort(s, e);
        for (int* q = s + 2; q < e; ++q)
            if (q[0] == q[-2]) return true;
    }
    return false;
}

// coo_to_crs (crs_io.cpp:19-70) step for step: one std::sort of the entry
// indices by (row, column) with the reference's comparator, then the
// duplicates of each (row, column) summed in the order the sort left them.
// The same libstdc++ std::sort on the same sequence and comparator makes
// the same moves, so triples are summed in the reference's order.
CRS coo_to_crs_like_reference(int nrows, const std::vector<int>& I, const std::vector<int>& J,
                              const std::vector<double>& V)
{
    const size_t nnz = I.size();
    std::vector<size_t> ord(nnz);
    std::iota(ord.begin(), ord.end(), (size_t)0);
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
        if (I[a] != I[b]) return I[a] < I[b];
        return J[a] < J[b];
    });
    CRS A;
    A.n = nrows;
    A.rowptr.assign((size_t)nrows + 1, 0);
    A.colind.reserve(nnz);
    A.val.reserve(nnz);
    for (size_t idx = 0; idx < nnz;) {
        const int r = I[ord[idx]], c = J[ord[idx]];
        double s = 0.0;
        do {
            s += V[ord[idx]];
            ++idx;
        } while (idx < nnz && I[ord[idx]] == r && J[ord[idx]] == c);
        A.colind.push_back(c);
        A.val.push_back(s);
        A.rowptr[(size_t)r + 1]++;
    }
    for (int i = 0; i < nrows; ++i) A.rowptr[(size_t)i + 1] += A.rowptr[(size_t)i];
    return A;
}

}  // namespace

// read_matrix_market_crs (crs_io.cpp:73-159) with coo_to_crs (crs_io.cpp:19-70).
// Same accepted formats and error cases; parsing is a single pass over the
// file in memory.  Duplicate entries are summed in the reference's order.
CRS read_matrix_market_crs(const std::string& path)
{
    std::string buf = slurp(path);
    Lines L{buf.data(), buf.data() + buf.size()};
    const char *b, *e;
    if (!L.next(b, e)) throw Error(ICCG_ERR_IO, "Empty file");
    std::string banner, mtx, storage, field, symmetry;
    {
        const char* p = b;
        if (!(next_token(p, e, banner) && next_token(p, e, mtx) && next_token(p, e, storage) &&
              next_token(p, e, field) && next_token(p, e, symmetry)))
            throw Error(ICCG_ERR_IO, "Invalid MatrixMarket header");
        if (banner != "%%MatrixMarket") throw Error(ICCG_ERR_IO, "Not a MatrixMarket file");
        mtx = lower(mtx); storage = lower(storage); field = lower(field); symmetry = lower(symmetry);
        if (mtx != "matrix" || storage != "coordinate")
            throw Error(ICCG_ERR_IO, "Only 'matrix coordinate' is supported");
        if (!(field == "real" || field == "integer" || field == "pattern"))
            throw Error(ICCG_ERR_IO, "Unsupported field: " + field);
        if (!(symmetry == "general" || symmetry == "symmetric"))
            throw Error(ICCG_ERR_IO, "Unsupported symmetry: " + symmetry);
    }
    // skip comment lines, then the size line
    bool got = false;
    while (L.next(b, e)) {
        if (e > b && *b == '%') continue;
        got = true;
        break;
    }
    if (!got) throw Error(ICCG_ERR_IO, "Missing size line");
    long long nr, nc, nz;
    {
        const char* p = b;
        if (!(parse_ll(p, e, nr) && parse_ll(p, e, nc) && parse_ll(p, e, nz)))
            throw Error(ICCG_ERR_IO, "Invalid size line");
    }
    const int nrows = (int)nr, ncols = (int)nc, nnz = (int)nz;
    const bool sym = symmetry == "symmetric";
    const bool pattern = field == "pattern";
    std::vector<int> I, J;
    std::vector<double> V;
    size_t cap = (size_t)std::max(nnz, 0) * (sym ? 2 : 1);
    I.reserve(cap); J.reserve(cap); V.reserve(cap);
    auto push = [&](int i, int j, double v) {
        if (i < 0 || i >= nrows || j < 0 || j >= ncols) throw Error(ICCG_ERR_IO, "Index out of range");
        I.push_back(i); J.push_back(j); V.push_back(v);
    };
    for (int k = 0; k < nnz; ++k) {
        if (!L.next(b, e)) throw Error(ICCG_ERR_IO, "Unexpected EOF");
        if (e == b || *b == '%') { --k; continue; }
        const char* p = b;
        long long ii, jj;
        if (!(parse_ll(p, e, ii) && parse_ll(p, e, jj)))
            throw Error(ICCG_ERR_IO, "Invalid entry line (indices)");
        double v = 1.0;
        if (!pattern && !parse_double(p, e, v)) throw Error(ICCG_ERR_IO, "Invalid entry line (value)");
        int i = (int)(ii - 1), j = (int)(jj - 1);
        push(i, j, v);
        if (sym && i != j) push(j, i, v);
    }
    // COO -> CRS: bucket by row (stable), sort each row by column (stable),
    // sum duplicates in order.  Two entries of one (row, column) sum to the
    // same double in either order; three or more may not, and the reference
    // sums them in the order its std::sort over the whole entry list leaves
    // them (crs_io.cpp:27-45; introsort does not keep input order), so that
    // case is redone with the same call.
    CRS A;
    A.n = nrows;
    const size_t m = I.size();
    if (has_triple_entry(nrows, I, J)) return coo_to_crs_like_reference(nrows, I, J, V);
    std::vector<int> cnt((size_t)nrows + 1, 0);
    for (size_t t = 0; t < m; ++t) cnt[(size_t)I[t] + 1]++;
    for (int r = 0; r < nrows; ++r) cnt[(size_t)r + 1] += cnt[(size_t)r];
    std::vector<int> ord(m);
    {
        std::vector<int> cur(cnt.begin(), cnt.end() - 1);
        for (size_t t = 0; t < m; ++t) ord[(size_t)cur[(size_t)I[t]]++] = (int)t;
    }
    A.rowptr.assign((size_t)nrows + 1, 0);
    A.colind.reserve(m);
    A.val.reserve(m);
    for (int r = 0; r < nrows; ++r) {
        int* s = ord.data() + cnt[(size_t)r];
        int* t = ord.data() + cnt[(size_t)r + 1];
        if (t - s <= 32) {
            // short rows: stable insertion sort by column
            for (int* a = s + 1; a < t; ++a) {
                const int x = *a, cx = J[(size_t)x];
                int* b = a;
                while (b > s && J[(size_t)b[-1]] > cx) { *b = b[-1]; --b; }
                *b = x;
            }
        } else {
            std::stable_sort(s, t, [&](int a, int c) { return J[(size_t)a] < J[(size_t)c]; });
        }
        for (int* q = s; q < t;) {
            int c = J[(size_t)*q];
            double acc = 0.0;
            do { acc += V[(size_t)*q]; ++q; } while (q < t && J[(size_t)*q] == c);
            A.colind.push_back(c);
            A.val.push_back(acc);
        }
        A.rowptr[(size_t)r + 1] = (int)A.colind.size();
    }
    return A;
}

void write_matrix_market(const std::string& path, const CRS& A, bool symmetric_lower)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(ICCG_ERR_IO, "cannot write " + path);
    long long cnt = 0;
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k)
            if (!symmetric_lower || A.colind[k] <= i) ++cnt;
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real %s\n",
                 symmetric_lower ? "symmetric" : "general");
    std::fprintf(f, "%d %d %lld\n", A.n, A.n, cnt);
    // entry lines "i j v" with v as %.17g (std::to_chars with general format
    // and precision 17 prints exactly what printf does), formatted into one
    // buffer per chunk of rows and written with one call
    std::string out;
    out.reserve((size_t)std::min<long long>(cnt, 1 << 20) * 40 + 64);
    char num[96];  // one line needs at most 11 + 1 + 11 + 1 + 24 + 1 bytes
    char* const num_end = num + sizeof num;
    auto put = [&]() {
        if (!out.empty() && std::fwrite(out.data(), 1, out.size(), f) != out.size()) {
            std::fclose(f);
            throw Error(ICCG_ERR_IO, "cannot write " + path);
        }
        out.clear();
    };
    for (int i = 0; i < A.n; ++i) {
        for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k)
            if (!symmetric_lower || A.colind[k] <= i) {
                // each conversion leaves room for the separator after it
                char* q = std::to_chars(num, num_end - 1, i + 1).ptr;
                *q++ = ' ';
                q = std::to_chars(q, num_end - 1, A.colind[k] + 1).ptr;
                *q++ = ' ';
                q = std::to_chars(q, num_end - 1, A.val[k], std::chars_format::general, 17).ptr;
                *q++ = '\n';
                out.append(num, q);
            }
        if (out.size() > (32u << 20)) put();
    }
    put();
    std::fclose(f);
}

// ReadColorFile_1Based (color.cpp:14-47), ReadBlockFile_1Based
// (block.cpp:15-51), ReadBlockColorFile_1Based (block.cpp:53-89).
std::vector<int> read_assignment_1based(int kind, const std::string& path, int n_expected, int& k_out)
{
    static const char* what[3] = {"color", "block", "block-color"};
    if (kind < 0 || kind > 2) throw Error(ICCG_ERR_ARG, "bad assignment kind");
    std::string buf;
    try {
        buf = slurp(path);
    } catch (const Error&) {
        throw Error(ICCG_ERR_IO, std::string("cannot open ") + what[kind] + " file: " + path);
    }
    const char* p = buf.data();
    const char* e = p + buf.size();
    auto skipws = [&] { while (p < e && (is_ws(*p) || *p == '\n')) ++p; };
    auto read_int = [&](int& v) -> bool {
        skipws();
        if (p >= e) return false;
        char tmp[32];
        size_t len = 0;
        while (p + len < e && !is_ws(p[len]) && p[len] != '\n' && len < 31) { tmp[len] = p[len]; ++len; }
        tmp[len] = 0;
        char* q;
        long x = std::strtol(tmp, &q, 10);
        if (q == tmp) return false;
        p += (q - tmp);
        v = (int)x;
        return true;
    };
    int K = 0;
    if (!read_int(K)) throw Error(ICCG_ERR_IO, std::string("failed to read first line of ") + what[kind] + " file");
    if (K <= 0) throw Error(ICCG_ERR_IO, std::string(what[kind]) + " count must be positive");
    std::vector<int> out((size_t)std::max(n_expected, 0), -1);
    int assigned = 0, id, v;
    while (read_int(id) && read_int(v)) {
        if (id < 1 || id > n_expected)
            throw Error(ICCG_ERR_IO, std::string("id out of range in ") + what[kind] + " file: " + std::to_string(id));
        if (v < 1 || v > K)
            throw Error(ICCG_ERR_IO, std::string("value out of range in ") + what[kind] + " file: " + std::to_string(v));
        if (out[(size_t)id - 1] == -1) ++assigned;
        out[(size_t)id - 1] = v - 1;
    }
    if (assigned != n_expected)
        throw Error(ICCG_ERR_IO, std::string(what[kind]) + " file does not assign all ids: assigned=" +
                                     std::to_string(assigned) + " expected=" + std::to_string(n_expected));
    k_out = K;
    return out;
}

void write_assignment_1based(const std::string& path, const int* v0, int n, int k)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(ICCG_ERR_IO, "cannot write " + path);
    std::fprintf(f, "%d\n", k);
    for (int i = 0; i < n; ++i) std::fprintf(f, "%d %d\n", i + 1, v0[i] + 1);
    std::fclose(f);
}

namespace {

// stable counting sort of ids [0,n) by key[id] (ids ascending within a key)
std::vector<int> counting_order(const std::vector<int>& key, const std::vector<int>& ids_in)
{
    int lo = 0, hi = -1;
    for (int id : ids_in) { lo = std::min(lo, key[(size_t)id]); hi = std::max(hi, key[(size_t)id]); }
    std::vector<int> out(ids_in.size());
    if (ids_in.empty()) return out;
    long range = (long)hi - lo + 1;
    if (range > (long)ids_in.size() * 4 + 1024) {
        out = ids_in;
        std::stable_sort(out.begin(), out.end(), [&](int a, int b) { return key[(size_t)a] < key[(size_t)b]; });
        return out;
    }
    std::vector<int> cnt((size_t)range + 1, 0);
    for (int id : ids_in) cnt[(size_t)(key[(size_t)id] - lo) + 1]++;
    for (long r = 0; r < range; ++r) cnt[(size_t)r + 1] += cnt[(size_t)r];
    for (int id : ids_in) out[(size_t)cnt[(size_t)(key[(size_t)id] - lo)]++] = id;
    return out;
}

}  // namespace

// BuildPermutationByColor (color.cpp:50-63): order = ids sorted by
// (color, old id); new_of_old[order[k]] = k.
std::vector<int> build_permutation_by_color(const std::vector<int>& color)
{
    const int n = (int)color.size();
    std::vector<int> ids((size_t)n);
    std::iota(ids.begin(), ids.end(), 0);
    std::vector<int> order = counting_order(color, ids);
    std::vector<int> new_of_old((size_t)n);
    for (int k = 0; k < n; ++k) new_of_old[(size_t)order[(size_t)k]] = k;
    return new_of_old;
}

// BuildPermutationByBlockColor (block.cpp:92-114): sort by
// (block_color[block], block, old id), done as two stable counting passes.
std::vector<int> build_permutation_by_block_color(const std::vector<int>& block_of_old,
                                                  const std::vector<int>& block_color)
{
    const int n = (int)block_of_old.size();
    std::vector<int> ids((size_t)n);
    std::iota(ids.begin(), ids.end(), 0);
    std::vector<int> by_block = counting_order(block_of_old, ids);
    std::vector<int> ckey((size_t)n);
    for (int i = 0; i < n; ++i) ckey[(size_t)i] = block_color[(size_t)block_of_old[(size_t)i]];
    std::vector<int> order = counting_order(ckey, by_block);
    std::vector<int> new_of_old((size_t)n);
    for (int k = 0; k < n; ++k) new_of_old[(size_t)order[(size_t)k]] = k;
    return new_of_old;
}

namespace {

// Places the entries that a scan over input rows produces into the rows of
// a CRS matrix, keeping in each output row the order of a single scan over
// all input rows.  The input rows are split into parts; each part counts its
// entries per output row, and a part's entries land after those of the
// parts before it.  scan(i0, i1, put) calls put(row, col, val) for every
// entry that input rows [i0, i1) produce, in order.
template <class Scan>
void scatter_rows(int n_out, const std::vector<int>& parts, const Scan& scan, std::vector<int>& ptr,
                  std::vector<int>& col, std::vector<double>& val)
{
    const int T = (int)parts.size() - 1;
    std::vector<std::vector<int>> at((size_t)T);
    for (auto& a : at) a.reserve((size_t)n_out);  // filled (and first touched) by each part's thread
    run_parts(T, [&](int t) {
        std::vector<int>& c = at[(size_t)t];
        c.resize((size_t)n_out);
        scan(parts[(size_t)t], parts[(size_t)t + 1], [&](int r, int, double) { ++c[(size_t)r]; });
    });
    std::vector<int> ob((size_t)T + 1);
    for (int t = 0; t <= T; ++t) ob[(size_t)t] = (int)((long long)n_out * t / T);
    std::vector<long long> tot((size_t)T + 1, 0);
    run_parts(T, [&](int t) {
        long long s = 0;
        for (int r = ob[(size_t)t]; r < ob[(size_t)t + 1]; ++r)
            for (int u = 0; u < T; ++u) s += at[(size_t)u][(size_t)r];
        tot[(size_t)t + 1] = s;
    });
    scan_parts(tot);
    if (tot[(size_t)T] > 2147483647LL) throw Error(ICCG_ERR_ARG, "matrix exceeds int32 nnz");
    size_for_fill(ptr, (size_t)n_out + 1);
    // each part's count becomes the slot of its first entry in the row
    run_parts(T, [&](int t) {
        int a = (int)tot[(size_t)t];
        for (int r = ob[(size_t)t]; r < ob[(size_t)t + 1]; ++r) {
            ptr[(size_t)r] = a;
            for (int u = 0; u < T; ++u) {
                const int c = at[(size_t)u][(size_t)r];
                at[(size_t)u][(size_t)r] = a;
                a += c;
            }
        }
    });
    ptr[(size_t)n_out] = (int)tot[(size_t)T];
    size_for_fill(col, (size_t)tot[(size_t)T]);
    size_for_fill(val, (size_t)tot[(size_t)T]);
    run_parts(T, [&](int t) {
        std::vector<int>& next = at[(size_t)t];
        scan(parts[(size_t)t], parts[(size_t)t + 1], [&](int r, int c, double v) {
            const int p = next[(size_t)r]++;
            col[(size_t)p] = c;
            val[(size_t)p] = v;
        });
    });
}

// threads for scatter_rows over `entries` entries into n_out rows: each
// thread holds n_out counters, so their total stays within twice the entries
int scatter_threads(int n_out, long long entries)
{
    const long long cap = std::max(1ll, 2 * entries / std::max(1, n_out));
    return (int)std::max(1ll, std::min({(long long)host_threads(entries), (long long)std::max(1, n_out), cap}));
}

// stable insertion sort of (col, val)[b, e) by column
void sort_row_short(int* col, double* val, int b, int e)
{
    for (int t = b + 1; t < e; ++t) {
        const int c = col[t];
        const double v = val[t];
        int u = t - 1;
        while (u >= b && col[u] > c) {
            col[u + 1] = col[u];
            val[u + 1] = val[u];
            --u;
        }
        col[u + 1] = c;
        val[u + 1] = v;
    }
}

// Sorts (col, val)[b, e) by column as the reference's per-row std::sort of
// (column, value) pairs does (color.cpp:111-112): up to 16 entries that
// sort is an insertion sort, which keeps equal columns in input order (the
// routine above); longer rows go through the same std::sort call on the
// same sequence, so equal columns end in the reference's order and a long
// row costs O(m log m).
void sort_row_like_reference(int* col, double* val, int b, int e, std::vector<std::pair<int, double>>& tmp)
{
    if (e - b <= 16) {
        sort_row_short(col, val, b, e);
        return;
    }
    tmp.resize((size_t)(e - b));
    for (int q = b; q < e; ++q) tmp[(size_t)(q - b)] = {col[q], val[q]};
    std::sort(tmp.begin(), tmp.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (int q = b; q < e; ++q) {
        col[q] = tmp[(size_t)(q - b)].first;
        val[q] = tmp[(size_t)(q - b)].second;
    }
}

void check_indices(int n, const int* rp, const int* ci, const int* perm, const std::vector<int>& parts,
                   const char* what)
{
    const int T = (int)parts.size() - 1;
    std::vector<unsigned char> bad((size_t)T, 0);
    run_parts(T, [&](int t) {
        for (int i = parts[(size_t)t]; i < parts[(size_t)t + 1]; ++i) {
            if (perm && (perm[i] < 0 || perm[i] >= n)) bad[(size_t)t] = 1;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (ci[k] < 0 || ci[k] >= n) bad[(size_t)t] = 1;
        }
    });
    for (int t = 0; t < T; ++t)
        if (bad[(size_t)t]) throw Error(ICCG_ERR_ARG, std::string(what) + ": index out of range");
}

}  // namespace

// Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141).  Uses only j <= i of
// the input, folds each entry to (max(ip,jp), min(ip,jp)), sorts every row by
// column as the reference's std::sort does, sums duplicate columns in that
// order and drops sums equal to 0.0.
CRS permute_ptap_lower(int n, const int* rp, const int* ci, const double* v, const int* new_of_old)
{
    const int T = scatter_threads(n, n > 0 ? rp[n] : 0);
    const std::vector<int> parts = row_parts(n, rp, T);
    check_indices(n, rp, ci, new_of_old, parts, "Permute_PtAP");
    std::vector<int> bp, bc;
    std::vector<double> bv;
    scatter_rows(n, parts, [&](int i0, int i1, auto&& put) {
        for (int i = i0; i < i1; ++i) {
            const int ip = new_of_old[i];
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (j > i) continue;
                const int jp = new_of_old[j];
                put(std::max(ip, jp), std::min(ip, jp), v[k]);
            }
        }
    }, bp, bc, bv);
    // each row: sorted by column, equal columns summed in order, zero sums
    // dropped; the kept entries move to the front of the row's range
    CRS B;
    B.n = n;
    size_for_fill(B.rowptr, (size_t)n + 1);
    std::vector<int> ob((size_t)T + 1);
    for (int t = 0; t <= T; ++t) ob[(size_t)t] = (int)((long long)n * t / T);
    std::vector<long long> kept((size_t)T + 1, 0);
    std::vector<unsigned char> failed((size_t)T, 0);
    run_parts(T, [&](int t) {
      try {
        std::vector<std::pair<int, double>> tmp;
        long long s = 0;
        for (int r = ob[(size_t)t]; r < ob[(size_t)t + 1]; ++r) {
            const int b = bp[(size_t)r], e = bp[(size_t)r + 1];
            sort_row_like_reference(bc.data(), bv.data(), b, e, tmp);
            int w = b;
            if (e > b) {
                int cur_c = bc[(size_t)b];
                double acc = bv[(size_t)b];
                for (int q = b + 1; q < e; ++q) {
                    if (bc[(size_t)q] == cur_c) {
                        acc += bv[(size_t)q];
                    } else {
                        if (acc != 0.0) { bc[(size_t)w] = cur_c; bv[(size_t)w] = acc; ++w; }
                        cur_c = bc[(size_t)q];
                        acc = bv[(size_t)q];
                    }
                }
                if (acc != 0.0) { bc[(size_t)w] = cur_c; bv[(size_t)w] = acc; ++w; }
            }
            B.rowptr[(size_t)r] = w - b;
            s += w - b;
        }
        kept[(size_t)t + 1] = s;
      } catch (...) {
        failed[(size_t)t] = 1;
      }
    });
    for (int t = 0; t < T; ++t)
        if (failed[(size_t)t]) throw Error(ICCG_ERR_NOMEM, "Permute_PtAP: out of host memory");
    scan_parts(kept);
    run_parts(T, [&](int t) {
        int a = (int)kept[(size_t)t];
        for (int r = ob[(size_t)t]; r < ob[(size_t)t + 1]; ++r) {
            const int c = B.rowptr[(size_t)r];
            B.rowptr[(size_t)r] = a;
            a += c;
        }
    });
    B.rowptr[(size_t)n] = (int)kept[(size_t)T];
    size_for_fill(B.colind, (size_t)kept[(size_t)T]);
    size_for_fill(B.val, (size_t)kept[(size_t)T]);
    run_parts(T, [&](int t) {
        for (int r = ob[(size_t)t]; r < ob[(size_t)t + 1]; ++r) {
            const int d = B.rowptr[(size_t)r], m = B.rowptr[(size_t)r + 1] - d, b = bp[(size_t)r];
            std::copy(bc.begin() + b, bc.begin() + b + m, B.colind.begin() + d);
            std::copy(bv.begin() + b, bv.begin() + b + m, B.val.begin() + d);
        }
    });
    return B;
}

CRS permute_ptap_lower(const CRS& A, const std::vector<int>& new_of_old)
{
    const int n = A.n;
    if ((int)new_of_old.size() != n) throw Error(ICCG_ERR_ARG, "Permute_PtAP: new_of_old size mismatch");
    if ((int)A.rowptr.size() != n + 1) throw Error(ICCG_ERR_ARG, "Permute_PtAP: A.rowptr size mismatch");
    return permute_ptap_lower(n, A.rowptr.data(), A.colind.data(), A.val.data(), new_of_old.data());
}

// expand_lower_to_full (crs_io.cpp:163-227): diagonal once, (i,j) and (j,i)
// for each off-diagonal; columns sorted per row.  Row i of the output is
// (lower part of row i) followed by (transposed entries from rows k > i); for
// a lower, sorted input both arrive ascending and no row needs sorting.
CRS expand_lower_to_full(int n, const int* rp, const int* ci, const double* v)
{
    const int T = scatter_threads(n, n > 0 ? 2ll * rp[n] : 0);
    const std::vector<int> parts = row_parts(n, rp, T);
    check_indices(n, rp, ci, nullptr, parts, "expand_lower_to_full");
    CRS F;
    F.n = n;
    scatter_rows(n, parts, [&](int i0, int i1, auto&& put) {
        for (int i = i0; i < i1; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                put(i, j, v[k]);
                if (j != i) put(j, i, v[k]);
            }
    }, F.rowptr, F.colind, F.val);
    // per-row sort by column, as the reference's index sort (crs_io.cpp:
    // 203-219): rows of up to 16 entries are insertion-sorted by that
    // std::sort, which keeps equal columns in input order; a longer row with
    // equal columns goes through the same std::sort call on the same index
    // sequence, so its equal columns end in the reference's order; a row with
    // distinct columns has one sorted order
    std::vector<int> ob((size_t)T + 1);
    for (int t = 0; t <= T; ++t) ob[(size_t)t] = (int)((long long)n * t / T);
    std::vector<unsigned char> failed((size_t)T, 0);
    run_parts(T, [&](int t) {
        try {
            std::vector<std::pair<int, double>> row;
            std::vector<int> idx;
            for (int i = ob[(size_t)t]; i < ob[(size_t)t + 1]; ++i) {
                const int s = F.rowptr[(size_t)i], e = F.rowptr[(size_t)i + 1];
                bool sorted = true, distinct = true;
                for (int q = s + 1; q < e; ++q) {
                    if (F.colind[(size_t)q] < F.colind[(size_t)q - 1]) sorted = false;
                    if (F.colind[(size_t)q] == F.colind[(size_t)q - 1]) distinct = false;
                }
                if (sorted && (distinct || e - s <= 16)) continue;
                if (e - s <= 16) {
                    sort_row_short(F.colind.data(), F.val.data(), s, e);
                    continue;
                }
                row.clear();
                for (int q = s; q < e; ++q) row.emplace_back(F.colind[(size_t)q], F.val[(size_t)q]);
                if (distinct) {
                    std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
                } else {
                    idx.resize((size_t)(e - s));
                    std::iota(idx.begin(), idx.end(), 0);
                    std::sort(idx.begin(), idx.end(),
                              [&](int a, int b) { return row[(size_t)a].first < row[(size_t)b].first; });
                    std::vector<std::pair<int, double>> srt(idx.size());
                    for (size_t k = 0; k < idx.size(); ++k) srt[k] = row[(size_t)idx[k]];
                    row.swap(srt);
                }
                for (int q = s; q < e; ++q) {
                    F.colind[(size_t)q] = row[(size_t)(q - s)].first;
                    F.val[(size_t)q] = row[(size_t)(q - s)].second;
                }
            }
        } catch (...) {
            failed[(size_t)t] = 1;
        }
    });
    for (int t = 0; t < T; ++t)
        if (failed[(size_t)t]) throw Error(ICCG_ERR_NOMEM, "expand_lower_to_full: out of host memory");
    return F;
}

CRS expand_lower_to_full(const CRS& L)
{
    if ((int)L.rowptr.size() != L.n + 1) throw Error(ICCG_ERR_ARG, "expand_lower_to_full: rowptr size mismatch");
    return expand_lower_to_full(L.n, L.rowptr.data(), L.colind.data(), L.val.data());
}

// BuildColorPtrRows_FromPermutationAndColor (color.cpp:164-197)
void build_color_schedule(const std::vector<int>& color, int nc, const std::vector<int>& new_of_old,
                          std::vector<int>& color_ptr, std::vector<int>& rows_of_color)
{
    const int n = (int)color.size();
    if ((int)new_of_old.size() != n) throw Error(ICCG_ERR_ARG, "size mismatch");
    std::vector<int> old_of_new((size_t)n, -1);
    for (int o = 0; o < n; ++o) {
        const int id = new_of_old[(size_t)o];
        if (id < 0 || id >= n) throw Error(ICCG_ERR_ARG, "invert_permutation: out of range");
        old_of_new[(size_t)id] = o;
    }
    color_ptr.assign((size_t)nc + 1, 0);
    for (int i = 0; i < n; ++i) {
        const int c = color[(size_t)old_of_new[(size_t)i]];
        if ((unsigned)c >= (unsigned)nc) throw Error(ICCG_ERR_ARG, "color out of range");
        color_ptr[(size_t)c + 1]++;
    }
    for (int c = 0; c < nc; ++c) color_ptr[(size_t)c + 1] += color_ptr[(size_t)c];
    rows_of_color.assign((size_t)n, -1);
    std::vector<int> cur(color_ptr.begin(), color_ptr.end() - 1);
    for (int i = 0; i < n; ++i) rows_of_color[(size_t)cur[(size_t)color[(size_t)old_of_new[(size_t)i]]]++] = i;
}

// BuildABMCSchedule (block.cpp:116-174)
void build_abmc_schedule(const std::vector<int>& new_of_old, const std::vector<int>& block_of_old,
                         const std::vector<int>& block_color, int nb, int nc,
                         std::vector<int>& color_ptr_blk, std::vector<int>& blocks_of_color,
                         std::vector<int>& block_ptr, std::vector<int>& rows_of_block)
{
    const int n = (int)new_of_old.size();
    std::vector<int> old_of_new((size_t)n, -1);
    for (int o = 0; o < n; ++o) {
        const int id = new_of_old[(size_t)o];
        if (id < 0 || id >= n) throw Error(ICCG_ERR_ARG, "new_of_old out of range");
        old_of_new[(size_t)id] = o;
    }
    for (int o = 0; o < n; ++o) {
        const int b = block_of_old[(size_t)o];
        if (b < 0 || b >= nb) throw Error(ICCG_ERR_ARG, "block id out of range");
        if (block_color[(size_t)b] < 0 || block_color[(size_t)b] >= nc) throw Error(ICCG_ERR_ARG, "block color out of range");
    }
    std::vector<char> seen((size_t)nb, 0);
    color_ptr_blk.assign((size_t)nc + 1, 0);
    for (int i = 0; i < n; ++i) {
        const int b = block_of_old[(size_t)old_of_new[(size_t)i]];
        if (!seen[(size_t)b]) { seen[(size_t)b] = 1; color_ptr_blk[(size_t)block_color[(size_t)b] + 1]++; }
    }
    for (int c = 0; c < nc; ++c) color_ptr_blk[(size_t)c + 1] += color_ptr_blk[(size_t)c];
    blocks_of_color.assign((size_t)nb, -1);
    std::vector<int> cur(color_ptr_blk.begin(), color_ptr_blk.end() - 1);
    std::fill(seen.begin(), seen.end(), 0);
    for (int i = 0; i < n; ++i) {
        const int b = block_of_old[(size_t)old_of_new[(size_t)i]];
        if (!seen[(size_t)b]) { seen[(size_t)b] = 1; blocks_of_color[(size_t)cur[(size_t)block_color[(size_t)b]]++] = b; }
    }
    block_ptr.assign((size_t)nb + 1, 0);
    for (int i = 0; i < n; ++i) block_ptr[(size_t)block_of_old[(size_t)old_of_new[(size_t)i]] + 1]++;
    for (int b = 0; b < nb; ++b) block_ptr[(size_t)b + 1] += block_ptr[(size_t)b];
    rows_of_block.assign((size_t)n, -1);
    std::vector<int> cur2(block_ptr.begin(), block_ptr.end() - 1);
    for (int i = 0; i < n; ++i) rows_of_block[(size_t)cur2[(size_t)block_of_old[(size_t)old_of_new[(size_t)i]]]++] = i;
}

}  // namespace iccg
