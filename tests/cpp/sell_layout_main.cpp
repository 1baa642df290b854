// sell_layout_main.cpp -- runs the host SELL-32 layout builder on one input
// for the CPU tests (tests/test_host_layouts.py).
//
//   sell_layout_main <in> <out> <threads>
//   in : int32 nq, nslices, slices[2 * nslices], n, nnz, rp[n+1], ci[nnz],
//        has_map, src_map[nnz if has_map], q2r[nq], r2q[n], unit_of[n],
//        step_of[n], encode
//   out: int32 status (0 built, 1 refused by the encoding, else the iccg.h
//        error code); on an error the message; when built: int64 slots,
//        int32 max_nin, then h_ptr h_col h_len src (int32) and prev_only
//        unit_only (uint8), each as int64 length + data
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../iccg_b200/csrc/host.hpp"

static FILE* g_in;

static int rd1()
{
    int32_t v = 0;
    if (std::fread(&v, sizeof(v), 1, g_in) != 1) std::exit(2);
    return v;
}

static std::vector<int> rdv(size_t n)
{
    std::vector<int> v(n);
    if (n && std::fread(v.data(), sizeof(int), n, g_in) != n) std::exit(2);
    return v;
}

template <class T>
static void wr(FILE* f, const std::vector<T>& v)
{
    const int64_t n = (int64_t)v.size();
    std::fwrite(&n, sizeof(n), 1, f);
    if (n) std::fwrite(v.data(), sizeof(T), v.size(), f);
}

int main(int argc, char** argv)
{
    if (argc != 4 || !(g_in = std::fopen(argv[1], "rb"))) return 2;
    iccg::SellOrder o;
    o.nq = rd1();
    const int ns = rd1();
    std::vector<std::pair<int, int>> slices((size_t)ns);
    for (auto& s : slices) {
        s.first = rd1();
        s.second = rd1();
    }
    const int n = rd1(), nnz = rd1();
    const std::vector<int> rp = rdv((size_t)n + 1), ci = rdv((size_t)nnz);
    const int has_map = rd1();
    const std::vector<int> map = rdv(has_map ? (size_t)nnz : 0);
    const std::vector<int> q2r = rdv((size_t)o.nq), r2q = rdv((size_t)n), unit_of = rdv((size_t)n),
                           step_of = rdv((size_t)n);
    const int encode = rd1();
    std::fclose(g_in);
    o.q2r = q2r.data();
    o.r2q = r2q.data();
    o.unit_of = unit_of.data();
    o.step_of = step_of.data();
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    iccg::SellLayout M;
    int32_t status = 0;
    try {
        if (!iccg::build_sell_layout(slices, rp.data(), ci.data(), has_map ? map.data() : nullptr, o, encode, M,
                                     std::atoi(argv[3])))
            status = 1;
    } catch (const iccg::Error& e) {
        status = e.code;
        std::fwrite(&status, sizeof(status), 1, out);
        std::fputs(e.what(), out);
        std::fclose(out);
        return 0;
    }
    std::fwrite(&status, sizeof(status), 1, out);
    if (status == 0) {
        const int64_t slots = M.slots;
        const int32_t nin = M.max_nin;
        std::fwrite(&slots, sizeof(slots), 1, out);
        std::fwrite(&nin, sizeof(nin), 1, out);
        for (const auto* v : {&M.h_ptr, &M.h_col, &M.h_len, &M.src}) wr(out, *v);
        wr(out, M.prev_only);
        wr(out, M.unit_only);
    }
    std::fclose(out);
    return 0;
}
