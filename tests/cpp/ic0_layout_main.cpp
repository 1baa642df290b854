// ic0_layout_main.cpp -- runs the host IC(0) layout builder on one matrix
// for the CPU tests (tests/test_host_layouts.py).
//
//   ic0_layout_main <in> <out> <threads>
//   in : int32 n, int32 nnz, int32 rowptr[n+1], int32 colind[nnz], float64 val[nnz]
//   out: int32 status (0 or the iccg.h error code); on error the message,
//        else each array as int64 length + data, in the order
//        Lp Li dpos Up Ui ut_src Sp Si s_src Tp Ti t_src (int32) Lx0 (float64)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../iccg_b200/csrc/host.hpp"

template <class T>
static bool rd(FILE* f, T* p, size_t n)
{
    return std::fread(p, sizeof(T), n, f) == n;
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
    if (argc != 4) return 2;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int32_t n = 0, nnz = 0;
    if (!rd(in, &n, 1) || !rd(in, &nnz, 1) || n < 0 || nnz < 0) return 2;
    std::vector<int> rp((size_t)n + 1), ci((size_t)nnz);
    std::vector<double> val((size_t)nnz);
    if (!rd(in, rp.data(), rp.size()) || !rd(in, ci.data(), ci.size()) || !rd(in, val.data(), val.size())) return 2;
    std::fclose(in);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    iccg::Ic0Layout L;
    std::vector<double> Lx0;
    int32_t status = 0;
    try {
        iccg::build_ic0_layout(n, rp.data(), ci.data(), val.data(), L, Lx0, std::atoi(argv[3]));
    } catch (const iccg::Error& e) {
        status = e.code;
        std::fwrite(&status, sizeof(status), 1, out);
        std::fputs(e.what(), out);
        std::fclose(out);
        return 0;
    }
    std::fwrite(&status, sizeof(status), 1, out);
    for (const auto* v : {&L.Lp, &L.Li, &L.dpos, &L.Up, &L.Ui, &L.ut_src, &L.Sp, &L.Si, &L.s_src, &L.Tp, &L.Ti, &L.t_src})
        wr(out, *v);
    wr(out, Lx0);
    std::fclose(out);
    return 0;
}
