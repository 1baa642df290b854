// dropin_check.cpp -- the reference's own conjugate_gradient<Precond>
// template (cg_crs.cpp:89-162, compiled from the reference sources) driven
// by the GPU preconditioner adapter iccg::GpuIC0 (include/iccg_precond.hpp)
// in place of IC0, next to the same template with the reference's IC0.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref (it
// contains reference code), run by the GPU tests.
//
// usage: dropin_check A.mtx B.blk C.bcol [tol] [max_iter]
// Replays the set-up of the reference's main for abmc_crs
// (cg_crs.cpp:377-481) with b = 1, prints one JSON line.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "crs_io.hpp"
#include "color.hpp"
#include "block.hpp"
#include "ic0.hpp"

#define main iccg_reference_main
#include "cg_crs.cpp"
#undef main

#include "iccg_precond.hpp"

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s A.mtx B.blk C.bcol [tol] [max_iter]\n", argv[0]);
        return 2;
    }
    const double tol = argc >= 5 ? std::atof(argv[4]) : 1e-8;
    const int max_iter = argc >= 6 ? std::atoi(argv[5]) : 10000;
    CRS A = read_matrix_market_crs(argv[1]);
    int nbs = 0, nbc = 0;
    std::vector<int> block_of_old = ReadBlockFile_1Based(argv[2], A.n, nbs);
    std::vector<int> block_color = ReadBlockColorFile_1Based(argv[3], nbs, nbc);
    std::vector<int> new_of_old = BuildPermutationByBlockColor(block_of_old, block_color);
    CRS Ap = Permute_PtAP_LowerCRS_to_LowerCRS(A, new_of_old);
    Ap = expand_lower_to_full(Ap);
    std::vector<int> color_ptr_blk, blocks_of_color, block_ptr, rows_of_block;
    BuildABMCSchedule(new_of_old, block_of_old, block_color, nbs, nbc, color_ptr_blk, blocks_of_color, block_ptr,
                      rows_of_block);
    ColorSchedule sched;
    sched.mode = ColorSchedule::ABMC_BLOCK;
    sched.nc = nbc;
    sched.nb = nbs;
    sched.color_ptr_blk = color_ptr_blk.data();
    sched.blocks_of_color = blocks_of_color.data();
    sched.block_ptr = block_ptr.data();
    sched.rows_of_block = rows_of_block.data();

    std::vector<double> b(A.n, 1.0);
    std::vector<double> x_ref(A.n, 0.0), x_gpu(A.n, 0.0), x_full(A.n, 0.0);
    IC0 M(Ap, 0.0);
    CGResult r_ref = conjugate_gradient(Ap, b, x_ref, M, max_iter, tol, &sched);
    // the same template, the GPU preconditioner behind the same interface
    iccg::GpuIC0 G(Ap, 0.0);
    CGResult r_gpu = conjugate_gradient(Ap, b, x_gpu, G, max_iter, tol, &sched);
    // the whole solve on the device
    iccg::GpuCGResult r_full = iccg::gpu_conjugate_gradient(b, x_full, G, max_iter, tol, &sched);
    double d1 = 0, d2 = 0, nx = 0;
    for (int i = 0; i < A.n; ++i) {
        d1 += (x_gpu[i] - x_ref[i]) * (x_gpu[i] - x_ref[i]);
        d2 += (x_full[i] - x_ref[i]) * (x_full[i] - x_ref[i]);
        nx += x_ref[i] * x_ref[i];
    }
    std::printf("{\"n\": %d, \"ref_iters\": %d, \"ref_rel\": %.17g, \"adapter_iters\": %d, \"adapter_rel\": %.17g, "
                "\"adapter_x_rel_err\": %.3e, \"gpu_iters\": %d, \"gpu_converged\": %d, \"gpu_x_rel_err\": %.3e, "
                "\"name\": \"%s\"}\n",
                A.n, r_ref.iters, r_ref.rel_resid, r_gpu.iters, r_gpu.rel_resid, std::sqrt(d1 / nx), r_full.iters,
                r_full.converged ? 1 : 0, std::sqrt(d2 / nx), G.name().c_str());
    return 0;
}
