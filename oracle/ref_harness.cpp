// ref_harness.cpp -- C entry points around the UNMODIFIED reference sources.
//
// TEST INFRASTRUCTURE ONLY (the oracle side).  The Makefile in this directory
// compiles this file together with the reference's crs_io.cpp, ic0.cpp,
// color.cpp and block.cpp, straight from the reference checkout, into
// oracle/_ref/libiccg_ref.so.  Nothing here is shipped with, or called by,
// the product library.
//
// cg_crs.cpp is #included with its `main` renamed, so spmv / dot / nrm2 /
// conjugate_gradient (cg_crs.cpp:33-162) are the reference's own code.  The
// driver steps of main (cg_crs.cpp:377-484) are replayed by ref_problem_create
// for the five reference binaries (Makefile:18-53):
//   variant 0 cg_crs    (-DNOPRE)  Identity,  A_run = A
//   variant 1 dcg_crs   (-DJAC)    Jacobi,    A_run = A
//   variant 2 iccg_crs  (-DIC)     IC0,       A_run = A, no schedule
//   variant 3 piccg_crs (-DPIC)    IC0 + MC schedule on P^T A P
//   variant 4 abmc_crs  (-DABMC)   IC0 + ABMC schedule on P^T A P
// The harness is compiled once with -DIC -DPIC -DABMC; with a null schedule
// IC0::apply takes the sequential path of the non-PIC build (ic0.cpp:368).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

#include "crs_io.hpp"
#include "color.hpp"
#include "block.hpp"
#include "precond.hpp"   // Identity / Jacobi: cg_crs.cpp includes it only without -DIC
// The factor arrays of IC0 are private; the oracle reads them for parity.
#define private public
#include "ic0.hpp"
#undef private

#define main iccg_reference_main
#include "cg_crs.cpp"
#undef main

namespace {

thread_local std::string g_err;

struct RefProblem {
    int variant = 0;
    CRS A;          // as given (original order)
    CRS Ap;         // A_run for variants 3/4
    std::vector<int> new_of_old, color;
    std::vector<int> color_ptr, rows_of_color;
    std::vector<int> color_ptr_blk, blocks_of_color, block_ptr, rows_of_block;
    int nc = 0, nb = 0;
    ColorSchedule sched;
    const ColorSchedule* sched_ptr = nullptr;
    std::unique_ptr<Identity> M0;
    std::unique_ptr<Jacobi> M1;
    std::unique_ptr<IC0> M2;
    const CRS& arun() const { return variant >= 3 ? Ap : A; }
};

CRS make_crs(int n, const int* rowptr, const int* colind, const double* val)
{
    CRS A;
    A.n = n;
    int nnz = rowptr[n];
    A.rowptr.assign(rowptr, rowptr + n + 1);
    A.colind.assign(colind, colind + nnz);
    A.val.assign(val, val + nnz);
    return A;
}

template <class F>
int guarded(F&& f)
{
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }
void ref_set_threads(int t) { omp_set_num_threads(t); }
int ref_max_threads(void) { return omp_get_max_threads(); }

// variant: see the header comment.  color0 = node colors (variant 3, 0-based,
// nc colors) or block_of_old (variant 4, nb blocks); bcolor0 = block colors
// (variant 4, nc colors).  shift is the IC0 shift (the reference's main
// passes 0.0, cg_crs.cpp:454).
void* ref_problem_create(int variant, int n, const int* rowptr, const int* colind,
                         const double* val, const int* color0, int k0,
                         const int* bcolor0, int nc, double shift)
{
    RefProblem* P = new RefProblem;
    int rc = guarded([&] {
        P->variant = variant;
        P->A = make_crs(n, rowptr, colind, val);
        if (variant == 3) {
            P->nc = k0;
            P->color.assign(color0, color0 + n);
            P->new_of_old = BuildPermutationByColor(P->color);
        } else if (variant == 4) {
            P->nb = k0;
            P->nc = nc;
            std::vector<int> block_of_old(color0, color0 + n);
            std::vector<int> block_color(bcolor0, bcolor0 + k0);
            P->color.resize(n);
            for (int i = 0; i < n; ++i) P->color[i] = block_color[block_of_old[i]];
            P->new_of_old = BuildPermutationByBlockColor(block_of_old, block_color);
            BuildABMCSchedule(P->new_of_old, block_of_old, block_color, P->nb, P->nc,
                              P->color_ptr_blk, P->blocks_of_color, P->block_ptr,
                              P->rows_of_block);
        }
        if (variant >= 3) {
            P->Ap = Permute_PtAP_LowerCRS_to_LowerCRS(P->A, P->new_of_old);
            P->Ap = expand_lower_to_full(P->Ap);
            BuildColorPtrRows_FromPermutationAndColor(P->color, P->nc, P->new_of_old,
                                                      P->color_ptr, P->rows_of_color);
        }
        if (variant == 0) P->M0.reset(new Identity(P->arun()));
        if (variant == 1) P->M1.reset(new Jacobi(P->arun()));
        if (variant >= 2) P->M2.reset(new IC0(P->arun(), shift));
        if (variant == 3) {
            P->sched.nc = P->nc;
            P->sched.color_ptr = P->color_ptr.data();
            P->sched.rows_of_color = P->rows_of_color.data();
            P->sched_ptr = &P->sched;
        } else if (variant == 4) {
            P->sched.mode = ColorSchedule::ABMC_BLOCK;
            P->sched.nc = P->nc;
            P->sched.nb = P->nb;
            P->sched.color_ptr_blk = P->color_ptr_blk.data();
            P->sched.blocks_of_color = P->blocks_of_color.data();
            P->sched.block_ptr = P->block_ptr.data();
            P->sched.rows_of_block = P->rows_of_block.data();
            P->sched_ptr = &P->sched;
        }
    });
    if (rc) { delete P; return nullptr; }
    return P;
}

void ref_problem_free(void* h) { delete static_cast<RefProblem*>(h); }

int ref_problem_n(void* h) { return static_cast<RefProblem*>(h)->arun().n; }
int ref_problem_nnz(void* h) { return (int)static_cast<RefProblem*>(h)->arun().colind.size(); }

void ref_problem_arun(void* h, int* rowptr, int* colind, double* val)
{
    const CRS& A = static_cast<RefProblem*>(h)->arun();
    std::copy(A.rowptr.begin(), A.rowptr.end(), rowptr);
    std::copy(A.colind.begin(), A.colind.end(), colind);
    std::copy(A.val.begin(), A.val.end(), val);
}

void ref_problem_perm(void* h, int* new_of_old)
{
    auto* P = static_cast<RefProblem*>(h);
    std::copy(P->new_of_old.begin(), P->new_of_old.end(), new_of_old);
}

int ref_problem_nc(void* h) { return static_cast<RefProblem*>(h)->nc; }
int ref_problem_nb(void* h) { return static_cast<RefProblem*>(h)->nb; }

void ref_problem_sched_mc(void* h, int* color_ptr, int* rows_of_color)
{
    auto* P = static_cast<RefProblem*>(h);
    std::copy(P->color_ptr.begin(), P->color_ptr.end(), color_ptr);
    std::copy(P->rows_of_color.begin(), P->rows_of_color.end(), rows_of_color);
}

void ref_problem_sched_abmc(void* h, int* color_ptr_blk, int* blocks_of_color,
                            int* block_ptr, int* rows_of_block)
{
    auto* P = static_cast<RefProblem*>(h);
    std::copy(P->color_ptr_blk.begin(), P->color_ptr_blk.end(), color_ptr_blk);
    std::copy(P->blocks_of_color.begin(), P->blocks_of_color.end(), blocks_of_color);
    std::copy(P->block_ptr.begin(), P->block_ptr.end(), block_ptr);
    std::copy(P->rows_of_block.begin(), P->rows_of_block.end(), rows_of_block);
}

int ref_problem_ic0_nnz(void* h)
{
    auto* P = static_cast<RefProblem*>(h);
    return P->M2 ? (int)P->M2->L_colind.size() : -1;
}

void ref_problem_ic0_export(void* h, int* Lp, int* Li, double* Lx, int* Up, int* Ui, double* Ux)
{
    auto* P = static_cast<RefProblem*>(h);
    const IC0& M = *P->M2;
    std::copy(M.L_rowptr.begin(), M.L_rowptr.end(), Lp);
    std::copy(M.L_colind.begin(), M.L_colind.end(), Li);
    std::copy(M.L_val.begin(), M.L_val.end(), Lx);
    std::copy(M.LT_colptr.begin(), M.LT_colptr.end(), Up);
    std::copy(M.LT_rowind.begin(), M.LT_rowind.end(), Ui);
    std::copy(M.LT_val.begin(), M.LT_val.end(), Ux);
}

void ref_apply(void* h, const double* r, double* z)
{
    auto* P = static_cast<RefProblem*>(h);
    int n = P->arun().n;
    std::vector<double> rv(r, r + n), zv(n);
    if (P->M0) P->M0->apply(rv, zv, P->sched_ptr);
    if (P->M1) P->M1->apply(rv, zv, P->sched_ptr);
    if (P->M2) P->M2->apply(rv, zv, P->sched_ptr);
    std::copy(zv.begin(), zv.end(), z);
}

void ref_spmv(void* h, const double* x, double* y)
{
    auto* P = static_cast<RefProblem*>(h);
    int n = P->arun().n;
    std::vector<double> xv(x, x + n), yv(n);
    spmv(P->arun(), xv, yv);
    std::copy(yv.begin(), yv.end(), y);
}

double ref_dot(int n, const double* a, const double* b)
{
    std::vector<double> av(a, a + n), bv(b, b + n);
    return dot(av, bv);
}

double ref_nrm2(int n, const double* a)
{
    std::vector<double> av(a, a + n);
    return nrm2(av);
}

// conjugate_gradient on A_run with the problem's preconditioner; x in/out.
// elapsed_us: time of conjugate_gradient alone (cg_crs.cpp:507-510, in us).
int ref_cg(void* h, const double* b, double* x, int max_iter, double tol,
           int* iters, double* rel, int* converged, double* elapsed_us)
{
    auto* P = static_cast<RefProblem*>(h);
    int n = P->arun().n;
    std::vector<double> bv(b, b + n), xv(x, x + n);
    CGResult out;
    auto t0 = std::chrono::steady_clock::now();
    if (P->M0) out = conjugate_gradient(P->arun(), bv, xv, *P->M0, max_iter, tol, P->sched_ptr);
    if (P->M1) out = conjugate_gradient(P->arun(), bv, xv, *P->M1, max_iter, tol, P->sched_ptr);
    if (P->M2) out = conjugate_gradient(P->arun(), bv, xv, *P->M2, max_iter, tol, P->sched_ptr);
    auto t1 = std::chrono::steady_clock::now();
    if (elapsed_us) *elapsed_us = std::chrono::duration<double, std::micro>(t1 - t0).count();
    std::copy(xv.begin(), xv.end(), x);
    *iters = out.iters;
    *rel = out.rel_resid;
    *converged = out.converged ? 1 : 0;
    return 0;
}

// Readers: the reference's own parsers (crs_io.cpp:73-159, color.cpp:14-47,
// block.cpp:15-89).  ref_read_mm returns a heap CRS handle.
void* ref_read_mm(const char* path)
{
    CRS* A = new CRS;
    int rc = guarded([&] { *A = read_matrix_market_crs(path); });
    if (rc) { delete A; return nullptr; }
    return A;
}
int ref_crs_n(void* h) { return static_cast<CRS*>(h)->n; }
int ref_crs_nnz(void* h) { return (int)static_cast<CRS*>(h)->colind.size(); }
void ref_crs_copy(void* h, int* rowptr, int* colind, double* val)
{
    CRS* A = static_cast<CRS*>(h);
    std::copy(A->rowptr.begin(), A->rowptr.end(), rowptr);
    std::copy(A->colind.begin(), A->colind.end(), colind);
    std::copy(A->val.begin(), A->val.end(), val);
}
void ref_crs_free(void* h) { delete static_cast<CRS*>(h); }

// Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141) and
// expand_lower_to_full (crs_io.cpp:163-227) themselves, on caller arrays;
// the result is returned as a heap CRS handle (ref_crs_* accessors).
void* ref_ptap_lower(int n, const int* rowptr, const int* colind, const double* val, const int* new_of_old)
{
    CRS* B = new CRS;
    int rc = guarded([&] {
        CRS A = make_crs(n, rowptr, colind, val);
        std::vector<int> p(new_of_old, new_of_old + n);
        *B = Permute_PtAP_LowerCRS_to_LowerCRS(A, p);
    });
    if (rc) { delete B; return nullptr; }
    return B;
}

void* ref_expand_lower_to_full(int n, const int* rowptr, const int* colind, const double* val)
{
    CRS* B = new CRS;
    int rc = guarded([&] { *B = expand_lower_to_full(make_crs(n, rowptr, colind, val)); });
    if (rc) { delete B; return nullptr; }
    return B;
}

// kind: 0 color file, 1 block file, 2 block-color file
int ref_read_assignment(int kind, const char* path, int n_expected, int* out, int* k_out)
{
    return guarded([&] {
        int k = 0;
        std::vector<int> v;
        if (kind == 0) v = ReadColorFile_1Based(path, n_expected, k);
        else if (kind == 1) v = ReadBlockFile_1Based(path, n_expected, k);
        else v = ReadBlockColorFile_1Based(path, n_expected, k);
        std::copy(v.begin(), v.end(), out);
        *k_out = k;
    });
}

}  // extern "C"
