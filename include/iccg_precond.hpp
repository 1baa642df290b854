// iccg_precond.hpp -- header-only C++ adapters over the C ABI (iccg.h) that
// satisfy the preconditioner concept of stomo0511/ICCG's
// conjugate_gradient<Precond> (cg_crs.cpp:89-98):
//
//   explicit P(const CRS&)  /  IC0(const CRS&, double shift)   (ic0.hpp:13)
//   void apply(const std::vector<double>& r, std::vector<double>& z,
//              const ColorSchedule* sched) const                (precond.hpp:12,
//                                                                precond.hpp:38,
//                                                                ic0.hpp:34)
//   std::string name() const                                    (precond.hpp:16,44)
//
// so the reference's own CG template can drive the GPU preconditioner
// unchanged, and iccg::gpu_conjugate_gradient() replaces the whole solve.
// Template parameters let the caller's CRS / ColorSchedule types (the
// reference's structs, crs_io.hpp:10-49 and color.hpp:9-22) be used directly;
// only their documented members are read.  Failing C ABI calls are rethrown
// as std::runtime_error, as the reference reports errors.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "iccg.h"

namespace iccg {

inline void check(int rc, iccg_ctx* ctx)
{
    if (rc != ICCG_OK) throw std::runtime_error(ctx ? iccg_ctx_last_error(ctx) : iccg_last_error());
}

// One device context holding A_run, the schedule and the preconditioner.
class GpuSystem {
public:
    template <class CRS>
    explicit GpuSystem(const CRS& A, int device = 0)
    {
        check(iccg_ctx_create(device, &ctx_), nullptr);
        n_ = A.n;
        check(iccg_matrix_upload(ctx_, A.n, A.rowptr.data(), A.colind.data(), A.val.data()), ctx_);
    }
    ~GpuSystem() { iccg_ctx_destroy(ctx_); }
    GpuSystem(const GpuSystem&) = delete;
    GpuSystem& operator=(const GpuSystem&) = delete;

    // IC0::apply's dispatch on the schedule (ic0.cpp:366-393).  The
    // schedule is sent to the device again whenever its contents differ from
    // the last one sent: the same object refilled, or another object at a
    // reused address, is not taken for the old schedule.  The check copies
    // and compares the schedule's arrays (O(n) host work per call).
    template <class Sched>
    void set_schedule(const Sched* s)
    {
        std::vector<int> key;
        int mode = 0;  // 0 none, 1 MC, 2 ABMC
        if (s && s->nc > 0) {
            if (s->mode == Sched::ABMC_BLOCK && s->color_ptr_blk && s->blocks_of_color && s->block_ptr &&
                s->rows_of_block)
                mode = 2;
            else if (s->color_ptr && s->rows_of_color)
                mode = 1;
        }
        key.push_back(mode);
        if (mode == 1) {
            key.push_back(s->nc);
            key.insert(key.end(), s->color_ptr, s->color_ptr + s->nc + 1);
            key.insert(key.end(), s->rows_of_color, s->rows_of_color + n_);
        } else if (mode == 2) {
            key.push_back(s->nc);
            key.push_back(s->nb);
            key.insert(key.end(), s->color_ptr_blk, s->color_ptr_blk + s->nc + 1);
            key.insert(key.end(), s->blocks_of_color, s->blocks_of_color + s->nb);
            key.insert(key.end(), s->block_ptr, s->block_ptr + s->nb + 1);
            key.insert(key.end(), s->rows_of_block, s->rows_of_block + n_);
        }
        if (have_key_ && key == key_) return;
        have_key_ = false;
        if (mode == 2) {
            check(iccg_schedule_abmc(ctx_, s->nc, s->nb, s->color_ptr_blk, s->blocks_of_color, s->block_ptr,
                                     s->rows_of_block),
                  ctx_);
        } else if (mode == 1) {
            check(iccg_schedule_mc(ctx_, s->nc, s->color_ptr, s->rows_of_color), ctx_);
        } else {
            check(iccg_schedule_none(ctx_), ctx_);
        }
        key_.swap(key);
        have_key_ = true;
    }
    iccg_ctx* ctx() const { return ctx_; }
    int n() const { return n_; }

private:
    iccg_ctx* ctx_ = nullptr;
    int n_ = 0;
    bool have_key_ = false;
    std::vector<int> key_;  // mode, sizes and arrays of the schedule on the device
};

// Precond::apply over the device; z is resized like the reference does.
template <int KIND>
class GpuPrecond {
public:
    template <class CRS>
    explicit GpuPrecond(const CRS& A, double shift = 1e-12, int device = 0, int storage = ICCG_STORE_FP64)
        : sys_(new GpuSystem(A, device)), storage_(storage)
    {
        check(iccg_precond_build(sys_->ctx(), KIND, shift, 0), sys_->ctx());
    }
    ~GpuPrecond() { delete sys_; }
    GpuPrecond(const GpuPrecond&) = delete;
    GpuPrecond& operator=(const GpuPrecond&) = delete;

    template <class Sched>
    void apply(const std::vector<double>& r, std::vector<double>& z, const Sched* sched) const
    {
        sys_->set_schedule(sched);
        if ((int)z.size() != sys_->n()) z.resize(sys_->n());
        check(iccg_precond_apply(sys_->ctx(), r.data(), z.data(), storage_), sys_->ctx());
    }
    std::string name() const
    {
        return KIND == ICCG_PRECOND_NONE ? "No preconditioner"
               : KIND == ICCG_PRECOND_JACOBI ? "Jacobi preconditioner"
                                             : "IC preconditioner with multi-coloring";
    }
    GpuSystem& system() const { return *sys_; }

private:
    GpuSystem* sys_;
    int storage_;
};

using GpuIdentity = GpuPrecond<ICCG_PRECOND_NONE>;
using GpuJacobi = GpuPrecond<ICCG_PRECOND_JACOBI>;
using GpuIC0 = GpuPrecond<ICCG_PRECOND_IC0>;

struct GpuCGResult {
    int iters = 0;
    double rel_resid = 0.0;
    bool converged = false;
    double true_rel_resid = 0.0;
    double solve_ms = 0.0;
};

// The whole conjugate_gradient (cg_crs.cpp:89-162) on the device: x holds x0
// on entry and the solution on return.
template <class Sched, int KIND>
GpuCGResult gpu_conjugate_gradient(const std::vector<double>& b, std::vector<double>& x, const GpuPrecond<KIND>& M,
                                   int max_iter, double tol, const Sched* sched,
                                   const iccg_solve_opts* opts = nullptr)
{
    M.system().set_schedule(sched);
    iccg_result res{};
    check(iccg_solve(M.system().ctx(), b.data(), x.data(), max_iter, tol, opts, &res), M.system().ctx());
    GpuCGResult out;
    out.iters = res.iters;
    out.rel_resid = res.rel_resid;
    out.converged = res.converged != 0;
    out.true_rel_resid = res.true_rel_resid;
    out.solve_ms = res.solve_ms;
    return out;
}

}  // namespace iccg
