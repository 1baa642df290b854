// kernels.cuh -- sm_100a kernels of the ICCG hot path.
//
// Every floating-point step is evaluated with the rounding the reference
// build gets from g++ (-O3, x86-64-v3 with FMA): the substitution sweeps
// (ic0.cpp:153-339, `acc -= L*y`), the two-pointer dot of the IC(0) factor
// (ic0.cpp:64-81) and the CG vector updates (cg_crs.cpp:137-141, 155-157)
// are fused multiply-adds, written as explicit fma(); the spmv row sum
// (cg_crs.cpp:73-75) and the IC(0) sum of squares (ic0.cpp:93-99) are a
// separately rounded product and sum, which g++ does not contract.  The file
// is compiled with --fmad=false so nvcc adds no contraction of its own.  The
// FP64 kernels therefore reproduce the reference's bits.  Inner products use
// the double-double reductions of dd.cuh.
//
// Reductions end in a "last block" step: every CTA writes its partial to a
// fixed slot, the CTA that takes the last ticket sums the slots in index
// order and runs the CG scalar logic of the reference (breakdown test, alpha,
// convergence test, beta) on the device.  Kernels of the fused path start
// with a uniform read of the solver status and return when the solve has
// already finished, so a CUDA graph may replay iterations past convergence.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd.cuh"

namespace iccg {

constexpr int kRunning = -1;
constexpr int kConverged = 0;
constexpr int kBreakdown = 1;
constexpr int kMaxIter = 2;
constexpr int kNonFinite = 3;
constexpr int kTrueCheck = 4;  // stopped: the recurrence residual passed the tolerance and the
                               // host is to confirm it with an FP64 residual (mixed precision)

// Device-resident CG state (one per context).
struct SolverState {
    double normb, rz_old, alpha, beta, rel_resid, tol;
    int k;            // iterations started
    int iters;        // CGResult::iters
    int status;       // kRunning / kConverged / ...
    int max_iter;
    int rr_interval;  // 0: FP64 path, no replacement
    int rr_flag;      // replacement requested by the update step
    int n_rr;
    int pend;         // a stop decided by the persistent apply's own reductions (kRunning: none);
                      // the p update that follows the apply moves it into `status`
    unsigned int ticket;
    int true_check;   // 1: a recurrence residual below tol asks for an FP64 residual check in the same
                      // iteration (rr_flag) instead of stopping with kTrueCheck (the batched solves)
    unsigned long long t_stop;  // %globaltimer (ns) when the solve stopped (0 while running)
    unsigned long long t_start; // %globaltimer (ns) when a batched solve was admitted
    int xdefer_k;     // the last iteration whose x += alpha p waits for the p update (FIN_UPDX); -1: none
    int xp;           // 1: the solve stopped before that x update (applied by k_apply_xp)
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

enum Fin {
    FIN_NONE = 0,
    FIN_STORE,  // write the rounded sums to out[]
    FIN_INIT,   // (b.b, r.r): normb, initial convergence test
    FIN_RZ0,    // (r.z): rz_old
    FIN_PAP,    // (p.Ap, p.p, Ap.Ap): breakdown test, alpha
    FIN_UPD,    // (r.r): rel, convergence / replacement trigger
    FIN_TRUE,   // (r.r) of the replaced residual: convergence
    FIN_RZ,     // (r.z): beta, rz_old
    FIN_UPDX,   // FIN_UPD where x += alpha p waits for the p update (the update fused into the
                // forward sweep): a stop here, or at this iteration's beta, leaves it pending (xp)
};

struct RedBuf {
    dd* partials;   // [slots * NV]
    double* out;    // FIN_STORE destination
};

// Programmatic dependent launch: wait until the preceding kernel in the
// stream has finished and its writes are visible (a no-op for a launch
// without the attribute).  Every kernel begins with this, before any global
// memory access.
__device__ __forceinline__ void grid_dep_begin() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Lets the next kernel start placing its CTAs once every CTA of this one has
// called it (or exited).  The per-iteration kernels call it after their main
// loop, before the final reduction, so the next launch overlaps only their
// tail; the next kernel still waits for this one to finish (grid_dep_begin).
__device__ __forceinline__ void grid_dep_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ bool st_done(const SolverState* st)
{
    return st != nullptr && *(volatile const int*)&st->status != kRunning;
}

// CG scalar logic of cg_crs.cpp:108-159, run by one thread.  With DEFER a
// stop is recorded in st->pend instead of st->status: the persistent apply
// (persist.cuh) gates every warp on st->status, which must not change while
// it runs, so its own reductions defer their decisions to the p update.
template <int FIN, bool DEFER = false>
__device__ void finish(const double* v, SolverState* st, double* out)
{
    if (FIN == FIN_STORE) {
        out[0] = v[0];
        return;
    }
    int& status = DEFER ? st->pend : st->status;
    if (FIN == FIN_INIT) {
        double normb = sqrt(v[0]);
        if (normb == 0.0) normb = 1.0;
        st->normb = normb;
        double rel = sqrt(v[1]) / normb;
        st->rel_resid = rel;
        st->iters = 0;
        if (rel < st->tol) status = kConverged;
        else if (st->max_iter <= 0) status = kMaxIter;
        return;
    }
    if (FIN == FIN_RZ0) {
        st->rz_old = v[0];
        return;
    }
    if (FIN == FIN_PAP) {
        const double pAp = v[0];
        const double eps = 2.220446049250313080847e-16;
        const double thr = eps * sqrt(v[1]) * sqrt(v[2]);
        if (pAp <= thr) {
            st->iters = st->k;
            status = kBreakdown;
            return;
        }
        if (!isfinite(pAp)) {
            st->iters = st->k;
            status = kNonFinite;
            return;
        }
        st->alpha = st->rz_old / pAp;
        return;
    }
    if (FIN == FIN_UPD || FIN == FIN_UPDX) {
        if (FIN == FIN_UPDX) st->xdefer_k = st->k;
        const double rel = sqrt(v[0]) / st->normb;
        st->iters = st->k + 1;
        st->rel_resid = rel;
        if (!isfinite(rel)) {
            status = kNonFinite;
            if (FIN == FIN_UPDX) st->xp = 1;
            return;
        }
        if (st->rr_interval <= 0) {
            if (rel < st->tol) status = kConverged;
        } else if (rel < st->tol) {
            if (st->true_check) st->rr_flag = 1;
            else status = kTrueCheck;
        } else if ((st->k + 1) % st->rr_interval == 0) {
            st->rr_flag = 1;
        }
        if (FIN == FIN_UPDX && status != kRunning) st->xp = 1;
        return;
    }
    if (FIN == FIN_TRUE) {
        const double rel = sqrt(v[0]) / st->normb;
        st->rel_resid = rel;
        st->rr_flag = 0;
        st->n_rr += 1;
        if (rel < st->tol) status = kConverged;
        return;
    }
    if (FIN == FIN_RZ) {
        const double rz = v[0];
        st->beta = rz / st->rz_old;
        st->rz_old = rz;
        if (!isfinite(st->beta)) {
            status = kNonFinite;
            st->iters = st->k + 1;
            if (st->xdefer_k == st->k) st->xp = 1;
        }
        return;
    }
}

// Block-reduce NV accumulators, publish the CTA's partial at slot `slot`,
// and let the CTA that completes the set of `nslots` partials finish.
template <int NV, int FIN>
__device__ __forceinline__ void reduce_finish(acc2 (&a)[NV], RedBuf red, SolverState* st,
                                              unsigned int* ticket, int slot, int nslots)
{
    __shared__ dd sm[NV * 32];
    __shared__ bool last;
    dd v[NV], tot[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = acc2_dd(a[q]);
    block_reduce_dd<NV>(v, sm, tot);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) red.partials[(size_t)slot * NV + q] = tot[q];
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        last = (t == (unsigned)nslots - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    dd s[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) s[q] = dd{0.0, 0.0};
    for (int b = threadIdx.x; b < nslots; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            dd p;
            p.hi = __ldcg(&red.partials[(size_t)b * NV + q].hi);
            p.lo = __ldcg(&red.partials[(size_t)b * NV + q].lo);
            s[q] = dd_add(s[q], p);
        }
    block_reduce_dd<NV>(s, sm, tot);
    if (threadIdx.x == 0) {
        double r[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) r[q] = dd_round(tot[q]);
        if (FIN == FIN_STORE) {
#pragma unroll
            for (int q = 0; q < NV; ++q) red.out[q] = r[q];
        } else {
            finish<FIN>(r, st, red.out);
        }
        *ticket = 0u;
    }
}

// ---------------------------------------------------------------------------
// SpMV (cg_crs.cpp:54-79): y_i = sum over row i of a_ik * x_c in CSR order,
// product and sum rounded separately.  FIN_PAP also forms p.Ap, p.p, Ap.Ap
// (cg_crs.cpp:127-129) with x = p.
// ---------------------------------------------------------------------------
template <class T, int FIN>
__global__ void __launch_bounds__(256) k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                              const T* __restrict__ v, const double* __restrict__ x,
                                              double* __restrict__ y, SolverState* st, RedBuf red,
                                              unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sum = 0.0;
        const int e = rp[i + 1];
        for (int k = rp[i]; k < e; ++k) sum = sum + (double)v[k] * x[ci[k]];
        y[i] = sum;
        if (FIN == FIN_PAP) {
            const double xi = x[i];
            acc2_fma(a[0], xi, sum);
            acc2_fma(a[1], xi, xi);
            acc2_fma(a[2], sum, sum);
        }
    }
    grid_dep_trigger();
    if (FIN == FIN_PAP) reduce_finish<3, FIN_PAP>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// r = b - A x with the FP64 matrix (cg_crs.cpp:102-106); FIN_INIT also
// forms b.b and r.r, FIN_TRUE forms r.r (residual replacement, only when the
// update step asked for it).
template <int FIN>
__global__ void __launch_bounds__(256) k_residual(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                  const double* __restrict__ v, const double* __restrict__ x,
                                                  const double* __restrict__ b, double* __restrict__ r,
                                                  SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    if (FIN == FIN_TRUE && *(volatile int*)&st->rr_flag == 0) return;
    acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sum = 0.0;
        const int e = rp[i + 1];
        for (int k = rp[i]; k < e; ++k) sum = sum + v[k] * x[ci[k]];
        const double bi = b[i];
        const double ri = bi - sum;
        r[i] = ri;
        if (FIN == FIN_INIT) {
            acc2_fma(a[0], bi, bi);
            acc2_fma(a[1], ri, ri);
        }
        if (FIN == FIN_TRUE) acc2_fma(a[0], ri, ri);
    }
    grid_dep_trigger();
    if (FIN == FIN_INIT) reduce_finish<2, FIN_INIT>(a, red, st, ticket, blockIdx.x, gridDim.x);
    if (FIN == FIN_TRUE) {
        acc2 t[1] = {a[0]};
        reduce_finish<1, FIN_TRUE>(t, red, st, ticket, blockIdx.x, gridDim.x);
    }
}

// x += alpha p; r -= alpha Ap (cg_crs.cpp:137-141), then r.r (cg_crs.cpp:143).
// alpha comes from the state (fused) or from the argument (st == nullptr).
// FIN_UPDX leaves x += alpha p to the p update (k_xpay with x), which reads
// p anyway: 8 bytes per row less, a stop in between marks it pending.
template <int FIN>
__global__ void __launch_bounds__(256) k_update(int n, double alpha_arg, const double* __restrict__ p,
                                                const double* __restrict__ Ap, double* __restrict__ x,
                                                double* __restrict__ r, SolverState* st, RedBuf red,
                                                unsigned int* ticket, int early)
{
    constexpr bool DOX = FIN != FIN_UPDX;
    // pairs of elements as 16-byte accesses, two pairs in flight per thread
    // (all vectors 16-byte aligned; otherwise one element at a time)
    const bool vec = (((uintptr_t)Ap | (uintptr_t)r | (DOX ? ((uintptr_t)p | (uintptr_t)x) : 0)) & 15) == 0;
    const int n2 = n >> 1;
    const int stride = gridDim.x * blockDim.x;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double2* __restrict__ p2 = reinterpret_cast<const double2*>(p);
    const double2* __restrict__ q2 = reinterpret_cast<const double2*>(Ap);
    double2* __restrict__ x2 = reinterpret_cast<double2*>(x);
    double2* __restrict__ r2 = reinterpret_cast<double2*>(r);
    // early: r, x and p of the thread's first two pairs were written before
    // the launch just before this one (the SpMV), so they load before the
    // wait on it, and the next launch is let in right after the wait
    const bool ew = early && vec;
    if (!ew) grid_dep_begin();
    double2 pre[2][3];
    if (ew) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int ik = i0 + k * stride;
            if (ik < n2) {
                pre[k][0] = __ldcg(r2 + ik);
                if (DOX) {
                    pre[k][1] = __ldcg(p2 + ik);
                    pre[k][2] = __ldcg(x2 + ik);
                }
            }
        }
        grid_dep_begin();
        grid_dep_trigger();
    }
    if (st_done(st)) return;
    const double alpha = st ? st->alpha : alpha_arg;
    acc2 a[1] = {{0.0, 0.0}};
    if (!vec) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            if (DOX) x[k] = fma(alpha, p[k], x[k]);
            const double rk = fma(-alpha, Ap[k], r[k]);
            r[k] = rk;
            if (FIN != FIN_NONE) acc2_fma(a[0], rk, rk);
        }
        grid_dep_trigger();
        if (FIN != FIN_NONE) reduce_finish<1, FIN>(a, red, st, ticket, blockIdx.x, gridDim.x);
        return;
    }
    // k < 0: load the pair; k = 0, 1: the pair loaded before the wait
    auto pair = [&](int i, int k) {
        const double2 qv = q2[i];
        double2 rv = k < 0 ? r2[i] : pre[k][0];
        if (DOX) {
            const double2 pv = k < 0 ? p2[i] : pre[k][1];
            double2 xv = k < 0 ? x2[i] : pre[k][2];
            xv.x = fma(alpha, pv.x, xv.x);
            xv.y = fma(alpha, pv.y, xv.y);
            x2[i] = xv;
        }
        rv.x = fma(-alpha, qv.x, rv.x);
        rv.y = fma(-alpha, qv.y, rv.y);
        r2[i] = rv;
        if (FIN != FIN_NONE) {
            acc2_fma(a[0], rv.x, rv.x);
            acc2_fma(a[0], rv.y, rv.y);
        }
    };
    int i = i0;
    if (ew) {
        if (i + stride < n2) {
            pair(i, 0);
            pair(i + stride, 1);
            i += 2 * stride;
        } else if (i < n2) {
            pair(i, 0);
            i = n2;
        }
    }
    for (; i + stride < n2; i += 2 * stride) {
        pair(i, -1);
        pair(i + stride, -1);
    }
    if (i < n2) pair(i, -1);
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const int k = n - 1;
        if (DOX) x[k] = fma(alpha, p[k], x[k]);
        const double rk = fma(-alpha, Ap[k], r[k]);
        r[k] = rk;
        if (FIN != FIN_NONE) acc2_fma(a[0], rk, rk);
    }
    if (!ew) grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// p = z + beta p (cg_crs.cpp:155-157); the fused form then advances k and
// stops the solve after max_iter iterations (cg_crs.cpp:125).  With x
// (the update fused into the forward sweep) x += alpha p comes first, with
// the p of this iteration (cg_crs.cpp:137-138).
__global__ void __launch_bounds__(256) k_xpay(int n, double beta_arg, const double* __restrict__ z,
                                              double* __restrict__ p, SolverState* st, double* __restrict__ x,
                                              int early)
{
    const bool vec = (((uintptr_t)z | (uintptr_t)p | (uintptr_t)x) & 15) == 0;
    const int n2 = n >> 1;
    const int stride = gridDim.x * blockDim.x;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double2* __restrict__ z2 = reinterpret_cast<const double2*>(z);
    double2* __restrict__ p2 = reinterpret_cast<double2*>(p);
    double2* __restrict__ x2 = reinterpret_cast<double2*>(x);
    // early: p and x of the thread's first two pairs were written before
    // the launch just before this one (the preconditioner apply, which
    // writes z), so they load before the wait on it, and the next launch is
    // let in right after the wait
    const bool ew = early && vec;
    if (!ew) grid_dep_begin();
    double2 pre[2][2];
    if (ew) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int ik = i0 + k * stride;
            if (ik < n2) {
                pre[k][0] = __ldcg(p2 + ik);
                if (x) pre[k][1] = __ldcg(x2 + ik);
            }
        }
        grid_dep_begin();
        grid_dep_trigger();
    }
    if (st) {
        // a stop the persistent apply deferred: make it the solve's status
        const int pd = *(volatile const int*)&st->pend;
        if (pd != kRunning) {
            if (blockIdx.x == 0 && threadIdx.x == 0 && st->status == kRunning) st->status = pd;
            return;
        }
    }
    if (st_done(st)) return;
    const double beta = st ? st->beta : beta_arg;
    const double alpha = (st && x) ? st->alpha : 0.0;
    if (!vec) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            if (x) x[k] = fma(alpha, p[k], x[k]);
            p[k] = fma(beta, p[k], z[k]);
        }
    } else {
        // k < 0: load the pair; k = 0, 1: the pair loaded before the wait
        auto pair = [&](int i, int k) {
            const double2 zv = z2[i];
            double2 pv = k < 0 ? p2[i] : pre[k][0];
            if (x) {
                double2 xv = k < 0 ? x2[i] : pre[k][1];
                xv.x = fma(alpha, pv.x, xv.x);
                xv.y = fma(alpha, pv.y, xv.y);
                x2[i] = xv;
            }
            pv.x = fma(beta, pv.x, zv.x);
            pv.y = fma(beta, pv.y, zv.y);
            p2[i] = pv;
        };
        int i = i0;
        if (ew) {
            if (i + stride < n2) {
                pair(i, 0);
                pair(i + stride, 1);
                i += 2 * stride;
            } else if (i < n2) {
                pair(i, 0);
                i = n2;
            }
        }
        for (; i + stride < n2; i += 2 * stride) {
            pair(i, -1);
            pair(i + stride, -1);
        }
        if (i < n2) pair(i, -1);
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
            if (x) x[n - 1] = fma(alpha, p[n - 1], x[n - 1]);
            p[n - 1] = fma(beta, p[n - 1], z[n - 1]);
        }
    }
    if (!ew) grid_dep_trigger();
    if (st && blockIdx.x == 0 && threadIdx.x == 0) {
        const int k1 = st->k + 1;
        st->k = k1;
        if (k1 >= st->max_iter) st->status = kMaxIter;
    }
}

// x += alpha p of a solve that stopped between the fused update and the p
// update (xp set by FIN_UPDX / FIN_RZ); k_clear_xp clears the mark after it
__global__ void __launch_bounds__(256) k_apply_xp(int n, const double* __restrict__ p, double* __restrict__ x,
                                                  const SolverState* st)
{
    grid_dep_begin();
    if (!st->xp) return;
    const double alpha = st->alpha;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        x[k] = fma(alpha, p[k], x[k]);
}

__global__ void k_clear_xp(SolverState* st)
{
    grid_dep_begin();
    st->xp = 0;
}

// resumes a solve stopped at kTrueCheck with the replacement requested
__global__ void k_resume_true_check(SolverState* st)
{
    grid_dep_begin();
    if (st->status == kTrueCheck) {
        st->status = kRunning;
        st->pend = kRunning;
        st->rr_flag = 1;
    }
}

__global__ void __launch_bounds__(256) k_copy(int n, const double* __restrict__ a, double* __restrict__ b,
                                              SolverState* st)
{
    grid_dep_begin();
    if (st_done(st)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

__global__ void __launch_bounds__(256) k_sub(int n, const double* __restrict__ b, const double* __restrict__ ax,
                                             double* __restrict__ r)
{
    grid_dep_begin();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] = b[i] - ax[i];
}

// generic dot a.b (FIN_STORE) -- dot()/nrm2() of cg_crs.cpp:33-50
__global__ void __launch_bounds__(256) k_dot(int n, const double* __restrict__ a, const double* __restrict__ b,
                                             RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    acc2 s[1] = {{0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc2_fma(s[0], a[i], b[i]);
    grid_dep_trigger();
    reduce_finish<1, FIN_STORE>(s, red, nullptr, ticket, blockIdx.x, gridDim.x);
}

// Identity (precond.hpp:12-14, inv == nullptr) or Jacobi (precond.hpp:38-42)
// z = inv .* r, with r.z for FIN_RZ0 / FIN_RZ.
template <int FIN>
__global__ void __launch_bounds__(256) k_diag_apply(int n, const double* __restrict__ inv,
                                                    const double* __restrict__ r, double* __restrict__ z,
                                                    SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    acc2 a[1] = {{0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = r[i];
        const double zi = inv ? inv[i] * ri : ri;
        z[i] = zi;
        if (FIN != FIN_NONE) acc2_fma(a[0], ri, zi);
    }
    grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Substitution sweep over one level of a schedule plan.
//
// A plan lists, per level, independent units; a unit is a sequence of rows
// computed in order by one thread (MC: one row; ABMC: the rows of a block in
// ascending (forward) or descending (backward) order; natural order: level
// sets of single rows).  Row i computes
//     out_i = (in_i - sum_k S_ik out_{c_k}) / d_i
// with the sum as a chain of fused multiply-adds in column order, exactly as
// forward_solve_mc / forward_solve_abmc (ic0.cpp:201-214, 280-295) for S =
// strict lower part of L and backward_solve_mc / _abmc (ic0.cpp:229-244,
// 319-334) for S = strict upper part of L^T.  FIN_RZ0 / FIN_RZ accumulate
// r.z over all levels of the sweep (one slot per CTA of every level launch).
// ---------------------------------------------------------------------------
struct SweepArgs {
    const int* unit_ptr;   // nullptr: one row per unit
    const int* rows;
    const int* Sp;
    const int* Si;
    const void* Sx;
    const void* d;
    const double* in;
    double* out;
    const double* rdot;    // r for the fused r.z
};

template <class T, int FIN>
__global__ void __launch_bounds__(256) k_sweep(SweepArgs a, int u0, int u1, int slot0, int nslots,
                                               SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    const T* __restrict__ Sx = (const T*)a.Sx;
    const T* __restrict__ d = (const T*)a.d;
    const int* __restrict__ Sp = a.Sp;
    const int* __restrict__ Si = a.Si;
    acc2 acc[1] = {{0.0, 0.0}};
    for (int u = u0 + blockIdx.x * blockDim.x + threadIdx.x; u < u1; u += gridDim.x * blockDim.x) {
        const int t0 = a.unit_ptr ? a.unit_ptr[u] : u;
        const int t1 = a.unit_ptr ? a.unit_ptr[u + 1] : u + 1;
        for (int t = t0; t < t1; ++t) {
            const int i = a.rows[t];
            double s = a.in[i];
            const int e = Sp[i + 1];
            for (int k = Sp[i]; k < e; ++k) s = fma(-(double)Sx[k], a.out[Si[k]], s);
            const double v = s / (double)d[i];
            a.out[i] = v;
            if (FIN != FIN_NONE) acc2_fma(acc[0], a.rdot[i], v);
        }
    }
    grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(acc, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// ---------------------------------------------------------------------------
// Lane-interleaved kernels (the default path).
//
// The device keeps the system in an internal row order Q built from the
// schedule: within each level (color), the units (ABMC blocks; single rows
// for MC and level sets) are taken 32 at a time, longest first, and their
// rows are numbered (step r, unit u) -- the r-th row of every unit of the
// group, then the (r+1)-th, ...  A warp owns a group and lane u owns unit u,
// so one warp step advances 32 independent chains by one row each, and rows
// of one step are consecutive.
//
// Matrices are stored as SELL-32 over Q: a slice holds up to 32 consecutive
// Q rows, entry j of the slice's lane l at ptr[slice] + 32 j + l, so every
// load of a warp step is one coalesced 128-byte line per array.  Each row
// keeps the reference's entry order (column indices are relabelled to Q, not
// re-sorted), so every row's chain of operations is the reference's and the
// results keep its bits.  Vectors live in Q order; they are permuted only at
// the API boundary.
// ---------------------------------------------------------------------------
// The CG update fused into the forward sweep (FIN_UPDX): r -= alpha Ap
// (cg_crs.cpp:139-141) for each row as the sweep stages it -- r and Ap come
// into the tile with the batch's other arrays -- and the new r is written
// back, is the row's input, and r.r is reduced by the sweep's launches (the
// residual test of cg_crs.cpp:143).  x += alpha p (cg_crs.cpp:137-138) waits
// for the p update, which reads p anyway (k_xpay with x); a stop in between
// leaves it pending in the state (xp) for k_apply_xp.  The arithmetic of
// each element is k_update's.
struct UpdArgs {
    double* r;
    const double* Ap;
};

struct SellMat {
    const int* ptr;       // first slot of each slice
    const int* col;       // column (Q index) per slot
    const void* val;      // value per slot (float or double)
    const int* len;       // entries of each Q row
    const int2* pk;       // FP32 values with their columns, one 8-byte word per slot (or null)
};

// pk[s] = (value bits, column) of slot s: one load per entry in the SpMV
__global__ void __launch_bounds__(256) k_pack_sell(long long m, const float* __restrict__ v,
                                                   const int* __restrict__ col, int2* __restrict__ pk)
{
    grid_dep_begin();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        pk[i] = make_int2(__float_as_int(v[i]), col[i]);
}

// y = A x over regular 32-row slices (slice s = Q rows [32 s, 32 s + 32)),
// product and sum rounded separately as in spmv (cg_crs.cpp:73-75).  PK:
// FP32 values read with their columns as one 8-byte word (A.pk).
template <class T, int FIN, bool PK = false>
__global__ void __launch_bounds__(256, PK ? 4 : 0) k_spmv_q(int n, SellMat A, const double* __restrict__ x,
                                                double* __restrict__ y, SolverState* st, RedBuf red,
                                                unsigned int* ticket, int early)
{
    const T* __restrict__ val = (const T*)A.val;
    const int* __restrict__ col = A.col;
    acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    const int lane = threadIdx.x & 31;
    const int nslices = (n + 31) >> 5;
    const int stride = (gridDim.x * blockDim.x) >> 5;
    // Software pipeline over the warp's slices: the row length, columns and
    // values of the next slice (up to K entries per row) are loaded while
    // the current slice's x gathers and sums run.  Rows longer than K take
    // the rest of their entries in a tail loop.
    constexpr int K = 8;
    int L = 0, c[K];
    T v[K];
    // FP32 values packed with their columns: one 8-byte load per entry
    static_assert(!PK || sizeof(T) == 4, "packed words hold FP32 values");
    const int2* __restrict__ pk = A.pk;
    auto load = [&](int s) {
        const int i = (s << 5) + lane;
        L = i < n ? A.len[i] : 0;
        const int p0 = A.ptr[s] + lane;
        if (PK) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const int2 e = j < L ? __ldcs(pk + p0 + 32 * j) : make_int2(0, 0);
                c[j] = e.y;
                v[j] = (T)__int_as_float(e.x);
            }
        } else {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                c[j] = j < L ? __ldcs(col + p0 + 32 * j) : 0;
                v[j] = j < L ? __ldcs(val + p0 + 32 * j) : (T)0;
            }
        }
    };
    // early: the first slice's matrix words do not depend on the launch
    // just before, so they load before the wait on it, and the next launch
    // is let in right after the wait
    if (!early) grid_dep_begin();
    int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s < nslices) load(s);
    if (early) {
        grid_dep_begin();
        grid_dep_trigger();
    }
    if (st_done(st)) return;
    for (; s < nslices; s += stride) {
        const int Lc = L;
        int cc[K];
        T vc[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            cc[j] = c[j];
            vc[j] = v[j];
        }
        const int sn = s + stride;
        if (sn < nslices) load(sn);
        double xv[K];
#pragma unroll
        for (int j = 0; j < K; ++j) xv[j] = j < Lc ? __ldg(x + cc[j]) : 0.0;
        const int i = (s << 5) + lane;
        double sum = 0.0;
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (j < Lc) sum = sum + (double)vc[j] * xv[j];
        if (Lc > K) {
            const int p0 = A.ptr[s] + lane;
            for (int j = K; j < Lc; ++j) {
                const int pa = p0 + 32 * j;
                sum = sum + (double)__ldcs(val + pa) * __ldg(x + __ldcs(col + pa));
            }
        }
        if (i < n) {
            y[i] = sum;
            if (FIN == FIN_PAP) {
                const double xi = __ldg(x + i);
                acc2_fma(a[0], xi, sum);
                acc2_fma(a[1], xi, xi);
                acc2_fma(a[2], sum, sum);
            }
        }
    }
    if (!early) grid_dep_trigger();
    if (FIN == FIN_PAP) reduce_finish<3, FIN_PAP>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// The FP32 SpMV with TPR threads per row (2 or 4) for matrices with long
// rows: TPR warps share a slice, warp w of the slice takes the row entries
// j = w, w + TPR, ... (coalesced: one 8-byte packed word per lane per j) and
// sums them in that order; the TPR partial sums of a row are then added in
// warp order.  The result is deterministic but not the single sum in CSR
// order of k_spmv_q, so only the mixed form (FP32 storage) offers it.
template <int TPR, int FIN>
__global__ void __launch_bounds__(256) k_spmv_qt(int n, SellMat A, const double* __restrict__ x,
                                                 double* __restrict__ y, SolverState* st, RedBuf red,
                                                 unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    constexpr int SPC = 8 / TPR;  // slices per CTA iteration
    constexpr int K = 8;          // entries per warp in flight
    __shared__ double part[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = warp / TPR, w = warp % TPR;
    const int nslices = (n + 31) >> 5;
    const int2* __restrict__ pk = A.pk;
    acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    // every warp of the CTA runs the same number of iterations
    for (int s0 = blockIdx.x * SPC; s0 < nslices; s0 += gridDim.x * SPC) {
        const int s = s0 + sl;
        const int i = (s << 5) + lane;
        double sum = 0.0;
        if (s < nslices && i < n) {
            const int L = A.len[i];
            const int p0 = A.ptr[s] + lane;
            for (int j0 = w; j0 < L; j0 += K * TPR) {
                int c[K];
                float v[K];
#pragma unroll
                for (int u = 0; u < K; ++u) {
                    const int j = j0 + u * TPR;
                    const int2 e = j < L ? __ldcs(pk + p0 + 32 * j) : make_int2(0, 0);
                    c[u] = e.y;
                    v[u] = __int_as_float(e.x);
                }
                double xv[K];
#pragma unroll
                for (int u = 0; u < K; ++u) xv[u] = j0 + u * TPR < L ? __ldg(x + c[u]) : 0.0;
#pragma unroll
                for (int u = 0; u < K; ++u)
                    if (j0 + u * TPR < L) sum = sum + (double)v[u] * xv[u];
            }
        }
        part[warp][lane] = sum;
        __syncthreads();
        if (w == 0 && s < nslices && i < n) {
            double t = part[warp][lane];
#pragma unroll
            for (int q = 1; q < TPR; ++q) t = t + part[warp + q][lane];
            y[i] = t;
            if (FIN == FIN_PAP) {
                const double xi = __ldg(x + i);
                acc2_fma(a[0], xi, t);
                acc2_fma(a[1], xi, xi);
                acc2_fma(a[2], t, t);
            }
        }
        __syncthreads();
    }
    grid_dep_trigger();
    if (FIN == FIN_PAP) reduce_finish<3, FIN_PAP>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// r = b - A x with the FP64 matrix in Q order (FIN_INIT: b.b and r.r;
// FIN_TRUE: residual replacement when requested, r.r).
template <int FIN>
__global__ void __launch_bounds__(256) k_residual_q(int n, SellMat A, const double* __restrict__ x,
                                                    const double* __restrict__ b, double* __restrict__ r,
                                                    SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    if (FIN == FIN_TRUE && *(volatile int*)&st->rr_flag == 0) return;
    const double* __restrict__ val = (const double*)A.val;
    acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
    const int lane = threadIdx.x & 31;
    const int nslices = (n + 31) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices; s += (gridDim.x * blockDim.x) >> 5) {
        const int i = (s << 5) + lane;
        if (i < n) {
            const int L = A.len[i];
            const int p0 = A.ptr[s] + lane;
            double sum = 0.0;
            for (int j = 0; j < L; ++j) {
                const int pa = p0 + 32 * j;
                sum = sum + __ldcs(val + pa) * __ldg(x + __ldcs(A.col + pa));
            }
            const double bi = b[i];
            const double ri = bi - sum;
            r[i] = ri;
            if (FIN == FIN_INIT) {
                acc2_fma(a[0], bi, bi);
                acc2_fma(a[1], ri, ri);
            }
            if (FIN == FIN_TRUE) acc2_fma(a[0], ri, ri);
        }
    }
    grid_dep_trigger();
    if (FIN == FIN_INIT) reduce_finish<2, FIN_INIT>(a, red, st, ticket, blockIdx.x, gridDim.x);
    if (FIN == FIN_TRUE) {
        acc2 t[1] = {a[0]};
        reduce_finish<1, FIN_TRUE>(t, red, st, ticket, blockIdx.x, gridDim.x);
    }
}

// One level of a substitution sweep in Q order.  Group g (a warp) holds up
// to 32 units; lane u's unit has glen[32 g + u] rows (lanes sorted by
// length, longest first, so the active lanes of step r are a prefix and the
// rows of step r are Q rows gbase[g] + off_r + [0, cnt_r)).  Slice
// sl0[g] + r of M holds the entries of step r's rows.  Forward steps run
// r = 0, 1, ...; backward steps run the units' rows in reverse.  Row q:
//     out_q = (in_q - sum_k M_qk out_{c_k}) / d_q
// with the sum a chain of fused multiply-adds in the reference's entry order
// (ic0.cpp:201-214, 229-244, 280-295, 319-334).  Earlier-level values come
// from global memory; in-unit values were written by the same lane at an
// earlier step (the value of the row just before is kept in a register).
template <class T, bool FWD, int FIN>
__global__ void __launch_bounds__(256) k_sweep_q(int g0, int g1, const int* __restrict__ gbase,
                                                 const int* __restrict__ glen, const int* __restrict__ sl0,
                                                 SellMat M, const T* __restrict__ dg,
                                                 const double* __restrict__ in, double* out,
                                                 const double* __restrict__ rdot, int slot0, int nslots,
                                                 SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    const T* __restrict__ val = (const T*)M.val;
    const int* __restrict__ col = M.col;
    const int lane = threadIdx.x & 31;
    acc2 rz[1] = {{0.0, 0.0}};
    for (int g = g0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); g < g1;
         g += (gridDim.x * blockDim.x) >> 5) {
        const int len = glen[(size_t)g * 32 + lane];
        const int base = gbase[g];
        const int s0 = sl0[g];
        const int maxlen = __reduce_max_sync(0xffffffffu, (unsigned)len);
        int prev_q = -1;
        double prev_v = 0.0;
        for (int t = 0; t < maxlen; ++t) {
            const int r = FWD ? t : (maxlen - 1 - t);
            const int off = (int)__reduce_add_sync(0xffffffffu, (unsigned)min(len, r));
            if (r < len) {
                const int q = base + off + lane;
                const int p0 = M.ptr[s0 + r] + lane;
                const int L = M.len[q] & 0xffff;
                double acc = in[q];
                for (int j = 0; j < L; ++j) {
                    const int pa = p0 + 32 * j;
                    const int c = col[pa];
                    const double xv = (c == prev_q) ? prev_v : out[c];
                    acc = fma(-(double)val[pa], xv, acc);
                }
                const double v = acc / (double)dg[q];
                out[q] = v;
                prev_q = q;
                prev_v = v;
                if (FIN != FIN_NONE) acc2_fma(rz[0], rdot[q], v);
            }
        }
    }
    grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(rz, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// The earlier-level part of a substitution row: a - sum_j v_j prev[c_j] over
// entries j in [j0, j1), one fused multiply-add per entry in the order of j
// (the reference's).  KT gathers are issued before their multiply-adds, so a
// long row waits for one gather latency per KT entries, not per entry.
// Entry j sits at slot pb + 32 j of a SELL matrix in global memory ...
template <int KT, class T>
__device__ __forceinline__ double fold_ext_global(double a, int pb, int j0, int j1, const int* __restrict__ col,
                                                  const T* __restrict__ val, const double* __restrict__ prev)
{
    for (int jc = j0; jc < j1; jc += KT) {
        int c[KT];
        T v[KT];
        double x[KT];
#pragma unroll
        for (int u = 0; u < KT; ++u) {
            const int pa = pb + 32 * (jc + u < j1 ? jc + u : jc);
            c[u] = col[pa];
            v[u] = val[pa];
        }
#pragma unroll
        for (int u = 0; u < KT; ++u) x[u] = jc + u < j1 ? __ldg(prev + c[u]) : 0.0;
#pragma unroll
        for (int u = 0; u < KT; ++u)
            if (jc + u < j1) a = fma(-(double)v[u], x[u], a);
    }
    return a;
}

// An earlier-level value.  COH: written by other CTAs of the running launch
// (the persistent apply), so read through L2 (ld.global.cg); otherwise read
// only, through the read-only path.
template <bool COH>
__device__ __forceinline__ double ld_prev(const double* p)
{
    return COH ? __ldcg(p) : __ldg(p);
}

// ... or at e + 32 j of the staged slot arrays in shared memory
template <int KT, class T, bool COH = false>
__device__ __forceinline__ double fold_ext_staged(double a, int e, int j0, int j1, const int* s_col, const T* s_val,
                                                  const double* prev)
{
    for (int jc = j0; jc < j1; jc += KT) {
        double x[KT];
#pragma unroll
        for (int u = 0; u < KT; ++u) x[u] = jc + u < j1 ? ld_prev<COH>(prev + s_col[e + 32 * (jc + u)]) : 0.0;
#pragma unroll
        for (int u = 0; u < KT; ++u)
            if (jc + u < j1) a = fma(-(double)s_val[e + 32 * (jc + u)], x[u], a);
    }
    return a;
}

// the gathered values of entries [j0, j1), parked beside the staged entries
// (the exact backward order applies them after the in-unit entries)
template <int KT, bool COH = false>
__device__ __forceinline__ void park_ext_staged(int e, int j0, int j1, const int* s_col, double* s_pv,
                                                const double* prev)
{
    for (int jc = j0; jc < j1; jc += KT) {
        double x[KT];
#pragma unroll
        for (int u = 0; u < KT; ++u) x[u] = jc + u < j1 ? ld_prev<COH>(prev + s_col[e + 32 * (jc + u)]) : 0.0;
#pragma unroll
        for (int u = 0; u < KT; ++u)
            if (jc + u < j1) s_pv[e + 32 * (jc + u)] = x[u];
    }
}

// Step slices of the two-phase sweeps: first Q row, SELL slot pointers of
// the forward (S) and backward (T) matrices, and a packed word
// rows | step << 6 | widthS << 12 | widthT << 20 (widths clamped to 255).
struct SliceMeta {
    int q0, pS, pT, w;
};

// Two-phase substitution over one level (groups [g0, g1)), used when every
// unit has at most 64 rows.  Row lengths are stored as L | nint << 16 and the
// nint in-unit entries of a row carry col = -(step + 1) (the unit's own row
// at that step); they are the last entries of a forward row and the first of
// a backward row, as in the reference's column order.
//
// A CTA (8 warps) takes gpc groups at a time; their step slices are
// consecutive, slices [sl0[gb], sl0[gb + gpc]), and map one-to-one onto a
// shared tile of tile * 32 rows.
//  Phase A, all warps, one warp per slice: one metadata load, then the
//    slice's entries (loaded speculatively up to KS per row, coalesced),
//    pivots and inputs; each row's chain over its entries from earlier
//    levels (final values, not written by this launch) is computed; the
//    partial value, pivot, row index, first NI in-unit entries and (with a
//    reduction) r_q go to the tile.
//  Phase B, one warp per group: the steps of its 32 units, reading the tile
//    only: in-unit entries use the unit's earlier results, the row divides
//    by its pivot, the result is stored and r.z accumulated.  Rows with more
//    than NI in-unit entries, and the exact backward order, read the rest of
//    the row from global memory.
// Forward rows: earlier-level entries come first in the reference's order,
// so the split keeps its bits.  Backward rows put the in-unit entries first;
// EXACT keeps that order (phase B applies the earlier-level entries after the
// in-unit ones); otherwise the earlier-level entries are applied first, in
// phase A (the FP32-storage path, which has no reference rounding to keep).
template <class T, bool FWD, int FIN, bool EXACT, int NI, int KS>
__global__ void __launch_bounds__(256) k_sweep_q2(int g0, int g1, int gpc, int tile, int slow,
                                                  const int* __restrict__ sl0, const int* __restrict__ glen,
                                                  const SliceMeta* __restrict__ meta, SellMat M,
                                                  const T* __restrict__ dg, const double* __restrict__ in,
                                                  double* out, const double* __restrict__ rdot, int slot0,
                                                  int nslots, SolverState* st, RedBuf red, unsigned int* ticket)
{
    grid_dep_begin();
    if (st_done(st)) return;
    constexpr bool ext_first = FWD || !EXACT;
    constexpr bool with_r = FIN != FIN_NONE;
    // tile layout: partial sums / results and r (double), pivots and in-unit
    // values (T), row index, slow-path slot and length word (int), in-unit
    // steps (int8, -1 if none)
    extern __shared__ double smem_d[];
    const int R = tile * 32;
    double* s_acc = smem_d;
    double* s_rd = smem_d + R;                                       // [R] if with_r
    T* s_piv = reinterpret_cast<T*>(smem_d + (with_r ? 2 : 1) * R);
    T* s_iv = s_piv + R;                                             // [NI][R]
    int* s_q = reinterpret_cast<int*>(s_iv + NI * R);                // [R]
    int* s_p0 = s_q + R;                                             // [R] if slow
    int* s_lw = s_p0 + R;                                            // [R] if slow
    signed char* s_ii = reinterpret_cast<signed char*>(slow ? s_lw + R : s_p0);  // [NI][R]
    const T* __restrict__ val = (const T*)M.val;
    const int* __restrict__ col = M.col;
    const int* __restrict__ mlen = M.len;
    const double* __restrict__ prev = out;  // earlier-level values: read-only in this launch
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    acc2 rz[1] = {{0.0, 0.0}};
    for (int gb = g0 + blockIdx.x * gpc; gb < g1; gb += gridDim.x * gpc) {
        const int ng = min(gpc, g1 - gb);
        const int sb = sl0[gb], se = sl0[gb + ng];
        // phase A
        for (int t = warp; t < se - sb; t += 8) {
            const SliceMeta m = meta[sb + t];
            const int cnt = m.w & 63;
            const int w = FWD ? (m.w >> 12) & 255 : (m.w >> 20) & 255;
            const int pb = (FWD ? m.pS : m.pT) + lane;
            if (lane < cnt) {
                const int q = m.q0 + lane;
                const int rr = t * 32 + lane;
                const int lw = mlen[q];
                double a = in[q];
                const T piv = dg[q];
                double rq = 0.0;
                if (with_r) rq = rdot[q];
                int cj[KS];
                T vj[KS];
#pragma unroll
                for (int j = 0; j < KS; ++j) {
                    cj[j] = 0;
                    vj[j] = (T)0;
                    if (j < w) {
                        cj[j] = col[pb + 32 * j];
                        vj[j] = val[pb + 32 * j];
                    }
                }
                const int L = lw & 0xffff, ni = lw >> 16;
                if (ext_first) {
                    const int j0 = FWD ? 0 : ni, j1 = FWD ? L - ni : L;
                    double xg[KS];
#pragma unroll
                    for (int j = 0; j < KS; ++j) xg[j] = (j >= j0 && j < j1) ? __ldg(prev + cj[j]) : 0.0;
#pragma unroll
                    for (int j = 0; j < KS; ++j)
                        if (j >= j0 && j < j1) a = fma(-(double)vj[j], xg[j], a);
                    a = fold_ext_global<8>(a, pb, max(KS, j0), j1, col, val, prev);
                }
                s_acc[rr] = a;
                if (with_r) s_rd[rr] = rq;
                s_piv[rr] = piv;
                s_q[rr] = q;
                const int jin = FWD ? L - ni : 0;
#pragma unroll
                for (int k = 0; k < NI; ++k) {
                    int idx = -1;
                    if (k < ni) {
                        const int pa = pb + 32 * (jin + k);
                        s_iv[k * R + rr] = val[pa];
                        idx = -col[pa] - 1;
                    }
                    s_ii[k * R + rr] = (signed char)idx;
                }
                if (slow) {
                    s_p0[rr] = (ni > NI || !ext_first) ? pb : -1;
                    s_lw[rr] = lw;
                }
            }
        }
        __syncthreads();
        // phase B
        if (warp < ng) {
            const int g = gb + warp;
            const int len = glen[(size_t)g * 32 + lane];
            const int maxlen = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            const int base = (sl0[g] - sb) * 32 + lane;
            for (int t = 0; t < maxlen; ++t) {
                const int r = FWD ? t : maxlen - 1 - t;
                if (r < len) {
                    const int rr = base + r * 32;
                    double a = s_acc[rr];
#pragma unroll
                    for (int k = 0; k < NI; ++k) {
                        const int idx = s_ii[k * R + rr];
                        if (idx >= 0) a = fma(-(double)s_iv[k * R + rr], s_acc[base + idx * 32], a);
                    }
                    const int p0 = slow ? s_p0[rr] : -1;
                    if (p0 >= 0) {
                        const int lw = s_lw[rr];
                        const int L = lw & 0xffff, ni = lw >> 16;
                        const int jin = FWD ? L - ni : 0;
                        for (int k = NI; k < ni; ++k) {
                            const int pa = p0 + 32 * (jin + k);
                            a = fma(-(double)val[pa], s_acc[base + (-col[pa] - 1) * 32], a);
                        }
                        if (!ext_first) a = fold_ext_global<8>(a, p0, ni, L, col, val, prev);
                    }
                    const double v = a / (double)s_piv[rr];
                    s_acc[rr] = v;
                    out[s_q[rr]] = v;
                    if (with_r) acc2_fma(rz[0], s_rd[rr], v);
                }
            }
        }
        __syncthreads();
    }
    grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(rz, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// ---------------------------------------------------------------------------
// Staged substitution over one level (the default when a batch fits shared
// memory).
//
// A batch is up to 16 consecutive groups of one level.  Its Q rows [qb, qe),
// its step slices [sb, se) and the SELL slots of those slices are contiguous,
// so everything the batch reads except the earlier-level values is a handful
// of contiguous ranges: slice metadata, inputs, r (with a reduction), pivots,
// row words, column indices and values.  A CTA takes batches b0 + blockIdx.x,
// + gridDim.x, ... and copies them into shared memory with cp.async (16-byte
// chunks, nothing held in registers).  With NB = 1 (the default) it has one
// buffer, refilled after each batch, so twice as many CTAs fit an SM and
// overlap each other's copies; with NB = 2 it copies batch i + 1 into the
// other half of a double buffer while it works on batch i.  Per batch:
//  G, all warps, one slice per warp and UG slices at a time: the
//    earlier-level values of each row's entries are gathered (the only
//    scattered reads) and folded into the row's partial sum in the tile, or,
//    for the exact backward order, parked beside the entries; the row's
//    in-unit entries (count, first two steps and values) are packed for C;
//  C, one warp per group and one lane per unit: the in-unit chains, from
//    the tile only; each result goes to out and stays in the tile for the
//    unit's later steps; r.z is accumulated.
// The order of the floating-point operations of every row is the one of
// k_sweep_q2 (and of the reference for EXACT).  Without EXACT (FP32
// storage) dg holds reciprocal pivots and the division is a product.
// ---------------------------------------------------------------------------
struct BatchDesc {
    int sb, se;    // step slices [sb, se)
    int qb, qe;    // Q rows [qb, qe)
    int ps0, ps1;  // SELL slots of the slices in S (forward matrix)
    int pt0, pt1;  // SELL slots of the slices in T (backward matrix)
    int gb, ng;    // groups [gb, gb + ng), ng <= 16
    int flags;     // bit 0 / 1: forward / backward chains are regular; bit 2: full slices (below)
    int pad1;
};

// Byte offsets of one stage buffer.  Row arrays get room for the 16-byte
// alignment of their first and last chunk; slot ranges start on a slice
// boundary (a multiple of 32 slots), so only their end is rounded.
struct StageLayout {
    int meta, in, rd, piv, len, col, val, pv, iw, iv, bytes;
};

__host__ __device__ inline int stage_al16(int x) { return (x + 15) & ~15; }

__host__ __device__ inline StageLayout stage_layout(int rows, int slots, int slices, int tsize, bool with_r,
                                                    bool with_pv)
{
    StageLayout L;
    int o = 0;
    L.meta = o;
    o += stage_al16(slices * 16);
    L.in = o;
    o += stage_al16((rows + 4) * 8);
    L.rd = o;
    if (with_r) o += stage_al16((rows + 4) * 8);
    L.piv = o;
    o += stage_al16((rows + 8) * tsize);
    L.len = o;
    o += stage_al16((rows + 8) * 4);
    L.col = o;
    o += stage_al16((slots + 4) * 4);
    L.val = o;
    o += stage_al16((slots + 4) * tsize);
    L.pv = o;
    if (with_pv) o += stage_al16(slots * 8);
    L.iw = o;  // per row: in-unit count and the steps of the first two in-unit entries
    o += stage_al16(rows * 4);
    L.iv = o;  // per row: the values of those two entries
    o += stage_al16(2 * rows * tsize);
    L.bytes = o;
    return L;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copies elements [first, first + count) of src (esize bytes each) into dst
// in 16-byte chunks, starting at the chunk that holds `first`; returns the
// element offset of `first` in dst.
// Threads tid = 0 .. nthr - 1 of the CTA share the copy (by default all).
__device__ __forceinline__ int stage_range(unsigned char* dst, const void* src, int esize, int first, int count,
                                           int tid = -1, int nthr = 0)
{
    if (tid < 0) {
        tid = threadIdx.x;
        nthr = blockDim.x;
    }
    const int per = 16 / esize;
    const int a0 = first & ~(per - 1);
    const int a1 = (first + count + per - 1) & ~(per - 1);
    const int chunks = (a1 - a0) / per;
    const unsigned char* s = (const unsigned char*)src + (size_t)a0 * esize;
    for (int k = tid; k < chunks; k += nthr) cp_async16(dst + 16 * k, s + 16 * k);
    return first - a0;
}

// Parts of a staged batch: the level's own arrays (slice words, pivots, row
// words, columns, values: the same in every sweep), the input rows and r.
enum StagePart { SP_MAT = 1, SP_IN = 2, SP_RD = 4, SP_ALL = 7, SP_EARLY = 8 };

// STAGE_IN = false leaves the inputs to the caller (the persistent apply's
// fused update writes them into the tile itself).  `parts` selects what is
// copied; COMMIT closes the copy group (a batch staged in two calls commits
// with the second).
// SP_MAT split in two: SP_GEO, the row words, columns and values, which a
// regular chain phase does not read, and SP_HEAD, the slice words and
// pivots, which it does (with the inputs, r and the packed in-unit words).
constexpr int SP_GEO = 16;
constexpr int SP_HEAD = 32;

template <class T, bool FWD, bool WITH_R, bool STAGE_IN = true, bool COMMIT = true>
__device__ __forceinline__ void stage_batch(unsigned char* base, const StageLayout& Ly, const BatchDesc& d,
                                            const SliceMeta* meta, const SellMat& M, const T* dg,
                                            const double* in, const double* rdot, int parts = SP_ALL,
                                            int tid = -1, int nthr = 0)
{
    const int rows = d.qe - d.qb;
    const int p0 = FWD ? d.ps0 : d.pt0, p1 = FWD ? d.ps1 : d.pt1;
    if (parts & (SP_MAT | SP_HEAD)) {
        stage_range(base + Ly.meta, meta, 16, d.sb, d.se - d.sb, tid, nthr);
        stage_range(base + Ly.piv, dg, (int)sizeof(T), d.qb, rows, tid, nthr);
    }
    if (parts & (SP_MAT | SP_GEO)) {
        stage_range(base + Ly.len, M.len, 4, d.qb, rows, tid, nthr);
        stage_range(base + Ly.col, M.col, 4, p0, p1 - p0, tid, nthr);
        stage_range(base + Ly.val, M.val, (int)sizeof(T), p0, p1 - p0, tid, nthr);
    }
    if (STAGE_IN && (parts & SP_IN)) stage_range(base + Ly.in, in, 8, d.qb, rows, tid, nthr);
    if (WITH_R && (parts & SP_RD)) stage_range(base + Ly.rd, rdot, 8, d.qb, rows, tid, nthr);
    if (COMMIT) cp_async_commit();
}

// Phase G of a staged batch (all threads): the earlier-level values of each
// row's entries are gathered and folded into the row's partial sum in the
// tile, or, for the exact backward order, parked beside the entries; each
// row's in-unit entries (count, first two steps and values) are packed for
// phase C.  COH reads the earlier-level values through L2 (the persistent
// apply, where other CTAs of the launch wrote them).
template <class T, bool FWD, bool EXACT, bool COH>
__device__ __forceinline__ void st_gather(const BatchDesc& cur, unsigned char* base, const StageLayout& Ly,
                                          int rows_cap, const double* prev)
{
    constexpr bool ext_first = FWD || !EXACT;
    constexpr int UG = 2;  // slices per warp in flight in G
    constexpr int KG = 4;  // earlier-level entries per row gathered at once
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SliceMeta* s_meta = reinterpret_cast<const SliceMeta*>(base + Ly.meta);
    double* s_in = reinterpret_cast<double*>(base + Ly.in) + (cur.qb & 1);
    const double* s_rd = reinterpret_cast<const double*>(base + Ly.rd) + (cur.qb & 1);
    const T* s_piv = reinterpret_cast<const T*>(base + Ly.piv) + (cur.qb & (16 / (int)sizeof(T) - 1));
    const int* s_len = reinterpret_cast<const int*>(base + Ly.len) + (cur.qb & 3);
    const int* s_col = reinterpret_cast<const int*>(base + Ly.col);
    const T* s_val = reinterpret_cast<const T*>(base + Ly.val);
    double* s_pv = reinterpret_cast<double*>(base + Ly.pv);
    int* s_iw = reinterpret_cast<int*>(base + Ly.iw);
    T* s_iv = reinterpret_cast<T*>(base + Ly.iv);
    const int p0 = FWD ? cur.ps0 : cur.pt0;
    const int ns = cur.se - cur.sb;
    (void)s_rd;

    // G, full batches (every slice 32 rows, so tile row rr is lane
    // rr % 32 of slice rr / 32): rows tid + 256 k, straight-line code
    // with predicated loads, RG rows of a thread in flight at once.
    if (cur.flags & 4) {
        constexpr int RG = 2;
        const int nrows = ns * 32;
        for (int rb = 0; rb < nrows; rb += 256 * RG) {
            int rr[RG], e[RG], j0[RG], j1[RG], ni[RG];
            bool act[RG];
            double xg[RG][KG];
#pragma unroll
            for (int k = 0; k < RG; ++k) {
                rr[k] = rb + (int)threadIdx.x + 256 * k;
                act[k] = rr[k] < nrows;
                const SliceMeta m = s_meta[act[k] ? rr[k] >> 5 : 0];
                const int lw = act[k] ? s_len[rr[k]] : 0;
                const int L = lw & 0xffff;
                ni[k] = lw >> 16;
                e[k] = (FWD ? m.pS : m.pT) - p0 + (rr[k] & 31);
                j0[k] = FWD ? 0 : ni[k];
                j1[k] = FWD ? L - ni[k] : L;
            }
#pragma unroll
            for (int k = 0; k < RG; ++k)
#pragma unroll
                for (int j = 0; j < KG; ++j) {
                    const bool pj = j0[k] + j < j1[k];
                    const int cj = s_col[pj ? e[k] + 32 * (j0[k] + j) : e[k]];
                    xg[k][j] = pj ? ld_prev<COH>(prev + cj) : 0.0;
                }
#pragma unroll
            for (int k = 0; k < RG; ++k) {
                if (!act[k]) continue;
                const int jin = FWD ? j1[k] : 0;
                const int ea = ni[k] > 0 ? e[k] + 32 * jin : e[k];
                const int eb = ni[k] > 1 ? e[k] + 32 * (jin + 1) : e[k];
                const int ca = s_col[ea], cb = s_col[eb];
                const T va = s_val[ea], vb = s_val[eb];
                int w = ni[k] << 16;
                w |= ni[k] > 0 ? -ca - 1 : 0;
                w |= ni[k] > 1 ? (-cb - 1) << 8 : 0;
                s_iw[rr[k]] = w;
                s_iv[rr[k]] = ni[k] > 0 ? va : (T)0;
                s_iv[rows_cap + rr[k]] = ni[k] > 1 ? vb : (T)0;
                if (ext_first) {
                    double a = s_in[rr[k]];
#pragma unroll
                    for (int j = 0; j < KG; ++j) {
                        const bool pj = j0[k] + j < j1[k];
                        const double v = (double)s_val[pj ? e[k] + 32 * (j0[k] + j) : e[k]];
                        a = pj ? fma(-v, xg[k][j], a) : a;
                    }
                    a = fold_ext_staged<8, T, COH>(a, e[k], j0[k] + KG, j1[k], s_col, s_val, prev);
                    s_in[rr[k]] = a;
                } else {
#pragma unroll
                    for (int j = 0; j < KG; ++j)
                        if (j0[k] + j < j1[k]) s_pv[e[k] + 32 * (j0[k] + j)] = xg[k][j];
                    park_ext_staged<8, COH>(e[k], j0[k] + KG, j1[k], s_col, s_pv, prev);
                }
            }
        }
    } else
    // G: earlier-level entries
    for (int t0 = warp; t0 < ns; t0 += 8 * UG) {
        int rr[UG], e[UG], j0[UG], j1[UG];
        bool act[UG];
#pragma unroll
        for (int u = 0; u < UG; ++u) {
            const int t = t0 + 8 * u;
            act[u] = false;
            rr[u] = e[u] = j0[u] = j1[u] = 0;
            if (t < ns) {
                const SliceMeta m = s_meta[t];
                if (lane < (m.w & 63)) {
                    act[u] = true;
                    rr[u] = m.q0 - cur.qb + lane;
                    const int lw = s_len[rr[u]];
                    const int L = lw & 0xffff, ni = lw >> 16;
                    e[u] = (FWD ? m.pS : m.pT) - p0 + lane;
                    j0[u] = FWD ? 0 : ni;
                    j1[u] = FWD ? L - ni : L;
                }
            }
        }
        double x[UG][KG];
#pragma unroll
        for (int u = 0; u < UG; ++u)
#pragma unroll
            for (int j = 0; j < KG; ++j)
                x[u][j] = (act[u] && j0[u] + j < j1[u]) ? ld_prev<COH>(prev + s_col[e[u] + 32 * (j0[u] + j)]) : 0.0;
        // in-unit entries of the row, for the chain: count and first two (step, value)
#pragma unroll
        for (int u = 0; u < UG; ++u) {
            if (!act[u]) continue;
            const int ni = FWD ? s_len[rr[u]] >> 16 : j0[u];
            const int jin = FWD ? j1[u] : 0;
            int w = ni << 16;
            T v0 = (T)0, v1 = (T)0;
            if (ni > 0) {
                w |= -s_col[e[u] + 32 * jin] - 1;
                v0 = s_val[e[u] + 32 * jin];
            }
            if (ni > 1) {
                w |= (-s_col[e[u] + 32 * (jin + 1)] - 1) << 8;
                v1 = s_val[e[u] + 32 * (jin + 1)];
            }
            s_iw[rr[u]] = w;
            s_iv[rr[u]] = v0;
            s_iv[rows_cap + rr[u]] = v1;
        }
#pragma unroll
        for (int u = 0; u < UG; ++u) {
            if (!act[u]) continue;
            if (ext_first) {
                double a = s_in[rr[u]];
#pragma unroll
                for (int j = 0; j < KG; ++j)
                    if (j0[u] + j < j1[u]) a = fma(-(double)s_val[e[u] + 32 * (j0[u] + j)], x[u][j], a);
                a = fold_ext_staged<8, T, COH>(a, e[u], j0[u] + KG, j1[u], s_col, s_val, prev);
                s_in[rr[u]] = a;
            } else {
#pragma unroll
                for (int j = 0; j < KG; ++j)
                    if (j0[u] + j < j1[u]) s_pv[e[u] + 32 * (j0[u] + j)] = x[u][j];
                park_ext_staged<8, COH>(e[u], j0[u] + KG, j1[u], s_col, s_pv, prev);
            }
        }
    }
}

// Phase C of a staged batch, one warp per group and one lane per unit: the
// in-unit chains, from the tile only; each result goes to out and stays in
// the tile for the unit's later steps; r.z (WITH_R) is accumulated.  gl / gs:
// this warp's groups' unit lengths and first slices (groups warp, warp + 8).
template <class T, bool FWD, bool EXACT, bool WITH_R>
__device__ __forceinline__ void st_chain(const BatchDesc& cur, unsigned char* base, const StageLayout& Ly,
                                         int rows_cap, const int (&gl)[2], const int (&gs)[2], double* out,
                                         acc2& rz)
{
    constexpr bool ext_first = FWD || !EXACT;
    constexpr bool with_r = WITH_R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SliceMeta* s_meta = reinterpret_cast<const SliceMeta*>(base + Ly.meta);
    double* s_in = reinterpret_cast<double*>(base + Ly.in) + (cur.qb & 1);
    const double* s_rd = reinterpret_cast<const double*>(base + Ly.rd) + (cur.qb & 1);
    const T* s_piv = reinterpret_cast<const T*>(base + Ly.piv) + (cur.qb & (16 / (int)sizeof(T) - 1));
    const int* s_len = reinterpret_cast<const int*>(base + Ly.len) + (cur.qb & 3);
    const int* s_col = reinterpret_cast<const int*>(base + Ly.col);
    const T* s_val = reinterpret_cast<const T*>(base + Ly.val);
    double* s_pv = reinterpret_cast<double*>(base + Ly.pv);
    int* s_iw = reinterpret_cast<int*>(base + Ly.iw);
    T* s_iv = reinterpret_cast<T*>(base + Ly.iv);
    const int p0 = FWD ? cur.ps0 : cur.pt0;
    (void)s_len;
    (void)s_col;
    (void)s_val;
    (void)s_pv;
    (void)p0;
    // C, regular batches: every group has 32 units of one length and
    // every in-unit entry is the row one step earlier in the sweep, so
    // step r of a group is tile row base + 32 r and the chain is one
    // fused multiply-add (selected by the row's in-unit count) and one
    // division / product per step, with no branches.  (The exact
    // backward order applies earlier-level entries inside the chain
    // and takes the general path.)
    if (ext_first && (cur.flags & (FWD ? 1 : 2))) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int gi = warp + 8 * k;
            if (gi >= cur.ng) break;
            const int len = gl[k];
            const int base = s_meta[gs[k] - cur.sb].q0 - cur.qb + lane;
            double last = 0.0;
            if constexpr (EXACT) {
                // FP64: one step's tile words are loaded a step ahead,
                // so the shared-memory latency stays off a chain whose
                // steps end in a division (it only carries `last`)
                struct Row {
                    double a, rd;
                    T iv, piv;
                    int iw;
                };
                auto row = [&](int t) {
                    const int rr = base + 32 * (FWD ? t : len - 1 - t);
                    Row q;
                    q.a = s_in[rr];
                    q.iv = s_iv[rr];
                    q.iw = s_iw[rr];
                    q.piv = s_piv[rr];
                    q.rd = with_r ? s_rd[rr] : 0.0;
                    return q;
                };
                Row R = len > 0 ? row(0) : Row{};
#pragma unroll 4
                for (int t = 0; t < len; ++t) {
                    const Row N = t + 1 < len ? row(t + 1) : R;
                    const int rr = base + 32 * (FWD ? t : len - 1 - t);
                    double a = R.a;
                    const double x = fma(-(double)R.iv, last, a);
                    a = (R.iw >> 16) ? x : a;
                    const double v = a / (double)R.piv;
                    out[cur.qb + rr] = v;
                    if (with_r) acc2_fma(rz, R.rd, v);
                    last = v;
                    R = N;
                }
            } else {
#pragma unroll 8
                for (int t = 0; t < len; ++t) {
                    const int rr = base + 32 * (FWD ? t : len - 1 - t);
                    double a = s_in[rr];
                    const double x = fma(-(double)s_iv[rr], last, a);
                    a = (s_iw[rr] >> 16) ? x : a;
                    const double v = EXACT ? a / (double)s_piv[rr] : a * (double)s_piv[rr];
                    s_in[rr] = v;
                    out[cur.qb + rr] = v;
                    if (with_r) acc2_fma(rz, s_rd[rr], v);
                    last = v;
                }
            }
        }
    } else {
    // C, general batches: in-unit chains of any shape.  The steps'
    // first Q rows sit in two registers per lane (steps lane and
    // lane + 32, shuffled out).
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int gi = warp + 8 * k;
        if (gi >= cur.ng) break;
        const int len = gl[k];
        const int sbase = gs[k] - cur.sb;
        const int maxlen = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
        const int qlo = lane < maxlen ? s_meta[sbase + lane].q0 - cur.qb : 0;
        const int qhi = lane + 32 < maxlen ? s_meta[sbase + lane + 32].q0 - cur.qb : 0;
        // row of step r for this lane; the shuffle needs the whole
        // warp, so only warp-uniform code (fetch) may call it
        auto row_of = [&](int r) {
            const int q = __shfl_sync(0xffffffffu, r < 32 ? qlo : qhi, r & 31);
            return q + lane;
        };
        // the same from the staged metadata, for per-lane code
        auto row_at = [&](int r) { return s_meta[sbase + r].q0 - cur.qb + lane; };
        double last = 0.0;
        int lastr = -1;
        struct Step {
            int rr, w;
            double a, rd, p, v0, v1;
        };
        auto fetch = [&](int t, Step& S) {
            const int r = FWD ? t : maxlen - 1 - t;
            S.rr = t < maxlen ? row_of(r) : 0;
            if (t < maxlen && r < len) {
                S.a = s_in[S.rr];
                S.p = (double)s_piv[S.rr];
                S.w = s_iw[S.rr];
                S.v0 = (double)s_iv[S.rr];
                S.v1 = (double)s_iv[rows_cap + S.rr];
                if (with_r) S.rd = s_rd[S.rr];
            }
        };
        // value of the unit's row at step idx: the register for the
        // step just done, else the tile (a volatile load, so that it
        // is only issued on the lanes and steps that need it and
        // never sits in front of the chain)
        auto unit_value = [&](int idx) {
            double x = last;
            if (idx != lastr) x = *reinterpret_cast<volatile const double*>(s_in + row_at(idx));
            return x;
        };
        auto step = [&](int t, const Step& S) {
            const int r = FWD ? t : maxlen - 1 - t;
            if (r >= len) return;
            double a = S.a;
            const int ni = S.w >> 16;
            if (ni > 0) a = fma(-S.v0, unit_value(S.w & 0xff), a);
            if (ni > 1) a = fma(-S.v1, unit_value((S.w >> 8) & 0xff), a);
            if (ni > 2 || !ext_first) {
                // more in-unit entries, and the exact backward order's
                // earlier-level entries: from the staged row
                const SliceMeta m = s_meta[sbase + r];
                const int L = s_len[S.rr] & 0xffff;
                const int e0 = (FWD ? m.pS : m.pT) - p0 + lane;
                const int jin = FWD ? L - ni : 0;
                for (int k2 = 2; k2 < ni; ++k2) {
                    const int ek = e0 + 32 * (jin + k2);
                    a = fma(-(double)s_val[ek], unit_value(-s_col[ek] - 1), a);
                }
                if (!ext_first)
                    for (int j = ni; j < L; ++j) {
                        const int ej = e0 + 32 * j;
                        a = fma(-(double)s_val[ej], s_pv[ej], a);
                    }
            }
            const double v = EXACT ? a / S.p : a * S.p;
            s_in[S.rr] = v;
            out[cur.qb + S.rr] = v;
            if (with_r) acc2_fma(rz, S.rd, v);
            last = v;
            lastr = r;
        };
        if constexpr (EXACT) {
            // FP64: each step's tile words are fetched a step ahead
            // (they are the row's own, never written by the steps
            // before it)
            Step A{}, B{};
            fetch(0, A);
            for (int t = 0; t < maxlen; ++t) {
                if (t + 1 < maxlen) fetch(t + 1, B);
                step(t, A);
                A = B;
            }
        } else {
            for (int t = 0; t < maxlen; ++t) {
                Step A{};
                fetch(t, A);
                step(t, A);
            }
        }
    }
    }
}

// EW (loads before the wait): the first batch's copy of the level's own
// arrays, and of the input rows / r where `early` (SP_IN / SP_RD bits) says
// the launch just before this one did not write them, is issued before the
// wait on that launch (griddepcontrol.wait), and the next launch is let in
// right after the wait; the rest of the batch follows the wait.  Every read
// of data the launch before may write (earlier-level values, the solver
// state) comes after the wait.  A template argument: as a run-time flag it
// made the forward FP32 form spill.
template <class T, bool FWD, int FIN, bool EXACT, int NB = 2, bool EW = false>
__global__ void __launch_bounds__(256) k_sweep_st(int b0, int b1, const BatchDesc* __restrict__ bd, int rows_cap,
                                                  int slots_cap, int slices_cap, const int* __restrict__ sl0,
                                                  const int* __restrict__ glen, const SliceMeta* __restrict__ meta,
                                                  SellMat M, const T* __restrict__ dg, const double* in,
                                                  double* out, const double* __restrict__ rdot, int slot0,
                                                  int nslots, SolverState* st, RedBuf red, unsigned int* ticket,
                                                  UpdArgs U, int early)
{
    // FIN_UPDX (forward, one buffer): the fused CG update; each batch's r
    // and Ap are staged (Ap in the area of the backward sweep's r)
    constexpr bool UPD = FIN == FIN_UPDX;
    static_assert(!UPD || (FWD && NB == 1), "the fused update runs in single-buffered forward sweeps");
    constexpr bool with_r = FIN == FIN_RZ || FIN == FIN_RZ0;
    constexpr bool with_pv = !(FWD || !EXACT);
    extern __shared__ __align__(16) unsigned char smem_st[];
    const StageLayout Ly = stage_layout(rows_cap, slots_cap, slices_cap, (int)sizeof(T), with_r || UPD, with_pv);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double* prev = out;  // earlier-level values: read-only in this launch
    acc2 rz[1] = {{0.0, 0.0}};
    const double* stage2 = UPD ? U.Ap : rdot;
    int b = b0 + blockIdx.x;
    constexpr bool ew = EW;
    // the parts of the first batch copied before the wait (none: wait first)
    const int first = ew ? SP_MAT | (UPD ? 0 : early & (SP_IN | SP_RD)) : 0;
    if (!ew) grid_dep_begin();
    if (ew && b < b1) {
        const BatchDesc d0 = bd[b];
        stage_batch<T, FWD, with_r || UPD, true, false>(smem_st, Ly, d0, meta, M, dg, in, stage2, first);
    }
    if (ew) {
        grid_dep_begin();
        grid_dep_trigger();
    }
    if (st_done(st)) {
        // the copies issued above are not in a group yet: close it, so the
        // wait covers them, before the CTA (and its shared memory) goes
        cp_async_commit();
        cp_async_wait<0>();
        return;
    }
    const double alpha = UPD ? st->alpha : 0.0;

    // the fused update of a staged batch's rows (after its copy landed):
    // r -= alpha Ap in the tile and back to r
    auto update = [&](unsigned char* base, const BatchDesc& d) {
        double* s_in = reinterpret_cast<double*>(base + Ly.in) + (d.qb & 1);
        const double* s_ap = reinterpret_cast<const double*>(base + Ly.rd) + (d.qb & 1);
        for (int i = threadIdx.x; i < d.qe - d.qb; i += blockDim.x) {
            const double rn = fma(-alpha, s_ap[i], s_in[i]);
            s_in[i] = rn;
            U.r[d.qb + i] = rn;
            acc2_fma(rz[0], rn, rn);
        }
    };
    if (b < b1) {
        BatchDesc cur = bd[b];
        stage_batch<T, FWD, with_r || UPD>(smem_st, Ly, cur, meta, M, dg, in, stage2, SP_ALL & ~first);
        bool has_next = b + (int)gridDim.x < b1;
        BatchDesc nxt = cur;
        if (has_next) nxt = bd[b + gridDim.x];
        for (int i = 0;; ++i) {
            // NB = 2: batch i + 1 is copied into the other half while batch i
            // is worked on; NB = 1: one buffer, refilled after each batch
            unsigned char* base = smem_st + (NB == 2 ? (i & 1) * Ly.bytes : 0);
            if (NB == 2 && has_next)
                stage_batch<T, FWD, with_r || UPD>(smem_st + ((i + 1) & 1) * Ly.bytes, Ly, nxt, meta, M, dg, in,
                                                   stage2);
            const bool has_nn = has_next && b + 2 * (int)gridDim.x < b1;
            BatchDesc nn = nxt;
            if (has_nn) nn = bd[b + 2 * gridDim.x];
            // group words for C (latency overlaps the wait)
            int gl[2] = {0, 0}, gs[2] = {0, 0};
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int gi = warp + 8 * k;
                if (gi < cur.ng) {
                    gl[k] = glen[(size_t)(cur.gb + gi) * 32 + lane];
                    gs[k] = sl0[cur.gb + gi];
                }
            }
            if (NB == 2 && has_next) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncthreads();
            if (UPD) {
                update(base, cur);
                __syncthreads();
            }

            st_gather<T, FWD, EXACT, false>(cur, base, Ly, rows_cap, prev);
            __syncthreads();

            // backward, single buffer, regular chain: the warps with no group
            // to chain copy the next batch's row words, columns and values
            // (read only by the gather) while the chains run.  (Not forward:
            // there it took the FP32 kernel from 48 to 60 registers, 5 to 4
            // CTAs per SM.)
            constexpr bool ext_first = FWD || !EXACT;
            const int busy = cur.ng < 8 ? cur.ng : 8;
            const bool geo = !FWD && NB == 1 && !UPD && ext_first && has_next && busy < 8 && (cur.flags & 2);
            if (geo && warp >= busy) {
                stage_batch<T, FWD, with_r || UPD>(smem_st, Ly, nxt, meta, M, dg, in, stage2, SP_GEO,
                                                   (int)threadIdx.x - 32 * busy, (int)blockDim.x - 32 * busy);
            }
            st_chain<T, FWD, EXACT, with_r>(cur, base, Ly, rows_cap, gl, gs, out, rz[0]);
            __syncthreads();
            if (!has_next) break;
            if (NB == 1)
                stage_batch<T, FWD, with_r || UPD>(smem_st, Ly, nxt, meta, M, dg, in, stage2,
                                                   geo ? SP_HEAD | SP_IN | SP_RD : SP_ALL);
            b += gridDim.x;
            cur = nxt;
            nxt = nn;
            has_next = has_nn;
        }
    }
    if (!ew) grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(rz, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// ---------------------------------------------------------------------------
// Chain-only levels: every row's entries are in-unit, at most one, on the
// unit's previous step in the sweep's order, and the groups are full (32
// units of one length, at most 16 steps).  A row is then
//     out_r = (in_r - v_r out_{r-1}) / d_r     (v_r absent on a unit's first row)
// with the fused multiply-add and the division / product of the staged
// kernel's regular chain, so the bits are the same.  One warp per group, one
// lane per unit; the steps' rows stream in chunks of CH, the next chunk's
// loads in flight while the current one is chained; no shared memory.
// ---------------------------------------------------------------------------
// `early` as in k_sweep_st: the group words and, for FP32 storage, the first
// chunk's level arrays and the inputs / r it names are loaded before the wait
// on the launch just before.  (The FP64 chunks stay after the wait: held
// across it they take the backward kernel from 114 to 142 registers, one CTA
// per SM, and the level to two waves.)
template <class T, bool FWD, int FIN, bool EXACT>
__global__ void __launch_bounds__(256) k_sweep_chain(int g0, int g1, const int* __restrict__ glen,
                                                     const int* __restrict__ sl0, const SliceMeta* __restrict__ meta,
                                                     SellMat M, const T* __restrict__ dg,
                                                     const double* in, double* __restrict__ out,
                                                     const double* __restrict__ rdot, int slot0, int nslots,
                                                     SolverState* st, RedBuf red, unsigned int* ticket, UpdArgs U,
                                                     int early)
{
    constexpr bool UPD = FIN == FIN_UPDX;  // forward: the fused CG update (r -= alpha Ap) on load
    constexpr bool with_r = FIN == FIN_RZ || FIN == FIN_RZ0;
    constexpr int CH = 4;
    const T* __restrict__ val = (const T*)M.val;
    const int lane = threadIdx.x & 31;
    acc2 rz[1] = {{0.0, 0.0}};
    struct Chunk {
        double a[CH], rd[CH];  // rd: r (backward r.z) or Ap (the fused update)
        T v[CH], p[CH];
        int L[CH], q[CH];
    };
    const int wg = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwg = (int)((gridDim.x * blockDim.x) >> 5);
    const bool ew = (early & SP_EARLY) != 0;
    early = UPD ? 0 : early & (SP_IN | SP_RD);
    int g = g0 + wg;
    int len = 0, my_q = 0, my_p = 0, my_w = 0;
    // lane r holds step r's first Q row, slot pointer and slice width
    auto group = [&](int gg) {
        len = glen[(size_t)gg * 32];  // every unit of the group has this length
        const int sb = sl0[gg];
        const SliceMeta mine = lane < len ? meta[sb + lane] : SliceMeta{0, 0, 0, 0};
        my_q = mine.q0;
        my_p = FWD ? mine.pS : mine.pT;
        my_w = FWD ? (mine.w >> 12) & 255 : (mine.w >> 20) & 255;
    };
    auto load = [&](int t0, Chunk& C, int parts) {
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int t = t0 + u;
            const bool ok = t < len;
            const int rs = ok ? (FWD ? t : len - 1 - t) : 0;
            const int q = __shfl_sync(0xffffffffu, my_q, rs) + lane;
            if (parts & SP_MAT) {
                const int p = __shfl_sync(0xffffffffu, my_p, rs) + lane;
                const int w = __shfl_sync(0xffffffffu, my_w, rs);
                C.q[u] = q;
                C.p[u] = ok ? dg[q] : (T)1;
                C.L[u] = ok ? M.len[q] & 0xffff : 0;
                C.v[u] = (ok && w > 0) ? val[p] : (T)0;
            }
            if (parts & SP_IN) C.a[u] = ok ? __ldcg(in + q) : 0.0;
            if (parts & SP_RD) C.rd[u] = ok ? (with_r ? __ldcg(rdot + q) : UPD ? __ldcg(U.Ap + q) : 0.0) : 0.0;
        }
    };
    Chunk A, B;
    const bool pre = ew && !EXACT;
    if (!ew) grid_dep_begin();
    if (g < g1) {
        group(g);
        if (pre) load(0, A, SP_MAT | early);
    }
    if (ew) {
        grid_dep_begin();
        grid_dep_trigger();
    }
    if (st_done(st)) return;
    const double alpha = UPD ? st->alpha : 0.0;
    for (bool first = true; g < g1; g += nwg, first = false) {
        if (first) {
            load(0, A, pre ? SP_ALL & ~(SP_MAT | early) : SP_ALL);
        } else {
            group(g);
            load(0, A, SP_ALL);
        }
        double last = 0.0;
        for (int t0 = 0; t0 < len; t0 += CH) {
            if (t0 + CH < len) load(t0 + CH, B, SP_ALL);
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                if (t0 + u < len) {
                    double a = A.a[u];
                    if (UPD) {
                        a = fma(-alpha, A.rd[u], a);
                        U.r[A.q[u]] = a;
                        acc2_fma(rz[0], a, a);
                    }
                    const double x = fma(-(double)A.v[u], last, a);
                    a = A.L[u] ? x : a;
                    const double v = EXACT ? a / (double)A.p[u] : a * (double)A.p[u];
                    out[A.q[u]] = v;
                    if (with_r) acc2_fma(rz[0], A.rd[u], v);
                    last = v;
                }
            }
            A = B;
        }
    }
    if (!ew) grid_dep_trigger();
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(rz, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// ---------------------------------------------------------------------------
// The CG update with the first forward level folded in, for a first level
// that is chain-only (k_sweep_chain's rows: at most one in-unit entry, on
// the unit's previous step).  One launch does
//   x += alpha p                       every row (a flat loop over pairs),
//   r -= alpha Ap                      rows [n0, n) in the flat loop, and the
//                                      first level's rows [0, n0) in the chains,
//   y = (r - v y_prev) / d             the first level's chains (warp per group),
// and reduces r.r over both parts (FIN_UPD).  Each element gets the fused
// multiply-adds of k_update and k_sweep_chain, so x, r and y keep their
// bits; the forward sweep then starts at level 1.  The chains run first in
// each warp: their steps are serial, and the flat loop's loads fill the SM
// behind them.  `early`: the flat loop's first two pairs of x, p and r
// (written two or more launches back) and the group words load before the
// wait on the SpMV.
// ---------------------------------------------------------------------------
template <class T, bool EXACT>
__global__ void __launch_bounds__(256) k_update_chain(int g0, int g1, const int* __restrict__ glen,
                                                      const int* __restrict__ sl0,
                                                      const SliceMeta* __restrict__ meta, SellMat M,
                                                      const T* __restrict__ dg, int n0, int n,
                                                      const double* __restrict__ p, const double* __restrict__ Ap,
                                                      double* __restrict__ x, double* __restrict__ r,
                                                      double* __restrict__ y, SolverState* st, RedBuf red,
                                                      unsigned int* ticket, int early)
{
    constexpr int CH = 4;
    const T* __restrict__ val = (const T*)M.val;
    const int lane = threadIdx.x & 31;
    acc2 a[1] = {{0.0, 0.0}};
    const int n2 = n >> 1;
    const int stride = gridDim.x * blockDim.x;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double2* __restrict__ p2 = reinterpret_cast<const double2*>(p);
    const double2* __restrict__ q2 = reinterpret_cast<const double2*>(Ap);
    double2* __restrict__ x2 = reinterpret_cast<double2*>(x);
    double2* __restrict__ r2 = reinterpret_cast<double2*>(r);
    const int wg = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwg = (int)((gridDim.x * blockDim.x) >> 5);
    int g = g0 + wg;
    int len = 0, my_q = 0, my_p = 0, my_w = 0;
    auto group = [&](int gg) {
        len = glen[(size_t)gg * 32];
        const int sb = sl0[gg];
        const SliceMeta mine = lane < len ? meta[sb + lane] : SliceMeta{0, 0, 0, 0};
        my_q = mine.q0;
        my_p = mine.pS;
        my_w = (mine.w >> 12) & 255;
    };
    // the pair's r update: whole (both rows >= n0), second row only, or none
    auto rmask = [&](int i) { return (2 * i >= n0 ? 1 : 0) + (2 * i + 1 >= n0 ? 1 : 0); };
    double2 pre[2][3];
    if (early) {
        if (g < g1) group(g);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int ik = i0 + k * stride;
            if (ik < n2) {
                pre[k][0] = __ldcg(p2 + ik);
                pre[k][1] = __ldcg(x2 + ik);
                if (rmask(ik)) pre[k][2] = __ldcg(r2 + ik);
            }
        }
        grid_dep_begin();
        grid_dep_trigger();
    } else {
        grid_dep_begin();
        if (g < g1) group(g);
    }
    if (st_done(st)) return;
    const double alpha = st->alpha;

    // x for every row, r for the rows from n0 on (k_update's pairs)
    auto pair = [&](int i, int k) {
        double2 pv, xv;
        if (k < 0) {
            pv = p2[i];
            xv = x2[i];
        } else {
            pv = pre[k][0];
            xv = pre[k][1];
        }
        xv.x = fma(alpha, pv.x, xv.x);
        xv.y = fma(alpha, pv.y, xv.y);
        x2[i] = xv;
        const int m = rmask(i);
        if (m == 2) {
            const double2 qv = q2[i];
            double2 rv = k < 0 ? r2[i] : pre[k][2];
            rv.x = fma(-alpha, qv.x, rv.x);
            rv.y = fma(-alpha, qv.y, rv.y);
            r2[i] = rv;
            acc2_fma(a[0], rv.x, rv.x);
            acc2_fma(a[0], rv.y, rv.y);
        } else if (m == 1) {
            const int e = 2 * i + 1;
            const double rk = fma(-alpha, Ap[e], r[e]);
            r[e] = rk;
            acc2_fma(a[0], rk, rk);
        }
    };
    // the pairs loaded before the wait go first (their registers are then
    // free for the chains)
    int i = i0;
    if (early) {
        if (i + stride < n2) {
            pair(i, 0);
            pair(i + stride, 1);
            i += 2 * stride;
        } else if (i < n2) {
            pair(i, 0);
            i = n2;
        }
    }
    // the first level's chains: r of the row, then the row of y
    struct Chunk {
        double r[CH], q[CH];
        T v[CH], d[CH];
        int L[CH], row[CH];
    };
    auto load = [&](int t0, Chunk& C) {
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int t = t0 + u;
            const bool ok = t < len;
            const int rs = ok ? t : 0;
            const int q = __shfl_sync(0xffffffffu, my_q, rs) + lane;
            const int pp = __shfl_sync(0xffffffffu, my_p, rs) + lane;
            const int w = __shfl_sync(0xffffffffu, my_w, rs);
            C.row[u] = q;
            C.r[u] = ok ? r[q] : 0.0;
            C.q[u] = ok ? Ap[q] : 0.0;
            C.d[u] = ok ? dg[q] : (T)1;
            C.L[u] = ok ? M.len[q] & 0xffff : 0;
            C.v[u] = (ok && w > 0) ? val[pp] : (T)0;
        }
    };
    for (bool first = true; g < g1; g += nwg, first = false) {
        if (!first) group(g);
        Chunk A, B;
        load(0, A);
        double last = 0.0;
        for (int t0 = 0; t0 < len; t0 += CH) {
            if (t0 + CH < len) load(t0 + CH, B);
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                if (t0 + u < len) {
                    double rn = fma(-alpha, A.q[u], A.r[u]);
                    r[A.row[u]] = rn;
                    acc2_fma(a[0], rn, rn);
                    const double xx = fma(-(double)A.v[u], last, rn);
                    rn = A.L[u] ? xx : rn;
                    const double v = EXACT ? rn / (double)A.d[u] : rn * (double)A.d[u];
                    y[A.row[u]] = v;
                    last = v;
                }
            }
            A = B;
        }
    }

    for (; i + stride < n2; i += 2 * stride) {
        pair(i, -1);
        pair(i + stride, -1);
    }
    if (i < n2) pair(i, -1);
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const int k = n - 1;
        x[k] = fma(alpha, p[k], x[k]);
        if (k >= n0) {
            const double rk = fma(-alpha, Ap[k], r[k]);
            r[k] = rk;
            acc2_fma(a[0], rk, rk);
        }
    }
    if (!early) grid_dep_trigger();
    reduce_finish<1, FIN_UPD>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// out[q] = in[perm[q]] (gather into Q order) / out[perm[q]] = in[q] (scatter)
__global__ void __launch_bounds__(256) k_gather_vec(int n, const int* __restrict__ perm,
                                                    const double* __restrict__ in, double* __restrict__ out)
{
    grid_dep_begin();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) out[q] = in[perm[q]];
}

__global__ void __launch_bounds__(256) k_scatter_vec(int n, const int* __restrict__ perm,
                                                     const double* __restrict__ in, double* __restrict__ out)
{
    grid_dep_begin();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) out[perm[q]] = in[q];
}

// ---------------------------------------------------------------------------
// IC(0) factorisation of one level (ic0.cpp:56-115), one thread per unit,
// rows of a unit in order.  Failures record (row << 34 | code << 32 | report
// row) with atomicMin, so the smallest failing row -- the one the reference's
// sequential loop throws at -- is reported.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_ic0_level(int u0, int u1, const int* __restrict__ unit_ptr,
                                                   const int* __restrict__ rows, const int* __restrict__ Lp,
                                                   const int* __restrict__ Li, double* Lx,
                                                   const int* __restrict__ dpos, double shift,
                                                   unsigned long long* err)
{
    grid_dep_begin();
    for (int u = u0 + blockIdx.x * blockDim.x + threadIdx.x; u < u1; u += gridDim.x * blockDim.x) {
        const int t0 = unit_ptr ? unit_ptr[u] : u;
        const int t1 = unit_ptr ? unit_ptr[u + 1] : u + 1;
        for (int t = t0; t < t1; ++t) {
            const int i = rows[t];
            const int bi = Lp[i], ei = Lp[i + 1];
            bool fail = false;
            for (int kij = bi; kij < ei; ++kij) {
                const int j = Li[kij];
                if (j >= i) break;
                double s = 0.0;
                int pi = bi, pj = Lp[j];
                const int ej = Lp[j + 1];
                while (pi < ei && pj < ej) {
                    const int c1 = Li[pi], c2 = Li[pj];
                    if (c1 >= j || c2 >= j) break;
                    if (c1 == c2) {
                        s = fma(Lx[pi], Lx[pj], s);
                        ++pi;
                        ++pj;
                    } else if (c1 < c2) {
                        ++pi;
                    } else {
                        ++pj;
                    }
                }
                const double Ljj = Lx[dpos[j]];
                if (fabs(Ljj) < 1e-30) {
                    atomicMin(err, ((unsigned long long)i << 34) | (1ull << 32) | (unsigned)j);
                    fail = true;
                    break;
                }
                Lx[kij] = (Lx[kij] - s) / Ljj;
            }
            if (fail) break;
            double s = 0.0;
            for (int k = bi; k < ei; ++k) {
                if (Li[k] >= i) break;
                s = s + Lx[k] * Lx[k];
            }
            const int di = dpos[i];
            double diag = Lx[di] - s;
            diag += shift;
            if (diag <= 0.0) {
                atomicMin(err, ((unsigned long long)i << 34) | (2ull << 32) | (unsigned)i);
                break;
            }
            Lx[di] = sqrt(diag);
        }
    }
}

// out[k] = (T) src[idx[k]]
template <class T>
__global__ void __launch_bounds__(256) k_gather(long long m, const int* __restrict__ idx,
                                                const double* __restrict__ src, T* __restrict__ out)
{
    grid_dep_begin();
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
        out[k] = (T)src[idx[k]];
}

// out[k] = (T) src[idx[k]], 0 where idx[k] < 0 (SELL padding)
template <class T>
__global__ void __launch_bounds__(256) k_gather_pad(long long m, const int* __restrict__ idx,
                                                    const double* __restrict__ src, T* __restrict__ out)
{
    grid_dep_begin();
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x) {
        const int i = idx[k];
        out[k] = i >= 0 ? (T)src[i] : (T)0;
    }
}

__global__ void __launch_bounds__(256) k_to_f32(long long m, const double* __restrict__ src, float* __restrict__ out)
{
    grid_dep_begin();
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
        out[k] = (float)src[k];
}

// out[k] = (float)(1 / src[k]): reciprocal pivots of the FP32-storage sweeps
__global__ void __launch_bounds__(256) k_recip_f32(long long m, const double* __restrict__ src, float* __restrict__ out)
{
    grid_dep_begin();
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
        out[k] = (float)(1.0 / src[k]);
}

}  // namespace iccg
