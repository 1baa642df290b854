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
    int pad;
    unsigned int ticket;
    unsigned int pad2;
};

enum Fin {
    FIN_NONE = 0,
    FIN_STORE,  // write the rounded sums to out[]
    FIN_INIT,   // (b.b, r.r): normb, initial convergence test
    FIN_RZ0,    // (r.z): rz_old
    FIN_PAP,    // (p.Ap, p.p, Ap.Ap): breakdown test, alpha
    FIN_UPD,    // (r.r): rel, convergence / replacement trigger
    FIN_TRUE,   // (r.r) of the replaced residual: convergence
    FIN_RZ,     // (r.z): beta, rz_old
};

struct RedBuf {
    dd* partials;   // [slots * NV]
    double* out;    // FIN_STORE destination
};

__device__ __forceinline__ bool st_done(const SolverState* st)
{
    return st != nullptr && *(volatile const int*)&st->status != kRunning;
}

// CG scalar logic of cg_crs.cpp:108-159, run by one thread.
template <int FIN>
__device__ void finish(const double* v, SolverState* st, double* out)
{
    if (FIN == FIN_STORE) {
        out[0] = v[0];
        return;
    }
    if (FIN == FIN_INIT) {
        double normb = sqrt(v[0]);
        if (normb == 0.0) normb = 1.0;
        st->normb = normb;
        double rel = sqrt(v[1]) / normb;
        st->rel_resid = rel;
        st->iters = 0;
        if (rel < st->tol) st->status = kConverged;
        else if (st->max_iter <= 0) st->status = kMaxIter;
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
            st->status = kBreakdown;
            return;
        }
        if (!isfinite(pAp)) {
            st->iters = st->k;
            st->status = kNonFinite;
            return;
        }
        st->alpha = st->rz_old / pAp;
        return;
    }
    if (FIN == FIN_UPD) {
        const double rel = sqrt(v[0]) / st->normb;
        st->iters = st->k + 1;
        st->rel_resid = rel;
        if (!isfinite(rel)) { st->status = kNonFinite; return; }
        if (st->rr_interval <= 0) {
            if (rel < st->tol) st->status = kConverged;
        } else if (rel < st->tol || (st->k + 1) % st->rr_interval == 0) {
            st->rr_flag = 1;
        }
        return;
    }
    if (FIN == FIN_TRUE) {
        const double rel = sqrt(v[0]) / st->normb;
        st->rel_resid = rel;
        st->rr_flag = 0;
        st->n_rr += 1;
        if (rel < st->tol) st->status = kConverged;
        return;
    }
    if (FIN == FIN_RZ) {
        const double rz = v[0];
        st->beta = rz / st->rz_old;
        st->rz_old = rz;
        if (!isfinite(st->beta)) { st->status = kNonFinite; st->iters = st->k + 1; }
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
    if (FIN == FIN_INIT) reduce_finish<2, FIN_INIT>(a, red, st, ticket, blockIdx.x, gridDim.x);
    if (FIN == FIN_TRUE) {
        acc2 t[1] = {a[0]};
        reduce_finish<1, FIN_TRUE>(t, red, st, ticket, blockIdx.x, gridDim.x);
    }
}

// x += alpha p; r -= alpha Ap (cg_crs.cpp:137-141), then r.r (cg_crs.cpp:143).
// alpha comes from the state (fused) or from the argument (st == nullptr).
template <int FIN>
__global__ void __launch_bounds__(256) k_update(int n, double alpha_arg, const double* __restrict__ p,
                                                const double* __restrict__ Ap, double* __restrict__ x,
                                                double* __restrict__ r, SolverState* st, RedBuf red,
                                                unsigned int* ticket)
{
    if (st_done(st)) return;
    const double alpha = st ? st->alpha : alpha_arg;
    acc2 a[1] = {{0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, Ap[i], r[i]);
        r[i] = ri;
        if (FIN != FIN_NONE) acc2_fma(a[0], ri, ri);
    }
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// p = z + beta p (cg_crs.cpp:155-157); the fused form then advances k and
// stops the solve after max_iter iterations (cg_crs.cpp:125).
__global__ void __launch_bounds__(256) k_xpay(int n, double beta_arg, const double* __restrict__ z,
                                              double* __restrict__ p, SolverState* st)
{
    if (st_done(st)) return;
    const double beta = st ? st->beta : beta_arg;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = fma(beta, p[i], z[i]);
    if (st && blockIdx.x == 0 && threadIdx.x == 0) {
        const int k1 = st->k + 1;
        st->k = k1;
        if (k1 >= st->max_iter) st->status = kMaxIter;
    }
}

__global__ void __launch_bounds__(256) k_copy(int n, const double* __restrict__ a, double* __restrict__ b,
                                              SolverState* st)
{
    if (st_done(st)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

__global__ void __launch_bounds__(256) k_sub(int n, const double* __restrict__ b, const double* __restrict__ ax,
                                             double* __restrict__ r)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] = b[i] - ax[i];
}

// generic dot a.b (FIN_STORE) -- dot()/nrm2() of cg_crs.cpp:33-50
__global__ void __launch_bounds__(256) k_dot(int n, const double* __restrict__ a, const double* __restrict__ b,
                                             RedBuf red, unsigned int* ticket)
{
    acc2 s[1] = {{0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc2_fma(s[0], a[i], b[i]);
    reduce_finish<1, FIN_STORE>(s, red, nullptr, ticket, blockIdx.x, gridDim.x);
}

// Identity (precond.hpp:12-14, inv == nullptr) or Jacobi (precond.hpp:38-42)
// z = inv .* r, with r.z for FIN_RZ0 / FIN_RZ.
template <int FIN>
__global__ void __launch_bounds__(256) k_diag_apply(int n, const double* __restrict__ inv,
                                                    const double* __restrict__ r, double* __restrict__ z,
                                                    SolverState* st, RedBuf red, unsigned int* ticket)
{
    if (st_done(st)) return;
    acc2 a[1] = {{0.0, 0.0}};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = r[i];
        const double zi = inv ? inv[i] * ri : ri;
        z[i] = zi;
        if (FIN != FIN_NONE) acc2_fma(a[0], ri, zi);
    }
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
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(acc, red, st, ticket, slot0 + blockIdx.x, nslots);
}

// ---------------------------------------------------------------------------
// Tiled kernels.
//
// A CTA tile is a range of at most 256 consecutive rows whose CSR entries
// [rowptr[R0], rowptr[R1]) are contiguous in memory.  The CTA first copies
// that segment (column indices and values) into shared memory with 16-byte
// vector loads marked streaming (evict-first: the matrix is read once per
// iteration and should not push the vectors out of L2), then one thread per
// row runs the row's arithmetic from shared memory in the reference's order.
// Segments start at the 4-entry boundary at or below rowptr[R0]; every
// device array carries 16 entries of padding, so the rounded-up tail of the
// last tile stays inside the allocation.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void stage_segment(const int* __restrict__ gcol, const T* __restrict__ gval, int ea,
                                              int cnt, int* s_col, T* s_val)
{
    const int nv = (cnt + 3) >> 2;  // 4-entry groups
    const int4* c4 = reinterpret_cast<const int4*>(gcol + ea);
    int4* sc4 = reinterpret_cast<int4*>(s_col);
    for (int v = threadIdx.x; v < nv; v += blockDim.x) sc4[v] = __ldcs(c4 + v);
    if (sizeof(T) == 4) {
        const float4* v4 = reinterpret_cast<const float4*>(gval + ea);
        float4* sv4 = reinterpret_cast<float4*>(s_val);
        for (int v = threadIdx.x; v < nv; v += blockDim.x) sv4[v] = __ldcs(v4 + v);
    } else {
        const double2* v2 = reinterpret_cast<const double2*>(gval + ea);
        double2* sv2 = reinterpret_cast<double2*>(s_val);
        for (int v = threadIdx.x; v < 2 * nv; v += blockDim.x) sv2[v] = __ldcs(v2 + v);
    }
}

// SpMV over CTA tiles (tile_row: ntiles+1 row boundaries); same arithmetic as
// k_spmv.  Dynamic shared memory: cap * (4 + sizeof(T)) bytes.
template <class T, int FIN>
__global__ void __launch_bounds__(256) k_spmv_tiled(int ntiles, const int* __restrict__ tile_row,
                                                    const int* __restrict__ rp, const int* __restrict__ ci,
                                                    const T* __restrict__ v, int cap,
                                                    const double* __restrict__ x, double* __restrict__ y,
                                                    SolverState* st, RedBuf red, unsigned int* ticket)
{
    if (st_done(st)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s_val = reinterpret_cast<T*>(smem_raw);
    int* s_col = reinterpret_cast<int*>(smem_raw + (size_t)cap * sizeof(T));
    acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int R0 = tile_row[t], R1 = tile_row[t + 1];
        const int e0 = rp[R0], e1 = rp[R1];
        const int ea = e0 & ~3;
        stage_segment<T>(ci, v, ea, e1 - ea, s_col, s_val);
        const int i = R0 + threadIdx.x;
        int rs = 0, re = 0;
        if (i < R1) {
            rs = rp[i] - ea;
            re = rp[i + 1] - ea;
        }
        __syncthreads();
        if (i < R1) {
            double sum = 0.0;
            for (int k = rs; k < re; ++k) sum = sum + (double)s_val[k] * __ldg(x + s_col[k]);
            y[i] = sum;
            if (FIN == FIN_PAP) {
                const double xi = __ldg(x + i);
                acc2_fma(a[0], xi, sum);
                acc2_fma(a[1], xi, xi);
                acc2_fma(a[2], sum, sum);
            }
        }
        __syncthreads();
    }
    if (FIN == FIN_PAP) reduce_finish<3, FIN_PAP>(a, red, st, ticket, blockIdx.x, gridDim.x);
}

// Warp tile of a substitution level: `nrows` (<= 32) consecutive rows from
// `row0`, made of whole units (blocks); bit l of `mask` is set where lane l
// starts a unit; `nsteps` is the longest unit.  Eight warp tiles form one CTA
// tile (rows contiguous across them; empty ones pad the end of a level).
struct WarpTile {
    int row0;
    int nrows;
    unsigned int mask;
    int nsteps;
};

// Forward (L y = r, FWD) or backward (L^T z = y) substitution over the CTA
// tiles [ct0, ct1) of one level of a contiguous schedule.  Lane l owns row
// i = row0 + l of its warp tile; its unit spans lanes [us, ue).
//
// Forward: the entries of row i with column below the unit's first row
// (earlier levels, final) are applied first, fully in parallel -- they come
// first in the reference's column order; the unit's own entries follow, one
// step per row of the unit: at step s the lane with position s in its unit
// applies its in-unit entries (their y values are in the shared tile) and
// divides.  Backward: in-unit entries come first in column order, so at its
// step (units run in descending row order) a lane applies its in-unit
// entries from the shared tile, then the later-level entries, whose values
// (and matrix entries) were fetched into registers before the steps began.
// The operation order per row equals the reference's sequential sweep.
template <class T, bool FWD, int KX, int FIN>
__global__ void __launch_bounds__(256) k_sweep_tiled(int ct0, int ct1, const WarpTile* __restrict__ wt,
                                                     const int* __restrict__ Sp, const int* __restrict__ Si,
                                                     const T* __restrict__ Sx, const T* __restrict__ dg,
                                                     int cap, const double* __restrict__ in, double* out,
                                                     const double* __restrict__ rdot, int slot0, int nslots,
                                                     SolverState* st, RedBuf red, unsigned int* ticket)
{
    if (st_done(st)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* s_y = reinterpret_cast<double*>(smem_raw);                       // 256 rows
    T* s_val = reinterpret_cast<T*>(smem_raw + 256 * sizeof(double));
    int* s_col = reinterpret_cast<int*>(smem_raw + 256 * sizeof(double) + (size_t)cap * sizeof(T));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    acc2 rz[1] = {{0.0, 0.0}};
    for (int ct = ct0 + blockIdx.x; ct < ct1; ct += gridDim.x) {
        // padding warp tiles start at the end row with nrows = 0
        const int R0 = wt[(size_t)ct * 8].row0;
        const WarpTile w7 = wt[(size_t)ct * 8 + 7];
        const int R1 = w7.row0 + w7.nrows;
        const int e0 = Sp[R0], e1 = Sp[R1];
        const int ea = e0 & ~3;
        stage_segment<T>(Si, Sx, ea, e1 - ea, s_col, s_val);
        const WarpTile w = wt[(size_t)ct * 8 + warp];
        const bool valid = lane < w.nrows;
        const int i = w.row0 + lane;
        // unit of this lane: lanes [us, ue)
        const unsigned int below = w.mask & (0xffffffffu >> (31 - lane));
        const int us = 31 - __clz(below);
        const unsigned int above = w.mask & ~(0xffffffffu >> (31 - lane));
        const int ue = above ? (__ffs(above) - 1) : w.nrows;
        const int pos = FWD ? (lane - us) : (ue - 1 - lane);
        const int urow0 = w.row0 + us, urow1 = w.row0 + ue;
        double acc = 0.0, dv = 1.0;
        int k = 0, ke = 0;
        if (valid) {
            acc = in[i];
            dv = (double)dg[i];
            k = Sp[i] - ea;
            ke = Sp[i + 1] - ea;
        }
        __syncthreads();
        double xv[KX > 0 ? KX : 1];
        T lv[KX > 0 ? KX : 1];
        int kin = k, nx = 0;
        if (valid) {
            if (FWD) {
                // earlier-level entries: parallel part of the chain
                while (k < ke && s_col[k] < urow0) {
                    acc = fma(-(double)s_val[k], out[s_col[k]], acc);
                    ++k;
                }
            } else {
                while (kin < ke && s_col[kin] < urow1) ++kin;
#pragma unroll
                for (int q = 0; q < KX; ++q) {
                    if (kin + q < ke) {
                        lv[q] = s_val[kin + q];
                        xv[q] = out[s_col[kin + q]];
                        ++nx;
                    }
                }
            }
        }
        double v = 0.0;
        for (int s = 0; s < w.nsteps; ++s) {
            if (valid && pos == s) {
                if (FWD) {
                    for (; k < ke; ++k) acc = fma(-(double)s_val[k], s_y[s_col[k] - R0], acc);
                } else {
                    for (int q = k; q < kin; ++q) acc = fma(-(double)s_val[q], s_y[s_col[q] - R0], acc);
#pragma unroll
                    for (int q = 0; q < KX; ++q)
                        if (q < nx) acc = fma(-(double)lv[q], xv[q], acc);
                    for (int q = kin + nx; q < ke; ++q) acc = fma(-(double)s_val[q], out[s_col[q]], acc);
                }
                v = acc / dv;
                s_y[i - R0] = v;
            }
            __syncwarp();
        }
        if (valid) {
            out[i] = v;
            if (FIN != FIN_NONE) acc2_fma(rz[0], rdot[i], v);
        }
        __syncthreads();
    }
    if (FIN != FIN_NONE) reduce_finish<1, FIN>(rz, red, st, ticket, slot0 + blockIdx.x, nslots);
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
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
        out[k] = (T)src[idx[k]];
}

__global__ void __launch_bounds__(256) k_to_f32(long long m, const double* __restrict__ src, float* __restrict__ out)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
        out[k] = (float)src[k];
}

}  // namespace iccg
