// persist.cuh -- the whole IC(0) apply (forward and backward substitution,
// every level) in one persistent launch.
//
// The sweeps of ic0.cpp:194-339 run level after level; launched one kernel
// per level, each level pays a launch, a ramp-up and a drain, and an apply
// is several launches plus the CG vector kernels around them.  Here the
// work of an apply is a list of items, the staged batches of the per-level
// kernel (k_sweep_st: up to 16 consecutive unit groups of one level, at most
// 512 rows or one larger group): the forward sweep's batches in level order,
// then the backward sweep's in reverse.  Every CTA works on its own: it
// takes the next item from a global ticket counter, waits until the items
// whose rows its entries read are done (per-item done flags, bounded waits),
// stages and computes the batch (phases G and C of the staged kernel) and
// publishes its flag.  A CTA holding ticket t only waits on tickets below t,
// which were taken by CTAs that are running, so the launch always makes
// progress whatever the number of resident CTAs.
//
// Tickets: one 64-bit counter per launch configuration that is never reset.
// A launch takes exactly M = 2 * items + CTAs tickets (each CTA takes
// tickets until it draws one past the items), so ticket D belongs to launch
// e = D / M as item D mod M, and an item's flag holds e + 1 once it is done
// in launch e.  A launch whose solve has already stopped takes no ticket.
//
// With the fused CG update (UPD), a forward batch first does x += alpha p,
// r -= alpha Ap for its rows and writes the new r into its tile as the
// sweep's input, and r.r is reduced with the items.
//
// The floating-point operations of every row are those of the staged
// kernel, so FP64 keeps the reference's bits.  Earlier-level values are read
// through L2 (other CTAs of the launch wrote them).
//
// Reductions (r.r of the fused update, r.z of the backward sweep) are exact
// and independent of which CTA took which item: each item's sum goes to its
// own slot, published with the item's done flag, and the CTA holding the
// sweep's last ticket adds all slots in a fixed order once every item of
// the sweep is done, then runs the CG scalar logic.
#pragma once
#include "kernels.cuh"

namespace iccg {

// per launch configuration
struct PCtl {
    unsigned long long draws;  // tickets taken, all launches
    unsigned int upd_done;     // launch index + 1 once the fused update's r.r has been finished
    unsigned int pad;
};

struct PArgs {
    int nitems;               // items of one sweep
    const BatchDesc* items;   // forward order; backward item b is items[nitems - 1 - b]
    const int* dep_ptr;       // per ticket (2 * nitems + 1)
    const int* dep_idx;       // tickets each ticket waits for
    unsigned int* flags;      // per ticket: launch index + 1 when done
    PCtl* ctl;
    dd* slot;                 // [2][nitems] per-item sums
    unsigned int* err;        // 1 + ticket of a dependency wait that gave up
    const int* glen;
    const int* sl0;
    const SliceMeta* meta;
    SellMat S, T;             // forward / backward matrices (in-unit entries encoded)
    const void* dg;           // pivots (FP64) or reciprocal pivots (FP32)
    double* r;                // forward input (r); r of the backward r.z
    double* y;                // forward output, backward input
    double* z;                // backward output
    double* x;                // fused update: x += alpha p
    const double* p;
    const double* Ap;
    SolverState* st;
};

constexpr int kPersistThreads = 256;
constexpr unsigned int kPersistSpin = 1u << 22;  // polls before a dependency wait gives up

__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int* p)
{
    return *reinterpret_cast<const volatile unsigned int*>(p);
}

// A batch's stage layout, sized to the batch itself (the backward one
// holds r for r.z, and with FP64 the gathered values parked for the exact
// order); the launch's shared memory is the largest over all batches.
template <class T, bool RED, bool EXACT>
__host__ __device__ inline StageLayout persist_layout(const BatchDesc& d, bool fwd)
{
    return fwd ? stage_layout(d.qe - d.qb, d.ps1 - d.ps0, d.se - d.sb, (int)sizeof(T), false, false)
               : stage_layout(d.qe - d.qb, d.pt1 - d.pt0, d.se - d.sb, (int)sizeof(T), RED, EXACT);
}

// Fixed-order warp sum of a double-double value (lane 0 holds the result).
__device__ __forceinline__ dd warp_sum_dd(dd v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = dd_add(v, dd_shfl_down(v, off));
    return v;
}

// Waits until the items of ticket t's dependency list are done in the
// launch tagged `tag` (threads poll in parallel; bounded waits), then makes
// their writes visible to the whole CTA: each polling thread fences after
// what it observed, and the CTA barrier orders the other threads' reads
// after those fences.  `first` is the thread's first flag read, issued
// earlier (see persist_batch), or ~0u.
__device__ __forceinline__ void persist_wait_deps(const PArgs& A, int t, unsigned int tag, unsigned int first)
{
    bool polled = false;
    for (int k = A.dep_ptr[t] + threadIdx.x; k < A.dep_ptr[t + 1]; k += blockDim.x) {
        const unsigned int* f = A.flags + A.dep_idx[k];
        unsigned int it = 0;
        unsigned int v = !polled ? first : ld_volatile_u32(f);
        polled = true;
        while (v != tag) {
            __nanosleep(32);
            v = ld_volatile_u32(f);
            // give up after the poll limit, or at once after another wait of
            // this launch gave up (no chain of timeouts)
            if (++it > kPersistSpin || ld_volatile_u32(A.err) != 0u) {
                atomicCAS(A.err, 0u, (unsigned int)t + 1u);
                break;
            }
        }
    }
    if (polled) __threadfence();
    __syncthreads();
}

// One batch of one sweep, all threads of the CTA.  What does not depend on
// other items -- the batch's matrix data (and, forward, its input r) staged
// by cp.async, and the fused update -- is started before the dependency
// wait, so the wait overlaps those copies; the backward input y and r
// (written by forward items of this launch) are staged after it.
template <class T, bool FWD, bool EXACT, bool UPD, bool RED>
__device__ __forceinline__ void persist_batch(const PArgs& A, int t, unsigned int tag, const BatchDesc& cur,
                                              unsigned char* base, acc2& red, double alpha)
{
    constexpr bool with_r = RED && !FWD;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const StageLayout Ly = persist_layout<T, RED, EXACT>(cur, FWD);
    const int rows = cur.qe - cur.qb;
    const SellMat& M = FWD ? A.S : A.T;
    const T* dg = (const T*)A.dg;
    double* out = FWD ? A.y : A.z;
    const int p0 = FWD ? cur.ps0 : cur.pt0, p1 = FWD ? cur.ps1 : cur.pt1;
    stage_range(base + Ly.meta, A.meta, 16, cur.sb, cur.se - cur.sb);
    stage_range(base + Ly.piv, dg, (int)sizeof(T), cur.qb, rows);
    stage_range(base + Ly.len, M.len, 4, cur.qb, rows);
    stage_range(base + Ly.col, M.col, 4, p0, p1 - p0);
    stage_range(base + Ly.val, M.val, (int)sizeof(T), p0, p1 - p0);
    if (FWD && !UPD) stage_range(base + Ly.in, A.r, 8, cur.qb, rows);
    cp_async_commit();
    // the thread's first dependency flag, read now so that its round trip
    // overlaps the update below
    unsigned int first = ~0u;
    {
        const int k = A.dep_ptr[t] + threadIdx.x;
        if (k < A.dep_ptr[t + 1]) first = ld_volatile_u32(A.flags + A.dep_idx[k]);
    }
    if (UPD) {
        // x += alpha p, r -= alpha Ap (cg_crs.cpp:137-141) for the batch's
        // rows; the new r is the sweep's input
        double* s_in = reinterpret_cast<double*>(base + Ly.in) + (cur.qb & 1);
        for (int i = threadIdx.x; i < rows; i += blockDim.x) {
            const int q = cur.qb + i;
            const double rq = __ldcg(A.r + q), apq = __ldg(A.Ap + q), pq = __ldg(A.p + q), xq = A.x[q];
            A.x[q] = fma(alpha, pq, xq);
            const double rn = fma(-alpha, apq, rq);
            A.r[q] = rn;
            s_in[i] = rn;
            acc2_fma(red, rn, rn);
        }
    }
    int gl[2] = {0, 0}, gs[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int gi = warp + 8 * k;
        if (gi < cur.ng) {
            gl[k] = __ldg(A.glen + (size_t)(cur.gb + gi) * 32 + lane);
            gs[k] = __ldg(A.sl0 + cur.gb + gi);
        }
    }
    persist_wait_deps(A, t, tag, first);
    if (!FWD) {
        stage_range(base + Ly.in, A.y, 8, cur.qb, rows);
        if (with_r) stage_range(base + Ly.rd, A.r, 8, cur.qb, rows);
        cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
    st_gather<T, FWD, EXACT, true>(cur, base, Ly, rows, out);
    __syncthreads();
    st_chain<T, FWD, EXACT, with_r>(cur, base, Ly, rows, gl, gs, out, red);
}

// The sweep's total: run by the CTA holding the sweep's last ticket once
// every item of the sweep is done (their per-item sums, in their slots, are
// covered by their done flags).  Each thread adds a fixed set of slots in
// order and the block adds the threads' sums in a fixed tree, so the total
// does not depend on which CTA runs it.  Then the CG scalar logic: FIN_UPD
// for the forward sweep's r.r (the fused update), FIN_RZ0 / FIN_RZ for the
// backward sweep's r.z, decisions deferred to st->pend.
template <int FIN, bool UPD>
__device__ __forceinline__ void persist_total(const PArgs& A, int dir, unsigned int tag, dd* s_red)
{
    const int t0 = dir ? A.nitems : 0;
    for (int k = threadIdx.x; k < A.nitems; k += blockDim.x) {
        const unsigned int* f = A.flags + t0 + k;
        unsigned int it = 0;
        while (ld_volatile_u32(f) != tag) {
            __nanosleep(64);
            if (++it > kPersistSpin || ld_volatile_u32(A.err) != 0u) {
                atomicCAS(A.err, 0u, 0x40000001u);
                break;
            }
        }
    }
    __threadfence();
    __syncthreads();
    dd acc{0.0, 0.0};
    for (int k = threadIdx.x; k < A.nitems; k += blockDim.x) {
        const dd* p = A.slot + (size_t)dir * A.nitems + k;
        dd w;
        w.hi = __ldcg(&p->hi);
        w.lo = __ldcg(&p->lo);
        acc = dd_add(acc, w);
    }
    dd v[1] = {acc}, tot[1];
    block_reduce_dd<1>(v, s_red, tot);
    if (threadIdx.x != 0) return;
    double rv[1] = {dd_round(tot[0])};
    SolverState* st = A.st;
    if (dir == 0) {
        // the fused update's r.r (FIN_UPD); the backward total waits for it
        finish<FIN_UPD, true>(rv, st, nullptr);
        __threadfence();
        *reinterpret_cast<volatile unsigned int*>(&A.ctl->upd_done) = tag;
        return;
    }
    if (UPD) {
        unsigned int it = 0;
        while (ld_volatile_u32(&A.ctl->upd_done) != tag) {
            __nanosleep(64);
            if (++it > kPersistSpin || ld_volatile_u32(A.err) != 0u) {
                atomicCAS(A.err, 0u, 0x40000000u);
                break;
            }
        }
        __threadfence();
        // the solve stopped at this iteration's update: r.z of its residual
        // is not used (the reference returns before z = M^-1 r)
        if (*reinterpret_cast<volatile int*>(&st->pend) != kRunning) return;
    }
    finish<FIN, true>(rv, st, nullptr);
}

template <class T, bool EXACT, bool UPD, int FIN>
__global__ void __launch_bounds__(kPersistThreads, 4) k_apply_persist(PArgs A)
{
    constexpr bool RED = FIN != FIN_NONE;
    grid_dep_begin();
    // st->status does not change while this kernel runs (its own decisions
    // go to st->pend), so every CTA takes the same branch here
    if (st_done(A.st)) return;
    extern __shared__ __align__(16) unsigned char smem_persist[];
    __shared__ unsigned long long s_draw;
    __shared__ dd s_red[kPersistThreads / 32];
    const int tid = threadIdx.x;
    const unsigned long long M = 2ull * (unsigned long long)A.nitems + (unsigned long long)gridDim.x;
    const double alpha = UPD ? A.st->alpha : 0.0;
    unsigned long long Dn = 0;
    if (tid == 0) Dn = atomicAdd(&A.ctl->draws, 1ull);
    for (;;) {
        if (tid == 0) s_draw = Dn;
        __syncthreads();
        const unsigned long long D = s_draw;
        const unsigned long long e = D / M;
        const int t = (int)(D - e * M);
        if (t >= 2 * A.nitems) break;
        const unsigned int tag = (unsigned int)e + 1u;
        // the next ticket is taken now, so its round trip overlaps this item
        // (a CTA waiting for it waits on a ticket above its own, which this
        // CTA only starts after this item: the lowest unfinished ticket is
        // always being worked on)
        if (tid == 0) Dn = atomicAdd(&A.ctl->draws, 1ull);
        const bool fwd = t < A.nitems;
        const int idx = fwd ? t : t - A.nitems;
        const BatchDesc cur = A.items[fwd ? t : A.nitems - 1 - idx];
        acc2 red = {0.0, 0.0};
        if (fwd) persist_batch<T, true, EXACT, UPD, false>(A, t, tag, cur, smem_persist, red, alpha);
        else persist_batch<T, false, EXACT, false, RED>(A, t, tag, cur, smem_persist, red, 0.0);
        const bool sums = fwd ? UPD : RED;
        if (sums) {
            // the item's sum into its slot, published with its flag
            dd v[1] = {acc2_dd(red)}, tot[1];
            block_reduce_dd<1>(v, s_red, tot);
            if (tid == 0) A.slot[(size_t)(fwd ? 0 : 1) * A.nitems + idx] = tot[0];
        }
        // publish: the CTA barrier orders every thread's stores before
        // thread 0's fence, which is cumulative, then the flag (the pattern
        // of a grid-wide barrier)
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            *reinterpret_cast<volatile unsigned int*>(A.flags + t) = tag;
        }
        if (sums && idx == A.nitems - 1) persist_total<FIN, UPD>(A, fwd ? 0 : 1, tag, s_red);
    }
    grid_dep_trigger();
}

}  // namespace iccg
