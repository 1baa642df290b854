// dd.cuh -- double-double arithmetic for the CG inner products.
//
// The reference accumulates dot() and nrm2() in x87 long double
// (cg_crs.cpp:33-50).  Here every thread accumulates its share with the
// compensated dot product of Ogita, Rump and Oishi ("Accurate sum and dot
// product", SIAM J. Sci. Comput. 26(6), 2005: TwoProduct via FMA plus
// TwoSum), partial results are combined with the double-double addition of
// Bailey's QD library (error-free TwoSum of the high and low parts), and the
// total is rounded once to double.  The result is the correctly rounded dot
// product in all but pathological cancellation cases, and it does not depend
// on timing: every reduction tree below has a fixed shape.
//
// This file must be compiled with --fmad=false: TwoSum and the final
// renormalisations are only exact when no addition is contracted.
#pragma once
#include <cuda_runtime.h>

namespace iccg {

struct dd {
    double hi, lo;
};

__device__ __forceinline__ dd dd_two_sum(double a, double b)
{
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

__device__ __forceinline__ dd dd_fast_two_sum(double a, double b)
{
    double s = a + b;
    double e = b - (s - a);
    return {s, e};
}

__device__ __forceinline__ dd dd_add(dd a, dd b)
{
    dd s = dd_two_sum(a.hi, b.hi);
    dd t = dd_two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = dd_fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return dd_fast_two_sum(s.hi, s.lo);
}

// per-thread compensated accumulator: value = s + c
struct acc2 {
    double s, c;
};

__device__ __forceinline__ void acc2_fma(acc2& a, double x, double y)
{
    double p = x * y;
    double ep = fma(x, y, -p);
    double s = a.s + p;
    double bb = s - a.s;
    double es = (a.s - (s - bb)) + (p - bb);
    a.s = s;
    a.c += ep + es;
}

__device__ __forceinline__ dd acc2_dd(acc2 a) { return dd_two_sum(a.s, a.c); }

__device__ __forceinline__ double dd_round(dd a) { return a.hi + a.lo; }

__device__ __forceinline__ dd dd_shfl_down(dd v, int off)
{
    dd r;
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
    return r;
}

// Fixed-shape block reduction of NV double-double values; the block's sums
// end up in out[] of thread 0.  `sm` needs NV * (blockDim.x / 32) entries.
template <int NV>
__device__ __forceinline__ void block_reduce_dd(dd (&v)[NV], dd* sm, dd (&out)[NV])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[q] = dd_add(v[q], dd_shfl_down(v[q], off));
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sm[q * nw + warp] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            dd x = (lane < nw) ? sm[q * nw + lane] : dd{0.0, 0.0};
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x = dd_add(x, dd_shfl_down(x, off));
            out[q] = x;
        }
    }
    __syncthreads();
}

}  // namespace iccg
