// setup_dev.cu -- a set-up step on the device: the permuted system A_run of
// the reference's caller, Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141)
// followed by expand_lower_to_full (crs_io.cpp:163-227, cg_crs.cpp:421).
//
// The reference takes the lower triangle of A (entries j <= i, color.cpp:91),
// maps each entry to (new_of_old[i], new_of_old[j]) folded to the lower
// triangle (:97-98), sorts each row, sums equal columns, drops entries equal
// to 0.0 (:123, :132), and mirrors the result to a full matrix with sorted
// rows.  Two entries of the lower triangle map to the same output position
// only if the input repeats an (i, j) pair, so when no pair repeats every
// output entry is one input value: the device result is then the same bits
// as the host routines.  Here each lower entry is written to its row and to
// its mirror row, each row is sorted by column, and zeros are dropped.  An
// input that repeats a pair (the summation order would matter) or has a row
// of more than kMaxRow entries is handed to the host routines instead, with
// the same result.

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/iccg.h"
#include "devbuf.hpp"
#include "host.hpp"

namespace iccg {

extern thread_local std::string g_host_err;  // host_capi.cpp

namespace ptap_dev {

constexpr int kThreads = 256;
constexpr int kMaxRow = 256;   // longer output rows go to the host routines
constexpr int kScanTile = 1024;

enum ErrBits { E_RANGE = 1, E_PERM = 2, E_DUP = 4, E_LONG = 8 };

// new_of_old must be a permutation of 0..n-1
__global__ void k_check_perm(int n, const int* __restrict__ p, int* __restrict__ seen, int* err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int q = p[i];
        if (q < 0 || q >= n || atomicExch(&seen[q], 1) != 0) atomicOr(err, E_PERM);
    }
}

// entries per output row: each lower entry (j <= i) lands in row p[i] and,
// off the diagonal, in row p[j]
__global__ void k_count(int n, const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ p,
                        int* __restrict__ cnt, int* err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int pi = p[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < 0 || j >= n) {
                atomicOr(err, E_RANGE);
                continue;
            }
            if (j > i) continue;
            atomicAdd(&cnt[pi], 1);
            if (j != i) atomicAdd(&cnt[p[j]], 1);
        }
    }
}

// exclusive scan of one tile of kScanTile counts per CTA; the tile sums go
// to tsum (scanned on the host, added back by k_scan_add)
__global__ void __launch_bounds__(kThreads) k_scan_tile(int m, const int* __restrict__ in, long long* __restrict__ out,
                                                        long long* __restrict__ tsum)
{
    __shared__ long long s[kScanTile];
    const int base = blockIdx.x * kScanTile;
    for (int t = threadIdx.x; t < kScanTile; t += blockDim.x) s[t] = base + t < m ? in[base + t] : 0;
    __syncthreads();
    // Hillis-Steele inclusive scan over the tile (log2 1024 = 10 rounds)
    for (int d = 1; d < kScanTile; d <<= 1) {
        long long v[kScanTile / kThreads];
#pragma unroll
        for (int u = 0; u < kScanTile / kThreads; ++u) {
            const int t = threadIdx.x + u * kThreads;
            v[u] = t >= d ? s[t - d] : 0;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kScanTile / kThreads; ++u) s[threadIdx.x + u * kThreads] += v[u];
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kScanTile; t += blockDim.x)
        if (base + t < m) out[base + t] = (t == 0 ? 0 : s[t - 1]);
    if (threadIdx.x == 0) tsum[blockIdx.x] = s[kScanTile - 1];
}

__global__ void k_scan_add(int m, long long* __restrict__ out, const long long* __restrict__ toff)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        out[i] += toff[i / kScanTile];
}

// every lower entry into its row (and its mirror row) at a free position
__global__ void k_scatter(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ val,
                          const int* __restrict__ p, int* __restrict__ cur, int* __restrict__ oc,
                          double* __restrict__ ov)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int pi = p[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < 0 || j >= n || j > i) continue;
            const int pj = p[j];
            const double v = val[k];
            int pos = atomicAdd(&cur[pi], 1);
            oc[pos] = pj;
            ov[pos] = v;
            if (j != i) {
                pos = atomicAdd(&cur[pj], 1);
                oc[pos] = pi;
                ov[pos] = v;
            }
        }
    }
}

// each row sorted by column (insertion sort, one thread per row); a repeated
// column or a row longer than kMaxRow sets the error word; nz[r] counts the
// entries that are not 0.0
__global__ void k_sort_rows(int n, const long long* __restrict__ off, int* __restrict__ oc, double* __restrict__ ov,
                            int* __restrict__ nz, int* err)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const long long a = off[r], e = off[r + 1];
        if (e - a > kMaxRow) {
            atomicOr(err, E_LONG);
            nz[r] = 0;
            continue;
        }
        for (long long k = a + 1; k < e; ++k) {
            const int c = oc[k];
            const double v = ov[k];
            long long m = k - 1;
            while (m >= a && oc[m] > c) {
                oc[m + 1] = oc[m];
                ov[m + 1] = ov[m];
                --m;
            }
            oc[m + 1] = c;
            ov[m + 1] = v;
        }
        int cnt = 0;
        for (long long k = a; k < e; ++k) {
            if (k > a && oc[k] == oc[k - 1]) atomicOr(err, E_DUP);
            cnt += ov[k] != 0.0 ? 1 : 0;
        }
        nz[r] = cnt;
    }
}

// the entries that are not 0.0, into the final rows
__global__ void k_compact(int n, const long long* __restrict__ off, const long long* __restrict__ noff,
                          const int* __restrict__ oc, const double* __restrict__ ov, int* __restrict__ rp_out,
                          int* __restrict__ c_out, double* __restrict__ v_out)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        long long w = noff[r];
        rp_out[r] = (int)w;
        for (long long k = off[r]; k < off[r + 1]; ++k)
            if (ov[k] != 0.0) {
                c_out[w] = oc[k];
                v_out[w] = ov[k];
                ++w;
            }
        if (r == n - 1) rp_out[n] = (int)w;
    }
}

// exclusive scan of m counts into out[0..m] (out[m] = total)
static long long scan(const int* cnt, long long* out, int m, long long* counter, cudaStream_t st)
{
    const int tiles = (m + kScanTile - 1) / kScanTile;
    Buf<long long> ts;
    ts.alloc((size_t)std::max(1, tiles), counter);
    k_scan_tile<<<std::max(1, tiles), kThreads, 0, st>>>(m, cnt, out, ts.get());
    CK(cudaGetLastError());
    std::vector<long long> h((size_t)std::max(1, tiles));
    CK(cudaMemcpyAsync(h.data(), ts.get(), sizeof(long long) * h.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    long long run = 0;
    for (auto& v : h) {
        const long long t = v;
        v = run;
        run += t;
    }
    CK(cudaMemcpyAsync(ts.get(), h.data(), sizeof(long long) * h.size(), cudaMemcpyHostToDevice, st));
    k_scan_add<<<std::max(1, std::min(tiles * 4, 4096)), kThreads, 0, st>>>(m, out, ts.get());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out + m, &run, sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return run;
}

// A_run into the caller's arrays; returns 1 if the device computed it, 0 if
// the host routines did (repeated pairs or very long rows)
static int run(int device, int n, const int* rowptr, const int* colind, const double* val, const int* p, int cap,
               int* rp_out, int* c_out, double* v_out, int* nnz_out)
{
    check_crs(n, rowptr, colind, val);
    if (n > 0 && !p) throw Error(ICCG_ERR_ARG, "null new_of_old");
    if (!rp_out || !nnz_out || (cap > 0 && (!c_out || !v_out))) throw Error(ICCG_ERR_ARG, "null output");
    auto host = [&]() {
        CRS L = permute_ptap_lower(n, rowptr, colind, val, p);
        CRS F = expand_lower_to_full(L);
        *nnz_out = F.nnz();
        if (F.nnz() > cap) throw Error(ICCG_ERR_ARG, "output capacity too small");
        copy_out(F, rp_out, c_out, v_out);
        return 0;
    };
    if (n == 0) return host();
    int prev = 0;
    CK(cudaGetDevice(&prev));
    CK(cudaSetDevice(device));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    cudaStream_t st = nullptr;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard()
        {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    long long counter = 0;
    const long long nnz = rowptr[n];
    Buf<int> drp, dci, dp, cnt, cur, err, seen, nz;
    Buf<double> dval;
    drp.upload(rowptr, (size_t)n + 1, &counter, st);
    dci.upload(colind, (size_t)std::max(1ll, nnz), &counter, st);
    dval.upload(val, (size_t)std::max(1ll, nnz), &counter, st);
    dp.upload(p, (size_t)n, &counter, st);
    cnt.alloc((size_t)n, &counter);
    seen.alloc((size_t)n, &counter);
    err.alloc(1, &counter);
    CK(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * (size_t)n, st));
    CK(cudaMemsetAsync(seen.get(), 0, sizeof(int) * (size_t)n, st));
    CK(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    const int grid = std::max(1, std::min((n + kThreads - 1) / kThreads, 148 * 16));
    k_check_perm<<<grid, kThreads, 0, st>>>(n, dp.get(), seen.get(), err.get());
    k_count<<<grid, kThreads, 0, st>>>(n, drp.get(), dci.get(), dp.get(), cnt.get(), err.get());
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr & E_RANGE) throw Error(ICCG_ERR_ARG, "column index out of range");
    if (herr & E_PERM) throw Error(ICCG_ERR_ARG, "new_of_old is not a permutation");
    Buf<long long> off, noff;
    off.alloc((size_t)n + 1, &counter);
    const long long total = scan(cnt.get(), off.get(), n, &counter, st);
    if (total > 2147483647LL) throw Error(ICCG_ERR_ARG, "expanded matrix exceeds int32 nnz");
    Buf<int> oc;
    Buf<double> ov;
    oc.alloc((size_t)std::max(1ll, total), &counter);
    ov.alloc((size_t)std::max(1ll, total), &counter);
    cur.alloc((size_t)n, &counter);
    // the write cursor of row r starts at off[r] (an int: total < 2^31)
    {
        std::vector<long long> ho((size_t)n + 1);
        CK(cudaMemcpyAsync(ho.data(), off.get(), sizeof(long long) * ho.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<int> hc((size_t)n);
        for (int r = 0; r < n; ++r) hc[(size_t)r] = (int)ho[(size_t)r];
        CK(cudaMemcpyAsync(cur.get(), hc.data(), sizeof(int) * hc.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    k_scatter<<<grid, kThreads, 0, st>>>(n, drp.get(), dci.get(), dval.get(), dp.get(), cur.get(), oc.get(), ov.get());
    nz.alloc((size_t)n, &counter);
    k_sort_rows<<<grid, kThreads, 0, st>>>(n, off.get(), oc.get(), ov.get(), nz.get(), err.get());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr & (E_DUP | E_LONG)) return host();
    noff.alloc((size_t)n + 1, &counter);
    const long long kept = scan(nz.get(), noff.get(), n, &counter, st);
    *nnz_out = (int)kept;
    if (kept > cap) throw Error(ICCG_ERR_ARG, "output capacity too small");
    Buf<int> frp, fc;
    Buf<double> fv;
    frp.alloc((size_t)n + 1, &counter);
    fc.alloc((size_t)std::max(1ll, kept), &counter);
    fv.alloc((size_t)std::max(1ll, kept), &counter);
    k_compact<<<grid, kThreads, 0, st>>>(n, off.get(), noff.get(), oc.get(), ov.get(), frp.get(), fc.get(), fv.get());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rp_out, frp.get(), sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
    if (kept > 0) {
        CK(cudaMemcpyAsync(c_out, fc.get(), sizeof(int) * (size_t)kept, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(v_out, fv.get(), sizeof(double) * (size_t)kept, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return 1;
}

}  // namespace ptap_dev
}  // namespace iccg

extern "C" {

int iccg_ptap_full_gpu(int device, int n, const int* rowptr, const int* colind, const double* val,
                       const int* new_of_old, int cap, int* out_rowptr, int* out_colind, double* out_val,
                       int* out_nnz, int* on_device)
{
    try {
        const int d = iccg::ptap_dev::run(device, n, rowptr, colind, val, new_of_old, cap, out_rowptr, out_colind,
                                          out_val, out_nnz);
        if (on_device) *on_device = d;
        return ICCG_OK;
    } catch (const iccg::Error& e) {
        iccg::g_host_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        iccg::g_host_err = "out of host memory";
        return ICCG_ERR_NOMEM;
    } catch (const std::exception& e) {
        iccg::g_host_err = e.what();
        return ICCG_ERR_ARG;
    }
}

}  // extern "C"
