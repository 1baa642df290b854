// ctx.cu -- device context, schedule plans, IC(0) build and the CG drivers
// behind the C ABI of include/iccg.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/iccg.h"
#include "host.hpp"
#include "kernels.cuh"

namespace iccg {

extern thread_local std::string g_host_err;  // host_capi.cpp

// ---------------------------------------------------------------------------
// small RAII device buffer with byte accounting
// ---------------------------------------------------------------------------
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    long long* counter = nullptr;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }
    void release()
    {
        if (p) {
            cudaFree(p);
            if (counter) *counter -= (long long)bytes;
        }
        p = nullptr;
        bytes = 0;
    }
};

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            throw Error(ICCG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

template <class T>
struct Buf {
    DevMem m;
    size_t n = 0;
    T* get() const { return (T*)m.p; }
    void alloc(size_t count, long long* counter)
    {
        if (count == n && m.p) return;
        m.release();
        n = count;
        // pad every array by 16 elements so vectorised tails stay in bounds
        size_t bytes = (count + 16) * sizeof(T);
        cudaError_t e = cudaMalloc(&m.p, bytes);
        if (e != cudaSuccess) {
            m.p = nullptr;
            n = 0;
            cudaGetLastError();
            throw Error(ICCG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        m.bytes = bytes;
        m.counter = counter;
        *counter += (long long)bytes;
    }
    void upload(const T* h, size_t count, long long* counter, cudaStream_t s)
    {
        alloc(count, counter);
        if (count) CK(cudaMemcpyAsync(m.p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void free() { m.release(); n = 0; }
};

// A substitution / factorisation schedule: levels of independent units,
// each unit a sequence of rows done in order by one thread.
struct Plan {
    int nlevels = 0;
    std::vector<int> level_ptr;  // units per level (host)
    std::vector<int> grid;       // CTAs per level launch
    std::vector<int> slot0;      // first reduction slot of each launch
    int nslots = 0;
    bool unit_is_row = true;
    Buf<int> unit_ptr, rows;
    std::vector<int> h_unit_ptr, h_rows;
};

struct Factor {
    bool built = false;
    int nnzL = 0;
    double shift = 0.0;
    std::vector<int> Lp, Li, dpos, Up, Ui, ut_src, Sp, Si, s_src, Tp, Ti, t_src;
    Buf<int> dLp, dLi, ddpos;
    Buf<double> dLx;
    Buf<int> dSp, dSi, dTp, dTi;
    Buf<double> S64, T64, d64;
    Buf<float> S32, T32, d32;
    bool has32 = false;
    void reset()
    {
        built = false;
        has32 = false;
        nnzL = 0;
        shift = 0.0;
        for (auto* v : {&Lp, &Li, &dpos, &Up, &Ui, &ut_src, &Sp, &Si, &s_src, &Tp, &Ti, &t_src}) v->clear();
        for (auto* b : {&dLp, &dLi, &ddpos, &dSp, &dSi, &dTp, &dTi}) b->free();
        for (auto* b : {&dLx, &S64, &T64, &d64}) b->free();
        for (auto* b : {&S32, &T32, &d32}) b->free();
    }
};

constexpr int kThreads = 256;

// warp tiles of a contiguous schedule (see build_sweep_tiles)
struct SweepTiles {
    bool ok = false;
    int version = -1;
    int cap = 0, kx = 4, nlevels = 0, bnslots = 0;
    std::vector<int> ct_ptr, fgrid, bgrid, bslot0;
    Buf<WarpTile> wt;
};

}  // namespace iccg

using namespace iccg;

struct iccg_ctx {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    long long dev_bytes = 0;
    // matrix (A_run)
    int n = 0, nnz = 0;
    std::vector<int> h_rowptr, h_colind;
    std::vector<double> h_val;
    Buf<int> rowptr, colind;
    Buf<double> val64;
    Buf<float> val32;
    bool has_val32 = false;
    // schedule
    int sched_kind = ICCG_SCHED_NONE;
    int sched_version = 0;
    Plan fwd, bwd;
    bool plans_ready = false;
    // tiled kernels
    bool use_tiled = true;
    bool spmv_ok = false;
    int spmv_cap = 0, spmv_ntiles = 0;
    Buf<int> spmv_tiles;
    SweepTiles tl;
    // preconditioner
    int pc_kind = -1;
    Buf<double> inv_diag;
    Factor F;
    // vectors
    Buf<double> vb, vx, vr, vp, vz, vy, vAp, vtmp;
    // reductions / state
    Buf<dd> partials;
    Buf<unsigned int> ticket;
    Buf<double> scalars;
    Buf<SolverState> state;
    Buf<unsigned long long> errword;
    SolverState* h_state = nullptr;   // pinned
    double* h_scalars = nullptr;      // pinned
    int* h_status = nullptr;          // pinned, 2 slots
    size_t partial_slots = 0;
    // graph of the fused iteration
    cudaGraphExec_t gexec = nullptr;
    long long gkey = -1;
    int gkernels = 0;
    // events
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs[2] = {nullptr, nullptr};
    // profiling
    bool profile = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    size_t ev_used = 0;
    std::vector<int> ev_cls;
    double prof_ms[5] = {0, 0, 0, 0, 0};
    long long prof_n[5] = {0, 0, 0, 0, 0};
};

namespace iccg {

static int grid_for(const iccg_ctx* c, long long work, int threads = kThreads)
{
    long long g = (work + threads - 1) / threads;
    long long cap = (long long)c->nsm * (2048 / threads);
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

static void ensure_partials(iccg_ctx* c, size_t slots)
{
    if (slots <= c->partial_slots) return;
    c->partials.alloc(slots * 4, &c->dev_bytes);
    c->partial_slots = slots;
}

// dynamic shared memory above 48 KB needs an opt-in per kernel; set when the
// tiles are built, never while a graph is being captured
template <class K>
static void smem_optin(K kernel, size_t bytes)
{
    if (bytes > 48 * 1024) CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// launch wrapper: counts launches and, when profiling, brackets with events
template <class K, class... Args>
static void launch_smem(iccg_ctx* c, int cls, K kernel, int grid, int block, size_t smem, Args... args)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->profile) {
        if (c->ev_used == c->ev_pool.size()) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            c->ev_pool.emplace_back(a, b);
            c->ev_cls.push_back(0);
        }
        e0 = c->ev_pool[c->ev_used].first;
        e1 = c->ev_pool[c->ev_used].second;
        c->ev_cls[c->ev_used] = cls;
        ++c->ev_used;
        CK(cudaEventRecord(e0, c->stream));
    }
    kernel<<<grid, block, smem, c->stream>>>(args...);
    CK(cudaGetLastError());
    if (c->profile) CK(cudaEventRecord(e1, c->stream));
    c->launches++;
}

template <class K, class... Args>
static void launch(iccg_ctx* c, int cls, K kernel, int grid, int block, Args... args)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->profile) {
        if (c->ev_used == c->ev_pool.size()) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            c->ev_pool.emplace_back(a, b);
            c->ev_cls.push_back(0);
        }
        e0 = c->ev_pool[c->ev_used].first;
        e1 = c->ev_pool[c->ev_used].second;
        c->ev_cls[c->ev_used] = cls;
        ++c->ev_used;
        CK(cudaEventRecord(e0, c->stream));
    }
    kernel<<<grid, block, 0, c->stream>>>(args...);
    CK(cudaGetLastError());
    if (c->profile) CK(cudaEventRecord(e1, c->stream));
    c->launches++;
}

static void collect_profile(iccg_ctx* c)
{
    if (!c->profile) return;
    CK(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < c->ev_used; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev_pool[k].first, c->ev_pool[k].second));
        c->prof_ms[c->ev_cls[k]] += ms;
        c->prof_n[c->ev_cls[k]] += 1;
    }
    c->ev_used = 0;
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------
static void finalize_plan(iccg_ctx* c, Plan& P)
{
    P.nlevels = (int)P.level_ptr.size() - 1;
    P.grid.assign((size_t)P.nlevels, 0);
    P.slot0.assign((size_t)P.nlevels, 0);
    int s = 0;
    for (int l = 0; l < P.nlevels; ++l) {
        const int units = P.level_ptr[(size_t)l + 1] - P.level_ptr[(size_t)l];
        P.grid[(size_t)l] = grid_for(c, units);
        P.slot0[(size_t)l] = s;
        s += P.grid[(size_t)l];
    }
    P.nslots = s;
    if (!P.unit_is_row) P.unit_ptr.upload(P.h_unit_ptr.data(), P.h_unit_ptr.size(), &c->dev_bytes, c->stream);
    else P.unit_ptr.free();
    P.rows.upload(P.h_rows.data(), P.h_rows.size(), &c->dev_bytes, c->stream);
    ensure_partials(c, (size_t)std::max(P.nslots, 1));
}

// Dependency check of a forward plan against the lower pattern of A_run:
// every j < i in row i must be finished before row i starts.
static void check_plan(iccg_ctx* c, const Plan& P)
{
    const int n = c->n;
    std::vector<int> lev((size_t)n, -1), unit((size_t)n, -1), pos((size_t)n, -1);
    for (int l = 0; l < P.nlevels; ++l)
        for (int u = P.level_ptr[(size_t)l]; u < P.level_ptr[(size_t)l + 1]; ++u) {
            const int t0 = P.unit_is_row ? u : P.h_unit_ptr[(size_t)u];
            const int t1 = P.unit_is_row ? u + 1 : P.h_unit_ptr[(size_t)u + 1];
            for (int t = t0; t < t1; ++t) {
                const int i = P.h_rows[(size_t)t];
                if (i < 0 || i >= n) throw Error(ICCG_ERR_SCHEDULE, "schedule row out of range");
                if (lev[(size_t)i] >= 0)
                    throw Error(ICCG_ERR_SCHEDULE, "row " + std::to_string(i) + " appears twice in the schedule");
                lev[(size_t)i] = l;
                unit[(size_t)i] = u;
                pos[(size_t)i] = t;
            }
        }
    for (int i = 0; i < n; ++i)
        if (lev[(size_t)i] < 0) throw Error(ICCG_ERR_SCHEDULE, "row " + std::to_string(i) + " missing from the schedule");
    long long bad = 0;
    for (int i = 0; i < n; ++i)
        for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k) {
            const int j = c->h_colind[(size_t)k];
            if (j >= i) continue;
            const bool ok = lev[(size_t)j] < lev[(size_t)i] ||
                            (unit[(size_t)j] == unit[(size_t)i] && pos[(size_t)j] < pos[(size_t)i]);
            if (!ok) ++bad;
        }
    if (bad)
        throw Error(ICCG_ERR_SCHEDULE, "schedule has " + std::to_string(bad) +
                                           " dependencies (j<i) inside one color across units or on a later "
                                           "color; the parallel substitution would race");
}

static void build_plans_none(iccg_ctx* c)
{
    const int n = c->n;
    // forward level sets over the lower pattern
    std::vector<int> lev((size_t)n, 0);
    int nl = 0;
    for (int i = 0; i < n; ++i) {
        int l = 0;
        for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k) {
            const int j = c->h_colind[(size_t)k];
            if (j < i) l = std::max(l, lev[(size_t)j] + 1);
        }
        lev[(size_t)i] = l;
        nl = std::max(nl, l + 1);
    }
    auto bucket = [&](Plan& P, const std::vector<int>& L, int nlev) {
        P.unit_is_row = true;
        P.level_ptr.assign((size_t)nlev + 1, 0);
        for (int i = 0; i < n; ++i) P.level_ptr[(size_t)L[(size_t)i] + 1]++;
        for (int l = 0; l < nlev; ++l) P.level_ptr[(size_t)l + 1] += P.level_ptr[(size_t)l];
        P.h_rows.assign((size_t)n, 0);
        std::vector<int> cur(P.level_ptr.begin(), P.level_ptr.end() - 1);
        for (int i = 0; i < n; ++i) P.h_rows[(size_t)cur[(size_t)L[(size_t)i]]++] = i;
        P.h_unit_ptr.clear();
    };
    bucket(c->fwd, lev, n ? nl : 0);
    // backward level sets over the upper pattern (L^T rows)
    std::vector<int> levb((size_t)n, 0);
    int nlb = 0;
    for (int i = n - 1; i >= 0; --i) {
        int l = 0;
        for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k) {
            const int j = c->h_colind[(size_t)k];
            if (j > i) l = std::max(l, levb[(size_t)j] + 1);
        }
        levb[(size_t)i] = l;
        nlb = std::max(nlb, l + 1);
    }
    bucket(c->bwd, levb, n ? nlb : 0);
    finalize_plan(c, c->fwd);
    finalize_plan(c, c->bwd);
}

static void build_plans_mc(iccg_ctx* c, int nc, const int* color_ptr, const int* rows_of_color)
{
    const int n = c->n;
    if (nc <= 0 || !color_ptr || !rows_of_color) throw Error(ICCG_ERR_ARG, "bad MC schedule");
    for (int k = 0; k < nc; ++k)
        if (color_ptr[k] > color_ptr[k + 1] || color_ptr[k] < 0 || color_ptr[k + 1] > n)
            throw Error(ICCG_ERR_SCHEDULE, "color_ptr is not a nondecreasing range in [0, n]");
    Plan& F = c->fwd;
    F.unit_is_row = true;
    F.level_ptr.clear();
    F.h_rows.clear();
    F.level_ptr.push_back(0);
    for (int k = 0; k < nc; ++k) {
        for (int t = color_ptr[k]; t < color_ptr[k + 1]; ++t) F.h_rows.push_back(rows_of_color[t]);
        F.level_ptr.push_back((int)F.h_rows.size());
    }
    F.nlevels = nc;
    check_plan(c, F);
    Plan& B = c->bwd;
    B.unit_is_row = true;
    B.level_ptr.clear();
    B.h_rows.clear();
    B.level_ptr.push_back(0);
    for (int k = nc - 1; k >= 0; --k) {
        for (int t = color_ptr[k]; t < color_ptr[k + 1]; ++t) B.h_rows.push_back(rows_of_color[t]);
        B.level_ptr.push_back((int)B.h_rows.size());
    }
    finalize_plan(c, F);
    finalize_plan(c, B);
}

static void build_plans_abmc(iccg_ctx* c, int nc, int nb, const int* color_ptr_blk, const int* blocks_of_color,
                             const int* block_ptr, const int* rows_of_block)
{
    const int n = c->n;
    if (nc <= 0 || nb <= 0 || !color_ptr_blk || !blocks_of_color || !block_ptr || !rows_of_block)
        throw Error(ICCG_ERR_ARG, "bad ABMC schedule");
    for (int k = 0; k < nc; ++k)
        if (color_ptr_blk[k] > color_ptr_blk[k + 1] || color_ptr_blk[k] < 0 || color_ptr_blk[k + 1] > nb)
            throw Error(ICCG_ERR_SCHEDULE, "color_ptr_blk is not a nondecreasing range in [0, nb]");
    Plan& F = c->fwd;
    Plan& B = c->bwd;
    for (Plan* P : {&F, &B}) {
        P->unit_is_row = false;
        P->level_ptr.assign(1, 0);
        P->h_unit_ptr.assign(1, 0);
        P->h_rows.clear();
    }
    auto add_color = [&](Plan& P, int k, bool reverse) {
        for (int kb = color_ptr_blk[k]; kb < color_ptr_blk[k + 1]; ++kb) {
            const int b = blocks_of_color[kb];
            if (b < 0 || b >= nb) throw Error(ICCG_ERR_SCHEDULE, "blocks_of_color entry out of range");
            const int s = block_ptr[b], e = block_ptr[b + 1];
            if (s < 0 || e > n || s > e) throw Error(ICCG_ERR_SCHEDULE, "block_ptr out of range");
            if (!reverse) for (int t = s; t < e; ++t) P.h_rows.push_back(rows_of_block[t]);
            else for (int t = e - 1; t >= s; --t) P.h_rows.push_back(rows_of_block[t]);
            P.h_unit_ptr.push_back((int)P.h_rows.size());
        }
        P.level_ptr.push_back((int)P.h_unit_ptr.size() - 1);
    };
    for (int k = 0; k < nc; ++k) add_color(F, k, false);
    for (int k = nc - 1; k >= 0; --k) add_color(B, k, true);
    F.nlevels = nc;
    check_plan(c, F);
    finalize_plan(c, F);
    finalize_plan(c, B);
}

// ---------------------------------------------------------------------------
// IC(0) on the device
// ---------------------------------------------------------------------------
static void build_factor_pattern(iccg_ctx* c)
{
    Factor& F = c->F;
    const int n = c->n;
    // extract_lower_with_diag (ic0.cpp:14-38) and diag_pos (ic0.cpp:47-54)
    F.Lp.assign((size_t)n + 1, 0);
    F.Li.clear();
    std::vector<int> src;
    for (int i = 0; i < n; ++i) {
        F.Lp[(size_t)i] = (int)F.Li.size();
        for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k)
            if (c->h_colind[(size_t)k] <= i) { F.Li.push_back(c->h_colind[(size_t)k]); src.push_back(k); }
    }
    F.Lp[(size_t)n] = (int)F.Li.size();
    F.nnzL = (int)F.Li.size();
    F.dpos.assign((size_t)n, -1);
    for (int i = 0; i < n; ++i) {
        for (int k = F.Lp[(size_t)i]; k < F.Lp[(size_t)i + 1]; ++k)
            if (F.Li[(size_t)k] == i) { F.dpos[(size_t)i] = k; break; }
        if (F.dpos[(size_t)i] < 0)
            throw Error(ICCG_ERR_DIAG, "IC(0): diagonal missing at row " + std::to_string(i));
    }
    // CSC of L (build_csc_from_crs, ic0.cpp:118-151)
    F.Up.assign((size_t)n + 1, 0);
    for (int k = 0; k < F.nnzL; ++k) F.Up[(size_t)F.Li[(size_t)k] + 1]++;
    for (int i = 0; i < n; ++i) F.Up[(size_t)i + 1] += F.Up[(size_t)i];
    F.Ui.assign((size_t)F.nnzL, 0);
    F.ut_src.assign((size_t)F.nnzL, 0);
    {
        std::vector<int> cur(F.Up.begin(), F.Up.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = F.Lp[(size_t)i]; k < F.Lp[(size_t)i + 1]; ++k) {
                const int pos = cur[(size_t)F.Li[(size_t)k]]++;
                F.Ui[(size_t)pos] = i;
                F.ut_src[(size_t)pos] = k;
            }
    }
    // sweep layout: strict lower part of L rows, strict upper part of L^T rows
    F.Sp.assign((size_t)n + 1, 0);
    F.Si.clear();
    F.s_src.clear();
    for (int i = 0; i < n; ++i) {
        F.Sp[(size_t)i] = (int)F.Si.size();
        for (int k = F.Lp[(size_t)i]; k < F.Lp[(size_t)i + 1]; ++k) {
            const int j = F.Li[(size_t)k];
            if (j < i) { F.Si.push_back(j); F.s_src.push_back(k); }
            else break;
        }
    }
    F.Sp[(size_t)n] = (int)F.Si.size();
    F.Tp.assign((size_t)n + 1, 0);
    F.Ti.clear();
    F.t_src.clear();
    for (int i = 0; i < n; ++i) {
        F.Tp[(size_t)i] = (int)F.Ti.size();
        for (int k = F.Up[(size_t)i]; k < F.Up[(size_t)i + 1]; ++k) {
            const int j = F.Ui[(size_t)k];
            if (j > i) { F.Ti.push_back(j); F.t_src.push_back(F.ut_src[(size_t)k]); }
        }
    }
    F.Tp[(size_t)n] = (int)F.Ti.size();
    // initial values of L = lower part of A (ic0.cpp:42-44)
    std::vector<double> Lx0((size_t)F.nnzL);
    for (size_t k = 0; k < src.size(); ++k) Lx0[k] = c->h_val[(size_t)src[k]];
    F.dLp.upload(F.Lp.data(), F.Lp.size(), &c->dev_bytes, c->stream);
    F.dLi.upload(F.Li.data(), F.Li.size(), &c->dev_bytes, c->stream);
    F.ddpos.upload(F.dpos.data(), F.dpos.size(), &c->dev_bytes, c->stream);
    F.dLx.upload(Lx0.data(), Lx0.size(), &c->dev_bytes, c->stream);
    CK(cudaStreamSynchronize(c->stream));
}

static unsigned long long factor_once(iccg_ctx* c, double shift)
{
    Factor& F = c->F;
    const Plan& P = c->fwd;
    const unsigned long long none = ~0ull;
    CK(cudaMemcpyAsync(c->errword.get(), &none, sizeof(none), cudaMemcpyHostToDevice, c->stream));
    for (int l = 0; l < P.nlevels; ++l) {
        const int u0 = P.level_ptr[(size_t)l], u1 = P.level_ptr[(size_t)l + 1];
        if (u1 <= u0) continue;
        launch(c, 3, k_ic0_level, grid_for(c, u1 - u0, 128), 128, u0, u1,
               (const int*)(P.unit_is_row ? nullptr : P.unit_ptr.get()), (const int*)P.rows.get(),
               (const int*)F.dLp.get(), (const int*)F.dLi.get(), F.dLx.get(), (const int*)F.ddpos.get(), shift,
               c->errword.get());
    }
    unsigned long long w = none;
    CK(cudaMemcpyAsync(&w, c->errword.get(), sizeof(w), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return w;
}

static void build_ic0(iccg_ctx* c, double shift, bool auto_shift)
{
    Factor& F = c->F;
    F.built = false;
    F.has32 = false;
    build_factor_pattern(c);
    std::vector<double> Lx0((size_t)F.nnzL);
    CK(cudaMemcpyAsync(Lx0.data(), F.dLx.get(), sizeof(double) * Lx0.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double max_aii = 0.0;
    for (int i = 0; i < c->n; ++i) max_aii = std::max(max_aii, std::fabs(Lx0[(size_t)F.dpos[(size_t)i]]));
    double s = shift;
    for (int attempt = 0;; ++attempt) {
        unsigned long long w = factor_once(c, s);
        if (w == ~0ull) break;
        const int row = (int)(w >> 34);
        const int code = (int)((w >> 32) & 3ull);
        const int rep = (int)(w & 0xffffffffull);
        // shifted IC(0): restart with shift = max(2 shift, 1e-3 max|a_ii|),
        // doubling up to 40 times (covers shifts up to ~1e9 max|a_ii|)
        if (code == 2 && auto_shift && attempt < 40) {
            s = std::max(2.0 * s, 1e-3 * max_aii);
            if (!(s > 0.0)) s = 1e-3;
            CK(cudaMemcpyAsync(F.dLx.get(), Lx0.data(), sizeof(double) * Lx0.size(), cudaMemcpyHostToDevice,
                               c->stream));
            continue;
        }
        (void)row;
        if (code == 1)
            throw Error(ICCG_ERR_PIVOT_ZERO, "IC(0): zero/near-zero pivot at row " + std::to_string(rep));
        throw Error(ICCG_ERR_PIVOT_NONPOS, "IC(0): non-positive pivot at row " + std::to_string(rep));
    }
    F.shift = s;
    // sweep arrays
    std::vector<int> dsrc(F.dpos);
    F.dSp.upload(F.Sp.data(), F.Sp.size(), &c->dev_bytes, c->stream);
    F.dSi.upload(F.Si.data(), F.Si.size(), &c->dev_bytes, c->stream);
    F.dTp.upload(F.Tp.data(), F.Tp.size(), &c->dev_bytes, c->stream);
    F.dTi.upload(F.Ti.data(), F.Ti.size(), &c->dev_bytes, c->stream);
    Buf<int> idx;
    auto gather = [&](const std::vector<int>& src, Buf<double>& out) {
        idx.upload(src.data(), src.size(), &c->dev_bytes, c->stream);
        out.alloc(src.size(), &c->dev_bytes);
        if (!src.empty())
            launch(c, 3, k_gather<double>, grid_for(c, (long long)src.size()), kThreads, (long long)src.size(),
                   (const int*)idx.get(), (const double*)F.dLx.get(), out.get());
        CK(cudaStreamSynchronize(c->stream));
    };
    gather(F.s_src, F.S64);
    gather(F.t_src, F.T64);
    gather(dsrc, F.d64);
    idx.free();
    CK(cudaStreamSynchronize(c->stream));
    F.built = true;
}

static void ensure_factor32(iccg_ctx* c)
{
    Factor& F = c->F;
    if (F.has32) return;
    auto conv = [&](const Buf<double>& a, Buf<float>& b) {
        b.alloc(a.n, &c->dev_bytes);
        if (a.n) launch(c, 3, k_to_f32, grid_for(c, (long long)a.n), kThreads, (long long)a.n, (const double*)a.get(), b.get());
    };
    conv(F.S64, F.S32);
    conv(F.T64, F.T32);
    conv(F.d64, F.d32);
    CK(cudaStreamSynchronize(c->stream));
    F.has32 = true;
}

static void ensure_val32(iccg_ctx* c)
{
    if (c->has_val32) return;
    c->val32.alloc((size_t)c->nnz, &c->dev_bytes);
    if (c->nnz) launch(c, 3, k_to_f32, grid_for(c, c->nnz), kThreads, (long long)c->nnz, (const double*)c->val64.get(), c->val32.get());
    CK(cudaStreamSynchronize(c->stream));
    c->has_val32 = true;
}

static void require_matrix(iccg_ctx* c)
{
    if (c->n <= 0 && c->h_rowptr.empty()) throw Error(ICCG_ERR_STATE, "no matrix uploaded");
}

static void require_precond(iccg_ctx* c)
{
    require_matrix(c);
    if (c->pc_kind < 0) throw Error(ICCG_ERR_STATE, "preconditioner not built");
    if (c->pc_kind == ICCG_PRECOND_IC0 && !c->F.built) throw Error(ICCG_ERR_STATE, "IC(0) factor not built");
}

// ---------------------------------------------------------------------------
// preconditioner apply: z = M^{-1} r  (IC0::apply, ic0.cpp:366-393)
// ---------------------------------------------------------------------------
// Warp tiles for a contiguous schedule: every unit of the forward plan is a
// run of consecutive rows (at most 32) and the units of a level follow each
// other.  MC plans with ascending rows per color and ABMC plans made by
// BuildPermutationByBlockColor + BuildABMCSchedule have this form.
static bool build_sweep_tiles(iccg_ctx* c)
{
    SweepTiles& T = c->tl;
    T.ok = false;
    const Plan& P = c->fwd;
    const Factor& F = c->F;
    if (!F.built || P.nlevels <= 0) return false;
    struct U { int r, m; };
    std::vector<std::vector<U>> lv((size_t)P.nlevels);
    for (int l = 0; l < P.nlevels; ++l) {
        int prev_end = -1;
        for (int u = P.level_ptr[(size_t)l]; u < P.level_ptr[(size_t)l + 1]; ++u) {
            const int t0 = P.unit_is_row ? u : P.h_unit_ptr[(size_t)u];
            const int t1 = P.unit_is_row ? u + 1 : P.h_unit_ptr[(size_t)u + 1];
            const int m = t1 - t0;
            if (m <= 0 || m > 32) return false;
            const int r = P.h_rows[(size_t)t0];
            for (int t = t0; t < t1; ++t)
                if (P.h_rows[(size_t)t] != r + (t - t0)) return false;
            if (prev_end >= 0 && r != prev_end) return false;
            prev_end = r + m;
            lv[(size_t)l].push_back({r, m});
        }
    }
    const std::vector<int>& Sp = F.Sp;
    const std::vector<int>& Tp = F.Tp;
    auto entries = [&](int a, int b) { return std::max(Sp[(size_t)b] - Sp[(size_t)a], Tp[(size_t)b] - Tp[(size_t)a]); };
    int cap = 1024;
    for (const auto& units : lv)
        for (const U& u : units) {
            // one full warp tile of such units must fit
            const int need = entries(u.r, u.r + u.m) * ((32 + u.m - 1) / u.m) + 8;
            while (cap < need && cap < 16384) cap *= 2;
        }
    for (const auto& units : lv)
        for (const U& u : units)
            if (entries(u.r, u.r + u.m) > cap - 4) return false;
    std::vector<WarpTile> wts;
    T.ct_ptr.assign(1, 0);
    for (int l = 0; l < P.nlevels; ++l) {
        std::vector<WarpTile> ws;
        int cta_r0 = lv[(size_t)l].empty() ? 0 : lv[(size_t)l][0].r;
        WarpTile cur{cta_r0, 0, 0u, 0};
        auto close_cta = [&](int end_row) {
            if (cur.nrows > 0) { ws.push_back(cur); }
            if (!ws.empty()) {
                while (ws.size() < 8) ws.push_back(WarpTile{end_row, 0, 0u, 0});
                wts.insert(wts.end(), ws.begin(), ws.end());
            }
            ws.clear();
            cur = WarpTile{end_row, 0, 0u, 0};
            cta_r0 = end_row;
        };
        for (const U& u : lv[(size_t)l]) {
            if (cur.nrows + u.m > 32) {
                ws.push_back(cur);
                cur = WarpTile{u.r, 0, 0u, 0};
                if (ws.size() == 8) close_cta(u.r);
            }
            if (entries(cta_r0, u.r + u.m) > cap - 4) close_cta(u.r);
            cur.mask |= 1u << cur.nrows;
            cur.nrows += u.m;
            cur.nsteps = std::max(cur.nsteps, u.m);
        }
        const int end_row = cur.row0 + cur.nrows;
        close_cta(end_row);
        T.ct_ptr.push_back((int)(wts.size() / 8));
    }
    // external (later-level) entries per backward row: register prefetch depth
    int maxx = 0;
    for (const auto& units : lv)
        for (const U& u : units)
            for (int i = u.r; i < u.r + u.m; ++i) {
                int cnt = 0;
                for (int k = Tp[(size_t)i]; k < Tp[(size_t)i + 1]; ++k)
                    if (F.Ti[(size_t)k] >= u.r + u.m) ++cnt;
                maxx = std::max(maxx, cnt);
            }
    T.kx = maxx <= 2 ? 2 : maxx <= 4 ? 4 : maxx <= 8 ? 8 : 16;
    T.cap = cap;
    {
        const size_t b32 = 256 * sizeof(double) + (size_t)cap * 8, b64 = 256 * sizeof(double) + (size_t)cap * 12;
        if (b64 > 200 * 1024) return false;
        smem_optin(k_sweep_tiled<float, true, 1, FIN_NONE>, b32);
        smem_optin(k_sweep_tiled<double, true, 1, FIN_NONE>, b64);
        auto bw = [&](auto k32a, auto k32b, auto k32c, auto k64a, auto k64b, auto k64c) {
            smem_optin(k32a, b32); smem_optin(k32b, b32); smem_optin(k32c, b32);
            smem_optin(k64a, b64); smem_optin(k64b, b64); smem_optin(k64c, b64);
        };
        switch (T.kx) {
#define ICCG_BW(KX) bw(k_sweep_tiled<float, false, KX, FIN_NONE>, k_sweep_tiled<float, false, KX, FIN_RZ0>, \
                       k_sweep_tiled<float, false, KX, FIN_RZ>, k_sweep_tiled<double, false, KX, FIN_NONE>, \
                       k_sweep_tiled<double, false, KX, FIN_RZ0>, k_sweep_tiled<double, false, KX, FIN_RZ>)
            case 2: ICCG_BW(2); break;
            case 4: ICCG_BW(4); break;
            case 8: ICCG_BW(8); break;
            default: ICCG_BW(16); break;
#undef ICCG_BW
        }
    }
    T.nlevels = P.nlevels;
    T.fgrid.assign((size_t)P.nlevels, 1);
    T.bgrid.assign((size_t)P.nlevels, 1);
    T.bslot0.assign((size_t)P.nlevels, 0);
    const int cta_cap = c->nsm * 8;
    for (int l = 0; l < P.nlevels; ++l) {
        const int nct = T.ct_ptr[(size_t)l + 1] - T.ct_ptr[(size_t)l];
        T.fgrid[(size_t)l] = std::max(1, std::min(nct, cta_cap));
        T.bgrid[(size_t)l] = T.fgrid[(size_t)l];
    }
    int s = 0;
    for (int l = P.nlevels - 1; l >= 0; --l) {
        T.bslot0[(size_t)l] = s;
        s += T.bgrid[(size_t)l];
    }
    T.bnslots = s;
    ensure_partials(c, (size_t)std::max(s, 1));
    T.wt.upload(wts.data(), wts.size(), &c->dev_bytes, c->stream);
    CK(cudaStreamSynchronize(c->stream));
    T.ok = true;
    return true;
}

static void ensure_sweep_tiles(iccg_ctx* c)
{
    if (c->tl.version == c->sched_version) return;
    build_sweep_tiles(c);
    c->tl.version = c->sched_version;
}

template <class T, int FIN>
static void apply_ic0_tiled(iccg_ctx* c, const double* r, double* y, double* z, SolverState* st)
{
    Factor& F = c->F;
    SweepTiles& TL = c->tl;
    const T* Sx = std::is_same<T, float>::value ? (const T*)(const void*)F.S32.get() : (const T*)(const void*)F.S64.get();
    const T* Tx = std::is_same<T, float>::value ? (const T*)(const void*)F.T32.get() : (const T*)(const void*)F.T64.get();
    const T* d = std::is_same<T, float>::value ? (const T*)(const void*)F.d32.get() : (const T*)(const void*)F.d64.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    const size_t smem = 256 * sizeof(double) + (size_t)TL.cap * (sizeof(T) + 4);
    const WarpTile* wt = TL.wt.get();
    for (int l = 0; l < TL.nlevels; ++l)
        launch_smem(c, 1, k_sweep_tiled<T, true, 1, FIN_NONE>, TL.fgrid[(size_t)l], kThreads, smem,
                    TL.ct_ptr[(size_t)l], TL.ct_ptr[(size_t)l + 1], wt, (const int*)F.dSp.get(),
                    (const int*)F.dSi.get(), Sx, d, TL.cap, r, y, (const double*)nullptr, 0, 0, st, red,
                    c->ticket.get());
    for (int l = TL.nlevels - 1; l >= 0; --l) {
        auto go = [&](auto kernel) {
            launch_smem(c, 2, kernel, TL.bgrid[(size_t)l], kThreads, smem, TL.ct_ptr[(size_t)l],
                        TL.ct_ptr[(size_t)l + 1], wt, (const int*)F.dTp.get(), (const int*)F.dTi.get(), Tx, d,
                        TL.cap, (const double*)y, z, r, TL.bslot0[(size_t)l], TL.bnslots, st, red,
                        c->ticket.get());
        };
        switch (TL.kx) {
            case 2: go(k_sweep_tiled<T, false, 2, FIN>); break;
            case 4: go(k_sweep_tiled<T, false, 4, FIN>); break;
            case 8: go(k_sweep_tiled<T, false, 8, FIN>); break;
            default: go(k_sweep_tiled<T, false, 16, FIN>); break;
        }
    }
}

template <class T, int FIN>
static void apply_ic0(iccg_ctx* c, const double* r, double* y, double* z, SolverState* st)
{
    ensure_sweep_tiles(c);
    if (c->tl.ok && c->use_tiled) {
        apply_ic0_tiled<T, FIN>(c, r, y, z, st);
        return;
    }
    Factor& F = c->F;
    const void* Sx = std::is_same<T, float>::value ? (const void*)F.S32.get() : (const void*)F.S64.get();
    const void* Tx = std::is_same<T, float>::value ? (const void*)F.T32.get() : (const void*)F.T64.get();
    const void* d = std::is_same<T, float>::value ? (const void*)F.d32.get() : (const void*)F.d64.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    SweepArgs a{};
    a.unit_ptr = c->fwd.unit_is_row ? nullptr : c->fwd.unit_ptr.get();
    a.rows = c->fwd.rows.get();
    a.Sp = F.dSp.get();
    a.Si = F.dSi.get();
    a.Sx = Sx;
    a.d = d;
    a.in = r;
    a.out = y;
    for (int l = 0; l < c->fwd.nlevels; ++l) {
        const int u0 = c->fwd.level_ptr[(size_t)l], u1 = c->fwd.level_ptr[(size_t)l + 1];
        launch(c, 1, k_sweep<T, FIN_NONE>, c->fwd.grid[(size_t)l], kThreads, a, u0, u1, 0, 0, st, red,
               c->ticket.get());
    }
    SweepArgs b = a;
    b.unit_ptr = c->bwd.unit_is_row ? nullptr : c->bwd.unit_ptr.get();
    b.rows = c->bwd.rows.get();
    b.Sp = F.dTp.get();
    b.Si = F.dTi.get();
    b.Sx = Tx;
    b.in = y;
    b.out = z;
    b.rdot = r;
    for (int l = 0; l < c->bwd.nlevels; ++l) {
        const int u0 = c->bwd.level_ptr[(size_t)l], u1 = c->bwd.level_ptr[(size_t)l + 1];
        launch(c, 2, k_sweep<T, FIN>, c->bwd.grid[(size_t)l], kThreads, b, u0, u1, c->bwd.slot0[(size_t)l],
               c->bwd.nslots, st, red, c->ticket.get());
    }
}

template <int FIN>
static void apply_pc(iccg_ctx* c, int storage, const double* r, double* z, SolverState* st)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    if (c->pc_kind == ICCG_PRECOND_IC0) {
        if (storage == ICCG_STORE_FP32) apply_ic0<float, FIN>(c, r, c->vy.get(), z, st);
        else apply_ic0<double, FIN>(c, r, c->vy.get(), z, st);
        return;
    }
    const double* inv = c->pc_kind == ICCG_PRECOND_JACOBI ? c->inv_diag.get() : nullptr;
    launch(c, 3, k_diag_apply<FIN>, grid_for(c, c->n), kThreads, c->n, inv, r, z, st, red, c->ticket.get());
}

// CTA tiles of the SpMV: at most 256 rows and cap - 4 entries each.
static void build_spmv_tiles(iccg_ctx* c)
{
    c->spmv_ok = false;
    const int n = c->n;
    int maxrow = 0;
    for (int i = 0; i < n; ++i) maxrow = std::max(maxrow, c->h_rowptr[(size_t)i + 1] - c->h_rowptr[(size_t)i]);
    const double avg = n ? (double)c->nnz / n : 0.0;
    int cap = (int)std::ceil(256.0 * avg * 1.15 / 256.0) * 256;
    cap = std::max(cap, 1024);
    while (cap - 4 < maxrow && cap < 16384) cap *= 2;
    if (cap - 4 < maxrow) return;  // very long rows: the untiled kernel
    std::vector<int> tr(1, 0);
    int r0 = 0;
    for (int i = 0; i < n; ++i) {
        const int rows = i + 1 - r0;
        const int ent = c->h_rowptr[(size_t)i + 1] - c->h_rowptr[(size_t)r0];
        if (rows > 256 || ent > cap - 4) {
            tr.push_back(i);
            r0 = i;
        }
    }
    tr.push_back(n);
    if ((size_t)cap * 12 > 200 * 1024) return;
    smem_optin(k_spmv_tiled<float, FIN_NONE>, (size_t)cap * 8);
    smem_optin(k_spmv_tiled<float, FIN_PAP>, (size_t)cap * 8);
    smem_optin(k_spmv_tiled<double, FIN_NONE>, (size_t)cap * 12);
    smem_optin(k_spmv_tiled<double, FIN_PAP>, (size_t)cap * 12);
    c->spmv_cap = cap;
    c->spmv_ntiles = (int)tr.size() - 1;
    c->spmv_tiles.upload(tr.data(), tr.size(), &c->dev_bytes, c->stream);
    c->spmv_ok = true;
}

template <int FIN>
static void spmv_launch(iccg_ctx* c, int storage, const double* x, double* y, SolverState* st)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    const int* rp = c->rowptr.get();
    const int* ci = c->colind.get();
    if (c->spmv_ok && c->use_tiled) {
        const int g = std::min(c->spmv_ntiles, c->nsm * 8);
        if (storage == ICCG_STORE_FP32)
            launch_smem(c, 0, k_spmv_tiled<float, FIN>, g, kThreads, (size_t)c->spmv_cap * 8, c->spmv_ntiles,
                        (const int*)c->spmv_tiles.get(), rp, ci, (const float*)c->val32.get(), c->spmv_cap, x, y, st,
                        red, c->ticket.get());
        else
            launch_smem(c, 0, k_spmv_tiled<double, FIN>, g, kThreads, (size_t)c->spmv_cap * 12, c->spmv_ntiles,
                        (const int*)c->spmv_tiles.get(), rp, ci, (const double*)c->val64.get(), c->spmv_cap, x, y,
                        st, red, c->ticket.get());
        return;
    }
    const int g = grid_for(c, c->n);
    if (storage == ICCG_STORE_FP32)
        launch(c, 0, k_spmv<float, FIN>, g, kThreads, c->n, rp, ci, (const float*)c->val32.get(), x, y, st, red,
               c->ticket.get());
    else
        launch(c, 0, k_spmv<double, FIN>, g, kThreads, c->n, rp, ci, (const double*)c->val64.get(), x, y, st, red,
               c->ticket.get());
}

static void spmv_dev(iccg_ctx* c, int storage, const double* x, double* y)
{
    if (storage == ICCG_STORE_FP32) ensure_val32(c);
    spmv_launch<FIN_NONE>(c, storage, x, y, nullptr);
}

static double dot_dev(iccg_ctx* c, int n, const double* a, const double* b)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    ensure_partials(c, (size_t)grid_for(c, n));
    red.partials = c->partials.get();
    launch(c, 3, k_dot, grid_for(c, n), kThreads, n, a, b, red, c->ticket.get());
    CK(cudaMemcpyAsync(c->h_scalars, c->scalars.get(), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return c->h_scalars[0];
}

// ---------------------------------------------------------------------------
// plain FP64 CG (cg_crs.cpp:89-162): one kernel per reference operation, the
// scalar logic on the host after reading each reduction back.
// ---------------------------------------------------------------------------
static void solve_plain(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, iccg_result* res)
{
    const int n = c->n;
    double* r = c->vr.get();
    double* p = c->vp.get();
    double* z = c->vz.get();
    double* Ap = c->vAp.get();
    double* Ax = c->vtmp.get();
    const int g = grid_for(c, n);
    spmv_dev(c, ICCG_STORE_FP64, x, Ax);
    launch(c, 3, k_sub, g, kThreads, n, b, (const double*)Ax, r);
    double normb = std::sqrt(dot_dev(c, n, b, b));
    if (normb == 0.0) normb = 1.0;
    apply_pc<FIN_NONE>(c, ICCG_STORE_FP64, r, z, nullptr);
    launch(c, 3, k_copy, g, kThreads, n, (const double*)z, p, (SolverState*)nullptr);
    double rz_old = dot_dev(c, n, r, z);
    res->iters = 0;
    res->converged = 0;
    res->status = kMaxIter;
    res->rel_resid = std::sqrt(dot_dev(c, n, r, r)) / normb;
    if (res->rel_resid < tol) {
        res->converged = 1;
        res->status = kConverged;
        return;
    }
    for (int k = 0; k < max_iter; ++k) {
        spmv_dev(c, ICCG_STORE_FP64, p, Ap);
        const double pAp = dot_dev(c, n, p, Ap);
        const double eps = 2.220446049250313080847e-16;
        const double thr = eps * std::sqrt(dot_dev(c, n, p, p)) * std::sqrt(dot_dev(c, n, Ap, Ap));
        if (pAp <= thr) {
            res->iters = k;
            res->status = kBreakdown;
            return;
        }
        const double alpha = rz_old / pAp;
        RedBuf red{c->partials.get(), c->scalars.get()};
        launch(c, 3, k_update<FIN_NONE>, g, kThreads, n, alpha, (const double*)p, (const double*)Ap, x, r,
               (SolverState*)nullptr, red, c->ticket.get());
        const double rel = std::sqrt(dot_dev(c, n, r, r)) / normb;
        res->iters = k + 1;
        res->rel_resid = rel;
        if (rel < tol) {
            res->converged = 1;
            res->status = kConverged;
            return;
        }
        apply_pc<FIN_NONE>(c, ICCG_STORE_FP64, r, z, nullptr);
        const double rz_new = dot_dev(c, n, r, z);
        const double beta = rz_new / rz_old;
        launch(c, 3, k_xpay, g, kThreads, n, beta, (const double*)z, p, (SolverState*)nullptr);
        rz_old = rz_new;
    }
    res->status = kMaxIter;
}

// ---------------------------------------------------------------------------
// fused CG: device-side scalars, graph-replayed iterations
// ---------------------------------------------------------------------------
template <class T>
static void fused_iteration(iccg_ctx* c, int storage, bool rr, const double* b, double* x)
{
    const int n = c->n;
    const int g = grid_for(c, n);
    SolverState* st = c->state.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    const T* Av = std::is_same<T, float>::value ? (const T*)c->val32.get() : (const T*)c->val64.get();
    (void)Av;
    spmv_launch<FIN_PAP>(c, storage, (const double*)c->vp.get(), c->vAp.get(), st);
    launch(c, 3, k_update<FIN_UPD>, g, kThreads, n, 0.0, (const double*)c->vp.get(), (const double*)c->vAp.get(), x,
           c->vr.get(), st, red, c->ticket.get());
    if (rr)
        launch(c, 4, k_residual<FIN_TRUE>, g, kThreads, n, (const int*)c->rowptr.get(), (const int*)c->colind.get(),
               (const double*)c->val64.get(), (const double*)x, b, c->vr.get(), st, red, c->ticket.get());
    apply_pc<FIN_RZ>(c, storage, c->vr.get(), c->vz.get(), st);
    launch(c, 3, k_xpay, g, kThreads, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st);
}

static void solve_fused(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, const iccg_solve_opts& o,
                        iccg_result* res)
{
    const int n = c->n;
    const int storage = o.storage;
    const bool rr = storage == ICCG_STORE_FP32 && o.rr_interval > 0;
    if (storage == ICCG_STORE_FP32) {
        ensure_val32(c);
        if (c->pc_kind == ICCG_PRECOND_IC0) ensure_factor32(c);
    }
    SolverState s0{};
    s0.tol = tol;
    s0.k = 0;
    s0.iters = 0;
    s0.status = kRunning;
    s0.max_iter = max_iter;
    s0.rr_interval = storage == ICCG_STORE_FP32 ? std::max(0, o.rr_interval) : 0;
    if (storage == ICCG_STORE_FP32 && s0.rr_interval == 0) s0.rr_interval = 0;
    *c->h_state = s0;
    CK(cudaMemcpyAsync(c->state.get(), c->h_state, sizeof(SolverState), cudaMemcpyHostToDevice, c->stream));
    unsigned int zero = 0;
    CK(cudaMemcpyAsync(c->ticket.get(), &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    const int g = grid_for(c, n);
    SolverState* st = c->state.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    // r0 = b - A x0, ||b||, z0 = M^{-1} r0, rz, p = z  (cg_crs.cpp:102-123)
    launch(c, 4, k_residual<FIN_INIT>, g, kThreads, n, (const int*)c->rowptr.get(), (const int*)c->colind.get(),
           (const double*)c->val64.get(), (const double*)x, b, c->vr.get(), st, red, c->ticket.get());
    apply_pc<FIN_RZ0>(c, storage, c->vr.get(), c->vz.get(), st);
    launch(c, 3, k_copy, g, kThreads, n, (const double*)c->vz.get(), c->vp.get(), st);

    const int m = std::max(1, o.graph_iters);
    const bool use_graph = !c->profile;
    auto one_batch = [&]() {
        for (int it = 0; it < m; ++it) {
            if (storage == ICCG_STORE_FP32) fused_iteration<float>(c, storage, rr, b, x);
            else fused_iteration<double>(c, storage, rr, b, x);
        }
    };
    if (use_graph) {
        const long long key = ((long long)c->sched_version << 24) ^ ((long long)storage << 20) ^
                              ((long long)rr << 19) ^ ((long long)m << 4) ^ (long long)c->pc_kind ^
                              ((long long)(uintptr_t)x << 32) ^ ((long long)(uintptr_t)b << 40);
        if (!c->gexec || c->gkey != key) {
            if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
            cudaGraph_t graph;
            const long long before = c->launches;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            try {
                one_batch();
            } catch (...) {
                cudaStreamEndCapture(c->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            CK(cudaStreamEndCapture(c->stream, &graph));
            CK(cudaGraphInstantiate(&c->gexec, graph, 0));
            cudaGraphDestroy(graph);
            c->gkernels = (int)(c->launches - before);
            c->launches = before;
            c->gkey = key;
        }
    }
    // launch batches; poll the status of batch i-1 while batch i runs
    for (int batch = 0;; ++batch) {
        if (use_graph) {
            CK(cudaGraphLaunch(c->gexec, c->stream));
            c->launches += c->gkernels;
        } else {
            one_batch();
        }
        CK(cudaMemcpyAsync(&c->h_status[batch & 1], &st->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaEventRecord(c->evs[batch & 1], c->stream));
        if (batch > 0) {
            CK(cudaEventSynchronize(c->evs[(batch - 1) & 1]));
            if (c->h_status[(batch - 1) & 1] != kRunning) break;
        }
        if ((long long)(batch + 1) * m > (long long)max_iter + m) {
            CK(cudaEventSynchronize(c->evs[batch & 1]));
            break;
        }
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaMemcpyAsync(c->h_state, st, sizeof(SolverState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const SolverState& sf = *c->h_state;
    res->iters = sf.iters;
    res->status = sf.status == kRunning ? kMaxIter : sf.status;
    res->converged = sf.status == kConverged ? 1 : 0;
    res->rel_resid = sf.rel_resid;
    res->n_replacements = sf.n_rr;
}

static double true_resid(iccg_ctx* c, const double* b, const double* x)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    launch(c, 4, k_residual<FIN_NONE>, grid_for(c, c->n), kThreads, c->n, (const int*)c->rowptr.get(),
           (const int*)c->colind.get(), (const double*)c->val64.get(), x, b, c->vtmp.get(), (SolverState*)nullptr,
           red, c->ticket.get());
    const double nr = dot_dev(c, c->n, c->vtmp.get(), c->vtmp.get());
    const double nb = dot_dev(c, c->n, b, b);
    return std::sqrt(nr) / std::sqrt(nb);
}

static void solve_dev(iccg_ctx* c, const double* b, double* x, int max_iter, double tol,
                      const iccg_solve_opts* opts, iccg_result* res)
{
    require_precond(c);
    iccg_solve_opts o{ICCG_MODE_FUSED, ICCG_STORE_FP64, 50, 8};
    if (opts) o = *opts;
    if (o.graph_iters <= 0) o.graph_iters = 8;
    if (o.mode == ICCG_MODE_PLAIN && o.storage != ICCG_STORE_FP64)
        throw Error(ICCG_ERR_ARG, "the plain path computes in FP64 storage only");
    std::memset(res, 0, sizeof(*res));
    if (o.mode == ICCG_MODE_PLAIN) {
        CK(cudaEventRecord(c->ev0, c->stream));
        solve_plain(c, b, x, max_iter, tol, res);
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    } else {
        solve_fused(c, b, x, max_iter, tol, o, res);
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    res->solve_ms = ms;
    collect_profile(c);
    // A converged FP32-storage solve ends on a residual replacement, whose
    // convergence test is already ||b - A x|| / ||b|| with the FP64 matrix.
    if (o.mode == ICCG_MODE_FUSED && o.storage == ICCG_STORE_FP32 && o.rr_interval > 0 && res->converged)
        res->true_rel_resid = res->rel_resid;
    else
        res->true_rel_resid = true_resid(c, b, x);
}

static void ensure_vectors(iccg_ctx* c)
{
    const size_t n = (size_t)c->n;
    for (Buf<double>* v : {&c->vb, &c->vx, &c->vr, &c->vp, &c->vz, &c->vy, &c->vAp, &c->vtmp}) v->alloc(n, &c->dev_bytes);
    ensure_partials(c, (size_t)grid_for(c, c->n));
}

template <class F>
static int guard(iccg_ctx* c, F&& f)
{
    if (!c) return ICCG_ERR_ARG;
    try {
        CK(cudaSetDevice(c->device));
        f();
        return ICCG_OK;
    } catch (const Error& e) {
        c->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        c->err = "out of host memory";
        return ICCG_ERR_NOMEM;
    } catch (const std::exception& e) {
        c->err = e.what();
        return ICCG_ERR_ARG;
    }
}

}  // namespace iccg

extern "C" {

int iccg_ctx_create(int device, iccg_ctx** out)
{
    if (!out) return ICCG_ERR_ARG;
    *out = nullptr;
    auto* c = new iccg_ctx;
    c->device = device;
    int rc = guard(c, [&] {
        int ndev = 0;
        CK(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw Error(ICCG_ERR_ARG, "no such CUDA device");
        CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        CK(cudaEventCreateWithFlags(&c->evs[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->evs[1], cudaEventDisableTiming));
        CK(cudaMallocHost(&c->h_state, sizeof(SolverState)));
        CK(cudaMallocHost(&c->h_scalars, 8 * sizeof(double)));
        CK(cudaMallocHost(&c->h_status, 2 * sizeof(int)));
        c->ticket.alloc(4, &c->dev_bytes);
        c->scalars.alloc(8, &c->dev_bytes);
        c->state.alloc(1, &c->dev_bytes);
        c->errword.alloc(1, &c->dev_bytes);
        CK(cudaMemsetAsync(c->ticket.get(), 0, 4 * sizeof(unsigned int), c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
    if (rc) {
        iccg::g_host_err = c->err;
        iccg_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return ICCG_OK;
}

int iccg_ctx_destroy(iccg_ctx* c)
{
    if (!c) return ICCG_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    for (auto& e : c->ev_pool) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto e : c->evs) if (e) cudaEventDestroy(e);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    if (c->h_status) cudaFreeHost(c->h_status);
    cudaStream_t s = c->stream;
    delete c;  // buffers free themselves
    if (s) cudaStreamDestroy(s);
    return ICCG_OK;
}

const char* iccg_ctx_last_error(const iccg_ctx* c) { return c ? c->err.c_str() : "null context"; }
void* iccg_ctx_stream(iccg_ctx* c) { return c ? (void*)c->stream : nullptr; }
long long iccg_ctx_launch_count(const iccg_ctx* c) { return c ? c->launches : 0; }
long long iccg_ctx_device_bytes(const iccg_ctx* c) { return c ? c->dev_bytes : 0; }

int iccg_matrix_upload(iccg_ctx* c, int n, const int* rowptr, const int* colind, const double* val)
{
    return guard(c, [&] {
        if (n <= 0 || !rowptr || !colind || !val) throw Error(ICCG_ERR_ARG, "bad matrix arguments");
        if (rowptr[0] != 0) throw Error(ICCG_ERR_ARG, "rowptr[0] must be 0");
        for (int i = 0; i < n; ++i) {
            if (rowptr[i + 1] < rowptr[i]) throw Error(ICCG_ERR_ARG, "rowptr must be nondecreasing");
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
                if (colind[k] < 0 || colind[k] >= n) throw Error(ICCG_ERR_ARG, "column index out of range");
                if (k > rowptr[i] && colind[k] <= colind[k - 1])
                    throw Error(ICCG_ERR_ARG, "columns must be strictly ascending within each row");
            }
        }
        const int nnz = rowptr[n];
        c->n = n;
        c->nnz = nnz;
        c->h_rowptr.assign(rowptr, rowptr + n + 1);
        c->h_colind.assign(colind, colind + nnz);
        c->h_val.assign(val, val + nnz);
        c->rowptr.upload(rowptr, (size_t)n + 1, &c->dev_bytes, c->stream);
        c->colind.upload(colind, (size_t)nnz, &c->dev_bytes, c->stream);
        c->val64.upload(val, (size_t)nnz, &c->dev_bytes, c->stream);
        c->val32.free();
        c->has_val32 = false;
        ensure_vectors(c);
        build_spmv_tiles(c);
        // a new matrix invalidates the schedule and the preconditioner
        c->pc_kind = -1;
        c->F.reset();
        c->sched_kind = ICCG_SCHED_NONE;
        build_plans_none(c);
        c->sched_version++;
        if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_mc(iccg_ctx* c, int nc, const int* color_ptr, const int* rows_of_color)
{
    return guard(c, [&] {
        require_matrix(c);
        build_plans_mc(c, nc, color_ptr, rows_of_color);
        c->sched_kind = ICCG_SCHED_MC;
        c->sched_version++;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_abmc(iccg_ctx* c, int nc, int nb, const int* color_ptr_blk, const int* blocks_of_color,
                       const int* block_ptr, const int* rows_of_block)
{
    return guard(c, [&] {
        require_matrix(c);
        build_plans_abmc(c, nc, nb, color_ptr_blk, blocks_of_color, block_ptr, rows_of_block);
        c->sched_kind = ICCG_SCHED_ABMC;
        c->sched_version++;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_none(iccg_ctx* c)
{
    return guard(c, [&] {
        require_matrix(c);
        build_plans_none(c);
        c->sched_kind = ICCG_SCHED_NONE;
        c->sched_version++;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_precond_build(iccg_ctx* c, int kind, double shift, int auto_shift)
{
    return guard(c, [&] {
        require_matrix(c);
        c->pc_kind = -1;
        if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
        c->sched_version++;
        if (kind == ICCG_PRECOND_NONE) {
            c->inv_diag.free();
        } else if (kind == ICCG_PRECOND_JACOBI) {
            // Jacobi::Jacobi (precond.hpp:23-36)
            std::vector<double> inv((size_t)c->n, 1.0);
            for (int i = 0; i < c->n; ++i) {
                double d = 0.0;
                for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k)
                    if (c->h_colind[(size_t)k] == i) { d = c->h_val[(size_t)k]; break; }
                inv[(size_t)i] = (std::fabs(d) > 0.0) ? 1.0 / d : 1.0;
            }
            c->inv_diag.upload(inv.data(), inv.size(), &c->dev_bytes, c->stream);
            CK(cudaStreamSynchronize(c->stream));
        } else if (kind == ICCG_PRECOND_IC0) {
            build_ic0(c, shift, auto_shift != 0);
        } else {
            throw Error(ICCG_ERR_ARG, "unknown preconditioner kind");
        }
        c->pc_kind = kind;
    });
}

double iccg_precond_shift(const iccg_ctx* c) { return c ? c->F.shift : 0.0; }

int iccg_precond_apply_dev(iccg_ctx* c, const double* r, double* z, int storage)
{
    return guard(c, [&] {
        require_precond(c);
        if (storage == ICCG_STORE_FP32 && c->pc_kind == ICCG_PRECOND_IC0) ensure_factor32(c);
        apply_pc<FIN_NONE>(c, storage, r, z, nullptr);
        collect_profile(c);
    });
}

int iccg_precond_apply(iccg_ctx* c, const double* r, double* z, int storage)
{
    return guard(c, [&] {
        require_precond(c);
        if (storage == ICCG_STORE_FP32 && c->pc_kind == ICCG_PRECOND_IC0) ensure_factor32(c);
        CK(cudaMemcpyAsync(c->vb.get(), r, sizeof(double) * (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
        apply_pc<FIN_NONE>(c, storage, c->vb.get(), c->vtmp.get(), nullptr);
        CK(cudaMemcpyAsync(z, c->vtmp.get(), sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        collect_profile(c);
    });
}

int iccg_precond_nnz(const iccg_ctx* c, int* nnzL)
{
    if (!c || !nnzL) return ICCG_ERR_ARG;
    if (!c->F.built) return ICCG_ERR_STATE;
    *nnzL = c->F.nnzL;
    return ICCG_OK;
}

int iccg_precond_export(iccg_ctx* c, int* Lp, int* Li, double* Lx, int* Up, int* Ui, double* Ux)
{
    return guard(c, [&] {
        if (!c->F.built) throw Error(ICCG_ERR_STATE, "IC(0) factor not built");
        const Factor& F = c->F;
        std::vector<double> lx((size_t)F.nnzL);
        CK(cudaMemcpyAsync(lx.data(), F.dLx.get(), sizeof(double) * lx.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (Lp) std::memcpy(Lp, F.Lp.data(), sizeof(int) * F.Lp.size());
        if (Li) std::memcpy(Li, F.Li.data(), sizeof(int) * F.Li.size());
        if (Lx) std::memcpy(Lx, lx.data(), sizeof(double) * lx.size());
        if (Up) std::memcpy(Up, F.Up.data(), sizeof(int) * F.Up.size());
        if (Ui) std::memcpy(Ui, F.Ui.data(), sizeof(int) * F.Ui.size());
        if (Ux) for (size_t k = 0; k < F.ut_src.size(); ++k) Ux[k] = lx[(size_t)F.ut_src[k]];
    });
}

int iccg_spmv_dev(iccg_ctx* c, const double* x, double* y, int storage)
{
    return guard(c, [&] {
        require_matrix(c);
        spmv_dev(c, storage, x, y);
        CK(cudaStreamSynchronize(c->stream));
        collect_profile(c);
    });
}

int iccg_spmv(iccg_ctx* c, const double* x, double* y, int storage)
{
    return guard(c, [&] {
        require_matrix(c);
        CK(cudaMemcpyAsync(c->vb.get(), x, sizeof(double) * (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
        spmv_dev(c, storage, c->vb.get(), c->vtmp.get());
        CK(cudaMemcpyAsync(y, c->vtmp.get(), sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        collect_profile(c);
    });
}

int iccg_dot_dev(iccg_ctx* c, int n, const double* a, const double* b, double* out)
{
    return guard(c, [&] {
        if (n < 0 || !out) throw Error(ICCG_ERR_ARG, "bad dot arguments");
        *out = dot_dev(c, n, a, b);
    });
}

int iccg_solve_dev(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, const iccg_solve_opts* opts,
                   iccg_result* res)
{
    return guard(c, [&] {
        if (!b || !x || !res) throw Error(ICCG_ERR_ARG, "null argument");
        solve_dev(c, b, x, max_iter, tol, opts, res);
    });
}

int iccg_solve(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, const iccg_solve_opts* opts,
               iccg_result* res)
{
    return guard(c, [&] {
        if (!b || !x || !res) throw Error(ICCG_ERR_ARG, "null argument");
        require_precond(c);
        const size_t bytes = sizeof(double) * (size_t)c->n;
        CK(cudaMemcpyAsync(c->vb.get(), b, bytes, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->vx.get(), x, bytes, cudaMemcpyHostToDevice, c->stream));
        solve_dev(c, c->vb.get(), c->vx.get(), max_iter, tol, opts, res);
        CK(cudaMemcpyAsync(x, c->vx.get(), bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_ctx_set_option(iccg_ctx* c, int option, long long value)
{
    return guard(c, [&] {
        if (option == ICCG_OPT_TILED) {
            c->use_tiled = value != 0;
            c->sched_version++;  // re-capture graphs
        } else {
            throw Error(ICCG_ERR_ARG, "unknown option");
        }
    });
}

int iccg_profile_enable(iccg_ctx* c, int enable)
{
    return guard(c, [&] {
        c->profile = enable != 0;
        for (int k = 0; k < 5; ++k) { c->prof_ms[k] = 0.0; c->prof_n[k] = 0; }
    });
}

int iccg_profile_read(iccg_ctx* c, int cls, double* total_ms, long long* launches)
{
    if (!c || cls < 0 || cls >= 5) return ICCG_ERR_ARG;
    if (total_ms) *total_ms = c->prof_ms[cls];
    if (launches) *launches = c->prof_n[cls];
    return ICCG_OK;
}

}  // extern "C"
