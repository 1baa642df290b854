// context.hpp -- the device context behind iccg_ctx.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "devbuf.hpp"
#include "kernels.cuh"
#include "persist.cuh"

namespace iccg {

constexpr int kThreads = 256;

// A substitution / factorisation schedule in A_run row numbering: levels of
// independent units, each unit a sequence of rows done in order.
struct Plan {
    int nlevels = 0;
    std::vector<int> level_ptr;  // units per level (host)
    std::vector<int> grid;       // CTAs per level launch (simple kernels)
    std::vector<int> slot0;      // first reduction slot of each launch
    int nslots = 0;
    bool unit_is_row = true;
    Buf<int> unit_ptr, rows;
    std::vector<int> h_unit_ptr, h_rows;
};

// IC(0) factor in the reference's layout (L rows, A_run numbering) plus the
// strict-lower / strict-upper split used by the substitutions.
struct Factor : Ic0Layout {
    bool built = false;
    int nnzL = 0;
    double shift = 0.0;
    Buf<int> dLp, dLi, ddpos;
    Buf<double> dLx;
    // simple-path arrays (A_run numbering)
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

// A SELL-32 matrix over Q rows (see kernels.cuh, "Lane-interleaved kernels").
// The host arrays (SellLayout) keep h_ptr, src, prev_only and unit_only;
// h_col and h_len are released once they are on the device.
struct SellDev : SellLayout {
    Buf<int> ptr, col, len;
    Buf<double> v64;
    Buf<float> v32;
    Buf<int2> pk;          // FP32 values packed with their columns (the SpMV's matrix)
    bool has32 = false;
    bool haspk = false;
    SellMat view(bool fp32) const
    {
        return SellMat{ptr.get(), col.get(), fp32 ? (const void*)v32.get() : (const void*)v64.get(), len.get(),
                       fp32 && haspk ? pk.get() : nullptr};
    }
    void reset()
    {
        for (auto* b : {&ptr, &col, &len}) b->free();
        v64.free();
        v32.free();
        pk.free();
        has32 = false;
        haspk = false;
        slots = 0;
        max_nin = 0;
        src.clear();
        h_ptr.clear();
        h_col.clear();
        h_len.clear();
        prev_only.clear();
        unit_only.clear();
    }
};

// The persistent IC(0) apply (persist.cuh): its work items, their
// dependencies, and per launch configuration the ticket counter, done
// flags and reduction slots.
struct PersistVar {
    Buf<PCtl> ctl;
    Buf<unsigned int> flags;
    Buf<dd> slot;
    int grid = 0;
    size_t smem = 0;
    bool ready = false;
};

struct PersistPlan {
    bool ok = false;
    bool used = false;   // launched since the error word was last read
    int nitems = 0;
    size_t smem[2] = {0, 0};  // dynamic shared memory per CTA: [0] FP64, [1] FP32
    long long ndeps = 0;
    Buf<int> dep_ptr, dep_idx;
    Buf<unsigned int> err;
    PersistVar var[8];
    void reset()
    {
        ok = used = false;
        nitems = 0;
        smem[0] = smem[1] = 0;
        ndeps = 0;
        dep_ptr.free();
        dep_idx.free();
        for (auto& v : var) v.ready = false;
    }
};

// The lane-interleaved device system.
struct QSys {
    bool ok = false;
    int version = -1;         // schedule version it was built for
    int factor_version = -1;  // factor build it holds
    std::vector<int> q2r, r2q;
    Buf<int> dq2r;
    // sweep groups
    int nlevels = 0, ngroups = 0;
    std::vector<int> level_g;   // groups per level (nlevels+1)
    std::vector<int> fgrid, bslot0;
    int bnslots = 0;
    Buf<int> gbase, glen, sl0;
    std::vector<int> h_gbase, h_glen, h_sl0;
    std::vector<std::pair<int, int>> steps;  // step slices: (first Q row, rows)
    std::vector<int> step_r;                 // step index of each slice within its unit group
    Buf<SliceMeta> meta;                     // per slice (two-phase sweeps)
    int tile = 0;                            // slices of one two-phase batch (gpc * maxu)
    int ks = 8;                              // entries loaded speculatively per row
    std::vector<int> unit_of, step_of;       // per A_run row: unit id, row index in the unit
    int maxu = 0;                            // longest unit
    bool two_phase = false;                  // S/T carry in-unit entries as -(step + 1)
    int gpc = 1;                             // groups per CTA of the two-phase kernel
    bool q2_big = false;                     // its tile needs more than 48 KB (opt-in shared memory)
    int ni = 1;                              // in-unit entries staged per row (1, 2 or 4)
    std::vector<int> g2grid, b2slot0;        // its grids and backward reduction slots
    int b2nslots = 0;
    // staged sweeps (k_sweep_st): batches of groups, per-level buffer
    // capacities, and grids / backward reduction slots per value type
    // ([0] FP64, [1] FP32)
    bool staged = false;
    Buf<BatchDesc> bdesc;
    std::vector<BatchDesc> h_bdesc;                       // the batches, host copy (persistent apply plan)
    std::vector<int> lb;                                  // first batch of each level (nlevels + 1)
    std::vector<int> st_rows, st_slotsS, st_slotsT, st_slices;
    std::vector<int> st_fit;                              // 1: the level's batches fit the stage budget
    std::vector<int> st_one;                              // 1: ... in one stage buffer only (single-buffered kernel)
    std::vector<int> st_fit64;                            // 1: ... with FP64 values too (forward sweep)
    // levels whose rows have in-unit entries only, one per row, the previous
    // step, in full groups of at most 16 steps: the chain-only kernel
    std::vector<int> chainS, chainT;
    std::vector<int> st_fgrid[2], st_bgrid[2];
    std::vector<int> st1_fgrid[2], st1_bgrid[2];          // the same with one stage buffer
    std::vector<int> ch_grid[2];                          // chain-only kernel grids per level
    Buf<float> r32;                                       // FP32 reciprocal pivots
    bool r32_ok = false;
    // matrices
    SellDev A, S, T;
    Buf<double> d64, inv_diag;
    Buf<float> d32;
    bool d32_ok = false;
    PersistPlan pp;
    void reset()
    {
        pp.reset();
        ok = false;
        version = factor_version = -1;
        q2r.clear();
        r2q.clear();
        dq2r.free();
        nlevels = ngroups = 0;
        level_g.clear();
        fgrid.clear();
        bslot0.clear();
        bnslots = 0;
        gbase.free();
        glen.free();
        sl0.free();
        h_gbase.clear();
        h_glen.clear();
        h_sl0.clear();
        steps.clear();
        step_r.clear();
        meta.free();
        tile = 0;
        ks = 8;
        unit_of.clear();
        step_of.clear();
        maxu = 0;
        two_phase = false;
        gpc = 1;
        q2_big = false;
        g2grid.clear();
        b2slot0.clear();
        b2nslots = 0;
        staged = false;
        bdesc.free();
        h_bdesc.clear();
        lb.clear();
        for (auto* v : {&st_rows, &st_slotsS, &st_slotsT, &st_slices, &st_fit, &st_one, &st_fit64, &chainS, &chainT})
            v->clear();
        for (int k = 0; k < 2; ++k) {
            st_fgrid[k].clear();
            st_bgrid[k].clear();
            ch_grid[k].clear();
            st1_fgrid[k].clear();
            st1_bgrid[k].clear();
        }
        r32.free();
        r32_ok = false;
        A.reset();
        S.reset();
        T.reset();
        d64.free();
        inv_diag.free();
        d32.free();
        d32_ok = false;
    }
};

// What a captured iteration graph was recorded for: a graph is replayed
// only for a solve whose key equals it field by field (the graphs bake in
// the system, its kernels and the x / b device pointers).
// iterations per graph launch of a single-system solve when the caller does
// not choose: the 128^3 mixed solve took 20.10 / 19.92 / 19.80 / 19.79 ms
// with 4 / 8 / 16 / 32 (the replay loop shrinks the last graphs to 4, 2, 1)
constexpr int kGraphIters = 16;

struct GraphKey {
    int sched_version = -1, factor_version = -1, storage = -1, rri = -1, use_q = -1, m = -1, pc_kind = -1,
        sweep_kernel = -1;
    const void* x = nullptr;
    const void* b = nullptr;
    bool operator==(const GraphKey& o) const
    {
        return sched_version == o.sched_version && factor_version == o.factor_version && storage == o.storage &&
               rri == o.rri && use_q == o.use_q && m == o.m && pc_kind == o.pc_kind &&
               sweep_kernel == o.sweep_kernel && x == o.x && b == o.b;
    }
    bool operator!=(const GraphKey& o) const { return !(*this == o); }
};

}  // namespace iccg

struct iccg_ctx {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    long long dev_bytes = 0;
    // A_run
    int n = 0, nnz = 0;
    std::vector<int> h_rowptr, h_colind;
    std::vector<double> h_val;
    iccg::Buf<int> rowptr, colind;
    iccg::Buf<double> val64;
    iccg::Buf<float> val32;
    bool has_val32 = false;
    // schedule
    int sched_kind = ICCG_SCHED_NONE;
    // the natural-order plans are due but not built: an upload leaves them
    // to the first call that needs them, since a schedule usually follows
    bool plans_pending = false;
    int sched_version = 0;
    iccg::Plan fwd, bwd;
    // lane-interleaved system (default) or the simple one-thread-per-row path
    bool use_q = true;
    int sweep_kernel = 0;   // ICCG_OPT_SWEEP: 0 staged where it fits, 1 two-phase per-slice kernel
    bool pdl = true;        // ICCG_OPT_PDL: programmatic dependent launch
    int stage_kb = 0;       // ICCG_OPT_STAGE_KB: staged-sweep buffer budget (0: the opt-in maximum)
    int stage_rows = 256;   // ICCG_OPT_STAGE_ROWS: rows of a staged batch at most (one group may exceed it)
    int stage_bufs = 1;     // ICCG_OPT_STAGE_BUFS: staged-sweep buffers per CTA (1 or 2)
    int smem_optin = 0;     // largest dynamic shared memory per CTA
    bool persist = false;   // ICCG_OPT_PERSIST: the IC(0) apply as one persistent launch where planned
    bool fuse_update = false; // ICCG_OPT_FUSE_UPDATE: the CG update inside the forward sweep's launches
    bool defer_x = false;     // ICCG_OPT_DEFER_X: x += alpha p with the p update instead of the r update
    bool spmv_pack = true;    // ICCG_OPT_SPMV_PACK: FP32 SpMV reads (value, column) words
    int spmv_tpr = 1;         // ICCG_OPT_SPMV_TPR: threads per row of the FP32 SpMV (1, 2 or 4)
    bool update_chain = false;  // ICCG_OPT_UPDATE_CHAIN: the update does the first (chain-only) forward level
    int early = 1;            // ICCG_OPT_EARLY: loads before the wait on the previous launch
                              // (bit 0: FP32 storage solves, bit 1: FP64)
    iccg::QSys Q;
    // preconditioner
    int pc_kind = -1;
    int factor_version = 0;
    iccg::Buf<double> inv_diag;
    iccg::Factor F;
    // vectors: A_run-order staging (vb, vx) and work vectors (path order)
    iccg::Buf<double> vb, vx, qb, qx, vr, vp, vz, vy, vAp, vtmp;
    // reductions / state
    iccg::Buf<iccg::dd> partials;
    iccg::Buf<unsigned int> ticket;
    iccg::Buf<double> scalars;
    iccg::Buf<iccg::SolverState> state;
    iccg::Buf<unsigned long long> errword;
    iccg::SolverState* h_state = nullptr;  // pinned
    double* h_scalars = nullptr;           // pinned
    int* h_status = nullptr;               // pinned, 2 slots
    iccg::SolverState* h_obs = nullptr;    // pinned, 2 slots: the state after each graph launch
    size_t partial_slots = 0;
    // graph of the fused iteration
    // graphs of the fused iterations: one per pattern of residual-replacement
    // positions within a batch, all for the same system / vectors (gkey)
    struct GraphEntry {
        unsigned mask;   // iterations with the FP64 residual replacement
        int size;        // iterations in the graph
        cudaGraphExec_t exec;
        int kernels;
    };
    std::vector<GraphEntry> graphs;
    bool gkey_valid = false;
    iccg::GraphKey gkey;
    // events
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs[2] = {nullptr, nullptr};
    // profiling
    bool profile = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    size_t ev_used = 0;
    std::vector<int> ev_cls;
    double prof_ms[6] = {0, 0, 0, 0, 0, 0};
    long long prof_n[6] = {0, 0, 0, 0, 0, 0};
};
