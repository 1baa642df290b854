// qsys.inl -- the lane-interleaved (Q-ordered) device system (included by
// ctx.cu inside namespace iccg).
//
// Q order from the forward plan: level by level; the level's units sorted by
// length, longest first (stable); groups of 32 consecutive units; inside a
// group the rows (step r, unit u) in r-major order.  Lane u of a warp owns
// unit u, so the active lanes of every step are a prefix and the rows of a
// step are consecutive Q rows.  The backward sweep runs the same groups with
// levels and steps reversed, which is a valid order because every backward
// dependency is a forward dependency reversed.

static void build_persist(iccg_ctx* c);  // persist.inl

// encode: 0 plain columns; 1 forward rows, 2 backward rows -- in-unit entries
// become -(step + 1) and each row's length word carries their count in its
// high half; returns false (and leaves plain columns) when a row's in-unit
// entries are not its last (forward) / first (backward) entries.
static bool sell_build(iccg_ctx* c, const std::vector<std::pair<int, int>>& slices, const std::vector<int>& rp,
                       const std::vector<int>& ci, const std::vector<int>* src_map, SellDev& M, int encode = 0)
{
    const QSys& Q = c->Q;
    const SellOrder order{(int)Q.q2r.size(), Q.q2r.data(), Q.r2q.data(), Q.unit_of.data(), Q.step_of.data()};
    if (!build_sell_layout(slices, rp.data(), ci.data(), src_map ? src_map->data() : nullptr, order, encode, M,
                           host_threads((long long)ci.size())))
        return false;
    M.ptr.upload(M.h_ptr.data(), M.h_ptr.size(), &c->dev_bytes, c->stream);
    M.col.upload(M.h_col.data(), M.h_col.size(), &c->dev_bytes, c->stream);
    M.len.upload(M.h_len.data(), M.h_len.size(), &c->dev_bytes, c->stream);
    M.has32 = false;
    M.v32.free();
    CK(cudaStreamSynchronize(c->stream));
    std::vector<int>().swap(M.h_col);
    std::vector<int>().swap(M.h_len);
    return true;
}

// M.v64[slot] = src[M.src[slot]] (0 on padding)
static void sell_values(iccg_ctx* c, SellDev& M, const double* src)
{
    Buf<int> idx;
    idx.upload(M.src.data(), M.src.size(), &c->dev_bytes, c->stream);
    M.v64.alloc((size_t)M.slots, &c->dev_bytes);
    if (M.slots)
        launch(c, 3, k_gather_pad<double>, grid_for(c, M.slots), kThreads, (long long)M.slots,
               (const int*)idx.get(), src, M.v64.get());
    CK(cudaStreamSynchronize(c->stream));
    M.has32 = false;
}

static void sell_f32(iccg_ctx* c, SellDev& M)
{
    if (M.has32) return;
    M.v32.alloc((size_t)M.slots, &c->dev_bytes);
    if (M.slots)
        launch(c, 3, k_to_f32, grid_for(c, M.slots), kThreads, (long long)M.slots, (const double*)M.v64.get(),
               M.v32.get());
    CK(cudaStreamSynchronize(c->stream));
    M.has32 = true;
}

static void build_q_order(iccg_ctx* c)
{
    QSys& Q = c->Q;
    const Plan& P = c->fwd;
    Q.q2r.clear();
    Q.q2r.reserve((size_t)c->n);
    Q.level_g.assign(1, 0);
    Q.h_gbase.clear();
    Q.h_glen.clear();
    Q.h_sl0.clear();
    Q.steps.clear();
    struct U { int t0, m; };
    std::vector<U> units;
    Q.unit_of.assign((size_t)c->n, -1);
    Q.step_of.assign((size_t)c->n, 0);
    Q.step_r.clear();
    Q.maxu = 0;
    int unit_id = 0;
    for (int l = 0; l < P.nlevels; ++l) {
        units.clear();
        for (int u = P.level_ptr[(size_t)l]; u < P.level_ptr[(size_t)l + 1]; ++u) {
            const int t0 = P.unit_is_row ? u : P.h_unit_ptr[(size_t)u];
            const int t1 = P.unit_is_row ? u + 1 : P.h_unit_ptr[(size_t)u + 1];
            if (t1 > t0) units.push_back({t0, t1 - t0});
        }
        std::stable_sort(units.begin(), units.end(), [](const U& a, const U& b) { return a.m > b.m; });
        for (size_t g0 = 0; g0 < units.size(); g0 += 32) {
            const size_t g1 = std::min(units.size(), g0 + 32);
            Q.h_gbase.push_back((int)Q.q2r.size());
            Q.h_sl0.push_back((int)Q.steps.size());
            for (size_t u = g0; u < g0 + 32; ++u) Q.h_glen.push_back(u < g1 ? units[u].m : 0);
            const int maxlen = units[g0].m;
            Q.maxu = std::max(Q.maxu, maxlen);
            for (int r = 0; r < maxlen; ++r) {
                int cnt = 0;
                while (g0 + (size_t)cnt < g1 && units[g0 + (size_t)cnt].m > r) ++cnt;
                Q.steps.emplace_back((int)Q.q2r.size(), cnt);
                Q.step_r.push_back(r);
                for (int u = 0; u < cnt; ++u) {
                    const int row = P.h_rows[(size_t)(units[g0 + (size_t)u].t0 + r)];
                    Q.q2r.push_back(row);
                    if (row >= 0 && row < c->n) {
                        Q.unit_of[(size_t)row] = unit_id + (int)(g0 + (size_t)u);
                        Q.step_of[(size_t)row] = r;
                    }
                }
            }
        }
        unit_id += (int)units.size();
        Q.level_g.push_back((int)Q.h_gbase.size());
    }
    if ((int)Q.q2r.size() != c->n) throw Error(ICCG_ERR_SCHEDULE, "schedule does not cover every row once");
    Q.h_gbase.push_back((int)Q.q2r.size());
    Q.h_sl0.push_back((int)Q.steps.size());
    Q.r2q.assign((size_t)c->n, -1);
    for (int q = 0; q < c->n; ++q) Q.r2q[(size_t)Q.q2r[(size_t)q]] = q;
    Q.nlevels = P.nlevels;
    Q.ngroups = (int)Q.h_sl0.size() - 1;
    Q.fgrid.assign((size_t)Q.nlevels, 1);
    Q.bslot0.assign((size_t)Q.nlevels, 0);
    const int cap = c->nsm * 8;
    for (int l = 0; l < Q.nlevels; ++l) {
        const int groups = Q.level_g[(size_t)l + 1] - Q.level_g[(size_t)l];
        Q.fgrid[(size_t)l] = std::max(1, std::min(cap, (groups + 7) / 8));  // 8 warps per CTA
    }
    int s = 0;
    for (int l = Q.nlevels - 1; l >= 0; --l) {
        Q.bslot0[(size_t)l] = s;
        s += Q.fgrid[(size_t)l];
    }
    Q.bnslots = s;
    ensure_partials(c, (size_t)std::max(s, 1));
    Q.dq2r.upload(Q.q2r.data(), Q.q2r.size(), &c->dev_bytes, c->stream);
    Q.gbase.upload(Q.h_gbase.data(), Q.h_gbase.size(), &c->dev_bytes, c->stream);
    Q.glen.upload(Q.h_glen.data(), Q.h_glen.size(), &c->dev_bytes, c->stream);
    Q.sl0.upload(Q.h_sl0.data(), Q.h_sl0.size(), &c->dev_bytes, c->stream);
    // A_run in Q order, regular 32-row slices
    std::vector<std::pair<int, int>> sl;
    for (int q = 0; q < c->n; q += 32) sl.emplace_back(q, std::min(32, c->n - q));
    sell_build(c, sl, c->h_rowptr, c->h_colind, nullptr, Q.A);
    sell_values(c, Q.A, c->val64.get());
}

// bytes per row of the two-phase sweep's shared tile (see k_sweep_q2)
static size_t sweep_row_bytes(size_t tsize, int ni, bool slow, bool with_r)
{
    return 8 + (with_r ? 8 : 0) + tsize * (1 + (size_t)ni) + 4 + (slow ? 8 : 0) + (size_t)ni;
}

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum less its static shared memory (once per kernel and device).
template <class K>
static void allow_smem(iccg_ctx* c, K kernel)
{
    // shared by every context of the process, which may run in several host
    // threads at once
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> done;
    std::lock_guard<std::mutex> lock(mu);
    const void* key = reinterpret_cast<const void*>(kernel);
    for (auto& e : done)
        if (e.first == key && e.second == c->device) return;
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, kernel));
    const int dyn = c->smem_optin - (int)fa.sharedSizeBytes;
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    done.push_back({key, c->device});
}

// Every k_sweep_q2 instantiation the sweeps launch, for tiles above the
// default 48 KB of dynamic shared memory (set at plan time, before any
// graph capture).
template <class T, int NI, int KS>
static void allow_q2_smem_t(iccg_ctx* c)
{
    constexpr bool f32 = std::is_same<T, float>::value;
    allow_smem(c, k_sweep_q2<T, true, FIN_NONE, true, NI, KS>);
    allow_smem(c, k_sweep_q2<T, false, FIN_NONE, !f32, NI, KS>);
    allow_smem(c, k_sweep_q2<T, false, FIN_RZ, !f32, NI, KS>);
    allow_smem(c, k_sweep_q2<T, false, FIN_RZ0, !f32, NI, KS>);
}

static void allow_q2_smem(iccg_ctx* c)
{
    allow_q2_smem_t<double, 1, 8>(c);
    allow_q2_smem_t<double, 1, 16>(c);
    allow_q2_smem_t<double, 2, 8>(c);
    allow_q2_smem_t<double, 2, 16>(c);
    allow_q2_smem_t<float, 1, 8>(c);
    allow_q2_smem_t<float, 1, 16>(c);
    allow_q2_smem_t<float, 2, 8>(c);
    allow_q2_smem_t<float, 2, 16>(c);
}

// Grids of the staged sweeps for value type T at each level: one CTA per
// batch up to what is resident at once at that level's buffer size.  The
// staged kernel runs forward sweeps in both types and backward sweeps with
// FP32 storage (FP64 backward sweeps use the per-slice kernel), so only
// those buffers are sized here; levels whose batches do not fit the stage
// budget keep grid 1 and run on the per-slice kernel.
template <class T>
static bool plan_staged_type(iccg_ctx* c, int k)
{
    QSys& Q = c->Q;
    constexpr bool exact = !std::is_same<T, float>::value;
    auto kf = k_sweep_st<T, true, FIN_NONE, exact>;
    auto kb = k_sweep_st<T, false, FIN_RZ, exact>;
    auto kf1 = k_sweep_st<T, true, FIN_NONE, exact, 1>;
    auto kb1 = k_sweep_st<T, false, FIN_RZ, exact, 1>;
    allow_smem(c, kf);
    allow_smem(c, kb);
    allow_smem(c, kf1);
    allow_smem(c, kb1);
    const int L = Q.nlevels;
    Q.st_fgrid[k].assign((size_t)L, 1);
    Q.st_bgrid[k].assign((size_t)L, 1);
    Q.st1_fgrid[k].assign((size_t)L, 1);
    Q.st1_bgrid[k].assign((size_t)L, 1);
    // the kernel's static shared memory (reduction scratch) comes on top
    const size_t lim = (size_t)std::max(0, c->smem_optin - 2048);
    for (int l = 0; l < L; ++l) {
        if (!Q.st_fit[(size_t)l] || (exact && !Q.st_fit64[(size_t)l])) continue;
        const int nb = Q.lb[(size_t)l + 1] - Q.lb[(size_t)l];
        // levels marked st_one run single-buffered only
        const bool two = !Q.st_one[(size_t)l];
        const size_t fs = (size_t)stage_layout(Q.st_rows[(size_t)l], Q.st_slotsS[(size_t)l],
                                               Q.st_slices[(size_t)l], (int)sizeof(T), false, false).bytes;
        if ((two ? 2 : 1) * fs > lim) return false;
        int pf = 0, pf1 = 0;
        if (two) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, kf, kThreads, 2 * fs));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf1, kf1, kThreads, fs));
        if ((two && pf < 1) || pf1 < 1) return false;
        Q.st1_fgrid[k][(size_t)l] = std::max(1, std::min(nb, pf1 * c->nsm));
        Q.st_fgrid[k][(size_t)l] = two ? std::max(1, std::min(nb, pf * c->nsm)) : Q.st1_fgrid[k][(size_t)l];
        if (!exact) {
            const size_t bs = (size_t)stage_layout(Q.st_rows[(size_t)l], Q.st_slotsT[(size_t)l],
                                                   Q.st_slices[(size_t)l], (int)sizeof(T), true, false).bytes;
            if ((two ? 2 : 1) * bs > lim) return false;
            int pb = 0, pb1 = 0;
            if (two) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pb, kb, kThreads, 2 * bs));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pb1, kb1, kThreads, bs));
            if ((two && pb < 1) || pb1 < 1) return false;
            Q.st1_bgrid[k][(size_t)l] = std::max(1, std::min(nb, pb1 * c->nsm));
            Q.st_bgrid[k][(size_t)l] = two ? std::max(1, std::min(nb, pb * c->nsm)) : Q.st1_bgrid[k][(size_t)l];
        }
    }
    // chain-only levels: one warp per group
    int pc = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pc, k_sweep_chain<T, false, FIN_RZ, exact>, kThreads, 0));
    Q.ch_grid[k].assign((size_t)L, 1);
    for (int l = 0; l < L; ++l) {
        const int ng = Q.level_g[(size_t)l + 1] - Q.level_g[(size_t)l];
        Q.ch_grid[k][(size_t)l] = std::max(1, std::min((ng + 7) / 8, std::max(1, pc) * c->nsm));
    }
    // reduction slots of a sweep (the backward r.z, or the forward r.r of
    // the fused update), whichever kernels its levels use
    long long s = 0;
    for (int l = 0; l < L; ++l)
        s += std::max({Q.st_bgrid[k][(size_t)l], Q.st1_bgrid[k][(size_t)l], Q.st_fgrid[k][(size_t)l],
                       Q.st1_fgrid[k][(size_t)l], Q.ch_grid[k][(size_t)l], Q.two_phase ? Q.g2grid[(size_t)l] : 0,
                       Q.fgrid.empty() ? 0 : Q.fgrid[(size_t)l]});
    ensure_partials(c, (size_t)std::max<long long>(s, 1));
    return true;
}

// Batches of the staged sweeps: consecutive groups of one level, at most 16
// groups and ICCG_OPT_STAGE_ROWS rows (256), and as many groups as keep two stage buffers of every
// type the staged kernel runs with (FP64 and FP32 forward, FP32 backward)
// within the budget (ICCG_OPT_STAGE_KB, default the opt-in shared memory);
// the default single buffer per CTA then takes half of it.  A level with a group that alone exceeds the budget runs on the
// per-slice kernel.
static void plan_staged(iccg_ctx* c)
{
    QSys& Q = c->Q;
    Q.staged = false;
    const int cap_rows = c->stage_rows;
    const int gmax = std::max(1, std::min(16, cap_rows / (32 * std::max(1, Q.maxu))));
    const size_t lim = (size_t)std::max(0, c->smem_optin - 2048);
    const size_t budget = c->stage_kb > 0 ? std::min(lim, (size_t)c->stage_kb * 1024) : lim;
    std::vector<BatchDesc> bds;
    Q.lb.assign((size_t)Q.nlevels + 1, 0);
    Q.st_rows.assign((size_t)Q.nlevels, 0);
    Q.st_slotsS.assign((size_t)Q.nlevels, 0);
    Q.st_slotsT.assign((size_t)Q.nlevels, 0);
    Q.st_slices.assign((size_t)Q.nlevels, 0);
    Q.st_fit.assign((size_t)Q.nlevels, 1);
    Q.st_one.assign((size_t)Q.nlevels, 0);
    Q.st_fit64.assign((size_t)Q.nlevels, 1);
    Q.chainS.assign((size_t)Q.nlevels, 1);
    Q.chainT.assign((size_t)Q.nlevels, 1);
    // groups [g, g + ng) of a level as one batch (se <= sb: not a batch)
    auto describe = [&](int g, int ng) {
        BatchDesc d{};
        d.gb = g;
        d.ng = ng;
        d.sb = Q.h_sl0[(size_t)g];
        d.se = Q.h_sl0[(size_t)(g + ng)];
        if (d.se <= d.sb) return d;
        d.qb = Q.steps[(size_t)d.sb].first;
        d.qe = Q.steps[(size_t)d.se - 1].first + Q.steps[(size_t)d.se - 1].second;
        d.ps0 = Q.S.h_ptr[(size_t)d.sb];
        d.ps1 = Q.S.h_ptr[(size_t)d.se];
        d.pt0 = Q.T.h_ptr[(size_t)d.sb];
        d.pt1 = Q.T.h_ptr[(size_t)d.se];
        return d;
    };
    // the level's buffer holds its largest batch in every dimension: the
    // stage bytes of one buffer at the level's capacities grown by batch d
    // (FP32 forward and backward, and FP64 forward unless the level dropped it)
    auto stage_bytes1 = [&](int l, const BatchDesc& d) {
        const int rows = std::max(Q.st_rows[(size_t)l], d.qe - d.qb);
        const int slS = std::max(Q.st_slotsS[(size_t)l], d.ps1 - d.ps0);
        const int slT = std::max(Q.st_slotsT[(size_t)l], d.pt1 - d.pt0);
        const int slices = std::max(Q.st_slices[(size_t)l], d.se - d.sb);
        return (size_t)std::max({Q.st_fit64[(size_t)l] ? stage_layout(rows, slS, slices, 8, false, false).bytes : 0,
                                 stage_layout(rows, slS, slices, 4, false, false).bytes,
                                 stage_layout(rows, slT, slices, 4, true, false).bytes});
    };
    // two buffers (the double-buffered kernel), or one at levels whose
    // single groups need it (st_one)
    auto stage_bytes = [&](int l, const BatchDesc& d) {
        return (Q.st_one[(size_t)l] ? 1 : 2) * stage_bytes1(l, d);
    };
    for (int l = 0; l < Q.nlevels; ++l) {
        const int g1 = Q.level_g[(size_t)l + 1];
        for (int g = Q.level_g[(size_t)l]; g < g1; ++g)
            if (Q.h_glen[(size_t)g * 32] > 16) Q.chainS[(size_t)l] = Q.chainT[(size_t)l] = 0;
        for (int g = Q.level_g[(size_t)l]; g < g1;) {
            BatchDesc d = describe(g, 1);
            if (d.se <= d.sb) return;
            if (stage_bytes(l, d) > budget) {
                // a group too large for two buffers: the level runs single-buffered;
                // too large for one with FP64 values: FP64 leaves the staged kernel
                // there (the per-slice kernel, the same bits); too large still: the
                // level is not staged
                Q.st_one[(size_t)l] = 1;
                if (stage_bytes(l, d) > budget) Q.st_fit64[(size_t)l] = 0;
                if (stage_bytes(l, d) > budget) Q.st_fit[(size_t)l] = 0;
            }
            while (d.ng < gmax && g + d.ng < g1 && Q.st_fit[(size_t)l]) {
                const BatchDesc e = describe(g, d.ng + 1);
                if (e.qe - e.qb > cap_rows || stage_bytes(l, e) > budget) break;
                d = e;
            }
            for (int s = d.sb + 1; s < d.se; ++s)
                if (Q.steps[(size_t)s].first != Q.steps[(size_t)s - 1].first + Q.steps[(size_t)s - 1].second) return;
            // regular batch: every group full (32 units of one length) and
            // every row's in-unit entry, if any, the step just before
            bool full = true;
            for (int gi = 0; gi < d.ng && full; ++gi) {
                const int g0 = d.gb + gi;
                for (int u = 0; u < 32; ++u)
                    full = full && Q.h_glen[(size_t)g0 * 32 + (size_t)u] == Q.h_glen[(size_t)g0 * 32];
            }
            bool pS = full, pT = full;
            for (int q = d.qb; q < d.qe && (pS || pT); ++q) {
                pS = pS && Q.S.prev_only[(size_t)q];
                pT = pT && Q.T.prev_only[(size_t)q];
            }
            d.flags = (pS ? 1 : 0) | (pT ? 2 : 0) | (full ? 4 : 0);
            if (!full || !pS) Q.chainS[(size_t)l] = 0;
            if (!full || !pT) Q.chainT[(size_t)l] = 0;
            for (int q = d.qb; q < d.qe && (Q.chainS[(size_t)l] || Q.chainT[(size_t)l]); ++q) {
                if (!Q.S.unit_only[(size_t)q]) Q.chainS[(size_t)l] = 0;
                if (!Q.T.unit_only[(size_t)q]) Q.chainT[(size_t)l] = 0;
            }
            Q.st_rows[(size_t)l] = std::max(Q.st_rows[(size_t)l], d.qe - d.qb);
            Q.st_slotsS[(size_t)l] = std::max(Q.st_slotsS[(size_t)l], d.ps1 - d.ps0);
            Q.st_slotsT[(size_t)l] = std::max(Q.st_slotsT[(size_t)l], d.pt1 - d.pt0);
            Q.st_slices[(size_t)l] = std::max(Q.st_slices[(size_t)l], d.se - d.sb);
            bds.push_back(d);
            g += d.ng;
        }
        Q.lb[(size_t)l + 1] = (int)bds.size();
    }
    SetupPhase t("q.factor.staged_grids");
    if (!plan_staged_type<double>(c, 0) || !plan_staged_type<float>(c, 1)) return;
    Q.bdesc.upload(bds.data(), bds.size(), &c->dev_bytes, c->stream);
    CK(cudaStreamSynchronize(c->stream));
    Q.h_bdesc.swap(bds);
    Q.staged = true;
}

static void build_q_factor(iccg_ctx* c)
{
    QSys& Q = c->Q;
    Factor& F = c->F;
    // two-phase sweeps need units of at most 64 rows, in-unit entries last
    // (forward) / first (backward) in every row -- the reference's column
    // order gives that for schedules from BuildABMCSchedule -- and the tile
    // of one group in shared memory: up to 8 groups in 48 KB, or, for units
    // of 32 to 64 rows, one group in the opt-in shared memory
    auto build = [&](bool enc) {
        bool ok = sell_build(c, Q.steps, F.Sp, F.Si, &F.s_src, Q.S, enc ? 1 : 0) &&
                  sell_build(c, Q.steps, F.Tp, F.Ti, &F.t_src, Q.T, enc ? 2 : 0);
        return ok;
    };
    Q.staged = false;
    Q.r32_ok = false;
    Q.two_phase = Q.maxu <= 64 && build(true);
    if (Q.two_phase) {
        // NI in-unit entries staged per row; gpc groups per CTA so that the
        // tile (R = gpc * maxu * 32 rows of 24 + 12 NI bytes) stays within
        // 48 KB and holds at most 1024 rows
        const int mx = std::max(Q.S.max_nin, Q.T.max_nin);
        Q.ni = mx <= 1 ? 1 : 2;  // rows with more in-unit entries take the slow path
        // largest tile row: FP64 pivots and values plus the slow-path words
        const size_t row_bytes = sweep_row_bytes(8, Q.ni, true, true);
        const size_t per_group = (size_t)std::max(1, Q.maxu) * 32 * row_bytes;
        Q.gpc = (int)std::max<size_t>(
            1, std::min<size_t>({8, 48 * 1024 / per_group, 32 / (size_t)std::max(1, Q.maxu)}));
        Q.q2_big = per_group * Q.gpc > 48 * 1024;
        // the kernel's static shared memory (reduction scratch) comes on top
        if (Q.q2_big && per_group > (size_t)std::max(0, c->smem_optin - 4096)) Q.two_phase = false;
        if (Q.two_phase && Q.q2_big) allow_q2_smem(c);
    }
    if (!Q.two_phase) build(false);
    sell_values(c, Q.S, F.dLx.get());
    sell_values(c, Q.T, F.dLx.get());
    if (Q.two_phase) {
        Q.g2grid.assign((size_t)Q.nlevels, 1);
        Q.b2slot0.assign((size_t)Q.nlevels, 0);
        // resident CTAs of the FP32-storage backward kernel at its tile size
        Q.tile = Q.gpc * Q.maxu;
        int wmax = 0;
        for (size_t s = 0; s < Q.steps.size(); ++s)
            wmax = std::max({wmax, (Q.S.h_ptr[s + 1] - Q.S.h_ptr[s]) / 32, (Q.T.h_ptr[s + 1] - Q.T.h_ptr[s]) / 32});
        Q.ks = wmax <= 8 ? 8 : 16;
        std::vector<SliceMeta> mt(Q.steps.size());
        for (size_t s = 0; s < Q.steps.size(); ++s) {
            const int ws = std::min(255, (Q.S.h_ptr[s + 1] - Q.S.h_ptr[s]) / 32);
            const int wt = std::min(255, (Q.T.h_ptr[s + 1] - Q.T.h_ptr[s]) / 32);
            mt[s] = SliceMeta{Q.steps[s].first, Q.S.h_ptr[s], Q.T.h_ptr[s],
                              Q.steps[s].second | (Q.step_r[s] << 6) | (ws << 12) | (wt << 20)};
        }
        Q.meta.upload(mt.data(), mt.size(), &c->dev_bytes, c->stream);
        const size_t fast = (size_t)Q.tile * 32 * sweep_row_bytes(4, Q.ni, Q.T.max_nin > Q.ni, true);
        int per_sm = 1;
        if (Q.ni == 1)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_q2<float, false, FIN_RZ, false, 1, 8>,
                                                             kThreads, fast));
        else
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_q2<float, false, FIN_RZ, false, 2, 8>,
                                                             kThreads, fast));
        const int cap = c->nsm * std::max(1, per_sm);
        for (int l = 0; l < Q.nlevels; ++l) {
            const int groups = Q.level_g[(size_t)l + 1] - Q.level_g[(size_t)l];
            Q.g2grid[(size_t)l] = std::max(1, std::min(cap, (groups + Q.gpc - 1) / Q.gpc));
        }
        int s = 0;
        for (int l = Q.nlevels - 1; l >= 0; --l) {
            Q.b2slot0[(size_t)l] = s;
            s += Q.g2grid[(size_t)l];
        }
        Q.b2nslots = s;
        ensure_partials(c, (size_t)std::max(s, 1));
        plan_staged(c);
        build_persist(c);
    }
    std::vector<int> dsrc((size_t)c->n);
    for (int q = 0; q < c->n; ++q) dsrc[(size_t)q] = F.dpos[(size_t)Q.q2r[(size_t)q]];
    Buf<int> idx;
    idx.upload(dsrc.data(), dsrc.size(), &c->dev_bytes, c->stream);
    Q.d64.alloc((size_t)c->n, &c->dev_bytes);
    launch(c, 3, k_gather<double>, grid_for(c, c->n), kThreads, (long long)c->n, (const int*)idx.get(),
           (const double*)F.dLx.get(), Q.d64.get());
    CK(cudaStreamSynchronize(c->stream));
    Q.d32_ok = false;
}

static void ensure_q(iccg_ctx* c)
{
    QSys& Q = c->Q;
    if (!Q.ok || Q.version != c->sched_version) {
        SetupPhase t("q.order");
        Q.reset();
        build_q_order(c);
        Q.version = c->sched_version;
        Q.ok = true;
    }
    if (Q.factor_version != c->factor_version) {
        // a new preconditioner since the last build
        if (c->pc_kind == ICCG_PRECOND_IC0 && c->F.built) {
            SetupPhase t("q.factor");
            build_q_factor(c);
        }
        if (c->pc_kind == ICCG_PRECOND_JACOBI) {
            Q.inv_diag.alloc((size_t)c->n, &c->dev_bytes);
            launch(c, 3, k_gather<double>, grid_for(c, c->n), kThreads, (long long)c->n, (const int*)Q.dq2r.get(),
                   (const double*)c->inv_diag.get(), Q.inv_diag.get());
            CK(cudaStreamSynchronize(c->stream));
        }
        Q.factor_version = c->factor_version;
    }
}

static void ensure_q32(iccg_ctx* c)
{
    SetupPhase t("q.fp32_copies");
    QSys& Q = c->Q;
    sell_f32(c, Q.A);
    if ((c->spmv_pack || c->spmv_tpr > 1) && !Q.A.haspk) {
        Q.A.pk.alloc((size_t)Q.A.slots, &c->dev_bytes);
        if (Q.A.slots)
            launch(c, 3, k_pack_sell, grid_for(c, Q.A.slots), kThreads, (long long)Q.A.slots,
                   (const float*)Q.A.v32.get(), (const int*)Q.A.col.get(), Q.A.pk.get());
        CK(cudaStreamSynchronize(c->stream));
        Q.A.haspk = true;
    }
    if (c->pc_kind == ICCG_PRECOND_IC0 && c->F.built) {
        sell_f32(c, Q.S);
        sell_f32(c, Q.T);
        if (!Q.d32_ok) {
            Q.d32.alloc((size_t)c->n, &c->dev_bytes);
            launch(c, 3, k_to_f32, grid_for(c, c->n), kThreads, (long long)c->n, (const double*)Q.d64.get(),
                   Q.d32.get());
            CK(cudaStreamSynchronize(c->stream));
            Q.d32_ok = true;
        }
        if ((Q.staged || Q.pp.ok) && !Q.r32_ok) {
            Q.r32.alloc((size_t)c->n, &c->dev_bytes);
            launch(c, 3, k_recip_f32, grid_for(c, c->n), kThreads, (long long)c->n, (const double*)Q.d64.get(),
                   Q.r32.get());
            CK(cudaStreamSynchronize(c->stream));
            Q.r32_ok = true;
        }
    }
}
