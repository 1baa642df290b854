// plan.inl -- launch helpers and substitution / factorisation schedules
// (included by ctx.cu inside namespace iccg).

static int grid_for(const iccg_ctx* c, long long work, int threads = kThreads)
{
    long long g = (work + threads - 1) / threads;
    long long cap = (long long)c->nsm * (2048 / threads);
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// CTAs a grid-stride kernel should get: enough for the work, at most what is
// resident at once (the kernel's own occupancy at this block / shared memory
// size), so the work is spread over one wave instead of a full wave plus a
// ragged tail.
template <class K>
static int occ_grid(iccg_ctx* c, K kernel, long long work, int threads = kThreads, size_t smem = 0)
{
    static thread_local std::vector<std::pair<std::pair<const void*, size_t>, int>> cache;
    const void* key = reinterpret_cast<const void*>(kernel);
    int per_sm = 0;
    for (auto& e : cache)
        if (e.first.first == key && e.first.second == smem) per_sm = e.second;
    if (per_sm == 0) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
        if (per_sm < 1) per_sm = 1;
        cache.push_back({{key, smem}, per_sm});
    }
    long long g = (work + threads - 1) / threads;
    const long long cap = (long long)c->nsm * per_sm;
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

// One launch on the context's stream.  With c->pdl the launch allows
// programmatic dependent launch: its CTAs may be placed while the previous
// kernel drains; every kernel waits for its predecessor before touching
// global memory (grid_dep_begin), so the data dependencies are unchanged.
template <class... KArgs, class... Args>
static void launch_raw(iccg_ctx* c, void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args)
{
    if (c->pdl) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3((unsigned)block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, kernel, args...));
    } else {
        kernel<<<grid, block, smem, c->stream>>>(args...);
        CK(cudaGetLastError());
    }
}

// launch wrapper: counts launches and, when profiling, brackets each launch
// with CUDA events on the context's stream (class cls)
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
    launch_raw(c, kernel, grid, block, smem, args...);
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
    launch_raw(c, kernel, grid, block, 0, args...);
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


// launch of a grid-stride kernel over `work` items, one wave of CTAs
template <class K, class... Args>
static void launch_n(iccg_ctx* c, int cls, K kernel, long long work, Args... args)
{
    launch(c, cls, kernel, occ_grid(c, kernel, work), kThreads, args...);
}
