// persist.inl -- planning and launch of the persistent IC(0) apply
// (persist.cuh); included by ctx.cu inside namespace iccg.
//
// The items are the staged batches (plan_staged): consecutive unit groups
// of one level.  A forward item waits for the forward items that hold the
// columns of its rows' strictly lower entries (earlier levels); a backward
// item waits for the forward item of its own rows (its input y and r) and
// for the backward items that hold the columns of its rows' strictly upper
// entries (later levels, done earlier in the backward sweep).  Every such
// item has a lower ticket.

// launch configurations: [FP32 ? 4 : 0] + kind
enum PersistKind { PK_PLAIN = 0, PK_RZ0 = 1, PK_RZ = 2, PK_UPD_RZ = 3 };

static void build_persist(iccg_ctx* c)
{
    QSys& Q = c->Q;
    PersistPlan& PP = Q.pp;
    PP.reset();
    const Factor& F = c->F;
    // every level staged (batches within the shared-memory budget)
    if (!Q.staged || Q.h_bdesc.empty()) return;
    for (int l = 0; l < Q.nlevels; ++l)
        if (!Q.st_fit[(size_t)l]) return;
    SetupPhase tp("q.factor.persist_plan");
    const std::vector<BatchDesc>& items = Q.h_bdesc;
    const int ni = (int)items.size();
    std::vector<int> item_of_q((size_t)c->n, -1);
    for (int i = 0; i < ni; ++i)
        for (int q = items[(size_t)i].qb; q < items[(size_t)i].qe; ++q) item_of_q[(size_t)q] = i;
    for (int q = 0; q < c->n; ++q)
        if (item_of_q[(size_t)q] < 0) return;
    // dependencies per ticket: forward tickets 0..ni-1 are items 0..ni-1;
    // backward ticket ni + b is item ni - 1 - b
    std::vector<int> dptr((size_t)2 * ni + 1, 0), didx;
    std::vector<int> seen((size_t)2 * ni, -1);
    didx.reserve((size_t)ni * 8);
    auto add = [&](int t, int dep) {
        if (dep == t || seen[(size_t)dep] == t) return true;
        if (dep > t) return false;
        seen[(size_t)dep] = t;
        didx.push_back(dep);
        return true;
    };
    for (int t = 0; t < 2 * ni; ++t) {
        const bool fwd = t < ni;
        const int it = fwd ? t : 2 * ni - 1 - t;
        const BatchDesc& I = items[(size_t)it];
        if (!fwd && !add(t, it)) return;
        const std::vector<int>& rp = fwd ? F.Sp : F.Tp;
        const std::vector<int>& ci = fwd ? F.Si : F.Ti;
        for (int q = I.qb; q < I.qe; ++q) {
            const int row = Q.q2r[(size_t)q];
            for (int k = rp[(size_t)row]; k < rp[(size_t)row + 1]; ++k) {
                const int f = item_of_q[(size_t)Q.r2q[(size_t)ci[(size_t)k]]];
                if (!add(t, fwd ? f : 2 * ni - 1 - f)) return;  // a schedule the plan does not cover
            }
        }
        dptr[(size_t)t + 1] = (int)didx.size();
    }
    // shared memory per value type: the largest batch layout of either
    // sweep, with the backward reduction (and FP64's parked values)
    for (const BatchDesc& d : items) {
        PP.smem[0] = std::max({PP.smem[0], (size_t)persist_layout<double, true, true>(d, true).bytes,
                               (size_t)persist_layout<double, true, true>(d, false).bytes});
        PP.smem[1] = std::max({PP.smem[1], (size_t)persist_layout<float, true, false>(d, true).bytes,
                               (size_t)persist_layout<float, true, false>(d, false).bytes});
    }
    PP.nitems = ni;
    PP.dep_ptr.upload(dptr.data(), dptr.size(), &c->dev_bytes, c->stream);
    if (!didx.empty()) PP.dep_idx.upload(didx.data(), didx.size(), &c->dev_bytes, c->stream);
    else PP.dep_idx.alloc(1, &c->dev_bytes);
    PP.err.alloc(1, &c->dev_bytes);
    CK(cudaMemsetAsync(PP.err.get(), 0, sizeof(unsigned int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    PP.ndeps = (long long)didx.size();
    PP.ok = true;
}

template <class T, bool UPD, int FIN>
static auto persist_kernel()
{
    return k_apply_persist<T, !std::is_same<T, float>::value, UPD, FIN>;
}

// the launch configuration's counters, shared memory and grid, made on
// first use (before any graph capture: see prepare_persist_t)
template <class T, bool UPD, int FIN>
static PersistVar& persist_var(iccg_ctx* c, int v)
{
    PersistPlan& PP = c->Q.pp;
    PersistVar& V = PP.var[v];
    if (V.ready) return V;
    const int ni = PP.nitems;
    const size_t smem = PP.smem[std::is_same<T, float>::value ? 1 : 0];
    auto kern = persist_kernel<T, UPD, FIN>();
    V.ctl.alloc(1, &c->dev_bytes);
    V.flags.alloc((size_t)2 * ni, &c->dev_bytes);
    V.slot.alloc((size_t)2 * ni, &c->dev_bytes);
    CK(cudaMemsetAsync(V.ctl.get(), 0, sizeof(PCtl), c->stream));
    CK(cudaMemsetAsync(V.flags.get(), 0, sizeof(unsigned int) * 2 * (size_t)ni, c->stream));
    V.smem = smem;
    allow_smem(c, kern);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPersistThreads, V.smem));
    if (per_sm < 1) throw Error(ICCG_ERR_ARG, "persistent apply does not fit an SM");
    V.grid = per_sm * c->nsm;
    CK(cudaStreamSynchronize(c->stream));
    V.ready = true;
    return V;
}

// Makes the counters of every launch configuration a solve of this storage
// uses (initial apply, plain and fused iterations): their allocation and
// clearing must happen before the iterations are captured into a graph.
template <class T>
static void prepare_persist_t(iccg_ctx* c)
{
    constexpr int b = std::is_same<T, float>::value ? 4 : 0;
    persist_var<T, false, FIN_NONE>(c, b + PK_PLAIN);
    persist_var<T, false, FIN_RZ0>(c, b + PK_RZ0);
    persist_var<T, false, FIN_RZ>(c, b + PK_RZ);
    persist_var<T, true, FIN_RZ>(c, b + PK_UPD_RZ);
}

// true if the IC(0) apply of this storage runs as one persistent launch:
// planned, and its largest batch (with the kernel's own shared memory, at
// most 4 KB) fits one CTA's shared memory
static bool use_persist(const iccg_ctx* c, int storage)
{
    const QSys& Q = c->Q;
    if (!c->persist || !c->use_q || c->pc_kind != ICCG_PRECOND_IC0 || !Q.pp.ok) return false;
    const bool f32 = storage == ICCG_STORE_FP32;
    if (Q.pp.smem[f32 ? 1 : 0] + 4096 > (size_t)c->smem_optin) return false;
    return !f32 || Q.r32_ok;
}

// z = M^{-1} r (y: the forward result) in one launch; UPD first does the CG
// update x += alpha p, r -= alpha Ap of the forward rows and reduces r.r
template <class T, bool UPD, int FIN>
static void launch_persist(iccg_ctx* c, double* r, double* y, double* z, SolverState* st, double* x = nullptr)
{
    QSys& Q = c->Q;
    PersistPlan& PP = Q.pp;
    constexpr bool f32 = std::is_same<T, float>::value;
    const int kind = UPD ? PK_UPD_RZ : FIN == FIN_RZ0 ? PK_RZ0 : FIN == FIN_RZ ? PK_RZ : PK_PLAIN;
    PersistVar& V = persist_var<T, UPD, FIN>(c, (f32 ? 4 : 0) + kind);
    PArgs a{};
    a.nitems = PP.nitems;
    a.items = Q.bdesc.get();
    a.dep_ptr = PP.dep_ptr.get();
    a.dep_idx = PP.dep_idx.get();
    a.flags = V.flags.get();
    a.ctl = V.ctl.get();
    a.slot = V.slot.get();
    a.err = PP.err.get();
    a.glen = Q.glen.get();
    a.sl0 = Q.sl0.get();
    a.meta = (const SliceMeta*)Q.meta.get();
    a.S = Q.S.view(f32);
    a.T = Q.T.view(f32);
    a.dg = f32 ? (const void*)Q.r32.get() : (const void*)Q.d64.get();
    a.r = r;
    a.y = y;
    a.z = z;
    a.x = x;
    a.p = c->vp.get();
    a.Ap = c->vAp.get();
    a.st = st;
    launch_smem(c, 5, persist_kernel<T, UPD, FIN>(), V.grid, kPersistThreads, V.smem, a);
    PP.used = true;
}

// reads and clears the plan's error word (stream already synchronised)
static void check_persist(iccg_ctx* c)
{
    PersistPlan& PP = c->Q.pp;
    if (!PP.ok || !PP.used) return;
    unsigned int e = 0;
    CK(cudaMemcpy(&e, PP.err.get(), sizeof(e), cudaMemcpyDeviceToHost));
    PP.used = false;
    if (e == 0) return;
    CK(cudaMemset(PP.err.get(), 0, sizeof(e)));
    throw Error(ICCG_ERR_CUDA, e == 0x40000000u   ? "persistent apply: wait for the update's reduction gave up"
                               : e == 0x40000001u ? "persistent apply: wait for a sweep's items gave up"
                                                  : "persistent apply: dependency wait gave up at ticket " +
                                                        std::to_string(e - 1));
}
