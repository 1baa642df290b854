// solver.inl -- kernel dispatch on the active path and the CG drivers
// (included by ctx.cu inside namespace iccg).
//
// Two paths compute the same bits: the lane-interleaved path (c->use_q,
// default; vectors in Q order, SELL-32 matrices) and the simple path (A_run
// order, one thread per row / per unit on CRS arrays).  The drivers below
// take vectors already in the active path's order.

// --- simple-path substitutions -------------------------------------------
template <class T, int FIN>
static void apply_ic0_simple(iccg_ctx* c, const double* r, double* y, double* z, SolverState* st)
{
    Factor& F = c->F;
    const bool f32 = std::is_same<T, float>::value;
    RedBuf red{c->partials.get(), c->scalars.get()};
    SweepArgs a{};
    a.unit_ptr = c->fwd.unit_is_row ? nullptr : c->fwd.unit_ptr.get();
    a.rows = c->fwd.rows.get();
    a.Sp = F.dSp.get();
    a.Si = F.dSi.get();
    a.Sx = f32 ? (const void*)F.S32.get() : (const void*)F.S64.get();
    a.d = f32 ? (const void*)F.d32.get() : (const void*)F.d64.get();
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
    b.Sx = f32 ? (const void*)F.T32.get() : (const void*)F.T64.get();
    b.in = y;
    b.out = z;
    b.rdot = r;
    for (int l = 0; l < c->bwd.nlevels; ++l) {
        const int u0 = c->bwd.level_ptr[(size_t)l], u1 = c->bwd.level_ptr[(size_t)l + 1];
        launch(c, 2, k_sweep<T, FIN>, c->bwd.grid[(size_t)l], kThreads, b, u0, u1, c->bwd.slot0[(size_t)l],
               c->bwd.nslots, st, red, c->ticket.get());
    }
}

// --- lane-interleaved substitutions -----------------------------------------
// Each level (color) of a sweep runs on one of four kernels:
//  0 chain-only (k_sweep_chain): rows whose entries are all in-unit, one per
//    row on the previous step, in full groups of at most 16 steps;
//  1 staged (k_sweep_st): FP32 storage, and FP64 forward sweeps -- the exact
//    FP64 backward order would park every gathered value in the tile (twice
//    the shared memory), where the per-slice kernel measured faster -- at
//    levels whose batches fit the stage budget;
//  2 per-slice two-phase (k_sweep_q2); 3 one-phase (k_sweep_q), for units of
//    more than 64 rows.
// The backward sweep's r.z reduction spans all its launches: slots are laid
// out level after level over the grids actually launched.
struct SweepLevel {
    int kind, grid;
};

template <class T>
static SweepLevel sweep_level(iccg_ctx* c, int l, bool fwd)
{
    QSys& Q = c->Q;
    constexpr bool f32 = std::is_same<T, float>::value;
    constexpr int k = f32 ? 1 : 0;
    const size_t l_ = (size_t)l;
    const bool st_ok = Q.staged && c->sweep_kernel == 0 && (!f32 || Q.r32_ok);
    if (st_ok && (fwd ? Q.chainS[l_] : Q.chainT[l_])) return {0, Q.ch_grid[k][l_]};
    if (st_ok && Q.st_fit[l_] && (f32 || (fwd && Q.st_fit64[l_]))) {
        if (c->stage_bufs == 1 || Q.st_one[l_]) return {1, fwd ? Q.st1_fgrid[k][l_] : Q.st1_bgrid[k][l_]};
        return {1, fwd ? Q.st_fgrid[k][l_] : Q.st_bgrid[k][l_]};
    }
    if (Q.two_phase) return {2, Q.g2grid[l_]};
    return {3, Q.fgrid[l_]};
}

// 1 if this storage's solves load before the wait on the previous launch
// (ICCG_OPT_EARLY)
static int early_on(const iccg_ctx* c, int storage)
{
    return (c->early >> (storage == ICCG_STORE_FP32 ? 0 : 1)) & 1;
}

template <class T, int FIN, bool FWD, int NI, int KS>
static void launch_q2_level(iccg_ctx* c, int l, int grid, const double* in, double* out, const double* rdot,
                            int slot0, int nslots, SolverState* st, const SellMat& M, const T* d)
{
    QSys& Q = c->Q;
    RedBuf red{c->partials.get(), c->scalars.get()};
    // FP64 storage keeps the reference's backward order exactly
    constexpr bool exact = FWD || !std::is_same<T, float>::value;
    const int slow = FWD ? (Q.S.max_nin > NI ? 1 : 0) : ((exact || Q.T.max_nin > NI) ? 1 : 0);
    const size_t smem = (size_t)Q.tile * 32 * sweep_row_bytes(sizeof(T), NI, slow != 0, FIN != FIN_NONE);
    launch_smem(c, FWD ? 1 : 2, k_sweep_q2<T, FWD, FIN, exact, NI, KS>, grid, kThreads, smem,
                Q.level_g[(size_t)l], Q.level_g[(size_t)l + 1], Q.gpc, Q.tile, slow, (const int*)Q.sl0.get(),
                (const int*)Q.glen.get(), (const SliceMeta*)Q.meta.get(), M, d, in, out, rdot, slot0, nslots, st, red,
                c->ticket.get());
}

// early (SP_IN / SP_RD): `in` / `rdot` were not written by the launch just
// before this level's, so the chain-only and staged kernels may load them
// before their wait on it
template <class T, int FIN, bool FWD>
static void launch_sweep_level(iccg_ctx* c, int l, const SweepLevel& sl, const double* in, double* out,
                               const double* rdot, int slot0, int nslots, SolverState* st, UpdArgs U = UpdArgs{},
                               int early = 0)
{
    QSys& Q = c->Q;
    constexpr bool f32 = std::is_same<T, float>::value;
    constexpr bool exact = !f32;
    const size_t l_ = (size_t)l;
    RedBuf red{c->partials.get(), c->scalars.get()};
    const SellMat M = FWD ? Q.S.view(f32) : Q.T.view(f32);
    // pivots: reciprocal for the FP32 staged / chain kernels, plain otherwise
    const T* dg = f32 ? (const T*)(const void*)Q.r32.get() : (const T*)(const void*)Q.d64.get();
    const T* d = f32 ? (const T*)(const void*)Q.d32.get() : (const T*)(const void*)Q.d64.get();
    const int cls = FWD ? 1 : 2;
    early = early_on(c, f32 ? ICCG_STORE_FP32 : ICCG_STORE_FP64) ? early | SP_EARLY : 0;
    switch (sl.kind) {
    case 0:
        launch(c, cls, k_sweep_chain<T, FWD, FIN, exact>, sl.grid, kThreads, Q.level_g[l_], Q.level_g[l_ + 1],
               (const int*)Q.glen.get(), (const int*)Q.sl0.get(), (const SliceMeta*)Q.meta.get(), M, dg, in, out,
               rdot, slot0, nslots, st, red, c->ticket.get(), U, early);
        break;
    case 1: {
        // a staged level of fewer than two CTAs per SM runs without loads
        // before the wait: with them the 96^3 27-point ABMC B=16 solve, whose
        // levels hold about one 512-row batch per SM, went 50.1 -> 58.7 ms
        if (sl.grid < 2 * c->nsm) early = 0;
        const int slots = FWD ? Q.st_slotsS[l_] : Q.st_slotsT[l_];
        const int nbuf = (c->stage_bufs == 1 || Q.st_one[l_]) ? 1 : 2;
        // the fused update stages Ap in the area of the backward sweep's r
        constexpr bool with_r = FIN == FIN_RZ || FIN == FIN_RZ0 || FIN == FIN_UPDX;
        const size_t smem = nbuf * (size_t)stage_layout(Q.st_rows[l_], slots, Q.st_slices[l_], (int)sizeof(T),
                                                        with_r, !FWD && exact)
                                       .bytes;
        const bool ew = (early & SP_EARLY) != 0;
        if constexpr (FIN == FIN_UPDX) {
            // the fused update runs single-buffered only (fused_update_ok)
            auto kern = ew ? k_sweep_st<T, FWD, FIN, exact, 1, true> : k_sweep_st<T, FWD, FIN, exact, 1>;
            allow_smem(c, kern);
            launch_smem(c, cls, kern, sl.grid, kThreads, smem, Q.lb[l_], Q.lb[l_ + 1],
                        (const BatchDesc*)Q.bdesc.get(), Q.st_rows[l_], slots, Q.st_slices[l_],
                        (const int*)Q.sl0.get(), (const int*)Q.glen.get(), (const SliceMeta*)Q.meta.get(), M, dg, in,
                        out, rdot, slot0, nslots, st, red, c->ticket.get(), U, early);
        } else {
            auto kern = nbuf == 1 ? (ew ? k_sweep_st<T, FWD, FIN, exact, 1, true> : k_sweep_st<T, FWD, FIN, exact, 1>)
                                  : (ew ? k_sweep_st<T, FWD, FIN, exact, 2, true> : k_sweep_st<T, FWD, FIN, exact, 2>);
            allow_smem(c, kern);
            launch_smem(c, cls, kern, sl.grid, kThreads, smem, Q.lb[l_], Q.lb[l_ + 1],
                        (const BatchDesc*)Q.bdesc.get(), Q.st_rows[l_], slots, Q.st_slices[l_],
                        (const int*)Q.sl0.get(), (const int*)Q.glen.get(), (const SliceMeta*)Q.meta.get(), M, dg, in,
                        out, rdot, slot0, nslots, st, red, c->ticket.get(), U, early);
        }
        break;
    }
    case 2:
        if (Q.ni == 1 && Q.ks == 8) launch_q2_level<T, FIN, FWD, 1, 8>(c, l, sl.grid, in, out, rdot, slot0, nslots, st, M, d);
        else if (Q.ni == 1) launch_q2_level<T, FIN, FWD, 1, 16>(c, l, sl.grid, in, out, rdot, slot0, nslots, st, M, d);
        else if (Q.ks == 8) launch_q2_level<T, FIN, FWD, 2, 8>(c, l, sl.grid, in, out, rdot, slot0, nslots, st, M, d);
        else launch_q2_level<T, FIN, FWD, 2, 16>(c, l, sl.grid, in, out, rdot, slot0, nslots, st, M, d);
        break;
    default:
        launch(c, cls, k_sweep_q<T, FWD, FIN>, sl.grid, kThreads, Q.level_g[l_], Q.level_g[l_ + 1],
               (const int*)Q.gbase.get(), (const int*)Q.glen.get(), (const int*)Q.sl0.get(), M, d, in, out, rdot,
               slot0, nslots, st, red, c->ticket.get());
        break;
    }
}

// true if every forward level runs on a kernel with the fused CG update
// (chain-only, or single-buffered staged)
template <class T>
static bool fused_update_ok(iccg_ctx* c)
{
    const QSys& Q = c->Q;
    if (!c->use_q || c->pc_kind != ICCG_PRECOND_IC0 || c->stage_bufs != 1 || !c->fuse_update) return false;
    for (int l = 0; l < Q.nlevels; ++l) {
        const int k = sweep_level<T>(c, l, true).kind;
        if (k != 0 && k != 1) return false;
        // the staged form also stages Ap: its buffer must still fit
        if (k == 1 && stage_layout(Q.st_rows[(size_t)l], Q.st_slotsS[(size_t)l], Q.st_slices[(size_t)l],
                                   (int)sizeof(T), true, false).bytes > c->smem_optin - 2048)
            return false;
    }
    return true;
}

// z = M^{-1} r.  UPD: the forward levels first do the CG update r -= alpha
// Ap of their rows (U; x += alpha p waits for the p update) and reduce r.r
// over all their launches (FIN_UPDX at the last CTA of the last forward
// level).
// f0 = 1: the first forward level was done by the update (k_update_chain),
// which also wrote r; the forward sweep starts at level 1.
template <class T, int FIN, bool UPD = false>
static void apply_ic0_q(iccg_ctx* c, const double* r, double* y, double* z, SolverState* st, UpdArgs U = UpdArgs{},
                        int f0 = 0)
{
    QSys& Q = c->Q;
    if (!UPD && use_persist(c, std::is_same<T, float>::value ? ICCG_STORE_FP32 : ICCG_STORE_FP64)) {
        launch_persist<T, false, FIN>(c, const_cast<double*>(r), y, z, st);
        return;
    }
    if (UPD) {
        std::vector<SweepLevel> fl((size_t)Q.nlevels);
        int fslots = 0;
        for (int l = 0; l < Q.nlevels; ++l) {
            fl[(size_t)l] = sweep_level<T>(c, l, true);
            fslots += fl[(size_t)l].grid;
        }
        int s0 = 0;
        for (int l = 0; l < Q.nlevels; ++l) {
            launch_sweep_level<T, FIN_UPDX, true>(c, l, fl[(size_t)l], r, y, nullptr, s0, fslots, st, U);
            s0 += fl[(size_t)l].grid;
        }
    } else {
        // the first level's r may come from the launch just before (the
        // update or a residual); the later levels' r does not
        for (int l = f0; l < Q.nlevels; ++l)
            launch_sweep_level<T, FIN_NONE, true>(c, l, sweep_level<T>(c, l, true), r, y, nullptr, 0, 0, st,
                                                  UpdArgs{}, l > f0 ? SP_IN : 0);
    }
    std::vector<SweepLevel> bl((size_t)Q.nlevels);
    int nslots = 0;
    for (int l = Q.nlevels - 1; l >= 0; --l) {
        bl[(size_t)l] = sweep_level<T>(c, l, false);
        nslots += bl[(size_t)l].grid;
    }
    int slot0 = 0;
    // the backward level l reads the y rows the forward level l wrote (and,
    // with the fused update, its r rows): the launch just before only for
    // the last level; without the fused update r is older, unless no
    // forward level ran after the update
    for (int l = Q.nlevels - 1; l >= 0; --l) {
        const int early = l < Q.nlevels - 1 ? SP_IN | SP_RD : (UPD || l < f0) ? 0 : SP_RD;
        launch_sweep_level<T, FIN, false>(c, l, bl[(size_t)l], y, z, r, slot0, nslots, st, UpdArgs{}, early);
        slot0 += bl[(size_t)l].grid;
    }
}

// z = M^{-1} r (IC0::apply, ic0.cpp:366-393; Identity / Jacobi apply)
template <int FIN>
static void apply_path(iccg_ctx* c, int storage, const double* r, double* z, SolverState* st)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    const bool f32 = storage == ICCG_STORE_FP32;
    if (c->pc_kind == ICCG_PRECOND_IC0) {
        if (c->use_q) {
            if (f32) apply_ic0_q<float, FIN>(c, r, c->vy.get(), z, st);
            else apply_ic0_q<double, FIN>(c, r, c->vy.get(), z, st);
        } else {
            if (f32) apply_ic0_simple<float, FIN>(c, r, c->vy.get(), z, st);
            else apply_ic0_simple<double, FIN>(c, r, c->vy.get(), z, st);
        }
        return;
    }
    const double* inv = nullptr;
    if (c->pc_kind == ICCG_PRECOND_JACOBI) inv = c->use_q ? c->Q.inv_diag.get() : c->inv_diag.get();
    launch_n(c, 3, k_diag_apply<FIN>, (long long)c->n, c->n, inv, r, z, st, red, c->ticket.get());
}

// y = A x (spmv, cg_crs.cpp:54-79); FIN_PAP adds p.Ap, p.p, Ap.Ap
template <int FIN>
static void spmv_path(iccg_ctx* c, int storage, const double* x, double* y, SolverState* st)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    const bool f32 = storage == ICCG_STORE_FP32;
    const int g = grid_for(c, c->n);
    if (c->use_q) {
        const SellMat A = c->Q.A.view(f32);
        const int ew = early_on(c, storage);
        // TPR threads per row: TPR times the threads, but every CTA writes its
        // reduction slot, so the grid stays within the slots the partial-sum
        // buffer holds (sized for one thread per row; the kernel strides)
        const long long w = (long long)c->n * c->spmv_tpr;
        auto qt_grid = [&](auto kern) {
            return (int)std::max(1ll, std::min<long long>(occ_grid(c, kern, w), (long long)c->partial_slots));
        };
        if (f32 && A.pk && c->spmv_tpr == 2)
            launch(c, 0, k_spmv_qt<2, FIN>, qt_grid(k_spmv_qt<2, FIN>), kThreads, c->n, A, x, y, st, red,
                   c->ticket.get());
        else if (f32 && A.pk && c->spmv_tpr == 4)
            launch(c, 0, k_spmv_qt<4, FIN>, qt_grid(k_spmv_qt<4, FIN>), kThreads, c->n, A, x, y, st, red,
                   c->ticket.get());
        else if (f32 && c->spmv_pack && A.pk)
            launch_n(c, 0, k_spmv_q<float, FIN, true>, (long long)c->n, c->n, A, x, y, st, red, c->ticket.get(), ew);
        else if (f32) launch_n(c, 0, k_spmv_q<float, FIN>, (long long)c->n, c->n, A, x, y, st, red, c->ticket.get(), ew);
        else launch_n(c, 0, k_spmv_q<double, FIN>, (long long)c->n, c->n, A, x, y, st, red, c->ticket.get(), ew);
        return;
    }
    const int* rp = c->rowptr.get();
    const int* ci = c->colind.get();
    if (f32)
        launch_n(c, 0, k_spmv<float, FIN>, (long long)c->n, c->n, rp, ci, (const float*)c->val32.get(), x, y, st, red,
               c->ticket.get());
    else
        launch_n(c, 0, k_spmv<double, FIN>, (long long)c->n, c->n, rp, ci, (const double*)c->val64.get(), x, y, st, red,
               c->ticket.get());
}

// r = b - A x with the FP64 matrix
template <int FIN>
static void residual_path(iccg_ctx* c, const double* x, const double* b, double* r, SolverState* st)
{
    RedBuf red{c->partials.get(), c->scalars.get()};
    const int g = grid_for(c, c->n);
    if (c->use_q)
        launch_n(c, 4, k_residual_q<FIN>, (long long)c->n, c->n, c->Q.A.view(false), x, b, r, st, red, c->ticket.get());
    else
        launch_n(c, 4, k_residual<FIN>, (long long)c->n, c->n, (const int*)c->rowptr.get(), (const int*)c->colind.get(),
               (const double*)c->val64.get(), x, b, r, st, red, c->ticket.get());
}

// makes the arrays of the active path ready (outside graph capture)
static void prepare_path(iccg_ctx* c, int storage)
{
    if (c->use_q) {
        ensure_q(c);
        if (storage == ICCG_STORE_FP32) ensure_q32(c);
        if (use_persist(c, storage)) {
            if (storage == ICCG_STORE_FP32) prepare_persist_t<float>(c);
            else prepare_persist_t<double>(c);
        }
    } else if (storage == ICCG_STORE_FP32) {
        ensure_val32(c);
        if (c->pc_kind == ICCG_PRECOND_IC0) ensure_factor32(c);
    }
}

static double dot_dev(iccg_ctx* c, int n, const double* a, const double* b)
{
    ensure_partials(c, (size_t)grid_for(c, n));
    RedBuf red{c->partials.get(), c->scalars.get()};
    launch_n(c, 3, k_dot, (long long)n, n, a, b, red, c->ticket.get());
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
    RedBuf red{c->partials.get(), c->scalars.get()};
    spmv_path<FIN_NONE>(c, ICCG_STORE_FP64, x, Ax, nullptr);
    launch_n(c, 3, k_sub, (long long)c->n, n, b, (const double*)Ax, r);
    double normb = std::sqrt(dot_dev(c, n, b, b));
    if (normb == 0.0) normb = 1.0;
    apply_path<FIN_NONE>(c, ICCG_STORE_FP64, r, z, nullptr);
    launch_n(c, 3, k_copy, (long long)c->n, n, (const double*)z, p, (SolverState*)nullptr);
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
        spmv_path<FIN_NONE>(c, ICCG_STORE_FP64, p, Ap, nullptr);
        const double pAp = dot_dev(c, n, p, Ap);
        const double eps = 2.220446049250313080847e-16;
        const double thr = eps * std::sqrt(dot_dev(c, n, p, p)) * std::sqrt(dot_dev(c, n, Ap, Ap));
        if (pAp <= thr) {
            res->iters = k;
            res->status = kBreakdown;
            return;
        }
        const double alpha = rz_old / pAp;
        launch_n(c, 3, k_update<FIN_NONE>, (long long)c->n, n, alpha, (const double*)p, (const double*)Ap, x, r,
               (SolverState*)nullptr, red, c->ticket.get(), early_on(c, ICCG_STORE_FP64));
        const double rel = std::sqrt(dot_dev(c, n, r, r)) / normb;
        res->iters = k + 1;
        res->rel_resid = rel;
        if (rel < tol) {
            res->converged = 1;
            res->status = kConverged;
            return;
        }
        apply_path<FIN_NONE>(c, ICCG_STORE_FP64, r, z, nullptr);
        const double rz_new = dot_dev(c, n, r, z);
        const double beta = rz_new / rz_old;
        launch_n(c, 3, k_xpay, (long long)c->n, n, beta, (const double*)z, p, (SolverState*)nullptr, (double*)nullptr,
                 early_on(c, ICCG_STORE_FP64));
        rz_old = rz_new;
    }
    res->status = kMaxIter;
}

// ---------------------------------------------------------------------------
// fused CG: device-side scalars, iterations replayed as a CUDA graph
// ---------------------------------------------------------------------------

// true if the update can take the first forward level (ICCG_OPT_UPDATE_CHAIN):
// IC(0) in Q order whose first forward level runs on the chain-only kernel,
// the plain update path (no persistent apply, fused update or deferred x) and
// 16-byte aligned vectors
template <class T>
static bool update_chain_ok(iccg_ctx* c, const double* x)
{
    if (!c->update_chain || !c->use_q || c->pc_kind != ICCG_PRECOND_IC0 || c->fuse_update || c->defer_x) return false;
    if (c->Q.nlevels < 1 || use_persist(c, std::is_same<T, float>::value ? ICCG_STORE_FP32 : ICCG_STORE_FP64))
        return false;
    if (sweep_level<T>(c, 0, true).kind != 0) return false;
    const uintptr_t a = (uintptr_t)x | (uintptr_t)c->vp.get() | (uintptr_t)c->vAp.get() | (uintptr_t)c->vr.get();
    return (a & 15) == 0;
}

template <class T>
static void update_chain(iccg_ctx* c, double* x, SolverState* st)
{
    QSys& Q = c->Q;
    constexpr bool f32 = std::is_same<T, float>::value;
    constexpr bool exact = !f32;
    auto kern = k_update_chain<T, exact>;
    int per = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kThreads, 0));
    const int groups = Q.level_g[1] - Q.level_g[0];
    // a full wave; the chains want one warp per group
    int grid = std::max(1, per) * c->nsm;
    grid = std::max(grid, std::min((groups + 7) / 8, 8 * c->nsm));
    grid = std::min(grid, (int)c->partial_slots);
    const int n0 = Q.h_gbase[(size_t)Q.level_g[1]];
    const T* dg = f32 ? (const T*)(const void*)Q.r32.get() : (const T*)(const void*)Q.d64.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    launch(c, 3, kern, grid, kThreads, Q.level_g[0], Q.level_g[1], (const int*)Q.glen.get(), (const int*)Q.sl0.get(),
           (const SliceMeta*)Q.meta.get(), Q.S.view(f32), dg, n0, c->n, (const double*)c->vp.get(),
           (const double*)c->vAp.get(), x, c->vr.get(), c->vy.get(), st, red, c->ticket.get(),
           early_on(c, f32 ? ICCG_STORE_FP32 : ICCG_STORE_FP64));
}
static void fused_iteration(iccg_ctx* c, int storage, bool rr, const double* b, double* x)
{
    const int n = c->n;
    const int g = grid_for(c, n);
    SolverState* st = c->state.get();
    RedBuf red{c->partials.get(), c->scalars.get()};
    spmv_path<FIN_PAP>(c, storage, (const double*)c->vp.get(), c->vAp.get(), st);
    if (!rr && use_persist(c, storage)) {
        // update, both sweeps and the two reductions in one launch
        if (storage == ICCG_STORE_FP32) launch_persist<float, true, FIN_RZ>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, x);
        else launch_persist<double, true, FIN_RZ>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, x);
        launch_n(c, 3, k_xpay, (long long)c->n, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st, (double*)nullptr,
                 early_on(c, storage));
        return;
    }
    const bool f32 = storage == ICCG_STORE_FP32;
    if (!rr && (f32 ? fused_update_ok<float>(c) : fused_update_ok<double>(c))) {
        // the update inside the forward sweep's launches
        const UpdArgs U{c->vr.get(), c->vAp.get()};
        if (f32) apply_ic0_q<float, FIN_RZ, true>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, U);
        else apply_ic0_q<double, FIN_RZ, true>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, U);
        // x += alpha p, then p = z + beta p
        launch_n(c, 3, k_xpay, (long long)c->n, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st, x,
                 early_on(c, storage));
        return;
    }
    if (!rr && (f32 ? update_chain_ok<float>(c, x) : update_chain_ok<double>(c, x))) {
        // the update with the first forward level (chain-only) in its launch
        if (f32) update_chain<float>(c, x, st);
        else update_chain<double>(c, x, st);
        if (f32) apply_ic0_q<float, FIN_RZ>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, UpdArgs{}, 1);
        else apply_ic0_q<double, FIN_RZ>(c, c->vr.get(), c->vy.get(), c->vz.get(), st, UpdArgs{}, 1);
        launch_n(c, 3, k_xpay, (long long)c->n, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st, (double*)nullptr,
                 early_on(c, storage));
        return;
    }
    // x += alpha p with the p update (defer_x), except where the FP64
    // residual of this iteration needs the new x
    const bool dx = c->defer_x && !rr;
    const int ew = early_on(c, storage);
    if (dx)
        launch_n(c, 3, k_update<FIN_UPDX>, (long long)c->n, n, 0.0, (const double*)c->vp.get(),
                 (const double*)c->vAp.get(), x, c->vr.get(), st, red, c->ticket.get(), ew);
    else
        launch_n(c, 3, k_update<FIN_UPD>, (long long)c->n, n, 0.0, (const double*)c->vp.get(),
                 (const double*)c->vAp.get(), x, c->vr.get(), st, red, c->ticket.get(), ew);
    if (rr) residual_path<FIN_TRUE>(c, (const double*)x, b, c->vr.get(), st);
    apply_path<FIN_RZ>(c, storage, c->vr.get(), c->vz.get(), st);
    launch_n(c, 3, k_xpay, (long long)c->n, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st,
             dx ? x : (double*)nullptr, ew);
}

// releases every captured iteration graph of the context
static void drop_graph(iccg_ctx* c)
{
    for (auto& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
    c->gkey_valid = false;
}

static void solve_fused(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, const iccg_solve_opts& o,
                        iccg_result* res)
{
    const int n = c->n;
    const int storage = o.storage;
    const bool rr = storage == ICCG_STORE_FP32 && o.rr_interval > 0;
    SolverState s0{};
    s0.tol = tol;
    s0.status = kRunning;
    s0.pend = kRunning;
    s0.max_iter = max_iter;
    s0.rr_interval = rr ? o.rr_interval : 0;
    s0.xdefer_k = -1;
    *c->h_state = s0;
    CK(cudaMemcpyAsync(c->state.get(), c->h_state, sizeof(SolverState), cudaMemcpyHostToDevice, c->stream));
    unsigned int zero = 0;
    CK(cudaMemcpyAsync(c->ticket.get(), &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    const int g = grid_for(c, n);
    SolverState* st = c->state.get();
    // r0 = b - A x0, ||b||, z0 = M^{-1} r0, rz, p = z  (cg_crs.cpp:102-123)
    residual_path<FIN_INIT>(c, (const double*)x, b, c->vr.get(), st);
    apply_path<FIN_RZ0>(c, storage, c->vr.get(), c->vz.get(), st);
    launch_n(c, 3, k_copy, (long long)c->n, n, (const double*)c->vz.get(), c->vp.get(), st);

    const int m = std::max(1, o.graph_iters);
    const bool use_graph = !c->profile;
    // residual replacement every rr_interval iterations happens at iterations
    // the host can name: a batch of m iterations starting at iteration k0
    // carries the replacement kernel only where (k + 1) % rr_interval == 0
    const int rri = rr ? o.rr_interval : 0;
    auto rr_mask = [&](long long k0, int sz) {
        unsigned mk = 0;
        if (rri > 0)
            for (int it = 0; it < sz && it < 32; ++it)
                if ((k0 + it + 1) % rri == 0) mk |= 1u << it;
        return mk;
    };
    auto one_batch = [&](unsigned mk, int sz) {
        for (int it = 0; it < sz; ++it) fused_iteration(c, storage, it < 32 && ((mk >> it) & 1u), b, x);
    };
    GraphKey key;
    key.sched_version = c->sched_version;
    key.factor_version = c->factor_version;
    key.storage = storage;
    key.rri = rri;
    key.use_q = c->use_q ? 1 : 0;
    key.m = m;
    key.pc_kind = c->pc_kind;
    key.sweep_kernel = c->sweep_kernel;
    key.x = x;
    key.b = b;
    if (use_graph && (!c->gkey_valid || c->gkey != key)) {
        drop_graph(c);
        c->gkey = key;
        c->gkey_valid = true;
    }
    auto graph_for = [&](unsigned mk, int sz) -> iccg_ctx::GraphEntry& {
        for (auto& g : c->graphs)
            if (g.mask == mk && g.size == sz) return g;
        cudaGraph_t graph = nullptr;
        const long long before = c->launches;
        SetupPhase tg("solve.graph_capture");
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        try {
            one_batch(mk, sz);
        } catch (...) {
            cudaStreamEndCapture(c->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        CK(cudaStreamEndCapture(c->stream, &graph));
        iccg_ctx::GraphEntry e{mk, sz, nullptr, 0};
        const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
        cudaGraphDestroy(graph);
        CK(ie);
        e.kernels = (int)(c->launches - before);
        c->launches = before;
        c->graphs.push_back(e);
        return c->graphs.back();
    };
    auto run_batch = [&](long long k0, int sz) {
        const unsigned mk = rr_mask(k0, sz);
        if (use_graph) {
            auto& g = graph_for(mk, sz);
            CK(cudaGraphLaunch(g.exec, c->stream));
            c->launches += g.kernels;
        } else {
            one_batch(mk, sz);
        }
    };
    // Batches of iterations are launched ahead: the state after batch i - 1
    // is read while batch i runs, and a batch that finds the solve stopped
    // does nothing.  Near the end the recurrence residual's decay per
    // iteration, from the last two reads, predicts the stop: no batch is
    // queued past the predicted iteration, and the last batches shrink to
    // 4, 2 or 1 iterations, so few iterations run on after the stop.  A wrong
    // prediction costs one more read, never an iteration.
    const double ltol = std::log(tol);
    long long k_base = 0;  // iterations completed before the current run of batches
    for (;;) {
        long long k_next = k_base;  // first iteration of the next batch
        int nl = 0, nr = 0;         // batches launched / read
        bool have1 = false, have2 = false;
        long long k_last = 0, k_prev = 0;
        double lr_last = 0.0, lr_prev = 0.0;
        for (;;) {
            int sz = m;
            if (have2 && lr_last < lr_prev && k_last > k_prev) {
                const double slope = (lr_last - lr_prev) / (double)(k_last - k_prev);
                const double left = (ltol - lr_last) / slope - (double)(k_next - k_last);
                if (left <= 0.0) sz = 0;
                else if (left < (double)m) sz = left > 4.0 ? std::min(m, 4) : left > 2.0 ? std::min(m, 2) : 1;
            }
            if (sz == 0 && nl == nr) sz = 1;
            if (k_next >= (long long)max_iter + m) sz = 0;
            if (sz > 0 && nl - nr < 2) {
                run_batch(k_next, sz);
                k_next += sz;
                CK(cudaMemcpyAsync(&c->h_obs[nl & 1], st, sizeof(SolverState), cudaMemcpyDeviceToHost, c->stream));
                CK(cudaEventRecord(c->evs[nl & 1], c->stream));
                ++nl;
                if (nl - nr < 2) continue;  // keep one batch queued behind the one running
            }
            if (nl == nr) break;  // nothing to read: past max_iter
            CK(cudaEventSynchronize(c->evs[nr & 1]));
            const SolverState& ob = c->h_obs[nr & 1];
            ++nr;
            if (ob.status != kRunning) break;
            if (ob.k > k_last || !have1) {
                k_prev = k_last;
                lr_prev = lr_last;
                have2 = have1;
                k_last = ob.k;
                lr_last = std::log(std::max(ob.rel_resid, 1e-300));
                have1 = true;
            }
        }
        CK(cudaStreamSynchronize(c->stream));
        CK(cudaMemcpyAsync(c->h_state, st, sizeof(SolverState), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (c->h_state->status != kTrueCheck) break;
        // The recurrence residual passed the tolerance: replace it by the
        // FP64 residual b - A x (cg_crs.cpp:518-528 semantics), test that,
        // and, if it is not below the tolerance, finish this iteration
        // (z = M^-1 r, beta, p) and go on.
        CK(cudaStreamSynchronize(c->stream));
        // x += alpha p where the fused update left it to the p update
        launch_n(c, 3, k_apply_xp, (long long)c->n, n, (const double*)c->vp.get(), x, (const SolverState*)st);
        launch(c, 3, k_clear_xp, 1, 1, st);
        launch(c, 3, k_resume_true_check, 1, 1, st);
        residual_path<FIN_TRUE>(c, (const double*)x, b, c->vr.get(), st);
        apply_path<FIN_RZ>(c, storage, c->vr.get(), c->vz.get(), st);
        launch_n(c, 3, k_xpay, (long long)c->n, n, 0.0, (const double*)c->vz.get(), c->vp.get(), st, (double*)nullptr,
                 early_on(c, storage));
        CK(cudaMemcpyAsync(c->h_state, st, sizeof(SolverState), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (c->h_state->status != kRunning) break;
        k_base = c->h_state->k;
    }
    // a stop between the fused update and the p update leaves x += alpha p
    launch_n(c, 3, k_apply_xp, (long long)c->n, n, (const double*)c->vp.get(), x, (const SolverState*)st);
    launch(c, 3, k_clear_xp, 1, 1, st);
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
    residual_path<FIN_NONE>(c, x, b, c->vtmp.get(), nullptr);
    const double nr = dot_dev(c, c->n, c->vtmp.get(), c->vtmp.get());
    const double nb = dot_dev(c, c->n, b, b);
    return std::sqrt(nr) / std::sqrt(nb);
}

// conjugate_gradient with b, x in A_run order on the device
static void solve_dev(iccg_ctx* c, const double* b, double* x, int max_iter, double tol, const iccg_solve_opts* opts,
                      iccg_result* res)
{
    require_precond(c);
    iccg_solve_opts o{ICCG_MODE_FUSED, ICCG_STORE_FP64, 50, kGraphIters};
    if (opts) o = *opts;
    if (o.graph_iters <= 0) o.graph_iters = kGraphIters;
    if (o.mode == ICCG_MODE_PLAIN && o.storage != ICCG_STORE_FP64)
        throw Error(ICCG_ERR_ARG, "the plain path computes in FP64 storage only");
    std::memset(res, 0, sizeof(*res));
    prepare_path(c, o.storage);
    const double* bp = b;
    double* xp = x;
    const int g = grid_for(c, c->n);
    if (c->use_q) {
        launch_n(c, 3, k_gather_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), b, c->qb.get());
        launch_n(c, 3, k_gather_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), (const double*)x, c->qx.get());
        bp = c->qb.get();
        xp = c->qx.get();
    }
    if (o.mode == ICCG_MODE_PLAIN) {
        CK(cudaEventRecord(c->ev0, c->stream));
        solve_plain(c, bp, xp, max_iter, tol, res);
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    } else {
        solve_fused(c, bp, xp, max_iter, tol, o, res);
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    res->solve_ms = ms;
    collect_profile(c);
    check_persist(c);
    // A converged FP32-storage solve ends on a residual replacement, whose
    // convergence test is already ||b - A x|| / ||b|| with the FP64 matrix.
    if (o.mode == ICCG_MODE_FUSED && o.storage == ICCG_STORE_FP32 && o.rr_interval > 0 && res->converged)
        res->true_rel_resid = res->rel_resid;
    else
        res->true_rel_resid = true_resid(c, bp, xp);
    if (c->use_q) launch_n(c, 3, k_scatter_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), (const double*)xp, x);
    CK(cudaStreamSynchronize(c->stream));
}

// z = M^{-1} r and y = A x with vectors in A_run order on the device
static void apply_dev(iccg_ctx* c, int storage, const double* r, double* z)
{
    require_precond(c);
    prepare_path(c, storage);
    const int g = grid_for(c, c->n);
    if (c->use_q) {
        launch_n(c, 3, k_gather_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), r, c->qb.get());
        apply_path<FIN_NONE>(c, storage, c->qb.get(), c->qx.get(), nullptr);
        launch_n(c, 3, k_scatter_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), (const double*)c->qx.get(), z);
    } else {
        apply_path<FIN_NONE>(c, storage, r, z, nullptr);
    }
    CK(cudaStreamSynchronize(c->stream));
    collect_profile(c);
    check_persist(c);
}

static void spmv_dev(iccg_ctx* c, int storage, const double* x, double* y)
{
    require_matrix(c);
    prepare_path(c, storage);
    const int g = grid_for(c, c->n);
    if (c->use_q) {
        launch_n(c, 3, k_gather_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), x, c->qb.get());
        spmv_path<FIN_NONE>(c, storage, c->qb.get(), c->qx.get(), nullptr);
        launch_n(c, 3, k_scatter_vec, (long long)c->n, c->n, (const int*)c->Q.dq2r.get(), (const double*)c->qx.get(), y);
    } else {
        spmv_path<FIN_NONE>(c, storage, x, y, nullptr);
    }
    CK(cudaStreamSynchronize(c->stream));
    collect_profile(c);
}

static void ensure_vectors(iccg_ctx* c)
{
    const size_t n = (size_t)c->n;
    for (Buf<double>* v : {&c->vb, &c->vx, &c->qb, &c->qx, &c->vr, &c->vp, &c->vz, &c->vy, &c->vAp, &c->vtmp})
        v->alloc(n, &c->dev_bytes);
    ensure_partials(c, (size_t)grid_for(c, c->n));
}
