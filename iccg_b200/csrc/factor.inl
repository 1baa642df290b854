// factor.inl -- IC(0) factor built on the device (included by ctx.cu inside
// namespace iccg).

// ---------------------------------------------------------------------------
// IC(0) on the device
// ---------------------------------------------------------------------------
// L's layout, on the host and the device, and its initial values Lx0 (the
// lower part of A, ic0.cpp:42-44)
static void build_factor_pattern(iccg_ctx* c, std::vector<double>& Lx0)
{
    Factor& F = c->F;
    const int n = c->n;
    build_ic0_layout(n, c->h_rowptr.data(), c->h_colind.data(), c->h_val.data(), F, Lx0,
                     host_threads((long long)c->h_colind.size()));
    F.nnzL = (int)F.Li.size();
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
    std::vector<double> Lx0;  // A's lower entries: the factor's initial values
    {
        SetupPhase t("ic0.pattern");
        build_factor_pattern(c, Lx0);
    }
    std::optional<SetupPhase> tf(std::in_place, "ic0.factor");
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
    CK(cudaStreamSynchronize(c->stream));
    tf.reset();
    SetupPhase tsw("ic0.sweep_arrays");
    // sweep arrays
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
    gather(F.dpos, F.d64);
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

static void require_uploaded(iccg_ctx* c)
{
    if (c->n <= 0 && c->h_rowptr.empty()) throw Error(ICCG_ERR_STATE, "no matrix uploaded");
}

// a matrix with its sweep plans: the natural-order ones are built here when
// no schedule has replaced them since the upload
static void require_matrix(iccg_ctx* c)
{
    require_uploaded(c);
    if (c->plans_pending) {
        SetupPhase t("natural_order_plans");
        build_plans_none(c);
        c->plans_pending = false;
    }
}

static void require_precond(iccg_ctx* c)
{
    require_matrix(c);
    if (c->pc_kind < 0) throw Error(ICCG_ERR_STATE, "preconditioner not built");
    if (c->pc_kind == ICCG_PRECOND_IC0 && !c->F.built) throw Error(ICCG_ERR_STATE, "IC(0) factor not built");
}

