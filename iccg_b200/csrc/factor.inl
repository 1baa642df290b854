// factor.inl -- IC(0) factor built on the device (included by ctx.cu inside
// namespace iccg).

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
    {
        SetupPhase t("ic0.pattern");
        build_factor_pattern(c);
        CK(cudaStreamSynchronize(c->stream));
    }
    SetupPhase* tf = new SetupPhase("ic0.factor");
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
    CK(cudaStreamSynchronize(c->stream));
    delete tf;
    SetupPhase tsw("ic0.sweep_arrays");
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

