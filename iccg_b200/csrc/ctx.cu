// ctx.cu -- the C ABI of include/iccg.h over the device context.
//
// One CUDA translation unit: the kernels (kernels.cuh) and the host code
// that plans, factors and solves (plan.inl, factor.inl, qsys.inl,
// solver.inl) are compiled together here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/iccg.h"
#include "context.hpp"

namespace iccg {

extern thread_local std::string g_host_err;  // host_capi.cpp

#include "plan.inl"
#include "factor.inl"
#include "qsys.inl"
#include "persist.inl"
#include "solver.inl"
#include "batch.inl"

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

template <class F>
static int bguard(iccg_batch* B, F&& f)
{
    if (!B) return ICCG_ERR_ARG;
    try {
        CK(cudaSetDevice(B->device));
        f();
        return ICCG_OK;
    } catch (const Error& e) {
        B->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        B->err = "out of host memory";
        return ICCG_ERR_NOMEM;
    } catch (const std::exception& e) {
        B->err = e.what();
        return ICCG_ERR_ARG;
    }
}

}  // namespace iccg

using namespace iccg;

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
        CK(cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        CK(cudaEventCreateWithFlags(&c->evs[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->evs[1], cudaEventDisableTiming));
        CK(cudaMallocHost(&c->h_state, sizeof(SolverState)));
        CK(cudaMallocHost(&c->h_scalars, 8 * sizeof(double)));
        CK(cudaMallocHost(&c->h_status, 2 * sizeof(int)));
        CK(cudaMallocHost(&c->h_obs, 2 * sizeof(SolverState)));
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
    drop_graph(c);
    for (auto& e : c->ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto e : c->evs)
        if (e) cudaEventDestroy(e);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_obs) cudaFreeHost(c->h_obs);
    cudaStream_t s = c->stream;
    delete c;  // device buffers free themselves
    if (s) cudaStreamDestroy(s);
    return ICCG_OK;
}

const char* iccg_ctx_last_error(const iccg_ctx* c) { return c ? c->err.c_str() : "null context"; }
void* iccg_ctx_stream(iccg_ctx* c) { return c ? (void*)c->stream : nullptr; }
long long iccg_ctx_launch_count(const iccg_ctx* c) { return c ? c->launches : 0; }
long long iccg_ctx_device_bytes(const iccg_ctx* c) { return c ? c->dev_bytes : 0; }

int iccg_ctx_set_option(iccg_ctx* c, int option, long long value)
{
    return guard(c, [&] {
        if (option == ICCG_OPT_TILED) {
            c->use_q = value != 0;
        } else if (option == ICCG_OPT_SWEEP) {
            if (value != 0 && value != 1) throw Error(ICCG_ERR_ARG, "ICCG_OPT_SWEEP takes 0 or 1");
            c->sweep_kernel = (int)value;
        } else if (option == ICCG_OPT_PDL) {
            c->pdl = value != 0;
        } else if (option == ICCG_OPT_PERSIST) {
            c->persist = value != 0;
        } else if (option == ICCG_OPT_FUSE_UPDATE) {
            c->fuse_update = value != 0;
        } else if (option == ICCG_OPT_DEFER_X) {
            c->defer_x = value != 0;
        } else if (option == ICCG_OPT_SPMV_PACK) {
            c->spmv_pack = value != 0;
        } else if (option == ICCG_OPT_SPMV_TPR) {
            if (value != 1 && value != 2 && value != 4) throw Error(ICCG_ERR_ARG, "ICCG_OPT_SPMV_TPR takes 1, 2 or 4");
            c->spmv_tpr = (int)value;
        } else if (option == ICCG_OPT_UPDATE_CHAIN) {
            c->update_chain = value != 0;
        } else if (option == ICCG_OPT_EARLY) {
            if (value < 0 || value > 3) throw Error(ICCG_ERR_ARG, "ICCG_OPT_EARLY takes 0 to 3");
            c->early = (int)value;
        } else if (option == ICCG_OPT_STAGE_BUFS) {
            if (value != 1 && value != 2) throw Error(ICCG_ERR_ARG, "ICCG_OPT_STAGE_BUFS takes 1 or 2");
            c->stage_bufs = (int)value;
        } else if (option == ICCG_OPT_STAGE_ROWS) {
            if (value < 32 || value > 8192) throw Error(ICCG_ERR_ARG, "ICCG_OPT_STAGE_ROWS takes 32 to 8192");
            c->stage_rows = (int)value;
            if (c->Q.two_phase && !c->Q.steps.empty()) {
                CK(cudaStreamSynchronize(c->stream));
                plan_staged(c);
                build_persist(c);
            }
        } else if (option == ICCG_OPT_STAGE_KB) {
            if (value < 0 || value > 1024) throw Error(ICCG_ERR_ARG, "ICCG_OPT_STAGE_KB takes 0 to 1024");
            c->stage_kb = (int)value;
            if (c->Q.two_phase && !c->Q.steps.empty()) {
                CK(cudaStreamSynchronize(c->stream));
                plan_staged(c);
                build_persist(c);
            }
        } else {
            throw Error(ICCG_ERR_ARG, "unknown option");
        }
        drop_graph(c);
    });
}

int iccg_matrix_upload(iccg_ctx* c, int n, const int* rowptr, const int* colind, const double* val)
{
    return guard(c, [&] {
        SetupPhase all("upload");
        if (n <= 0 || !rowptr || !colind || !val) throw Error(ICCG_ERR_ARG, "bad matrix arguments");
        if (rowptr[0] != 0) throw Error(ICCG_ERR_ARG, "rowptr[0] must be 0");
        std::optional<SetupPhase> v(std::in_place, "upload.validate");
        for (int i = 0; i < n; ++i) {
            if (rowptr[i + 1] < rowptr[i]) throw Error(ICCG_ERR_ARG, "rowptr must be nondecreasing");
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
                if (colind[k] < 0 || colind[k] >= n) throw Error(ICCG_ERR_ARG, "column index out of range");
                if (k > rowptr[i] && colind[k] <= colind[k - 1])
                    throw Error(ICCG_ERR_ARG, "columns must be strictly ascending within each row");
            }
        }
        v.reset();
        drop_graph(c);
        const int nnz = rowptr[n];
        c->n = n;
        c->nnz = nnz;
        {
            SetupPhase t("upload.host_copy");
            size_for_fill(c->h_rowptr, (size_t)n + 1);
            size_for_fill(c->h_colind, (size_t)nnz);
            size_for_fill(c->h_val, (size_t)nnz);
            std::copy(rowptr, rowptr + n + 1, c->h_rowptr.begin());
            std::copy(colind, colind + nnz, c->h_colind.begin());
            std::copy(val, val + nnz, c->h_val.begin());
        }
        {
            SetupPhase t("upload.device_copy");
            c->rowptr.upload(rowptr, (size_t)n + 1, &c->dev_bytes, c->stream);
            c->colind.upload(colind, (size_t)nnz, &c->dev_bytes, c->stream);
            c->val64.upload(val, (size_t)nnz, &c->dev_bytes, c->stream);
            c->val32.free();
            c->has_val32 = false;
            ensure_vectors(c);
            CK(cudaStreamSynchronize(c->stream));
        }
        // a new matrix invalidates the schedule and the preconditioner
        c->pc_kind = -1;
        c->F.reset();
        c->Q.reset();
        c->sched_kind = ICCG_SCHED_NONE;
        c->plans_pending = true;
        c->sched_version++;
        c->factor_version++;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_mc(iccg_ctx* c, int nc, const int* color_ptr, const int* rows_of_color)
{
    return guard(c, [&] {
        require_uploaded(c);
        drop_graph(c);
        // until the new plans are complete the context is in the natural order
        c->sched_kind = ICCG_SCHED_NONE;
        c->plans_pending = true;
        c->sched_version++;
        build_plans_mc(c, nc, color_ptr, rows_of_color);
        c->plans_pending = false;
        c->sched_kind = ICCG_SCHED_MC;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_abmc(iccg_ctx* c, int nc, int nb, const int* color_ptr_blk, const int* blocks_of_color,
                       const int* block_ptr, const int* rows_of_block)
{
    return guard(c, [&] {
        require_uploaded(c);
        drop_graph(c);
        // until the new plans are complete the context is in the natural order
        c->sched_kind = ICCG_SCHED_NONE;
        c->plans_pending = true;
        c->sched_version++;
        build_plans_abmc(c, nc, nb, color_ptr_blk, blocks_of_color, block_ptr, rows_of_block);
        c->plans_pending = false;
        c->sched_kind = ICCG_SCHED_ABMC;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int iccg_schedule_none(iccg_ctx* c)
{
    return guard(c, [&] {
        require_uploaded(c);
        drop_graph(c);
        build_plans_none(c);
        c->plans_pending = false;
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
        drop_graph(c);
        c->factor_version++;
        if (kind == ICCG_PRECOND_NONE) {
            c->inv_diag.free();
        } else if (kind == ICCG_PRECOND_JACOBI) {
            // Jacobi::Jacobi (precond.hpp:23-36)
            std::vector<double> inv((size_t)c->n, 1.0);
            for (int i = 0; i < c->n; ++i) {
                double d = 0.0;
                for (int k = c->h_rowptr[(size_t)i]; k < c->h_rowptr[(size_t)i + 1]; ++k)
                    if (c->h_colind[(size_t)k] == i) {
                        d = c->h_val[(size_t)k];
                        break;
                    }
                inv[(size_t)i] = (std::fabs(d) > 0.0) ? 1.0 / d : 1.0;
            }
            c->inv_diag.upload(inv.data(), inv.size(), &c->dev_bytes, c->stream);
            CK(cudaStreamSynchronize(c->stream));
        } else if (kind == ICCG_PRECOND_IC0) {
            SetupPhase t("precond_build.ic0");
            build_ic0(c, shift, auto_shift != 0);
        } else {
            throw Error(ICCG_ERR_ARG, "unknown preconditioner kind");
        }
        c->pc_kind = kind;
        c->factor_version++;
    });
}

double iccg_precond_shift(const iccg_ctx* c) { return c ? c->F.shift : 0.0; }

int iccg_precond_apply_dev(iccg_ctx* c, const double* r, double* z, int storage)
{
    return guard(c, [&] { apply_dev(c, storage, r, z); });
}

int iccg_precond_apply(iccg_ctx* c, const double* r, double* z, int storage)
{
    return guard(c, [&] {
        require_precond(c);
        const size_t bytes = sizeof(double) * (size_t)c->n;
        CK(cudaMemcpyAsync(c->vb.get(), r, bytes, cudaMemcpyHostToDevice, c->stream));
        apply_dev(c, storage, c->vb.get(), c->vx.get());
        CK(cudaMemcpyAsync(z, c->vx.get(), bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
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
        if (Ux)
            for (size_t k = 0; k < F.ut_src.size(); ++k) Ux[k] = lx[(size_t)F.ut_src[k]];
    });
}

int iccg_spmv_dev(iccg_ctx* c, const double* x, double* y, int storage)
{
    return guard(c, [&] { spmv_dev(c, storage, x, y); });
}

int iccg_spmv(iccg_ctx* c, const double* x, double* y, int storage)
{
    return guard(c, [&] {
        require_matrix(c);
        const size_t bytes = sizeof(double) * (size_t)c->n;
        CK(cudaMemcpyAsync(c->vb.get(), x, bytes, cudaMemcpyHostToDevice, c->stream));
        spmv_dev(c, storage, c->vb.get(), c->vx.get());
        CK(cudaMemcpyAsync(y, c->vx.get(), bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
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

int iccg_profile_enable(iccg_ctx* c, int enable)
{
    return guard(c, [&] {
        c->profile = enable != 0;
        for (int k = 0; k < 6; ++k) {
            c->prof_ms[k] = 0.0;
            c->prof_n[k] = 0;
        }
    });
}

int iccg_profile_read(iccg_ctx* c, int cls, double* total_ms, long long* launches)
{
    if (!c || cls < 0 || cls >= 6) return ICCG_ERR_ARG;
    if (total_ms) *total_ms = c->prof_ms[cls];
    if (launches) *launches = c->prof_n[cls];
    return ICCG_OK;
}

int iccg_sweep_plan(iccg_ctx* c, int storage, int fwd, int* kinds, int* grids, int cap, int* nlevels)
{
    return guard(c, [&] {
        if (!nlevels || cap < 0 || (cap > 0 && (!kinds || !grids))) throw Error(ICCG_ERR_ARG, "bad argument");
        if (storage != ICCG_STORE_FP64 && storage != ICCG_STORE_FP32) throw Error(ICCG_ERR_ARG, "bad storage");
        require_precond(c);
        if (c->pc_kind != ICCG_PRECOND_IC0) throw Error(ICCG_ERR_STATE, "preconditioner has no substitution sweeps");
        prepare_path(c, storage);
        const bool f32 = storage == ICCG_STORE_FP32;
        if (!c->use_q) {
            const Plan& P = fwd ? c->fwd : c->bwd;
            *nlevels = P.nlevels;
            for (int l = 0; l < std::min(cap, P.nlevels); ++l) {
                kinds[l] = 4;
                grids[l] = P.grid[(size_t)l];
            }
            return;
        }
        *nlevels = c->Q.nlevels;
        if (use_persist(c, storage)) {
            // every level in the one persistent launch
            const PersistVar& V = f32 ? persist_var<float, false, FIN_NONE>(c, 4 + PK_PLAIN)
                                      : persist_var<double, false, FIN_NONE>(c, PK_PLAIN);
            for (int l = 0; l < std::min(cap, c->Q.nlevels); ++l) {
                kinds[l] = 5;
                grids[l] = V.grid;
            }
            return;
        }
        for (int l = 0; l < std::min(cap, c->Q.nlevels); ++l) {
            const SweepLevel s = f32 ? sweep_level<float>(c, l, fwd != 0) : sweep_level<double>(c, l, fwd != 0);
            kinds[l] = s.kind;
            grids[l] = s.grid;
        }
    });
}

// ---------------------------------------------------------------------------
// batched solves
// ---------------------------------------------------------------------------
static void batch_free(iccg_batch* B)
{
    bat::drop_graph(B);
    if (B->ev0) cudaEventDestroy(B->ev0);
    if (B->ev1) cudaEventDestroy(B->ev1);
    for (auto e : B->evs)
        if (e) cudaEventDestroy(e);
    if (B->h_running) cudaFreeHost(B->h_running);
    if (B->h_status) cudaFreeHost(B->h_status);
    cudaStream_t s = B->stream;
    delete B;  // device buffers free themselves
    if (s) cudaStreamDestroy(s);
}

int iccg_batch_create(int device, iccg_batch** out)
{
    if (!out) return ICCG_ERR_ARG;
    *out = nullptr;
    auto* B = new iccg_batch;
    B->device = device;
    const int rc = bguard(B, [&] {
        int ndev = 0;
        CK(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw Error(ICCG_ERR_ARG, "no such CUDA device");
        CK(cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, device));
        CK(cudaDeviceGetAttribute(&B->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        CK(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&B->ev0));
        CK(cudaEventCreate(&B->ev1));
        CK(cudaEventCreateWithFlags(&B->evs[0], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&B->evs[1], cudaEventDisableTiming));
        CK(cudaMallocHost(&B->h_running, 2 * sizeof(int)));
    });
    if (rc) {
        iccg::g_host_err = B->err;
        batch_free(B);
        return rc;
    }
    *out = B;
    return ICCG_OK;
}

int iccg_batch_destroy(iccg_batch* B)
{
    if (!B) return ICCG_OK;
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    batch_free(B);
    return ICCG_OK;
}

const char* iccg_batch_last_error(const iccg_batch* B) { return B ? B->err.c_str() : "null batch"; }
long long iccg_batch_launch_count(const iccg_batch* B) { return B ? B->launches : 0; }
long long iccg_batch_device_bytes(const iccg_batch* B) { return B ? B->dev_bytes : 0; }
double iccg_batch_device_ms(const iccg_batch* B) { return B ? B->last_ms : 0.0; }

int iccg_batch_add_system(iccg_batch* B, iccg_ctx* ctx, int* index)
{
    return bguard(B, [&] {
        if (!ctx || !index) throw Error(ICCG_ERR_ARG, "null argument");
        if (ctx->device != B->device) throw Error(ICCG_ERR_ARG, "context on another device");
        require_precond(ctx);
        for (const auto& h : B->sys)
            if (h->c == ctx) throw Error(ICCG_ERR_ARG, "context already in the batch");
        // a free entry (a removed system) is reused
        int k = -1;
        for (size_t i = 0; i < B->sys.size(); ++i)
            if (!B->sys[i]->c) {
                k = (int)i;
                break;
            }
        if (k < 0) {
            B->sys.push_back(std::make_unique<bat::SysHost>());
            k = (int)B->sys.size() - 1;
        }
        bat::SysHost& H = *B->sys[(size_t)k];
        H.c = ctx;
        H.storage = -1;
        H.active = 0;
        B->sys_dirty = true;
        *index = k;
    });
}

int iccg_batch_remove_system(iccg_batch* B, int index)
{
    return bguard(B, [&] {
        if (index < 0 || index >= (int)B->sys.size() || !B->sys[(size_t)index]->c)
            throw Error(ICCG_ERR_ARG, "no such system in the batch");
        bat::SysHost& H = *B->sys[(size_t)index];
        if (H.active) throw Error(ICCG_ERR_STATE, "the system has solves in the batch");
        CK(cudaStreamSynchronize(B->stream));
        H.c = nullptr;
        H.storage = -1;
        H.bdb.release();
        B->sys_dirty = true;
    });
}

int iccg_batch_clear(iccg_batch* B)
{
    return bguard(B, [&] {
        if (bat::in_flight(B)) throw Error(ICCG_ERR_STATE, "the batch has solves in flight");
        CK(cudaStreamSynchronize(B->stream));
        bat::drop_graph(B);
        B->sys.clear();
        B->sys_dirty = true;
        B->lists_dirty = true;
    });
}

int iccg_batch_solve(iccg_batch* B, int nsolve, const int* system, const double* const* b, double* const* x,
                     int max_iter, double tol, const iccg_solve_opts* opts, iccg_result* res)
{
    return bguard(B, [&] {
        if (nsolve <= 0 || !system || !b || !x || !res) throw Error(ICCG_ERR_ARG, "null argument or no solves");
        for (int s = 0; s < nsolve; ++s)
            if (!b[s] || !x[s]) throw Error(ICCG_ERR_ARG, "null right-hand side or solution");
        if (B->sys.empty()) throw Error(ICCG_ERR_STATE, "the batch holds no system");
        iccg_solve_opts o{ICCG_MODE_FUSED, ICCG_STORE_FP64, 50, kGraphIters};
        if (opts) o = *opts;
        if (o.storage == ICCG_STORE_FP32) bat::run<float>(B, nsolve, system, b, x, max_iter, tol, o, res);
        else bat::run<double>(B, nsolve, system, b, x, max_iter, tol, o, res);
    });
}

int iccg_batch_open(iccg_batch* B, int slots, const iccg_solve_opts* opts)
{
    return bguard(B, [&] {
        iccg_solve_opts o{ICCG_MODE_FUSED, ICCG_STORE_FP64, 50, kGraphIters};
        if (opts) o = *opts;
        bat::open_session(B, slots, o);
    });
}

int iccg_batch_submit(iccg_batch* B, int system, const double* b, const double* x0, int max_iter, double tol,
                      int* slot)
{
    return bguard(B, [&] {
        if (!slot) throw Error(ICCG_ERR_ARG, "null argument");
        *slot = bat::submit(B, system, b, x0, max_iter, tol);
    });
}

int iccg_batch_step(iccg_batch* B, int* stopped, int cap, int* nstopped, int* nrunning)
{
    return bguard(B, [&] {
        if (!nstopped || (cap > 0 && !stopped)) throw Error(ICCG_ERR_ARG, "null argument");
        if (B->storage < 0) throw Error(ICCG_ERR_STATE, "the batch is not open");
        if (B->storage == ICCG_STORE_FP32) bat::step<float>(B, nrunning);
        else bat::step<double>(B, nrunning);
        const int k = std::min(cap, (int)B->report.size());
        for (int i = 0; i < k; ++i) stopped[i] = B->report[(size_t)i];
        B->report.erase(B->report.begin(), B->report.begin() + k);
        *nstopped = k;
    });
}

int iccg_batch_retire(iccg_batch* B, int n, const int* slots, double* const* x, iccg_result* res)
{
    return bguard(B, [&] {
        if (n <= 0) return;
        if (!slots || !x || !res) throw Error(ICCG_ERR_ARG, "null argument");
        bat::retire(B, n, slots, x, res);
    });
}

int iccg_device_memory(int device, long long* free_bytes, long long* total_bytes)
{
    if (!free_bytes || !total_bytes) return ICCG_ERR_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return ICCG_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return ICCG_ERR_ARG;
    }
    size_t f = 0, t = 0;
    const cudaError_t e = cudaMemGetInfo(&f, &t);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ICCG_ERR_CUDA;
    }
    *free_bytes = (long long)f;
    *total_bytes = (long long)t;
    return ICCG_OK;
}

}  // extern "C"
