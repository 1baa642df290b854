// batch.inl -- many independent solves advanced together (included by
// ctx.cu inside namespace iccg).
//
// A batch holds systems built as ordinary contexts (matrix, schedule, IC(0)
// factor, lane-interleaved layout) and runs a set of solves -- (system,
// right-hand side) pairs, each the conjugate_gradient of cg_crs.cpp:89-162
// -- in lockstep: every kernel of a CG iteration is ONE launch over all the
// solves, taking its work from a device work list of (solve, row slices)
// items:
//   SpMV with p.Ap, p.p, Ap.Ap;  update x += alpha p, r -= alpha Ap with r.r;
//   FP64 residual b - A x for the solves that asked for one (every rr_interval
//   iterations, and once the recurrence residual is below tol);
//   one launch per level of the forward and the backward substitution (the
//   staged batches of every system's level l), r.z;  p = z + beta p.
// A solve's items in every launch read its own SolverState; a solve that has
// stopped skips its items.  A graph of a few iterations of the whole batch
// is replayed until every solve has stopped.
//
// Reductions are per solve: every item's sums go to the solve's slot for
// that item, and the item that completes the solve's set (an arrival counter
// per solve and reduction) adds the slots in slot order, in double-double,
// and runs the CG scalar logic for that solve.  The arithmetic of every row is
// the single-system kernels' (k_spmv_q, k_update, k_residual_q, the staged
// sweeps, k_xpay), so a solve gives the same bits alone and in any batch.

namespace bat {

// one system's device arrays (lane-interleaved order; value type of the
// batch's storage)
struct BSys {
    int n;
    SellMat A;        // A, storage values
    SellMat A64;      // A, FP64 values (residuals)
    SellMat S, T;     // strict parts of L / L^T, in-unit entries encoded
    const void* dg;   // pivots (FP64) or reciprocal pivots (FP32)
    const SliceMeta* meta;
    const int* glen;
    const int* sl0;
    const BatchDesc* bd;   // forward batches (the context's staged batches)
    const BatchDesc* bdb;  // backward batches: the same, or split by groups where the
                           // FP64 exact order's parked values would not fit shared memory
    const int* q2r;        // Q row -> A_run row
};

// one solve (a slot of the batch): its system and vectors (Q order),
// reduction slots and arrival counters (0 SpMV, 1 vector kernels and
// residuals, 2 backward sweep)
struct BSolve {
    int sys;
    int n;
    double *b, *x, *r, *p, *z, *y, *Ap;
    double *hb, *hx;  // b and x in the caller's (A_run) order: the host copies' staging
    dd* slots;
    unsigned int* arrive;
    int nitems[3];    // items of each reduction
};

// a work item: solve, range [a, b) (slices, rows, or a batch index in a),
// and its slot in the solve's reduction.  A launch takes the items
// [rng[0], rng[1]) of its list, the range read from device memory, so a
// captured graph stays valid while the lists are rewritten in place.
struct BItem {
    int solve, a, b, slot;
};

constexpr int kThreadsB = 256;
constexpr int kVecRows = 8192;   // rows per vector item (a multiple of 32)
constexpr int kSpmvSlices = 64;  // slices per SpMV item

// Adds an item's NV sums to its slot of the solve; the item completing the
// solve's set adds the slots in order and runs finish<FIN> (FIN_STORE: the
// sums into out).  Every thread of the CTA calls it.
template <int NV, int FIN>
__device__ void solve_reduce(acc2 (&a)[NV], const BSolve& S, int kind, int slot, SolverState* st, double* out)
{
    __shared__ dd sm[NV * (kThreadsB / 32)];
    __shared__ bool last;
    dd v[NV], tot[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = acc2_dd(a[q]);
    block_reduce_dd<NV>(v, sm, tot);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) S.slots[(size_t)slot * NV + q] = tot[q];
        __threadfence();
        const unsigned int c = atomicAdd(&S.arrive[kind], 1u);
        last = c == (unsigned int)S.nitems[kind] - 1u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    dd s[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) s[q] = dd{0.0, 0.0};
    for (int k = threadIdx.x; k < S.nitems[kind]; k += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            dd w;
            w.hi = __ldcg(&S.slots[(size_t)k * NV + q].hi);
            w.lo = __ldcg(&S.slots[(size_t)k * NV + q].lo);
            s[q] = dd_add(s[q], w);
        }
    block_reduce_dd<NV>(s, sm, tot);
    if (threadIdx.x == 0) {
        double r[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) r[q] = dd_round(tot[q]);
        if (FIN == FIN_STORE) {
#pragma unroll
            for (int q = 0; q < NV; ++q) out[q] = r[q];
        } else {
            finish<FIN>(r, st, nullptr);
            if (st->status != kRunning && st->t_stop == 0ull) st->t_stop = global_ns();
        }
        S.arrive[kind] = 0u;
    }
}

// y = A p (cg_crs.cpp:54-79, k_spmv_q's row arithmetic), with p.Ap, p.p,
// Ap.Ap and the breakdown test / alpha (cg_crs.cpp:127-135)
template <class T>
__global__ void __launch_bounds__(kThreadsB) k_bat_spmv(const BItem* __restrict__ items, const int* __restrict__ rng,
                                                         const BSys* __restrict__ sys, const BSolve* __restrict__ sol,
                                                         SolverState* states)
{
    grid_dep_begin();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = rng[0], i1 = rng[1];
    for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
        const BItem I = items[it];
        SolverState* st = states + I.solve;
        if (st_done(st)) continue;
        const BSolve S = sol[I.solve];
        const SellMat A = sys[S.sys].A;
        const T* __restrict__ val = (const T*)A.val;
        acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        for (int s = I.a + warp; s < I.b; s += kThreadsB / 32) {
            const int i = (s << 5) + lane;
            if (i < S.n) {
                const int L = A.len[i];
                const int p0 = A.ptr[s] + lane;
                // the row's first K entries: every column and value load,
                // then every gather, in flight before the sum (in CSR
                // order, as k_spmv_q)
                constexpr int K = 8;
                int c[K];
                double v[K], xv[K];
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    c[j] = j < L ? __ldg(A.col + p0 + 32 * j) : 0;
                    v[j] = j < L ? (double)__ldg(val + p0 + 32 * j) : 0.0;
                }
#pragma unroll
                for (int j = 0; j < K; ++j) xv[j] = j < L ? __ldg(S.p + c[j]) : 0.0;
                double sum = 0.0;
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (j < L) sum = sum + v[j] * xv[j];
                for (int j = K; j < L; ++j) {
                    const int pa = p0 + 32 * j;
                    sum = sum + (double)__ldg(val + pa) * __ldg(S.p + __ldg(A.col + pa));
                }
                S.Ap[i] = sum;
                const double xi = S.p[i];
                acc2_fma(a[0], xi, sum);
                acc2_fma(a[1], xi, xi);
                acc2_fma(a[2], sum, sum);
            }
        }
        solve_reduce<3, FIN_PAP>(a, S, 0, I.slot, st, nullptr);
    }
    grid_dep_trigger();
}

enum VecOp { V_UPDATE = 0, V_XPAY = 1, V_COPY = 2 };

// x += alpha p, r -= alpha Ap with r.r (cg_crs.cpp:137-149); p = z + beta p
// and the iteration count (cg_crs.cpp:155-157, 125); p = z (cg_crs.cpp:123)
template <int OP>
__global__ void __launch_bounds__(kThreadsB) k_bat_vec(const BItem* __restrict__ items, const int* __restrict__ rng,
                                                        const BSolve* __restrict__ sol, SolverState* states)
{
    grid_dep_begin();
    const int i0 = rng[0], i1 = rng[1];
    for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
        const BItem I = items[it];
        SolverState* st = states + I.solve;
        if (st_done(st)) continue;
        const BSolve S = sol[I.solve];
        if (OP == V_UPDATE) {
            const double alpha = st->alpha;
            acc2 a[1] = {{0.0, 0.0}};
            for (int k = I.a + threadIdx.x; k < I.b; k += blockDim.x) {
                S.x[k] = fma(alpha, S.p[k], S.x[k]);
                const double rk = fma(-alpha, S.Ap[k], S.r[k]);
                S.r[k] = rk;
                acc2_fma(a[0], rk, rk);
            }
            solve_reduce<1, FIN_UPD>(a, S, 1, I.slot, st, nullptr);
        } else if (OP == V_XPAY) {
            const double beta = st->beta;
            for (int k = I.a + threadIdx.x; k < I.b; k += blockDim.x) S.p[k] = fma(beta, S.p[k], S.z[k]);
            // the solve's first item advances the iteration count (the p of
            // a solve that stops here is not used again)
            if (I.slot == 0 && threadIdx.x == 0) {
                const int k1 = st->k + 1;
                st->k = k1;
                if (k1 >= st->max_iter) {
                    st->status = kMaxIter;
                    if (st->t_stop == 0ull) st->t_stop = global_ns();
                }
            }
        } else {
            for (int k = I.a + threadIdx.x; k < I.b; k += blockDim.x) S.p[k] = S.z[k];
        }
    }
    grid_dep_trigger();
}

// r = b - A x with the FP64 matrix (k_residual_q's arithmetic): FIN_INIT
// (b.b, r.r: ||b||, the initial test), FIN_TRUE (only solves that asked for
// it: the residual replacement and the FP64 confirmation of convergence),
// FIN_STORE (r.r and b.b into out[2 * solve]: the reported true residual)
template <int FIN>
__global__ void __launch_bounds__(kThreadsB) k_bat_residual(const BItem* __restrict__ items, const int* __restrict__ rng,
                                                             const BSys* __restrict__ sys,
                                                             const BSolve* __restrict__ sol, SolverState* states,
                                                             double* out)
{
    grid_dep_begin();
    constexpr int NV = FIN == FIN_TRUE ? 1 : 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = rng[0], i1 = rng[1];
    for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
        const BItem I = items[it];
        SolverState* st = states + I.solve;
        if (FIN != FIN_STORE && st_done(st)) continue;
        if (FIN == FIN_TRUE && *(volatile int*)&st->rr_flag == 0) continue;
        const BSolve S = sol[I.solve];
        const SellMat A = sys[S.sys].A64;
        const double* __restrict__ val = (const double*)A.val;
        acc2 a[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) a[q] = {0.0, 0.0};
        // vector items cover rows [a, b), a a multiple of 32: whole slices
        for (int s = (I.a >> 5) + warp; s < ((I.b + 31) >> 5); s += kThreadsB / 32) {
            const int i = (s << 5) + lane;
            if (i < I.b) {
                const int L = A.len[i];
                const int p0 = A.ptr[s] + lane;
                double sum = 0.0;
                for (int j = 0; j < L; ++j) {
                    const int pa = p0 + 32 * j;
                    sum = sum + __ldg(val + pa) * __ldg(S.x + __ldg(A.col + pa));
                }
                const double bi = S.b[i];
                const double ri = bi - sum;
                if (FIN != FIN_STORE) S.r[i] = ri;
                if (FIN == FIN_TRUE) {
                    acc2_fma(a[0], ri, ri);
                } else {
                    acc2_fma(a[0], FIN == FIN_INIT ? bi : ri, FIN == FIN_INIT ? bi : ri);
                    acc2_fma(a[NV - 1], FIN == FIN_INIT ? ri : bi, FIN == FIN_INIT ? ri : bi);
                }
            }
        }
        solve_reduce<NV, FIN>(a, S, 1, I.slot, st, out ? out + 2 * I.solve : nullptr);
    }
    grid_dep_trigger();
}

// One level of the forward or backward substitution over every solve: each
// item is one staged batch of a solve's system (phases G and C of the staged
// kernel, the same operations per row); the backward sweep reduces r.z over
// all its levels (FIN_RZ0 / FIN_RZ).
template <class T, bool FWD, int FIN, bool EXACT>
__global__ void __launch_bounds__(kThreadsB) k_bat_sweep(const BItem* __restrict__ items, const int* __restrict__ rng,
                                                          const BSys* __restrict__ sys,
                                                          const BSolve* __restrict__ sol, SolverState* states)
{
    grid_dep_begin();
    constexpr bool with_r = FIN == FIN_RZ || FIN == FIN_RZ0;
    extern __shared__ __align__(16) unsigned char smem_bat[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = rng[0], i1 = rng[1];
    for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
        const BItem I = items[it];
        SolverState* st = states + I.solve;
        if (st_done(st)) continue;
        const BSolve S = sol[I.solve];
        const BSys& Y = sys[S.sys];
        const BatchDesc cur = FWD ? Y.bd[I.a] : Y.bdb[I.a];
        const int rows = cur.qe - cur.qb;
        const StageLayout Ly = FWD ? stage_layout(rows, cur.ps1 - cur.ps0, cur.se - cur.sb, (int)sizeof(T), false, false)
                                   : stage_layout(rows, cur.pt1 - cur.pt0, cur.se - cur.sb, (int)sizeof(T), with_r,
                                                  EXACT);
        const SellMat M = FWD ? Y.S : Y.T;
        double* out = FWD ? S.y : S.z;
        stage_batch<T, FWD, with_r>(smem_bat, Ly, cur, Y.meta, M, (const T*)Y.dg, FWD ? S.r : S.y, S.r);
        int gl[2] = {0, 0}, gs[2] = {0, 0};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int gi = warp + 8 * k;
            if (gi < cur.ng) {
                gl[k] = __ldg(Y.glen + (size_t)(cur.gb + gi) * 32 + lane);
                gs[k] = __ldg(Y.sl0 + cur.gb + gi);
            }
        }
        cp_async_wait<0>();
        __syncthreads();
        st_gather<T, FWD, EXACT, false>(cur, smem_bat, Ly, rows, out);
        __syncthreads();
        acc2 rz[1] = {{0.0, 0.0}};
        st_chain<T, FWD, EXACT, with_r>(cur, smem_bat, Ly, rows, gl, gs, out, rz[0]);
        __syncthreads();
        if (with_r) solve_reduce<1, FIN>(rz, S, 2, I.slot, st, nullptr);
    }
    grid_dep_trigger();
}

// b and x0 from the staging (caller's order) into Q order (gather, which
// 0: b, 1: x), or x back into the staging (scatter)
__global__ void __launch_bounds__(kThreadsB) k_bat_perm(const BItem* __restrict__ items, const int* __restrict__ rng,
                                                         const BSys* __restrict__ sys,
                                                         const BSolve* __restrict__ sol, int which, int gather)
{
    grid_dep_begin();
    const int i0 = rng[0], i1 = rng[1];
    for (int it = i0 + (int)blockIdx.x; it < i1; it += gridDim.x) {
        const BItem I = items[it];
        const BSolve S = sol[I.solve];
        const int* perm = sys[S.sys].q2r;
        if (gather) {
            double* v = which == 0 ? S.b : S.x;
            const double* h = which == 0 ? S.hb : S.hx;
            for (int k = I.a + threadIdx.x; k < I.b; k += blockDim.x) v[k] = h[perm[k]];
        } else {
            for (int k = I.a + threadIdx.x; k < I.b; k += blockDim.x) S.hx[perm[k]] = S.x[k];
        }
    }
}

// status of every slot into out[], the number still running into *running
__global__ void k_bat_status(int nslot, const SolverState* states, int* out, int* running)
{
    grid_dep_begin();
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int c = 0;
    for (int s = threadIdx.x; s < nslot; s += blockDim.x) {
        const int st = states[s].status;
        if (out) out[s] = st;
        c += st == kRunning ? 1 : 0;
    }
    atomicAdd(&cnt, c);
    __syncthreads();
    if (threadIdx.x == 0) *running = cnt;
}

// the start time of the solves just admitted (%globaltimer, ns)
__global__ void k_bat_begin(const int* __restrict__ solves, int count, SolverState* states)
{
    grid_dep_begin();
    const unsigned long long t = global_ns();
    for (int i = threadIdx.x; i < count; i += blockDim.x) states[solves[i]].t_start = t;
}

}  // namespace bat

}  // namespace iccg

namespace iccg {
namespace bat {

constexpr int kIdle = 5;  // status of a slot that holds no solve (not kRunning)

// A system of the batch: its context and the device tables the batched
// kernels read for the batch's value type.
struct SysHost {
    iccg_ctx* c = nullptr;
    int storage = -1;        // value type the tables were built for
    int qver = -1, fver = -1;  // the context's layout and factor they were built from
    BSys y{};
    Buf<BatchDesc> bdb;      // backward batches (split by groups where needed)
    std::vector<int> blb;    // first backward batch of each level (+ end)
    std::vector<int> smem_f, smem_b;  // stage bytes per level
    int nlevels = 0;
    int active = 0;          // slots holding solves of it
};

// A slot: one solve's device memory and its table entry.
struct SlotHost {
    int state = 0;     // 0 free, 1 admitted (start-up pending), 2 running, 3 stopped, not retired
    int sys = -1;
    Buf<double> mem;   // vectors, staging of b and x, reduction slots
    BSolve v{};
};

}  // namespace bat

}  // namespace iccg

// The batch object behind iccg_batch (include/iccg.h).
struct iccg_batch {
    int device = 0;
    int nsm = 148;
    int smem_optin = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    double last_ms = 0.0;
    long long dev_bytes = 0;
    std::vector<std::unique_ptr<iccg::bat::SysHost>> sys;  // contexts owned by the caller
    // the open session: value type, options, slots
    int storage = -1;
    iccg_solve_opts opts{ICCG_MODE_FUSED, ICCG_STORE_FP64, 50, 8};
    std::vector<std::unique_ptr<iccg::bat::SlotHost>> slot;
    iccg::Buf<iccg::bat::BSys> dsys;
    iccg::Buf<iccg::bat::BSolve> dsol;
    iccg::Buf<iccg::SolverState> dstate;
    iccg::Buf<unsigned int> darrive;
    iccg::Buf<double> dtres;
    iccg::Buf<int> dstatus, drunning;
    bool sys_dirty = true, lists_dirty = true;
    // work lists of the running solves (the iteration graph), of the solves
    // just admitted (their start-up) and of the solves being retired; each
    // with its ranges: [0, 1] SpMV, [2, 3] vector items, then the forward
    // and backward level offsets
    iccg::Buf<iccg::bat::BItem> a_spmv, a_vec, a_fwd, a_bwd, s_vec, s_fwd, s_bwd, r_vec;
    iccg::Buf<int> a_rng, s_rng, r_rng, s_ids;
    int a_levels = 0;
    long long a_nspmv = 0, a_nvec = 0;
    std::vector<long long> a_nf, a_nb;    // items per level
    std::vector<int> a_smf, a_smb;        // stage bytes per level
    std::vector<int> report;              // stopped slots not yet reported by step
    // the captured iteration graph and what it was captured for
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> gkey;
    long long per_graph = 0;
    int* h_status = nullptr;   // pinned, one per slot
    size_t h_status_cap = 0;
    int* h_running = nullptr;  // pinned, 2
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs[2] = {nullptr, nullptr};
};

namespace iccg {
namespace bat {

template <class K, class... Args>
static void blaunch(iccg_batch* B, K kernel, int grid, size_t smem, Args... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)std::max(1, grid));
    cfg.blockDim = dim3((unsigned)kThreadsB);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = B->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kernel, args...));
    B->launches++;
}

// CTAs of a grid-stride launch over `items`: the next power of two, at most
// one resident wave (a bucketed grid keeps a captured graph valid while the
// item counts move within the bucket)
template <class K>
static int bgrid(iccg_batch* B, K kernel, size_t smem, long long items)
{
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreadsB, smem));
    long long p2 = 1;
    while (p2 < items) p2 <<= 1;
    return (int)std::max(1ll, std::min<long long>(p2, (long long)std::max(1, per_sm) * B->nsm));
}

// raises a kernel's dynamic shared-memory limit to the device's opt-in maximum
template <class K>
static void bsmem(iccg_batch* B, K kernel)
{
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, kernel));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            B->smem_optin - (int)fa.sharedSizeBytes));
}

// elements between a solve's vectors: an even count, so that every vector
// starts on a 16-byte boundary (the staged sweeps copy r and y in 16-byte
// chunks)
static long long vec_step(int n) { return ((long long)n + 3) & ~1ll; }

static void drop_graph(iccg_batch* B)
{
    if (B->exec) cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
    B->gkey.clear();
}

static bool in_flight(const iccg_batch* B)
{
    for (const auto& s : B->slot)
        if (s->state != 0) return true;
    return false;
}

// The system's tables for the session's value type: the lane-interleaved
// layout with every level staged; backward batches whose exact-order buffer
// (the gathered values parked beside the entries) exceeds shared memory are
// split into batches of one group each (the groups of a level are
// independent, and a group's rows and slices are contiguous).
static void sys_tables(iccg_batch* B, int k)
{
    SysHost& H = *B->sys[(size_t)k];
    iccg_ctx* c = H.c;
    if (!c) throw Error(ICCG_ERR_ARG, "no system " + std::to_string(k) + " in the batch");
    if (H.storage == B->storage && H.qver == c->Q.version && H.fver == c->Q.factor_version && c->Q.ok) return;
    if (H.active) throw Error(ICCG_ERR_STATE, "system " + std::to_string(k) + " changed while solves of it run");
    const bool f32 = B->storage == ICCG_STORE_FP32;
    const bool exact = !f32;
    const int tsize = f32 ? 4 : 8;
    require_precond(c);
    if (c->pc_kind != ICCG_PRECOND_IC0 || !c->use_q)
        throw Error(ICCG_ERR_STATE, "batched solves need IC(0) on the lane-interleaved path");
    prepare_path(c, B->storage);
    CK(cudaStreamSynchronize(c->stream));
    QSys& Q = c->Q;
    bool fit = Q.staged && Q.two_phase && (!f32 || Q.r32_ok);
    for (int l = 0; fit && l < Q.nlevels; ++l) fit = Q.st_fit[(size_t)l] != 0 && (f32 || Q.st_fit64[(size_t)l] != 0);
    if (!fit) throw Error(ICCG_ERR_STATE, "system " + std::to_string(k) + ": a level does not fit the staged sweep");
    const int lim = std::max(0, B->smem_optin - 2048);  // the reduction scratch comes on top
    auto fwd_bytes = [&](const BatchDesc& d) {
        return stage_layout(d.qe - d.qb, d.ps1 - d.ps0, d.se - d.sb, tsize, false, false).bytes;
    };
    auto bwd_bytes = [&](const BatchDesc& d) {
        return stage_layout(d.qe - d.qb, d.pt1 - d.pt0, d.se - d.sb, tsize, true, exact).bytes;
    };
    auto one_group = [&](const BatchDesc& d, int g) {
        BatchDesc e = d;
        e.gb = g;
        e.ng = 1;
        e.sb = Q.h_sl0[(size_t)g];
        e.se = Q.h_sl0[(size_t)g + 1];
        e.qb = Q.steps[(size_t)e.sb].first;
        e.qe = Q.steps[(size_t)e.se - 1].first + Q.steps[(size_t)e.se - 1].second;
        e.ps0 = Q.S.h_ptr[(size_t)e.sb];
        e.ps1 = Q.S.h_ptr[(size_t)e.se];
        e.pt0 = Q.T.h_ptr[(size_t)e.sb];
        e.pt1 = Q.T.h_ptr[(size_t)e.se];
        return e;
    };
    std::vector<BatchDesc> hbd;
    H.nlevels = Q.nlevels;
    H.blb.assign((size_t)Q.nlevels + 1, 0);
    H.smem_f.assign((size_t)Q.nlevels, 0);
    H.smem_b.assign((size_t)Q.nlevels, 0);
    for (int l = 0; l < Q.nlevels; ++l) {
        H.blb[(size_t)l] = (int)hbd.size();
        for (int bi = Q.lb[(size_t)l]; bi < Q.lb[(size_t)l + 1]; ++bi) {
            const BatchDesc& d = Q.h_bdesc[(size_t)bi];
            H.smem_f[(size_t)l] = std::max(H.smem_f[(size_t)l], fwd_bytes(d));
            if (bwd_bytes(d) <= lim) {
                hbd.push_back(d);
                continue;
            }
            for (int g = d.gb; g < d.gb + d.ng; ++g) {
                const BatchDesc e = one_group(d, g);
                if (bwd_bytes(e) > lim)
                    throw Error(ICCG_ERR_STATE, "system " + std::to_string(k) + ": a group of level " +
                                                    std::to_string(l) + " does not fit the staged sweep");
                hbd.push_back(e);
            }
        }
        for (int i = H.blb[(size_t)l]; i < (int)hbd.size(); ++i)
            H.smem_b[(size_t)l] = std::max(H.smem_b[(size_t)l], bwd_bytes(hbd[(size_t)i]));
    }
    H.blb[(size_t)Q.nlevels] = (int)hbd.size();
    if (hbd.empty()) hbd.push_back(BatchDesc{});
    H.bdb.upload(hbd.data(), hbd.size(), &B->dev_bytes, B->stream);
    BSys& y = H.y;
    y.n = c->n;
    y.A = Q.A.view(f32);
    y.A64 = Q.A.view(false);
    y.S = Q.S.view(f32);
    y.T = Q.T.view(f32);
    y.dg = f32 ? (const void*)Q.r32.get() : (const void*)Q.d64.get();
    y.meta = (const SliceMeta*)Q.meta.get();
    y.glen = Q.glen.get();
    y.sl0 = Q.sl0.get();
    y.bd = Q.bdesc.get();
    y.bdb = H.bdb.get();
    y.q2r = Q.dq2r.get();
    H.storage = B->storage;
    H.qver = Q.version;
    H.fver = Q.factor_version;
    B->sys_dirty = true;
}

static void upload_sys(iccg_batch* B)
{
    if (!B->sys_dirty) return;
    std::vector<BSys> hs(std::max<size_t>(1, B->sys.size()));
    for (size_t k = 0; k < B->sys.size(); ++k)
        if (B->sys[k]->c && B->sys[k]->storage == B->storage) hs[k] = B->sys[k]->y;
    B->dsys.upload(hs.data(), hs.size(), &B->dev_bytes, B->stream);
    B->sys_dirty = false;
}

// Opens a session: value type and options of the solves to come, `cap` slots.
static void open_session(iccg_batch* B, int cap, const iccg_solve_opts& o)
{
    if (in_flight(B)) throw Error(ICCG_ERR_STATE, "the batch has solves in flight");
    if (o.mode != ICCG_MODE_FUSED) throw Error(ICCG_ERR_ARG, "batched solves run the fused form only");
    if (o.storage != ICCG_STORE_FP32 && o.storage != ICCG_STORE_FP64) throw Error(ICCG_ERR_ARG, "unknown storage");
    if (cap <= 0) throw Error(ICCG_ERR_ARG, "a batch needs at least one slot");
    drop_graph(B);
    B->storage = o.storage;
    B->opts = o;
    if (B->opts.graph_iters <= 0) B->opts.graph_iters = 8;
    B->sys_dirty = true;
    B->lists_dirty = true;
    B->report.clear();
    while ((int)B->slot.size() < cap) B->slot.push_back(std::make_unique<SlotHost>());
    const size_t n = B->slot.size();
    B->dsol.alloc(n, &B->dev_bytes);
    B->darrive.alloc(3 * n, &B->dev_bytes);
    B->dtres.alloc(2 * n, &B->dev_bytes);
    B->dstatus.alloc(n, &B->dev_bytes);
    B->drunning.alloc(2, &B->dev_bytes);
    std::vector<SolverState> idle(n);
    for (auto& q : idle) {
        q = SolverState{};
        q.status = kIdle;
    }
    B->dstate.upload(idle.data(), n, &B->dev_bytes, B->stream);
    CK(cudaMemsetAsync(B->darrive.get(), 0, sizeof(unsigned int) * 3 * n, B->stream));
    if (B->h_status_cap < n) {
        if (B->h_status) cudaFreeHost(B->h_status);
        B->h_status = nullptr;
        B->h_status_cap = 0;
        CK(cudaMallocHost(&B->h_status, sizeof(int) * n));
        B->h_status_cap = n;
    }
    CK(cudaStreamSynchronize(B->stream));
}

// Admits a solve into a free slot: its vectors, b and x0 (A_run order) into
// the slot's staging; the start-up runs with the next step.
static int submit(iccg_batch* B, int k, const double* b, const double* x0, int max_iter, double tol)
{
    if (B->storage < 0) throw Error(ICCG_ERR_STATE, "the batch is not open");
    if (k < 0 || k >= (int)B->sys.size() || !B->sys[(size_t)k]->c)
        throw Error(ICCG_ERR_ARG, "solve names no system of the batch");
    if (!b) throw Error(ICCG_ERR_ARG, "null right-hand side");
    sys_tables(B, k);
    int s = -1;
    for (size_t i = 0; i < B->slot.size(); ++i)
        if (B->slot[i]->state == 0) {
            s = (int)i;
            break;
        }
    if (s < 0) throw Error(ICCG_ERR_STATE, "no free slot");
    SysHost& H = *B->sys[(size_t)k];
    SlotHost& S = *B->slot[(size_t)s];
    const int n = H.y.n;
    const long long step = vec_step(n);
    const int nslices = (n + 31) / 32;
    const int nspmv = (nslices + kSpmvSlices - 1) / kSpmvSlices;
    const int nvec = (n + kVecRows - 1) / kVecRows;
    const int nbwd = H.blb.back();
    const long long nred = std::max({3ll * nspmv, 2ll * nvec, (long long)nbwd, 1ll});
    S.mem.alloc((size_t)(9 * step + 2 * nred), &B->dev_bytes);
    BSolve& v = S.v;
    v = BSolve{};
    v.sys = k;
    v.n = n;
    double* base = S.mem.get();
    double** vp[9] = {&v.b, &v.x, &v.r, &v.p, &v.z, &v.y, &v.Ap, &v.hb, &v.hx};
    for (int q = 0; q < 9; ++q) *vp[q] = base + (size_t)q * step;
    v.slots = reinterpret_cast<dd*>(base + 9 * step);
    v.arrive = B->darrive.get() + 3 * (size_t)s;
    v.nitems[0] = nspmv;
    v.nitems[1] = nvec;
    v.nitems[2] = nbwd;
    SolverState q{};
    q.tol = tol;
    q.status = kRunning;
    q.pend = kRunning;
    q.max_iter = max_iter;
    q.rr_interval = B->storage == ICCG_STORE_FP32 ? B->opts.rr_interval : 0;
    q.true_check = 1;
    q.xdefer_k = -1;
    const size_t nb = sizeof(double) * (size_t)n;
    CK(cudaMemcpyAsync(B->dsol.get() + s, &v, sizeof(BSolve), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemcpyAsync(B->dstate.get() + s, &q, sizeof(SolverState), cudaMemcpyHostToDevice, B->stream));
    CK(cudaMemsetAsync(v.arrive, 0, 3 * sizeof(unsigned int), B->stream));
    CK(cudaMemcpyAsync(v.hb, b, nb, cudaMemcpyHostToDevice, B->stream));
    if (x0) CK(cudaMemcpyAsync(v.hx, x0, nb, cudaMemcpyHostToDevice, B->stream));
    else CK(cudaMemsetAsync(v.hx, 0, nb, B->stream));
    S.state = 1;
    S.sys = k;
    H.active++;
    return s;
}

// the items of a set of slots: vector and SpMV items, and the sweep items
// level by level (in a level system by system and batch by batch, the solves
// of one system next to each other, so that its matrix data is read from
// DRAM once and from L2 for the others); rng as described at iccg_batch
struct Lists {
    std::vector<BItem> spmv, vec, fwd, bwd;
    std::vector<int> rng;
    std::vector<long long> nf, nb;
    std::vector<int> smf, smb;
    int levels = 0;
};

static Lists make_lists(iccg_batch* B, const std::vector<int>& slots)
{
    Lists L;
    std::vector<std::vector<int>> of(B->sys.size());
    for (int s : slots) {
        const SlotHost& S = *B->slot[(size_t)s];
        of[(size_t)S.sys].push_back(s);
        L.levels = std::max(L.levels, B->sys[(size_t)S.sys]->nlevels);
        const int n = S.v.n, nslices = (n + 31) / 32;
        int ns = 0, nv = 0;
        for (int a = 0; a < nslices; a += kSpmvSlices)
            L.spmv.push_back(BItem{s, a, std::min(nslices, a + kSpmvSlices), ns++});
        for (int a = 0; a < n; a += kVecRows) L.vec.push_back(BItem{s, a, std::min(n, a + kVecRows), nv++});
    }
    const int NL = L.levels;
    std::vector<int> bslot(B->slot.size(), 0);
    std::vector<int> foff((size_t)NL + 1, 0), boff((size_t)NL + 1, 0);
    L.nf.assign((size_t)NL, 0);
    L.nb.assign((size_t)NL, 0);
    L.smf.assign((size_t)NL, 0);
    L.smb.assign((size_t)NL, 0);
    // backward slots: levels from the last to the first
    std::vector<std::vector<BItem>> bl((size_t)NL);
    for (int l = NL - 1; l >= 0; --l)
        for (size_t k = 0; k < B->sys.size(); ++k) {
            if (of[k].empty()) continue;
            const SysHost& H = *B->sys[k];
            if (l >= H.nlevels) continue;
            for (int bi = H.blb[(size_t)l]; bi < H.blb[(size_t)l + 1]; ++bi)
                for (int s : of[k]) bl[(size_t)l].push_back(BItem{s, bi, 0, bslot[(size_t)s]++});
            L.smb[(size_t)l] = std::max(L.smb[(size_t)l], H.smem_b[(size_t)l]);
        }
    for (int l = 0; l < NL; ++l) {
        foff[(size_t)l] = (int)L.fwd.size();
        for (size_t k = 0; k < B->sys.size(); ++k) {
            if (of[k].empty()) continue;
            const SysHost& H = *B->sys[k];
            if (l >= H.nlevels) continue;
            const QSys& Q = H.c->Q;
            for (int bi = Q.lb[(size_t)l]; bi < Q.lb[(size_t)l + 1]; ++bi)
                for (int s : of[k]) L.fwd.push_back(BItem{s, bi, 0, 0});
            L.smf[(size_t)l] = std::max(L.smf[(size_t)l], H.smem_f[(size_t)l]);
        }
        L.nf[(size_t)l] = (long long)L.fwd.size() - foff[(size_t)l];
        boff[(size_t)l] = (int)L.bwd.size();
        L.bwd.insert(L.bwd.end(), bl[(size_t)l].begin(), bl[(size_t)l].end());
        L.nb[(size_t)l] = (long long)bl[(size_t)l].size();
    }
    foff[(size_t)NL] = (int)L.fwd.size();
    boff[(size_t)NL] = (int)L.bwd.size();
    L.rng = {0, (int)L.spmv.size(), 0, (int)L.vec.size()};
    L.rng.insert(L.rng.end(), foff.begin(), foff.end());
    L.rng.insert(L.rng.end(), boff.begin(), boff.end());
    for (auto* v : {&L.spmv, &L.vec, &L.fwd, &L.bwd})
        if (v->empty()) v->push_back(BItem{0, 0, 0, 0});
    return L;
}

// the typed kernels of the session
template <class T>
struct Kern {
    static constexpr bool exact = !std::is_same<T, float>::value;
    decltype(&k_bat_spmv<T>) spmv = k_bat_spmv<T>;
    decltype(&k_bat_vec<V_UPDATE>) upd = k_bat_vec<V_UPDATE>, xpay = k_bat_vec<V_XPAY>, copy = k_bat_vec<V_COPY>;
    decltype(&k_bat_residual<FIN_INIT>) init = k_bat_residual<FIN_INIT>, tru = k_bat_residual<FIN_TRUE>,
                                        store = k_bat_residual<FIN_STORE>;
    decltype(&k_bat_sweep<T, true, FIN_NONE, exact>) f = k_bat_sweep<T, true, FIN_NONE, exact>,
                                                    b0 = k_bat_sweep<T, false, FIN_RZ0, exact>,
                                                    b = k_bat_sweep<T, false, FIN_RZ, exact>;
    explicit Kern(iccg_batch* B)
    {
        static std::mutex mu;
        static std::vector<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (std::find(done.begin(), done.end(), B->device) != done.end()) return;
        bsmem(B, f);
        bsmem(B, b0);
        bsmem(B, b);
        done.push_back(B->device);
    }
};

// both sweeps over lists (items, ranges at rng + 4 / rng + 5 + levels)
template <class T>
static void launch_sweeps(iccg_batch* B, const Kern<T>& K, int fin_b, const BItem* F, const BItem* Bk, const int* rng,
                          int levels, const std::vector<long long>& nf, const std::vector<long long>& nb,
                          const std::vector<int>& smf, const std::vector<int>& smb)
{
    const BSys* ds = B->dsys.get();
    const BSolve* dv = B->dsol.get();
    SolverState* st = B->dstate.get();
    for (int l = 0; l < levels; ++l)
        if (nf[(size_t)l] > 0)
            blaunch(B, K.f, bgrid(B, K.f, (size_t)smf[(size_t)l], nf[(size_t)l]), (size_t)smf[(size_t)l], F, rng + 4 + l,
                    ds, dv, st);
    for (int l = levels - 1; l >= 0; --l) {
        if (nb[(size_t)l] <= 0) continue;
        const int* r = rng + 5 + levels + l;
        const size_t sm = (size_t)smb[(size_t)l];
        if (fin_b == FIN_RZ0) blaunch(B, K.b0, bgrid(B, K.b0, sm, nb[(size_t)l]), sm, Bk, r, ds, dv, st);
        else blaunch(B, K.b, bgrid(B, K.b, sm, nb[(size_t)l]), sm, Bk, r, ds, dv, st);
    }
}

// Start-up of the solves admitted since the last step: b and x0 into Q
// order, r0 = b - A x0 with ||b|| and the initial test, z0 = M^-1 r0, r.z,
// p = z (cg_crs.cpp:102-123).
template <class T>
static void flush_admissions(iccg_batch* B)
{
    std::vector<int> ids;
    for (size_t s = 0; s < B->slot.size(); ++s)
        if (B->slot[s]->state == 1) ids.push_back((int)s);
    if (ids.empty()) return;
    upload_sys(B);
    const Kern<T> K(B);
    Lists L = make_lists(B, ids);
    B->s_vec.upload(L.vec.data(), L.vec.size(), &B->dev_bytes, B->stream);
    B->s_fwd.upload(L.fwd.data(), L.fwd.size(), &B->dev_bytes, B->stream);
    B->s_bwd.upload(L.bwd.data(), L.bwd.size(), &B->dev_bytes, B->stream);
    B->s_rng.upload(L.rng.data(), L.rng.size(), &B->dev_bytes, B->stream);
    B->s_ids.upload(ids.data(), ids.size(), &B->dev_bytes, B->stream);
    const BSys* ds = B->dsys.get();
    const BSolve* dv = B->dsol.get();
    SolverState* st = B->dstate.get();
    const long long nv = L.rng[3];
    const int* R = B->s_rng.get();
    blaunch(B, k_bat_begin, 1, 0, (const int*)B->s_ids.get(), (int)ids.size(), st);
    const int gp = bgrid(B, k_bat_perm, 0, nv);
    blaunch(B, k_bat_perm, gp, 0, (const BItem*)B->s_vec.get(), R + 2, ds, dv, 0, 1);
    blaunch(B, k_bat_perm, gp, 0, (const BItem*)B->s_vec.get(), R + 2, ds, dv, 1, 1);
    blaunch(B, K.init, bgrid(B, K.init, 0, nv), 0, (const BItem*)B->s_vec.get(), R + 2, ds, dv, st, (double*)nullptr);
    launch_sweeps<T>(B, K, FIN_RZ0, B->s_fwd.get(), B->s_bwd.get(), R, L.levels, L.nf, L.nb, L.smf, L.smb);
    blaunch(B, K.copy, bgrid(B, K.copy, 0, nv), 0, (const BItem*)B->s_vec.get(), R + 2, dv, st);
    for (int s : ids) B->slot[(size_t)s]->state = 2;
    B->lists_dirty = true;
}

// the lists of the running solves
static void rebuild_active(iccg_batch* B)
{
    if (!B->lists_dirty) return;
    std::vector<int> ids;
    for (size_t s = 0; s < B->slot.size(); ++s)
        if (B->slot[s]->state == 2) ids.push_back((int)s);
    Lists L = make_lists(B, ids);
    B->a_spmv.upload(L.spmv.data(), L.spmv.size(), &B->dev_bytes, B->stream);
    B->a_vec.upload(L.vec.data(), L.vec.size(), &B->dev_bytes, B->stream);
    B->a_fwd.upload(L.fwd.data(), L.fwd.size(), &B->dev_bytes, B->stream);
    B->a_bwd.upload(L.bwd.data(), L.bwd.size(), &B->dev_bytes, B->stream);
    B->a_rng.upload(L.rng.data(), L.rng.size(), &B->dev_bytes, B->stream);
    B->a_levels = L.levels;
    B->a_nspmv = L.rng[1];
    B->a_nvec = L.rng[3];
    B->a_nf = L.nf;
    B->a_nb = L.nb;
    B->a_smf = L.smf;
    B->a_smb = L.smb;
    B->lists_dirty = false;
}

// The graph of graph_iters CG iterations over the running solves
// (cg_crs.cpp:125-160): SpMV with p.Ap, p.p, Ap.Ap and alpha; the update
// with r.r; the FP64 residual where a solve asked for it; both sweeps with
// r.z and beta; p = z + beta p.  Captured again when the lists' storage,
// the level count, a grid bucket or a stage size changes.
template <class T>
static void ensure_graph(iccg_batch* B)
{
    const Kern<T> K(B);
    const int m = B->opts.graph_iters;
    const int L = B->a_levels;
    const int gs = bgrid(B, K.spmv, 0, B->a_nspmv), gv = bgrid(B, K.upd, 0, B->a_nvec);
    const int gr = bgrid(B, K.tru, 0, B->a_nvec);
    std::vector<long long> key = {(long long)(uintptr_t)B->a_spmv.get(), (long long)(uintptr_t)B->a_vec.get(),
                                  (long long)(uintptr_t)B->a_fwd.get(), (long long)(uintptr_t)B->a_bwd.get(),
                                  (long long)(uintptr_t)B->a_rng.get(), (long long)(uintptr_t)B->dsys.get(),
                                  (long long)(uintptr_t)B->dsol.get(), (long long)(uintptr_t)B->dstate.get(),
                                  B->storage, m, L, gs, gv, gr};
    for (int l = 0; l < L; ++l) {
        key.push_back(B->a_nf[(size_t)l] > 0 ? bgrid(B, K.f, (size_t)B->a_smf[(size_t)l], B->a_nf[(size_t)l]) : 0);
        key.push_back(B->a_nb[(size_t)l] > 0 ? bgrid(B, K.b, (size_t)B->a_smb[(size_t)l], B->a_nb[(size_t)l]) : 0);
        key.push_back(B->a_smf[(size_t)l]);
        key.push_back(B->a_smb[(size_t)l]);
    }
    if (B->exec && key == B->gkey) return;
    drop_graph(B);
    const BSys* ds = B->dsys.get();
    const BSolve* dv = B->dsol.get();
    SolverState* st = B->dstate.get();
    const int* R = B->a_rng.get();
    auto iteration = [&] {
        blaunch(B, K.spmv, gs, 0, (const BItem*)B->a_spmv.get(), R, ds, dv, st);
        blaunch(B, K.upd, gv, 0, (const BItem*)B->a_vec.get(), R + 2, dv, st);
        blaunch(B, K.tru, gr, 0, (const BItem*)B->a_vec.get(), R + 2, ds, dv, st, (double*)nullptr);
        launch_sweeps<T>(B, K, FIN_RZ, B->a_fwd.get(), B->a_bwd.get(), R, L, B->a_nf, B->a_nb, B->a_smf, B->a_smb);
        blaunch(B, K.xpay, gv, 0, (const BItem*)B->a_vec.get(), R + 2, dv, st);
    };
    cudaGraph_t graph = nullptr;
    const long long before = B->launches;
    CK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    try {
        for (int it = 0; it < m; ++it) iteration();
    } catch (...) {
        cudaStreamEndCapture(B->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        B->launches = before;
        throw;
    }
    CK(cudaStreamEndCapture(B->stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    B->per_graph = B->launches - before;
    B->launches = before;
    CK(ie);
    B->exec = exec;
    B->gkey = key;
}

template <class T>
static bool prepare_step(iccg_batch* B)
{
    upload_sys(B);
    flush_admissions<T>(B);
    rebuild_active(B);
    if (B->a_nvec == 0) return false;
    ensure_graph<T>(B);
    return true;
}

// One graph launch (graph_iters iterations) over the running solves; the
// slots that stopped in it are queued for the report.
template <class T>
static void step(iccg_batch* B, int* nrunning)
{
    const int n = (int)B->slot.size();
    if (prepare_step<T>(B)) {
        CK(cudaGraphLaunch(B->exec, B->stream));
        B->launches += B->per_graph;
    }
    blaunch(B, k_bat_status, 1, 0, n, (const SolverState*)B->dstate.get(), B->dstatus.get(), B->drunning.get());
    CK(cudaMemcpyAsync(B->h_status, B->dstatus.get(), sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, B->stream));
    CK(cudaStreamSynchronize(B->stream));
    int run = 0;
    for (int s = 0; s < n; ++s) {
        SlotHost& S = *B->slot[(size_t)s];
        if (S.state != 2) continue;
        if (B->h_status[s] == kRunning) {
            ++run;
        } else {
            S.state = 3;
            B->report.push_back(s);
            B->lists_dirty = true;
        }
    }
    for (const auto& S : B->slot) run += S->state == 1 ? 1 : 0;
    if (nrunning) *nrunning = run;
}

// Retires stopped solves: the reported true residual ||b - A x|| / ||b|| in
// FP64, x back in the caller's order, the results; the slots become free.
static void retire(iccg_batch* B, int count, const int* slots, double* const* x, iccg_result* res)
{
    std::vector<int> ids(slots, slots + count);
    for (size_t i = 0; i < ids.size(); ++i) {
        const int s = ids[i];
        if (s < 0 || s >= (int)B->slot.size() || B->slot[(size_t)s]->state != 3)
            throw Error(ICCG_ERR_STATE, "slot " + std::to_string(s) + " holds no stopped solve");
        if (std::count(ids.begin(), ids.end(), s) != 1) throw Error(ICCG_ERR_ARG, "a slot named twice");
        if (!x[i]) throw Error(ICCG_ERR_ARG, "null solution array");
    }
    upload_sys(B);
    std::vector<BItem> vi;
    for (int s : ids) {
        const int n = B->slot[(size_t)s]->v.n;
        int nv = 0;
        for (int a = 0; a < n; a += kVecRows) vi.push_back(BItem{s, a, std::min(n, a + kVecRows), nv++});
    }
    const int rng[2] = {0, (int)vi.size()};
    B->r_vec.upload(vi.data(), vi.size(), &B->dev_bytes, B->stream);
    B->r_rng.upload(rng, 2, &B->dev_bytes, B->stream);
    const BSys* ds = B->dsys.get();
    const BSolve* dv = B->dsol.get();
    SolverState* st = B->dstate.get();
    auto kstore = k_bat_residual<FIN_STORE>;
    blaunch(B, kstore, bgrid(B, kstore, 0, (long long)vi.size()), 0, (const BItem*)B->r_vec.get(),
            (const int*)B->r_rng.get(), ds, dv, st, B->dtres.get());
    blaunch(B, k_bat_perm, bgrid(B, k_bat_perm, 0, (long long)vi.size()), 0, (const BItem*)B->r_vec.get(),
            (const int*)B->r_rng.get(), ds, dv, 1, 0);
    std::vector<SolverState> sf(ids.size());
    std::vector<double> tr(2 * ids.size());
    for (size_t i = 0; i < ids.size(); ++i) {
        const int s = ids[i];
        const SlotHost& S = *B->slot[(size_t)s];
        CK(cudaMemcpyAsync(&sf[i], st + s, sizeof(SolverState), cudaMemcpyDeviceToHost, B->stream));
        CK(cudaMemcpyAsync(&tr[2 * i], B->dtres.get() + 2 * s, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                           B->stream));
        CK(cudaMemcpyAsync(x[i], S.v.hx, sizeof(double) * (size_t)S.v.n, cudaMemcpyDeviceToHost, B->stream));
    }
    CK(cudaStreamSynchronize(B->stream));
    const bool f32 = B->storage == ICCG_STORE_FP32;
    for (size_t i = 0; i < ids.size(); ++i) {
        const SolverState& q = sf[i];
        iccg_result& r = res[i];
        std::memset(&r, 0, sizeof(r));
        r.iters = q.iters;
        r.status = q.status == kRunning ? kMaxIter : q.status;
        r.converged = q.status == kConverged ? 1 : 0;
        r.rel_resid = q.rel_resid;
        r.n_replacements = q.n_rr;
        // as a solve alone reports it: a converged mixed-precision solve ends
        // on an FP64 residual replacement, whose test is the true residual
        if (f32 && B->opts.rr_interval > 0 && r.converged) r.true_rel_resid = r.rel_resid;
        else r.true_rel_resid = std::sqrt(tr[2 * i]) / std::sqrt(tr[2 * i + 1]);
        r.solve_ms = q.t_stop > q.t_start ? (double)(q.t_stop - q.t_start) * 1e-6 : 0.0;
        SlotHost& S = *B->slot[(size_t)ids[i]];
        B->sys[(size_t)S.sys]->active--;
        S.state = 0;
        S.sys = -1;
    }
    for (int s : ids) B->report.erase(std::remove(B->report.begin(), B->report.end(), s), B->report.end());
}

// A whole solve set: every solve admitted at once, graph launches until none
// runs (the count after launch i - 1 is read while launch i runs), then all
// retired.
template <class T>
static void run(iccg_batch* B, int nsolve, const int* sys_of, const double* const* bh, double* const* xh, int max_iter,
                double tol, const iccg_solve_opts& o, iccg_result* res)
{
    open_session(B, std::max(nsolve, (int)B->slot.size()), o);
    std::vector<int> slot_of((size_t)nsolve);
    for (int s = 0; s < nsolve; ++s) slot_of[(size_t)s] = submit(B, sys_of[s], bh[s], xh[s], max_iter, tol);
    upload_sys(B);
    CK(cudaEventRecord(B->ev0, B->stream));
    const bool any = prepare_step<T>(B);
    const int n = (int)B->slot.size();
    const int m = B->opts.graph_iters;
    const long long nb_max = (long long)max_iter / m + 2;
    for (long long bi = 0; any; ++bi) {
        CK(cudaGraphLaunch(B->exec, B->stream));
        B->launches += B->per_graph;
        blaunch(B, k_bat_status, 1, 0, n, (const SolverState*)B->dstate.get(), (int*)nullptr,
                B->drunning.get() + (bi & 1));
        CK(cudaMemcpyAsync(&B->h_running[bi & 1], B->drunning.get() + (bi & 1), sizeof(int), cudaMemcpyDeviceToHost,
                           B->stream));
        CK(cudaEventRecord(B->evs[bi & 1], B->stream));
        if (bi > 0) {
            CK(cudaEventSynchronize(B->evs[(bi - 1) & 1]));
            if (B->h_running[(bi - 1) & 1] == 0) break;
        }
        if (bi >= nb_max) {
            CK(cudaEventSynchronize(B->evs[bi & 1]));
            break;
        }
    }
    CK(cudaEventRecord(B->ev1, B->stream));
    for (int s : slot_of) B->slot[(size_t)s]->state = 3;
    B->lists_dirty = true;
    std::vector<iccg_result> out((size_t)nsolve);
    retire(B, nsolve, slot_of.data(), xh, out.data());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    B->last_ms = ms;
    for (int s = 0; s < nsolve; ++s) {
        res[s] = out[(size_t)s];
        if (res[s].solve_ms <= 0.0) res[s].solve_ms = ms;
    }
}

}  // namespace bat
