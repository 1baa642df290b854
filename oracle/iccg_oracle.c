/*
 * iccg_oracle.c -- CPU restatement of the ICCG hot path of stomo0511/ICCG.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark may call it; the
 * product library (iccg_b200) never links, loads or executes it.
 *
 * It restates, in plain C, every function on the reference's hot path, each
 * one citing the reference file:line it follows.  Floating-point operations
 * are written out exactly as g++ 13 -O3 -march=x86-64-v3 evaluates the
 * reference, as read from the x86 assembly of that build: the substitution
 * sweeps (`acc -= L*y`), the two-pointer dot of build_ic0 and the CG vector
 * updates are fused multiply-adds; the spmv row sum and the IC(0) sum of
 * squares are NOT fused (g++ leaves those loop-carried reduction chains
 * uncontracted); dot/nrm2 accumulate in x87 long double.  This file is
 * compiled with -ffp-contract=off so only the explicit fma() calls are fused.
 *
 * Pinning: the restatement is checked bit-for-bit against the reference
 * itself (compiled from its own sources into oracle/_ref by the Makefile in
 * this directory) and against the committed fixtures in tests/golden/ that
 * were produced from that build.
 *
 * Known gap: where the reference sorts with std::sort (per PtAP row,
 * color.cpp:111-112; per expanded row, crs_io.cpp:203-219; the whole COO
 * list of the MatrixMarket reader, crs_io.cpp:27-30) this file keeps equal
 * keys in input order.  libstdc++'s std::sort does the same for ranges of
 * at most 16 elements (it insertion-sorts them) but not for longer ones, so
 * a row of more than 16 entries that repeats a column (three or more times
 * for the summing routines) can come out in a different order here.  Those
 * inputs are checked against the compiled reference instead.
 *
 * All functions return 0 on success or a negative error code; where the
 * reference throws std::runtime_error the restatement returns ORC_E*.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>

#define ORC_OK 0
#define ORC_EARG (-1)     /* size / range errors (reference: runtime_error)   */
#define ORC_EDIAG (-2)    /* IC(0): diagonal missing        (ic0.cpp:52-53)   */
#define ORC_EPIVZ (-3)    /* IC(0): near-zero pivot         (ic0.cpp:86-87)   */
#define ORC_EPIVN (-4)    /* IC(0): non-positive pivot      (ic0.cpp:104-113) */
#define ORC_EIO (-5)      /* file format errors (crs_io.cpp, color.cpp, block.cpp) */
#define ORC_ENOMEM (-6)

static int g_err_row = -1; /* row of the last IC(0) failure */
int orc_last_error_row(void) { return g_err_row; }

/* ------------------------------------------------------------------------ */
/* small helpers                                                             */
/* ------------------------------------------------------------------------ */

typedef struct { int c; double v; int ord; } orc_cv;

/* stable merge sort of (c, v) pairs by c (insertion order kept for ties) */
static void orc_sort_cv(orc_cv* a, orc_cv* tmp, int n)
{
    if (n < 2) return;
    if (n <= 16) {
        for (int i = 1; i < n; ++i) {
            orc_cv x = a[i];
            int j = i - 1;
            while (j >= 0 && a[j].c > x.c) { a[j + 1] = a[j]; --j; }
            a[j + 1] = x;
        }
        return;
    }
    int h = n / 2;
    orc_sort_cv(a, tmp, h);
    orc_sort_cv(a + h, tmp, n - h);
    int i = 0, j = h, k = 0;
    while (i < h && j < n) tmp[k++] = (a[j].c < a[i].c) ? a[j++] : a[i++];
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, sizeof(orc_cv) * (size_t)n);
}

/* key arrays for the permutation sorts; keys are unique (old id is the last
 * key), so any correct sort reproduces std::stable_sort exactly. */
static const int* g_k1; static const int* g_k2;
static int cmp_by_color(const void* pa, const void* pb)
{
    int a = *(const int*)pa, b = *(const int*)pb;
    if (g_k1[a] != g_k1[b]) return g_k1[a] < g_k1[b] ? -1 : 1;
    return (a > b) - (a < b);
}
static int cmp_by_block_color(const void* pa, const void* pb)
{
    int a = *(const int*)pa, b = *(const int*)pb;
    int ba = g_k1[a], bb = g_k1[b];
    int ca = g_k2[ba], cb = g_k2[bb];
    if (ca != cb) return ca < cb ? -1 : 1;
    if (ba != bb) return ba < bb ? -1 : 1;
    return (a > b) - (a < b);
}

/* ------------------------------------------------------------------------ */
/* a5: BuildPermutationByColor (color.cpp:50-63)                             */
/* new_of_old from a stable sort of old ids by (color, old id).              */
/* ------------------------------------------------------------------------ */
int orc_perm_by_color(int n, const int* color, int* new_of_old)
{
    if (n < 0) return ORC_EARG;
    int* order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!order) return ORC_ENOMEM;
    for (int i = 0; i < n; ++i) order[i] = i;
    g_k1 = color;
    qsort(order, (size_t)n, sizeof(int), cmp_by_color);
    for (int k = 0; k < n; ++k) new_of_old[order[k]] = k;
    free(order);
    return ORC_OK;
}

/* a6: BuildPermutationByBlockColor (block.cpp:92-114): sort by
 * (block_color[block], block, old id). */
int orc_perm_by_block_color(int n, const int* block_of_old, const int* block_color,
                            int* new_of_old)
{
    if (n < 0) return ORC_EARG;
    int* order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!order) return ORC_ENOMEM;
    for (int i = 0; i < n; ++i) order[i] = i;
    g_k1 = block_of_old; g_k2 = block_color;
    qsort(order, (size_t)n, sizeof(int), cmp_by_block_color);
    for (int k = 0; k < n; ++k) new_of_old[order[k]] = k;
    free(order);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a7: Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141)                  */
/* Only entries with j <= i of the input are used (color.cpp:91); each is     */
/* mapped to (max(ip,jp), min(ip,jp)) (color.cpp:97-98), rows are sorted by   */
/* column, duplicates are summed and sums equal to 0.0 are dropped            */
/* (color.cpp:123,132).  The output capacity must be >= the number of lower   */
/* input entries; *out_nnz receives the actual count.                        */
/* Ties between duplicate columns are summed in insertion order (the          */
/* reference's std::sort keeps that order for rows of <= 16 entries only).   */
/* ------------------------------------------------------------------------ */
int orc_ptap_lower(int n, const int* rowptr, const int* colind, const double* val,
                   const int* new_of_old, int cap,
                   int* out_rowptr, int* out_colind, double* out_val, int* out_nnz)
{
    if (n < 0) return ORC_EARG;
    int* cnt = (int*)calloc((size_t)n + 1, sizeof(int));
    if (!cnt) return ORC_ENOMEM;
    long total = 0;
    for (int i = 0; i < n; ++i) {
        int ip = new_of_old[i];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            if (j > i) continue;
            int jp = new_of_old[j];
            int r = ip > jp ? ip : jp;
            cnt[r + 1]++;
            total++;
        }
    }
    for (int r = 0; r < n; ++r) cnt[r + 1] += cnt[r];
    orc_cv* buf = (orc_cv*)malloc(sizeof(orc_cv) * (size_t)(total > 0 ? total : 1));
    orc_cv* tmp = (orc_cv*)malloc(sizeof(orc_cv) * (size_t)(total > 0 ? total : 1));
    int* cur = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    if (!buf || !tmp || !cur) { free(cnt); free(buf); free(tmp); free(cur); return ORC_ENOMEM; }
    memcpy(cur, cnt, sizeof(int) * (size_t)(n + 1));
    for (int i = 0; i < n; ++i) {
        int ip = new_of_old[i];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            if (j > i) continue;
            int jp = new_of_old[j];
            int r = ip, c = jp;
            if (c > r) { int t = r; r = c; c = t; }
            orc_cv e; e.c = c; e.v = val[k]; e.ord = 0;
            buf[cur[r]++] = e;
        }
    }
    int nz = 0;
    out_rowptr[0] = 0;
    for (int r = 0; r < n; ++r) {
        int b = cnt[r], e = cnt[r + 1];
        if (e > b) {
            orc_sort_cv(buf + b, tmp, e - b);
            int cur_c = buf[b].c;
            double acc = buf[b].v;
            for (int t = b + 1; t < e; ++t) {
                if (buf[t].c == cur_c) {
                    acc += buf[t].v;
                } else {
                    if (acc != 0.0) {
                        if (nz >= cap) goto overflow;
                        out_colind[nz] = cur_c; out_val[nz] = acc; ++nz;
                    }
                    cur_c = buf[t].c; acc = buf[t].v;
                }
            }
            if (acc != 0.0) {
                if (nz >= cap) goto overflow;
                out_colind[nz] = cur_c; out_val[nz] = acc; ++nz;
            }
        }
        out_rowptr[r + 1] = nz;
    }
    *out_nnz = nz;
    free(cnt); free(buf); free(tmp); free(cur);
    return ORC_OK;
overflow:
    free(cnt); free(buf); free(tmp); free(cur);
    return ORC_EARG;
}

/* ------------------------------------------------------------------------ */
/* a3: expand_lower_to_full (crs_io.cpp:163-227).  Output nnz = 2*nnzL - diag */
/* entries; each row's columns are sorted ascending afterwards.              */
/* ------------------------------------------------------------------------ */
int orc_expand_lower_to_full_nnz(int n, const int* rowptr, const int* colind)
{
    long nz = 0;
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) nz += (colind[k] == i) ? 1 : 2;
    return (int)nz;
}

int orc_expand_lower_to_full(int n, const int* rowptr, const int* colind, const double* val,
                             int* frow, int* fcol, double* fval)
{
    int* cntr = (int*)calloc((size_t)n + 1, sizeof(int));
    if (!cntr) return ORC_ENOMEM;
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            cntr[i]++;
            if (j != i) cntr[j]++;
        }
    frow[0] = 0;
    for (int i = 0; i < n; ++i) frow[i + 1] = frow[i] + cntr[i];
    int* cur = cntr;
    for (int i = 0; i < n; ++i) cur[i] = frow[i];
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            double v = val[k];
            int p = cur[i]++;
            fcol[p] = j; fval[p] = v;
            if (j != i) { int q = cur[j]++; fcol[q] = i; fval[q] = v; }
        }
    /* per-row sort by column (crs_io.cpp:206-225) */
    int maxlen = 0;
    for (int i = 0; i < n; ++i) if (frow[i + 1] - frow[i] > maxlen) maxlen = frow[i + 1] - frow[i];
    orc_cv* a = (orc_cv*)malloc(sizeof(orc_cv) * (size_t)(maxlen > 0 ? maxlen : 1));
    orc_cv* t = (orc_cv*)malloc(sizeof(orc_cv) * (size_t)(maxlen > 0 ? maxlen : 1));
    if (!a || !t) { free(cntr); free(a); free(t); return ORC_ENOMEM; }
    for (int i = 0; i < n; ++i) {
        int rs = frow[i], re = frow[i + 1];
        for (int k = rs; k < re; ++k) { a[k - rs].c = fcol[k]; a[k - rs].v = fval[k]; }
        orc_sort_cv(a, t, re - rs);
        for (int k = rs; k < re; ++k) { fcol[k] = a[k - rs].c; fval[k] = a[k - rs].v; }
    }
    free(cntr); free(a); free(t);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a8: BuildColorPtrRows_FromPermutationAndColor (color.cpp:164-197)         */
/* color_ptr[nc+1]; rows_of_color[n] lists NEW ids, ascending within a color */
/* ------------------------------------------------------------------------ */
int orc_color_schedule(int n, const int* color, int nc, const int* new_of_old,
                       int* color_ptr, int* rows_of_color)
{
    int* old_of_new = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* cur = (int*)calloc((size_t)nc + 1, sizeof(int));
    if (!old_of_new || !cur) { free(old_of_new); free(cur); return ORC_ENOMEM; }
    for (int i = 0; i < n; ++i) old_of_new[i] = -1;
    for (int o = 0; o < n; ++o) {              /* invert_permutation (color.cpp:144-153) */
        int id = new_of_old[o];
        if (id < 0 || id >= n) { free(old_of_new); free(cur); return ORC_EARG; }
        old_of_new[id] = o;
    }
    for (int c = 0; c <= nc; ++c) color_ptr[c] = 0;
    for (int i = 0; i < n; ++i) {
        int c = color[old_of_new[i]];
        if ((unsigned)c >= (unsigned)nc) { free(old_of_new); free(cur); return ORC_EARG; }
        color_ptr[c + 1]++;
    }
    for (int c = 0; c < nc; ++c) color_ptr[c + 1] += color_ptr[c];
    for (int c = 0; c <= nc; ++c) cur[c] = color_ptr[c];
    for (int i = 0; i < n; ++i) rows_of_color[cur[color[old_of_new[i]]]++] = i;
    free(old_of_new); free(cur);
    return ORC_OK;
}

/* a9: BuildABMCSchedule (block.cpp:116-174).  blocks_of_color lists blocks in
 * first-appearance order along the new ids (tail stays -1 if a block has no
 * rows); block_ptr is indexed by block id; rows_of_block lists new ids. */
int orc_abmc_schedule(int n, const int* new_of_old, const int* block_of_old,
                      const int* block_color, int nb, int nc,
                      int* color_ptr_blk, int* blocks_of_color, int* block_ptr,
                      int* rows_of_block)
{
    int* old_of_new = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    char* seen = (char*)calloc((size_t)nb + 1, 1);
    int* cur = (int*)malloc(sizeof(int) * (size_t)((nc > nb ? nc : nb) + 1));
    if (!old_of_new || !seen || !cur) { free(old_of_new); free(seen); free(cur); return ORC_ENOMEM; }
    for (int o = 0; o < n; ++o) old_of_new[new_of_old[o]] = o;
    for (int c = 0; c <= nc; ++c) color_ptr_blk[c] = 0;
    for (int i = 0; i < n; ++i) {
        int b = block_of_old[old_of_new[i]];
        if (!seen[b]) { seen[b] = 1; color_ptr_blk[block_color[b] + 1]++; }
    }
    for (int c = 0; c < nc; ++c) color_ptr_blk[c + 1] += color_ptr_blk[c];
    for (int b = 0; b < nb; ++b) blocks_of_color[b] = -1;
    for (int c = 0; c <= nc; ++c) cur[c] = color_ptr_blk[c];
    memset(seen, 0, (size_t)nb + 1);
    for (int i = 0; i < n; ++i) {
        int b = block_of_old[old_of_new[i]];
        if (!seen[b]) { seen[b] = 1; blocks_of_color[cur[block_color[b]]++] = b; }
    }
    for (int b = 0; b <= nb; ++b) block_ptr[b] = 0;
    for (int i = 0; i < n; ++i) block_ptr[block_of_old[old_of_new[i]] + 1]++;
    for (int b = 0; b < nb; ++b) block_ptr[b + 1] += block_ptr[b];
    for (int b = 0; b <= nb; ++b) cur[b] = block_ptr[b];
    for (int i = 0; i < n; ++i) rows_of_block[cur[block_of_old[old_of_new[i]]]++] = i;
    free(old_of_new); free(seen); free(cur);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a11: spmv (cg_crs.cpp:54-79), OpenMP branch: y_i = sum_k a_ik x_ck in CSR */
/* order; g++ keeps the product and the sum separately rounded here          */
/* (vmulsd + vaddsd: the reduction chain is not contracted).                */
/* ------------------------------------------------------------------------ */
void orc_spmv(int n, const int* rowptr, const int* colind, const double* val,
              const double* x, double* y)
{
    for (int i = 0; i < n; ++i) {
        double sum = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) sum = sum + val[k] * x[colind[k]];
        y[i] = sum;
    }
}

/* a12: dot / nrm2 (cg_crs.cpp:33-50): x87 long double accumulation. */
double orc_dot(int n, const double* a, const double* b)
{
    long double s = 0.0L;
    for (int i = 0; i < n; ++i) s += (long double)a[i] * b[i];
    return (double)s;
}

double orc_nrm2(int n, const double* a)
{
    long double s = 0.0L;
    for (int i = 0; i < n; ++i) s += (long double)a[i] * a[i];
    return sqrt((double)s);
}

/* ------------------------------------------------------------------------ */
/* IC(0) factor (ic0.cpp:6-151)                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n;
    int *Lp, *Li;  double* Lx;    /* L: lower + diagonal, CRS              */
    int* diag_pos;
    int *Up, *Ui;  double* Ux;    /* L^T as CSC of L (= CRS of L^T)        */
    int* LT_diag_pos;
} orc_ic0;

/* extract_lower_with_diag (ic0.cpp:14-38): entries with j <= i, row order kept */
static int orc_extract_lower(int n, const int* rowptr, const int* colind, const double* val,
                             int** Lp, int** Li, double** Lx)
{
    long nz = 0;
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) if (colind[k] <= i) ++nz;
    *Lp = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    *Li = (int*)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
    *Lx = (double*)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
    if (!*Lp || !*Li || !*Lx) return ORC_ENOMEM;
    int p = 0;
    for (int i = 0; i < n; ++i) {
        (*Lp)[i] = p;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (colind[k] <= i) { (*Li)[p] = colind[k]; (*Lx)[p] = val[k]; ++p; }
    }
    (*Lp)[n] = p;
    return ORC_OK;
}

void orc_ic0_free(orc_ic0* f)
{
    if (!f) return;
    free(f->Lp); free(f->Li); free(f->Lx); free(f->diag_pos);
    free(f->Up); free(f->Ui); free(f->Ux); free(f->LT_diag_pos);
    free(f);
}

/* IC0::IC0 -> extract_lower_with_diag, build_ic0 (ic0.cpp:40-116),
 * build_csc_from_crs (ic0.cpp:118-151). */
int orc_ic0_create(int n, const int* rowptr, const int* colind, const double* val,
                   double shift, orc_ic0** out)
{
    *out = NULL;
    orc_ic0* f = (orc_ic0*)calloc(1, sizeof(orc_ic0));
    if (!f) return ORC_ENOMEM;
    f->n = n;
    int rc = orc_extract_lower(n, rowptr, colind, val, &f->Lp, &f->Li, &f->Lx);
    if (rc) { orc_ic0_free(f); return rc; }
    int *Lp = f->Lp, *Li = f->Li; double* Lx = f->Lx;
    f->diag_pos = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        f->diag_pos[i] = -1;
        for (int k = Lp[i]; k < Lp[i + 1]; ++k) if (Li[k] == i) { f->diag_pos[i] = k; break; }
        if (f->diag_pos[i] < 0) { g_err_row = i; orc_ic0_free(f); return ORC_EDIAG; }
    }
    for (int i = 0; i < n; ++i) {
        for (int kij = Lp[i]; kij < Lp[i + 1]; ++kij) {
            int j = Li[kij];
            if (j >= i) break;
            double s = 0.0;
            int pi = Lp[i], pj = Lp[j];
            const int ei = Lp[i + 1], ej = Lp[j + 1];
            while (pi < ei && pj < ej) {           /* two-pointer dot (ic0.cpp:69-81) */
                int ci = Li[pi], cj = Li[pj];
                if (ci >= j || cj >= j) break;
                if (ci == cj) { s = fma(Lx[pi], Lx[pj], s); ++pi; ++pj; }
                else if (ci < cj) ++pi;
                else ++pj;
            }
            double Ljj = Lx[f->diag_pos[j]];
            if (fabs(Ljj) < 1e-30) { g_err_row = j; orc_ic0_free(f); return ORC_EPIVZ; }
            Lx[kij] = (Lx[kij] - s) / Ljj;
        }
        double s = 0.0;                          /* not contracted by g++ */
        for (int k = Lp[i]; k < Lp[i + 1]; ++k) {
            int j = Li[k];
            if (j >= i) break;
            s = s + Lx[k] * Lx[k];
        }
        int di = f->diag_pos[i];
        double diag = Lx[di] - s;
        diag += shift;
        if (diag <= 0.0) { g_err_row = i; orc_ic0_free(f); return ORC_EPIVN; }
        Lx[di] = sqrt(diag);
    }
    /* CSC of L (ic0.cpp:118-151) */
    int nz = Lp[n];
    f->Up = (int*)calloc((size_t)n + 1, sizeof(int));
    f->Ui = (int*)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
    f->Ux = (double*)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
    f->LT_diag_pos = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* ctr = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    if (!f->Up || !f->Ui || !f->Ux || !f->LT_diag_pos || !ctr) { free(ctr); orc_ic0_free(f); return ORC_ENOMEM; }
    for (int i = 0; i < n; ++i) f->LT_diag_pos[i] = -1;
    for (int k = 0; k < nz; ++k) f->Up[Li[k] + 1]++;
    for (int c = 0; c < n; ++c) f->Up[c + 1] += f->Up[c];
    memcpy(ctr, f->Up, sizeof(int) * (size_t)(n + 1));
    for (int i = 0; i < n; ++i)
        for (int k = Lp[i]; k < Lp[i + 1]; ++k) {
            int c = Li[k];
            int pos = ctr[c]++;
            f->Ui[pos] = i; f->Ux[pos] = Lx[k];
            if (i == c) f->LT_diag_pos[i] = pos;
        }
    free(ctr);
    *out = f;
    return ORC_OK;
}

int orc_ic0_nnz(const orc_ic0* f) { return f->Lp[f->n]; }

void orc_ic0_export(const orc_ic0* f, int* Lp, int* Li, double* Lx, int* Up, int* Ui, double* Ux)
{
    int n = f->n, nz = f->Lp[n];
    if (Lp) memcpy(Lp, f->Lp, sizeof(int) * (size_t)(n + 1));
    if (Li) memcpy(Li, f->Li, sizeof(int) * (size_t)nz);
    if (Lx) memcpy(Lx, f->Lx, sizeof(double) * (size_t)nz);
    if (Up) memcpy(Up, f->Up, sizeof(int) * (size_t)(n + 1));
    if (Ui) memcpy(Ui, f->Ui, sizeof(int) * (size_t)nz);
    if (Ux) memcpy(Ux, f->Ux, sizeof(double) * (size_t)nz);
}

/* a17: forward_solve / backward_solve (ic0.cpp:153-184) */
static void orc_fwd_seq(const orc_ic0* f, const double* b, double* y)
{
    for (int i = 0; i < f->n; ++i) {
        double s = b[i], di = 1.0;
        for (int k = f->Lp[i]; k < f->Lp[i + 1]; ++k) {
            int j = f->Li[k];
            if (j < i) s = fma(-f->Lx[k], y[j], s);
            else if (j == i) di = f->Lx[k];
            else break;
        }
        y[i] = s / di;
    }
}

static void orc_bwd_seq(const orc_ic0* f, const double* y, double* x)
{
    for (int i = f->n - 1; i >= 0; --i) {
        double s = y[i], di = 1.0;
        for (int k = f->Up[i]; k < f->Up[i + 1]; ++k) {
            int j = f->Ui[k];
            if (j > i) s = fma(-f->Ux[k], x[j], s);
            else if (j == i) di = f->Ux[k];
        }
        x[i] = s / di;
    }
}

/* one row of forward_solve_mc / forward_solve_abmc (ic0.cpp:201-214, 280-295) */
static void orc_fwd_row(const orc_ic0* f, int i, const double* r, double* y)
{
    double di = f->Lx[f->diag_pos[i]];
    double acc = r[i];
    for (int jj = f->Lp[i]; jj < f->Lp[i + 1]; ++jj) {
        int j = f->Li[jj];
        if (j < i) acc = fma(-f->Lx[jj], y[j], acc);
        else if (j == i) { }
        else break;
    }
    y[i] = acc / di;
}

/* one row of backward_solve_mc / backward_solve_abmc (ic0.cpp:229-244, 319-334) */
static void orc_bwd_row(const orc_ic0* f, int i, const double* y, double* x)
{
    double di = f->Ux[f->LT_diag_pos[i]];
    double acc = y[i];
    for (int jj = f->Up[i]; jj < f->Up[i + 1]; ++jj) {
        int j = f->Ui[jj];
        if (j > i) acc = fma(-f->Ux[jj], x[j], acc);
    }
    x[i] = acc / di;
}

/* ColorSchedule (color.hpp:9-22) */
typedef struct {
    int nc;
    const int* color_ptr;
    const int* rows_of_color;
    int mode;                 /* 0 = MC_NODE, 1 = ABMC_BLOCK */
    int nb;
    const int* color_ptr_blk;
    const int* blocks_of_color;
    const int* block_ptr;
    const int* rows_of_block;
} orc_sched;

/* a18/a19/a20: IC0::apply(r, z, sched) dispatch (ic0.cpp:366-393).  For a
 * schedule whose colors respect the dependencies the parallel loops of the
 * reference compute every row from finished inputs, so the restatement runs
 * them in schedule order on one thread.  y starts zero-filled as the
 * reference's std::vector<double> y(n) does (ic0.cpp:372). */
int orc_ic0_apply(const orc_ic0* f, const double* r, double* z, const orc_sched* s)
{
    int n = f->n;
    double* y = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    if (!y) return ORC_ENOMEM;
    if (!s || s->nc <= 0) {
        orc_fwd_seq(f, r, y);
        orc_bwd_seq(f, y, z);
    } else if (s->mode == 1 && s->color_ptr_blk && s->blocks_of_color && s->block_ptr && s->rows_of_block) {
        for (int c = 0; c < s->nc; ++c)
            for (int kb = s->color_ptr_blk[c]; kb < s->color_ptr_blk[c + 1]; ++kb) {
                int b = s->blocks_of_color[kb];
                for (int t = s->block_ptr[b]; t < s->block_ptr[b + 1]; ++t)
                    orc_fwd_row(f, s->rows_of_block[t], r, y);
            }
        for (int c = s->nc - 1; c >= 0; --c)
            for (int kb = s->color_ptr_blk[c]; kb < s->color_ptr_blk[c + 1]; ++kb) {
                int b = s->blocks_of_color[kb];
                for (int t = s->block_ptr[b + 1] - 1; t >= s->block_ptr[b]; --t)
                    orc_bwd_row(f, s->rows_of_block[t], y, z);
            }
    } else if (s->color_ptr && s->rows_of_color) {
        for (int c = 0; c < s->nc; ++c)
            for (int k = s->color_ptr[c]; k < s->color_ptr[c + 1]; ++k)
                orc_fwd_row(f, s->rows_of_color[k], r, y);
        for (int c = s->nc - 1; c >= 0; --c)
            for (int k = s->color_ptr[c]; k < s->color_ptr[c + 1]; ++k)
                orc_bwd_row(f, s->rows_of_color[k], y, z);
    } else {
        orc_fwd_seq(f, r, y);
        orc_bwd_seq(f, y, z);
    }
    free(y);
    return ORC_OK;
}

/* a14: Jacobi (precond.hpp:19-45): inv_diag from the first diagonal entry of
 * each row, 1.0 where it is zero or missing; apply z_i = inv_diag_i * r_i. */
void orc_jacobi_inv_diag(int n, const int* rowptr, const int* colind, const double* val, double* inv)
{
    for (int i = 0; i < n; ++i) {
        double d = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (colind[k] == i) { d = val[k]; break; }
        inv[i] = (fabs(d) > 0.0) ? 1.0 / d : 1.0;
    }
}

/* ------------------------------------------------------------------------ */
/* a13: conjugate_gradient<Precond> (cg_crs.cpp:89-162)                       */
/* kind: 0 Identity (precond.hpp:8-17), 1 Jacobi, 2 IC0.                     */
/* history (optional, length max_iter+1): rel_resid after each iteration.    */
/* ------------------------------------------------------------------------ */
typedef struct { int iters; double rel_resid; int converged; } orc_cg_result;

static void orc_precond(int kind, const double* inv, const orc_ic0* f, const orc_sched* s,
                        int n, const double* r, double* z)
{
    if (kind == 0) { memcpy(z, r, sizeof(double) * (size_t)n); }
    else if (kind == 1) { for (int i = 0; i < n; ++i) z[i] = inv[i] * r[i]; }
    else orc_ic0_apply(f, r, z, s);
}

int orc_cg(int n, const int* rowptr, const int* colind, const double* val,
           const double* b, double* x, int kind, const double* inv_diag,
           const orc_ic0* f, const orc_sched* s, int max_iter, double tol,
           orc_cg_result* res, double* history)
{
    double* r = (double*)calloc((size_t)n + 1, sizeof(double));
    double* p = (double*)calloc((size_t)n + 1, sizeof(double));
    double* z = (double*)calloc((size_t)n + 1, sizeof(double));
    double* Ap = (double*)calloc((size_t)n + 1, sizeof(double));
    double* Ax = (double*)calloc((size_t)n + 1, sizeof(double));
    if (!r || !p || !z || !Ap || !Ax) { free(r); free(p); free(z); free(Ap); free(Ax); return ORC_ENOMEM; }
    orc_spmv(n, rowptr, colind, val, x, Ax);
    for (int i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    double normb = orc_nrm2(n, b);
    if (normb == 0.0) normb = 1.0;
    orc_precond(kind, inv_diag, f, s, n, r, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz_old = orc_dot(n, r, z);
    res->iters = 0; res->converged = 0;
    res->rel_resid = orc_nrm2(n, r) / normb;
    if (history) history[0] = res->rel_resid;
    if (res->rel_resid < tol) { res->converged = 1; res->iters = 0; goto done; }
    for (int k = 0; k < max_iter; ++k) {
        orc_spmv(n, rowptr, colind, val, p, Ap);
        double pAp = orc_dot(n, p, Ap);
        double eps = 2.220446049250313080847e-16;
        double thr = eps * orc_nrm2(n, p) * orc_nrm2(n, Ap);
        if (pAp <= thr) { res->iters = k; goto done; }
        double alpha = rz_old / pAp;
        for (int i = 0; i < n; ++i) {
            x[i] = fma(alpha, p[i], x[i]);
            r[i] = fma(-alpha, Ap[i], r[i]);
        }
        double rel = orc_nrm2(n, r) / normb;
        res->iters = k + 1;
        res->rel_resid = rel;
        if (history) history[k + 1] = rel;
        if (rel < tol) { res->converged = 1; goto done; }
        orc_precond(kind, inv_diag, f, s, n, r, z);
        double rz_new = orc_dot(n, r, z);
        double beta = rz_new / rz_old;
        for (int i = 0; i < n; ++i) p[i] = fma(beta, p[i], z[i]);
        rz_old = rz_new;
    }
done:
    free(r); free(p); free(z); free(Ap); free(Ax);
    return ORC_OK;
}

/* a21: true residual ||A x - b|| / ||b|| (cg_crs.cpp:518-528) evaluated on
 * one thread (the reference's OpenMP reduction partial order is not fixed). */
double orc_true_resid(int n, const int* rowptr, const int* colind, const double* val,
                      const double* x, const double* b)
{
    double* Ax = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (!Ax) return NAN;
    orc_spmv(n, rowptr, colind, val, x, Ax);
    double nr = 0.0, nb = 0.0;
    for (int i = 0; i < n; ++i) {
        double d = Ax[i] - b[i];
        nr = nr + d * d;
        nb = nb + b[i] * b[i];
    }
    free(Ax);
    return sqrt(nr) / sqrt(nb);
}

/* ------------------------------------------------------------------------ */
/* a22: schedule hazard checkers (cg_crs.cpp:171-224, 259-336).              */
/* ------------------------------------------------------------------------ */
/* DebugCheck_InterBlockSameColorEdges: edges (i<j) between different blocks
 * of the same color; per-color counts into conflicts_by_color (length nc). */
long orc_check_interblock_same_color(int n, const int* rowptr, const int* colind,
                                     const int* block_of_old, const int* block_color,
                                     int nb, int nc, long* conflicts_by_color)
{
    long total = 0;
    for (int c = 0; c < nc; ++c) if (conflicts_by_color) conflicts_by_color[c] = 0;
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            if (j <= i) continue;
            int bi = block_of_old[i], bj = block_of_old[j];
            if (bi < 0 || bi >= nb || bj < 0 || bj >= nb) return -1;
            if (bi == bj) continue;
            int ci = block_color[bi], cj = block_color[bj];
            if (ci < 0 || ci >= nc || cj < 0 || cj >= nc) return -1;
            if (ci == cj) { if (conflicts_by_color) conflicts_by_color[ci]++; ++total; }
        }
    return total;
}

/* DebugCheck_ScheduleHazards_OnLower: same-color dependencies j<i in the
 * lower pattern of the permuted matrix, split into same-block / cross-block
 * when block ids are given (block_of_old may be NULL). */
long orc_check_schedule_hazards(int n, const int* rowptr, const int* colind,
                                const int* new_of_old, const int* color_old,
                                const int* block_of_old, long* same_block, long* cross_block)
{
    int* old_of_new = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!old_of_new) return -1;
    for (int o = 0; o < n; ++o) {
        int id = new_of_old[o];
        if (id < 0 || id >= n) { free(old_of_new); return -1; }
        old_of_new[id] = o;
    }
    long total = 0, sb = 0, xb = 0;
    for (int i = 0; i < n; ++i) {
        int ci = color_old[old_of_new[i]];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colind[k];
            if (j > i) continue;           /* lower pattern: j <= i      */
            if (j >= i) break;             /* cg_crs.cpp:305             */
            if (color_old[old_of_new[j]] == ci) {
                ++total;
                if (block_of_old) {
                    if (block_of_old[old_of_new[i]] == block_of_old[old_of_new[j]]) ++sb;
                    else ++xb;
                }
            }
        }
    }
    free(old_of_new);
    if (same_block) *same_block = sb;
    if (cross_block) *cross_block = xb;
    return total;
}

/* ------------------------------------------------------------------------ */
/* a2: read_matrix_market_crs / coo_to_crs (crs_io.cpp:19-159)                */
/* Two calls: orc_mm_read parses into a heap COO -> CRS held by the handle.  */
/* Duplicate (i,j) entries are summed in file order.                         */
/* ------------------------------------------------------------------------ */
typedef struct { int n, nnz; int* rowptr; int* colind; double* val; } orc_crs;

void orc_crs_free(orc_crs* a)
{
    if (!a) return;
    free(a->rowptr); free(a->colind); free(a->val); free(a);
}
int orc_crs_n(const orc_crs* a) { return a->n; }
int orc_crs_nnz(const orc_crs* a) { return a->nnz; }
void orc_crs_copy(const orc_crs* a, int* rowptr, int* colind, double* val)
{
    memcpy(rowptr, a->rowptr, sizeof(int) * (size_t)(a->n + 1));
    memcpy(colind, a->colind, sizeof(int) * (size_t)a->nnz);
    memcpy(val, a->val, sizeof(double) * (size_t)a->nnz);
}

static void orc_lower(char* s) { for (; *s; ++s) *s = (char)tolower((unsigned char)*s); }

typedef struct { int i, j; double v; long ord; } orc_coo;
static int cmp_coo(const void* pa, const void* pb)
{
    const orc_coo* a = (const orc_coo*)pa; const orc_coo* b = (const orc_coo*)pb;
    if (a->i != b->i) return a->i < b->i ? -1 : 1;
    if (a->j != b->j) return a->j < b->j ? -1 : 1;
    return (a->ord > b->ord) - (a->ord < b->ord);
}

static int orc_getline(FILE* f, char** buf, size_t* cap)
{
    size_t len = 0;
    int ch;
    if (!*buf) { *cap = 256; *buf = (char*)malloc(*cap); }
    while ((ch = fgetc(f)) != EOF) {
        if (len + 2 > *cap) { *cap *= 2; *buf = (char*)realloc(*buf, *cap); }
        if (ch == '\n') break;
        (*buf)[len++] = (char)ch;
    }
    if (ch == EOF && len == 0) return -1;
    (*buf)[len] = 0;
    return (int)len;
}

int orc_mm_read(const char* path, orc_crs** out)
{
    *out = NULL;
    FILE* f = fopen(path, "r");
    if (!f) return ORC_EIO;
    char* line = NULL; size_t cap = 0;
    char banner[64], mtx[64], storage[64], field[64], sym[64];
    if (orc_getline(f, &line, &cap) < 0) goto bad;
    if (sscanf(line, "%63s %63s %63s %63s %63s", banner, mtx, storage, field, sym) != 5) goto bad;
    if (strcmp(banner, "%%MatrixMarket") != 0) goto bad;
    orc_lower(mtx); orc_lower(storage); orc_lower(field); orc_lower(sym);
    if (strcmp(mtx, "matrix") || strcmp(storage, "coordinate")) goto bad;
    int is_pattern = !strcmp(field, "pattern");
    if (!(is_pattern || !strcmp(field, "real") || !strcmp(field, "integer"))) goto bad;
    int is_sym = !strcmp(sym, "symmetric");
    if (!(is_sym || !strcmp(sym, "general"))) goto bad;
    int nrows = 0, ncols = 0, nnz = 0;
    for (;;) {                                   /* skip_comments + size line */
        if (orc_getline(f, &line, &cap) < 0) goto bad;
        if (line[0] == '%') continue;
        if (sscanf(line, "%d %d %d", &nrows, &ncols, &nnz) != 3) goto bad;
        break;
    }
    orc_coo* e = (orc_coo*)malloc(sizeof(orc_coo) * (size_t)(2 * (long)nnz + 1));
    if (!e) goto bad;
    long m = 0;
    for (int k = 0; k < nnz; ++k) {
        if (orc_getline(f, &line, &cap) < 0) { free(e); goto bad; }
        if (line[0] == 0 || line[0] == '%') { --k; continue; }
        char* p = line; char* q;
        long long ii = strtoll(p, &q, 10); if (q == p) { free(e); goto bad; } p = q;
        long long jj = strtoll(p, &q, 10); if (q == p) { free(e); goto bad; } p = q;
        double v = 1.0;
        if (!is_pattern) { v = strtod(p, &q); if (q == p) { free(e); goto bad; } }
        int i = (int)(ii - 1), j = (int)(jj - 1);
        if (i < 0 || i >= nrows || j < 0 || j >= ncols) { free(e); goto bad; }
        e[m].i = i; e[m].j = j; e[m].v = v; e[m].ord = m; ++m;
        if (is_sym && i != j) { e[m].i = j; e[m].j = i; e[m].v = v; e[m].ord = m; ++m; }
    }
    qsort(e, (size_t)m, sizeof(orc_coo), cmp_coo);
    orc_crs* a = (orc_crs*)calloc(1, sizeof(orc_crs));
    a->n = nrows;
    a->rowptr = (int*)calloc((size_t)nrows + 1, sizeof(int));
    a->colind = (int*)malloc(sizeof(int) * (size_t)(m + 1));
    a->val = (double*)malloc(sizeof(double) * (size_t)(m + 1));
    long u = 0;
    for (long idx = 0; idx < m;) {
        int r = e[idx].i, c = e[idx].j;
        double s = 0.0;
        do { s += e[idx].v; ++idx; } while (idx < m && e[idx].i == r && e[idx].j == c);
        a->colind[u] = c; a->val[u] = s; a->rowptr[r + 1]++; ++u;
    }
    for (int i = 0; i < nrows; ++i) a->rowptr[i + 1] += a->rowptr[i];
    a->nnz = (int)u;
    free(e); free(line); fclose(f);
    *out = a;
    return ORC_OK;
bad:
    free(line); fclose(f);
    return ORC_EIO;
}

/* a4: ReadColorFile_1Based (color.cpp:14-47), ReadBlockFile_1Based
 * (block.cpp:15-51), ReadBlockColorFile_1Based (block.cpp:53-89): first
 * integer = count K (> 0); then pairs "id value" (1-based), id in [1..n],
 * value in [1..K]; duplicates overwrite; every id must be assigned.
 * Output is 0-based; *k_out receives K. */
int orc_read_assignment(const char* path, int n_expected, int* out, int* k_out)
{
    FILE* f = fopen(path, "r");
    if (!f) return ORC_EIO;
    int K;
    if (fscanf(f, "%d", &K) != 1 || K <= 0) { fclose(f); return ORC_EIO; }
    for (int i = 0; i < n_expected; ++i) out[i] = -1;
    int assigned = 0, id, v;
    while (fscanf(f, "%d %d", &id, &v) == 2) {
        if (id < 1 || id > n_expected || v < 1 || v > K) { fclose(f); return ORC_EIO; }
        if (out[id - 1] == -1) ++assigned;
        out[id - 1] = v - 1;
    }
    fclose(f);
    if (assigned != n_expected) return ORC_EIO;
    *k_out = K;
    return ORC_OK;
}
