// host_gen.cpp -- synthetic SPD problems, colorings and ABMC blockings.
//
// The reference ships none of these: its inputs are SuiteSparse matrices and
// .col/.blk/.bcol files made by an external tool (run_mc.sh:14,
// run_abmc.sh:19-20, check_igraph.cpp:1-13).  Everything here is seeded and
// deterministic, and feeds the oracle and the GPU path the same arrays.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

#include "host.hpp"
#include "../../include/iccg.h"

namespace iccg {

void gen_uniform(int n, uint64_t seed, double* out)
{
    uint64_t s = seed;
    for (int i = 0; i < n; ++i) out[i] = u01(s) * 2.0 - 1.0;
}

// 5-point (2D) / 7-point (3D) Dirichlet stencils in lexicographic order
// (x fastest).  Off-diagonals -w per direction, diagonal 2*sum(w).
CRS gen_stencil(int kind, int nx, int ny, int nz, double wx, double wy, double wz)
{
    if (nx <= 0 || ny <= 0 || (kind == ICCG_GEN_3D7 && nz <= 0)) throw Error(ICCG_ERR_ARG, "bad grid");
    if (kind != ICCG_GEN_2D5 && kind != ICCG_GEN_3D7) throw Error(ICCG_ERR_ARG, "bad stencil kind");
    const bool three = kind == ICCG_GEN_3D7;
    if (!three) nz = 1;
    const long long nl = (long long)nx * ny * nz;
    if (nl * (three ? 7 : 5) > 2147483647LL) throw Error(ICCG_ERR_ARG, "grid too large for int32 CRS");
    const int n = (int)nl;
    CRS A;
    A.n = n;
    A.rowptr.resize((size_t)n + 1);
    A.colind.reserve((size_t)n * (three ? 7 : 5));
    A.val.reserve((size_t)n * (three ? 7 : 5));
    const double diag = three ? 2.0 * (wx + wy + wz) : 2.0 * (wx + wy);
    const int sxy = nx * ny;
    A.rowptr[0] = 0;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int id = x + nx * (y + ny * z);
                auto put = [&](int c, double v) { A.colind.push_back(c); A.val.push_back(v); };
                if (three && z > 0) put(id - sxy, -wz);
                if (y > 0) put(id - nx, -wy);
                if (x > 0) put(id - 1, -wx);
                put(id, diag);
                if (x + 1 < nx) put(id + 1, -wx);
                if (y + 1 < ny) put(id + nx, -wy);
                if (three && z + 1 < nz) put(id + sxy, -wz);
                A.rowptr[(size_t)id + 1] = (int)A.colind.size();
            }
    return A;
}

// 27-point cell-centred diffusion.  kappa = exp(sigma * g), g a Gaussian
// field (Box-Muller on splitmix64) smoothed by a 3x3x3 box filter (mean over
// the cells inside the grid) and normalised to zero mean, unit variance;
// sigma = ln(contrast) / (max g - min g), so max kappa / min kappa = contrast.
// The coupling of cells p and q (q in the 26-neighbourhood) is
// -w * 2 kp kq / (kp + kq), with w = 1 (face), 1/2 (edge), 1/4 (corner).
// The diagonal sums the couplings of all 26 neighbours, those outside the
// grid taken with kappa_q = kappa_p (Dirichlet), so A is an SPD M-matrix.
CRS gen_diffusion27(int nx, int ny, int nz, double contrast, uint64_t seed)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !(contrast >= 1.0)) throw Error(ICCG_ERR_ARG, "bad diffusion27 args");
    const long long nl = (long long)nx * ny * nz;
    if (nl * 27 > 2147483647LL) throw Error(ICCG_ERR_ARG, "grid too large for int32 CRS");
    const int n = (int)nl;
    std::vector<double> g0((size_t)n), g((size_t)n);
    uint64_t s = seed;
    for (int i = 0; i < n; i += 2) {
        double u1 = u01(s), u2 = u01(s);
        if (u1 < 1e-300) u1 = 1e-300;
        double rad = std::sqrt(-2.0 * std::log(u1)), th = 2.0 * M_PI * u2;
        g0[(size_t)i] = rad * std::cos(th);
        if (i + 1 < n) g0[(size_t)i + 1] = rad * std::sin(th);
    }
    auto idx = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); };
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double acc = 0.0;
                int cnt = 0;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            int X = x + dx, Y = y + dy, Z = z + dz;
                            if (X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz) continue;
                            acc += g0[idx(X, Y, Z)];
                            ++cnt;
                        }
                g[idx(x, y, z)] = acc / cnt;
            }
    double mean = 0.0;
    for (double v : g) mean += v;
    mean /= n;
    double var = 0.0;
    for (double v : g) var += (v - mean) * (v - mean);
    double sd = std::sqrt(var / n);
    if (!(sd > 0.0)) sd = 1.0;
    double gmin = 1e300, gmax = -1e300;
    for (double& v : g) {
        v = (v - mean) / sd;
        gmin = std::min(gmin, v);
        gmax = std::max(gmax, v);
    }
    const double sigma = (gmax > gmin) ? std::log(contrast) / (gmax - gmin) : 0.0;
    std::vector<double> kap((size_t)n);
    for (int i = 0; i < n; ++i) kap[(size_t)i] = std::exp(sigma * g[(size_t)i]);
    auto hm = [](double a, double b) { return 2.0 * a * b / (a + b); };
    CRS A;
    A.n = n;
    A.rowptr.resize((size_t)n + 1);
    A.rowptr[0] = 0;
    A.colind.reserve((size_t)n * 27);
    A.val.reserve((size_t)n * 27);
    static const double wt[4] = {0.0, 1.0, 0.5, 0.25};
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t p = idx(x, y, z);
                const double kp = kap[p];
                double diag = 0.0;
                size_t diag_slot = 0;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            const int m = std::abs(dx) + std::abs(dy) + std::abs(dz);
                            if (m == 0) {
                                diag_slot = A.colind.size();
                                A.colind.push_back((int)p);
                                A.val.push_back(0.0);
                                continue;
                            }
                            int X = x + dx, Y = y + dy, Z = z + dz;
                            const bool inside = !(X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz);
                            const double c = wt[m] * hm(kp, inside ? kap[idx(X, Y, Z)] : kp);
                            diag += c;
                            if (inside) {
                                A.colind.push_back((int)idx(X, Y, Z));
                                A.val.push_back(-c);
                            }
                        }
                A.val[diag_slot] = diag;
                A.rowptr[p + 1] = (int)A.colind.size();
            }
    return A;
}

// Symmetrised k-NN graph Laplacian on npts uniform points in [0,1)^2:
// edge (i,j) if j is among the k nearest of i or i among those of j, weight
// 1/dist; A = D - W + diag_shift * I.  Neighbour search on a uniform grid.
CRS gen_knn_laplacian(int npts, int k, double diag_shift, uint64_t seed)
{
    if (npts <= 1 || k <= 0 || k >= npts) throw Error(ICCG_ERR_ARG, "bad knn args");
    const int n = npts;
    std::vector<double> px((size_t)n), py((size_t)n);
    uint64_t s = seed;
    for (int i = 0; i < n; ++i) { px[(size_t)i] = u01(s); py[(size_t)i] = u01(s); }
    // about 4 points per grid cell (the search is exact for any cell size:
    // it widens by rings until no point outside can be nearer than the k-th)
    const int G = std::max(1, (int)std::sqrt((double)n / 4.0));
    std::vector<int> cell_ptr((size_t)G * G + 1, 0), cell_pts((size_t)n);
    auto cell_of = [&](double v) { int c = (int)(v * G); return c >= G ? G - 1 : c; };
    for (int i = 0; i < n; ++i) cell_ptr[(size_t)cell_of(px[(size_t)i]) + (size_t)G * cell_of(py[(size_t)i]) + 1]++;
    for (size_t c = 0; c < (size_t)G * G; ++c) cell_ptr[c + 1] += cell_ptr[c];
    {
        std::vector<int> cur(cell_ptr.begin(), cell_ptr.end() - 1);
        for (int i = 0; i < n; ++i) cell_pts[(size_t)cur[(size_t)cell_of(px[(size_t)i]) + (size_t)G * cell_of(py[(size_t)i])]++] = i;
    }
    std::vector<int> nbr((size_t)n * k);
    std::vector<std::pair<double, int>> cand;
    for (int i = 0; i < n; ++i) {
        const int cx = cell_of(px[(size_t)i]), cy = cell_of(py[(size_t)i]);
        cand.clear();
        for (int ring = 0;; ++ring) {
            for (int yy = cy - ring; yy <= cy + ring; ++yy)
                for (int xx = cx - ring; xx <= cx + ring; ++xx) {
                    if (std::max(std::abs(xx - cx), std::abs(yy - cy)) != ring) continue;
                    if (xx < 0 || yy < 0 || xx >= G || yy >= G) continue;
                    const size_t c = (size_t)xx + (size_t)G * yy;
                    for (int t = cell_ptr[c]; t < cell_ptr[c + 1]; ++t) {
                        const int j = cell_pts[(size_t)t];
                        if (j == i) continue;
                        const double dx = px[(size_t)i] - px[(size_t)j], dy = py[(size_t)i] - py[(size_t)j];
                        cand.emplace_back(dx * dx + dy * dy, j);
                    }
                }
            // points outside the searched square are at least ring/G away
            if ((int)cand.size() >= k) {
                std::nth_element(cand.begin(), cand.begin() + (k - 1), cand.end());
                const double rk = (double)ring / G;
                if (cand[(size_t)k - 1].first <= rk * rk || ring > G) break;
            }
            if (ring > G) break;
        }
        std::partial_sort(cand.begin(), cand.begin() + k, cand.end());
        for (int t = 0; t < k; ++t) nbr[(size_t)i * k + t] = cand[(size_t)t].second;
    }
    // symmetrise: row i holds its k neighbours and every point that has i
    // among its neighbours, ascending, without repeats (per-row buckets,
    // each sorted on its own)
    std::vector<int> deg((size_t)n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int t = 0; t < k; ++t) {
            deg[(size_t)i + 1]++;
            deg[(size_t)nbr[(size_t)i * k + t] + 1]++;
        }
    for (int i = 0; i < n; ++i) deg[(size_t)i + 1] += deg[(size_t)i];
    std::vector<int> adj((size_t)deg[(size_t)n]);
    {
        std::vector<int> cur(deg.begin(), deg.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int t = 0; t < k; ++t) {
                const int j = nbr[(size_t)i * k + t];
                adj[(size_t)cur[(size_t)i]++] = j;
                adj[(size_t)cur[(size_t)j]++] = i;
            }
    }
    std::vector<int> ulen((size_t)n);
    for (int i = 0; i < n; ++i) {
        auto b = adj.begin() + deg[(size_t)i], e = adj.begin() + deg[(size_t)i + 1];
        std::sort(b, e);
        ulen[(size_t)i] = (int)(std::unique(b, e) - b);
    }
    CRS A;
    A.n = n;
    A.rowptr.assign((size_t)n + 1, 0);
    for (int i = 0; i < n; ++i) A.rowptr[(size_t)i + 1] = A.rowptr[(size_t)i] + ulen[(size_t)i] + 1;  // + diagonal
    A.colind.resize((size_t)A.rowptr[(size_t)n]);
    A.val.resize((size_t)A.rowptr[(size_t)n]);
    for (int i = 0; i < n; ++i) {
        int pos = A.rowptr[(size_t)i];
        double dsum = 0.0;
        int dslot = -1;
        bool placed = false;
        for (int t = 0; t < ulen[(size_t)i]; ++t) {
            const int j = adj[(size_t)deg[(size_t)i] + t];
            if (!placed && j > i) { dslot = pos; A.colind[(size_t)pos++] = i; placed = true; }
            const double dx = px[(size_t)i] - px[(size_t)j], dy = py[(size_t)i] - py[(size_t)j];
            const double w = 1.0 / std::max(std::sqrt(dx * dx + dy * dy), 1e-12);
            A.colind[(size_t)pos] = j;
            A.val[(size_t)pos++] = -w;
            dsum += w;
        }
        if (!placed) { dslot = pos; A.colind[(size_t)pos++] = i; }
        A.val[(size_t)dslot] = dsum + diag_shift;
    }
    return A;
}

// Greedy coloring in natural order: each node takes the smallest color not
// used by an already colored neighbour.  Returns the number of colors.
int color_greedy(int n, const int* rowptr, const int* colind, int* color)
{
    std::vector<int> mark;
    int nc = 0;
    for (int i = 0; i < n; ++i) color[i] = -1;
    for (int i = 0; i < n; ++i) {
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int j = colind[k];
            if (j != i && color[j] >= 0) {
                if ((size_t)color[j] >= mark.size()) mark.resize((size_t)color[j] + 1, -1);
                mark[(size_t)color[j]] = i;
            }
        }
        int c = 0;
        while ((size_t)c < mark.size() && mark[(size_t)c] == i) ++c;
        color[i] = c;
        nc = std::max(nc, c + 1);
    }
    return nc;
}

// ABMC blocking.  method 0: block = id / B.  method 1: breadth-first
// aggregation -- the smallest unassigned node seeds a block that grows over
// unassigned neighbours (in column order) until it holds B nodes.
int block_partition(int n, const int* rowptr, const int* colind, int B, int method, int* block_of_old)
{
    if (B <= 0) throw Error(ICCG_ERR_ARG, "block size must be positive");
    if (method == 0) {
        for (int i = 0; i < n; ++i) block_of_old[i] = i / B;
        return (n + B - 1) / B;
    }
    if (method != 1) throw Error(ICCG_ERR_ARG, "bad blocking method");
    for (int i = 0; i < n; ++i) block_of_old[i] = -1;
    std::vector<int> queue;
    queue.reserve(1024);
    int nb = 0;
    for (int seed = 0; seed < n; ++seed) {
        if (block_of_old[seed] >= 0) continue;
        queue.clear();
        queue.push_back(seed);
        size_t head = 0;
        int cnt = 0;
        while (head < queue.size() && cnt < B) {
            const int u = queue[head++];
            if (block_of_old[u] >= 0) continue;
            block_of_old[u] = nb;
            ++cnt;
            for (int k = rowptr[u]; k < rowptr[u + 1]; ++k) {
                const int v = colind[k];
                if (block_of_old[v] < 0) queue.push_back(v);
            }
        }
        ++nb;
    }
    return nb;
}

// Greedy coloring of the block quotient graph (blocks adjacent when any of
// their nodes are), blocks visited in id order.
int color_blocks(int n, const int* rowptr, const int* colind, const int* block_of_old, int nb,
                 int* block_color)
{
    std::vector<int> bptr((size_t)nb + 1, 0), rows((size_t)n);
    for (int i = 0; i < n; ++i) {
        if (block_of_old[i] < 0 || block_of_old[i] >= nb) throw Error(ICCG_ERR_ARG, "block id out of range");
        bptr[(size_t)block_of_old[i] + 1]++;
    }
    for (int b = 0; b < nb; ++b) bptr[(size_t)b + 1] += bptr[(size_t)b];
    {
        std::vector<int> cur(bptr.begin(), bptr.end() - 1);
        for (int i = 0; i < n; ++i) rows[(size_t)cur[(size_t)block_of_old[i]]++] = i;
    }
    for (int b = 0; b < nb; ++b) block_color[b] = -1;
    std::vector<int> mark;
    int nc = 0;
    for (int b = 0; b < nb; ++b) {
        for (int t = bptr[(size_t)b]; t < bptr[(size_t)b + 1]; ++t) {
            const int i = rows[(size_t)t];
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
                const int bj = block_of_old[colind[k]];
                if (bj == b) continue;
                const int c = block_color[bj];
                if (c >= 0) {
                    if ((size_t)c >= mark.size()) mark.resize((size_t)c + 1, -1);
                    mark[(size_t)c] = b;
                }
            }
        }
        int c = 0;
        while ((size_t)c < mark.size() && mark[(size_t)c] == b) ++c;
        block_color[b] = c;
        nc = std::max(nc, c + 1);
    }
    return nc;
}

}  // namespace iccg
