// host.hpp -- host-side data structures and set-up routines of iccg_b200.
//
// The CRS container and ColorSchedule view keep the reference's layout
// (crs_io.hpp:10-49, color.hpp:9-22).  Every ordering routine here is a new
// implementation that reproduces the reference's output bit for bit; the
// file:line of the reference function each one stands in for is given at
// its definition.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace iccg {

struct CRS {
    int n = 0;
    std::vector<int> rowptr;   // n+1
    std::vector<int> colind;   // nnz
    std::vector<double> val;   // nnz
    int nnz() const { return (int)colind.size(); }
};

struct ColorSchedule {
    int nc = 0;
    const int* color_ptr = nullptr;
    const int* rows_of_color = nullptr;
    enum Mode { MC_NODE, ABMC_BLOCK } mode = MC_NODE;
    int nb = 0;
    const int* color_ptr_blk = nullptr;
    const int* blocks_of_color = nullptr;
    const int* block_ptr = nullptr;
    const int* rows_of_block = nullptr;
};

// Error carrying an iccg.h status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---- formats ----
CRS read_matrix_market_crs(const std::string& path);
void write_matrix_market(const std::string& path, const CRS& A, bool symmetric_lower);
std::vector<int> read_assignment_1based(int kind, const std::string& path, int n_expected,
                                        int& k_out);
void write_assignment_1based(const std::string& path, const int* v0, int n, int k);

// ---- orderings / schedules ----
std::vector<int> build_permutation_by_color(const std::vector<int>& color);
std::vector<int> build_permutation_by_block_color(const std::vector<int>& block_of_old,
                                                  const std::vector<int>& block_color);
CRS permute_ptap_lower(const CRS& A, const std::vector<int>& new_of_old);
CRS expand_lower_to_full(const CRS& L);
void build_color_schedule(const std::vector<int>& color, int nc,
                          const std::vector<int>& new_of_old, std::vector<int>& color_ptr,
                          std::vector<int>& rows_of_color);
void build_abmc_schedule(const std::vector<int>& new_of_old, const std::vector<int>& block_of_old,
                         const std::vector<int>& block_color, int nb, int nc,
                         std::vector<int>& color_ptr_blk, std::vector<int>& blocks_of_color,
                         std::vector<int>& block_ptr, std::vector<int>& rows_of_block);

// ---- generators ----
CRS gen_stencil(int kind, int nx, int ny, int nz, double wx, double wy, double wz);
CRS gen_diffusion27(int nx, int ny, int nz, double contrast, uint64_t seed);
CRS gen_knn_laplacian(int npts, int k, double diag_shift, uint64_t seed);
void gen_uniform(int n, uint64_t seed, double* out);
int color_greedy(int n, const int* rowptr, const int* colind, int* color);
int block_partition(int n, const int* rowptr, const int* colind, int B, int method,
                    int* block_of_old);
int color_blocks(int n, const int* rowptr, const int* colind, const int* block_of_old, int nb,
                 int* block_color);

// splitmix64 step
inline uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double u01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * 0x1.0p-53; }

}  // namespace iccg
