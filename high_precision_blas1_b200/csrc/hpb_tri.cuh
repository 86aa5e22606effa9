// Sparse triangular solves and the ILU(0) factorization on CSR matrices.
//
// Replaces csr::gpu_matrix::triangular_solve_lower / triangular_solve_upper
// (common/csr/gpu_matrix.h:142-311: cuSPARSE csrsv2 with a per-call
// analysis and cudaMalloc'd buffer) and gives csr::preconditioner
// (common/csr/preconditioner.h:32-85) and csr::gpu_ilu0_preconditioner
// (common/csr/gpu_ilu0_preconditioner.h:32-80) their factors.
//
// An analysis (hpb_csr_tri) is made once per sparsity pattern and triangle:
// rows are cut into tiles of kTriTile consecutive rows; inside a tile each
// row gets its level (longest chain of in-tile dependencies), and the tile's
// rows are stored in level order as packed descriptors.  A solve is one
// kernel: each block takes the next tile by ticket (ascending for a lower,
// descending for an upper triangle), keeps the tile's solution in shared
// memory, and its warps take the tile's levels round-robin, so a warp loads
// the rows of its next level while earlier levels finish.  Dependencies on
// other tiles are read from x itself (x is pre-filled with a signalling-NaN
// sentinel), by a receiver warp per block that streams them into shared
// memory ahead of need; the factorization, whose rows are read as a whole,
// uses per-row flags (release/acquire at GPU scope).  Every wait has a time
// limit after which the kernel records a timeout and carries on, so a
// launch always ends.
#pragma once

#include "hpb_common.cuh"

namespace hpb {
namespace tri {

constexpr int kTriTile = 8192;      // rows per tile
constexpr int kTriThreads = 512;    // threads per solve block (16 warps)

// Error bits of Plan::err (device).
constexpr int kErrUnsorted = 1;     // column indices of a row not strictly increasing
constexpr int kErrColumn = 2;       // column index outside [0, rows)
constexpr int kErrTimeout = 4;      // a bounded wait gave up
constexpr int kErrZeroPivot = 8;    // ILU(0): zero pivot

struct Plan {
    int device = 0;
    int upper = 0;                  // 0: strictly lower part, 1: strictly upper part
    int all_diag = 0;               // every row stores its diagonal
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t ntiles = 0;
    int32_t max_levels = 0;         // largest level count of a tile
    int64_t sum_levels = 0;         // levels summed over tiles
    const int32_t* rp = nullptr;    // caller's structure; must stay valid and unchanged
    const int32_t* ci = nullptr;
    int4* desc = nullptr;           // n: (row, first dependency, dependency count, diagonal position) in level order
    int4* dcol = nullptr;           // n: columns of the first four dependencies (-1: none), in level order
    int4* dslot = nullptr;          // n: halo slot of each of those that lies in another tile (-1: none)
    int32_t* hoff = nullptr;        // ntiles + 1: first halo slot of each tile in hrow
    int32_t* hrow = nullptr;        // halo slots: the other-tile row each one is filled from
    int32_t* lvlptr = nullptr;      // ntiles * (kTriTile + 1): level starts within the tile
    int32_t* nlev = nullptr;        // ntiles
    int32_t* dpos = nullptr;        // n: position of the diagonal entry of each row, -1 if absent
    unsigned* flags = nullptr;      // n + 1: per-row done flags (factorization), then the tile ticket
    void* scratch = nullptr;        // n * 16 bytes, allocated on the first in-place solve
    int* err = nullptr;             // error bits
    int* err_row = nullptr;         // ILU(0): first row with a zero pivot
    unsigned long long wait_ns = 0; // solve: limit of each bounded wait (0: the default, 4 s)
    int32_t withhold_row = -1;      // solve, testing aid: this row's value is never published to x
};

int analyse(hpb_context* ctx, int upper, int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci, Plan* P);
void release(Plan* P);

// x := op^-1 (alpha b) for the plan's triangle; unit: the diagonal is taken
// as 1 (stored diagonal entries are ignored).  Stream-ordered, no host sync;
// b and x must not overlap.  Two graph-capturable launches (the sentinel
// fill of x, the solve).
template <class E>
cudaError_t launch_trsv(const Plan& P, int unit, const E* val, E alpha, const E* b, E* x, cudaStream_t s);

// Approximate x ~ T^-1 (alpha b) by Jacobi sweeps (x_0 = 0, then `sweeps`
// passes x_{k+1} = D^-1 (alpha b - (T - D) x_k)); tmp: n elements; b must
// not overlap x or tmp.  sweeps + 1 launches, graph-capturable.
template <class E>
cudaError_t launch_trsv_sweeps(const Plan& P, int unit, const E* val, E alpha, const E* b, E* x, E* tmp, int sweeps,
                               cudaStream_t s);

// ILU(0) in place on val (lower plan): val := L\U with L unit lower
// (strictly lower entries stored) and U upper (diagonal included).
template <class E>
cudaError_t launch_ilu0(const Plan& P, E* val, cudaStream_t s);

}  // namespace tri

// 1 in each element type (the alpha of a plain solve)
template <class E> inline E unit_of();
template <> inline float unit_of<float>() { return 1.0f; }
template <> inline double unit_of<double>() { return 1.0; }
template <> inline cf unit_of<cf>() { return cf{1.0f, 0.0f}; }
template <> inline cd unit_of<cd>() { return cd{1.0, 0.0}; }

}  // namespace hpb

// The C ABI handle is the plan.
struct hpb_csr_tri {
    hpb::tri::Plan plan;
};
