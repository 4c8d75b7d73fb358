// ensemble.cuh — one persistent launch that advances a batched ensemble of small grids.
//
// The launch advances every member of a dns2d_batch by K steps.  Its CTAs (all co-resident:
// a cooperative launch of at most as many CTAs as fit on the GPU at once) take numbered work
// items from one global ticket counter:
//   step s:  all row items (ROWS physical rows of one member; the row pass of k_rows_step),
//            then all column items (CG columns of one member; the column pass of k_cols_step),
//   step s+1, ...
// A column item of member m at step s needs every row item of (m, s); a row item of (m, s)
// needs every column item of (m, s - 1).  Both are counted per member (rows_done, cols_done,
// cumulative over the launch).  Every dependency of an item has a smaller number, and every
// smaller number is held by a running CTA or finished, so the waits always end; members of
// different sizes and speeds interleave with no kernel boundary between passes.  A wait polls
// its counter at most spin_limit times and then records a time-out in *status and returns; the
// other CTAs see the status and stop (no trap, the context stays usable).
//
// The per-mode arithmetic and every butterfly are those of k_rows_step / k_cols_step on the
// size's default radix plan, so a member's field equals the one the standalone kernels give on
// that plan, bit for bit;
// the FP64 energy/enstrophy partials are summed per item instead of per column (same values to
// rounding).  Global loads of data that another CTA of the launch wrote (U, W, D, E, om2,
// fnm1) go through L2 only: an SM can hold stale L1 lines of those addresses from an earlier
// item.
#pragma once
#include "dns2d_kernels.cuh"

namespace dns2d {

constexpr int kEnsThreads = 384;   // threads per CTA (the N = 512 row pass width)
constexpr int kEnsMaxGroups = 8;   // size groups per launch
constexpr int kEnsRows = 4;        // physical rows per row item

// columns per column item: the largest divisor of H with CG * NTA <= kEnsThreads
template <int N>
constexpr int ens_cols_per_item()
{
    int cg = kEnsThreads / Cfg<N>::NTA;
    while (cg > 1 && (Cfg<N>::H % cg) != 0) --cg;
    return cg < 1 ? 1 : cg;
}

template <int N>
constexpr size_t ens_smem_bytes()
{
    constexpr size_t r = (size_t)kEnsRows * Cfg<N>::LP, c = (size_t)2 * ens_cols_per_item<N>() * Cfg<N>::LP;
    return (r > c ? r : c) * sizeof(float2);
}

// the sizes a persistent launch serves (the single-CTA generic sizes of the ensemble configs)
__host__ __device__ constexpr bool ens_supported(int N)
{
    return N == 64 || N == 128 || N == 256 || N == 512;
}

struct EnsGroupDev {
    int N = 0, count = 0;
    int member0 = 0;                 // index of the group's member 0 in the counters
    int row_items = 0, col_items = 0;  // per member and step
    int tiles_per_item = 1;          // row tiles (kEnsRows rows each) per row item
    int groups_per_item = 1;         // column groups (ens_cols_per_item columns each) per column item
    int row_begin = 0, col_begin = 0;  // first item of this group in a step's row / column block
    Pointers p;                      // group pointers, member strides set
};

struct EnsLaunch {
    EnsGroupDev g[kEnsMaxGroups];
    int ngroups = 0, steps = 0, first = 0;
    int rows_per_step = 0, cols_per_step = 0;
    unsigned int *ticket = nullptr, *rows_done = nullptr, *cols_done = nullptr;
    int *status = nullptr;       // 0: running / done; 1: a wait ran out
    long long spin_limit = 0;    // polls of a counter before a wait gives up
    int stall_member = -1;       // >= 0: that member's column items wait for a count never reached
};

// host side (ensemble.cu): occupancy-sized cooperative launch; returns the CUDA error
cudaError_t ens_launch(const EnsLaunch &q, cudaStream_t stream, int *grid_out);

}  // namespace dns2d
