// Host-side launch entry points shared between the .cu files of libavbd6.
#pragma once
#include "common.cuh"

namespace avbd {

// Kernels enqueued by the launch functions on this thread (for the
// per-substep launch count reported in the stats).
extern thread_local long long g_kernel_launches;

void scan_launch(const Dev& d, const int* in, int* out, int n_cap, const int* n_dev, int* total_out,
                 cudaStream_t st);
void radix_sort_launch(Dev& d, cudaStream_t st);
void launch_collision(Dev& d, const AvbdParams& P, const AvbdDims& dims, int grid, cudaStream_t st, bool rebuild = true);

// Solve: coloring + predict + prelude + iterations + cache refresh.
// persistent = one cooperative launch; otherwise one launch per phase.
cudaError_t launch_solve(Dev& d, const AvbdParams& P, int persistent, int grid, int block, cudaStream_t st,
                         int variant);
// Resident CTAs per SM of the persistent kernel built for `variant` (2 or 3)
// CTAs per SM.
int solve_occupancy(int block, int variant);
void launch_reset(Dev& d, cudaStream_t st);
int count_conflicts(Dev& d, cudaStream_t st);
void launch_hash_scrub(Dev& d, cudaStream_t st);
void launch_cache_load(Dev& d, int n, const int* abc, const unsigned long long* keys, const float* st,
                       cudaStream_t s);

}  // namespace avbd
