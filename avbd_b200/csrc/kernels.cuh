// Host-side launch entry points shared between the .cu files of libavbd6.
#pragma once
#include "common.cuh"

namespace avbd {

// Kernels enqueued by the launch functions on this thread (for the
// per-substep launch count reported in the stats).
extern thread_local long long g_kernel_launches;

// Stage timing of one collision pipeline (avbd_profile_next_substep): while
// a timer is installed on this thread, the launch functions record an event
// after each stage (captured into a one-off graph, so no host launch gaps
// sit between the stages).
struct StageTimer {
  static const int kMax = 48;
  cudaEvent_t ev[kMax];
  const char* name[kMax];
  int n;
};
extern thread_local StageTimer* g_stage_timer;
inline void stage_mark(cudaStream_t st, const char* name) {
  StageTimer* t = g_stage_timer;
  if (t && t->n < StageTimer::kMax) {
    // an event-record node when the pipeline is being captured
    cudaEventRecordWithFlags(t->ev[t->n], st, cudaEventRecordExternal);
    t->name[t->n] = name;
    t->n++;
  }
}

void scan_launch(const Dev& d, const int* in, int* out, int n_cap, const int* n_dev, int* total_out,
                 cudaStream_t st);
void radix_sort_launch(Dev& d, cudaStream_t st);
void launch_collision(Dev& d, const AvbdParams& P, const AvbdDims& dims, int grid, cudaStream_t st, bool rebuild = true);

// Solve: coloring + predict + prelude + iterations + cache refresh.
// persistent = one cooperative launch; otherwise one launch per phase.
// With the flag-ordered sweep (P.flag_sweep) the persistent path is three
// cooperative launches: head, the sweep (k_flag_sweep, `sweep_grid` CTAs),
// tail.
cudaError_t launch_solve(Dev& d, const AvbdParams& P, int persistent, int grid, int block, cudaStream_t st,
                         int variant, int sweep_grid, int sweep_minb);
// CTAs of the standalone flag-sweep kernel for `group_size` lanes per body
// (batched: the batched-scene instantiation) built for `blocks_per_sm` (2 or
// 3) CTAs per SM that fit on the GPU at once.
int sweep_grid_size(int group_size, bool batched, int num_sms, int blocks_per_sm);
// Resident CTAs per SM of the persistent kernel built for `variant` (2 or 3)
// CTAs per SM.
int solve_occupancy(int block, int variant);
void launch_reset(Dev& d, cudaStream_t st);
// Scene build: the 8 corner groups of each floor block at its group offset
// (scene.cu).
cudaError_t launch_floor_groups(const Dev& d, int nblk, const int* blk_body, const float4* blk_he_fy,
                                const float4* blk_mat, const int* blk_row0, const int* blk_per, const int* blk_goff,
                                cudaStream_t st);
int count_conflicts(Dev& d, cudaStream_t st);
void launch_hash_scrub(Dev& d, cudaStream_t st);
void launch_cache_load(Dev& d, int n, const int* abc, const unsigned long long* keys, const float* st,
                       cudaStream_t s);

}  // namespace avbd
