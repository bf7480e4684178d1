/*
 * avbd6.h -- C ABI of libavbd6.so, the B200 (sm_100a) implementation of the
 * Solver6DOF substep of nanli9/AVBD (package avbd3d).
 *
 * The reference drives its substep from Python through Warp launches
 * (src/avbd3d/solver_6dof.py:1178-1464, kernels in src/avbd3d/kernels_6dof.py).
 * This library replaces that whole launch sequence.  Conventions:
 *
 *  - Memory: the caller owns every device buffer.  The library describes one
 *    device arena (avbd_layout: byte offset of each array); the caller
 *    allocates it (PyTorch in the shipped host code), fills the scene arrays
 *    and passes the base pointer to avbd_create.  The library allocates only
 *    its context and CUDA graph objects.  An arena must not be freed or moved
 *    while a context uses it.
 *  - Errors: every call returns 0 or a negative AVBD_E_* code; the device
 *    status bits (AVBD_ERR_*) are reported through avbd_read_stats.
 *  - Streams: `stream` is a cudaStream_t passed as void*; calls enqueue work
 *    asynchronously except avbd_read_stats (synchronises the stream).
 *  - Threads: one context per host thread at a time.
 */
#ifndef AVBD6_H
#define AVBD6_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AVBD_OK 0
#define AVBD_E_INVALID -1    /* bad argument or size */
#define AVBD_E_CUDA -2       /* a CUDA call failed */
#define AVBD_E_TIMEOUT -3    /* a bounded device wait ran out */
#define AVBD_E_OVERFLOW -4   /* a pool overflowed (contacts dropped) */

/* Device status bits (AvbdStats.err). */
#define AVBD_ERR_BARRIER_TIMEOUT 1
#define AVBD_ERR_HASH_FULL 2
#define AVBD_ERR_PAIR_OVERFLOW 4
#define AVBD_ERR_ROW_OVERFLOW 8
#define AVBD_ERR_NONFINITE 16
#define AVBD_ERR_NBR_OVERFLOW 32
#define AVBD_ERR_BVH 64

/* Sizes that fix the arena layout.  Mirrors the capacities the reference
 * sizes in Solver6DOF._flush (solver_6dof.py:937-943, 1150-1163). */
typedef struct AvbdDims {
  int n_bodies;
  int n_static_groups; /* floor corners, pins: fixed at scene build */
  int n_static_rows;   /* rows of those groups (reference row numbering) */
  int pair_cap;        /* broadphase pairs i<j (reference _bp_max_pairs) */
  int dyn_row_cap;     /* dynamic contact rows (reference n_dyn_capacity) */
  int dyn_group_cap;   /* dynamic contact groups (<= dyn_row_cap) */
  int hash_cap;        /* contact-cache slots, power of two */
  int mlp_floats;      /* learned warm-start weights: 0 or AVBD_MLP_FLOATS */
  int new_cap;         /* new contacts queued per substep for the learned
                          warm start / training log (0 = none) */
  int n_scenes;        /* batched independent scenes (0 = one scene).  With
                          n > 0 the arena's SCENE_OF gives each body's scene
                          and SCENE_TAB per scene (substep dt, iterations,
                          substeps per frame, 0) as float4; bodies of
                          different scenes never collide.  AvbdParams then
                          gives the maximum iterations and substeps. */
  int anchor_keys;     /* contact-cache key: 0 = (a, b, manifold ordinal) as
                          the reference's live cache; 1 = (a, b, contact point
                          in a's frame at 5 mm) as its documented cache */
} AvbdDims;

/* Scalars of Solver6DOF.__init__ (solver_6dof.py:180-201). */
typedef struct AvbdParams {
  float dt; /* frame dt; a substep uses dt / substeps */
  int iterations;     /* 0..256 (AVBD_MAX_VIOL_ITERS) */
  float gravity[3];
  float alpha, beta, gamma;
  int post_stabilize;
  float max_linear_speed, max_angular_speed;
  int substeps;
  float friction_static_mult;
  int coloring_mode;         /* 0 = jacobi (speculative), 1 = jones_plassmann */
  int recolor_every_substep; /* 1 = recolor every substep, 0 = on conflict */
  int self_collide;
  float self_friction;
  int group_size;      /* lanes per body in the primal: 1,2,4,8,16,32 */
  int use_graph;       /* capture one substep as a CUDA graph and replay it */
  int persistent;      /* 1 = one cooperative kernel per substep solve */
  int record_violation;/* store the max constraint violation per iteration */
  int mlp_warm_start;  /* 1 = learned warm start for new contacts */
  int debug_skip_arrive; /* test hook: block 0 skips one barrier arrival */
  int blocks_per_sm;   /* persistent grid: CTAs per SM, 2 or 3, each with its
                          own register budget (128 / 80 registers); 0 = 2 */
  int timing;          /* stamp the persistent kernel's phase boundaries */
  int log_new_contacts;/* queue the features of every new contact (training) */
  int flag_sweep;      /* persistent solve: order the color passes by per-body
                          completion flags (each body waits only for its own
                          neighbours) instead of a grid barrier per color */
  int bvh_rebuild_every; /* collision: rebuild the LBVH every this many
                          substeps and refit it in between (the pair list
                          is the same either way); 0 or 1 = every substep */
  int adaptive_lanes;  /* barrier sweep: a color whose bodies, at twice the
                          lanes per body, still fit in one round of the
                          resident warps gets twice the lanes (repeatedly,
                          up to 32); group_size is then the lane count of
                          the large colors */
  int resting_floor;   /* barrier sweep (flag_sweep = 0): 1 = a floor corner
                          that rests above the floor in its substep-start
                          state (no force, multipliers 0, minimum penalties)
                          is evaluated from the body's pose alone, without
                          reading or writing its group: the same sums and
                          poses as reading it (the stored tangent multipliers
                          may differ in the sign of zero); 0 = every group is
                          read.  The flag sweep always reads. */
} AvbdParams;

/* Iterations whose max violation a substep records (record_violation). */
#define AVBD_MAX_VIOL_ITERS 256

typedef struct AvbdStats {
  int n_pairs_found, n_pairs, n_dyn_groups, n_dyn_rows, n_dyn_rows_req;
  int n_contacts_req, n_colors, recolored, conflicts, err, err_where;
  int n_cache_hits, n_new_contacts, max_dg, n_viol;
  unsigned epoch;
  int graph_state;  /* bit 0: collision graph live, bit 1: solve graph live,
                       bit 2: the last avbd_step ran as one whole-frame graph
                       (all substeps, collision and solve; bits 0-1 set too) */
  int capture_err;  /* 1000 * collision capture error + solve capture error */
  long long kernels_launched; /* kernels enqueued by this context so far */
  float viol[AVBD_MAX_VIOL_ITERS];
  int n_new_logged;   /* new contacts queued last substep (may exceed new_cap) */
  int n_mlp_applied;  /* of those, warm-started by the MLP */
  int n_mlp_fallback; /* of those, kept at the zero start (separated, non-finite,
                         outside the static friction cone) */
  int n_mlp_reverted; /* learned starts reset to the zero start at their first
                         dual update because the contact separated (the
                         predicted force raised the complementarity residual) */
  float viol_contact[AVBD_MAX_VIOL_ITERS]; /* per-iteration max violation over box-box contacts */
} AvbdStats;

typedef struct AvbdCtx AvbdCtx;

/* Arena layout.  `offsets` receives avbd_num_arrays() byte offsets. */
int avbd_num_arrays(void);
const char* avbd_array_name(int id);
int avbd_layout(const AvbdDims* dims, size_t* offsets, size_t* total_bytes);

/* Replaces Solver6DOF._flush's device allocation (solver_6dof.py:904-1174):
 * binds a filled arena.  */
int avbd_create(const AvbdDims* dims, void* arena, size_t arena_bytes, AvbdCtx** out);
int avbd_destroy(AvbdCtx* ctx);

/* Scalars; no recapture is needed when they change (they live on device). */
int avbd_set_params(AvbdCtx* ctx, const AvbdParams* p, void* stream);

/* Marks every body uncolored, empties the contact cache and zeroes counters
 * (the fresh-flush state of solver_6dof.py:1010-1035, 1150-1156). */
int avbd_reset_state(AvbdCtx* ctx, void* stream);

/* Forces a recolor on the next substep (solver_6dof.py:605-624 sets
 * _color_dirty when the coloring mode changes). */
int avbd_mark_color_dirty(AvbdCtx* ctx, void* stream);

/* One substep of `dt` (replaces _step_one, solver_6dof.py:1232-1464). */
int avbd_substep(AvbdCtx* ctx, float dt, void* stream);

/* One frame: params.substeps substeps of dt/substeps (Solver6DOF.step,
 * solver_6dof.py:1178-1197). */
int avbd_step(AvbdCtx* ctx, void* stream);

/* Device counters of the last substep; synchronises `stream`. */
int avbd_read_stats(AvbdCtx* ctx, AvbdStats* out, void* stream);

/* Diagnostic: active two-body contact pairs whose bodies share a color
 * (count_color_conflicts, solver_6dof.py:846-862).  Synchronises. */
int avbd_count_color_conflicts(AvbdCtx* ctx, void* stream);

/* Replaces the contact cache with n entries: abc = n x (a, b, ordinal)
 * int32 and state = n x 8 floats (lambda n/t/b, penalty n/t/b, was_static
 * t/b), both device pointers; the next substep's emission looks them up.
 * The reference keeps this state in hash_keys/hash_state
 * (solver_6dof.py:1150-1156, kernels_6dof.py:2923-2995). */
int avbd_cache_load(AvbdCtx* ctx, int n, const int* abc, const float* state, void* stream);

/* The same with the cache's raw 50-bit keys (bits 50-63 ignored): the only
 * form for an anchor-keyed cache (AvbdDims.anchor_keys = 1), any cache's keys
 * as read back from the arena's H_KEY. */
int avbd_cache_load_keys(AvbdCtx* ctx, int n, const unsigned long long* keys, const float* state, void* stream);

/* Clears the sticky device error bits. */
int avbd_clear_errors(AvbdCtx* ctx, void* stream);

/* Device time of the last substep's collision and solve parts, in ms
 * (replaces broadphase_ms, solver_6dof.py:1786-1787, 1916).  Synchronises. */
int avbd_step_ms(AvbdCtx* ctx, float* collide_ms, float* solve_ms);

/* Phase timestamps of the last substep's solve (params.timing = 1): up to
 * `cap` (globaltimer ns, phase id) pairs; returns the count.  Synchronises. */
int avbd_read_phase_marks(AvbdCtx* ctx, long long* t_ns, int* phase, int cap, void* stream);

/* Scene build on the device (replaces the per-row loops of _flush,
 * solver_6dof.py:1067-1129, for the rows of add_floor_contact_box,
 * :474-541): writes the 8 corner groups of each of `nblk` floor blocks
 * into the static group arrays of the arena.  Per block (device arrays):
 * body; half extents and floor height (float4); mu, mu_s, stiffness
 * (float4, 4th unused); first row number; rows per corner (3 with
 * friction, else 1); first group index (blocks and explicit groups sorted
 * by body, then first row).  Call after avbd_create, with the bodies' half
 * extents (BHE) already in the arena. */
int avbd_build_floor_groups(AvbdCtx* ctx, int nblk, const int* blk_body, const float* blk_he_fy,
                            const float* blk_mat, const int* blk_row0, const int* blk_per, const int* blk_goff,
                            void* stream);

/* Collision stage profile (no counterpart in the reference; it serves the
 * per-kernel bandwidth report of the benchmark).  After
 * avbd_profile_next_substep, the next substep runs its collision pipeline
 * as a one-off CUDA graph with an event-record node after each stage (and
 * synchronises); avbd_collision_profile then writes up to `cap` stage
 * durations in ms and returns their count;
 * avbd_collision_stage names stage i ("k_aabb", "radix_sort", "k_bp_count",
 * ..., a scan stage covers its three launches). */
int avbd_profile_next_substep(AvbdCtx* ctx);
int avbd_collision_profile(AvbdCtx* ctx, float* ms, int cap);
const char* avbd_collision_stage(AvbdCtx* ctx, int i);

/* Exclusive prefix sum of n int32 (out[0..n], out[n] = total) that allocates
 * no device memory.  No counterpart in the reference: it serves callers that
 * cannot call cudaMalloc (a host that owns the device-memory budget, a
 * real-time loop).  Its scratch is a fixed 16 KiB device array of this
 * library, so n is limited to 8,388,607 (larger n returns AVBD_E_INVALID).
 * The first call on a device looks the array up (cudaGetSymbolAddress); make
 * that first call before any stream capture.  All calls on a device share the
 * array: calls that overlap on the GPU race, so serialise them.  The looked-up
 * address is kept for the process: do not call this after cudaDeviceReset.
 * `in` and `out` are device pointers; asynchronous on `stream`. */
int avbd_exclusive_scan_noalloc(const int* in, int* out, int n, void* stream);

/* ---------------------------------------------------------------------
 * Learned warm start.  No counterpart in the reference: it replaces the
 * cache-miss defaults of gpu_pool_emit_rows (kernels_6dof.py:2864-2879:
 * lambda 0, penalties (1e6, 1, 1)) with a prediction, which the prelude
 * (kernels_6dof.py:1596-1609) then treats like a cached value.
 *
 * Network: 20 features -> 64 -> 64 -> 4, SiLU, FP32 master weights.
 * Features of a new contact (reference body a, incident body b):
 *   0-2  contact normal in a's body frame     3  penetration depth (m)
 *   4-6  relative contact-point velocity (a - b) along (t, b, n)
 *   7-8  inverse masses of a, b               9-10  n^T I^-1 n of a, b
 *   11   static friction mu_s                 12  dynamic friction mu
 *   13-19  one-hot SAT axis class of the pair (A = the lower body index):
 *          face of A (x, y, z), face of B (x, y, z), edge-edge.
 * Outputs (targets, before the stored normalisation):
 *   y0 = log1p(-lambda_n), y1 = lambda_t1 / (|lambda_n| + 1),
 *   y2 = lambda_t2 / (|lambda_n| + 1), y3 = log(k_n).
 *
 * AVBD_MLP_PARAMS master parameters, in order: W1[64][20], b1[64],
 * W2[64][64], b2[64], W3[4][64], b3[4] (row-major, out x in).
 * AVBD_MLP_FLOATS packed inference block (floats; bf16 pairs in uint32):
 *   [0,32) feature mean  [32,64) 1/feature std  [64,68) target mean
 *   [68] lambda scale zeta (the decoded forces are multiplied by it)
 *   [72,80) target std  [80,144) b1  [144,208) b2  [208,216) b3
 *   [216,1240) W1 bf16 [64][32]  [1240,3288) W2 bf16 [64][64]
 *   [3288,3544) W3 bf16 [8][64]  (zero padded).
 */
#define AVBD_MLP_IN 20
#define AVBD_MLP_OUT 4
#define AVBD_MLP_PARAMS 5764
#define AVBD_MLP_FLOATS 3544

/* Builds the packed inference block from master parameters `theta` and the
 * normalisation `norm` (feature mean[20], feature std[20], target mean[4],
 * target std[4], lambda scale zeta[1]: 49 floats).  Device pointers. */
int avbd_mlp_pack(const float* theta, const float* norm, float* packed, void* stream);

/* BF16 tensor-core forward (the solver's path) of n raw feature rows:
 * out = n x 4 targets (denormalised).  Device pointers. */
int avbd_mlp_infer(const float* packed, const float* feat, int n, float* out, void* stream);

/* Bytes of scratch avbd_mlp_loss_grad needs for n samples. */
size_t avbd_mlp_scratch_bytes(int n);

/* FP32 loss and gradient over n normalised samples x (n x 20) with targets
 * y (n x 4): loss = mean over samples of the summed squared error of the 4
 * outputs; grad has AVBD_MLP_PARAMS floats.  Deterministic (fixed reduction
 * order).  Device pointers; `loss` receives one float. */
int avbd_mlp_loss_grad(const float* theta, const float* x, const float* y, int n, float* grad, float* loss,
                       void* scratch, size_t scratch_bytes, void* stream);

/* One Adam step (bias-corrected, step number t >= 1) on AVBD_MLP_PARAMS
 * parameters with moment buffers m, v. */
int avbd_mlp_adam(float* theta, const float* grad, float* m, float* v, int t, float lr, float beta1, float beta2,
                  float eps, void* stream);

/* Last error text of this thread. */
const char* avbd_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* AVBD6_H */
