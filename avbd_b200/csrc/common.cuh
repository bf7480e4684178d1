// Shared device definitions for the B200 Solver6DOF substep.
//
// Data model:
//  * bodies are SoA float4 arrays (x.xyz + mass, q, v, w, ...);
//  * constraints are stored as *contact groups*: a normal row plus its two
//    friction rows (floor corner or box-box contact), a 1-row frictionless
//    contact, or the three axis rows of a pin.  A group's rows share bodies
//    and anchors, so the primal reads the geometry once for up to three rows.
//    The reference's row numbering (c_* arrays, solver_6dof.py:1067-1129) is
//    kept through g_row0, so row-indexed API results are unchanged.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/avbd6.h"

namespace avbd {

// Device-wide exclusive scan (collide.cu: k_scan_reduce / k_scan_parts /
// k_scan_down): SCAN_T threads per block, SCAN_V ints per thread, so one
// block covers SCAN_CHUNK ints and writes one block partial.
#define SCAN_T 256
#define SCAN_V 8
#define SCAN_CHUNK (SCAN_T * SCAN_V)

// Group kinds.  The row types they carry are those of solver_6dof.py:31-34.
enum : int { KIND_FLOOR = 0, KIND_PIN = 1, KIND_BOX = 2 };
// g_meta bit layout.
//   bits 0-1 kind, bit 2: three rows (else one), bit 3: hard (stiffness=inf),
//   bits 4-5 contact ordinal within the pair manifold (box groups).
__host__ __device__ inline int meta_kind(int m) { return m & 3; }
__host__ __device__ inline int meta_nrows(int m) { return (m & 4) ? 3 : 1; }
__host__ __device__ inline bool meta_hard(int m) { return (m & 8) != 0; }
__host__ __device__ inline int meta_cidx(int m) { return (m >> 4) & 3; }
__host__ __device__ inline int make_meta(int kind, int three, int hard, int cidx) {
  return kind | (three ? 4 : 0) | (hard ? 8 : 0) | (cidx << 4);
}
// Implicit floor corners (bit 9): the 8 corner groups of one floor block
// (solver_6dof.py:474-541) store no geometry.  The corner offset is the
// body's half extents with the signs of corner index c = bits 6-8 (x: bit 2,
// y: bit 1, z: bit 0; set = +, the reference's sx, sy, sz loop order), and
// g_mat.w, the fracture threshold of other groups (never reached by floor
// rows), holds the floor height.
#define META_IMPLICIT 512
__host__ __device__ inline bool meta_implicit(int m) { return (m & META_IMPLICIT) != 0; }
__device__ __forceinline__ float4 implicit_corner(float4 he, int meta, float floor_y) {
  int c = (meta >> 6) & 7;
  return make_float4((c & 4) ? he.x : -he.x, (c & 2) ? he.y : -he.y, (c & 1) ? he.z : -he.z, floor_y);
}
// g_flags bit layout: bits 0-2 row active, bit 3 normal row was_static,
// bits 4/5 the friction rows' own was_static (carried to the cache), bit 6:
// body_b owns the group (runs its dual update; else body_a), bit 7: a new
// contact whose prelude runs in the learned-warm-start phase, bit 8: its
// start came from the network (checked at its first dual update), bit 9:
// that start was reverted to the zero start.
enum : int {
  FL_ACT0 = 1, FL_ACT1 = 2, FL_ACT2 = 4, FL_WAS = 8, FL_WAST = 16, FL_WASB = 32, FL_OWNB = 64, FL_NEW = 128,
  FL_LRN = 256, FL_REV = 512
};

// Penalty constants: kernels_6dof.py:50-52.
#define PEN_MIN 1.0e6f
#define PEN_MIN_T 1.0f
#define PEN_MAX 1.0e9f
#define MAX_COLORS 32
#define JP_ROUNDS 24
#define COLL_MARGIN 0.005f
#define BP_SLOTS 32

// Learned warm start: layer widths and the packed inference block (floats;
// layout documented with AVBD_MLP_FLOATS in avbd6.h).
#define MLP_IN AVBD_MLP_IN
#define MLP_H 64
#define MLP_OUT AVBD_MLP_OUT
#define MLPO_FMEAN 0
#define MLPO_FISTD 32
#define MLPO_OMEAN 64
#define MLPO_OSTD 72
#define MLPO_B1 80
#define MLPO_B2 144
#define MLPO_B3 208
#define MLPO_W1 216   // bf16 [64][32] as 1024 bf16 pairs
#define MLPO_W2 1240  // bf16 [64][64] as 2048 pairs
#define MLPO_W3 3288  // bf16 [8][64] as 256 pairs
static_assert(MLPO_W3 + 256 == AVBD_MLP_FLOATS, "packed MLP block size");

// Error bits of the device status word.
enum : int {
  ERR_BARRIER_TIMEOUT = 1,
  ERR_HASH_FULL = 2,
  ERR_PAIR_OVERFLOW = 4,
  ERR_ROW_OVERFLOW = 8,
  ERR_NONFINITE = 16,
  ERR_NBR_OVERFLOW = 32,
  ERR_BVH = 64,
};

// Counters written on the device, read by the host once per frame.
struct DevCounters {
  int n_pairs_found;     // canonical (i<j) broadphase pairs found this substep
  int n_nbr_found;       // directed neighbour entries found (2 * pairs)
  int n_pairs;           // pairs kept (<= pair_cap)
  int n_dyn_groups;      // dynamic contact groups kept
  int n_dyn_rows;        // dynamic rows kept
  int n_dyn_rows_req;    // dynamic rows requested (may exceed capacity)
  int n_contacts_req;    // contacts found by the manifold
  int n_colors;          // active colors
  int recolored;         // 1 if the last substep recolored
  int conflicts;         // same-color edges seen by the recolor gate
  int uncolored;         // scratch for the coloring convergence test
  int color_dirty;       // host request: force a recolor on the next substep
  int err;               // error bits (ERR_*)
  int err_where;         // barrier index of a timeout
  unsigned epoch;        // contact-cache epoch (substeps since the last clear)
  int n_cache_hits;      // warm-start cache hits in the last emission
  int n_new_contacts;    // cache misses in the last emission
  int max_dg;            // longest per-body dynamic incidence list
  unsigned viol_bits[AVBD_MAX_VIOL_ITERS];  // per-iteration max violation (float bits, >= 0)
  int n_viol;
  int n_marks;           // phase timestamps recorded (timing mode)
  int n_new_logged;      // new contacts queued for the learned warm start / log
  int n_mlp_applied;     // new contacts that took the learned warm start
  int n_mlp_fallback;    // new contacts that fell back to the zero start
  int n_mlp_reverted;    // learned starts reverted at their first dual (residual rose)
  int slot;              // substep slot within the frame (batched scenes)
  int slot_next;         // slot of the next substep (reset by the host at frame start)
  int pad[8];
  unsigned long long mark_t[256];  // globaltimer after each grid barrier
  int mark_id[256];                // phase id of that barrier (PH_*)
  // grid barrier state (each counter on its own 128-byte line): blocks
  // arrive on one of BAR_SUB sub-counters; the last of each sub-group
  // arrives on the top counter; the last of those bumps the generation.
  unsigned bar_count;
  unsigned pad2[31];
  unsigned bar_gen;
  unsigned pad3[31];
  unsigned bar_sub[16][32];
  int round_unc[2];  // uncolored counts of alternate coloring rounds
  int work_ctr[4];   // color passes: next chunk to hand out (pass q uses q & 3)
  int pad4[26];
  unsigned vc_max_bits[AVBD_MAX_VIOL_ITERS];  // per-iteration max violation over box-box contact groups (float bits)
  int vc_cnt[AVBD_MAX_VIOL_ITERS];            // and their count (record_violation)
};
#define BAR_SUB 16

// Scalars read by the kernels from device memory, so a captured graph sees
// parameter changes without being re-captured.
struct DevParams {
  float dt;  // substep dt
  int iterations;
  float gx, gy, gz;
  float alpha, beta, gamma;
  int post_stab;
  float max_lin, max_ang;  // +inf when the cap is off
  float fsm;
  int color_mode;  // 0 jacobi, 1 jones-plassmann
  int recolor_every;
  float self_friction;
  int group_size;
  int record_violation;
  int debug_skip_arrive;
  int mlp_on;
  unsigned long long barrier_timeout_ns;
  int timing;   // record phase timestamps in the counters
  int log_new;  // queue every new contact's features (training-data log)
  int batched;  // bodies belong to scenes with their own dt / iterations / substeps
  int flag_sweep;  // color passes ordered by per-body completion flags instead of grid barriers
  int adaptive_lanes;  // small colors get more lanes per body (barrier sweep)
  int resting_floor;   // resting floor corners evaluated from the pose alone (fsep)
  int pad[2];
};

// Phase ids of the persistent kernel's timestamps.
enum : int {
  PH_START = 0, PH_GATE_PRELUDE, PH_COLOR_RESET, PH_ROUND, PH_BUCKET, PH_PREDICT, PH_PRIMAL, PH_DUAL, PH_COLLECT,
  PH_COUNT
};

// Every device pointer and size one substep needs.  Passed by value.
struct Dev {
  const DevParams* prm;
  // sizes
  int nb, n_sg, n_static_rows, g_cap, row_cap, pair_cap, nbr_cap, hash_cap;
  int n_sg_rows_unused;
  // bodies
  float4 *x, *q, *v, *w, *pv, *pw, *x0, *q0, *xin, *qin, *iw0, *iw1, *iloc, *he;
  float* prio;
  int *color, *color2, *color_starts, *color_bodies;
  int *sg_start;
  int *dg_start, *dg_cnt, *dg_idx;
  int* dg_other;  // beside dg_idx: 2 * other body + (this body is the group's second body)
  // groups
  int2* g_body;
  int *g_meta, *g_row0, *g_flags;
  float4 *g_offa, *g_offb, *g_n, *g_mat, *g_lam, *g_pen, *g_ac0;
  // broad phase
  float4 *aabb_lo, *aabb_hi;
  unsigned *morton, *morton2;
  int *order, *order2;
  float4 *node_lo, *node_hi;
  int *node_left, *node_right, *node_parent, *node_flag;
  float4* node_rec;  // per internal node: its grandchildren's (or leaf children's) boxes (traversal copy)
  float* bounds;  // 6 floats (lo xyz, hi xyz) as ordered ints
  int *nbr_cnt, *nbr_start, *nbr_idx, *nbr_pair;
  int *up_cnt, *pair_start;
  int* bp_tmp;  // BP_SLOTS upper neighbours per body from the traversal
  int2* pair_ab;
  int* pair_info;     // overlap | sat_idx<<1 | count<<6 | ref_is_a<<9
  float4* pair_nrm;   // manifold normal (inc -> ref), w = SAT depth
  float4* pair_off;   // 8 per pair: off_ref[4], off_inc[4]
  int *pair_gcnt, *pair_gstart, *pair_rstart, *pair_kept;
  // contact cache
  unsigned long long* h_key;
  float4 *h_s0, *h_s1;
  // scan scratch
  int* scan_part;
  int scan_part_cap;
  // radix sort scratch
  int* sort_hist;
  // coloring scratch
  int *c_used, *c_lost, *c_hist;
  // learned warm start (optional): packed weights, null when disabled
  const float* mlp_w;
  int new_cap;      // capacity of the new-contact queue
  int* new_list;    // group id of each queued new contact
  float* mlp_feat;  // MLP_IN raw features of each queued new contact
  // batched scenes (null when the arena holds one scene)
  int n_scenes;
  const int* scene_of;       // scene of each body
  const float4* scene_tab;   // per scene: (substep dt, iterations, substeps per frame, 0)
  // flag-ordered sweep: passes each body has completed in this substep
  int* done;
  // per body, the floor height when its first eight static groups are its
  // floor corners in the resting start state (implicit corners 0-7, all rows
  // active, no force, minimum penalties, no alpha offset), else NaN; set by
  // predict, cleared by the sweep once a corner's state changes
  float* fsep;
  // anchor-keyed cache (null: keys are (a, b, ordinal))
  unsigned long long* g_key;
  // counters
  DevCounters* ctr;
};

// ---------------------------------------------------------------------------
// Small vector / quaternion math (float).  Quaternions are XYZW.
// ---------------------------------------------------------------------------
struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 mk(float a, float b, float c) { return V3{a, b, c}; }
__host__ __device__ __forceinline__ V3 xyz(float4 a) { return V3{a.x, a.y, a.z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Hamilton product.
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
  return make_float4(a.w * b.x + b.w * a.x + (a.y * b.z - a.z * b.y), a.w * b.y + b.w * a.y + (a.z * b.x - a.x * b.z),
                     a.w * b.z + b.w * a.z + (a.x * b.y - a.y * b.x), a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z));
}
__device__ __forceinline__ float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
// v' = (2w^2-1) v + 2 (q.v) q + 2 w (q x v)
__device__ __forceinline__ V3 qrot(float4 q, V3 v) {
  float c = 2.0f * q.w * q.w - 1.0f;
  float d = 2.0f * (q.x * v.x + q.y * v.y + q.z * v.z);
  float w2 = q.w * 2.0f;
  return V3{v.x * c + q.x * d + (q.y * v.z - q.z * v.y) * w2, v.y * c + q.y * d + (q.z * v.x - q.x * v.z) * w2,
            v.z * c + q.z * d + (q.x * v.y - q.y * v.x) * w2};
}
struct M3 {
  float m[3][3];
};
__host__ __device__ __forceinline__ M3 qmat(float4 q) {
  float x = q.x, y = q.y, z = q.z, w = q.w;
  M3 R;
  R.m[0][0] = 1.0f - 2.0f * (y * y + z * z);
  R.m[0][1] = 2.0f * (x * y - z * w);
  R.m[0][2] = 2.0f * (x * z + y * w);
  R.m[1][0] = 2.0f * (x * y + z * w);
  R.m[1][1] = 1.0f - 2.0f * (x * x + z * z);
  R.m[1][2] = 2.0f * (y * z - x * w);
  R.m[2][0] = 2.0f * (x * z - y * w);
  R.m[2][1] = 2.0f * (y * z + x * w);
  R.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
  return R;
}
__host__ __device__ __forceinline__ V3 mcol(const M3& R, int k) { return V3{R.m[0][k], R.m[1][k], R.m[2][k]}; }
__host__ __device__ __forceinline__ V3 mtv(const M3& R, V3 v) {
  return V3{R.m[0][0] * v.x + R.m[1][0] * v.y + R.m[2][0] * v.z, R.m[0][1] * v.x + R.m[1][1] * v.y + R.m[2][1] * v.z,
            R.m[0][2] * v.x + R.m[1][2] * v.y + R.m[2][2] * v.z};
}

// Rotation vector -> unit quaternion: kernels_6dof.py:63-73.
__device__ __forceinline__ float4 quat_from_rotvec(V3 rv) {
  float th = sqrtf(dot(rv, rv));
  if (th < 1.0e-9f) return make_float4(0.5f * rv.x, 0.5f * rv.y, 0.5f * rv.z, 1.0f);
  float s, c;
  sincosf(0.5f * th, &s, &c);
  s = s / th;
  return make_float4(s * rv.x, s * rv.y, s * rv.z, c);
}
// Unit quaternion -> rotation vector in [-pi, pi]: kernels_6dof.py:76-97.
__device__ __forceinline__ V3 quat_to_rotvec(float4 q) {
  if (q.w < 0.0f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
  V3 qv{q.x, q.y, q.z};
  float l = sqrtf(dot(qv, qv));
  if (l < 1.0e-9f) return V3{0.0f, 0.0f, 0.0f};
  float ang = 2.0f * atan2f(l, q.w);
  return qv * (ang / l);
}
__device__ __forceinline__ float4 qnormalize(float4 q) {
  float l = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  if (l > 0.0f) {
    float s = 1.0f / l;
    return make_float4(q.x * s, q.y * s, q.z * s, q.w * s);
  }
  return q;
}

// Duff et al. 2017 tangent of n: kernels_6dof.py:2208-2218.
__host__ __device__ __forceinline__ V3 orthonormal_basis(V3 n) {
  float sign = n.z >= 0.0f ? 1.0f : -1.0f;
  float a = -1.0f / (sign + n.z);
  float b = n.x * n.y * a;
  return V3{1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x};
}

// 64-bit contact-cache key (a < b, ordinal c).  The epoch tag lives in bits
// 50-63 of the stored slot.
__host__ __device__ __forceinline__ unsigned long long cache_key(int a, int b, int c) {
  return ((unsigned long long)(unsigned)a << 26) | ((unsigned long long)(unsigned)b << 2) | (unsigned long long)c;
}
#define KEY_MASK ((1ull << 50) - 1ull)
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z ^= z >> 31;
  z *= 0x7fb5d329728ea185ull;
  z ^= z >> 27;
  z *= 0x81dadef4bc2dd44dull;
  z ^= z >> 33;
  return z;
}
__host__ __device__ __forceinline__ unsigned epoch_tag(unsigned epoch) { return 1u + (epoch % 16000u); }

// Anchor-keyed cache (the 5 mm-quantized key of the reference's documented
// cache, PERFORMANCE_PROGRESS.md:122-125): bodies a < b plus the contact
// point in the body frame of a (the lower index), each coordinate rounded to
// 5 mm, folded into a 50-bit fingerprint.  A contact keeps its warm start
// while its anchor stays in the same 5 mm cell, whatever its ordinal in the
// manifold.
#define KEY_MASK50 ((1ull << 50) - 1ull)
__host__ __device__ __forceinline__ int quant_5mm(float x) {
#ifdef __CUDA_ARCH__
  float s = __fmul_rn(x, 200.0f);
  int q = __float2int_rn(s);  // round half to even
#else
  float s = x * 200.0f;
  int q = (int)nearbyintf(s);
#endif
  return q < -32767 ? -32767 : (q > 32767 ? 32767 : q);
}
__host__ __device__ __forceinline__ unsigned long long anchor_key(int a, int b, float ox, float oy, float oz) {
  unsigned long long k1 = ((unsigned long long)(unsigned)a << 32) | (unsigned long long)(unsigned)b;
  unsigned long long k2 = ((unsigned long long)(unsigned short)(short)quant_5mm(ox) << 32) |
                          ((unsigned long long)(unsigned short)(short)quant_5mm(oy) << 16) |
                          (unsigned long long)(unsigned short)(short)quant_5mm(oz);
  return mix64(k1 ^ mix64(k2 + 0x9E3779B97F4A7C15ull)) & KEY_MASK50;
}
// Two contacts of one pair in the same cells get distinct keys (the later
// ordinal is rehashed), so every contact has its own cache entry.
__host__ __device__ __forceinline__ unsigned long long anchor_key_rehash(unsigned long long k, int c) {
  return mix64(k + (unsigned long long)(c + 1)) & KEY_MASK50;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

}  // namespace avbd
