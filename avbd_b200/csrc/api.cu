// C ABI of libavbd6.so (declared in include/avbd6.h): arena layout, context,
// parameters, substep / frame launch (optionally replayed from one CUDA
// graph per substep), device counters.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"
#include "kernels.cuh"

using namespace avbd;

namespace avbd {
thread_local long long g_kernel_launches = 0;
}

namespace {

thread_local std::string g_err;

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
  g_err = what;
  if (e != cudaSuccess) {
    g_err += ": ";
    g_err += cudaGetErrorString(e);
  }
  return code;
}

// Arena arrays: id, element bytes, element count (from the dims).
#define AVBD_ARRAYS(X)                                                                                        \
  X(BX, 16, N) X(BQ, 16, N) X(BV, 16, N) X(BW, 16, N) X(BPV, 16, N) X(BPW, 16, N) X(BX0, 16, N) X(BQ0, 16, N) \
  X(BXIN, 16, N) X(BQIN, 16, N) X(BIW0, 16, N) X(BIW1, 16, N) X(BILOC, 16, N) X(BHE, 16, N) X(BPRIO, 4, N)    \
  X(COLOR, 4, N) X(COLOR2, 4, N) X(COLOR_STARTS, 4, 64) X(COLOR_BODIES, 4, N) X(SG_START, 4, N + 1)           \
  X(DG_START, 4, N + 1) X(DG_CNT, 4, N) X(DG_IDX, 4, 2 * DG) X(G_BODY, 8, G) X(G_META, 4, G) X(G_ROW0, 4, G)    \
  X(G_FLAGS, 4, G) X(G_OFFA, 16, G) X(G_OFFB, 16, G) X(G_N, 16, G) X(G_MAT, 16, G) X(G_LAM, 16, G)             \
  X(G_PEN, 16, G) X(G_AC0, 16, G) X(AABB_LO, 16, N) X(AABB_HI, 16, N) X(MORTON, 4, N) X(MORTON2, 4, N)        \
  X(ORDER, 4, N) X(ORDER2, 4, N) X(NODE_LO, 16, 2 * N) X(NODE_HI, 16, 2 * N) X(NODE_LEFT, 4, N)                \
  X(NODE_RIGHT, 4, N) X(NODE_PARENT, 4, 2 * N) X(NODE_FLAG, 4, N) X(BOUNDS, 4, 8) X(UP_CNT, 4, N)              \
  X(PAIR_START, 4, N + 1) X(PAIR_AB, 8, P) X(PAIR_INFO, 4, P) X(PAIR_NRM, 16, P) X(PAIR_OFF, 16, 8 * P)        \
  X(PAIR_GCNT, 4, P) X(PAIR_GSTART, 4, P + 1) X(PAIR_RSTART, 4, P + 1) X(PAIR_KEPT, 4, P + 1) X(H_KEY, 8, H)   \
  X(H_S0, 16, H) X(H_S1, 16, H) X(SCAN_PART, 4, 2 * SP) X(SORT_HIST, 4, SH) X(C_USED, 4, N) X(C_LOST, 4, N)        \
  X(C_HIST, 4, 64 * 128) X(MLP_W, 4, M) X(PARAMS, 1, (long long)sizeof(DevParams))                             \
  X(COUNTERS, 1, (long long)sizeof(DevCounters)) X(BP_TMP, 4, N * BP_SLOTS) X(NEW_LIST, 4, NC)                 \
  X(MLP_FEAT, 4, NC * MLP_IN) X(SCENE_OF, 4, NS > 0 ? N : 0) X(SCENE_TAB, 16, NS) X(DONE, 4, N)              \
  X(G_KEY, 8, KEYS ? G : 0) X(NODE_REC, 128, N) X(DG_OTHER, 4, 2 * DG) X(FSEP, 4, N)

enum ArrayId {
#define X(id, sz, cnt) A_##id,
  AVBD_ARRAYS(X)
#undef X
      A_COUNT
};
const char* kNames[] = {
#define X(id, sz, cnt) #id,
    AVBD_ARRAYS(X)
#undef X
};

bool compute_layout(const AvbdDims* dm, size_t* off, size_t* total) {
  if (!dm || dm->n_bodies < 0 || dm->n_static_groups < 0 || dm->pair_cap < 0 || dm->dyn_group_cap < 0 ||
      dm->dyn_row_cap < 0 || dm->hash_cap < 1 || (dm->hash_cap & (dm->hash_cap - 1)) != 0 ||
      (dm->mlp_floats != 0 && dm->mlp_floats != AVBD_MLP_FLOATS) || dm->new_cap < 0 || dm->n_scenes < 0 ||
      dm->anchor_keys < 0 || dm->anchor_keys > 1)
    return false;
  long long N = dm->n_bodies > 0 ? dm->n_bodies : 1;
  long long DG = dm->dyn_group_cap;
  long long G = (long long)dm->n_static_groups + DG;
  if (G < 1) G = 1;
  long long P = dm->pair_cap > 0 ? dm->pair_cap : 1;
  long long H = dm->hash_cap;
  long long M = dm->mlp_floats;
  long long NC = dm->new_cap;
  long long NS = dm->n_scenes;
  long long KEYS = dm->anchor_keys;
  long long nblk = (N + 2047) / 2048;
  long long SH = 256 * nblk + 1;
  long long big = P > SH ? P : SH;
  if (N > big) big = N;
  long long SP = big / 2048 + 4;
  size_t o = 0;
  int k = 0;
#define X(id, sz, cnt)                             \
  o = (o + 255) & ~(size_t)255;                    \
  off[k++] = o;                                    \
  o += (size_t)(sz) * (size_t)((cnt) > 0 ? (cnt) : 1);
  AVBD_ARRAYS(X)
#undef X
  *total = (o + 255) & ~(size_t)255;
  return true;
}

}  // namespace

namespace avbd {
// Error text for entry points defined in other translation units.
void set_error_text(const char* what, cudaError_t e) { fail(0, what, e); }
}  // namespace avbd

struct AvbdCtx {
  AvbdDims dims;
  AvbdParams P;
  DevParams dp;
  Dev d;
  char* arena;
  size_t bytes;
  int num_sms;
  int coll_grid;
  int solve_grid, solve_block, solve_variant;
  int sweep_grid;  // CTAs of the standalone flag-sweep launch (0: the sweep runs inside the persistent kernel)
  int sweep_minb;  // CTAs per SM the sweep launch is built for (2: 320 threads, 3: 256 threads)
  // parts: 0 = collision with an LBVH rebuild, 1 = solve, 2 = collision
  // that refits the previous tree
  cudaGraphExec_t exec[3];
  cudaGraph_t graph[3];
  bool graph_ok[3];
  int graph_key[3][4];
  int capture_err[3];
  int part_kernels[3];
  // Whole-frame graphs (avbd_step): the frame's substeps, each its
  // collision part and solve part with event-record nodes between them, in
  // one graph; one graph per pattern of LBVH rebuilds over the substeps.
  static const int kFrameGraphs = 8;
  cudaGraphExec_t fexec[kFrameGraphs];
  cudaGraph_t fgraph[kFrameGraphs];
  unsigned fpattern[kFrameGraphs];
  int fkey[kFrameGraphs][16];
  int fkernels[kFrameGraphs];
  int nframe;
  int frame_capture_err;
  int frame_graph_used;  // the last avbd_step ran as one whole-frame graph
  int bvh_age;        // substeps since the last LBVH rebuild (0: none yet)
  int last_coll_part; // collision part of the last substep
  long long kernels_launched;
  long long substeps_done;
  float cur_dt;
  cudaEvent_t ev[3];
  StageTimer timer;      // stage events of a profiled collision pipeline
  int profile_next;      // the next substep runs its collision pipeline eagerly, timed
  int profile_ready;     // timer holds a completed profile
};

extern "C" {
static void drop_graph(AvbdCtx* c, int part);
}

// Any error a runtime call left behind is recorded here and cleared, so it
// never surfaces later inside the caller's own CUDA calls.
static int settle_errors(int code, const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess && code == AVBD_OK) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return AVBD_E_CUDA;
  }
  return code;
}

extern "C" {

int avbd_num_arrays(void) { return A_COUNT; }
const char* avbd_array_name(int id) { return (id >= 0 && id < A_COUNT) ? kNames[id] : nullptr; }
const char* avbd_last_error(void) { return g_err.c_str(); }

int avbd_layout(const AvbdDims* dims, size_t* offsets, size_t* total_bytes) {
  if (!offsets || !total_bytes) return fail(AVBD_E_INVALID, "null output");
  if (!compute_layout(dims, offsets, total_bytes)) return fail(AVBD_E_INVALID, "invalid dims");
  return AVBD_OK;
}

int avbd_create(const AvbdDims* dims, void* arena, size_t arena_bytes, AvbdCtx** out) {
  if (!out || !arena) return fail(AVBD_E_INVALID, "null argument");
  size_t off[A_COUNT], total = 0;
  if (!compute_layout(dims, off, &total)) return fail(AVBD_E_INVALID, "invalid dims");
  if (arena_bytes < total) return fail(AVBD_E_INVALID, "arena smaller than the layout");
  if (((uintptr_t)arena & 255) != 0) return fail(AVBD_E_INVALID, "arena not 256-byte aligned");
  AvbdCtx* c = new AvbdCtx();
  std::memset(c, 0, sizeof(*c));
  c->dims = *dims;
  c->arena = (char*)arena;
  c->bytes = arena_bytes;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (c->num_sms <= 0) c->num_sms = 148;
  c->coll_grid = c->num_sms * 4;
  Dev& d = c->d;
  char* a = c->arena;
#define PTR(T, id) reinterpret_cast<T>(a + off[A_##id])
  d.prm = PTR(const DevParams*, PARAMS);
  d.nb = dims->n_bodies;
  d.n_sg = dims->n_static_groups;
  d.n_static_rows = dims->n_static_rows;
  d.g_cap = dims->n_static_groups + dims->dyn_group_cap;
  d.row_cap = dims->n_static_rows + dims->dyn_row_cap;
  d.pair_cap = dims->pair_cap;
  d.nbr_cap = 0;
  d.hash_cap = dims->hash_cap;
  d.x = PTR(float4*, BX); d.q = PTR(float4*, BQ); d.v = PTR(float4*, BV); d.w = PTR(float4*, BW);
  d.pv = PTR(float4*, BPV); d.pw = PTR(float4*, BPW); d.x0 = PTR(float4*, BX0); d.q0 = PTR(float4*, BQ0);
  d.xin = PTR(float4*, BXIN); d.qin = PTR(float4*, BQIN); d.iw0 = PTR(float4*, BIW0); d.iw1 = PTR(float4*, BIW1);
  d.iloc = PTR(float4*, BILOC); d.he = PTR(float4*, BHE); d.prio = PTR(float*, BPRIO);
  d.color = PTR(int*, COLOR); d.color2 = PTR(int*, COLOR2); d.color_starts = PTR(int*, COLOR_STARTS);
  d.color_bodies = PTR(int*, COLOR_BODIES); d.sg_start = PTR(int*, SG_START); d.dg_start = PTR(int*, DG_START);
  d.dg_cnt = PTR(int*, DG_CNT); d.dg_idx = PTR(int*, DG_IDX);
  d.dg_other = PTR(int*, DG_OTHER);
  d.g_body = PTR(int2*, G_BODY); d.g_meta = PTR(int*, G_META); d.g_row0 = PTR(int*, G_ROW0);
  d.g_flags = PTR(int*, G_FLAGS); d.g_offa = PTR(float4*, G_OFFA); d.g_offb = PTR(float4*, G_OFFB);
  d.g_n = PTR(float4*, G_N); d.g_mat = PTR(float4*, G_MAT); d.g_lam = PTR(float4*, G_LAM);
  d.g_pen = PTR(float4*, G_PEN); d.g_ac0 = PTR(float4*, G_AC0);
  d.aabb_lo = PTR(float4*, AABB_LO); d.aabb_hi = PTR(float4*, AABB_HI);
  d.morton = PTR(unsigned*, MORTON); d.morton2 = PTR(unsigned*, MORTON2);
  d.order = PTR(int*, ORDER); d.order2 = PTR(int*, ORDER2);
  d.node_lo = PTR(float4*, NODE_LO); d.node_hi = PTR(float4*, NODE_HI); d.node_left = PTR(int*, NODE_LEFT);
  d.node_right = PTR(int*, NODE_RIGHT); d.node_parent = PTR(int*, NODE_PARENT); d.node_flag = PTR(int*, NODE_FLAG);
  d.node_rec = PTR(float4*, NODE_REC);
  d.bounds = PTR(float*, BOUNDS);
  d.nbr_cnt = d.nbr_start = d.nbr_idx = d.nbr_pair = nullptr;
  d.up_cnt = PTR(int*, UP_CNT); d.pair_start = PTR(int*, PAIR_START); d.bp_tmp = PTR(int*, BP_TMP);
  d.pair_ab = PTR(int2*, PAIR_AB); d.pair_info = PTR(int*, PAIR_INFO); d.pair_nrm = PTR(float4*, PAIR_NRM);
  d.pair_off = PTR(float4*, PAIR_OFF); d.pair_gcnt = PTR(int*, PAIR_GCNT); d.pair_gstart = PTR(int*, PAIR_GSTART);
  d.pair_rstart = PTR(int*, PAIR_RSTART); d.pair_kept = PTR(int*, PAIR_KEPT);
  d.h_key = PTR(unsigned long long*, H_KEY); d.h_s0 = PTR(float4*, H_S0); d.h_s1 = PTR(float4*, H_S1);
  d.scan_part = PTR(int*, SCAN_PART); d.sort_hist = PTR(int*, SORT_HIST);
  d.c_used = PTR(int*, C_USED); d.c_lost = PTR(int*, C_LOST); d.c_hist = PTR(int*, C_HIST);
  d.mlp_w = dims->mlp_floats > 0 ? PTR(const float*, MLP_W) : nullptr;
  d.new_cap = dims->new_cap;
  d.new_list = PTR(int*, NEW_LIST);
  d.mlp_feat = PTR(float*, MLP_FEAT);
  d.n_scenes = dims->n_scenes;
  d.scene_of = dims->n_scenes > 0 ? PTR(const int*, SCENE_OF) : nullptr;
  d.scene_tab = dims->n_scenes > 0 ? PTR(const float4*, SCENE_TAB) : nullptr;
  d.done = PTR(int*, DONE);
  d.fsep = PTR(float*, FSEP);
  d.g_key = dims->anchor_keys ? PTR(unsigned long long*, G_KEY) : nullptr;
  d.ctr = PTR(DevCounters*, COUNTERS);
#undef PTR
  int occ = solve_occupancy(256, 2);
  c->solve_block = 256;
  c->solve_variant = 2;
  c->solve_grid = c->num_sms * (occ > 0 ? occ : 1);
  c->P.dt = 1.0f / 60.0f;
  c->P.iterations = 10;
  c->P.substeps = 1;
  c->P.group_size = 16;
  c->P.use_graph = 1;
  c->P.persistent = 1;
  for (int k = 0; k < 3; ++k) cudaEventCreate(&c->ev[k]);
  for (int k = 0; k < StageTimer::kMax; ++k) cudaEventCreate(&c->timer.ev[k]);
  *out = c;
  return AVBD_OK;
}

static void drop_frame_graphs(AvbdCtx* c) {
  for (int k = 0; k < c->nframe; ++k) {
    if (c->fexec[k]) cudaGraphExecDestroy(c->fexec[k]);
    if (c->fgraph[k]) cudaGraphDestroy(c->fgraph[k]);
    c->fexec[k] = nullptr;
    c->fgraph[k] = nullptr;
  }
  c->nframe = 0;
}

int avbd_destroy(AvbdCtx* c) {
  if (!c) return AVBD_OK;
  for (int part = 0; part < 3; ++part) drop_graph(c, part);
  drop_frame_graphs(c);
  for (int k = 0; k < 3; ++k)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  for (int k = 0; k < StageTimer::kMax; ++k)
    if (c->timer.ev[k]) cudaEventDestroy(c->timer.ev[k]);
  delete c;
  return AVBD_OK;
}

static void fill_devparams(AvbdCtx* c, float dt_sub) {
  const AvbdParams& P = c->P;
  DevParams& q = c->dp;
  std::memset(&q, 0, sizeof(q));
  q.dt = dt_sub;
  q.iterations = P.iterations;
  q.gx = P.gravity[0];
  q.gy = P.gravity[1];
  q.gz = P.gravity[2];
  q.alpha = P.alpha;
  q.beta = P.beta;
  q.gamma = P.gamma;
  q.post_stab = P.post_stabilize ? 1 : 0;
  // solver_6dof.py:1514-1522: both caps must be positive and finite, else off.
  bool caps = P.max_linear_speed > 0.0f && std::isfinite(P.max_linear_speed) && P.max_angular_speed > 0.0f &&
              std::isfinite(P.max_angular_speed);
  q.max_lin = caps ? P.max_linear_speed : INFINITY;
  q.max_ang = caps ? P.max_angular_speed : INFINITY;
  q.fsm = P.friction_static_mult;
  q.color_mode = P.coloring_mode;
  q.recolor_every = P.recolor_every_substep;
  q.self_friction = P.self_friction;
  int g = P.group_size;
  q.group_size = (g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32) ? g : 16;
  q.record_violation = P.record_violation;
  q.debug_skip_arrive = P.debug_skip_arrive;
  q.mlp_on = P.mlp_warm_start && c->dims.mlp_floats > 0 && c->dims.new_cap > 0;
  q.log_new = P.log_new_contacts && c->dims.new_cap > 0;
  q.batched = c->dims.n_scenes > 0;
  q.flag_sweep = P.flag_sweep;
  q.adaptive_lanes = P.adaptive_lanes;
  q.resting_floor = P.resting_floor;
  q.barrier_timeout_ns = P.debug_skip_arrive ? 200000000ull : 2000000000ull;
  q.timing = P.timing;
}

int avbd_set_params(AvbdCtx* c, const AvbdParams* p, void* stream) {
  if (!c || !p) return fail(AVBD_E_INVALID, "null argument");
  if (p->iterations < 0 || p->iterations > AVBD_MAX_VIOL_ITERS || p->substeps < 1)
    return fail(AVBD_E_INVALID, "iterations must be in [0, 256] and substeps >= 1");
  c->P = *p;
  c->cur_dt = p->dt / (float)p->substeps;
  fill_devparams(c, c->cur_dt);
  cudaError_t e = cudaMemcpyAsync((void*)c->d.prm, &c->dp, sizeof(DevParams), cudaMemcpyHostToDevice, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "params upload", e);
  // Persistent grid: `blocks_per_sm` CTAs per SM (0 = 2), using the
  // register budget built for it, capped by the measured occupancy.
  // With the flag sweep as its own launch, blocks_per_sm shapes that launch;
  // the persistent head and tail keep the 2-CTA build (the 3-CTA build
  // spills 2.8 KB per thread).
  int want = p->blocks_per_sm > 0 ? p->blocks_per_sm : 2;
  c->sweep_minb = want >= 3 ? 3 : 2;
  if (p->flag_sweep) want = 2;
  c->solve_variant = want >= 3 ? 3 : 2;
  int occ = solve_occupancy(256, c->solve_variant);
  int b = want < occ ? want : occ;
  c->solve_grid = c->num_sms * (b > 0 ? b : 1);
  c->sweep_grid = p->flag_sweep ? sweep_grid_size(p->group_size, c->d.n_scenes > 0, c->num_sms, c->sweep_minb) : 0;
  return AVBD_OK;
}

int avbd_reset_state(AvbdCtx* c, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  launch_reset(c->d, (cudaStream_t)stream);
  c->substeps_done = 0;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "reset", e);
}

int avbd_mark_color_dirty(AvbdCtx* c, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  int one = 1;
  cudaError_t e = cudaMemcpyAsync(&c->d.ctr->color_dirty, &one, sizeof(int), cudaMemcpyHostToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "mark dirty", e);
}

// Part 0 = collision pipeline, part 1 = solve.  Each part is captured as its
// own CUDA graph; the timing events are recorded between the graph launches.
static cudaError_t enqueue_part(AvbdCtx* c, int part, cudaStream_t st) {
  long long before = g_kernel_launches;
  cudaError_t e;
  if (part != 1) {
    launch_collision(c->d, c->P, c->dims, c->coll_grid, st, part == 0);
    e = cudaGetLastError();
  } else {
    e = launch_solve(c->d, c->P, c->P.persistent, c->solve_grid, c->solve_block, st, c->solve_variant,
                     c->sweep_grid, c->sweep_minb);
  }
  c->part_kernels[part] = (int)(g_kernel_launches - before);
  return e;
}

static void part_key(AvbdCtx* c, int part, int key[4]) {
  if (part != 1) {
    key[0] = c->P.self_collide; key[1] = c->coll_grid; key[2] = 0; key[3] = 0;
  } else {
    key[0] = c->P.persistent + 10 * c->solve_variant; key[1] = c->solve_grid;
    key[2] = c->P.persistent ? (c->P.flag_sweep ? 1000 + c->P.group_size : 0)
                             : c->P.iterations + 100 * c->P.post_stabilize;
    key[3] = c->P.persistent ? c->sweep_grid : c->P.coloring_mode;
  }
}

static void drop_graph(AvbdCtx* c, int part) {
  if (c->exec[part]) { cudaGraphExecDestroy(c->exec[part]); c->exec[part] = nullptr; }
  if (c->graph[part]) { cudaGraphDestroy(c->graph[part]); c->graph[part] = nullptr; }
  c->graph_ok[part] = false;
}

// Capture one part; on failure remember the error and stop trying.
static void capture_part(AvbdCtx* c, int part, cudaStream_t st) {
  drop_graph(c, part);
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    c->capture_err[part] = (int)e;
    cudaGetLastError();
    return;
  }
  cudaError_t le = enqueue_part(c, part, st);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(st, &g);
  cudaGraphExec_t ex = nullptr;
  if (le == cudaSuccess && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
    c->graph[part] = g;
    c->exec[part] = ex;
    c->graph_ok[part] = true;
    part_key(c, part, c->graph_key[part]);
    c->capture_err[part] = 0;
  } else {
    c->capture_err[part] = (int)(le != cudaSuccess ? le : (e != cudaSuccess ? e : cudaErrorUnknown));
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
}

static cudaError_t run_part(AvbdCtx* c, int part, cudaStream_t st) {
  if (c->P.use_graph && st != nullptr && c->capture_err[part] == 0) {
    int key[4];
    part_key(c, part, key);
    if (c->graph_ok[part] && std::memcmp(key, c->graph_key[part], sizeof(key)) != 0) drop_graph(c, part);
    if (!c->graph_ok[part]) capture_part(c, part, st);
    if (c->graph_ok[part]) {
      c->kernels_launched += c->part_kernels[part];
      return cudaGraphLaunch(c->exec[part], st);
    }
  }
  cudaError_t e = enqueue_part(c, part, st);
  c->kernels_launched += c->part_kernels[part];
  return e;
}

// Collision part of the next substep by the LBVH cadence (rebuild every
// bvh_rebuild_every substeps, refit in between); advances the cadence.
static int next_collision_part(AvbdCtx* c) {
  bool collide = c->P.self_collide && c->d.nb >= 2;
  int every = c->P.bvh_rebuild_every > 1 ? c->P.bvh_rebuild_every : 1;
  bool rebuild = !collide || c->bvh_age == 0 || c->bvh_age >= every;
  c->bvh_age = !collide ? 0 : (rebuild ? 1 : c->bvh_age + 1);
  return rebuild ? 0 : 2;
}

static int run_substep(AvbdCtx* c, cudaStream_t st) {
  if (c->d.nb == 0) return AVBD_OK;
  if (c->substeps_done > 0 && c->substeps_done % 8192 == 0) launch_hash_scrub(c->d, st);
  // The pair list does not depend on the tree (pairs come out sorted by
  // body), so between rebuilds the LBVH is only refit to the new boxes.
  int part = next_collision_part(c);
  c->last_coll_part = part;
  cudaEventRecord(c->ev[0], st);
  cudaError_t e;
  if (c->profile_next) {  // a one-off graph of the pipeline with an event node after each stage
    c->timer.n = 0;
    c->profile_next = 0;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      g_stage_timer = &c->timer;
      cudaError_t le = enqueue_part(c, part, st);
      g_stage_timer = nullptr;
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(st, &g);
      if (le != cudaSuccess) e = le;
      cudaGraphExec_t ex = nullptr;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
      if (e == cudaSuccess) e = cudaGraphLaunch(ex, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (ex) cudaGraphExecDestroy(ex);
      if (g) cudaGraphDestroy(g);
    }
    c->kernels_launched += c->part_kernels[part];
    c->profile_ready = e == cudaSuccess;
  } else {
    e = run_part(c, part, st);
  }
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "collision launch", e);
  cudaEventRecord(c->ev[1], st);
  e = run_part(c, 1, st);
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "solve launch", e);
  cudaEventRecord(c->ev[2], st);
  c->substeps_done++;
  return AVBD_OK;
}

// Batched scenes: a frame is slots 0..substeps-1; a scene takes part in the
// first `its substeps` slots.  The device counts slots from this reset.
static int reset_slot(AvbdCtx* c, cudaStream_t st) {
  if (c->dims.n_scenes <= 0) return AVBD_OK;
  cudaError_t e = cudaMemsetAsync(&c->d.ctr->slot_next, 0, sizeof(int), st);
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "slot reset", e);
}

static int substep_impl(AvbdCtx* c, float dt, cudaStream_t st) {
  if (dt != c->cur_dt) {
    c->cur_dt = dt;
    fill_devparams(c, dt);
    cudaError_t e = cudaMemcpyAsync((void*)c->d.prm, &c->dp, sizeof(DevParams), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(AVBD_E_CUDA, "params upload", e);
  }
  return settle_errors(run_substep(c, st), "substep");
}

int avbd_substep(AvbdCtx* c, float dt, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  cudaStream_t st = (cudaStream_t)stream;
  int r = reset_slot(c, st);  // batched: one substep = slot 0, every scene at its own dt
  c->frame_graph_used = 0;
  return r != AVBD_OK ? r : substep_impl(c, dt, st);
}

static void frame_key(AvbdCtx* c, unsigned pattern, int key[16]) {
  std::memset(key, 0, 16 * sizeof(int));
  part_key(c, 0, key);
  part_key(c, 1, key + 4);
  part_key(c, 2, key + 8);
  key[12] = c->P.substeps;
  key[13] = (int)pattern;
}

// Captures one frame: per substep, event ev[0], collision part, ev[1], solve
// part, ev[2] (event-record nodes, so avbd_step_ms reads the last substep's
// parts as with the per-part graphs).
static int capture_frame(AvbdCtx* c, unsigned pattern, cudaStream_t st) {
  if (c->nframe >= AvbdCtx::kFrameGraphs) drop_frame_graphs(c);
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    c->frame_capture_err = (int)e;
    cudaGetLastError();
    return -1;
  }
  long long before = g_kernel_launches;
  cudaError_t le = cudaSuccess;
  for (int s = 0; s < c->P.substeps && le == cudaSuccess; ++s) {
    int part = ((pattern >> s) & 1u) ? 0 : 2;
    le = cudaEventRecordWithFlags(c->ev[0], st, cudaEventRecordExternal);
    if (le == cudaSuccess) le = enqueue_part(c, part, st);
    if (le == cudaSuccess) le = cudaEventRecordWithFlags(c->ev[1], st, cudaEventRecordExternal);
    if (le == cudaSuccess) le = enqueue_part(c, 1, st);
    if (le == cudaSuccess) le = cudaEventRecordWithFlags(c->ev[2], st, cudaEventRecordExternal);
  }
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(st, &g);
  cudaGraphExec_t ex = nullptr;
  if (le == cudaSuccess && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
    int k = c->nframe++;
    c->fgraph[k] = g;
    c->fexec[k] = ex;
    c->fpattern[k] = pattern;
    frame_key(c, pattern, c->fkey[k]);
    c->fkernels[k] = (int)(g_kernel_launches - before);
    cudaGetLastError();
    return k;
  }
  c->frame_capture_err = (int)(le != cudaSuccess ? le : (e != cudaSuccess ? e : cudaErrorUnknown));
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  return -1;
}

int avbd_step(AvbdCtx* c, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  cudaStream_t st = (cudaStream_t)stream;
  float dt = c->P.dt / (float)c->P.substeps;
  int r = reset_slot(c, st);
  bool frame = c->P.use_graph && st != nullptr && c->d.nb > 0 && c->P.substeps <= 32 && !c->profile_next &&
               c->frame_capture_err == 0;
  if (r == AVBD_OK && frame) {
    if (dt != c->cur_dt) {
      c->cur_dt = dt;
      fill_devparams(c, dt);
      cudaError_t e = cudaMemcpyAsync((void*)c->d.prm, &c->dp, sizeof(DevParams), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return fail(AVBD_E_CUDA, "params upload", e);
    }
    // the contact-cache scrub, every 8192 substeps, runs before the frame it falls in
    long long s0 = c->substeps_done;
    for (int s = 0; s < c->P.substeps; ++s)
      if (s0 + s > 0 && (s0 + s) % 8192 == 0) launch_hash_scrub(c->d, st);
    int age0 = c->bvh_age;
    unsigned pattern = 0;
    int last = 0;
    for (int s = 0; s < c->P.substeps; ++s) {
      last = next_collision_part(c);
      if (last == 0) pattern |= 1u << s;
    }
    int key[16];
    frame_key(c, pattern, key);
    int k = -1;
    for (int j = 0; j < c->nframe; ++j)
      if (std::memcmp(key, c->fkey[j], sizeof(key)) == 0) k = j;
    if (k < 0) k = capture_frame(c, pattern, st);
    if (k >= 0) {
      cudaError_t e = cudaGraphLaunch(c->fexec[k], st);
      if (e != cudaSuccess) return fail(AVBD_E_CUDA, "frame graph launch", e);
      c->kernels_launched += c->fkernels[k];
      c->substeps_done += c->P.substeps;
      c->last_coll_part = last;
      c->frame_graph_used = 1;
      return settle_errors(AVBD_OK, "step");
    }
    c->bvh_age = age0;  // capture failed: the per-substep path below replays the cadence
  }
  c->frame_graph_used = 0;
  for (int s = 0; s < c->P.substeps && r == AVBD_OK; ++s) r = substep_impl(c, dt, st);
  return r;
}

int avbd_read_stats(AvbdCtx* c, AvbdStats* out, void* stream) {
  if (!c || !out) return fail(AVBD_E_INVALID, "null argument");
  DevCounters h;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(&h, c->d.ctr, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "stats readback", e);
  std::memset(out, 0, sizeof(*out));
  out->n_pairs_found = h.n_pairs_found;
  out->n_pairs = h.n_pairs;
  out->n_dyn_groups = h.n_dyn_groups;
  out->n_dyn_rows = h.n_dyn_rows;
  out->n_dyn_rows_req = h.n_dyn_rows_req;
  out->n_contacts_req = h.n_contacts_req;
  out->n_colors = h.n_colors;
  out->recolored = h.recolored;
  out->conflicts = h.conflicts;
  out->err = h.err;
  out->err_where = h.err_where;
  out->n_cache_hits = h.n_cache_hits;
  out->n_new_contacts = h.n_new_contacts;
  out->max_dg = h.max_dg;
  out->n_viol = h.n_viol;
  out->epoch = h.epoch;
  out->graph_state = c->frame_graph_used ? 7 : ((c->graph_ok[c->last_coll_part] ? 1 : 0) | (c->graph_ok[1] ? 2 : 0));
  out->capture_err = c->capture_err[c->last_coll_part] * 1000 + c->capture_err[1];
  out->kernels_launched = c->kernels_launched;
  out->n_new_logged = h.n_new_logged;
  out->n_mlp_applied = h.n_mlp_applied;
  out->n_mlp_fallback = h.n_mlp_fallback;
  out->n_mlp_reverted = h.n_mlp_reverted;
  for (int k = 0; k < AVBD_MAX_VIOL_ITERS; ++k) {
    unsigned b = h.vc_max_bits[k];
    float f;
    memcpy(&f, &b, sizeof f);
    out->viol_contact[k] = f;
  }
  for (int k = 0; k < AVBD_MAX_VIOL_ITERS; ++k) {
    unsigned b = h.viol_bits[k];
    float f;
    std::memcpy(&f, &b, 4);
    out->viol[k] = f;
  }
  if (h.err & AVBD_ERR_BARRIER_TIMEOUT) return fail(AVBD_E_TIMEOUT, "device barrier timed out");
  return settle_errors(AVBD_OK, "read_stats");
}

int avbd_cache_load(AvbdCtx* c, int n, const int* abc, const float* state, void* stream) {
  if (!c || n < 0 || (n > 0 && (!abc || !state))) return fail(AVBD_E_INVALID, "bad cache arguments");
  if (n > 0 && c->dims.anchor_keys) return fail(AVBD_E_INVALID, "anchor-keyed cache: use avbd_cache_load_keys");
  launch_cache_load(c->d, n, abc, nullptr, state, (cudaStream_t)stream);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "cache load", e);
}

int avbd_cache_load_keys(AvbdCtx* c, int n, const unsigned long long* keys, const float* state, void* stream) {
  if (!c || n < 0 || (n > 0 && (!keys || !state))) return fail(AVBD_E_INVALID, "bad cache arguments");
  launch_cache_load(c->d, n, nullptr, keys, state, (cudaStream_t)stream);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "cache load", e);
}

int avbd_clear_errors(AvbdCtx* c, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  cudaError_t e = cudaMemsetAsync(&c->d.ctr->err, 0, 2 * sizeof(int), (cudaStream_t)stream);
  // a solve that stopped early may leave the coloring flags set
  if (e == cudaSuccess && c->d.nb > 0)
    e = cudaMemsetAsync(c->d.c_lost, 0, (size_t)c->d.nb * sizeof(int), (cudaStream_t)stream);
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "clear errors", e);
}

int avbd_step_ms(AvbdCtx* c, float* collide_ms, float* solve_ms) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  cudaError_t e = cudaEventSynchronize(c->ev[2]);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(AVBD_E_CUDA, "event sync", e);
  }
  float a = 0.0f, b = 0.0f;
  if (cudaEventElapsedTime(&a, c->ev[0], c->ev[1]) != cudaSuccess) a = 0.0f;
  if (cudaEventElapsedTime(&b, c->ev[1], c->ev[2]) != cudaSuccess) b = 0.0f;
  cudaGetLastError();
  if (collide_ms) *collide_ms = a;
  if (solve_ms) *solve_ms = b;
  return AVBD_OK;
}

int avbd_read_phase_marks(AvbdCtx* c, long long* t_ns, int* phase, int cap, void* stream) {
  if (!c || !t_ns || !phase || cap < 0) return fail(AVBD_E_INVALID, "bad arguments");
  DevCounters h;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(&h, c->d.ctr, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "marks readback", e);
  int n = h.n_marks < cap ? h.n_marks : cap;
  if (n > 256) n = 256;
  for (int k = 0; k < n; ++k) {
    t_ns[k] = (long long)h.mark_t[k];
    phase[k] = h.mark_id[k];
  }
  return n;
}

int avbd_count_color_conflicts(AvbdCtx* c, void* stream) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  return count_conflicts(c->d, (cudaStream_t)stream);
}


int avbd_profile_next_substep(AvbdCtx* c) {
  if (!c) return fail(AVBD_E_INVALID, "null ctx");
  c->profile_next = 1;
  c->profile_ready = 0;
  return AVBD_OK;
}

int avbd_collision_profile(AvbdCtx* c, float* ms, int cap) {
  // (the profiled pipeline ran as a one-off graph; its events are complete)
  if (!c || (!ms && cap > 0)) return fail(AVBD_E_INVALID, "null argument");
  if (!c->profile_ready) return fail(AVBD_E_INVALID, "no profiled substep has run");
  int n = c->timer.n;
  if (n < 1) return 0;
  cudaError_t e = cudaEventSynchronize(c->timer.ev[n - 1]);
  if (e != cudaSuccess) return fail(AVBD_E_CUDA, "profile events", e);
  int k = 0;
  for (; k + 1 < n && k < cap; ++k) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, c->timer.ev[k], c->timer.ev[k + 1]);
    ms[k] = t;
  }
  return k;
}

const char* avbd_collision_stage(AvbdCtx* c, int i) {
  if (!c || !c->profile_ready || i < 0 || i + 1 >= c->timer.n) return "";
  return c->timer.name[i + 1];
}

int avbd_build_floor_groups(AvbdCtx* c, int nblk, const int* blk_body, const float* blk_he_fy,
                            const float* blk_mat, const int* blk_row0, const int* blk_per, const int* blk_goff,
                            void* stream) {
  if (!c || nblk < 0 || (nblk > 0 && (!blk_body || !blk_he_fy || !blk_mat || !blk_row0 || !blk_per || !blk_goff)))
    return fail(AVBD_E_INVALID, "bad floor-block arguments");
  if (8LL * nblk > c->d.n_sg) return fail(AVBD_E_INVALID, "more floor corners than static groups");
  if (nblk == 0) return AVBD_OK;
  cudaError_t e = launch_floor_groups(c->d, nblk, blk_body, reinterpret_cast<const float4*>(blk_he_fy),
                                      reinterpret_cast<const float4*>(blk_mat), blk_row0, blk_per, blk_goff,
                                      (cudaStream_t)stream);
  return e == cudaSuccess ? AVBD_OK : fail(AVBD_E_CUDA, "floor groups", e);
}

}  // extern "C"
