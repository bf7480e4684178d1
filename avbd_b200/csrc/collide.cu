// Collision pipeline of one substep: AABBs, LBVH broad phase, 15-axis SAT +
// contact manifold, contact-group emission with the warm-start cache lookup,
// and the body -> dynamic-group incidence lists.
//
// Compiled with -fmad=false: the SAT axis choice, the clip tests and the
// contact selection take the same branches as the oracle's float code
// (compiled with -ffp-contract=off), operation for operation.
//
// Reference: solver_6dof.py:1774-1916 (driver), kernels_6dof.py:1922-2130
// (AABB, BVH query, SAT), :2208-2537 (manifold), :2695-2912 (emission),
// :2588-2603 (cache key/hash), :2626-2692 (CSR).
#include <cuda/atomic>

#include "common.cuh"
#include "kernels.cuh"

namespace avbd {

// ---------------------------------------------------------------------------
// Grid-stride helpers.
// ---------------------------------------------------------------------------
#define GSTRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

__device__ __forceinline__ int f2ord(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// ---------------------------------------------------------------------------
// Substep start: reset counters and the scene bounds used for Morton codes.
// ---------------------------------------------------------------------------
__global__ void k_begin_substep(const __grid_constant__ Dev d) {
  if (blockIdx.x == 0 && d.prm->record_violation)  // per-iteration violation records of this substep
    for (int k = threadIdx.x; k < AVBD_MAX_VIOL_ITERS; k += blockDim.x) {
      d.ctr->viol_bits[k] = 0u;
      d.ctr->vc_max_bits[k] = 0u;
      d.ctr->vc_cnt[k] = 0;
    }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    DevCounters* c = d.ctr;
    c->n_pairs_found = 0;
    c->n_nbr_found = 0;
    c->n_pairs = 0;
    c->n_dyn_groups = 0;
    c->n_dyn_rows = 0;
    c->n_dyn_rows_req = 0;
    c->n_contacts_req = 0;
    c->conflicts = 0;
    c->n_cache_hits = 0;
    c->n_new_contacts = 0;
    c->n_new_logged = 0;
    c->n_mlp_applied = 0;
    c->n_mlp_fallback = 0;
    c->n_mlp_reverted = 0;
    for (int k = 0; k < 4; ++k) c->work_ctr[k] = 0;
    c->slot = c->slot_next;  // substep slot within the frame (batched scenes)
    c->slot_next = c->slot + 1;
    c->max_dg = 0;
    c->n_viol = 0;
    c->bar_count = 0;
    for (int k = 0; k < BAR_SUB; ++k) c->bar_sub[k][0] = 0;
    int* b = (int*)d.bounds;
    b[0] = b[1] = b[2] = 0x7fffffff;
    b[3] = b[4] = b[5] = (int)0x80000000;
  }
  GSTRIDE(i, d.nb) {
    d.dg_cnt[i] = 0;
  }
}

// OBB -> world AABB with margin (kernels_6dof.py:1922-1943), plus the bounds
// of the AABB centres for the Morton grid.
__global__ void k_aabb(const __grid_constant__ Dev d) {
  __shared__ int sb[6];
  if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? 0x7fffffff : (int)0x80000000;
  __syncthreads();
  GSTRIDE(i, d.nb) {
    float4 x = d.x[i];
    float4 he = d.he[i];
    M3 R = qmat(d.q[i]);
    float ex = fabsf(R.m[0][0]) * he.x + fabsf(R.m[0][1]) * he.y + fabsf(R.m[0][2]) * he.z + COLL_MARGIN;
    float ey = fabsf(R.m[1][0]) * he.x + fabsf(R.m[1][1]) * he.y + fabsf(R.m[1][2]) * he.z + COLL_MARGIN;
    float ez = fabsf(R.m[2][0]) * he.x + fabsf(R.m[2][1]) * he.y + fabsf(R.m[2][2]) * he.z + COLL_MARGIN;
    d.aabb_lo[i] = make_float4(x.x - ex, x.y - ey, x.z - ez, 0.0f);
    d.aabb_hi[i] = make_float4(x.x + ex, x.y + ey, x.z + ez, 0.0f);
    atomicMin(&sb[0], f2ord(x.x));
    atomicMin(&sb[1], f2ord(x.y));
    atomicMin(&sb[2], f2ord(x.z));
    atomicMax(&sb[3], f2ord(x.x));
    atomicMax(&sb[4], f2ord(x.y));
    atomicMax(&sb[5], f2ord(x.z));
  }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin((int*)d.bounds + threadIdx.x, sb[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax((int*)d.bounds + threadIdx.x, sb[threadIdx.x]);
}

__device__ __forceinline__ unsigned spread10(unsigned v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(const __grid_constant__ Dev d) {
  const int* b = (const int*)d.bounds;
  float lx = ord2f(b[0]), ly = ord2f(b[1]), lz = ord2f(b[2]);
  float hx = ord2f(b[3]), hy = ord2f(b[4]), hz = ord2f(b[5]);
  float sx = hx > lx ? 1023.0f / (hx - lx) : 0.0f;
  float sy = hy > ly ? 1023.0f / (hy - ly) : 0.0f;
  float sz = hz > lz ? 1023.0f / (hz - lz) : 0.0f;
  GSTRIDE(i, d.nb) {
    float4 x = d.x[i];
    unsigned ix = (unsigned)fminf(fmaxf((x.x - lx) * sx, 0.0f), 1023.0f);
    unsigned iy = (unsigned)fminf(fmaxf((x.y - ly) * sy, 0.0f), 1023.0f);
    unsigned iz = (unsigned)fminf(fmaxf((x.z - lz) * sz, 0.0f), 1023.0f);
    d.morton[i] = (spread10(ix) << 2) | (spread10(iy) << 1) | spread10(iz);
    d.order[i] = i;
  }
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan (three launches).  SCAN_CHUNK ints per block
// (common.cuh).  out[n] receives the total.
// ---------------------------------------------------------------------------

__device__ __forceinline__ int warp_incl_scan(int v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane_id() >= o) v += t;
  }
  return v;
}
// Block-wide exclusive scan of one value per thread (blockDim = SCAN_T).
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
  __shared__ int ws[SCAN_T / 32];
  int inc = warp_incl_scan(v);
  int w = threadIdx.x >> 5;
  if (lane_id() == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    int s = lane_id() < SCAN_T / 32 ? ws[lane_id()] : 0;
    int si = warp_incl_scan(s);
    if (lane_id() < SCAN_T / 32) ws[lane_id()] = si - s;
    if (lane_id() == SCAN_T / 32 - 1) *total = si;
  }
  __syncthreads();
  int r = ws[w] + inc - v;
  __syncthreads();
  return r;
}

__device__ __forceinline__ void scan_reduce_body(const int* in, int n, int* part) {
  int base = blockIdx.x * SCAN_CHUNK;
  int s = 0;
  if (base < n) {
    int i0 = base + threadIdx.x * SCAN_V;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k)
      if (i0 + k < n) s += in[i0 + k];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ int ws[SCAN_T / 32];
  if (lane_id() == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < SCAN_T / 32; ++w) t += ws[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_scan_reduce(const int* in, int n_host, const int* n_dev, int* part) {
  scan_reduce_body(in, n_dev ? *n_dev : n_host, part);
}

// Single block: exclusive scan of part[0..np) in place; part[np] = total.
__device__ __forceinline__ void scan_parts_body(int* part, int np) {
  __shared__ int carry;
  __shared__ int tot;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < np; base += SCAN_T) {
    int i = base + threadIdx.x;
    int v = i < np ? part[i] : 0;
    int e = block_excl_scan(v, &tot);
    if (i < np) part[i] = carry + e;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) part[np] = carry;
}

__global__ void k_scan_parts(int* part, int np) { scan_parts_body(part, np); }

__device__ __forceinline__ void scan_down_body(const int* in, int* out, int n, const int* part, int np,
                                               int* total_out) {
  int base = blockIdx.x * SCAN_CHUNK;
  if (base > n) return;
  int i0 = base + threadIdx.x * SCAN_V;
  int v[SCAN_V];
  int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    v[k] = (i0 + k < n) ? in[i0 + k] : 0;
    s += v[k];
  }
  __shared__ int tot;
  int e = block_excl_scan(s, &tot) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    if (i0 + k < n) out[i0 + k] = e;
    e += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    out[n] = part[np];
    if (total_out) *total_out = part[np];
  }
}

__global__ void k_scan_down(const int* in, int* out, int n_host, const int* n_dev, const int* part, int np,
                            int* total_out) {
  scan_down_body(in, out, n_dev ? *n_dev : n_host, part, np, total_out);
}

// Two scans of the same length in one set of three launches: blockIdx.y
// picks the array (its partials follow the first array's np + 1).
struct Scan2 {
  const int* in[2];
  int* out[2];
};
__global__ void k_scan2_reduce(Scan2 s, int n_host, const int* n_dev, int* part, int np) {
  const int y = blockIdx.y;
  scan_reduce_body(s.in[y], n_dev ? *n_dev : n_host, part + y * (np + 1));
}
__global__ void k_scan2_parts(int* part, int np) { scan_parts_body(part + blockIdx.y * (np + 1), np); }
__global__ void k_scan2_down(Scan2 s, int n_host, const int* n_dev, const int* part, int np) {
  const int y = blockIdx.y;
  scan_down_body(s.in[y], s.out[y], n_dev ? *n_dev : n_host, part + y * (np + 1), np, nullptr);
}

void scan2_launch(const Dev& d, const int* in0, int* out0, const int* in1, int* out1, int n_cap, const int* n_dev,
                  cudaStream_t st) {
  int np = (n_cap + SCAN_CHUNK) / SCAN_CHUNK;
  if (np < 1) np = 1;
  Scan2 s{{in0, in1}, {out0, out1}};
  k_scan2_reduce<<<dim3(np, 2), SCAN_T, 0, st>>>(s, n_cap, n_dev, d.scan_part, np);
  k_scan2_parts<<<dim3(1, 2), SCAN_T, 0, st>>>(d.scan_part, np);
  k_scan2_down<<<dim3(np, 2), SCAN_T, 0, st>>>(s, n_cap, n_dev, d.scan_part, np);
  g_kernel_launches += 3;
}

void scan_launch(const Dev& d, const int* in, int* out, int n_cap, const int* n_dev, int* total_out,
                 cudaStream_t st) {
  int np = (n_cap + SCAN_CHUNK) / SCAN_CHUNK;  // covers index n_cap for the total
  if (np < 1) np = 1;
  k_scan_reduce<<<np, SCAN_T, 0, st>>>(in, n_cap, n_dev, d.scan_part);
  k_scan_parts<<<1, SCAN_T, 0, st>>>(d.scan_part, np);
  k_scan_down<<<np, SCAN_T, 0, st>>>(in, out, n_cap, n_dev, d.scan_part, np, total_out);
  g_kernel_launches += 3;
}

// ---------------------------------------------------------------------------
// LSD radix sort of (morton, body) pairs, 8-bit digits, 4 passes, stable.
// ---------------------------------------------------------------------------
#define RS_T 256
#define RS_CHUNKS 8
#define RS_TILE (RS_T * RS_CHUNKS)

__global__ void k_radix_hist(const unsigned* keys, int n, int shift, int* hist, int nblk) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * RS_TILE;
  for (int k = 0; k < RS_CHUNKS; ++k) {
    int i = base + k * RS_T + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
  }
  __syncthreads();
  hist[threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_radix_scatter(const unsigned* keys, const int* vals, unsigned* okeys, int* ovals, int n, int shift,
                                const int* hist_scan, int nblk) {
  __shared__ int run[256];      // running count per digit within this tile
  __shared__ int wcnt[8][256];  // per-warp digit counts of the current chunk
  int w = threadIdx.x >> 5, l = lane_id();
  run[threadIdx.x] = hist_scan[threadIdx.x * nblk + blockIdx.x];
  int base = blockIdx.x * RS_TILE;
  for (int k = 0; k < RS_CHUNKS; ++k) {
    for (int u = 0; u < 8; ++u) wcnt[u][threadIdx.x] = 0;
    __syncthreads();
    int i = base + k * RS_T + threadIdx.x;
    bool valid = i < n;
    unsigned key = valid ? keys[i] : 0u;
    int dig = valid ? (int)((key >> shift) & 255u) : 256 + l;  // invalid lanes get unique dummies
    unsigned peers = __match_any_sync(0xffffffffu, dig);
    int rank = __popc(peers & ((1u << l) - 1u));
    if (valid && rank == 0) wcnt[w][dig] = __popc(peers);
    __syncthreads();
    if (valid) {
      int off = run[dig];
      for (int u = 0; u < w; ++u) off += wcnt[u][dig];
      int pos = off + rank;
      okeys[pos] = key;
      ovals[pos] = vals[i];
    }
    __syncthreads();
    int tot = 0;
    for (int u = 0; u < 8; ++u) tot += wcnt[u][threadIdx.x];
    run[threadIdx.x] += tot;
    __syncthreads();
  }
}

void radix_sort_launch(Dev& d, cudaStream_t st) {
  int n = d.nb;
  int nblk = (n + RS_TILE - 1) / RS_TILE;
  unsigned* ks[2] = {d.morton, d.morton2};
  int* vs[2] = {d.order, d.order2};
  for (int pass = 0; pass < 4; ++pass) {
    int src = pass & 1;
    k_radix_hist<<<nblk, RS_T, 0, st>>>(ks[src], n, pass * 8, d.sort_hist, nblk);
    scan_launch(d, d.sort_hist, d.sort_hist, 256 * nblk, nullptr, nullptr, st);
    k_radix_scatter<<<nblk, RS_T, 0, st>>>(ks[src], vs[src], ks[src ^ 1], vs[src ^ 1], n, pass * 8, d.sort_hist,
                                           nblk);
    g_kernel_launches += 2;
  }
  // four passes: the sorted result is back in (morton, order)
}

// ---------------------------------------------------------------------------
// Karras (2012) LBVH over the sorted Morton codes.  Nodes [0, n-1) are
// internal, [n-1, 2n-1) leaves (leaf k = k-th body in Morton order).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int delta(const unsigned* m, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  unsigned a = m[i], b = m[j];
  if (a == b) return 32 + __clz((unsigned)(i ^ j));
  return __clz(a ^ b);
}

__global__ void k_lbvh_build(const __grid_constant__ Dev d) {
  int n = d.nb;
  const unsigned* m = d.morton;
  GSTRIDE(i, n - 1) {
    int dir = (delta(m, n, i, i + 1) - delta(m, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(m, n, i, i - dir);
    int lmax = 2;
    while (delta(m, n, i, i + lmax * dir) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (delta(m, n, i, i + (l + t) * dir) > dmin) l += t;
    int j = i + l * dir;
    int dnode = delta(m, n, i, j);
    int s = 0;
    int len = l;
    int t = (len + 1) >> 1;
    while (true) {
      if (delta(m, n, i, i + (s + t) * dir) > dnode) s += t;
      if (t == 1) break;
      t = (t + 1) >> 1;
    }
    int split = i + s * dir + min(dir, 0);
    int first = min(i, j), last = max(i, j);
    int left = (first == split) ? (n - 1 + split) : split;
    int right = (last == split + 1) ? (n - 1 + split + 1) : split + 1;
    d.node_left[i] = left;
    d.node_right[i] = right;
    d.node_parent[left] = i;
    d.node_parent[right] = i;
    d.node_flag[i] = 0;
  }
  GSTRIDE(k, n) {
    int b = d.order[k];
    d.node_lo[n - 1 + k] = d.aabb_lo[b];
    d.node_hi[n - 1 + k] = d.aabb_hi[b];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.node_parent[0] = -1;
}

// Between rebuilds: the tree keeps its topology and leaf order; leaves take
// the bodies' new boxes and the refit below recomputes the internal ones.
__global__ void k_lbvh_leaves(const __grid_constant__ Dev d) {
  int n = d.nb;
  GSTRIDE(i, n - 1) d.node_flag[i] = 0;
  GSTRIDE(k, n) {
    int b = d.order[k];
    d.node_lo[n - 1 + k] = d.aabb_lo[b];
    d.node_hi[n - 1 + k] = d.aabb_hi[b];
  }
}

__global__ void k_lbvh_refit(const __grid_constant__ Dev d) {
  int n = d.nb;
  GSTRIDE(k, n) {
    int node = n - 1 + k;
    int p = d.node_parent[node];
    int guard = 0;
    while (p >= 0 && guard < 128) {
      // acq_rel: this thread's box store above is released with the
      // arrival, and the second child to arrive acquires its sibling's box
      cuda::atomic_ref<int, cuda::thread_scope_device> arrivals(d.node_flag[p]);
      if (arrivals.fetch_add(1, cuda::memory_order_acq_rel) == 0) break;  // first child to arrive stops
      int l = d.node_left[p], r = d.node_right[p];
      float4 a = __ldcg(&d.node_lo[l]), b = __ldcg(&d.node_lo[r]);
      float4 c = __ldcg(&d.node_hi[l]), e = __ldcg(&d.node_hi[r]);
      d.node_lo[p] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.0f);
      d.node_hi[p] = make_float4(fmaxf(c.x, e.x), fmaxf(c.y, e.y), fmaxf(c.z, e.z), 0.0f);
      p = d.node_parent[p];
      ++guard;
    }
    if (guard >= 128) atomicOr(&d.ctr->err, ERR_BVH);
  }
}

// Traversal copy of the tree, two levels per record: internal node p's
// record lists up to four entries -- each child that is a leaf, and the two
// children of each child that is internal -- as (lo, code) (hi, static), 32
// bytes each, 128 per record.  code >= 0: an internal node (descend into its
// record); code <= -2: a leaf, body -code - 2 (no lookup of the Morton order
// during the walk), static flag in hi.w; -1: no entry.  A walk loads half the
// records a binary walk would.  Written after every refit.
__device__ __forceinline__ void pack_entry(const Dev& d, int n, int c, float4* e) {
  float4 lo = d.node_lo[c], hi = d.node_hi[c];
  int code = c;
  float st = 0.0f;
  if (c >= n - 1) {
    int b = d.order[c - (n - 1)];
    code = -2 - b;
    st = d.x[b].w <= 0.0f ? 1.0f : 0.0f;
  }
  e[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(code));
  e[1] = make_float4(hi.x, hi.y, hi.z, st);
}

__global__ void k_lbvh_pack(const __grid_constant__ Dev d) {
  int n = d.nb;
  GSTRIDE(p, n - 1) {
    float4* rec = d.node_rec + 8 * (size_t)p;
    int k = 0;
    int ch[2] = {d.node_left[p], d.node_right[p]};
    for (int a = 0; a < 2; ++a) {
      int c = ch[a];
      if (c >= n - 1) {
        pack_entry(d, n, c, rec + 2 * k++);
      } else {
        pack_entry(d, n, d.node_left[c], rec + 2 * k++);
        pack_entry(d, n, d.node_right[c], rec + 2 * k++);
      }
    }
    for (; k < 4; ++k) {
      rec[2 * k] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
      rec[2 * k + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
}

__device__ __forceinline__ bool overlap(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  return alo.x <= bhi.x && blo.x <= ahi.x && alo.y <= bhi.y && blo.y <= ahi.y && alo.z <= bhi.z && blo.z <= ahi.z;
}

// Query body i's AABB; calls fn(j) for every body j > i that overlaps and is
// not static-static (kernels_6dof.py:1946-1978, closed-interval test).
template <class F>
__device__ __forceinline__ void bvh_query_upper(const Dev& d, int i, F fn) {
  int n = d.nb;
  float4 lo = d.aabb_lo[i], hi = d.aabb_hi[i];
  bool si = d.x[i].w <= 0.0f;
  int sc = d.scene_of ? d.scene_of[i] : 0;  // batched scenes never collide with each other
  auto report = [&](int j, bool sj) {
    if (j > i && !(si && sj) && (!d.scene_of || d.scene_of[j] == sc)) fn(j);
  };
  if (!overlap(lo, hi, d.node_lo[0], d.node_hi[0])) return;
  if (n - 1 <= 0) {  // a single body: the root is its leaf
    report(d.order[0], d.x[d.order[0]].w <= 0.0f);
    return;
  }
  // Entries are tested before they are pushed: overlapping leaves are
  // reported at once, the first overlapping internal entry is descended
  // into directly, and the others are pushed.
  constexpr int STACK = 96;
  int stack[STACK];
  int sp = 0;
  int node = 0;
  while (true) {
    const float4* rec = d.node_rec + 8 * (size_t)node;
    float4 r[8];  // the whole record in one round trip
#pragma unroll
    for (int e = 0; e < 8; ++e) r[e] = __ldg(rec + e);
    int next = -1;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float4 elo = r[2 * e], ehi = r[2 * e + 1];
      int code = __float_as_int(elo.w);
      if (code == -1 || !overlap(lo, hi, elo, ehi)) continue;
      if (code <= -2) {
        report(-2 - code, ehi.w != 0.0f);
      } else if (next < 0) {
        next = code;
      } else {
        if (sp + 1 > STACK) {
          atomicOr(&d.ctr->err, ERR_BVH);
          return;
        }
        stack[sp++] = code;
      }
    }
    if (next >= 0) {
      node = next;
    } else {
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
}

// One traversal per body, threads in Morton order (a warp walks nearby
// bodies, so its traversals share tree nodes).  The first BP_SLOTS upper
// neighbours are kept in a per-body buffer for k_bp_fill.
__global__ void k_bp_count(const __grid_constant__ Dev d) {
  GSTRIDE(k, d.nb) {
    int i = d.order[k];
    int c = 0;
    int* slot = d.bp_tmp + (size_t)i * BP_SLOTS;
    bvh_query_upper(d, i, [&](int j) {
      if (c < BP_SLOTS) slot[c] = j;
      ++c;
    });
    d.up_cnt[i] = c;
  }
}

// Writes body i's upper neighbours (j > i) as canonical pairs at
// pair_start[i].., sorted by j, keeping those below pair_cap, so the pair
// list is ordered by (i, j).  Bodies with more than BP_SLOTS upper neighbours
// traverse again.
__global__ void k_bp_fill(const __grid_constant__ Dev d) {
  int cap = d.pair_cap;
  GSTRIDE(k, d.nb) {
    int i = d.order[k];
    int s = d.pair_start[i];
    int n = d.up_cnt[i];
    if (s >= cap || n == 0) continue;
    if (n <= BP_SLOTS) {
      int v[BP_SLOTS];
      const int* slot = d.bp_tmp + (size_t)i * BP_SLOTS;
      for (int a = 0; a < n; ++a) {  // insertion sort by j
        int x = slot[a];
        int b = a - 1;
        while (b >= 0 && v[b] > x) {
          v[b + 1] = v[b];
          --b;
        }
        v[b + 1] = x;
      }
      int e = min(n, cap - s);
      for (int a = 0; a < e; ++a) d.pair_ab[s + a] = make_int2(i, v[a]);
      continue;
    }
    // Rare: more neighbours than slots.  Keep the smallest j's below the cap
    // by repeated selection over fresh traversals (bounded by n).
    int e = min(n, cap - s);
    int last = -1;
    for (int a = 0; a < e; ++a) {
      int best = 0x7fffffff;
      bvh_query_upper(d, i, [&](int j) {
        if (j > last && j < best) best = j;
      });
      d.pair_ab[s + a] = make_int2(i, best);
      last = best;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int found = d.pair_start[d.nb];
    d.ctr->n_pairs_found = found;
    d.ctr->n_pairs = min(found, cap);
    if (found > cap) atomicOr(&d.ctr->err, ERR_PAIR_OVERFLOW);
  }
}

// ---------------------------------------------------------------------------
// 15-axis SAT (kernels_6dof.py:1991-2130) and contact manifold
// (kernels_6dof.py:2221-2537).  One thread per pair.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float proj_radius(V3 L, V3 c0, V3 c1, V3 c2, V3 he) {
  return he.x * fabsf(dot(L, c0)) + he.y * fabsf(dot(L, c1)) + he.z * fabsf(dot(L, c2));
}

struct Manifold {
  int overlap, sat_idx, count, ref_is_a;
  V3 n;  // SAT normal (B -> A)
  float depth;
  V3 nn;  // contact normal (inc -> ref)
  V3 off_ref[4], off_inc[4];
  float pen[4];  // penetration depth of each contact (>0 when penetrating)
};

// The clip polygons of one thread in shared memory: 2 buffers x 8 vertices x
// 3 floats, float s of the thread at s * NARROW_BLOCK (a warp's accesses hit
// 32 banks), instead of 192 bytes of local memory per thread that the
// narrow phase's occupancy pushed out of L1.
#define NARROW_BLOCK 128
struct ClipPoly {
  float* col;  // this thread's column
  __device__ __forceinline__ V3 get(int b, int k) const {
    const float* p = col + (b * 8 + k) * 3 * NARROW_BLOCK;
    return V3{p[0], p[NARROW_BLOCK], p[2 * NARROW_BLOCK]};
  }
  __device__ __forceinline__ void set(int b, int k, V3 v) const {
    float* p = col + (b * 8 + k) * 3 * NARROW_BLOCK;
    p[0] = v.x;
    p[NARROW_BLOCK] = v.y;
    p[2 * NARROW_BLOCK] = v.z;
  }
};

__device__ void sat_manifold(V3 cA, M3 RA, V3 eA, V3 cB, M3 RB, V3 eB, Manifold& o, ClipPoly poly) {
  o.overlap = 0;
  o.sat_idx = -1;
  o.count = 0;
  o.ref_is_a = 0;
  V3 t = cB - cA;
  V3 A[3] = {mcol(RA, 0), mcol(RA, 1), mcol(RA, 2)};
  V3 B[3] = {mcol(RB, 0), mcol(RB, 1), mcol(RB, 2)};
  float best = 1.0e20f;
  int bi = -1;
  V3 ba{0.0f, 0.0f, 0.0f};
  for (int k = 0; k < 3; ++k) {
    V3 L = A[k];
    float rA = comp(eA, k);
    float rB = proj_radius(L, B[0], B[1], B[2], eB);
    float tl = dot(t, L);
    float ov = rA + rB - fabsf(tl);
    if (ov < -COLL_MARGIN) return;
    if (ov < best) { best = ov; bi = k; ba = tl > 0.0f ? -L : L; }
  }
  for (int k = 0; k < 3; ++k) {
    V3 L = B[k];
    float rA = proj_radius(L, A[0], A[1], A[2], eA);
    float rB = comp(eB, k);
    float tl = dot(t, L);
    float ov = rA + rB - fabsf(tl);
    if (ov < -COLL_MARGIN) return;
    if (ov < best) { best = ov; bi = 3 + k; ba = tl > 0.0f ? -L : L; }
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      V3 L = cross(A[i], B[j]);
      float nl = sqrtf(dot(L, L));
      if (nl < 1.0e-6f) continue;
      L = L / nl;
      float rA = proj_radius(L, A[0], A[1], A[2], eA);
      float rB = proj_radius(L, B[0], B[1], B[2], eB);
      float tl = dot(t, L);
      float ov = rA + rB - fabsf(tl);
      if (ov < 0.0f) return;
      if (ov < best) { best = ov; bi = 6 + 3 * i + j; ba = tl > 0.0f ? -L : L; }
    }
  o.overlap = 1;
  o.sat_idx = bi;
  o.n = ba;
  o.depth = best;

  if (bi >= 6) {  // edge-edge: Ericson 5.1.9 closest points, one contact
    int e = bi - 6, kA = e / 3, kB = e % 3;
    V3 eAd = A[kA], eBd = B[kB];
    V3 cr = cross(eAd, eBd);
    if (sqrtf(dot(cr, cr)) < 1.0e-4f) return;
    int kA1 = (kA + 1) % 3, kA2 = (kA + 2) % 3;
    V3 toB = cB - cA;
    float sbA = dot(toB, A[kA1]) >= 0.0f ? 1.0f : -1.0f;
    float scA = dot(toB, A[kA2]) >= 0.0f ? 1.0f : -1.0f;
    V3 midA = (cA + A[kA1] * (sbA * comp(eA, kA1))) + A[kA2] * (scA * comp(eA, kA2));
    V3 P1 = midA - eAd * comp(eA, kA);
    V3 Q1 = midA + eAd * comp(eA, kA);
    int kB1 = (kB + 1) % 3, kB2 = (kB + 2) % 3;
    V3 toA = cA - cB;
    float sbB = dot(toA, B[kB1]) >= 0.0f ? 1.0f : -1.0f;
    float scB = dot(toA, B[kB2]) >= 0.0f ? 1.0f : -1.0f;
    V3 midB = (cB + B[kB1] * (sbB * comp(eB, kB1))) + B[kB2] * (scB * comp(eB, kB2));
    V3 P2 = midB - eBd * comp(eB, kB);
    V3 Q2 = midB + eBd * comp(eB, kB);
    V3 d1 = Q1 - P1, d2 = Q2 - P2, r = P1 - P2;
    float a = dot(d1, d1), ev = dot(d2, d2), f = dot(d2, r);
    const float eps = 1.0e-12f;
    float s = 0.0f, tp = 0.0f;
    if (a <= eps && ev <= eps) {
      s = 0.0f;
      tp = 0.0f;
    } else if (a <= eps) {
      s = 0.0f;
      tp = fminf(fmaxf(f / fmaxf(ev, eps), 0.0f), 1.0f);
    } else if (ev <= eps) {
      tp = 0.0f;
      float c = dot(d1, r);
      s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
    } else {
      float c = dot(d1, r), b = dot(d1, d2);
      float den = a * ev - b * b;
      s = den != 0.0f ? fminf(fmaxf((b * f - c * ev) / den, 0.0f), 1.0f) : 0.0f;
      tp = (b * s + f) / ev;
      if (tp < 0.0f) {
        tp = 0.0f;
        s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
      } else if (tp > 1.0f) {
        tp = 1.0f;
        s = fminf(fmaxf((b - c) / a, 0.0f), 1.0f);
      }
    }
    V3 pA = P1 + d1 * s, pB = P2 + d2 * tp;
    float gap = dot(pA - pB, ba);
    if (gap > COLL_MARGIN) return;
    o.count = 1;
    o.ref_is_a = 1;
    o.nn = ba;
    o.off_ref[0] = mtv(RA, pA - cA);
    o.off_inc[0] = mtv(RB, pB - cB);
    o.pen[0] = -gap;
    return;
  }
  // face-face: Sutherland-Hodgman clip of the incident face by the
  // reference face's side planes, keep points within the margin, top 4.
  int ref_is_a = bi < 3 ? 1 : 0;
  o.ref_is_a = ref_is_a;
  int ref_axis = ref_is_a ? bi : bi - 3;
  V3 nu = ref_is_a ? ba : -ba;
  V3 ref_c = ref_is_a ? cA : cB, inc_c = ref_is_a ? cB : cA;
  V3 e_ref = ref_is_a ? eA : eB, e_inc = ref_is_a ? eB : eA;
  const M3& Rr = ref_is_a ? RA : RB;
  const M3& Ri = ref_is_a ? RB : RA;
  V3 rca = mcol(Rr, ref_axis);
  float rsign = dot(rca, nu) > 0.0f ? -1.0f : 1.0f;
  V3 rfn = rca * rsign;
  V3 rfc = ref_c + rfn * comp(e_ref, ref_axis);
  int ax1 = (ref_axis + 1) % 3, ax2 = (ref_axis + 2) % 3;
  V3 u = mcol(Rr, ax1), v = mcol(Rr, ax2);
  float eu = comp(e_ref, ax1), evv = comp(e_ref, ax2);
  int ia = 0;
  float isg = 1.0f, bd = -1.0e20f;
  for (int k = 0; k < 3; ++k) {
    float dp = dot(mcol(Ri, k), nu);
    if (dp > bd) { bd = dp; ia = k; isg = 1.0f; }
    float dn = -dp;
    if (dn > bd) { bd = dn; ia = k; isg = -1.0f; }
  }
  V3 ifn = mcol(Ri, ia) * isg;
  V3 ifc = inc_c + ifn * comp(e_inc, ia);
  int ia1 = (ia + 1) % 3, ia2 = (ia + 2) % 3;
  V3 iu = mcol(Ri, ia1), iv = mcol(Ri, ia2);
  float ieu = comp(e_inc, ia1), iev = comp(e_inc, ia2);
  int cur = 0;
  poly.set(0, 0, (ifc + iu * ieu) + iv * iev);
  poly.set(0, 1, (ifc - iu * ieu) + iv * iev);
  poly.set(0, 2, (ifc - iu * ieu) - iv * iev);
  poly.set(0, 3, (ifc + iu * ieu) - iv * iev);
  int len = 4;
  for (int pl = 0; pl < 4; ++pl) {
    V3 pp, pn;
    if (pl == 0) { pp = rfc + u * eu; pn = u; }
    else if (pl == 1) { pp = rfc - u * eu; pn = -u; }
    else if (pl == 2) { pp = rfc + v * evv; pn = v; }
    else { pp = rfc - v * evv; pn = -v; }
    if (len == 0) return;
    int ol = 0, nx = cur ^ 1;
    for (int k = 0; k < len; ++k) {
      V3 ap = poly.get(cur, k);
      V3 bp = poly.get(cur, (k + 1) % len);
      float da = dot(ap - pp, pn), db = dot(bp - pp, pn);
      if (da <= 0.0f) {
        if (ol < 8) poly.set(nx, ol++, ap);
        if (db > 0.0f) {
          float tt = da / (da - db);
          if (ol < 8) poly.set(nx, ol++, ap + (bp - ap) * tt);
        }
      } else if (db <= 0.0f) {
        float tt = da / (da - db);
        if (ol < 8) poly.set(nx, ol++, ap + (bp - ap) * tt);
      }
    }
    cur = nx;
    len = ol;
  }
  if (len == 0) return;
  float bdp[4] = {-1.0e30f, -1.0e30f, -1.0e30f, -1.0e30f};
  int bix[4] = {-1, -1, -1, -1};
  int nbst = 0;
  for (int k = 0; k < len; ++k) {
    float ds = dot(poly.get(cur, k) - rfc, rfn);
    if (ds < COLL_MARGIN) {
      float depth = -ds;
      if (nbst < 4) {
        bdp[nbst] = depth;
        bix[nbst] = k;
        ++nbst;
      } else {
        int mp = 0;
        float mv = bdp[0];
        for (int q = 1; q < 4; ++q)
          if (bdp[q] < mv) { mv = bdp[q]; mp = q; }
        if (depth > mv) { bdp[mp] = depth; bix[mp] = k; }
      }
    }
  }
  if (nbst == 0) return;
  for (int a = 0; a < nbst - 1; ++a) {
    int mp = a;
    for (int k = a + 1; k < nbst; ++k)
      if (bdp[k] > bdp[mp]) mp = k;
    if (mp != a) {
      float td = bdp[a]; bdp[a] = bdp[mp]; bdp[mp] = td;
      int ti = bix[a]; bix[a] = bix[mp]; bix[mp] = ti;
    }
  }
  o.nn = nu;
  o.count = nbst;
  for (int c = 0; c < nbst; ++c) {
    V3 pi = poly.get(cur, bix[c]);
    float ds = dot(pi - rfc, rfn);
    V3 pr = pi - rfn * ds;
    o.off_ref[c] = mtv(Rr, pr - ref_c);
    o.off_inc[c] = mtv(Ri, pi - inc_c);
    o.pen[c] = bdp[c];
  }
}

// SAT + manifold per pair; writes the per-pair group/row counts for the scans.
// The counters every thread adds to are summed per warp first: one atomic
// per warp instead of one per pair on a single address.
__global__ void k_narrow(const __grid_constant__ Dev d) {
  int np = d.ctr->n_pairs;
  float self_friction = d.prm->self_friction;
  int creq = 0;
  __shared__ float clip_sm[48 * NARROW_BLOCK];
  const ClipPoly poly{clip_sm + threadIdx.x};
  GSTRIDE(p, np) {
    int2 ab = d.pair_ab[p];
    float4 xa = d.x[ab.x], xb = d.x[ab.y];
    float4 ha = d.he[ab.x], hb = d.he[ab.y];
    Manifold o;
    sat_manifold(xyz(xa), qmat(d.q[ab.x]), xyz(ha), xyz(xb), qmat(d.q[ab.y]), xyz(hb), o, poly);
    d.pair_info[p] = o.overlap | ((o.sat_idx & 31) << 1) | (o.count << 6) | (o.ref_is_a << 9);
    d.pair_nrm[p] = make_float4(o.nn.x, o.nn.y, o.nn.z, o.depth);
    for (int c = 0; c < o.count; ++c) {
      d.pair_off[8 * p + c] = make_float4(o.off_ref[c].x, o.off_ref[c].y, o.off_ref[c].z, o.pen[c]);
      d.pair_off[8 * p + 4 + c] = make_float4(o.off_inc[c].x, o.off_inc[c].y, o.off_inc[c].z, 0.0f);
    }
    // friction of the contact (kernels_6dof.py:2775-2780): sqrt(mu_ref mu_inc)
    // if either body has friction, else the default.
    float mr = ha.w, mi = hb.w;
    float mu = (mr > 0.0f || mi > 0.0f) ? sqrtf(mr * mi) : self_friction;
    int rpc = mu <= 0.0f ? 1 : 3;
    d.pair_gcnt[p] = o.count;
    d.pair_kept[p] = o.count * rpc;  // rows requested (scanned next)
    creq += o.count;
  }
  creq = __reduce_add_sync(0xffffffffu, creq);
  if ((threadIdx.x & 31) == 0 && creq) atomicAdd(&d.ctr->n_contacts_req, creq);
}

// Contact-cache lookup of key k written by the previous substep's refresh.
__device__ __forceinline__ int cache_find(const Dev& d, unsigned long long k, unsigned tag) {
  unsigned mask = (unsigned)d.hash_cap - 1u;
  unsigned h = (unsigned)mix64(k) & mask;
  unsigned long long want = k | ((unsigned long long)tag << 50);
  for (int probe = 0; probe < 4096; ++probe) {
    unsigned s = (h + probe) & mask;
    unsigned long long v = d.h_key[s];
    if (v == want) return (int)s;
    if ((unsigned)(v >> 50) != tag) return -1;
  }
  return -1;
}

// The 20 inputs of the learned warm start for one new contact (ref body a,
// incident body b): normal in a's frame (3), penetration depth (1), relative
// contact-point velocity in the (t, b, n) contact frame (3), inverse masses
// (2), n^T I^-1 n of both bodies (2), mu_s, mu_d (2), one-hot SAT axis class
// of the pair, A being its lower body index (face of A x/y/z, face of B
// x/y/z, edge-edge) (7).
__device__ void contact_features(const Dev& d, int a, int b, float4 nn, float4 offa, float4 offb, int sat, float mu,
                                 float mus, float* out) {
  V3 n = xyz(nn);
  float4 xa = d.x[a], xb = d.x[b];
  M3 Ra = qmat(d.q[a]), Rb = qmat(d.q[b]);
  V3 na = mtv(Ra, n), nb = mtv(Rb, n);
  V3 ra = V3{Ra.m[0][0] * offa.x + Ra.m[0][1] * offa.y + Ra.m[0][2] * offa.z,
             Ra.m[1][0] * offa.x + Ra.m[1][1] * offa.y + Ra.m[1][2] * offa.z,
             Ra.m[2][0] * offa.x + Ra.m[2][1] * offa.y + Ra.m[2][2] * offa.z};
  V3 rb = V3{Rb.m[0][0] * offb.x + Rb.m[0][1] * offb.y + Rb.m[0][2] * offb.z,
             Rb.m[1][0] * offb.x + Rb.m[1][1] * offb.y + Rb.m[1][2] * offb.z,
             Rb.m[2][0] * offb.x + Rb.m[2][1] * offb.y + Rb.m[2][2] * offb.z};
  V3 va = xyz(d.v[a]) + cross(xyz(d.w[a]), ra);
  V3 vb = xyz(d.v[b]) + cross(xyz(d.w[b]), rb);
  V3 vr = va - vb;
  V3 t = orthonormal_basis(n);
  V3 bt = cross(n, t);
  float4 ia = d.iloc[a], ib = d.iloc[b];
  float nia = (ia.x > 0.0f ? na.x * na.x / ia.x : 0.0f) + (ia.y > 0.0f ? na.y * na.y / ia.y : 0.0f) +
              (ia.z > 0.0f ? na.z * na.z / ia.z : 0.0f);
  float nib = (ib.x > 0.0f ? nb.x * nb.x / ib.x : 0.0f) + (ib.y > 0.0f ? nb.y * nb.y / ib.y : 0.0f) +
              (ib.z > 0.0f ? nb.z * nb.z / ib.z : 0.0f);
  out[0] = na.x;
  out[1] = na.y;
  out[2] = na.z;
  out[3] = offa.w;
  out[4] = dot(vr, t);
  out[5] = dot(vr, bt);
  out[6] = dot(vr, n);
  out[7] = xa.w > 0.0f ? 1.0f / xa.w : 0.0f;
  out[8] = xb.w > 0.0f ? 1.0f / xb.w : 0.0f;
  out[9] = nia;
  out[10] = nib;
  out[11] = mus;
  out[12] = mu;
  int cls = sat < 6 ? sat : 6;
  for (int k = 0; k < 7; ++k) out[13 + k] = k == cls ? 1.0f : 0.0f;
}

// Emission (kernels_6dof.py:2695-2912): one contact group per contact, rows
// numbered after the static rows in pair order; contacts whose rows would
// pass the dynamic row capacity are dropped (:2795-2800).  Warm start from
// the contact cache, else lambda = 0, k = (1e6, 1, 1).
// Eight blocks per SM (64 registers, a small spill): a pair's contacts are a
// chain of dependent cache probes, so more pairs in flight beat the spill
// (0.091 -> 0.079 ms on the 100k pile).
__global__ void __launch_bounds__(128, 8) k_emit(const __grid_constant__ Dev d, int dyn_row_cap, int dyn_group_cap) {
  int np = d.ctr->n_pairs;
  float self_friction = d.prm->self_friction, fsm = d.prm->fsm;
  unsigned tag = epoch_tag(d.ctr->epoch);
  int n_groups = 0, n_rows = 0, n_hits = 0, n_new = 0;  // summed per warp after the loop
  GSTRIDE(p, np) {
    int info = d.pair_info[p];
    int cnt = (info >> 6) & 7;
    int kept = 0;
    if (cnt > 0) {
      int2 ab = d.pair_ab[p];
      int ref_is_a = (info >> 9) & 1;
      int ref = ref_is_a ? ab.x : ab.y, inc = ref_is_a ? ab.y : ab.x;
      float mr = d.he[ref].w, mi = d.he[inc].w;
      float mu = (mr > 0.0f || mi > 0.0f) ? sqrtf(mr * mi) : self_friction;
      float mus = mu * fsm;
      int rpc = mu <= 0.0f ? 1 : 3;
      int rs = d.pair_rstart[p], gs = d.pair_gstart[p];
      float4 nn = d.pair_nrm[p];
      int hits = 0;
      // anchor keys: the contact point in the lower body's (ab.x) frame
      unsigned long long akey[4] = {0ull, 0ull, 0ull, 0ull};
      if (d.g_key) {
        for (int c = 0; c < cnt; ++c) {
          float4 o = d.pair_off[8 * p + (ref_is_a ? 0 : 4) + c];
          unsigned long long k = anchor_key(ab.x, ab.y, o.x, o.y, o.z);
          for (int c2 = 0; c2 < c; ++c2)
            if (akey[c2] == k) k = anchor_key_rehash(k, c);
          akey[c] = k;
        }
      }
      for (int c = 0; c < cnt; ++c) {
        if (rs + (c + 1) * rpc > dyn_row_cap || gs + c + 1 > dyn_group_cap) break;
        int g = d.n_sg + gs + c;
        d.g_body[g] = make_int2(ref, inc);
        d.g_meta[g] = make_meta(KIND_BOX, rpc == 3, 1, c);
        d.g_row0[g] = d.n_static_rows + rs + c * rpc;
        d.g_offa[g] = d.pair_off[8 * p + c];
        d.g_offb[g] = d.pair_off[8 * p + 4 + c];
        d.g_n[g] = make_float4(nn.x, nn.y, nn.z, 0.0f);
        d.g_mat[g] = make_float4(mu, mus, __int_as_float(0x7f800000), __int_as_float(0x7f800000));
        float4 s0 = make_float4(0.0f, 0.0f, 0.0f, PEN_MIN);
        float4 s1 = make_float4(PEN_MIN_T, PEN_MIN_T, 0.0f, 0.0f);
        bool queued = false;
        unsigned long long key = d.g_key ? akey[c] : cache_key(ab.x, ab.y, c);
        if (d.g_key) d.g_key[g] = key;
        int slot = cache_find(d, key, tag);
        if (slot >= 0) {
          s0 = d.h_s0[slot];
          s1 = d.h_s1[slot];
          ++hits;
        } else if (d.prm->mlp_on || d.prm->log_new) {
          // A new contact: queue it (with its features) for the learned
          // warm start (its prelude then runs in that phase) or for the
          // training log.
          int k = atomicAdd(&d.ctr->n_new_logged, 1);
          if (k < d.new_cap) {
            queued = d.prm->mlp_on != 0;
            d.new_list[k] = g;
            contact_features(d, ref, inc, nn, d.pair_off[8 * p + c], d.pair_off[8 * p + 4 + c], (info >> 1) & 31, mu,
                             mus, d.mlp_feat + (size_t)MLP_IN * k);
          }
        }
        d.g_lam[g] = make_float4(s0.x, s0.y, s0.z, 0.0f);
        d.g_pen[g] = make_float4(s0.w, s1.x, s1.y, 0.0f);
        d.g_ac0[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int act = rpc == 3 ? (FL_ACT0 | FL_ACT1 | FL_ACT2) : FL_ACT0;
        int fl = act;
        if (rpc == 3) fl |= ((int)s1.z != 0 ? FL_WAST : 0) | ((int)s1.w != 0 ? FL_WASB : 0);
        if (queued) fl |= FL_NEW;
        d.g_flags[g] = fl;
        ++kept;
      }
      if (kept) {
        n_groups += kept;
        n_rows += kept * rpc;
        atomicAdd(&d.dg_cnt[ab.x], kept);
        atomicAdd(&d.dg_cnt[ab.y], kept);
      }
      if (kept < cnt) atomicOr(&d.ctr->err, ERR_ROW_OVERFLOW);
      n_hits += hits;
      n_new += max(kept - hits, 0);
    }
    d.pair_kept[p] = kept;
  }
  n_groups = __reduce_add_sync(0xffffffffu, n_groups);
  n_rows = __reduce_add_sync(0xffffffffu, n_rows);
  n_hits = __reduce_add_sync(0xffffffffu, n_hits);
  n_new = __reduce_add_sync(0xffffffffu, n_new);
  if ((threadIdx.x & 31) == 0) {
    if (n_groups) atomicAdd(&d.ctr->n_dyn_groups, n_groups);
    if (n_rows) atomicAdd(&d.ctr->n_dyn_rows, n_rows);
    if (n_hits) atomicAdd(&d.ctr->n_cache_hits, n_hits);
    if (n_new) atomicAdd(&d.ctr->n_new_contacts, n_new);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int np_ = d.ctr->n_pairs;
    d.ctr->n_dyn_rows_req = d.pair_rstart[np_];
  }
}

// Per-body dynamic incidence lists (group ids), then sorted ascending so the
// primal's summation order is reproducible.
__global__ void k_dg_fill(const __grid_constant__ Dev d) {
  int np = d.ctr->n_pairs;
  GSTRIDE(p, np) {
    int kept = d.pair_kept[p];
    if (kept == 0) continue;
    int2 ab = d.pair_ab[p];
    int g0 = d.n_sg + d.pair_gstart[p];
    int pa = d.dg_start[ab.x] + atomicAdd(&d.dg_cnt[ab.x], kept);
    int pb = d.dg_start[ab.y] + atomicAdd(&d.dg_cnt[ab.y], kept);
    // the groups' bodies are (ref, inc) (k_emit); ab.x is the first when it is the reference
    int a_second = ((d.pair_info[p] >> 9) & 1) ? 0 : 1;
    for (int c = 0; c < kept; ++c) {
      d.dg_idx[pa + c] = g0 + c;
      d.dg_idx[pb + c] = g0 + c;
      d.dg_other[pa + c] = 2 * ab.y + a_second;
      d.dg_other[pb + c] = 2 * ab.x + (1 - a_second);
    }
  }
}

__global__ void k_dg_zero(const __grid_constant__ Dev d) {
  GSTRIDE(i, d.nb) d.dg_cnt[i] = 0;
}

__global__ void k_dg_sort(const __grid_constant__ Dev d) {
  int mx = 0;  // longest list, reduced per warp after the loop
  constexpr int CAP = 32;  // lists up to this long are sorted in a local copy
  GSTRIDE(i, d.nb) {
    int s = d.dg_start[i], e = d.dg_start[i + 1];
    if (e - s <= CAP) {
      // (group, entry) packed into one key, group in the high word: group
      // indices are unique in a body's list, so this sorts by group.  One
      // pass of independent loads in, one pass of stores out.
      unsigned long long kv[CAP];
      const int n = e - s;
      for (int k = 0; k < n; ++k)
        kv[k] = ((unsigned long long)(unsigned)d.dg_idx[s + k] << 32) | (unsigned)d.dg_other[s + k];
      for (int a = 1; a < n; ++a) {
        unsigned long long v = kv[a];
        int b = a - 1;
        while (b >= 0 && kv[b] > v) {
          kv[b + 1] = kv[b];
          --b;
        }
        kv[b + 1] = v;
      }
      for (int k = 0; k < n; ++k) {
        d.dg_idx[s + k] = (int)(kv[k] >> 32);
        d.dg_other[s + k] = (int)(kv[k] & 0xffffffffull);
      }
      mx = max(mx, n);
      continue;
    }
    for (int a = s + 1; a < e; ++a) {
      int v = d.dg_idx[a], w = d.dg_other[a];
      int b = a - 1;
      while (b >= s && d.dg_idx[b] > v) {
        d.dg_idx[b + 1] = d.dg_idx[b];
        d.dg_other[b + 1] = d.dg_other[b];
        --b;
      }
      d.dg_idx[b + 1] = v;
      d.dg_other[b + 1] = w;
    }
    mx = max(mx, e - s);
  }
  mx = __reduce_max_sync(0xffffffffu, mx);
  if ((threadIdx.x & 31) == 0 && mx > 0) atomicMax(&d.ctr->max_dg, mx);
}

// Empties dynamic incidence lists when self collision is off (static-only scenes).
__global__ void k_dg_clear(const __grid_constant__ Dev d) {
  GSTRIDE(i, d.nb + 1) d.dg_start[i] = 0;
}

// ---------------------------------------------------------------------------
// Host-side launch sequence of the collision pipeline.
// ---------------------------------------------------------------------------
thread_local StageTimer* g_stage_timer = nullptr;

void launch_collision(Dev& d, const AvbdParams& P, const AvbdDims& dims, int grid, cudaStream_t st, bool rebuild) {
  stage_mark(st, "start");
  k_begin_substep<<<grid, 256, 0, st>>>(d);
  stage_mark(st, "k_begin_substep");
  bool collide = P.self_collide && d.nb >= 2;
  if (!collide) {
    k_dg_clear<<<grid, 256, 0, st>>>(d);
    stage_mark(st, "k_dg_clear");
    g_kernel_launches += 2;
    return;
  }
  k_aabb<<<grid, 256, 0, st>>>(d);
  stage_mark(st, "k_aabb");
  if (rebuild) {
    k_morton<<<grid, 256, 0, st>>>(d);
    stage_mark(st, "k_morton");
    radix_sort_launch(d, st);
    stage_mark(st, "radix_sort");
    k_lbvh_build<<<grid, 256, 0, st>>>(d);
    stage_mark(st, "k_lbvh_build");
  } else {
    k_lbvh_leaves<<<grid, 256, 0, st>>>(d);  // same topology, new leaf boxes
    stage_mark(st, "k_lbvh_leaves");
  }
  k_lbvh_refit<<<grid, 256, 0, st>>>(d);
  stage_mark(st, "k_lbvh_refit");
  k_lbvh_pack<<<grid, 256, 0, st>>>(d);
  stage_mark(st, "k_lbvh_pack");
  // One thread per body for the walks: a walk is a chain of dependent loads,
  // so a thread that walked twice would double the launch's duration.
  const int walk_grid = max(grid, (d.nb + 127) / 128);
  k_bp_count<<<walk_grid, 128, 0, st>>>(d);
  stage_mark(st, "k_bp_count");
  scan_launch(d, d.up_cnt, d.pair_start, d.nb, nullptr, nullptr, st);
  stage_mark(st, "scan_pair_offsets");
  k_bp_fill<<<walk_grid, 128, 0, st>>>(d);
  stage_mark(st, "k_bp_fill");
  k_narrow<<<grid, NARROW_BLOCK, 0, st>>>(d);
  stage_mark(st, "k_narrow");
  const int* npairs = &d.ctr->n_pairs;
  scan2_launch(d, d.pair_gcnt, d.pair_gstart, d.pair_kept, d.pair_rstart, d.pair_cap, npairs, st);
  stage_mark(st, "scan_contact_offsets");
  k_emit<<<2 * grid, 128, 0, st>>>(d, dims.dyn_row_cap, dims.dyn_group_cap);  // 8 blocks per SM
  stage_mark(st, "k_emit");
  scan_launch(d, d.dg_cnt, d.dg_start, d.nb, nullptr, nullptr, st);
  stage_mark(st, "scan_incidence_offsets");
  k_dg_zero<<<grid, 256, 0, st>>>(d);
  k_dg_fill<<<grid, 256, 0, st>>>(d);
  stage_mark(st, "k_dg_fill");
  k_dg_sort<<<grid, 128, 0, st>>>(d);
  stage_mark(st, "k_dg_sort");
  g_kernel_launches += rebuild ? 13 : 12;  // the direct launches above (scans and sort count themselves)
}

}  // namespace avbd
