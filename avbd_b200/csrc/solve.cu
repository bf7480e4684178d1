// Solve part of one substep on the GPU: recolor gate + Jones-Plassmann /
// speculative (jacobi) coloring, predict, prelude, the colored Gauss-Seidel
// primal (one warp sub-group per body), the dual update, BDF1 finalize,
// post-stabilization and the contact-cache refresh.
//
// Every phase is a __device__ function over a grid-stride index range.  The
// fast path runs all phases inside ONE cooperative (persistent) kernel with a
// bounded software grid barrier between them; the split path launches one
// small kernel per phase (same code) for debugging and as a fallback.
//
// Reference: solver_6dof.py:1232-1464 (substep), :1507-1679 (iteration loop),
// kernels_6dof.py:122-187 (predict), :322-582 + :1149-1414 (primal),
// :1451-1548 (dual), :1565-1672 (prelude), :1733-1811 (post-stab alpha*C0),
// :1871-1901 (finalize), :2915-2995 (cache refresh), :3022-3336 (coloring).
#include <cuda/atomic>

#include "common.cuh"
#include "kernels.cuh"

namespace avbd {

#define FINF __int_as_float(0x7f800000)

// ---------------------------------------------------------------------------
// Bounded grid barrier.  Co-residency is guaranteed by the cooperative
// launch; every wait gives up after prm->barrier_timeout_ns, sets
// ERR_BARRIER_TIMEOUT and the kernel returns.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool grid_barrier(const Dev& d, int idx) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    DevCounters* c = d.ctr;
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(c->bar_gen);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(c->bar_count);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(c->err);
    ok = 1;
    if (err.load(cuda::memory_order_relaxed) & ERR_BARRIER_TIMEOUT) {
      ok = 0;
    } else {
      unsigned g = gen.load(cuda::memory_order_acquire);
      __threadfence();
      bool skip = d.prm->debug_skip_arrive && blockIdx.x == 0 && idx == 0;
      bool last = false;
      if (!skip) {
        unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        if (arrived == gridDim.x - 1) {
          cnt.store(0u, cuda::memory_order_relaxed);
          gen.fetch_add(1u, cuda::memory_order_release);
          last = true;
        }
      }
      if (!last) {
        unsigned long long t0 = gtimer();
        unsigned long long budget = d.prm->barrier_timeout_ns;
        while (gen.load(cuda::memory_order_acquire) == g) {
          if (err.load(cuda::memory_order_relaxed) & ERR_BARRIER_TIMEOUT) {
            ok = 0;
            break;
          }
          if (gtimer() - t0 > budget) {
            err.fetch_or(ERR_BARRIER_TIMEOUT, cuda::memory_order_relaxed);
            atomicMax(&c->err_where, idx);
            ok = 0;
            break;
          }
          __nanosleep(40);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return ok != 0;
}

// ---------------------------------------------------------------------------
// Per-body 6x6 system accumulator (symmetric blocks A, D; full B; rhs).
// ---------------------------------------------------------------------------
struct Acc {
  float a[6];  // xx yy zz xy xz yz
  float b[9];  // row-major B = sum k ja jl^T
  float dd[6];
  float rl[3], ra[3];
};
__device__ __forceinline__ void acc_zero(Acc& s) {
#pragma unroll
  for (int k = 0; k < 6; ++k) s.a[k] = s.dd[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; ++k) s.b[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) s.rl[k] = s.ra[k] = 0.0f;
}
__device__ __forceinline__ float acc_get(const Acc& s, int k) {
  return k < 6 ? s.a[k] : (k < 15 ? s.b[k - 6] : (k < 21 ? s.dd[k - 15] : (k < 24 ? s.rl[k - 21] : s.ra[k - 24])));
}

// kernels_6dof.py:280-316 (column norms of the contact Hessian approximation).
__device__ __forceinline__ V3 geom_stiffness_diag(V3 n, V3 r) {
  float nr = dot(n, r);
  float h00 = n.x * r.x - nr, h10 = 0.5f * (n.y * r.x + r.y * n.x), h20 = 0.5f * (n.z * r.x + r.z * n.x);
  float h01 = 0.5f * (n.x * r.y + r.x * n.y), h11 = n.y * r.y - nr, h21 = 0.5f * (n.z * r.y + r.z * n.y);
  float h02 = 0.5f * (n.x * r.z + r.x * n.z), h12 = 0.5f * (n.y * r.z + r.y * n.z), h22 = n.z * r.z - nr;
  return V3{sqrtf(h00 * h00 + h10 * h10 + h20 * h20), sqrtf(h01 * h01 + h11 * h11 + h21 * h21),
            sqrtf(h02 * h02 + h12 * h12 + h22 * h22)};
}

// Force and Eq.14-rescaled stiffness of one row (kernels_6dof.py:1320-1348).
__device__ __forceinline__ void row_force(float C, bool hard, float ac0, float lam, float pen, float lo, float hi,
                                          float& f, float& kl) {
  if (hard) C = C - ac0;
  float le = hard ? lam : 0.0f;
  float lp = pen * C + le;
  f = fminf(fmaxf(lp, lo), hi);
  kl = pen;
  float aC = fabsf(C);
  if (aC > 1.0e-12f) {
    if (lp < lo) kl = fabsf(lo - lp) / aC;
    else if (lp > hi) kl = fabsf(hi - lp) / aC;
  }
}

// Row with a general Jacobian (jl, ja); n_g is the row direction for G~.
__device__ __forceinline__ void acc_row(Acc& s, V3 jl, V3 ja, V3 ng, V3 rs, float f, float kl) {
  s.a[0] += jl.x * jl.x * kl; s.a[1] += jl.y * jl.y * kl; s.a[2] += jl.z * jl.z * kl;
  s.a[3] += jl.x * jl.y * kl; s.a[4] += jl.x * jl.z * kl; s.a[5] += jl.y * jl.z * kl;
  s.b[0] += ja.x * jl.x * kl; s.b[1] += ja.x * jl.y * kl; s.b[2] += ja.x * jl.z * kl;
  s.b[3] += ja.y * jl.x * kl; s.b[4] += ja.y * jl.y * kl; s.b[5] += ja.y * jl.z * kl;
  s.b[6] += ja.z * jl.x * kl; s.b[7] += ja.z * jl.y * kl; s.b[8] += ja.z * jl.z * kl;
  s.dd[0] += ja.x * ja.x * kl; s.dd[1] += ja.y * ja.y * kl; s.dd[2] += ja.z * ja.z * kl;
  s.dd[3] += ja.x * ja.y * kl; s.dd[4] += ja.x * ja.z * kl; s.dd[5] += ja.y * ja.z * kl;
  float fm = fabsf(f);
  if (fm > 0.0f) {
    V3 g = geom_stiffness_diag(ng, rs);
    s.dd[0] += g.x * fm; s.dd[1] += g.y * fm; s.dd[2] += g.z * fm;
  }
  s.rl[0] += jl.x * f; s.rl[1] += jl.y * f; s.rl[2] += jl.z * f;
  s.ra[0] += ja.x * f; s.ra[1] += ja.y * f; s.ra[2] += ja.z * f;
}

// Row along world axis K (floor normal/tangents, pin axes): jl = e_K.
template <int K>
__device__ __forceinline__ void acc_axis(Acc& s, V3 rs, float f, float kl) {
  V3 ja = K == 0 ? V3{0.0f, rs.z, -rs.y} : (K == 1 ? V3{-rs.z, 0.0f, rs.x} : V3{rs.y, -rs.x, 0.0f});
  s.a[K] += kl;
  s.b[0 + K] += ja.x * kl; s.b[3 + K] += ja.y * kl; s.b[6 + K] += ja.z * kl;
  s.dd[0] += ja.x * ja.x * kl; s.dd[1] += ja.y * ja.y * kl; s.dd[2] += ja.z * ja.z * kl;
  s.dd[3] += ja.x * ja.y * kl; s.dd[4] += ja.x * ja.z * kl; s.dd[5] += ja.y * ja.z * kl;
  float fm = fabsf(f);
  if (fm > 0.0f) {
    V3 e = K == 0 ? V3{1.0f, 0.0f, 0.0f} : (K == 1 ? V3{0.0f, 1.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f});
    V3 g = geom_stiffness_diag(e, rs);
    s.dd[0] += g.x * fm; s.dd[1] += g.y * fm; s.dd[2] += g.z * fm;
  }
  s.rl[K] += f;
  s.ra[0] += ja.x * f; s.ra[1] += ja.y * f; s.ra[2] += ja.z * f;
}

// Contribution of group g to body i's system (rows in row order).
__device__ __forceinline__ void accumulate_group(const Dev& d, int g, int i, V3 xi, float4 qi, bool post, Acc& s) {
  int meta = d.g_meta[g];
  int fl = d.g_flags[g];
  int kind = meta_kind(meta);
  bool three = (meta & 4) != 0, hard = (meta & 8) != 0;
  float4 lam = d.g_lam[g], pen = d.g_pen[g], ac0 = d.g_ac0[g];
  if (post) {  // post-stabilization pass: alpha = 0 for non-friction rows (kernels_6dof.py:1733-1811)
    ac0.x = 0.0f;
    if (kind == KIND_PIN) { ac0.y = 0.0f; ac0.z = 0.0f; }
  }
  float f, kl;
  if (kind == KIND_FLOOR) {
    float4 oa = d.g_offa[g];
    V3 rs = qrot(qi, xyz(oa));
    if (fl & FL_ACT0) {
      row_force((xi.y + rs.y) - oa.w, hard, ac0.x, lam.x, pen.x, -FINF, 0.0f, f, kl);
      acc_axis<1>(s, rs, f, kl);
    }
    if (three) {
      float4 mat = d.g_mat[g];
      float bound = ((fl & FL_WAS) ? mat.y : mat.x) * fabsf(lam.x);
      if (fl & FL_ACT1) {
        row_force(xi.x + rs.x, hard, ac0.y, lam.y, pen.y, -bound, bound, f, kl);
        acc_axis<0>(s, rs, f, kl);
      }
      if (fl & FL_ACT2) {
        row_force(xi.z + rs.z, hard, ac0.z, lam.z, pen.z, -bound, bound, f, kl);
        acc_axis<2>(s, rs, f, kl);
      }
    }
  } else if (kind == KIND_PIN) {
    float4 oa = d.g_offa[g], an = d.g_n[g];
    V3 rs = qrot(qi, xyz(oa));
    V3 p = xi + rs;
    if (fl & FL_ACT0) { row_force(p.x - an.x, hard, ac0.x, lam.x, pen.x, -FINF, FINF, f, kl); acc_axis<0>(s, rs, f, kl); }
    if (fl & FL_ACT1) { row_force(p.y - an.y, hard, ac0.y, lam.y, pen.y, -FINF, FINF, f, kl); acc_axis<1>(s, rs, f, kl); }
    if (fl & FL_ACT2) { row_force(p.z - an.z, hard, ac0.z, lam.z, pen.z, -FINF, FINF, f, kl); acc_axis<2>(s, rs, f, kl); }
  } else {
    int2 bd = d.g_body[g];
    bool side_a = bd.x == i;
    int o = side_a ? bd.y : bd.x;
    float4 xo4 = d.x[o], qo = d.q[o];
    float4 oa = d.g_offa[g], ob = d.g_offb[g];
    V3 n = xyz(d.g_n[g]);
    V3 rs, dd;
    if (side_a) {
      rs = qrot(qi, xyz(oa));
      V3 ro = qrot(qo, xyz(ob));
      dd = (xi + rs) - (xyz(xo4) + ro);
    } else {
      V3 ro = qrot(qo, xyz(oa));
      rs = qrot(qi, xyz(ob));
      dd = (xyz(xo4) + ro) - (xi + rs);
    }
    float sg = side_a ? 1.0f : -1.0f;
    if (fl & FL_ACT0) {
      row_force(dot(n, dd), hard, ac0.x, lam.x, pen.x, -FINF, 0.0f, f, kl);
      acc_row(s, n * sg, cross(rs, n) * sg, n, rs, f, kl);
    }
    if (three) {
      float4 mat = d.g_mat[g];
      float bound = ((fl & FL_WAS) ? mat.y : mat.x) * fabsf(lam.x);
      V3 t = orthonormal_basis(n);
      V3 b = cross(n, t);
      if (fl & FL_ACT1) {
        row_force(dot(t, dd), hard, ac0.y, lam.y, pen.y, -bound, bound, f, kl);
        acc_row(s, t * sg, cross(rs, t) * sg, t, rs, f, kl);
      }
      if (fl & FL_ACT2) {
        row_force(dot(b, dd), hard, ac0.z, lam.z, pen.z, -bound, bound, f, kl);
        acc_row(s, b * sg, cross(rs, b) * sg, b, rs, f, kl);
      }
    }
  }
}

// 3x3 inverse by the adjugate (zero matrix when singular).
__device__ __forceinline__ void inv3(const float m[3][3], float r[3][3]) {
  float c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
  float c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  float c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  float det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
  if (det == 0.0f) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) r[a][b] = 0.0f;
    return;
  }
  float id = 1.0f / det;
  r[0][0] = c00 * id;
  r[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
  r[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
  r[1][0] = c01 * id;
  r[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
  r[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
  r[2][0] = c02 * id;
  r[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
  r[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
}

// Inertial terms + Schur-complement solve + pose update (kernels_6dof.py:1379-1414).
__device__ __forceinline__ void solve_body(const Dev& d, int i, float4 xi4, float4 qi, const Acc& s, float dt) {
  float m = xi4.w;
  float idt2 = 1.0f / (dt * dt);
  float mi = m * idt2;
  float4 w0 = d.iw0[i], w1 = d.iw1[i];  // (xx yy zz xy) (xz yz)
  float I[3][3] = {{w0.x, w0.w, w1.x}, {w0.w, w0.y, w1.y}, {w1.x, w1.y, w0.z}};
  float A[3][3] = {{s.a[0] + mi, s.a[3], s.a[4]}, {s.a[3], s.a[1] + mi, s.a[5]}, {s.a[4], s.a[5], s.a[2] + mi}};
  float D[3][3] = {{I[0][0] * idt2 + s.dd[0], I[0][1] * idt2 + s.dd[3], I[0][2] * idt2 + s.dd[4]},
                   {I[1][0] * idt2 + s.dd[3], I[1][1] * idt2 + s.dd[1], I[1][2] * idt2 + s.dd[5]},
                   {I[2][0] * idt2 + s.dd[4], I[2][1] * idt2 + s.dd[5], I[2][2] * idt2 + s.dd[2]}};
  float B[3][3] = {{s.b[0], s.b[1], s.b[2]}, {s.b[3], s.b[4], s.b[5]}, {s.b[6], s.b[7], s.b[8]}};
  float4 xin = d.xin[i], qin = d.qin[i];
  V3 rl = V3{(xi4.x - xin.x) * mi + s.rl[0], (xi4.y - xin.y) * mi + s.rl[1], (xi4.z - xin.z) * mi + s.rl[2]};
  V3 dth = quat_to_rotvec(qmul(qi, qconj(qin)));
  V3 th = dth * idt2;
  V3 ra = V3{I[0][0] * th.x + I[0][1] * th.y + I[0][2] * th.z + s.ra[0],
             I[1][0] * th.x + I[1][1] * th.y + I[1][2] * th.z + s.ra[1],
             I[2][0] * th.x + I[2][1] * th.y + I[2][2] * th.z + s.ra[2]};
  float Ai[3][3];
  inv3(A, Ai);
  float BA[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) BA[r][c] = B[r][0] * Ai[0][c] + B[r][1] * Ai[1][c] + B[r][2] * Ai[2][c];
  V3 rth = V3{ra.x - (BA[0][0] * rl.x + BA[0][1] * rl.y + BA[0][2] * rl.z),
              ra.y - (BA[1][0] * rl.x + BA[1][1] * rl.y + BA[1][2] * rl.z),
              ra.z - (BA[2][0] * rl.x + BA[2][1] * rl.y + BA[2][2] * rl.z)};
  float S[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) S[r][c] = D[r][c] - (BA[r][0] * B[c][0] + BA[r][1] * B[c][1] + BA[r][2] * B[c][2]);
  float Si[3][3];
  inv3(S, Si);
  V3 dt_ = V3{Si[0][0] * rth.x + Si[0][1] * rth.y + Si[0][2] * rth.z, Si[1][0] * rth.x + Si[1][1] * rth.y + Si[1][2] * rth.z,
              Si[2][0] * rth.x + Si[2][1] * rth.y + Si[2][2] * rth.z};
  V3 u = V3{rl.x - (B[0][0] * dt_.x + B[1][0] * dt_.y + B[2][0] * dt_.z),
            rl.y - (B[0][1] * dt_.x + B[1][1] * dt_.y + B[2][1] * dt_.z),
            rl.z - (B[0][2] * dt_.x + B[1][2] * dt_.y + B[2][2] * dt_.z)};
  V3 dx = V3{Ai[0][0] * u.x + Ai[0][1] * u.y + Ai[0][2] * u.z, Ai[1][0] * u.x + Ai[1][1] * u.y + Ai[1][2] * u.z,
             Ai[2][0] * u.x + Ai[2][1] * u.y + Ai[2][2] * u.z};
  float4 nx = make_float4(xi4.x - dx.x, xi4.y - dx.y, xi4.z - dx.z, m);
  float4 nq = qnormalize(qmul(quat_from_rotvec(-dt_), qi));
  if (!(isfinite(nx.x) && isfinite(nx.y) && isfinite(nx.z) && isfinite(nq.w))) atomicOr(&d.ctr->err, ERR_NONFINITE);
  d.x[i] = nx;
  d.q[i] = nq;
}

// Primal sweep of one color: G lanes per body, butterfly reduction of the
// 27 accumulators, lane 0 solves (kernels_6dof.py:1149-1414, in place).
template <int G>
__device__ void primal_color(const Dev& d, int c, bool post, float dt, int gtid, int gsize) {
  int cs0 = d.color_starts[c];
  int nbody = d.color_starts[c + 1] - cs0;
  int total = nbody * G;
  for (int base = 0; base < total; base += gsize) {
    int t = base + gtid;
    int slot = t / G, lane = t & (G - 1);
    bool valid = slot < nbody;
    int i = valid ? d.color_bodies[cs0 + slot] : 0;
    float4 xi4 = valid ? d.x[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool act = valid && xi4.w > 0.0f;
    Acc s;
    acc_zero(s);
    float4 qi = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    if (act) {
      qi = d.q[i];
      V3 xi = xyz(xi4);
      int s0 = d.sg_start[i], ns = d.sg_start[i + 1] - s0;
      int e0 = d.dg_start[i], nd = d.dg_start[i + 1] - e0;
      for (int k = lane; k < ns + nd; k += G) {
        int g = k < ns ? s0 + k : d.dg_idx[e0 + (k - ns)];
        accumulate_group(d, g, i, xi, qi, post, s);
      }
    }
    if (G > 1) {
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          s.a[k] += __shfl_xor_sync(0xffffffffu, s.a[k], o);
          s.dd[k] += __shfl_xor_sync(0xffffffffu, s.dd[k], o);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) s.b[k] += __shfl_xor_sync(0xffffffffu, s.b[k], o);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          s.rl[k] += __shfl_xor_sync(0xffffffffu, s.rl[k], o);
          s.ra[k] += __shfl_xor_sync(0xffffffffu, s.ra[k], o);
        }
      }
    }
    if (act && lane == 0) solve_body(d, i, xi4, qi, s, dt);
  }
}

__device__ void ph_primal(const Dev& d, int c, bool post, int gtid, int gsize) {
  float dt = d.prm->dt;
  switch (d.prm->group_size) {
    case 1: primal_color<1>(d, c, post, dt, gtid, gsize); break;
    case 2: primal_color<2>(d, c, post, dt, gtid, gsize); break;
    case 4: primal_color<4>(d, c, post, dt, gtid, gsize); break;
    case 8: primal_color<8>(d, c, post, dt, gtid, gsize); break;
    case 16: primal_color<16>(d, c, post, dt, gtid, gsize); break;
    default: primal_color<32>(d, c, post, dt, gtid, gsize); break;
  }
}

// ---------------------------------------------------------------------------
// Row values of a group at a pose (for prelude / dual).
// ---------------------------------------------------------------------------
struct GroupC {
  float c[3];
};
__device__ __forceinline__ GroupC group_values(const Dev& d, int g, int meta, const float4* X, const float4* Q) {
  GroupC r;
  int kind = meta_kind(meta);
  int2 bd = d.g_body[g];
  float4 oa = d.g_offa[g];
  float4 xa = X[bd.x], qa = Q[bd.x];
  V3 pa = xyz(xa) + qrot(qa, xyz(oa));
  if (kind == KIND_FLOOR) {
    r.c[0] = pa.y - oa.w;
    r.c[1] = pa.x;  // dot((1,0,0), x + R off)
    r.c[2] = pa.z;  // dot((0,0,1), x + R off)
  } else if (kind == KIND_PIN) {
    float4 an = d.g_n[g];
    r.c[0] = pa.x - an.x;
    r.c[1] = pa.y - an.y;
    r.c[2] = pa.z - an.z;
  } else {
    float4 ob = d.g_offb[g];
    V3 pb = xyz(X[bd.y]) + qrot(Q[bd.y], xyz(ob));
    V3 dd = pa - pb;
    V3 n = xyz(d.g_n[g]);
    r.c[0] = dot(n, dd);
    if (meta & 4) {
      V3 t = orthonormal_basis(n);
      V3 b = cross(n, t);
      r.c[1] = dot(t, dd);
      r.c[2] = dot(b, dd);
    } else {
      r.c[1] = r.c[2] = 0.0f;
    }
  }
  return r;
}

__device__ __forceinline__ int n_groups_live(const Dev& d) { return d.n_sg + d.ctr->n_dyn_groups; }

// Prelude (kernels_6dof.py:1565-1672), run BEFORE predict so x/q are the
// substep's initial pose.  Rows of a group in row order (Warp CPU order):
// the friction check of the first tangent sees the decayed normal and first
// tangent, and the second tangent's lambda before its own decay.
__device__ void ph_prelude(const Dev& d, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  int ng = n_groups_live(d);
  float main_alpha = P.post_stab ? 1.0f : P.alpha;
  for (int g = gtid; g < ng; g += gsize) {
    int meta = d.g_meta[g];
    int fl = d.g_flags[g];
    int kind = meta_kind(meta);
    bool three = (meta & 4) != 0;
    float4 lam = d.g_lam[g], pen = d.g_pen[g], mat = d.g_mat[g];
    float s = mat.z;
    bool tang = kind != KIND_PIN;  // rows 1, 2 of floor/box groups are friction rows
    float lm[3] = {lam.x, lam.y, lam.z}, pn[3] = {pen.x, pen.y, pen.z};
    int nr = three ? 3 : 1;
    for (int k = 0; k < nr; ++k) {
      float kf = (tang && k > 0) ? PEN_MIN_T : PEN_MIN;
      float p = fminf(fmaxf(pn[k] * P.gamma, kf), PEN_MAX);
      if (!P.post_stab) lm[k] = lm[k] * P.alpha * P.gamma;
      if (!isnan(s) && s < FINF) p = fminf(p, s);
      pn[k] = p;
      if (tang && k == 1 && (fl & FL_ACT1) && (fl & FL_ACT0)) {
        float ln = fabsf(lm[0]);
        if (ln < 1.0e-9f) fl &= ~FL_WAS;
        else {
          float lt = lm[1], lb = lm[2];  // lm[2] not decayed yet
          float ltb = sqrtf(lt * lt + lb * lb);
          if (ltb <= mat.y * ln) fl |= FL_WAS;
          else fl &= ~FL_WAS;
        }
      }
    }
    GroupC c0 = group_values(d, g, meta, d.x, d.q);
    float a[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < nr; ++k) {
      if (!(fl & (1 << k))) continue;
      float C0 = c0.c[k];
      if (tang && k > 0) a[k] = C0;
      else if (kind != KIND_PIN) a[k] = C0 > 0.0f ? 0.0f : main_alpha * C0;
      else a[k] = main_alpha * C0;
    }
    d.g_lam[g] = make_float4(lm[0], lm[1], lm[2], 0.0f);
    d.g_pen[g] = make_float4(pn[0], pn[1], pn[2], 0.0f);
    d.g_ac0[g] = make_float4(a[0], a[1], a[2], 0.0f);
    d.g_flags[g] = fl;
  }
}

// Dual update (kernels_6dof.py:1451-1548), rows of a group in row order.
// Optionally records the max constraint violation of this iteration.
__device__ void ph_dual(const Dev& d, int it, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  int ng = n_groups_live(d);
  float vmax = 0.0f;
  for (int g = gtid; g < ng; g += gsize) {
    int meta = d.g_meta[g];
    int fl = d.g_flags[g];
    if (!(fl & 7)) continue;
    int kind = meta_kind(meta);
    bool three = (meta & 4) != 0, hard = (meta & 8) != 0;
    float4 lam = d.g_lam[g], pen = d.g_pen[g], ac0 = d.g_ac0[g], mat = d.g_mat[g];
    GroupC cv = group_values(d, g, meta, d.x, d.q);
    float lm[3] = {lam.x, lam.y, lam.z}, pn[3] = {pen.x, pen.y, pen.z}, ac[3] = {ac0.x, ac0.y, ac0.z};
    bool tang = kind != KIND_PIN;
    int nr = three ? 3 : 1;
    for (int k = 0; k < nr; ++k) {
      if (!(fl & (1 << k))) continue;
      float Craw = cv.c[k];
      float C = hard ? Craw - ac[k] : Craw;
      float le = hard ? lm[k] : 0.0f;
      float lo, hi;
      bool is_t = tang && k > 0;
      bool used_static = false;
      if (is_t) {
        float mu = mat.x;
        if (fl & FL_WAS) { mu = mat.y; used_static = true; }
        float bound = mu * fabsf(lm[0]);
        lo = -bound;
        hi = bound;
      } else {
        lo = -FINF;
        hi = kind == KIND_PIN ? FINF : 0.0f;
        float v = kind == KIND_PIN ? fabsf(Craw) : fmaxf(0.0f, -Craw);
        vmax = fmaxf(vmax, v);
      }
      float nl = fminf(fmaxf(pn[k] * C + le, lo), hi);
      lm[k] = nl;
      if (fabsf(nl) >= mat.w) {
        fl &= ~(1 << k);
        lm[k] = 0.0f;
        pn[k] = 0.0f;
        continue;
      }
      if (nl > lo && nl < hi) {
        float up = fminf(PEN_MAX, mat.z);
        pn[k] = fminf(pn[k] + P.beta * fabsf(C), up);
      } else if (is_t && used_static) {
        fl &= ~FL_WAS;
      }
    }
    d.g_lam[g] = make_float4(lm[0], lm[1], lm[2], 0.0f);
    d.g_pen[g] = make_float4(pn[0], pn[1], pn[2], 0.0f);
    d.g_flags[g] = fl;
  }
  if (P.record_violation && it < 64) {
    for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if (lane_id() == 0 && vmax > 0.0f) atomicMax(&d.ctr->viol_bits[it], __float_as_uint(vmax));
  }
}

// Inertial target + warm start (kernels_6dof.py:122-187).
__device__ void ph_predict(const Dev& d, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  float dt = P.dt;
  for (int i = gtid; i < d.nb; i += gsize) {
    float4 x = d.x[i], q = d.q[i];
    float m = x.w;
    d.x0[i] = x;
    d.q0[i] = q;
    M3 R = qmat(q);
    float4 il = d.iloc[i];
    float I[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) I[a][b] = R.m[a][0] * il.x * R.m[b][0] + R.m[a][1] * il.y * R.m[b][1] + R.m[a][2] * il.z * R.m[b][2];
    d.iw0[i] = make_float4(I[0][0], I[1][1], I[2][2], I[0][1]);
    d.iw1[i] = make_float4(I[0][2], I[1][2], 0.0f, 0.0f);
    if (m <= 0.0f) {
      d.xin[i] = x;
      d.qin[i] = q;
      continue;
    }
    float4 v = d.v[i], w = d.w[i], pv = d.pv[i];
    V3 g = V3{P.gx, P.gy, P.gz};
    V3 gdt2 = g * (dt * dt);
    V3 xin = (xyz(x) + xyz(v) * dt) + gdt2;
    float4 dq = quat_from_rotvec(xyz(w) * dt);
    float4 qn = qmul(dq, q);
    d.xin[i] = make_float4(xin.x, xin.y, xin.z, m);
    d.qin[i] = qn;
    V3 acc = (xyz(v) - xyz(pv)) / dt;
    float gn = sqrtf(dot(g, g));
    float wgt = 0.0f;
    if (gn > 0.0f) {
      V3 gh = g / gn;
      wgt = fminf(fmaxf(dot(acc, gh) / gn, 0.0f), 1.0f);
    }
    V3 xw = (xyz(x) + xyz(v) * dt) + gdt2 * wgt;
    d.x[i] = make_float4(xw.x, xw.y, xw.z, m);
    d.q[i] = qn;
  }
}

// BDF1 velocities + caps (kernels_6dof.py:1871-1901).
__device__ void ph_finalize(const Dev& d, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  float dt = P.dt;
  for (int i = gtid; i < d.nb; i += gsize) {
    float4 v = d.v[i], w = d.w[i];
    d.pv[i] = v;
    d.pw[i] = w;
    float4 x = d.x[i];
    if (x.w > 0.0f) {
      float4 x0 = d.x0[i];
      V3 nv = V3{x.x - x0.x, x.y - x0.y, x.z - x0.z} / dt;
      V3 nw = quat_to_rotvec(qmul(d.q[i], qconj(d.q0[i]))) / dt;
      float sl = sqrtf(dot(nv, nv));
      if (sl > P.max_lin) nv = nv * (P.max_lin / sl);
      float sa = sqrtf(dot(nw, nw));
      if (sa > P.max_ang) nw = nw * (P.max_ang / sa);
      d.v[i] = make_float4(nv.x, nv.y, nv.z, 0.0f);
      d.w[i] = make_float4(nw.x, nw.y, nw.z, 0.0f);
    }
  }
}

// Contact-cache refresh (kernels_6dof.py:2923-2995) with an epoch tag in
// place of the full-table clear (kernels_6dof.py:2915-2920).
__device__ void ph_collect(const Dev& d, int gtid, int gsize) {
  int nd = d.ctr->n_dyn_groups;
  unsigned tag = epoch_tag(d.ctr->epoch + 1u);
  unsigned mask = (unsigned)d.hash_cap - 1u;
  for (int u = gtid; u < nd; u += gsize) {
    int g = d.n_sg + u;
    int fl = d.g_flags[g];
    if (!(fl & FL_ACT0)) continue;
    int meta = d.g_meta[g];
    int2 bd = d.g_body[g];
    int ka = min(bd.x, bd.y), kb = max(bd.x, bd.y);
    unsigned long long key = cache_key(ka, kb, meta_cidx(meta));
    unsigned long long want = key | ((unsigned long long)tag << 50);
    float4 lam = d.g_lam[g], pen = d.g_pen[g];
    float4 s0, s1;
    if (meta & 4) {
      s0 = make_float4(lam.x, lam.y, lam.z, pen.x);
      s1 = make_float4(pen.y, pen.z, (fl & FL_WAST) ? 1.0f : 0.0f, (fl & FL_WASB) ? 1.0f : 0.0f);
    } else {
      s0 = make_float4(lam.x, 0.0f, 0.0f, pen.x);
      s1 = make_float4(PEN_MIN_T, PEN_MIN_T, 0.0f, 0.0f);
    }
    unsigned h = (unsigned)mix64(key) & mask;
    bool done = false;
    for (int probe = 0; probe < 4096 && !done; ++probe) {
      unsigned sl = (h + probe) & mask;
      unsigned long long v = atomicAdd(&d.h_key[sl], 0ull);
      while (true) {
        if (v == want) {
          done = true;
          break;
        }
        if ((unsigned)(v >> 50) == tag) break;  // occupied this epoch: next slot
        unsigned long long old = atomicCAS(&d.h_key[sl], v, want);
        if (old == v) {
          done = true;
          break;
        }
        v = old;
      }
      if (done) {
        d.h_s0[sl] = s0;
        d.h_s1[sl] = s1;
      }
    }
    if (!done) atomicOr(&d.ctr->err, ERR_HASH_FULL);
  }
}

// ---------------------------------------------------------------------------
// Coloring (edge parallel; snapshot semantics: every round reads the colors
// of the previous round).  Edges are broadphase pairs that emitted contacts.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool beats(const Dev& d, int a, int b) {  // a has priority over b
  float pa = d.prio[a], pb = d.prio[b];
  return pa > pb || (pa == pb && a < b);
}

__device__ void ph_gate(const Dev& d, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  if (d.ctr->color_dirty || P.recolor_every) return;
  int np = d.ctr->n_pairs;
  int cnt = 0;
  for (int p = gtid; p < np; p += gsize) {
    if (d.pair_kept[p] == 0) continue;
    int2 ab = d.pair_ab[p];
    if (d.color[ab.x] == d.color[ab.y]) ++cnt;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane_id() == 0 && cnt) atomicAdd(&d.ctr->conflicts, cnt);
}

__device__ __forceinline__ bool recolor_needed(const Dev& d) {
  return d.ctr->color_dirty || d.prm->recolor_every || d.ctr->conflicts > 0;
}

__device__ void ph_color_reset(const Dev& d, int gtid, int gsize) {
  for (int i = gtid; i < d.nb; i += gsize) {
    d.color[i] = -1;
    d.c_used[i] = 0;
    d.c_lost[i] = 0;
  }
  if (gtid == 0) {
    d.ctr->uncolored = 0;
    d.ctr->recolored = 1;
  }
}

// Round step 1: collect used colors of colored neighbours; for JP mark the
// lower-priority end of every uncolored-uncolored edge as a loser.
__device__ void ph_round_edges(const Dev& d, bool jp, int gtid, int gsize) {
  int np = d.ctr->n_pairs;
  for (int p = gtid; p < np; p += gsize) {
    if (d.pair_kept[p] == 0) continue;
    int2 ab = d.pair_ab[p];
    int ca = d.color[ab.x], cb = d.color[ab.y];
    if (ca < 0 && cb < 0) {
      if (jp) atomicOr(&d.c_lost[beats(d, ab.x, ab.y) ? ab.y : ab.x], 1);
    } else if (ca < 0) {
      if (cb < MAX_COLORS) atomicOr(&d.c_used[ab.x], 1 << cb);
    } else if (cb < 0) {
      if (ca < MAX_COLORS) atomicOr(&d.c_used[ab.y], 1 << ca);
    }
  }
}

__device__ __forceinline__ int first_fit(int used) {
  unsigned free_ = ~(unsigned)used;
  return free_ ? (__ffs((int)free_) - 1) : MAX_COLORS - 1;
}

// Round step 2: winners (JP) / every uncolored body (jacobi) take the
// smallest free color.  JP counts the bodies still uncolored.
__device__ void ph_round_assign(const Dev& d, bool jp, int gtid, int gsize) {
  int unc = 0;
  for (int i = gtid; i < d.nb; i += gsize) {
    if (d.color[i] >= 0) continue;
    if (jp && d.c_lost[i]) {
      ++unc;
    } else {
      d.color[i] = first_fit(d.c_used[i]);
    }
    d.c_used[i] = 0;
    d.c_lost[i] = 0;
  }
  if (jp) {
    for (int o = 16; o > 0; o >>= 1) unc += __shfl_xor_sync(0xffffffffu, unc, o);
    if (lane_id() == 0 && unc) atomicAdd(&d.ctr->uncolored, unc);
  }
}

// Jacobi resolve (kernels_6dof.py:3265-3296): of two same-colored
// neighbours, the lower-priority one is uncolored again.
__device__ void ph_resolve_edges(const Dev& d, int gtid, int gsize) {
  int np = d.ctr->n_pairs;
  for (int p = gtid; p < np; p += gsize) {
    if (d.pair_kept[p] == 0) continue;
    int2 ab = d.pair_ab[p];
    int ca = d.color[ab.x];
    if (ca >= 0 && ca == d.color[ab.y]) atomicOr(&d.c_lost[beats(d, ab.x, ab.y) ? ab.y : ab.x], 1);
  }
}

__device__ void ph_resolve_apply(const Dev& d, int gtid, int gsize) {
  int unc = 0;
  for (int i = gtid; i < d.nb; i += gsize) {
    if (d.c_lost[i]) {
      d.color[i] = -1;
      d.c_lost[i] = 0;
    }
    if (d.color[i] < 0) ++unc;
  }
  for (int o = 16; o > 0; o >>= 1) unc += __shfl_xor_sync(0xffffffffu, unc, o);
  if (lane_id() == 0 && unc) atomicAdd(&d.ctr->uncolored, unc);
}

// Bucketing of bodies by color, stable by body index: NCH chunks.
#define NCH 64
__device__ void ph_bucket_count(const Dev& d) {
  __shared__ int h[MAX_COLORS];
  int cs = (d.nb + NCH - 1) / NCH;
  for (int b = blockIdx.x; b < NCH; b += gridDim.x) {
    if (threadIdx.x < MAX_COLORS) h[threadIdx.x] = 0;
    __syncthreads();
    int s0 = b * cs, s1 = min(d.nb, s0 + cs);
    for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
      int c = d.color[i];
      if (c < 0) {  // stragglers take color 0 (kernels_6dof.py:3151-3165)
        c = 0;
        d.color[i] = 0;
      }
      atomicAdd(&h[c], 1);
    }
    __syncthreads();
    if (threadIdx.x < MAX_COLORS) d.c_hist[b * MAX_COLORS + threadIdx.x] = h[threadIdx.x];
    __syncthreads();
  }
}

__device__ void ph_bucket_scan(const Dev& d) {
  if (blockIdx.x != 0) return;
  __shared__ int tot[MAX_COLORS];
  int c = threadIdx.x;
  if (c < MAX_COLORS) {
    int run = 0;
    for (int b = 0; b < NCH; ++b) {
      int v = d.c_hist[b * MAX_COLORS + c];
      d.c_hist[b * MAX_COLORS + c] = run;
      run += v;
    }
    tot[c] = run;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0, mx = 0;
    for (int k = 0; k < MAX_COLORS; ++k) {
      d.color_starts[k] = acc;
      acc += tot[k];
      if (tot[k] > 0) mx = k;
    }
    d.color_starts[MAX_COLORS] = acc;
    d.ctr->n_colors = max(1, min(mx + 1, MAX_COLORS));
    d.ctr->color_dirty = 0;
  }
}

__device__ void ph_bucket_place(const Dev& d) {
  __shared__ int run[MAX_COLORS];
  __shared__ int wc[32][MAX_COLORS];
  int cs = (d.nb + NCH - 1) / NCH;
  int w = threadIdx.x >> 5, l = lane_id();
  int nw = blockDim.x >> 5;
  for (int b = blockIdx.x; b < NCH; b += gridDim.x) {
    if (threadIdx.x < MAX_COLORS) run[threadIdx.x] = d.color_starts[threadIdx.x] + d.c_hist[b * MAX_COLORS + threadIdx.x];
    int s0 = b * cs, s1 = min(d.nb, s0 + cs);
    for (int base = s0; base < s1; base += blockDim.x) {
      for (int k = threadIdx.x; k < 32 * MAX_COLORS; k += blockDim.x) (&wc[0][0])[k] = 0;
      __syncthreads();
      int i = base + threadIdx.x;
      bool valid = i < s1;
      int c = valid ? d.color[i] : MAX_COLORS + l;
      unsigned peers = __match_any_sync(0xffffffffu, c);
      int rank = __popc(peers & ((1u << l) - 1u));
      if (valid && rank == 0) wc[w][c] = __popc(peers);
      __syncthreads();
      if (valid) {
        int off = run[c];
        for (int u = 0; u < w; ++u) off += wc[u][c];
        d.color_bodies[off + rank] = i;
      }
      __syncthreads();
      if (threadIdx.x < MAX_COLORS) {
        int t = 0;
        for (int u = 0; u < nw; ++u) t += wc[u][threadIdx.x];
        run[threadIdx.x] += t;
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// The persistent substep kernel.
// ---------------------------------------------------------------------------
#define SOLVE_BLOCK 256

__global__ void __launch_bounds__(SOLVE_BLOCK, 1) k_solve_persistent(Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  int gsize = gridDim.x * blockDim.x;
  int bar = 0;
#define SYNC()                               \
  do {                                       \
    if (!grid_barrier(d, bar++)) return;     \
  } while (0)
  const DevParams& P = *d.prm;
  ph_gate(d, gtid, gsize);
  ph_prelude(d, gtid, gsize);  // reads x/q = the initial pose; predict runs after
  SYNC();
  if (recolor_needed(d)) {
    bool jp = P.color_mode == 1;
    ph_color_reset(d, gtid, gsize);
    SYNC();
    int rounds = jp ? JP_ROUNDS : MAX_COLORS;
    for (int r = 0; r < rounds; ++r) {
      ph_round_edges(d, jp, gtid, gsize);
      SYNC();
      ph_round_assign(d, jp, gtid, gsize);
      SYNC();
      if (!jp) {
        ph_resolve_edges(d, gtid, gsize);
        SYNC();
        ph_resolve_apply(d, gtid, gsize);
        SYNC();
      }
      int unc = *(volatile int*)&d.ctr->uncolored;
      SYNC();  // everyone has read the count before it is reset
      if (unc == 0) break;
      if (gtid == 0) d.ctr->uncolored = 0;
    }
    ph_bucket_count(d);
    SYNC();
    ph_bucket_scan(d);
    SYNC();
    ph_bucket_place(d);
  } else if (gtid == 0) {
    d.ctr->recolored = 0;
  }
  ph_predict(d, gtid, gsize);
  SYNC();
  int iters = P.iterations;
  int total = iters + (P.post_stab ? 1 : 0);
  int nc = *(volatile int*)&d.ctr->n_colors;
  for (int it = 0; it < total; ++it) {
    bool post = P.post_stab && it == iters;
    for (int c = 0; c < nc; ++c) {
      ph_primal(d, c, post, gtid, gsize);
      SYNC();
    }
    if (it < iters) {
      ph_dual(d, it, gtid, gsize);
      if (it == iters - 1) ph_finalize(d, gtid, gsize);
      SYNC();
    }
  }
  ph_collect(d, gtid, gsize);
  SYNC();
  if (gtid == 0) {
    d.ctr->epoch += 1u;
    d.ctr->n_viol = P.record_violation ? min(iters, 64) : 0;
  }
#undef SYNC
}

// ---------------------------------------------------------------------------
// Split path: one launch per phase, same phase functions.
// ---------------------------------------------------------------------------
#define GS int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x
__global__ void ks_gate_prelude(Dev d) { GS; ph_gate(d, gtid, gsize); ph_prelude(d, gtid, gsize); }
__global__ void ks_color_reset(Dev d) {
  GS;
  if (!recolor_needed(d)) {
    if (gtid == 0) d.ctr->recolored = 0;
    return;
  }
  ph_color_reset(d, gtid, gsize);
}
__global__ void ks_round_edges(Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0) return;
  ph_round_edges(d, d.prm->color_mode == 1, gtid, gsize);
}
__global__ void ks_round_assign(Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0) return;
  ph_round_assign(d, d.prm->color_mode == 1, gtid, gsize);
}
__global__ void ks_resolve_edges(Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0 || d.prm->color_mode == 1) return;
  ph_resolve_edges(d, gtid, gsize);
}
__global__ void ks_resolve_apply(Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0 || d.prm->color_mode == 1) return;
  ph_resolve_apply(d, gtid, gsize);
}
// After a round: uncolored == 0 -> mark done (-1), else reset the count.
__global__ void ks_round_end(Dev d) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && d.ctr->recolored && d.ctr->uncolored >= 0)
    d.ctr->uncolored = d.ctr->uncolored == 0 ? -1 : 0;
}
__global__ void ks_bucket_count(Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_count(d);
}
__global__ void ks_bucket_scan(Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_scan(d);
}
__global__ void ks_bucket_place(Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_place(d);
}
__global__ void ks_predict(Dev d) { GS; ph_predict(d, gtid, gsize); }
__global__ void ks_primal(Dev d, int it, int c) {
  GS;
  if (c >= d.ctr->n_colors) return;
  bool post = d.prm->post_stab && it == d.prm->iterations;
  ph_primal(d, c, post, gtid, gsize);
}
__global__ void ks_dual(Dev d, int it) {
  GS;
  int iters = d.prm->iterations;
  if (it < iters) {
    ph_dual(d, it, gtid, gsize);
    if (it == iters - 1) ph_finalize(d, gtid, gsize);
  }
}
__global__ void ks_collect(Dev d) { GS; ph_collect(d, gtid, gsize); }
__global__ void ks_end(Dev d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    d.ctr->epoch += 1u;
    d.ctr->n_viol = d.prm->record_violation ? min(d.prm->iterations, 64) : 0;
  }
}
#undef GS

int solve_occupancy(int block) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solve_persistent, block, 0);
  return n;
}

cudaError_t launch_solve(Dev& d, const AvbdParams& P, int persistent, int grid, int block, cudaStream_t st) {
  if (persistent) {
    void* args[] = {(void*)&d};
    g_kernel_launches += 1;
    return cudaLaunchCooperativeKernel((const void*)k_solve_persistent, dim3(grid), dim3(block), args, 0, st);
  }
  ks_gate_prelude<<<grid, block, 0, st>>>(d);
  ks_color_reset<<<grid, block, 0, st>>>(d);
  int rounds = P.coloring_mode == 1 ? JP_ROUNDS : MAX_COLORS;
  for (int r = 0; r < rounds; ++r) {
    ks_round_edges<<<grid, block, 0, st>>>(d);
    ks_round_assign<<<grid, block, 0, st>>>(d);
    ks_resolve_edges<<<grid, block, 0, st>>>(d);
    ks_resolve_apply<<<grid, block, 0, st>>>(d);
    ks_round_end<<<1, 32, 0, st>>>(d);
  }
  ks_bucket_count<<<NCH, block, 0, st>>>(d);
  ks_bucket_scan<<<1, block, 0, st>>>(d);
  ks_bucket_place<<<NCH, block, 0, st>>>(d);
  ks_predict<<<grid, block, 0, st>>>(d);
  int total = P.iterations + (P.post_stabilize ? 1 : 0);
  for (int it = 0; it < total; ++it) {
    for (int c = 0; c < MAX_COLORS; ++c) ks_primal<<<grid, block, 0, st>>>(d, it, c);
    ks_dual<<<grid, block, 0, st>>>(d, it);
  }
  ks_collect<<<grid, block, 0, st>>>(d);
  ks_end<<<1, 32, 0, st>>>(d);
  g_kernel_launches += 2 + 5 * rounds + 3 + 1 + total * (MAX_COLORS + 1) + 2;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// State reset, diagnostics, cache scrub.
// ---------------------------------------------------------------------------
__global__ void k_reset(Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  for (int i = gtid; i < d.nb; i += gsize) d.color[i] = -1;
  for (int s = gtid; s < d.hash_cap; s += gsize) d.h_key[s] = 0ull;
  if (gtid == 0) {
    DevCounters* c = d.ctr;
    c->err = 0;
    c->err_where = 0;
    c->epoch = 0;
    c->color_dirty = 1;
    c->n_colors = MAX_COLORS;
    c->recolored = 0;
    c->bar_count = 0;
    for (int k = 0; k < 64; ++k) c->viol_bits[k] = 0;
  }
}
void launch_reset(Dev& d, cudaStream_t st) { k_reset<<<148 * 4, 256, 0, st>>>(d); }

__global__ void k_conflicts(Dev d, int* out) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  int np = d.ctr->n_pairs;
  for (int p = gtid; p < np; p += gsize) {
    if (d.pair_kept[p] == 0) continue;
    int2 ab = d.pair_ab[p];
    if (d.color[ab.x] == d.color[ab.y]) atomicAdd(out, 1);
  }
}
int count_conflicts(Dev& d, cudaStream_t st) {
  int* dv = &d.ctr->pad[0];
  cudaMemsetAsync(dv, 0, sizeof(int), st);
  k_conflicts<<<148 * 2, 256, 0, st>>>(d, dv);
  int h = 0;
  cudaMemcpyAsync(&h, dv, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return h;
}

// Zero every cache slot whose tag is not the current one (keeps the live
// entries), so tags can wrap without a stale hit.
__global__ void k_hash_scrub(Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  unsigned tag = epoch_tag(d.ctr->epoch);
  for (int s = gtid; s < d.hash_cap; s += gsize) {
    unsigned long long v = d.h_key[s];
    if ((unsigned)(v >> 50) != tag) d.h_key[s] = 0ull;
  }
}
void launch_hash_scrub(Dev& d, cudaStream_t st) { k_hash_scrub<<<148 * 4, 256, 0, st>>>(d); }

// Host-provided cache contents, tagged with the current epoch so the next
// emission finds them.
__global__ void k_cache_clear(Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  for (int s = gtid; s < d.hash_cap; s += gsize) d.h_key[s] = 0ull;
}
__global__ void k_cache_insert(Dev d, int n, const int* abc, const float* st) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  unsigned tag = epoch_tag(d.ctr->epoch);
  unsigned mask = (unsigned)d.hash_cap - 1u;
  for (int k = gtid; k < n; k += gsize) {
    unsigned long long key = cache_key(abc[3 * k], abc[3 * k + 1], abc[3 * k + 2]);
    unsigned long long want = key | ((unsigned long long)tag << 50);
    unsigned h = (unsigned)mix64(key) & mask;
    bool done = false;
    for (int probe = 0; probe < 4096 && !done; ++probe) {
      unsigned sl = (h + probe) & mask;
      unsigned long long old = atomicCAS(&d.h_key[sl], 0ull, want);
      if (old == 0ull || old == want) {
        const float* s = st + 8 * k;
        d.h_s0[sl] = make_float4(s[0], s[1], s[2], s[3]);
        d.h_s1[sl] = make_float4(s[4], s[5], s[6], s[7]);
        done = true;
      }
    }
    if (!done) atomicOr(&d.ctr->err, ERR_HASH_FULL);
  }
}
void launch_cache_load(Dev& d, int n, const int* abc, const float* st, cudaStream_t s) {
  k_cache_clear<<<148 * 4, 256, 0, s>>>(d);
  if (n > 0) k_cache_insert<<<148 * 2, 256, 0, s>>>(d, n, abc, st);
}

}  // namespace avbd
