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
#include "mlp.cuh"

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

// ---------------------------------------------------------------------------
// Flag-ordered sweep primitives.  done[i] counts the color passes body i has
// finished in this substep.  A finished body publishes with a release store
// after its writes are fenced; a waiter polls with acquire loads, bounded by
// prm->barrier_timeout_ns (then ERR_BARRIER_TIMEOUT is set and every wait of
// the launch returns at once, so the kernel ends).
// ---------------------------------------------------------------------------
template <bool F, class T>
__device__ __forceinline__ T ldm(const T* p) {
  if constexpr (F) return __ldcg(p);  // written by another SM this substep: read through L2
  else return *p;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __noinline__ void wait_done_slow(const Dev& d, int o, int need) {
  unsigned long long t0 = gtimer();
  unsigned long long budget = d.prm->barrier_timeout_ns;
  for (unsigned spins = 1;; ++spins) {
    if (ld_acquire(d.done + o) >= need) return;
    if ((spins & 31u) == 0u) {
      if (*(volatile int*)&d.ctr->err & ERR_BARRIER_TIMEOUT) return;
      if (gtimer() - t0 > budget) {
        atomicOr(&d.ctr->err, ERR_BARRIER_TIMEOUT);
        return;
      }
    }
    __nanosleep(64);
  }
}

__device__ __forceinline__ void wait_done(const Dev& d, int o, int need) {
  if (ld_acquire(d.done + o) < need) wait_done_slow(d, o, need);
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
        // Two-level arrival: BAR_SUB sub-counters keep the serialized atomics
        // per address at about gridDim / BAR_SUB.
        unsigned nblk = gridDim.x;
        unsigned nsub = nblk < BAR_SUB ? nblk : BAR_SUB;
        unsigned sub = blockIdx.x % nsub;
        unsigned members = nblk / nsub + (sub < nblk % nsub ? 1u : 0u);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> sc(c->bar_sub[sub][0]);
        unsigned a_sub = sc.fetch_add(1u, cuda::memory_order_acq_rel);
        if (a_sub == members - 1) {
          sc.store(0u, cuda::memory_order_relaxed);
          unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
          if (arrived == nsub - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
            last = true;
          }
        }
      }
      if (!last) {
        // Poll the generation word; the timer and the abort flag are checked
        // every 64 polls so a healthy wait costs one L2 round trip per poll.
        unsigned long long t0 = gtimer();
        unsigned long long budget = d.prm->barrier_timeout_ns;
        unsigned spins = 0;
        while (gen.load(cuda::memory_order_acquire) == g) {
          if ((++spins & 63u) == 0u) {
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
          }
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

// Dual update of one group's rows in row order (kernels_6dof.py:1451-1548):
// a friction row sees its normal row's new lambda and was_static flag.
// Craw are the rows' constraint values at the current pose; ac the stored
// alpha*C0.  Returns the largest violation of the non-friction rows, measured
// on the value the update drives (C - alpha*C0 for hard rows).
__device__ __forceinline__ float dual_rows(int kind, int nr, bool hard, float4 mat, const float* Craw, const float* ac,
                                           float beta, float* lm, float* pn, int& fl) {
  bool tang = kind != KIND_PIN;
  float vmax = 0.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k >= nr || !(fl & (1 << k))) continue;
    float C = hard ? Craw[k] - ac[k] : Craw[k];
    float le = hard ? lm[k] : 0.0f;
    float lo, hi;
    bool is_t = tang && k > 0;
    bool used_static = false;
    if (is_t) {
      float mu = mat.x;
      if (fl & FL_WAS) {
        mu = mat.y;
        used_static = true;
      }
      float bound = mu * fabsf(lm[0]);
      lo = -bound;
      hi = bound;
    } else {
      lo = -FINF;
      hi = kind == KIND_PIN ? FINF : 0.0f;
      vmax = fmaxf(vmax, kind == KIND_PIN ? fabsf(C) : fmaxf(0.0f, -C));
    }
    float nl = fminf(fmaxf(pn[k] * C + le, lo), hi);
    lm[k] = nl;
    if (fabsf(nl) >= mat.w) {  // fracture
      fl &= ~(1 << k);
      lm[k] = 0.0f;
      pn[k] = 0.0f;
      continue;
    }
    if (nl > lo && nl < hi) {
      pn[k] = fminf(pn[k] + beta * fabsf(C), fminf(PEN_MAX, mat.z));
    } else if (is_t && used_static) {
      fl &= ~FL_WAS;  // static -> dynamic friction (AVBD sec. 3.3)
    }
  }
  return vmax;
}

// The plain start as fallback when a learned start raised the residual.  At
// the contact's first dual update (iteration 0) the normal row's opening
// ce = C - alpha*C0 times its penalty k estimates how far the predicted
// force lambda_p overshoots the force the contact needs (k ce ~ lambda_p -
// lambda*).  The zero start's error is |lambda*|, so the prediction is worse
// than no prediction when k ce > |lambda_p| / 2; such a start is dropped and
// the group continues from lambda = 0 and the minimum penalties, as a new
// contact of the reference would.  Clears FL_LRN either way.
__device__ __forceinline__ void learned_check(const Dev& d, int kind, bool hard, const float* C, const float* ac,
                                              float* lm, float* pn, int& fl) {
  fl &= ~FL_LRN;
  float ce = hard ? C[0] - ac[0] : C[0];
  if (kind == KIND_BOX && lm[0] < 0.0f && ce * pn[0] > 0.5f * fabsf(lm[0])) {
    lm[0] = lm[1] = lm[2] = 0.0f;
    pn[0] = PEN_MIN;
    pn[1] = pn[2] = PEN_MIN_T;
    fl = (fl & ~FL_WAS) | FL_REV;  // counted by the cache refresh
  }
}

// A copy the compiler cannot see through: known group values enter the row
// code as runtime values, so they take the same instructions (and the same
// FMA contractions) as values read from memory.
__device__ __forceinline__ float opaque(float v) {
  float r;
  asm("mov.b32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ int opaque(int v) {
  int r;
  asm("mov.b32 %0, %1;" : "=r"(r) : "r"(v));
  return r;
}
__device__ __forceinline__ float4 opaque4(float x, float y, float z, float w) {
  return make_float4(opaque(x), opaque(y), opaque(z), opaque(w));
}
// g_meta of implicit floor corner c of a hard three-row floor block.
__device__ __forceinline__ int resting_corner_meta(int c) {
  return make_meta(KIND_FLOOR, 1, 1, 0) | META_IMPLICIT | (c << 6);
}

// Group g's contribution to body i's system, rows in row order.  When
// `dual` is set and body i owns g (the group's dynamic body with the lower
// color), the previous iteration's dual update of g is applied first: both
// bodies still hold their poses from the end of that iteration, because the
// owner's color runs before the other body's.  Returns the violation of the
// updated rows (0 when no dual ran); a box-box group's violation is also
// added to csum / ccnt (the contact-row statistics of record_violation).
//
// F (flag-ordered sweep): before a box-box group's state and the other
// body's pose are read, wait until the other body has finished the pass this
// one needs -- pass it+1 when it owns the group (lower color, already updated
// in this pass), pass it otherwise -- and read everything another SM may
// have written in this substep through L2 (__ldcg), never through L1.
//
// oe: for a box-box group, its incidence entry of body i (dg_other: 2 * the
// other body + whether i is the group's second body), so the other body is
// known without reading the group's body pair; -1 reads the pair.
//
// corner >= 0: g is floor corner `corner` of a body whose corners are in the
// resting start state (fsep: floor height fy).  While the corner stays above
// the floor its stored state is known -- rows active, multipliers 0,
// penalties (PEN_MIN, PEN_MIN_T, PEN_MIN_T), no alpha offset -- and its dual
// update leaves that state as it is (the normal multiplier clamps to 0 with
// the penalty unchanged; the friction bounds are then 0, so the friction
// multipliers clamp to 0 and their stiffness |lambda - k C| / |C| is exactly
// k = 1), so the group is neither read nor written: the known values go
// through the same row code as read ones.  A corner at or below the floor is
// read as usual; if its dual update writes it, *wrote is set.  Barrier sweep
// only: in the flag sweep a lane's floor corner is evaluated while the index
// of its next (box-box) group is in flight, so reading the corner costs no
// time there, and the extra live values made the flag sweep spill (measured
// 9 % slower).
template <bool F>
__device__ __forceinline__ float accumulate_group(const Dev& d, int g, int i, V3 xi, float4 qi, bool post, bool dual,
                                                  Acc& s, float& csum, int& ccnt, int it = 0, int ci = 0,
                                                  int oe = -1, int corner = -1, float fy = 0.0f,
                                                  bool* wrote = nullptr) {
  bool rest = false;
  if (!F && corner >= 0) {
    float4 oa = implicit_corner(d.he[i], resting_corner_meta(corner), fy);
    V3 rs = qrot(qi, xyz(oa));
    rest = (xi.y + rs.y) - oa.w > 0.0f;
  }
  int meta = rest ? resting_corner_meta(corner) : d.g_meta[g];
  int fl = rest ? opaque(7) : ldm<F>(d.g_flags + g);
  int kind = meta_kind(meta);
  bool three = (meta & 4) != 0, hard = (meta & 8) != 0;
  int nr = three ? 3 : 1;
  int o = -1;
  bool side_b = false;
  if (kind == KIND_BOX) {
    if (oe >= 0) {
      o = oe >> 1;
      side_b = (oe & 1) != 0;
    } else {
      int2 bd = d.g_body[g];
      side_b = bd.x != i;
      o = side_b ? bd.x : bd.y;
    }
  }
  if (F && kind == KIND_BOX) {
    // A neighbour of the same color (a coloring that kept a conflict) runs
    // concurrently, as in the barrier sweep; waiting there could deadlock.
    if (d.color[o] != ci) {
      bool own_b = (fl & FL_OWNB) != 0;  // set before the passes; stable during them
      bool i_owns = own_b == side_b;
      wait_done(d, o, i_owns ? it : it + 1);
      fl = ldm<F>(d.g_flags + g);  // after the owner's dual update of this pass
    }
  }
  float4 lam, pen, ac0, mat;
  if (rest) {
    lam = opaque4(0.0f, 0.0f, 0.0f, 0.0f);
    pen = opaque4(PEN_MIN, PEN_MIN_T, PEN_MIN_T, 0.0f);
    ac0 = opaque4(0.0f, 0.0f, 0.0f, 0.0f);
    mat = opaque4(0.0f, 0.0f, FINF, fy);  // friction coefficients only scale a zero bound
  } else {
    lam = ldm<F>(d.g_lam + g);
    pen = ldm<F>(d.g_pen + g);
    ac0 = d.g_ac0[g];
    mat = d.g_mat[g];
  }
  float lm[3] = {lam.x, lam.y, lam.z}, pn[3] = {pen.x, pen.y, pen.z}, ac[3] = {ac0.x, ac0.y, ac0.z};
  float C[3] = {0.0f, 0.0f, 0.0f};
  V3 rs, dirs[3], dd;
  float sg = 1.0f;
  bool own = true;
  if (kind == KIND_FLOOR) {
    float4 oa;
    if (meta_implicit(meta)) {
      oa = implicit_corner(d.he[i], meta, mat.w);
      mat.w = FINF;  // no fracture on floor rows
    } else {
      oa = d.g_offa[g];
    }
    rs = qrot(qi, xyz(oa));
    C[0] = (xi.y + rs.y) - oa.w;
    C[1] = xi.x + rs.x;  // dot((1,0,0), x + R off)
    C[2] = xi.z + rs.z;  // dot((0,0,1), x + R off)
  } else if (kind == KIND_PIN) {
    float4 oa = d.g_offa[g], an = d.g_n[g];
    rs = qrot(qi, xyz(oa));
    V3 p = xi + rs;
    C[0] = p.x - an.x;
    C[1] = p.y - an.y;
    C[2] = p.z - an.z;
  } else {
    bool side_a = !side_b;
    own = ((fl & FL_OWNB) != 0) == !side_a;
    float4 xo4 = ldm<F>(d.x + o), qo = ldm<F>(d.q + o);
    float4 oa = d.g_offa[g], ob = d.g_offb[g];
    V3 n = xyz(d.g_n[g]);
    if (side_a) {
      rs = qrot(qi, xyz(oa));
      V3 ro = qrot(qo, xyz(ob));
      dd = (xi + rs) - (xyz(xo4) + ro);
    } else {
      V3 ro = qrot(qo, xyz(oa));
      rs = qrot(qi, xyz(ob));
      dd = (xyz(xo4) + ro) - (xi + rs);
    }
    sg = side_a ? 1.0f : -1.0f;
    dirs[0] = n;
    C[0] = dot(n, dd);
    if (three) {
      dirs[1] = orthonormal_basis(n);
      dirs[2] = cross(n, dirs[1]);
      C[1] = dot(dirs[1], dd);
      C[2] = dot(dirs[2], dd);
    }
  }
  float viol = 0.0f;
  if (dual && own) {
    if (fl & FL_LRN) learned_check(d, kind, hard, C, ac, lm, pn, fl);
    viol = dual_rows(kind, nr, hard, mat, C, ac, d.prm->beta, lm, pn, fl);
    if (!rest) {
      d.g_lam[g] = make_float4(lm[0], lm[1], lm[2], 0.0f);
      d.g_pen[g] = make_float4(pn[0], pn[1], pn[2], 0.0f);
      d.g_flags[g] = fl;
      if (!F && corner >= 0) *wrote = true;
    }
    if (kind == KIND_BOX && (fl & FL_ACT0)) {
      csum = fmaxf(csum, viol);
      ++ccnt;
    }
  }
  if (post) {  // post-stabilization pass: alpha = 0 for non-friction rows (kernels_6dof.py:1733-1811)
    ac[0] = 0.0f;
    if (kind == KIND_PIN) ac[1] = ac[2] = 0.0f;
  }
  float f, kl;
  if (kind == KIND_FLOOR) {
    if (fl & FL_ACT0) {
      row_force(C[0], hard, ac[0], lm[0], pn[0], -FINF, 0.0f, f, kl);
      acc_axis<1>(s, rs, f, kl);
    }
    if (three) {
      float bound = ((fl & FL_WAS) ? mat.y : mat.x) * fabsf(lm[0]);
      if (fl & FL_ACT1) {
        row_force(C[1], hard, ac[1], lm[1], pn[1], -bound, bound, f, kl);
        acc_axis<0>(s, rs, f, kl);
      }
      if (fl & FL_ACT2) {
        row_force(C[2], hard, ac[2], lm[2], pn[2], -bound, bound, f, kl);
        acc_axis<2>(s, rs, f, kl);
      }
    }
  } else if (kind == KIND_PIN) {
    if (fl & FL_ACT0) { row_force(C[0], hard, ac[0], lm[0], pn[0], -FINF, FINF, f, kl); acc_axis<0>(s, rs, f, kl); }
    if (fl & FL_ACT1) { row_force(C[1], hard, ac[1], lm[1], pn[1], -FINF, FINF, f, kl); acc_axis<1>(s, rs, f, kl); }
    if (fl & FL_ACT2) { row_force(C[2], hard, ac[2], lm[2], pn[2], -FINF, FINF, f, kl); acc_axis<2>(s, rs, f, kl); }
  } else {
    if (fl & FL_ACT0) {
      row_force(C[0], hard, ac[0], lm[0], pn[0], -FINF, 0.0f, f, kl);
      acc_row(s, dirs[0] * sg, cross(rs, dirs[0]) * sg, dirs[0], rs, f, kl);
    }
    if (three) {
      float bound = ((fl & FL_WAS) ? mat.y : mat.x) * fabsf(lm[0]);
      for (int k = 1; k < 3; ++k) {
        if (!(fl & (1 << k))) continue;
        row_force(C[k], hard, ac[k], lm[k], pn[k], -bound, bound, f, kl);
        acc_row(s, dirs[k] * sg, cross(rs, dirs[k]) * sg, dirs[k], rs, f, kl);
      }
    }
  }
  return viol;
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

// The per-body constants of the solve: world inertia (xx yy zz xy) (xz yz)
// and the inertial target.  They do not change during the passes, so the
// sweeps load them before the lane reduction and their round trip overlaps it.
struct BodyConst {
  float4 w0, w1, xin, qin;
};
__device__ __forceinline__ BodyConst load_body_const(const Dev& d, int i) {
  return BodyConst{d.iw0[i], d.iw1[i], d.xin[i], d.qin[i]};
}

// Inertial terms + Schur-complement solve + pose update (kernels_6dof.py:1379-1414).
__device__ __forceinline__ void solve_body(const Dev& d, int i, float4 xi4, float4 qi, const Acc& s, float dt,
                                           const BodyConst& bc) {
  float m = xi4.w;
  float idt2 = 1.0f / (dt * dt);
  float mi = m * idt2;
  const float4 w0 = bc.w0, w1 = bc.w1;
  float I[3][3] = {{w0.x, w0.w, w1.x}, {w0.w, w0.y, w1.y}, {w1.x, w1.y, w0.z}};
  float A[3][3] = {{s.a[0] + mi, s.a[3], s.a[4]}, {s.a[3], s.a[1] + mi, s.a[5]}, {s.a[4], s.a[5], s.a[2] + mi}};
  float D[3][3] = {{I[0][0] * idt2 + s.dd[0], I[0][1] * idt2 + s.dd[3], I[0][2] * idt2 + s.dd[4]},
                   {I[1][0] * idt2 + s.dd[3], I[1][1] * idt2 + s.dd[1], I[1][2] * idt2 + s.dd[5]},
                   {I[2][0] * idt2 + s.dd[4], I[2][1] * idt2 + s.dd[5], I[2][2] * idt2 + s.dd[2]}};
  float B[3][3] = {{s.b[0], s.b[1], s.b[2]}, {s.b[3], s.b[4], s.b[5]}, {s.b[6], s.b[7], s.b[8]}};
  const float4 xin = bc.xin, qin = bc.qin;
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

__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// L1 prefetch of the SoA records group g's evaluation reads (static groups
// are floor corners or pins; dynamic groups are box-box contacts).
__device__ __forceinline__ void prefetch_group(const Dev& d, int g, bool box) {
  prefetch_l1(d.g_meta + g);
  prefetch_l1(d.g_flags + g);
  prefetch_l1(d.g_lam + g);
  prefetch_l1(d.g_pen + g);
  prefetch_l1(d.g_ac0 + g);
  prefetch_l1(d.g_mat + g);
  prefetch_l1(d.g_offa + g);
  if (box) {
    prefetch_l1(d.g_body + g);
    prefetch_l1(d.g_offb + g);
    prefetch_l1(d.g_n + g);
  }
}

// Batched scenes: a scene takes part in the first `substeps` slots of a
// frame, at its own substep dt and iteration count (scene table entry
// (dt, iterations, substeps, 0)).
__device__ __forceinline__ float4 scene_entry(const Dev& d, int body) { return d.scene_tab[d.scene_of[body]]; }
__device__ __forceinline__ bool scene_on(const Dev& d, float4 t) { return d.ctr->slot < (int)t.z; }
__device__ __forceinline__ bool group_on(const Dev& d, int g) {
  return !d.prm->batched || scene_on(d, scene_entry(d, d.g_body[g].x));
}

// BDF1 velocities + caps of one body (kernels_6dof.py:1871-1901).
// x, q: the body's current pose.
__device__ __forceinline__ void finalize_body(const Dev& d, int i, float dt, float4 x, float4 q) {
  const DevParams& P = *d.prm;
  float4 v = d.v[i], w = d.w[i];
  d.pv[i] = v;
  d.pw[i] = w;
  if (x.w > 0.0f) {
    float4 x0 = d.x0[i];
    V3 nv = V3{x.x - x0.x, x.y - x0.y, x.z - x0.z} / dt;
    V3 nw = quat_to_rotvec(qmul(q, qconj(d.q0[i]))) / dt;
    float sl = sqrtf(dot(nv, nv));
    if (sl > P.max_lin) nv = nv * (P.max_lin / sl);
    float sa = sqrtf(dot(nw, nw));
    if (sa > P.max_ang) nw = nw * (P.max_ang / sa);
    d.v[i] = make_float4(nv.x, nv.y, nv.z, 0.0f);
    d.w[i] = make_float4(nw.x, nw.y, nw.z, 0.0f);
  }
}

// Which flags a color pass carries.
struct PassMode {
  bool post;      // post-stabilization primal (alpha = 0 for non-friction rows)
  bool dual;      // apply the previous iteration's dual update (owned groups)
  bool finalize;  // BDF1 finalize of the body before its primal
  int viol_slot;  // iteration whose violation is recorded (-1: none)
  int it;         // pass index (batched scenes derive their own flags from it)
};

// Folds a warp's violation statistics of iteration `slot` into the
// counters: the max over all rows, and the max and count over box-box
// contact groups (cmax: the rows a contact warm start sets).
__device__ __forceinline__ void record_violation(const Dev& d, int slot, float vmax, float cmax, int ccnt) {
  for (int o = 16; o > 0; o >>= 1) {
    vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    ccnt += __shfl_xor_sync(0xffffffffu, ccnt, o);
  }
  if (lane_id() == 0) {
    if (vmax > 0.0f) atomicMax(&d.ctr->viol_bits[slot], __float_as_uint(vmax));
    if (ccnt > 0) {
      if (cmax > 0.0f) atomicMax(&d.ctr->vc_max_bits[slot], __float_as_uint(cmax));
      atomicAdd(&d.ctr->vc_cnt[slot], ccnt);
    }
  }
}

// Primal sweep of one color: G lanes per body, butterfly reduction of the
// 27 accumulators, lane 0 solves (kernels_6dof.py:1149-1414, in place).
//
// Work is dealt in chunks of 32/G bodies, one chunk per warp: every warp
// starts on chunk (its warp index), and a warp that finishes takes the next
// undealt chunk from the pass's counter (heavy bodies come first in each
// color, so the light ones fill in behind them and the pass ends sooner than
// with a fixed stride).  Which warp runs a body never changes its result.
template <int G, bool B>
__device__ void primal_color(const Dev& d, int c, PassMode pm, float dt, int gtid, int gsize, int pass) {
  constexpr int W = 32 / G;
  const int post_stab = d.prm->post_stab;
  const int slot_now = B ? d.ctr->slot : 0;
  int cs0 = d.color_starts[c];
  int nbody = d.color_starts[c + 1] - cs0;
  const int nchunks = (nbody + W - 1) / W, nwarps = gsize >> 5;
  int* counter = &d.ctr->work_ctr[pass & 3];
  if (gtid == 0) d.ctr->work_ctr[(pass + 2) & 3] = 0;  // two passes ahead: no warp touches it now
  float vmax = 0.0f, csum = 0.0f;
  int ccnt = 0;
  for (int chunk = gtid >> 5; chunk < nchunks;) {
    int slot = chunk * W + (threadIdx.x & 31) / G, lane = threadIdx.x & (G - 1);
    bool valid = slot < nbody;
    int i = valid ? d.color_bodies[cs0 + slot] : 0;
    float4 xi4 = valid ? d.x[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool act = valid && xi4.w > 0.0f;
    bool solve = act;
    if (B) {
      // this body's scene: its own dt; pass `it` is a main iteration while
      // it < its, the post-stab pass (or, without it, the last dual and the
      // finalize) at it == its, and idle beyond or in a slot it skips
      float4 t = valid ? scene_entry(d, i) : make_float4(dt, 0.0f, 0.0f, 0.0f);
      int its = (int)t.y;
      dt = t.x;
      bool on = valid && slot_now < (int)t.z && pm.it <= its;
      pm.post = post_stab && pm.it == its;
      pm.dual = on && pm.it >= 1;
      pm.finalize = on && pm.it == its && its >= 1;
      act = act && on;
      solve = act && (pm.it < its || post_stab);
    }
    if (pm.finalize && valid && lane == 0) finalize_body(d, i, dt, xi4, d.q[i]);
    Acc s;
    acc_zero(s);
    float4 qi = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    bool wrote = false;
    if (act) {
      qi = d.q[i];
      V3 xi = xyz(xi4);
      int s0 = d.sg_start[i], ns = d.sg_start[i + 1] - s0;
      int e0 = d.dg_start[i], nd = d.dg_start[i + 1] - e0;
      // floor corners in the resting start state (fsep; an earlier pass of
      // this substep, on any SM, may have cleared it)
      float fy = d.prm->resting_floor ? __ldcg(d.fsep + i) : 0.0f;
      bool rest = d.prm->resting_floor && fy == fy;
      // Issue every group record this lane will read before evaluating any,
      // so the per-group dependent loads overlap instead of chaining.
      for (int k = lane; k < ns + nd; k += G) {
        if (k < ns) {
          if (!(rest && k < 8)) prefetch_group(d, s0 + k, false);
        } else {
          prefetch_group(d, d.dg_idx[e0 + (k - ns)], true);
        }
      }
      for (int k = lane; k < ns + nd; k += G) {
        int g = k < ns ? s0 + k : d.dg_idx[e0 + (k - ns)];
        int oe = k < ns ? -1 : d.dg_other[e0 + (k - ns)];
        vmax = fmaxf(vmax, accumulate_group<false>(d, g, i, xi, qi, pm.post, pm.dual, s, csum, ccnt, 0, 0, oe,
                                                   rest && k < 8 ? k : -1, fy, &wrote));
      }
    }
    {  // a resting corner whose group was written leaves the resting state
      constexpr unsigned BODY_LANES = G == 32 ? 0xffffffffu : (1u << G) - 1u;
      const unsigned wmask = __ballot_sync(0xffffffffu, wrote);
      if (lane == 0 && ((wmask >> ((threadIdx.x & 31) & ~(G - 1))) & BODY_LANES) != 0u)
        d.fsep[i] = __int_as_float(0x7fffffff);
    }
    BodyConst bc{};
    if (solve && lane == 0) bc = load_body_const(d, i);
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
    if (solve && lane == 0) solve_body(d, i, xi4, qi, s, dt, bc);
    int next = 0;
    if ((threadIdx.x & 31) == 0) next = nwarps + atomicAdd(counter, 1);
    chunk = __shfl_sync(0xffffffffu, next, 0);
  }
  if (pm.viol_slot >= 0) record_violation(d, pm.viol_slot, vmax, csum, ccnt);
}

// B: batched scenes (a separate instantiation, so the single-scene sweep's
// register allocation does not carry the per-scene state).
//
// adaptive_lanes: a pass's time has a floor of one chunk's chain of
// dependent loads, so a color too small to fill the resident warps runs
// faster with more lanes per body (fewer groups per lane): the lane count
// doubles while the color, at twice the lanes, still fits in one round of
// the resident warps.  Only
// the order of the per-body sums changes; the choice depends on the color's
// size alone, so runs stay reproducible.
template <bool B>
__device__ void ph_primal(const Dev& d, int c, PassMode pm, int gtid, int gsize, int pass) {
  float dt = d.prm->dt;
  int lanes = d.prm->group_size;
  if (d.prm->adaptive_lanes) {
    long long nbody = d.color_starts[c + 1] - d.color_starts[c];
    long long warp_lanes = (long long)(gsize >> 5) * 32;  // lanes of one round of the resident warps
    while (lanes < 32 && nbody * (2 * lanes) <= warp_lanes) lanes *= 2;
  }
  switch (lanes) {
    case 1: primal_color<1, B>(d, c, pm, dt, gtid, gsize, pass); break;
    case 2: primal_color<2, B>(d, c, pm, dt, gtid, gsize, pass); break;
    case 4: primal_color<4, B>(d, c, pm, dt, gtid, gsize, pass); break;
    case 8: primal_color<8, B>(d, c, pm, dt, gtid, gsize, pass); break;
    case 16: primal_color<16, B>(d, c, pm, dt, gtid, gsize, pass); break;
    default: primal_color<32, B>(d, c, pm, dt, gtid, gsize, pass); break;
  }
}

// Flags of iteration `it` of `total` (= iterations + post-stab pass).
__device__ __forceinline__ PassMode pass_mode(const DevParams& P, int it) {
  PassMode pm;
  int iters = P.iterations;
  pm.post = P.post_stab && it == iters;
  pm.dual = it >= 1 && it <= iters;  // dual of iteration it-1
  pm.finalize = P.post_stab && it == iters && iters >= 1;
  pm.viol_slot = (P.record_violation && pm.dual && it - 1 < AVBD_MAX_VIOL_ITERS && !P.batched) ? it - 1 : -1;
  pm.it = it;
  return pm;
}


// Flag-ordered sweep: all `total` passes over the colors without a grid
// barrier.  The work is cut into chunks of W = 32/G bodies of one color of
// one pass, numbered in (pass, color) order; warp w starts on chunk w and
// then takes the next undealt chunk from a counter, so chunks are dealt in
// increasing order to whichever warp is free.  A body waits only for its own
// previous pass and for its neighbours (lower color: this pass; higher
// color: the previous pass), so every chunk depends only on lower-numbered
// chunks, all of them already dealt, and the lowest unfinished chunk can
// always run (all warps are resident).  Each body's
// arithmetic and reduction order are those of primal_color, so the results
// are bit-identical to the barrier sweep.
template <int G, bool B>
__device__ void flag_sweep(const Dev& d, int total, int nc, int gtid, int gsize) {
  constexpr int W = 32 / G;
  const unsigned FULL = 0xffffffffu;
  const DevParams& P = *d.prm;
  const int lane = threadIdx.x & 31, slot = lane / G, gl = lane & (G - 1);
  const int post_stab = P.post_stab;
  const int slot_now = B ? d.ctr->slot : 0;
  // chunks per color (colors <= 32: one lane each), inclusive prefix
  int cnt = lane < nc ? d.color_starts[lane + 1] - d.color_starts[lane] : 0;
  int ch = (cnt + W - 1) / W;
  int incl = ch;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  const int per_pass = __shfl_sync(FULL, incl, 31);
  const long long n_chunks = (long long)per_pass * total;
  for (long long q = gtid >> 5; q < n_chunks;) {
    int it = (int)(q / per_pass), r = (int)(q - (long long)it * per_pass);
    int c = __ffs(__ballot_sync(FULL, incl > r)) - 1;
    int cntc = __shfl_sync(FULL, cnt, c);
    int k = (r - __shfl_sync(FULL, incl - ch, c)) * W + slot;
    bool valid = k < cntc;
    int i = valid ? d.color_bodies[d.color_starts[c] + k] : 0;
    PassMode pm = pass_mode(P, it);
    float dt = P.dt;
    bool act = valid && d.x0[i].w > 0.0f;  // mass is constant; x0 was written before the passes
    bool solve = act;
    if (B) {
      float4 t = valid ? scene_entry(d, i) : make_float4(dt, 0.0f, 0.0f, 0.0f);
      int its = (int)t.y;
      dt = t.x;
      bool on = valid && slot_now < (int)t.z && pm.it <= its;
      pm.post = post_stab && pm.it == its;
      pm.dual = on && pm.it >= 1;
      pm.finalize = on && pm.it == its && its >= 1;
      act = act && on;
      solve = act && (pm.it < its || post_stab);
    }
    // The incidence ranges and this lane's first group do not change during
    // the passes: their loads go out before the wait for the body's previous
    // pass, not after it.
    int s0 = 0, ns = 0, e0 = 0, nd = 0, g = 0, oe = -1;
    if (act) {
      s0 = d.sg_start[i];
      ns = d.sg_start[i + 1] - s0;
      e0 = d.dg_start[i];
      nd = d.dg_start[i + 1] - e0;
      g = gl < ns ? s0 + gl : (gl < ns + nd ? d.dg_idx[e0 + (gl - ns)] : 0);
      oe = gl >= ns && gl < ns + nd ? d.dg_other[e0 + (gl - ns)] : -1;
    }
    float4 xi4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), qi = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    if (act) {
      wait_done(d, i, it);  // its own previous pass (possibly on another SM)
      xi4 = __ldcg(d.x + i);
      qi = __ldcg(d.q + i);
    } else if (valid) {
      xi4 = d.x[i];  // a static body: never written by the passes
      qi = d.q[i];
    }
    if (pm.finalize && valid && gl == 0) finalize_body(d, i, dt, xi4, qi);
    Acc s;
    acc_zero(s);
    float vmax = 0.0f, csum = 0.0f;
    int ccnt = 0;
    if (act) {
      V3 xi = xyz(xi4);
      // No L1 prefetch here: the lines of a chunk's ~10 SoA arrays do not
      // survive in L1 until they are read (measured: 0.6 % faster without).
      // The next group's index is loaded before this group is evaluated, so
      // its round trip overlaps the evaluation (0.5-3.5 % faster on different
      // boxes; also loading the next group's body pair that early measured
      // slower).
      const int nt = ns + nd;
      for (int kk = gl; kk < nt; kk += G) {
        int kn = kk + G;
        int gn = kn < ns ? s0 + kn : (kn < nt ? d.dg_idx[e0 + (kn - ns)] : 0);
        int oen = kn >= ns && kn < nt ? d.dg_other[e0 + (kn - ns)] : -1;
        vmax = fmaxf(vmax, accumulate_group<true>(d, g, i, xi, qi, pm.post, pm.dual, s, csum, ccnt, it, c, oe));
        g = gn;
        oe = oen;
      }
    }
    BodyConst bc{};
    if (solve && gl == 0) bc = load_body_const(d, i);
    if (G > 1) {
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int kk = 0; kk < 6; ++kk) {
          s.a[kk] += __shfl_xor_sync(FULL, s.a[kk], o);
          s.dd[kk] += __shfl_xor_sync(FULL, s.dd[kk], o);
        }
#pragma unroll
        for (int kk = 0; kk < 9; ++kk) s.b[kk] += __shfl_xor_sync(FULL, s.b[kk], o);
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          s.rl[kk] += __shfl_xor_sync(FULL, s.rl[kk], o);
          s.ra[kk] += __shfl_xor_sync(FULL, s.ra[kk], o);
        }
      }
    }
    if (solve && gl == 0) solve_body(d, i, xi4, qi, s, dt, bc);
    // publish: the warp barrier orders every lane's writes (dual updates,
    // pose, finalize) before lane 0's release store, and the release is
    // cumulative over them, so one fence per body suffices (the pattern of a
    // grid barrier: block barrier, then one thread's fence).  A full fence in
    // every lane measured 4 % slower.
    __syncwarp();
    if (act && gl == 0) st_release(d.done + i, it + 1);
    if (pm.viol_slot >= 0) record_violation(d, pm.viol_slot, vmax, csum, ccnt);
    int next = 0;
    if (lane == 0) next = atomicAdd(&d.ctr->work_ctr[0], 1);  // zeroed at the substep start
    q = (gsize >> 5) + (long long)__shfl_sync(FULL, next, 0);
  }
}

template <bool B>
__device__ void ph_flag_sweep(const Dev& d, int total, int nc, int gtid, int gsize) {
  switch (d.prm->group_size) {
    case 1: flag_sweep<1, B>(d, total, nc, gtid, gsize); break;
    case 2: flag_sweep<2, B>(d, total, nc, gtid, gsize); break;
    case 4: flag_sweep<4, B>(d, total, nc, gtid, gsize); break;
    case 8: flag_sweep<8, B>(d, total, nc, gtid, gsize); break;
    case 16: flag_sweep<16, B>(d, total, nc, gtid, gsize); break;
    default: flag_sweep<32, B>(d, total, nc, gtid, gsize); break;
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
  float4 oa = meta_implicit(meta) ? implicit_corner(d.he[bd.x], meta, d.g_mat[g].w) : d.g_offa[g];
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
// tangent, and the second tangent's lambda before its own decay.  `lam`,
// `pen` are the group's stored (cached or default) state, or the learned
// start of a new contact.
__device__ __forceinline__ void prelude_group(const Dev& d, int g, int fl, float4 lam, float4 pen) {
  const DevParams& P = *d.prm;
  float main_alpha = P.post_stab ? 1.0f : P.alpha;
  {
    int meta = d.g_meta[g];
    int kind = meta_kind(meta);
    bool three = (meta & 4) != 0;
    float4 mat = d.g_mat[g];
    float s = mat.z;
    bool tang = kind != KIND_PIN;  // rows 1, 2 of floor/box groups are friction rows
    float lm[3] = {lam.x, lam.y, lam.z}, pn[3] = {pen.x, pen.y, pen.z};
    int nr = three ? 3 : 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k >= nr) break;
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
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k >= nr || !(fl & (1 << k))) continue;
      float C0 = c0.c[k];
      if (tang && k > 0) a[k] = C0;
      else if (kind != KIND_PIN) a[k] = C0 > 0.0f ? 0.0f : main_alpha * C0;
      else a[k] = main_alpha * C0;
    }
    d.g_lam[g] = make_float4(lm[0], lm[1], lm[2], 0.0f);
    d.g_pen[g] = make_float4(pn[0], pn[1], pn[2], 0.0f);
    d.g_ac0[g] = make_float4(a[0], a[1], a[2], 0.0f);
    d.g_flags[g] = fl & ~FL_NEW;
  }
}

template <bool B>
__device__ void ph_prelude(const Dev& d, int gtid, int gsize) {
  int ng = n_groups_live(d);
  for (int g = gtid; g < ng; g += gsize) {
    // the next group's fields into L1 while this one is evaluated (a warp's
    // six records span 16 lines, so they stay resident for one iteration)
    const int gn = g + gsize;
    if (gn < ng) {
      prefetch_l1(d.g_flags + gn);
      prefetch_l1(d.g_meta + gn);
      prefetch_l1(d.g_body + gn);
      prefetch_l1(d.g_lam + gn);
      prefetch_l1(d.g_pen + gn);
      prefetch_l1(d.g_mat + gn);
    }
    int fl = d.g_flags[g];
    if (fl & FL_NEW) continue;  // its prelude runs in ph_mlp_prelude
    if (B && !group_on(d, g)) continue;  // batched: its scene sits this substep out
    prelude_group(d, g, fl, d.g_lam[g], d.g_pen[g]);
  }
}

// Learned warm start of the new contacts the emission queued, fused with
// their prelude: each warp runs the network on 16-contact tiles (BF16
// mma.sync, weights staged once per block in shared memory), decodes the
// predicted (lambda_n, lambda_t1, lambda_t2, k_n), keeps the zero start for
// separated contacts, non-finite outputs and forces outside the static
// friction cone, and then runs the prelude of each contact on the start it
// chose.  Block-uniform (every thread of a block reaches the __syncthreads).
__device__ __noinline__ void ph_mlp_prelude(const Dev& d, int gtid, int gsize) {
  if (!d.prm->mlp_on || d.mlp_w == nullptr) return;
  int n = min(*(volatile int*)&d.ctr->n_new_logged, d.new_cap);
  if (n <= 0) return;
  extern __shared__ float sw[];  // AVBD_MLP_FLOATS (dynamic shared memory of the launch)
  stage_weights(d.mlp_w, sw);
  const int lane = threadIdx.x & 31;
  const float zeta = sw[MLPO_OMEAN + MLP_OUT];
  int applied = 0, fallback = 0;
  for (int tile = gtid >> 5; tile * 16 < n; tile += gsize >> 5) {
    int r0 = tile * 16, rows = min(16, n - r0);
    float y[4], og[4], og8[4];
    mlp_tile(sw, d.mlp_feat + (size_t)r0 * MLP_IN, rows, y);
    gather_rows(y, og, og8);
    if ((lane & 3) == 0) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        int row = (lane >> 2) + 8 * r;
        if (row >= rows) continue;
        int k = r0 + row;
        const float* f = d.mlp_feat + (size_t)k * MLP_IN;
        int g = d.new_list[k];
        if (!group_on(d, g)) continue;
        int fl = d.g_flags[g];
        float4 lam = d.g_lam[g], pen = d.g_pen[g];  // the zero start written by the emission
        float4 l2;
        float kn;
        if (decode_start(r ? og8 : og, f[3], f[11], zeta, l2, kn)) {
          if (!(d.g_meta[g] & 4)) l2.y = l2.z = 0.0f;
          lam = l2;
          pen.x = kn;
          fl |= FL_LRN;
          ++applied;
        } else {
          ++fallback;
        }
        prelude_group(d, g, fl, lam, pen);
      }
    }
  }
  __syncthreads();  // the shared weights are not reused before every warp is done
  for (int o = 16; o > 0; o >>= 1) {
    applied += __shfl_xor_sync(0xffffffffu, applied, o);
    fallback += __shfl_xor_sync(0xffffffffu, fallback, o);
  }
  if (lane == 0) {
    if (applied) atomicAdd(&d.ctr->n_mlp_applied, applied);
    if (fallback) atomicAdd(&d.ctr->n_mlp_fallback, fallback);
  }
}


// Stand-alone dual update of every group (kernels_6dof.py:1451-1548); used
// after the last iteration when there is no post-stabilization pass to carry
// it, and by the split path.  Optionally records the iteration's violation.
__device__ void ph_dual(const Dev& d, int it, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  int ng = n_groups_live(d);
  float vmax = 0.0f, csum = 0.0f;
  int ccnt = 0;
  for (int g = gtid; g < ng; g += gsize) {
    int meta = d.g_meta[g];
    int fl = d.g_flags[g];
    if (!(fl & 7)) continue;
    int kind = meta_kind(meta);
    bool three = (meta & 4) != 0, hard = (meta & 8) != 0;
    float4 lam = d.g_lam[g], pen = d.g_pen[g], ac0 = d.g_ac0[g], mat = d.g_mat[g];
    if (meta_implicit(meta)) mat.w = FINF;  // w holds the floor height
    GroupC cv = group_values(d, g, meta, d.x, d.q);
    float lm[3] = {lam.x, lam.y, lam.z}, pn[3] = {pen.x, pen.y, pen.z}, ac[3] = {ac0.x, ac0.y, ac0.z};
    if (fl & FL_LRN) learned_check(d, kind, hard, cv.c, ac, lm, pn, fl);
    float v = dual_rows(kind, three ? 3 : 1, hard, mat, cv.c, ac, P.beta, lm, pn, fl);
    vmax = fmaxf(vmax, v);
    if (kind == KIND_BOX && (fl & FL_ACT0)) {
      csum += v;
      ++ccnt;
    }
    d.g_lam[g] = make_float4(lm[0], lm[1], lm[2], 0.0f);
    d.g_pen[g] = make_float4(pn[0], pn[1], pn[2], 0.0f);
    d.g_flags[g] = fl;
  }
  if (P.record_violation && it < AVBD_MAX_VIOL_ITERS) record_violation(d, it, vmax, csum, ccnt);
}

// Inertial target + warm start (kernels_6dof.py:122-187), plus the owner of
// every contact group for the fused dual: its dynamic body with the lower
// color (a static body never runs a primal, so it never owns).
template <bool B>
__device__ void ph_predict(const Dev& d, int gtid, int gsize) {
  const DevParams& P = *d.prm;
  for (int i = gtid; i < d.nb; i += gsize) {
    float dt = P.dt;
    float4 x = d.x[i], q = d.q[i];
    float m = x.w;
    // flag sweep: passes done so far; a body that never runs counts as done
    d.done[i] = m > 0.0f ? 0 : 0x3fffffff;
    if (B) {
      float4 t = scene_entry(d, i);
      if (!scene_on(d, t)) {  // the scene sits this substep out: state untouched
        d.done[i] = 0x3fffffff;
        continue;
      }
      dt = t.x;
    }
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
  int nd = d.ctr->n_dyn_groups;
  for (int u = gtid; u < nd; u += gsize) {
    int g = d.n_sg + u;
    int2 bd = d.g_body[g];
    bool sa = d.x[bd.x].w <= 0.0f, sb = d.x[bd.y].w <= 0.0f;  // mass in .w is never changed by predict
    bool ownb = sa || (!sb && d.color[bd.y] < d.color[bd.x]);
    int fl = d.g_flags[g];
    d.g_flags[g] = ownb ? (fl | FL_OWNB) : (fl & ~FL_OWNB);
  }
  if (P.resting_floor && !P.flag_sweep) {
    // fsep: eight lanes per body, lane c checks the body's static group c
    // (after the prelude, so this is the state the passes start from).  The
    // trip count is a multiple of 32, so every lane of a warp runs the same
    // iterations and the eight lanes of a body are one aligned octet.
    const long long n8 = 8LL * d.nb, lim = (n8 + 31) & ~31LL;
    const int lane = threadIdx.x & 31;
    for (long long t = gtid; t < lim; t += gsize) {
      int i = (int)(t >> 3), c = (int)(t & 7);
      bool ok = false;
      float fyc = 0.0f;
      if (t < n8 && d.x[i].w > 0.0f) {  // mass in .w is never changed by predict
        int s0 = d.sg_start[i];
        if (d.sg_start[i + 1] - s0 >= 8) {
          int g = s0 + c;
          float4 lam = d.g_lam[g], pen = d.g_pen[g], ac0 = d.g_ac0[g], mat = d.g_mat[g];
          ok = d.g_meta[g] == resting_corner_meta(c) && (d.g_flags[g] & (7 | FL_WAS | FL_LRN)) == 7 &&
               lam.x == 0.0f && lam.y == 0.0f && lam.z == 0.0f && pen.x == PEN_MIN && pen.y == PEN_MIN_T &&
               pen.z == PEN_MIN_T && ac0.x == 0.0f && isfinite(mat.x) && isfinite(mat.y) && isfinite(mat.w);
          fyc = mat.w;
        }
      }
      float fy0 = __shfl_sync(0xffffffffu, fyc, lane & ~7);
      unsigned m = __ballot_sync(0xffffffffu, ok && fyc == fy0);
      if (t < n8 && c == 0) d.fsep[i] = ((m >> lane) & 0xffu) == 0xffu ? fy0 : __int_as_float(0x7fffffff);
    }
  }
}

// BDF1 velocities + caps of every body (kernels_6dof.py:1871-1901).
__device__ void ph_finalize(const Dev& d, int gtid, int gsize) {
  float dt = d.prm->dt;
  for (int i = gtid; i < d.nb; i += gsize) finalize_body(d, i, dt, d.x[i], d.q[i]);
}

// Contact-cache refresh (kernels_6dof.py:2923-2995) with an epoch tag in
// place of the full-table clear (kernels_6dof.py:2915-2920).
__device__ void ph_collect(const Dev& d, int gtid, int gsize) {
  int nd = d.ctr->n_dyn_groups;
  unsigned tag = epoch_tag(d.ctr->epoch + 1u);
  unsigned mask = (unsigned)d.hash_cap - 1u;
  int reverted = 0;
  for (int u = gtid; u < nd; u += gsize) {
    int g = d.n_sg + u;
    int fl = d.g_flags[g];
    if (fl & FL_REV) ++reverted;
    if (!(fl & FL_ACT0)) continue;
    int meta = d.g_meta[g];
    int2 bd = d.g_body[g];
    int ka = min(bd.x, bd.y), kb = max(bd.x, bd.y);
    unsigned long long key = d.g_key ? d.g_key[g] : cache_key(ka, kb, meta_cidx(meta));
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
      // a plain L2 read: the compare-and-swap below validates it
      unsigned long long v = __ldcg(&d.h_key[sl]);
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
  for (int o = 16; o > 0; o >>= 1) reverted += __shfl_xor_sync(0xffffffffu, reverted, o);
  if (lane_id() == 0 && reverted) atomicAdd(&d.ctr->n_mlp_reverted, reverted);
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
  // two pairs per iteration, every load issued before any test (a pair's
  // bodies are valid indices whether or not it kept contacts): two dependent
  // round trips per pair of pairs instead of three per pair
  for (int p = gtid; p < np; p += 2 * gsize) {
    const int p1 = p + gsize;
    const bool h1 = p1 < np;
    int k0 = d.pair_kept[p], k1 = h1 ? d.pair_kept[p1] : 0;
    int2 a0 = d.pair_ab[p], a1 = h1 ? d.pair_ab[p1] : make_int2(0, 0);
    int c00 = d.color[a0.x], c01 = d.color[a0.y], c10 = d.color[a1.x], c11 = d.color[a1.y];
    cnt += (k0 != 0 && c00 == c01) ? 1 : 0;
    cnt += (k1 != 0 && c10 == c11) ? 1 : 0;
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
    d.ctr->round_unc[0] = 0;
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
__device__ void ph_round_assign(const Dev& d, bool jp, int* unc_out, int gtid, int gsize) {
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
    if (lane_id() == 0 && unc) atomicAdd(unc_out, unc);
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

__device__ void ph_resolve_apply(const Dev& d, int* unc_out, int gtid, int gsize) {
  int unc = 0;
  for (int i = gtid; i < d.nb; i += gsize) {
    if (d.c_lost[i]) {
      d.color[i] = -1;
      d.c_lost[i] = 0;
    }
    if (d.color[i] < 0) ++unc;
  }
  for (int o = 16; o > 0; o >>= 1) unc += __shfl_xor_sync(0xffffffffu, unc, o);
  if (lane_id() == 0 && unc) atomicAdd(unc_out, unc);
}

// Jones-Plassmann as one dataflow phase (persistent kernel only: it needs
// every thread of the grid resident).  A JP round colors a body once every
// higher-priority neighbour is colored, with the smallest color none of them
// holds, so the result is the greedy coloring in decreasing priority, and the
// round that colors body i is r(i) = 1 + max r over its higher-priority
// neighbours (0 with none).  A body with r(i) >= JP_ROUNDS is still
// uncolored after the last round and the bucket phase gives it color 0.
// Here each body publishes st[i] = 1 + 64 r(i) + color (color 63 =
// uncolored) once all its higher-priority neighbours have published: the
// same colors as the round loop, without its 2 x JP_ROUNDS grid barriers.
// The published word is the only data exchanged, so plain relaxed loads
// and stores suffice.  Neighbours are the other bodies of the body's contact
// groups (the kept-pair graph of the round loop; a pair's groups are
// adjacent in the sorted incidence list, so repeats are adjacent too).
//
// Progress: a thread takes its bodies (gtid, gtid + gsize, ...) in
// decreasing priority.  For the current body it collects up to DF_HP
// higher-priority neighbours, polls all of them at once, and never waits
// inside a step.  The highest-priority body not yet published is its
// thread's current body, and everything it waits for has published, so it
// always advances.  Returns false (nothing done) when a thread would hold
// more than 32 bodies; the caller then runs the round loop.
//
// It runs speculatively, before the gate has decided whether to recolor:
// it reads only the contact graph and the priorities and writes color2 (-1
// = uncolored) and st = c_lost, which must be zero on entry (the arena
// starts zeroed; the persistent kernel clears it after every use, and so
// does avbd_clear_errors after a launch that stopped early).  When the gate
// keeps the old coloring, color2 is simply not used.
#define DF_HP 8
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __noinline__ bool ph_color_dataflow(const Dev& d, int gtid, int gsize) {
  const int nb = d.nb;
  if ((long long)nb > 32LL * gsize) return false;
  int* st = d.c_lost;  // zeroed by ph_color_reset
  int nk = gtid < nb ? (nb - 1 - gtid) / gsize + 1 : 0;
  unsigned todo = nk >= 32 ? 0xffffffffu : ((1u << nk) - 1u);
  int cur = -1, kp = 0, ke = 0, rmax = -1, last = -1, pending = 0;
  float pcur = 0.0f;
  unsigned used = 0;
  int hp[DF_HP];
  auto take_next = [&]() {
    cur = -1;
    for (unsigned m = todo; m; m &= m - 1) {
      int j = gtid + (__ffs(m) - 1) * gsize;
      float pj = d.prio[j];
      if (cur < 0 || pj > pcur || (pj == pcur && j < cur)) {
        cur = j;
        pcur = pj;
      }
    }
    if (cur >= 0) {
      todo &= ~(1u << ((cur - gtid) / gsize));
      kp = d.dg_start[cur];
      ke = d.dg_start[cur + 1];
      rmax = -1;
      last = -1;
      used = 0;
    }
  };
  // Next batch of higher-priority neighbours into hp[0..pending).
  auto collect = [&]() {
#pragma unroll
    for (int j = 0; j < DF_HP; ++j) hp[j] = -1;
    pending = 0;
    for (; kp < ke && pending < DF_HP; ++kp) {
      int o = d.dg_other[kp] >> 1;
      if (o == last) continue;
      last = o;
      float po = d.prio[o];
      if (!(po > pcur || (po == pcur && o < cur))) continue;
#pragma unroll
      for (int j = DF_HP - 1; j > 0; --j) hp[j] = hp[j - 1];  // shift: keeps hp[] in registers
      hp[0] = o;
      ++pending;
    }
  };
  take_next();
  unsigned long long t0 = 0;
  const unsigned long long budget = d.prm->barrier_timeout_ns;
  unsigned polls = 0;
  while (cur >= 0) {
    if (pending == 0 && kp < ke) collect();
    if (pending > 0) {
#pragma unroll
      for (int j = 0; j < DF_HP; ++j) {
        if (hp[j] < 0) continue;
        int s = ld_relaxed(st + hp[j]);
        if (s == 0) continue;
        --s;
        rmax = max(rmax, s >> 6);
        if ((s & 63) < MAX_COLORS) used |= 1u << (s & 63);
        hp[j] = -1;
        --pending;
      }
      if (rmax + 1 >= JP_ROUNDS) {  // uncolored whatever the other neighbours hold
        pending = 0;
        kp = ke;
      }
    }
    if (pending == 0 && kp >= ke) {
      int r = rmax + 1, c = 63;
      if (r >= JP_ROUNDS) {
        r = JP_ROUNDS;
      } else {
        c = first_fit((int)used);
      }
      d.color2[cur] = c < MAX_COLORS ? c : -1;
      asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(st + cur), "r"(1 + (r << 6) + c) : "memory");
      take_next();
      continue;
    }
    if (pending == 0) continue;  // more neighbours to collect
    if ((++polls & 31u) == 0u) {
      if (*(volatile int*)&d.ctr->err & ERR_BARRIER_TIMEOUT) return true;
      unsigned long long now = gtimer();
      if (t0 == 0) t0 = now;
      else if (now - t0 > budget) {
        atomicOr(&d.ctr->err, ERR_BARRIER_TIMEOUT);
        return true;
      }
    }
    __nanosleep(32);
  }
  return true;
}

// Bucketing of bodies by color.  Within a color, bodies come in four work
// buckets, heaviest first: more than 24, 17-24, 9-16 and at most 8 incident
// groups, i.e. by the lane rounds a body takes at 8 lanes.  The longest jobs
// start in the first wave of a pass, and a 4-body chunk mostly holds bodies
// with the same number of rounds, so few lanes idle.  Then by body index;
// deterministic.  Key = 4 * color + bucket.
#define NCH 64
#define NBK 4
#define NKEY (NBK * MAX_COLORS)
#define BUCKET_WARPS 8  // ph_bucket_place runs with 256-thread blocks (launch_solve checks)
__device__ __forceinline__ int bucket_key(const Dev& d, int i, int c) {
  int work = (d.sg_start[i + 1] - d.sg_start[i]) + (d.dg_start[i + 1] - d.dg_start[i]);
  return NBK * c + (work > 24 ? 0 : work > 16 ? 1 : work > 8 ? 2 : 3);
}

// from_color2: the colors come from the speculative dataflow coloring.
__device__ void ph_bucket_count(const Dev& d, bool from_color2 = false) {
  __shared__ int h[NKEY];
  int cs = (d.nb + NCH - 1) / NCH;
  for (int b = blockIdx.x; b < NCH; b += gridDim.x) {
    if (threadIdx.x < NKEY) h[threadIdx.x] = 0;
    __syncthreads();
    int s0 = b * cs, s1 = min(d.nb, s0 + cs);
    for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
      int c = from_color2 ? d.color2[i] : d.color[i];
      if (c < 0 || from_color2) {  // stragglers take color 0 (kernels_6dof.py:3151-3165)
        c = max(c, 0);
        d.color[i] = c;
      }
      atomicAdd(&h[bucket_key(d, i, c)], 1);
    }
    __syncthreads();
    if (threadIdx.x < NKEY) d.c_hist[b * NKEY + threadIdx.x] = h[threadIdx.x];
    __syncthreads();
  }
}

__device__ void ph_bucket_scan(const Dev& d) {
  if (blockIdx.x != 0) return;
  __shared__ int tot[NKEY];
  __shared__ int kstart[NKEY + 1];
  int k = threadIdx.x;
  if (k < NKEY) {
    int run = 0;
    for (int b = 0; b < NCH; ++b) {
      int v = d.c_hist[b * NKEY + k];
      d.c_hist[b * NKEY + k] = run;
      run += v;
    }
    tot[k] = run;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0, mx = 0;
    for (int u = 0; u < NKEY; ++u) {
      kstart[u] = acc;
      acc += tot[u];
      if (tot[u] > 0) mx = u / NBK;
    }
    kstart[NKEY] = acc;
    for (int c = 0; c <= MAX_COLORS; ++c) d.color_starts[c] = kstart[NBK * c < NKEY ? NBK * c : NKEY];
    d.ctr->n_colors = max(1, min(mx + 1, MAX_COLORS));
    d.ctr->color_dirty = 0;
  }
  __syncthreads();
  // chunk offsets become absolute positions
  if (k < NKEY)
    for (int b = 0; b < NCH; ++b) d.c_hist[b * NKEY + k] += kstart[k];
}

__device__ void ph_bucket_place(const Dev& d) {
  __shared__ int run[NKEY];
  __shared__ int wc[BUCKET_WARPS][NKEY];
  int cs = (d.nb + NCH - 1) / NCH;
  int w = threadIdx.x >> 5, l = lane_id();
  int nw = blockDim.x >> 5;
  for (int b = blockIdx.x; b < NCH; b += gridDim.x) {
    if (threadIdx.x < NKEY) run[threadIdx.x] = d.c_hist[b * NKEY + threadIdx.x];
    int s0 = b * cs, s1 = min(d.nb, s0 + cs);
    for (int base = s0; base < s1; base += blockDim.x) {
      for (int k = threadIdx.x; k < BUCKET_WARPS * NKEY; k += blockDim.x) (&wc[0][0])[k] = 0;
      __syncthreads();
      int i = base + threadIdx.x;
      bool valid = i < s1;
      int key = valid ? bucket_key(d, i, d.color[i]) : NKEY + l;
      unsigned peers = __match_any_sync(0xffffffffu, key);
      int rank = __popc(peers & ((1u << l) - 1u));
      if (valid && rank == 0) wc[w][key] = __popc(peers);
      __syncthreads();
      if (valid) {
        int off = run[key];
        for (int u = 0; u < w; ++u) off += wc[u][key];
        d.color_bodies[off + rank] = i;
      }
      __syncthreads();
      if (threadIdx.x < NKEY) {
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
// Two register budgets of the same kernel: 2 CTAs/SM (128 registers) or
// 3 CTAs/SM (80 registers); the host picks one (params.blocks_per_sm).

// `mode`: 0 = the whole substep; 1 = the head (gate, prelude, coloring,
// predict) only; 2 = the tail (last dual without post-stabilization,
// collect) only.  Modes 1 and 2 bracket the flag-ordered sweep when it runs
// as its own launch (k_flag_sweep), so the sweep gets a register budget of
// its own.
template <int MINB, bool BATCHED>
__global__ void __launch_bounds__(SOLVE_BLOCK, MINB) k_solve_persistent(const __grid_constant__ Dev d, int mode) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  int gsize = gridDim.x * blockDim.x;
  int bar = 0;
  const DevParams& P = *d.prm;
  const bool timing = P.timing != 0;
  // SYNC(id): grid barrier; in timing mode thread 0 stamps the end of phase id.
#define MARK(id)                                                     \
  do {                                                               \
    if (timing && gtid == 0) {                                       \
      int m_ = d.ctr->n_marks;                                       \
      if (m_ < 256) {                                                \
        d.ctr->mark_t[m_] = gtimer();                                \
        d.ctr->mark_id[m_] = (id);                                   \
        d.ctr->n_marks = m_ + 1;                                     \
      }                                                              \
    }                                                                \
  } while (0)
#define SYNC(id)                                                     \
  do {                                                               \
    if (!grid_barrier(d, bar++)) return;                             \
    MARK(id);                                                        \
  } while (0)
  const bool jp = P.color_mode == 1;
  // Jones-Plassmann: the dataflow coloring runs alongside the gate and the
  // prelude, into color2, and is used only if the gate asks for new colors.
  const bool spec = jp && (long long)d.nb <= 32LL * gsize;
  int iters = P.iterations;
  if (mode != 2) {
    if (timing && gtid == 0) {
      d.ctr->mark_t[0] = gtimer();
      d.ctr->mark_id[0] = PH_START;
      d.ctr->n_marks = 1;
    }
    ph_gate(d, gtid, gsize);
    ph_prelude<BATCHED>(d, gtid, gsize);  // reads x/q = the initial pose; predict runs after
    ph_mlp_prelude(d, gtid, gsize);
    if (spec) ph_color_dataflow(d, gtid, gsize);
    SYNC(PH_GATE_PRELUDE);
    if (recolor_needed(d)) {
      if (spec) {
        if (gtid == 0) d.ctr->recolored = 1;
      } else {
        ph_color_reset(d, gtid, gsize);
        SYNC(PH_COLOR_RESET);
      }
      // Round r counts its uncolored bodies into round_unc[r & 1]; every block
      // reads it after the round's last barrier.  The other slot is cleared
      // during round r's second phase, when all blocks have read it.
      int rounds = spec ? 0 : (jp ? JP_ROUNDS : MAX_COLORS);
      for (int r = 0; r < rounds; ++r) {
        int* unc_slot = &d.ctr->round_unc[r & 1];
        ph_round_edges(d, jp, gtid, gsize);
        SYNC(PH_ROUND);
        if (gtid == 0) d.ctr->round_unc[(r + 1) & 1] = 0;
        ph_round_assign(d, jp, unc_slot, gtid, gsize);
        SYNC(PH_ROUND);
        if (!jp) {
          ph_resolve_edges(d, gtid, gsize);
          SYNC(PH_ROUND);
          ph_resolve_apply(d, unc_slot, gtid, gsize);
          SYNC(PH_ROUND);
        }
        if (*(volatile int*)unc_slot == 0) break;
      }
      ph_bucket_count(d, spec);
      SYNC(PH_BUCKET);
      ph_bucket_scan(d);
      SYNC(PH_BUCKET);
      ph_bucket_place(d);
    } else if (gtid == 0) {
      d.ctr->recolored = 0;
    }
    ph_predict<BATCHED>(d, gtid, gsize);
    SYNC(PH_PREDICT);
    if (mode == 1) return;
    // batched scenes: one pass beyond the most iterations, where each scene
    // runs its post-stab pass or its last dual + finalize
    int total = iters + ((P.post_stab || P.batched) ? 1 : 0);
    int nc = *(volatile int*)&d.ctr->n_colors;
    // Pass `it` applies iteration it-1's dual update inside the color passes
    // (owner-first), so each iteration is nc barriers; without a
    // post-stabilization pass the last dual and the finalize run on their own.
    if (P.flag_sweep && nc > 0) {
      // all passes at once, each body ordered against its neighbours only
      ph_flag_sweep<BATCHED>(d, total, nc, gtid, gsize);
      SYNC(PH_PRIMAL);
    } else {
      for (int it = 0; it < total; ++it) {
        PassMode pm = pass_mode(P, it);
        for (int c = 0; c < nc; ++c) {
          ph_primal<BATCHED>(d, c, pm, gtid, gsize, it * nc + c);
          SYNC(PH_PRIMAL);
        }
      }
    }
  } else {
    MARK(PH_PRIMAL);  // the sweep launch ended
  }
  if (!P.post_stab && !P.batched && iters >= 1) {
    ph_dual(d, iters - 1, gtid, gsize);
    ph_finalize(d, gtid, gsize);
    SYNC(PH_DUAL);
  }
  ph_collect(d, gtid, gsize);
  if (spec)
    for (int i = gtid; i < d.nb; i += gsize) d.c_lost[i] = 0;  // the dataflow's flags, for the next launch
  SYNC(PH_COLLECT);
  if (gtid == 0) {
    d.ctr->epoch += 1u;
    d.ctr->n_viol = P.record_violation ? min(iters, AVBD_MAX_VIOL_ITERS) : 0;
  }
#undef SYNC
#undef MARK
}

// The flag-ordered sweep as a launch of its own, between the head and the
// tail of the persistent kernel: G fixed at compile time and 20 warps per SM
// (320 threads x 2 CTAs, 96 registers; inside the persistent kernel it runs
// at 16 warps with every lane count's code in one register budget), or 24
// warps per SM (256 threads x 3 CTAs, 80 registers, more spills).  A
// cooperative launch, so every CTA is resident: a warp's first chunk is
// its index, and later chunks wait only on lower ones already running.
#define SWEEP_BLOCK_FOR(minb) ((minb) >= 3 ? 256 : 320)
template <int G, bool B, int MINB>
__global__ void __launch_bounds__(SWEEP_BLOCK_FOR(MINB), MINB) k_flag_sweep(const __grid_constant__ Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  int gsize = gridDim.x * blockDim.x;
  const DevParams& P = *d.prm;
  int total = P.iterations + ((P.post_stab || P.batched) ? 1 : 0);
  int nc = *(volatile int*)&d.ctr->n_colors;
  if (nc > 0) flag_sweep<G, B>(d, total, nc, gtid, gsize);
}

// ---------------------------------------------------------------------------
// Split path: one launch per phase, same phase functions.
// ---------------------------------------------------------------------------
#define GS int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x
__global__ void ks_gate_prelude(const __grid_constant__ Dev d) {
  GS;
  ph_gate(d, gtid, gsize);
  if (d.prm->batched) ph_prelude<true>(d, gtid, gsize);
  else ph_prelude<false>(d, gtid, gsize);
}
__global__ void ks_mlp_prelude(const __grid_constant__ Dev d) { GS; ph_mlp_prelude(d, gtid, gsize); }
__global__ void ks_color_reset(const __grid_constant__ Dev d) {
  GS;
  if (!recolor_needed(d)) {
    if (gtid == 0) d.ctr->recolored = 0;
    return;
  }
  ph_color_reset(d, gtid, gsize);
}
__global__ void ks_round_edges(const __grid_constant__ Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0) return;
  ph_round_edges(d, d.prm->color_mode == 1, gtid, gsize);
}
__global__ void ks_round_assign(const __grid_constant__ Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0) return;
  ph_round_assign(d, d.prm->color_mode == 1, &d.ctr->uncolored, gtid, gsize);
}
__global__ void ks_resolve_edges(const __grid_constant__ Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0 || d.prm->color_mode == 1) return;
  ph_resolve_edges(d, gtid, gsize);
}
__global__ void ks_resolve_apply(const __grid_constant__ Dev d) {
  GS;
  if (!d.ctr->recolored || d.ctr->uncolored < 0 || d.prm->color_mode == 1) return;
  ph_resolve_apply(d, &d.ctr->uncolored, gtid, gsize);
}
// After a round: uncolored == 0 -> mark done (-1), else reset the count.
__global__ void ks_round_end(const __grid_constant__ Dev d) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && d.ctr->recolored && d.ctr->uncolored >= 0)
    d.ctr->uncolored = d.ctr->uncolored == 0 ? -1 : 0;
}
__global__ void ks_bucket_count(const __grid_constant__ Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_count(d);
}
__global__ void ks_bucket_scan(const __grid_constant__ Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_scan(d);
}
__global__ void ks_bucket_place(const __grid_constant__ Dev d) {
  if (!d.ctr->recolored) return;
  ph_bucket_place(d);
}
__global__ void ks_predict(const __grid_constant__ Dev d) {
  GS;
  if (d.prm->batched) ph_predict<true>(d, gtid, gsize);
  else ph_predict<false>(d, gtid, gsize);
}
__global__ void ks_primal(const __grid_constant__ Dev d, int it, int c) {
  GS;
  if (c >= d.ctr->n_colors) return;
  int pass = it * d.ctr->n_colors + c;
  if (d.prm->batched) ph_primal<true>(d, c, pass_mode(*d.prm, it), gtid, gsize, pass);
  else ph_primal<false>(d, c, pass_mode(*d.prm, it), gtid, gsize, pass);
}
__global__ void ks_tail(const __grid_constant__ Dev d) {
  GS;
  int iters = d.prm->iterations;
  if (!d.prm->post_stab && !d.prm->batched && iters >= 1) {
    ph_dual(d, iters - 1, gtid, gsize);
    ph_finalize(d, gtid, gsize);
  }
}
__global__ void ks_collect(const __grid_constant__ Dev d) { GS; ph_collect(d, gtid, gsize); }
__global__ void ks_end(const __grid_constant__ Dev d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    d.ctr->epoch += 1u;
    d.ctr->n_viol = d.prm->record_violation ? min(d.prm->iterations, AVBD_MAX_VIOL_ITERS) : 0;
  }
}
#undef GS

int solve_occupancy(int block, int variant) {
  int n = 0;
  // sized with the learned warm start's shared weights, whether used or not
  size_t smem = sizeof(float) * AVBD_MLP_FLOATS;
  int nb = 0;
  if (variant >= 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solve_persistent<3, false>, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_solve_persistent<3, true>, block, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solve_persistent<2, false>, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_solve_persistent<2, true>, block, smem);
  }
  if (nb < n) n = nb;  // one grid size serves both instantiations
  return n;
}

template <int MINB>
static const void* sweep_kernel_m(int group_size, bool b) {
  switch (group_size) {
    case 1: return b ? (const void*)k_flag_sweep<1, true, MINB> : (const void*)k_flag_sweep<1, false, MINB>;
    case 2: return b ? (const void*)k_flag_sweep<2, true, MINB> : (const void*)k_flag_sweep<2, false, MINB>;
    case 4: return b ? (const void*)k_flag_sweep<4, true, MINB> : (const void*)k_flag_sweep<4, false, MINB>;
    case 8: return b ? (const void*)k_flag_sweep<8, true, MINB> : (const void*)k_flag_sweep<8, false, MINB>;
    case 16: return b ? (const void*)k_flag_sweep<16, true, MINB> : (const void*)k_flag_sweep<16, false, MINB>;
    default: return b ? (const void*)k_flag_sweep<32, true, MINB> : (const void*)k_flag_sweep<32, false, MINB>;
  }
}
static const void* sweep_kernel(int group_size, bool b, int minb) {
  return minb >= 3 ? sweep_kernel_m<3>(group_size, b) : sweep_kernel_m<2>(group_size, b);
}

int sweep_block_size(int blocks_per_sm) { return SWEEP_BLOCK_FOR(blocks_per_sm); }

int sweep_grid_size(int group_size, bool batched, int num_sms, int blocks_per_sm) {
  int minb = blocks_per_sm >= 3 ? 3 : 2;
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_kernel(group_size, batched, minb), SWEEP_BLOCK_FOR(minb), 0);
  if (n > minb) n = minb;
  return num_sms * (n > 0 ? n : 1);
}

cudaError_t launch_solve(Dev& d, const AvbdParams& P, int persistent, int grid, int block, cudaStream_t st,
                         int variant, int sweep_grid, int sweep_minb) {
  // the bucket phases size their per-warp tables for this block size
  if (block != SOLVE_BLOCK) return cudaErrorInvalidConfiguration;
  // dynamic shared memory: the learned warm start's weights, when present
  size_t mlp_smem = d.mlp_w != nullptr ? sizeof(float) * AVBD_MLP_FLOATS : 0;
  if (persistent) {
    const bool b = d.n_scenes > 0;
    const void* fn = variant >= 3 ? (b ? (const void*)k_solve_persistent<3, true> : (const void*)k_solve_persistent<3, false>)
                                  : (b ? (const void*)k_solve_persistent<2, true> : (const void*)k_solve_persistent<2, false>);
    if (!P.flag_sweep || sweep_grid <= 0) {
      int mode = 0;
      void* args[] = {(void*)&d, (void*)&mode};
      g_kernel_launches += 1;
      return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, mlp_smem, st);
    }
    int head = 1, tail = 2;
    void* a_head[] = {(void*)&d, (void*)&head};
    void* a_sweep[] = {(void*)&d};
    void* a_tail[] = {(void*)&d, (void*)&tail};
    g_kernel_launches += 3;
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), a_head, mlp_smem, st);
    if (e != cudaSuccess) return e;
    e = cudaLaunchCooperativeKernel(sweep_kernel(P.group_size, b, sweep_minb), dim3(sweep_grid),
                                    dim3(SWEEP_BLOCK_FOR(sweep_minb)), a_sweep, 0, st);
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), a_tail, mlp_smem, st);
  }
  ks_gate_prelude<<<grid, block, 0, st>>>(d);
  if (mlp_smem) {
    ks_mlp_prelude<<<grid, block, mlp_smem, st>>>(d);
    g_kernel_launches += 1;
  }
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
  int total = P.iterations + ((P.post_stabilize || d.n_scenes > 0) ? 1 : 0);
  for (int it = 0; it < total; ++it)
    for (int c = 0; c < MAX_COLORS; ++c) ks_primal<<<grid, block, 0, st>>>(d, it, c);
  ks_tail<<<grid, block, 0, st>>>(d);
  ks_collect<<<grid, block, 0, st>>>(d);
  ks_end<<<1, 32, 0, st>>>(d);
  g_kernel_launches += 2 + 5 * rounds + 3 + 1 + total * MAX_COLORS + 3;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// State reset, diagnostics, cache scrub.
// ---------------------------------------------------------------------------
__global__ void k_reset(const __grid_constant__ Dev d) {
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
    for (int k = 0; k < BAR_SUB; ++k) c->bar_sub[k][0] = 0;
    for (int k = 0; k < AVBD_MAX_VIOL_ITERS; ++k) {
      c->viol_bits[k] = 0;
      c->vc_max_bits[k] = 0u;
      c->vc_cnt[k] = 0;
    }
  }
}
void launch_reset(Dev& d, cudaStream_t st) { k_reset<<<148 * 4, 256, 0, st>>>(d); }

__global__ void k_conflicts(const __grid_constant__ Dev d, int* out) {
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
__global__ void k_hash_scrub(const __grid_constant__ Dev d) {
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
__global__ void k_cache_clear(const __grid_constant__ Dev d) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  for (int s = gtid; s < d.hash_cap; s += gsize) d.h_key[s] = 0ull;
}
// Entries are (a, b, ordinal) triples, or raw 50-bit keys when `keys` is set.
__global__ void k_cache_insert(const __grid_constant__ Dev d, int n, const int* abc, const unsigned long long* keys,
                               const float* st) {
  int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsize = gridDim.x * blockDim.x;
  unsigned tag = epoch_tag(d.ctr->epoch);
  unsigned mask = (unsigned)d.hash_cap - 1u;
  for (int k = gtid; k < n; k += gsize) {
    unsigned long long key = keys ? (keys[k] & KEY_MASK50) : cache_key(abc[3 * k], abc[3 * k + 1], abc[3 * k + 2]);
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
void launch_cache_load(Dev& d, int n, const int* abc, const unsigned long long* keys, const float* st,
                       cudaStream_t s) {
  k_cache_clear<<<148 * 4, 256, 0, s>>>(d);
  if (n > 0) k_cache_insert<<<148 * 2, 256, 0, s>>>(d, n, abc, keys, st);
}

}  // namespace avbd
