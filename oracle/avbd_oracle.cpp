// CPU oracle for the Solver6DOF substep -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++, the algorithm of the reference
// `Solver6DOF` substep (nanli9/AVBD, package avbd3d) row by row, the way the
// reference's Warp kernels run on Warp's CPU device (one thread after another
// in launch order).  It is the checker the GPU product is compared against:
// only the test-suite, `__graft_entry__.smoke()` and the `cpu_baseline` leg of
// `bench.py` load it.  The product library never links it.
//
// Every function cites the reference file:line it follows.  File paths are
// relative to the reference project root.
//
// Two precisions are built from one template: `float` (the reference's own
// storage type) and `double` (the FP64 replay used by the parity tests).  The
// collision pipeline (AABB, pair set, SAT, manifold) always runs in float on
// float copies of the pose, exactly like the reference, so that its discrete
// outputs can be compared bit-for-bit with the GPU.
//
// Defined semantics where the reference is order dependent (the GPU kernels
// implement the same ones):
//  * pair order: pairs are sorted by (min body, max body); rows are emitted in
//    pair order, contacts in manifold order;
//  * coloring: every Jones-Plassmann / speculative round reads the previous
//    round's colors (snapshot semantics);
//  * dual/prelude: rows are processed in ascending row order (Warp CPU order),
//    so a tangent row sees its normal row's freshly updated lambda;
//  * the body->row CSR is rebuilt every substep (the reference skips the
//    rebuild when the live row count is zero and keeps a stale CSR).
//
// Compile with -ffp-contract=off so float collision math matches the GPU's
// -fmad=false collision kernels operation for operation.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// Constraint type codes: solver_6dof.py:31-34, kernels_6dof.py:44-47.
enum { FLOOR = 0, TANGENT = 1, PIN = 2, BOXBOX = 3 };
// Penalty constants: kernels_6dof.py:50-52.
static const double PEN_MIN = 1.0e6, PEN_MIN_T = 1.0, PEN_MAX = 1.0e9;
// kernels_6dof.py:2582-2585.
static const int MAX_COLORS = 32, JP_ROUNDS = 24;
static const float MARGIN = 0.005f;  // solver_6dof.py:1789
static const float FINF = std::numeric_limits<float>::infinity();

template <class T> struct V3 { T x, y, z; };
template <class T> struct Q4 { T x, y, z, w; };
template <class T> struct M3 { T m[3][3]; };

template <class T> static inline V3<T> v3(T a, T b, T c) { return V3<T>{a, b, c}; }
template <class T> static inline V3<T> add(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> static inline V3<T> sub(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> static inline V3<T> mul(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> static inline V3<T> divs(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> static inline V3<T> neg(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> static inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> static inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> static inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> static inline T comp(V3<T> a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
template <class T> static inline T clampv(T x, T lo, T hi) { return std::min(std::max(x, lo), hi); }

// Hamilton product, XYZW storage (Warp convention, kernels_6dof.py:58-60).
template <class T> static inline Q4<T> qmul(Q4<T> a, Q4<T> b) {
  return {a.w * b.x + b.w * a.x + (a.y * b.z - a.z * b.y),
          a.w * b.y + b.w * a.y + (a.z * b.x - a.x * b.z),
          a.w * b.z + b.w * a.z + (a.x * b.y - a.y * b.x),
          a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z)};
}
template <class T> static inline Q4<T> qconj(Q4<T> q) { return {-q.x, -q.y, -q.z, q.w}; }
// Rotation of v by unit q: v' = (2w^2-1) v + 2 (q.v) q + 2 w (q x v).
template <class T> static inline V3<T> qrot(Q4<T> q, V3<T> v) {
  T c = T(2) * q.w * q.w - T(1);
  T d = T(2) * (q.x * v.x + q.y * v.y + q.z * v.z);
  T w2 = q.w * T(2);
  return {v.x * c + q.x * d + (q.y * v.z - q.z * v.y) * w2,
          v.y * c + q.y * d + (q.z * v.x - q.x * v.z) * w2,
          v.z * c + q.z * d + (q.x * v.y - q.y * v.x) * w2};
}
template <class T> static inline M3<T> qmat(Q4<T> q) {
  T x = q.x, y = q.y, z = q.z, w = q.w;
  M3<T> R;
  R.m[0][0] = T(1) - T(2) * (y * y + z * z);
  R.m[0][1] = T(2) * (x * y - z * w);
  R.m[0][2] = T(2) * (x * z + y * w);
  R.m[1][0] = T(2) * (x * y + z * w);
  R.m[1][1] = T(1) - T(2) * (x * x + z * z);
  R.m[1][2] = T(2) * (y * z - x * w);
  R.m[2][0] = T(2) * (x * z - y * w);
  R.m[2][1] = T(2) * (y * z + x * w);
  R.m[2][2] = T(1) - T(2) * (x * x + y * y);
  return R;
}
template <class T> static inline V3<T> col(const M3<T>& R, int k) { return {R.m[0][k], R.m[1][k], R.m[2][k]}; }
template <class T> static inline V3<T> mtv(const M3<T>& R, V3<T> v) {  // R^T v
  return {R.m[0][0] * v.x + R.m[1][0] * v.y + R.m[2][0] * v.z,
          R.m[0][1] * v.x + R.m[1][1] * v.y + R.m[2][1] * v.z,
          R.m[0][2] * v.x + R.m[1][2] * v.y + R.m[2][2] * v.z};
}
template <class T> static inline V3<T> mv(const M3<T>& A, V3<T> v) {
  return {A.m[0][0] * v.x + A.m[0][1] * v.y + A.m[0][2] * v.z,
          A.m[1][0] * v.x + A.m[1][1] * v.y + A.m[1][2] * v.z,
          A.m[2][0] * v.x + A.m[2][1] * v.y + A.m[2][2] * v.z};
}
template <class T> static inline M3<T> mm(const M3<T>& A, const M3<T>& B) {
  M3<T> C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C.m[i][j] = A.m[i][0] * B.m[0][j] + A.m[i][1] * B.m[1][j] + A.m[i][2] * B.m[2][j];
  return C;
}
template <class T> static inline M3<T> mt(const M3<T>& A) {
  M3<T> C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C.m[i][j] = A.m[j][i];
  return C;
}
template <class T> static inline M3<T> zero3() { M3<T> A; std::memset(&A, 0, sizeof(A)); return A; }
// 3x3 inverse by the adjugate; a singular matrix gives the zero matrix.
template <class T> static inline M3<T> inv3(const M3<T>& a) {
  const T(*m)[3] = a.m;
  T c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
  T c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  T c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  T det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
  M3<T> r = zero3<T>();
  if (det == T(0)) return r;
  T id = T(1) / det;
  r.m[0][0] = c00 * id;
  r.m[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
  r.m[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
  r.m[1][0] = c01 * id;
  r.m[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
  r.m[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
  r.m[2][0] = c02 * id;
  r.m[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
  r.m[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
  return r;
}
template <class T> static inline Q4<T> qnormalize(Q4<T> q) {
  T l = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  if (l > T(0)) { T s = T(1) / l; return {q.x * s, q.y * s, q.z * s, q.w * s}; }
  return q;
}
// kernels_6dof.py:63-73
template <class T> static inline Q4<T> quat_from_rotvec(V3<T> rv) {
  T th = length(rv);
  if (th < T(1.0e-9)) return {T(0.5) * rv.x, T(0.5) * rv.y, T(0.5) * rv.z, T(1)};
  T half = T(0.5) * th;
  T s = std::sin(half) / th;
  return {s * rv.x, s * rv.y, s * rv.z, std::cos(half)};
}
// kernels_6dof.py:76-97
template <class T> static inline V3<T> quat_to_rotvec(Q4<T> q) {
  T qw = q.w, qx = q.x, qy = q.y, qz = q.z;
  if (qw < T(0)) { qw = -qw; qx = -qx; qy = -qy; qz = -qz; }
  V3<T> qv{qx, qy, qz};
  T l = length(qv);
  if (l < T(1.0e-9)) return {T(0), T(0), T(0)};
  T ang = T(2) * std::atan2(l, qw);
  return mul(qv, ang / l);
}
// kernels_6dof.py:280-316
template <class T> static inline V3<T> geom_stiffness_diag(V3<T> n, V3<T> r) {
  T nr = dot(n, r);
  T h00 = n.x * r.x - nr, h10 = T(0.5) * (n.y * r.x + r.y * n.x), h20 = T(0.5) * (n.z * r.x + r.z * n.x);
  T h01 = T(0.5) * (n.x * r.y + r.x * n.y), h11 = n.y * r.y - nr, h21 = T(0.5) * (n.z * r.y + r.z * n.y);
  T h02 = T(0.5) * (n.x * r.z + r.x * n.z), h12 = T(0.5) * (n.y * r.z + r.y * n.z), h22 = n.z * r.z - nr;
  return {std::sqrt(h00 * h00 + h10 * h10 + h20 * h20), std::sqrt(h01 * h01 + h11 * h11 + h21 * h21),
          std::sqrt(h02 * h02 + h12 * h12 + h22 * h22)};
}
// kernels_6dof.py:2208-2218 (Duff et al. 2017)
static inline V3<float> orthonormal_basis(V3<float> n) {
  float sign = n.z >= 0.0f ? 1.0f : -1.0f;
  float a = -1.0f / (sign + n.z);
  float b = n.x * n.y * a;
  return {1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x};
}

// ---------------------------------------------------------------------------
// Collision pipeline (float).
// ---------------------------------------------------------------------------
struct PairOut {
  int a, b, overlap, sat_idx;
  V3<float> n;
  float depth;
  int count, ref_is_a;
  V3<float> nn, tt, bb;
  V3<float> off_ref[4], off_inc[4];
};

// kernels_6dof.py:1922-1943
static inline void aabb_of(V3<float> c, Q4<float> q, V3<float> he, V3<float>& lo, V3<float>& hi) {
  M3<float> R = qmat(q);
  float ex = std::fabs(R.m[0][0]) * he.x + std::fabs(R.m[0][1]) * he.y + std::fabs(R.m[0][2]) * he.z + MARGIN;
  float ey = std::fabs(R.m[1][0]) * he.x + std::fabs(R.m[1][1]) * he.y + std::fabs(R.m[1][2]) * he.z + MARGIN;
  float ez = std::fabs(R.m[2][0]) * he.x + std::fabs(R.m[2][1]) * he.y + std::fabs(R.m[2][2]) * he.z + MARGIN;
  lo = {c.x - ex, c.y - ey, c.z - ez};
  hi = {c.x + ex, c.y + ey, c.z + ez};
}

// kernels_6dof.py:1981-1988
static inline float proj_radius(V3<float> L, V3<float> c0, V3<float> c1, V3<float> c2, V3<float> he) {
  return he.x * std::fabs(dot(L, c0)) + he.y * std::fabs(dot(L, c1)) + he.z * std::fabs(dot(L, c2));
}

// kernels_6dof.py:1991-2130 (obb_sat_pairs)
static void sat(V3<float> cA, M3<float> RA, V3<float> eA, V3<float> cB, M3<float> RB, V3<float> eB, PairOut& o) {
  V3<float> t = sub(cB, cA);
  V3<float> A[3] = {col(RA, 0), col(RA, 1), col(RA, 2)};
  V3<float> B[3] = {col(RB, 0), col(RB, 1), col(RB, 2)};
  float best = 1.0e20f;
  int bi = -1;
  V3<float> ba{0, 0, 0};
  for (int k = 0; k < 3; ++k) {
    V3<float> L = A[k];
    float rA = comp(eA, k);
    float rB = proj_radius(L, B[0], B[1], B[2], eB);
    float tl = dot(t, L);
    float ov = rA + rB - std::fabs(tl);
    if (ov < -MARGIN) { o.overlap = 0; return; }
    if (ov < best) { best = ov; bi = k; ba = tl > 0.0f ? neg(L) : L; }
  }
  for (int k = 0; k < 3; ++k) {
    V3<float> L = B[k];
    float rA = proj_radius(L, A[0], A[1], A[2], eA);
    float rB = comp(eB, k);
    float tl = dot(t, L);
    float ov = rA + rB - std::fabs(tl);
    if (ov < -MARGIN) { o.overlap = 0; return; }
    if (ov < best) { best = ov; bi = 3 + k; ba = tl > 0.0f ? neg(L) : L; }
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      V3<float> L = cross(A[i], B[j]);
      float nl = length(L);
      if (nl < 1.0e-6f) continue;
      L = divs(L, nl);
      float rA = proj_radius(L, A[0], A[1], A[2], eA);
      float rB = proj_radius(L, B[0], B[1], B[2], eB);
      float tl = dot(t, L);
      float ov = rA + rB - std::fabs(tl);
      if (ov < 0.0f) { o.overlap = 0; return; }
      if (ov < best) { best = ov; bi = 6 + 3 * i + j; ba = tl > 0.0f ? neg(L) : L; }
    }
  o.overlap = 1;
  o.sat_idx = bi;
  o.n = ba;
  o.depth = best;
}

// kernels_6dof.py:2221-2537 (obb_contact_manifold_6dof)
static void manifold(V3<float> cA, M3<float> RA, V3<float> eA, V3<float> cB, M3<float> RB, V3<float> eB, PairOut& o) {
  o.count = 0;
  if (!o.overlap) return;
  int sat_idx = o.sat_idx;
  V3<float> nin = o.n;
  if (sat_idx >= 6) {
    int e = sat_idx - 6, kA = e / 3, kB = e % 3;
    V3<float> eAd = col(RA, kA), eBd = col(RB, kB);
    if (length(cross(eAd, eBd)) < 1.0e-4f) return;
    int kA1 = (kA + 1) % 3, kA2 = (kA + 2) % 3;
    V3<float> A1c = col(RA, kA1), A2c = col(RA, kA2);
    V3<float> toB = sub(cB, cA);
    float sbA = dot(toB, A1c) >= 0.0f ? 1.0f : -1.0f;
    float scA = dot(toB, A2c) >= 0.0f ? 1.0f : -1.0f;
    V3<float> midA = add(add(cA, mul(A1c, sbA * comp(eA, kA1))), mul(A2c, scA * comp(eA, kA2)));
    V3<float> P1 = sub(midA, mul(eAd, comp(eA, kA)));
    V3<float> Q1 = add(midA, mul(eAd, comp(eA, kA)));
    int kB1 = (kB + 1) % 3, kB2 = (kB + 2) % 3;
    V3<float> B1c = col(RB, kB1), B2c = col(RB, kB2);
    V3<float> toA = sub(cA, cB);
    float sbB = dot(toA, B1c) >= 0.0f ? 1.0f : -1.0f;
    float scB = dot(toA, B2c) >= 0.0f ? 1.0f : -1.0f;
    V3<float> midB = add(add(cB, mul(B1c, sbB * comp(eB, kB1))), mul(B2c, scB * comp(eB, kB2)));
    V3<float> P2 = sub(midB, mul(eBd, comp(eB, kB)));
    V3<float> Q2 = add(midB, mul(eBd, comp(eB, kB)));
    V3<float> d1 = sub(Q1, P1), d2 = sub(Q2, P2), r = sub(P1, P2);
    float a = dot(d1, d1), ev = dot(d2, d2), f = dot(d2, r);
    const float eps = 1.0e-12f;
    float s = 0.0f, tp = 0.0f;
    if (a <= eps && ev <= eps) {
      s = 0.0f; tp = 0.0f;
    } else if (a <= eps) {
      s = 0.0f; tp = clampv(f / std::max(ev, eps), 0.0f, 1.0f);
    } else if (ev <= eps) {
      tp = 0.0f; float c = dot(d1, r); s = clampv(-c / a, 0.0f, 1.0f);
    } else {
      float c = dot(d1, r), b = dot(d1, d2);
      float den = a * ev - b * b;
      s = den != 0.0f ? clampv((b * f - c * ev) / den, 0.0f, 1.0f) : 0.0f;
      tp = (b * s + f) / ev;
      if (tp < 0.0f) { tp = 0.0f; s = clampv(-c / a, 0.0f, 1.0f); }
      else if (tp > 1.0f) { tp = 1.0f; s = clampv((b - c) / a, 0.0f, 1.0f); }
    }
    V3<float> pA = add(P1, mul(d1, s)), pB = add(P2, mul(d2, tp));
    float gap = dot(sub(pA, pB), nin);
    if (gap > MARGIN) return;
    V3<float> t_hat = orthonormal_basis(nin);
    o.count = 1;
    o.ref_is_a = 1;
    o.nn = nin;
    o.tt = t_hat;
    o.bb = cross(nin, t_hat);
    o.off_ref[0] = mtv(RA, sub(pA, cA));
    o.off_inc[0] = mtv(RB, sub(pB, cB));
    return;
  }
  int ref_is_a = sat_idx < 3 ? 1 : 0;
  o.ref_is_a = ref_is_a;
  int ref_axis;
  V3<float> nu, ref_c, inc_c, e_ref, e_inc;
  M3<float> Rr, Ri;
  if (sat_idx < 3) {
    ref_axis = sat_idx; nu = nin; ref_c = cA; Rr = RA; e_ref = eA; inc_c = cB; Ri = RB; e_inc = eB;
  } else {
    ref_axis = sat_idx - 3; nu = neg(nin); ref_c = cB; Rr = RB; e_ref = eB; inc_c = cA; Ri = RA; e_inc = eA;
  }
  V3<float> rca = col(Rr, ref_axis);
  float rsign = dot(rca, nu) > 0.0f ? -1.0f : 1.0f;
  V3<float> rfn = mul(rca, rsign);
  V3<float> rfc = add(ref_c, mul(rfn, comp(e_ref, ref_axis)));
  int ax1 = (ref_axis + 1) % 3, ax2 = (ref_axis + 2) % 3;
  V3<float> u = col(Rr, ax1), v = col(Rr, ax2);
  float eu = comp(e_ref, ax1), evv = comp(e_ref, ax2);
  int ia = 0;
  float isg = 1.0f, bd = -1.0e20f;
  for (int k = 0; k < 3; ++k) {
    float dp = dot(col(Ri, k), nu);
    if (dp > bd) { bd = dp; ia = k; isg = 1.0f; }
    float dn = -dp;
    if (dn > bd) { bd = dn; ia = k; isg = -1.0f; }
  }
  V3<float> ifn = mul(col(Ri, ia), isg);
  V3<float> ifc = add(inc_c, mul(ifn, comp(e_inc, ia)));
  int ia1 = (ia + 1) % 3, ia2 = (ia + 2) % 3;
  V3<float> iu = col(Ri, ia1), iv = col(Ri, ia2);
  float ieu = comp(e_inc, ia1), iev = comp(e_inc, ia2);
  V3<float> poly[2][8];
  int cur = 0;
  poly[0][0] = add(add(ifc, mul(iu, ieu)), mul(iv, iev));
  poly[0][1] = add(sub(ifc, mul(iu, ieu)), mul(iv, iev));
  poly[0][2] = sub(sub(ifc, mul(iu, ieu)), mul(iv, iev));
  poly[0][3] = sub(add(ifc, mul(iu, ieu)), mul(iv, iev));
  int len = 4;
  for (int pl = 0; pl < 4; ++pl) {
    V3<float> pp, pn;
    if (pl == 0) { pp = add(rfc, mul(u, eu)); pn = u; }
    else if (pl == 1) { pp = sub(rfc, mul(u, eu)); pn = neg(u); }
    else if (pl == 2) { pp = add(rfc, mul(v, evv)); pn = v; }
    else { pp = sub(rfc, mul(v, evv)); pn = neg(v); }
    if (len == 0) return;
    int ol = 0;
    int nx = cur ^ 1;
    for (int iv_ = 0; iv_ < len; ++iv_) {
      V3<float> ap = poly[cur][iv_];
      V3<float> bp = poly[cur][(iv_ + 1) % len];
      float da = dot(sub(ap, pp), pn);
      float db = dot(sub(bp, pp), pn);
      if (da <= 0.0f) {
        if (ol < 8) poly[nx][ol++] = ap;
        if (db > 0.0f) {
          float tt = da / (da - db);
          if (ol < 8) poly[nx][ol++] = add(ap, mul(sub(bp, ap), tt));
        }
      } else if (db <= 0.0f) {
        float tt = da / (da - db);
        if (ol < 8) poly[nx][ol++] = add(ap, mul(sub(bp, ap), tt));
      }
    }
    cur = nx;
    len = ol;
  }
  if (len == 0) return;
  float bdp[4] = {-1.0e30f, -1.0e30f, -1.0e30f, -1.0e30f};
  int bidx[4] = {-1, -1, -1, -1};
  int nb = 0;
  for (int iv_ = 0; iv_ < len; ++iv_) {
    float ds = dot(sub(poly[cur][iv_], rfc), rfn);
    if (ds < MARGIN) {
      float depth = -ds;
      if (nb < 4) { bdp[nb] = depth; bidx[nb] = iv_; ++nb; }
      else {
        int mp = 0;
        float mvv = bdp[0];
        for (int k = 1; k < 4; ++k)
          if (bdp[k] < mvv) { mvv = bdp[k]; mp = k; }
        if (depth > mvv) { bdp[mp] = depth; bidx[mp] = iv_; }
      }
    }
  }
  if (nb == 0) return;
  for (int i = 0; i < nb - 1; ++i) {
    int mp = i;
    for (int k = i + 1; k < nb; ++k)
      if (bdp[k] > bdp[mp]) mp = k;
    if (mp != i) { std::swap(bdp[i], bdp[mp]); std::swap(bidx[i], bidx[mp]); }
  }
  V3<float> t_hat = orthonormal_basis(nu);
  o.nn = nu;
  o.tt = t_hat;
  o.bb = cross(nu, t_hat);
  o.count = nb;
  for (int c = 0; c < nb; ++c) {
    V3<float> pi = poly[cur][bidx[c]];
    float ds = dot(sub(pi, rfc), rfn);
    V3<float> pr = sub(pi, mul(rfn, ds));
    o.off_ref[c] = mtv(Rr, sub(pr, ref_c));
    o.off_inc[c] = mtv(Ri, sub(pi, inc_c));
  }
}

// Contact-cache key (a, b, contact ordinal), 64-bit: (a << 26) | (b << 2) | c.
// The reference packs (a*16384+b)*4+c into int32 (kernels_6dof.py:2588-2594),
// which wraps above 16383 bodies; the 64-bit key is the intended mapping.
static inline uint64_t pair_key(int a, int b, int c) {
  return ((uint64_t)(uint32_t)a << 26) | ((uint64_t)(uint32_t)b << 2) | (uint64_t)c;
}

// The 5 mm anchor key (documented cache of the reference,
// PERFORMANCE_PROGRESS.md:122-125): bodies a < b and the contact point in
// a's body frame rounded to 5 mm (round half to even), folded into 50 bits
// with a 64-bit finalizer; a later contact of the same pair in the same
// cells is rehashed with its ordinal.  Same arithmetic as the device.
static inline uint64_t mix64(uint64_t z) {
  z ^= z >> 31;
  z *= 0x7fb5d329728ea185ull;
  z ^= z >> 27;
  z *= 0x81dadef4bc2dd44dull;
  z ^= z >> 33;
  return z;
}
static inline int quant_5mm(float x) {
  float s = x * 200.0f;
  int q = (int)std::nearbyint(s);
  return q < -32767 ? -32767 : (q > 32767 ? 32767 : q);
}
static const uint64_t KEY_MASK50 = (1ull << 50) - 1ull;
static inline uint64_t anchor_key(int a, int b, V3<float> o) {
  uint64_t k1 = ((uint64_t)(uint32_t)a << 32) | (uint64_t)(uint32_t)b;
  uint64_t k2 = ((uint64_t)(uint16_t)(int16_t)quant_5mm(o.x) << 32) | ((uint64_t)(uint16_t)(int16_t)quant_5mm(o.y) << 16) |
                (uint64_t)(uint16_t)(int16_t)quant_5mm(o.z);
  return mix64(k1 ^ mix64(k2 + 0x9E3779B97F4A7C15ull)) & KEY_MASK50;
}

// ---------------------------------------------------------------------------
// The simulation state.
// ---------------------------------------------------------------------------
template <class R> struct Sim {
  // parameters (solver_6dof.py:180-304)
  R dt = R(1.0 / 60.0);
  int iterations = 10;
  V3<R> g{0, R(-9.81), 0};
  R alpha = R(0.99), beta = R(1e5), gamma = R(0.99);
  int post_stab = 1;
  R max_lin = R(30), max_ang = R(50);
  int substeps = 1;
  float fsm = 1.5f;
  int color_mode = 0;  // 0 = jacobi, 1 = jones_plassmann
  int recolor_every = 0;
  int self_collide = 0;
  float self_friction = 0.0f;
  int threads = 1;

  // bodies
  int nb = 0;
  std::vector<V3<R>> x, v, w, pv, pw, x0, xin;
  std::vector<Q4<R>> q, q0, qin;
  std::vector<M3<R>> Iw;
  std::vector<float> mass, fric, prio;
  std::vector<V3<float>> he, Iloc;  // box inertia is diagonal (solver_6dof.py:132-142)

  // rows: static prefix [0, n_static), dynamic tail up to cap
  int n_static = 0, cap = 0, n_rows = 0;
  long long n_rows_reserved = 0;
  int pair_cap = 0;
  long long pairs_found = 0;
  std::vector<int> type, ba, bb, sib, par;
  std::vector<V3<float>> anchor, offa, offb;
  std::vector<float> stiff, fract, fmin, fmax, mu, mus;
  std::vector<R> lam, pen, ac0;
  std::vector<int> active, was;

  // contact cache
  struct Entry { R s[8]; };
  std::unordered_map<uint64_t, Entry> cache;
  struct Pool { int n, t, b, c; uint64_t key; };
  int key_mode = 0;  // 0: (a, b, ordinal) keys; 1: 5 mm anchor keys
  std::vector<Pool> pool;

  // coloring
  std::vector<int> color;
  int n_colors = 1;
  int color_dirty = 1;
  int recolored_last = 0;
  std::vector<int> color_starts, color_bodies;

  // CSR body -> rows
  std::vector<int> csr_start, csr_idx;

  // debug outputs of the last substep
  std::vector<PairOut> pairs;
  std::vector<int> row_c;  // contact ordinal of each dynamic normal row (-1 otherwise)
  // per-iteration max violation of the last substep
  std::vector<double> viol;
  int record_viol = 0;

  void resize_rows(int c) {
    cap = c;
    type.resize(c, 0); ba.resize(c, -1); bb.resize(c, -1); sib.resize(c, -1); par.resize(c, -1);
    anchor.resize(c, {0, 0, 0}); offa.resize(c, {0, 0, 0}); offb.resize(c, {0, 0, 0});
    stiff.resize(c, 0); fract.resize(c, 0); fmin.resize(c, 0); fmax.resize(c, 0); mu.resize(c, 0); mus.resize(c, 0);
    lam.resize(c, 0); pen.resize(c, 1); ac0.resize(c, 0); active.resize(c, 0); was.resize(c, 0);
    row_c.resize(c, -1);
  }

  // ---- collision: solver_6dof.py:1774-1916 --------------------------------
  void collide() {
    pairs.clear();
    pool.clear();
    pairs_found = 0;
    if (!(self_collide && nb >= 2)) return;
    std::vector<V3<float>> lo(nb), hi(nb), cf(nb);
    std::vector<Q4<float>> qf(nb);
    for (int i = 0; i < nb; ++i) {
      cf[i] = {(float)x[i].x, (float)x[i].y, (float)x[i].z};
      qf[i] = {(float)q[i].x, (float)q[i].y, (float)q[i].z, (float)q[i].w};
      aabb_of(cf[i], qf[i], he[i], lo[i], hi[i]);
    }
    // Pair set: every i<j whose AABBs overlap (closed intervals), skipping
    // static-static (kernels_6dof.py:1946-1978).  Sweep along x.
    std::vector<int> ord(nb);
    for (int i = 0; i < nb; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return lo[a].x < lo[b].x || (lo[a].x == lo[b].x && a < b); });
    std::vector<std::pair<int, int>> pl;
    for (int s = 0; s < nb; ++s) {
      int i = ord[s];
      for (int u = s + 1; u < nb; ++u) {
        int j = ord[u];
        if (lo[j].x > hi[i].x) break;
        if (lo[i].x <= hi[j].x && lo[i].y <= hi[j].y && lo[j].y <= hi[i].y && lo[i].z <= hi[j].z && lo[j].z <= hi[i].z) {
          if (mass[i] <= 0.0f && mass[j] <= 0.0f) continue;
          pl.push_back({std::min(i, j), std::max(i, j)});
        }
      }
    }
    std::sort(pl.begin(), pl.end());
    pairs_found = (long long)pl.size();
    if ((int)pl.size() > pair_cap) pl.resize(pair_cap);
    pairs.resize(pl.size());
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long p = 0; p < (long)pl.size(); ++p) {
      PairOut& o = pairs[p];
      o.a = pl[p].first; o.b = pl[p].second;
      o.count = 0; o.sat_idx = -1; o.ref_is_a = 0;
      M3<float> RA = qmat(qf[o.a]), RB = qmat(qf[o.b]);
      sat(cf[o.a], RA, he[o.a], cf[o.b], RB, he[o.b], o);
      manifold(cf[o.a], RA, he[o.a], cf[o.b], RB, he[o.b], o);
    }
    // Row emission (kernels_6dof.py:2695-2912), pair order.
    long long nr = n_rows;
    for (size_t p = 0; p < pairs.size(); ++p) {
      const PairOut& o = pairs[p];
      if (o.count == 0) continue;
      int ref = o.ref_is_a ? o.a : o.b, inc = o.ref_is_a ? o.b : o.a;
      float mr = fric[ref], mi = fric[inc];
      float m = self_friction;
      if (mr > 0.0f || mi > 0.0f) m = std::sqrt(mr * mi);
      float ms = m * fsm;
      int ka = std::min(ref, inc), kb = std::max(ref, inc);
      uint64_t keys[4];
      for (int c = 0; c < o.count; ++c) {
        if (key_mode) {
          uint64_t k = anchor_key(ka, kb, ka == ref ? o.off_ref[c] : o.off_inc[c]);
          for (int c2 = 0; c2 < c; ++c2)
            if (keys[c2] == k) k = mix64(k + (uint64_t)(c + 1)) & KEY_MASK50;
          keys[c] = k;
        } else {
          keys[c] = pair_key(ka, kb, c);
        }
      }
      for (int c = 0; c < o.count; ++c) {
        int rpc = m <= 0.0f ? 1 : 3;
        long long base = nr;
        nr += rpc;
        if (base + rpc > cap) break;  // capacity guard (:2799-2800)
        int n = (int)base;
        auto setrow = [&](int r, int ty, V3<float> an, float fmn, float fmx, int sb, int pr, float mu_, float mus_) {
          type[r] = ty; ba[r] = ref; bb[r] = inc; anchor[r] = an; offa[r] = o.off_ref[c]; offb[r] = o.off_inc[c];
          stiff[r] = FINF; fmin[r] = fmn; fmax[r] = fmx; ac0[r] = 0; active[r] = 1; fract[r] = FINF;
          sib[r] = sb; par[r] = pr; mu[r] = mu_; mus[r] = mus_; row_c[r] = -1;
        };
        setrow(n, BOXBOX, o.nn, -FINF, 0.0f, -1, -1, 0.0f, 0.0f);
        row_c[n] = c;
        int t = -1, b = -1;
        if (m > 0.0f) {
          t = n + 1; b = n + 2;
          setrow(t, TANGENT, o.tt, -FINF, FINF, n, b, m, ms);
          setrow(b, TANGENT, o.bb, -FINF, FINF, n, t, m, ms);
        }
        R s[8] = {0, 0, 0, R(PEN_MIN), R(PEN_MIN_T), R(PEN_MIN_T), 0, 0};
        auto it = cache.find(keys[c]);
        if (it != cache.end())
          for (int k = 0; k < 8; ++k) s[k] = it->second.s[k];
        lam[n] = s[0]; pen[n] = s[3]; was[n] = 0;
        if (t >= 0) { lam[t] = s[1]; pen[t] = s[4]; was[t] = (int)s[6]; }
        if (b >= 0) { lam[b] = s[2]; pen[b] = s[5]; was[b] = (int)s[7]; }
        pool.push_back({n, t, b, c, keys[c]});
      }
    }
    n_rows_reserved = nr;
    n_rows = (int)std::min<long long>(nr, cap);
  }

  // ---- coloring: solver_6dof.py:680-862, kernels_6dof.py:3022-3336 ------
  bool edge_row(int j) const {
    if (type[j] == PIN) return false;
    int a = ba[j], b = bb[j];
    return !(a < 0 || b < 0 || a == b);
  }
  long conflicts() const {
    long c = 0;
    for (int j = 0; j < n_rows; ++j)
      if (edge_row(j) && color[ba[j]] == color[bb[j]]) ++c;
    return c;
  }
  void recolor() {
    std::vector<int> ns(nb + 1, 0), nidx;
    for (int j = 0; j < n_rows; ++j)
      if (edge_row(j)) { ns[ba[j] + 1]++; ns[bb[j] + 1]++; }
    for (int i = 0; i < nb; ++i) ns[i + 1] += ns[i];
    nidx.resize(ns[nb]);
    std::vector<int> cur(ns.begin(), ns.end() - 1);
    for (int j = 0; j < n_rows; ++j)
      if (edge_row(j)) { nidx[cur[ba[j]]++] = bb[j]; nidx[cur[bb[j]]++] = ba[j]; }
    std::vector<int> c(nb, -1), nx(nb);
    auto first_fit = [&](int i, const std::vector<int>& snap) {
      uint32_t used = 0;
      for (int k = ns[i]; k < ns[i + 1]; ++k) {
        int cc = snap[nidx[k]];
        if (cc >= 0 && cc < MAX_COLORS) used |= (1u << cc);
      }
      int ch = MAX_COLORS - 1;
      for (int cc = 0; cc < MAX_COLORS; ++cc)
        if (!(used & (1u << cc))) { ch = cc; break; }
      return ch;
    };
    if (color_mode == 1) {  // Jones-Plassmann (kernels_6dof.py:3099-3148)
      for (int r = 0; r < JP_ROUNDS; ++r) {
        bool any = false;
        for (int i = 0; i < nb; ++i) {
          nx[i] = c[i];
          if (c[i] != -1) continue;
          any = true;
          float my = prio[i];
          bool win = true;
          for (int k = ns[i]; k < ns[i + 1] && win; ++k) {
            int nbr = nidx[k];
            if (c[nbr] == -1 && prio[nbr] >= my && (prio[nbr] > my || nbr < i)) win = false;
          }
          if (win) nx[i] = first_fit(i, c);
        }
        if (!any) break;
        c.swap(nx);
      }
    } else {  // speculative jacobi (kernels_6dof.py:3233-3296, solver_6dof.py:795-844)
      for (int r = 0; r < MAX_COLORS; ++r) {
        std::vector<int> as(c);
        for (int i = 0; i < nb; ++i)
          if (c[i] == -1) as[i] = first_fit(i, c);
        int unc = 0;
        for (int i = 0; i < nb; ++i) {
          int ci = as[i];
          nx[i] = ci;
          if (ci >= 0) {
            float my = prio[i];
            for (int k = ns[i]; k < ns[i + 1]; ++k) {
              int nbr = nidx[k];
              if (as[nbr] == ci && (prio[nbr] > my || (prio[nbr] == my && nbr < i))) { nx[i] = -1; break; }
            }
          }
          if (nx[i] == -1) ++unc;
        }
        c.swap(nx);
        if (unc == 0) break;
      }
    }
    int mx = 0;
    for (int i = 0; i < nb; ++i) {
      if (c[i] == -1) c[i] = 0;  // gpu_color_finalize (:3151-3165)
      mx = std::max(mx, c[i]);
    }
    color = c;
    n_colors = std::max(1, std::min(mx + 1, MAX_COLORS));
    color_dirty = 0;
  }
  void bucket_colors() {
    color_starts.assign(MAX_COLORS + 1, 0);
    for (int i = 0; i < nb; ++i) color_starts[color[i] + 1]++;
    for (int k = 0; k < MAX_COLORS; ++k) color_starts[k + 1] += color_starts[k];
    color_bodies.resize(nb);
    std::vector<int> cur(color_starts.begin(), color_starts.end() - 1);
    for (int i = 0; i < nb; ++i) color_bodies[cur[color[i]]++] = i;
  }

  // ---- body->row CSR: kernels_6dof.py:2626-2692 (ascending row order) ----
  void build_csr() {
    csr_start.assign(nb + 1, 0);
    for (int j = 0; j < n_rows; ++j) {
      if (ba[j] >= 0) csr_start[ba[j] + 1]++;
      if (type[j] != PIN && bb[j] >= 0) csr_start[bb[j] + 1]++;
    }
    for (int i = 0; i < nb; ++i) csr_start[i + 1] += csr_start[i];
    csr_idx.resize(csr_start[nb]);
    std::vector<int> cur(csr_start.begin(), csr_start.end() - 1);
    for (int j = 0; j < n_rows; ++j) {
      if (ba[j] >= 0) csr_idx[cur[ba[j]]++] = j;
      if (type[j] != PIN && bb[j] >= 0) csr_idx[cur[bb[j]]++] = j;
    }
  }

  // ---- predict: kernels_6dof.py:122-187 ----------------------------------
  void predict() {
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int i = 0; i < nb; ++i) {
      R m = (R)mass[i];
      x0[i] = x[i];
      q0[i] = q[i];
      M3<R> Rm = qmat(q[i]);
      M3<R> I = zero3<R>();
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          I.m[a][b] = Rm.m[a][0] * (R)Iloc[i].x * Rm.m[b][0] + Rm.m[a][1] * (R)Iloc[i].y * Rm.m[b][1] +
                      Rm.m[a][2] * (R)Iloc[i].z * Rm.m[b][2];
      Iw[i] = I;
      if (m <= R(0)) { xin[i] = x[i]; qin[i] = q[i]; continue; }
      V3<R> gdt2 = mul(g, dt * dt);
      xin[i] = add(add(x[i], mul(v[i], dt)), gdt2);
      Q4<R> dq = quat_from_rotvec(mul(w[i], dt));
      qin[i] = qmul(dq, q[i]);
      V3<R> acc = divs(sub(v[i], pv[i]), dt);
      R gn = length(g);
      R wgt = 0;
      if (gn > R(0)) {
        V3<R> gh = divs(g, gn);
        wgt = clampv(dot(acc, gh) / gn, R(0), R(1));
      }
      x[i] = add(add(x[i], mul(v[i], dt)), mul(gdt2, wgt));
      q[i] = qmul(dq, q[i]);
    }
  }

  // ---- constraint value of row j at pose (xs, qs) ----------------------
  R eval_C(int j, const std::vector<V3<R>>& xs, const std::vector<Q4<R>>& qs) const {
    int t = type[j], a = ba[j];
    V3<R> an{(R)anchor[j].x, (R)anchor[j].y, (R)anchor[j].z};
    V3<R> oa{(R)offa[j].x, (R)offa[j].y, (R)offa[j].z};
    if (t == FLOOR) return add(xs[a], qrot(qs[a], oa)).y - an.y;
    if (t == PIN) {
      V3<R> p = add(xs[a], qrot(qs[a], oa));
      int ax = bb[j];
      return ax == 0 ? p.x - an.x : (ax == 1 ? p.y - an.y : p.z - an.z);
    }
    V3<R> ra = add(xs[a], qrot(qs[a], oa));
    if (t == TANGENT && bb[j] < 0) return dot(an, ra);
    V3<R> ob{(R)offb[j].x, (R)offb[j].y, (R)offb[j].z};
    V3<R> rb = add(xs[bb[j]], qrot(qs[bb[j]], ob));
    return dot(an, sub(ra, rb));
  }

  // ---- prelude: kernels_6dof.py:1565-1672 --------------------------------
  // Rows of one contact (normal + its tangents) are consecutive; they are
  // processed by one worker in row order so a tangent sees the partner row
  // exactly as Warp's serial CPU launch leaves it.
  void prelude_row(int j, R main_alpha) {
    R kf = type[j] == TANGENT ? R(PEN_MIN_T) : R(PEN_MIN);
    R p = clampv(pen[j] * gamma, kf, R(PEN_MAX));
    if (!post_stab) lam[j] = lam[j] * alpha * gamma;
    float s = stiff[j];
    if (!std::isnan(s) && s < FINF) p = std::min(p, (R)s);
    pen[j] = p;
    if (type[j] == TANGENT && active[j]) {
      int sb = sib[j];
      if (sb >= 0 && active[sb]) {
        int pr = par[j];
        if (pr < 0 || pr >= j) {
          R ln = std::fabs(lam[sb]);
          if (ln < R(1.0e-9)) was[sb] = 0;
          else {
            R lt = lam[j], lb = pr >= 0 ? lam[pr] : R(0);
            R ltb = std::sqrt(lt * lt + lb * lb);
            was[sb] = ltb <= (R)mus[j] * ln ? 1 : 0;
          }
        }
      }
    }
    if (!active[j]) { ac0[j] = 0; return; }
    R C0 = eval_C(j, x0, q0);
    if (type[j] == TANGENT) { ac0[j] = C0; return; }
    bool uni = type[j] == FLOOR || type[j] == BOXBOX;
    ac0[j] = (uni && C0 > R(0)) ? R(0) : main_alpha * C0;
  }

  // ---- post-stabilization alpha*C0 with alpha = 0: kernels_6dof.py:1733-1811
  void cache_ac0_zero() {
    for (int j = 0; j < n_rows; ++j) {
      if (!active[j]) { ac0[j] = 0; continue; }
      R C0 = eval_C(j, x0, q0);
      if (type[j] == TANGENT) { ac0[j] = C0; continue; }
      bool uni = type[j] == FLOOR || type[j] == BOXBOX;
      ac0[j] = (uni && C0 > R(0)) ? R(0) : R(0) * C0;
    }
  }

  // ---- primal: kernels_6dof.py:322-582 (serial, in place) ---------------
  void primal_body(int i) {
    R m = (R)mass[i];
    if (m <= R(0)) return;
    R idt2 = R(1) / (dt * dt);
    const M3<R>& I = Iw[i];
    M3<R> A = zero3<R>(), B = zero3<R>(), D;
    A.m[0][0] = A.m[1][1] = A.m[2][2] = m * idt2;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) D.m[a][b] = I.m[a][b] * idt2;
    V3<R> rl = mul(sub(x[i], xin[i]), m * idt2);
    V3<R> dth = quat_to_rotvec(qmul(q[i], qconj(qin[i])));
    V3<R> ra = mv(I, mul(dth, idt2));
    Q4<R> qi = q[i];
    V3<R> xi = x[i];
    for (int k = csr_start[i]; k < csr_start[i + 1]; ++k) {
      int j = csr_idx[k];
      if (!active[j]) continue;
      int t = type[j];
      float s = stiff[j];
      R kp = pen[j];
      V3<R> oa{(R)offa[j].x, (R)offa[j].y, (R)offa[j].z};
      V3<R> an{(R)anchor[j].x, (R)anchor[j].y, (R)anchor[j].z};
      V3<R> jl{0, 0, 0}, ja{0, 0, 0}, rs{0, 0, 0}, nG{0, 0, 0};
      R C = 0;
      if (t == FLOOR) {
        rs = qrot(qi, oa);
        V3<R> n{0, 1, 0};
        jl = n; ja = cross(rs, n);
        C = (xi.y + rs.y) - an.y;
        nG = n;
      } else if (t == TANGENT || t == BOXBOX) {
        int b = bb[j];
        if (t == TANGENT && b < 0) {
          rs = qrot(qi, oa);
          jl = an; ja = cross(rs, an);
          C = dot(an, add(xi, rs));
        } else {
          int a = ba[j];
          V3<R> ob{(R)offb[j].x, (R)offb[j].y, (R)offb[j].z};
          if (a == i) {
            rs = qrot(qi, oa);
            V3<R> ro = qrot(q[b], ob);
            C = dot(an, sub(add(xi, rs), add(x[b], ro)));
            jl = an; ja = cross(rs, an);
          } else {
            V3<R> ro = qrot(q[a], oa);
            rs = qrot(qi, ob);
            C = dot(an, sub(add(x[a], ro), add(xi, rs)));
            jl = neg(an); ja = neg(cross(rs, an));
          }
        }
        nG = an;
      } else if (t == PIN) {
        int ax = bb[j];
        rs = qrot(qi, oa);
        V3<R> p = add(xi, rs);
        V3<R> n{0, 0, 0};
        if (ax == 0) { n = {1, 0, 0}; C = p.x - an.x; }
        else if (ax == 1) { n = {0, 1, 0}; C = p.y - an.y; }
        else { n = {0, 0, 1}; C = p.z - an.z; }
        jl = n; ja = cross(rs, n); nG = n;
      }
      bool hard = s >= FINF;
      if (hard) C = C - ac0[j];
      R le = hard ? lam[j] : R(0);
      R lp = kp * C + le;
      R lo, hi;
      if (t == TANGENT) {
        int sb = sib[j];
        R muv = was[sb] != 0 ? (R)mus[j] : (R)mu[j];
        R bound = muv * std::fabs(lam[sb]);
        lo = -bound; hi = bound;
      } else { lo = (R)fmin[j]; hi = (R)fmax[j]; }
      R f = clampv(lp, lo, hi);
      R kl = kp;
      R aC = std::fabs(C);
      if (aC > R(1.0e-12)) {
        if (lp < lo) kl = std::fabs(lo - lp) / aC;
        else if (lp > hi) kl = std::fabs(hi - lp) / aC;
      }
      R jlv[3] = {jl.x, jl.y, jl.z}, jav[3] = {ja.x, ja.y, ja.z};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          A.m[a][b] += jlv[a] * jlv[b] * kl;
          B.m[a][b] += jav[a] * jlv[b] * kl;
          D.m[a][b] += jav[a] * jav[b] * kl;
        }
      R fm = std::fabs(f);
      if (fm > R(0)) {
        V3<R> gd = mul(geom_stiffness_diag(nG, rs), fm);
        D.m[0][0] += gd.x; D.m[1][1] += gd.y; D.m[2][2] += gd.z;
      }
      rl = add(rl, mul(jl, f));
      ra = add(ra, mul(ja, f));
    }
    M3<R> Ai = inv3(A);
    M3<R> BAi = mm(B, Ai);
    V3<R> rth = sub(ra, mv(BAi, rl));
    M3<R> S = D;
    M3<R> BABt = mm(BAi, mt(B));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) S.m[a][b] -= BABt.m[a][b];
    V3<R> dth2 = mv(inv3(S), rth);
    V3<R> dx = mv(Ai, sub(rl, mv(mt(B), dth2)));
    x[i] = sub(x[i], dx);
    q[i] = qnormalize(qmul(quat_from_rotvec(neg(dth2)), q[i]));
  }

  // ---- dual: kernels_6dof.py:1451-1548 -----------------------------------
  void dual_row(int j) {
    if (!active[j]) return;
    int t = type[j];
    R C = eval_C(j, x, q);
    float s = stiff[j];
    if (s >= FINF) C = C - ac0[j];
    R le = s >= FINF ? lam[j] : R(0);
    R lo = (R)fmin[j], hi = (R)fmax[j];
    bool tan = t == TANGENT;
    int sb = -1;
    bool used_static = false;
    if (tan) {
      sb = sib[j];
      R muv = (R)mu[j];
      if (was[sb] != 0) { muv = (R)mus[j]; used_static = true; }
      R bound = muv * std::fabs(lam[sb]);
      lo = -bound; hi = bound;
    }
    R nl = clampv(pen[j] * C + le, lo, hi);
    lam[j] = nl;
    if (std::fabs(nl) >= (R)fract[j]) { active[j] = 0; lam[j] = 0; pen[j] = 0; return; }
    if (nl > lo && nl < hi) {
      R up = std::min(R(PEN_MAX), (R)s);
      pen[j] = std::min(pen[j] + beta * std::fabs(C), up);
    } else if (tan && used_static) {
      was[sb] = 0;
    }
  }

  // Max constraint violation: max(0,-C) for unilateral rows, |C| for pins,
  // C being the value the dual update drives (kernels_6dof.py:1484-1507):
  // hard rows are measured relative to their stored alpha*C0.
  double violation() const {
    double mx = 0;
    for (int j = 0; j < n_rows; ++j) {
      if (!active[j]) continue;
      int t = type[j];
      if (t == TANGENT) continue;
      double C = (double)eval_C(j, x, q);
      if (stiff[j] >= FINF) C -= (double)ac0[j];
      double vv = t == PIN ? std::fabs(C) : std::max(0.0, -C);
      mx = std::max(mx, vv);
    }
    return mx;
  }

  // ---- finalize: kernels_6dof.py:1871-1901 ----------------------------------
  void finalize() {
    R ml = max_lin, ma = max_ang;
    if (!(ml > R(0) && std::isfinite((double)ml) && ma > R(0) && std::isfinite((double)ma))) {
      ml = std::numeric_limits<R>::infinity(); ma = ml;
    }
    for (int i = 0; i < nb; ++i) {
      pv[i] = v[i]; pw[i] = w[i];
      if (mass[i] > 0.0f) {
        V3<R> nv = divs(sub(x[i], x0[i]), dt);
        V3<R> nw = divs(quat_to_rotvec(qmul(q[i], qconj(q0[i]))), dt);
        R sl = length(nv);
        if (sl > ml) nv = mul(nv, ml / sl);
        R sa = length(nw);
        if (sa > ma) nw = mul(nw, ma / sa);
        v[i] = nv; w[i] = nw;
      }
    }
  }

  // ---- contact-cache refresh: kernels_6dof.py:2915-2995 -------------------
  void hash_collect() {
    if (!self_collide) return;
    cache.clear();
    for (const Pool& p : pool) {
      if (!active[p.n]) continue;
      Entry e;
      e.s[0] = lam[p.n]; e.s[3] = pen[p.n];
      e.s[1] = 0; e.s[2] = 0; e.s[4] = R(PEN_MIN_T); e.s[5] = R(PEN_MIN_T); e.s[6] = 0; e.s[7] = 0;
      if (p.t >= 0) { e.s[1] = lam[p.t]; e.s[4] = pen[p.t]; e.s[6] = (R)was[p.t]; }
      if (p.b >= 0) { e.s[2] = lam[p.b]; e.s[5] = pen[p.b]; e.s[7] = (R)was[p.b]; }
      cache[p.key] = e;
    }
  }

  // Group leaders: rows that are not tangents; the tangents of a leader
  // follow it directly (solver_6dof.py:488-539, kernels_6dof.py:2795-2862).
  std::vector<int> leaders;
  void build_leaders() {
    leaders.clear();
    for (int j = 0; j < n_rows; ++j)
      if (type[j] != TANGENT || sib[j] < 0) leaders.push_back(j);
  }
  template <class F> void over_groups(F fn) {
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long u = 0; u < (long)leaders.size(); ++u) {
      int j0 = leaders[u];
      int j1 = (u + 1 < (long)leaders.size()) ? leaders[u + 1] : n_rows;
      for (int j = j0; j < j1; ++j) fn(j);
    }
  }

  // ---- one substep: solver_6dof.py:1232-1464 --------------------------------
  void substep() {
    if (nb == 0) return;
    n_rows = n_static;
    collide();
    recolored_last = 0;
    bool need = color_dirty || recolor_every || conflicts() > 0;
    if (need) { recolor(); recolored_last = 1; }
    bucket_colors();
    build_csr();
    predict();
    build_leaders();
    R main_alpha = post_stab ? R(1) : alpha;
    over_groups([&](int j) { prelude_row(j, main_alpha); });
    int total = iterations + (post_stab ? 1 : 0);
    viol.clear();
    for (int it = 0; it < total; ++it) {
      if (post_stab && it == iterations) cache_ac0_zero();
      for (int c = 0; c < n_colors; ++c) {
        int s0 = color_starts[c], s1 = color_starts[c + 1];
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
        for (int u = s0; u < s1; ++u) primal_body(color_bodies[u]);
      }
      if (record_viol) viol.push_back(violation());
      if (it < iterations) over_groups([&](int j) { dual_row(j); });
      if (it == iterations - 1) finalize();
    }
    hash_collect();
  }

  void step() {
    if (substeps <= 1) { substep(); return; }
    R full = dt;
    dt = full / R(substeps);
    for (int s = 0; s < substeps; ++s) substep();
    dt = full;
  }
};

}  // namespace orc

using namespace orc;

struct OrcHandle {
  int prec;
  Sim<float>* f;
  Sim<double>* d;
};

template <class F> static auto dispatch(OrcHandle* h, F fn) {
  if (h->prec == 0) return fn(*h->f);
  return fn(*h->d);
}

extern "C" {

void* orc_create(int precision) {
  OrcHandle* h = new OrcHandle();
  h->prec = precision;
  h->f = precision == 0 ? new Sim<float>() : nullptr;
  h->d = precision == 0 ? nullptr : new Sim<double>();
  return h;
}

void orc_destroy(void* p) {
  OrcHandle* h = (OrcHandle*)p;
  delete h->f;
  delete h->d;
  delete h;
}

// Scalars, in the order of Solver6DOF.__init__ (solver_6dof.py:180-201).
int orc_set_params(void* p, double dt, int iterations, double gx, double gy, double gz, double alpha, double beta,
                   double gamma, int post_stab, double max_lin, double max_ang, int substeps, double fsm,
                   int color_mode, int recolor_every, int self_collide, double self_friction, int threads) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    s.dt = (R)dt; s.iterations = iterations; s.g = {(R)gx, (R)gy, (R)gz};
    s.alpha = (R)alpha; s.beta = (R)beta; s.gamma = (R)gamma; s.post_stab = post_stab;
    s.max_lin = (R)max_lin; s.max_ang = (R)max_ang; s.substeps = substeps < 1 ? 1 : substeps;
    s.fsm = (float)fsm; s.color_mode = color_mode; s.recolor_every = recolor_every;
    s.self_collide = self_collide; s.self_friction = (float)self_friction; s.threads = threads < 1 ? 1 : threads;
    return 0;
  });
}

// Upload the scene (solver_6dof.py:904-1174).  Bodies: x3, q4 (xyzw), v3, w3,
// mass, half extents, friction, local inertia diagonal, coloring priority.
// Rows: the static prefix in the reference's _Row layout.
int orc_load_scene(void* p, int nb, const float* x, const float* q, const float* v, const float* w, const float* mass,
                   const float* he, const float* fric, const float* iloc, const float* prio, int nrows,
                   const int* type, const int* ba, const int* bb, const float* anchor, const float* offa,
                   const float* offb, const float* stiff, const float* fract, const float* fmin, const float* fmax,
                   const int* sib, const int* par, const float* mu, const float* mus, int pair_cap, int dyn_cap) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    s.nb = nb;
    s.x.resize(nb); s.q.resize(nb); s.v.resize(nb); s.w.resize(nb); s.pv.assign(nb, {0, 0, 0}); s.pw.assign(nb, {0, 0, 0});
    s.x0.resize(nb); s.q0.resize(nb); s.xin.resize(nb); s.qin.resize(nb); s.Iw.resize(nb);
    s.mass.resize(nb); s.fric.resize(nb); s.prio.resize(nb); s.he.resize(nb); s.Iloc.resize(nb);
    for (int i = 0; i < nb; ++i) {
      s.x[i] = {(R)x[3 * i], (R)x[3 * i + 1], (R)x[3 * i + 2]};
      s.q[i] = {(R)q[4 * i], (R)q[4 * i + 1], (R)q[4 * i + 2], (R)q[4 * i + 3]};
      s.v[i] = {(R)v[3 * i], (R)v[3 * i + 1], (R)v[3 * i + 2]};
      s.w[i] = {(R)w[3 * i], (R)w[3 * i + 1], (R)w[3 * i + 2]};
      s.mass[i] = mass[i]; s.fric[i] = fric[i]; s.prio[i] = prio[i];
      s.he[i] = {he[3 * i], he[3 * i + 1], he[3 * i + 2]};
      s.Iloc[i] = {iloc[3 * i], iloc[3 * i + 1], iloc[3 * i + 2]};
    }
    s.n_static = nrows;
    s.pair_cap = pair_cap;
    s.type.clear(); s.ba.clear(); s.bb.clear(); s.sib.clear(); s.par.clear(); s.anchor.clear(); s.offa.clear();
    s.offb.clear(); s.stiff.clear(); s.fract.clear(); s.fmin.clear(); s.fmax.clear(); s.mu.clear(); s.mus.clear();
    s.lam.clear(); s.pen.clear(); s.ac0.clear(); s.active.clear(); s.was.clear(); s.row_c.clear();
    s.resize_rows(nrows + dyn_cap);
    for (int j = 0; j < nrows; ++j) {
      s.type[j] = type[j]; s.ba[j] = ba[j]; s.bb[j] = bb[j]; s.sib[j] = sib[j]; s.par[j] = par[j];
      s.anchor[j] = {anchor[3 * j], anchor[3 * j + 1], anchor[3 * j + 2]};
      s.offa[j] = {offa[3 * j], offa[3 * j + 1], offa[3 * j + 2]};
      s.offb[j] = {offb[3 * j], offb[3 * j + 1], offb[3 * j + 2]};
      s.stiff[j] = stiff[j]; s.fract[j] = fract[j]; s.fmin[j] = fmin[j]; s.fmax[j] = fmax[j];
      s.mu[j] = mu[j]; s.mus[j] = mus[j];
      s.lam[j] = 0; s.pen[j] = 1; s.active[j] = 1; s.was[j] = 0; s.ac0[j] = 0;
    }
    s.n_rows = nrows;
    s.cache.clear();
    s.color.assign(nb, -1);
    s.color_dirty = 1;
    s.n_colors = MAX_COLORS;
    return 0;
  });
}

// Grow the pair and dynamic-row capacities, keeping the rows already stored.
int orc_set_caps(void* p, int pair_cap, int dyn_cap) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    s.pair_cap = pair_cap;
    if (s.n_static + dyn_cap > s.cap) s.resize_rows(s.n_static + dyn_cap);
    return 0;
  });
}

int orc_step(void* p) { return dispatch((OrcHandle*)p, [&](auto& s) { s.step(); return 0; }); }
int orc_substep(void* p) { return dispatch((OrcHandle*)p, [&](auto& s) { s.substep(); return 0; }); }
int orc_set_dt(void* p, double dt) {
  return dispatch((OrcHandle*)p, [&](auto& s) { s.dt = (decltype(s.dt))dt; return 0; });
}
int orc_set_record_violation(void* p, int on) {
  return dispatch((OrcHandle*)p, [&](auto& s) { s.record_viol = on; return 0; });
}
int orc_get_violation(void* p, double* out, int cap) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    int n = (int)s.viol.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = s.viol[k];
    return n;
  });
}

// Body state as doubles: x3, q4, v3, w3, prev_v3, prev_w3 (any may be null).
int orc_get_bodies(void* p, double* x, double* q, double* v, double* w, double* pv, double* pw) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    for (int i = 0; i < s.nb; ++i) {
      if (x) { x[3 * i] = s.x[i].x; x[3 * i + 1] = s.x[i].y; x[3 * i + 2] = s.x[i].z; }
      if (q) { q[4 * i] = s.q[i].x; q[4 * i + 1] = s.q[i].y; q[4 * i + 2] = s.q[i].z; q[4 * i + 3] = s.q[i].w; }
      if (v) { v[3 * i] = s.v[i].x; v[3 * i + 1] = s.v[i].y; v[3 * i + 2] = s.v[i].z; }
      if (w) { w[3 * i] = s.w[i].x; w[3 * i + 1] = s.w[i].y; w[3 * i + 2] = s.w[i].z; }
      if (pv) { pv[3 * i] = s.pv[i].x; pv[3 * i + 1] = s.pv[i].y; pv[3 * i + 2] = s.pv[i].z; }
      if (pw) { pw[3 * i] = s.pw[i].x; pw[3 * i + 1] = s.pw[i].y; pw[3 * i + 2] = s.pw[i].z; }
    }
    return s.nb;
  });
}
int orc_set_bodies(void* p, const double* x, const double* q, const double* v, const double* w, const double* pv,
                   const double* pw) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    for (int i = 0; i < s.nb; ++i) {
      if (x) s.x[i] = {(R)x[3 * i], (R)x[3 * i + 1], (R)x[3 * i + 2]};
      if (q) s.q[i] = {(R)q[4 * i], (R)q[4 * i + 1], (R)q[4 * i + 2], (R)q[4 * i + 3]};
      if (v) s.v[i] = {(R)v[3 * i], (R)v[3 * i + 1], (R)v[3 * i + 2]};
      if (w) s.w[i] = {(R)w[3 * i], (R)w[3 * i + 1], (R)w[3 * i + 2]};
      if (pv) s.pv[i] = {(R)pv[3 * i], (R)pv[3 * i + 1], (R)pv[3 * i + 2]};
      if (pw) s.pw[i] = {(R)pw[3 * i], (R)pw[3 * i + 1], (R)pw[3 * i + 2]};
    }
    return 0;
  });
}

// Row counts: [n_static, n_rows (clamped), capacity, rows reserved, pairs found].
int orc_get_counts(void* p, long long* out) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    out[0] = s.n_static; out[1] = s.n_rows; out[2] = s.cap; out[3] = s.n_rows_reserved; out[4] = s.pairs_found;
    out[5] = (long long)s.pairs.size(); out[6] = s.n_colors; out[7] = s.recolored_last; out[8] = s.color_dirty;
    return 0;
  });
}
// Per-row state for rows [0, n): lambda, penalty, alpha*C0, active, was_static, type, body_a, body_b.
int orc_get_rows(void* p, int n, double* lam, double* pen, double* ac0, int* active, int* was, int* type, int* ba,
                 int* bb) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    int m = std::min(n, s.cap);
    for (int j = 0; j < m; ++j) {
      if (lam) lam[j] = s.lam[j];
      if (pen) pen[j] = s.pen[j];
      if (ac0) ac0[j] = s.ac0[j];
      if (active) active[j] = s.active[j];
      if (was) was[j] = s.was[j];
      if (type) type[j] = s.type[j];
      if (ba) ba[j] = s.ba[j];
      if (bb) bb[j] = s.bb[j];
    }
    return m;
  });
}
// Static-row state (rows [0, n_static)) as persistent across substeps.
int orc_set_static_rows(void* p, const double* lam, const double* pen, const int* active, const int* was) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    for (int j = 0; j < s.n_static; ++j) {
      s.lam[j] = (R)lam[j]; s.pen[j] = (R)pen[j]; s.active[j] = active[j]; s.was[j] = was[j];
    }
    return 0;
  });
}
// Contact cache: keys (a, b, c) as int triples and 8 state values each.
int orc_set_key_mode(void* p, int mode) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    s.key_mode = mode ? 1 : 0;
    s.cache.clear();
    return 0;
  });
}
// Contact cache as raw keys (either mode) and 8 state values each, keys sorted.
int orc_get_cache_keys(void* p, int cap, uint64_t* keys, double* st) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    std::vector<uint64_t> ks;
    for (auto& kv : s.cache) ks.push_back(kv.first);
    std::sort(ks.begin(), ks.end());
    int n = (int)ks.size();
    for (int k = 0; k < n && k < cap; ++k) {
      keys[k] = ks[k];
      const auto& e = s.cache[ks[k]];
      for (int u = 0; u < 8; ++u) st[8 * k + u] = e.s[u];
    }
    return n;
  });
}
int orc_set_cache_keys(void* p, int n, const uint64_t* keys, const double* st) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    s.cache.clear();
    for (int k = 0; k < n; ++k) {
      typename std::remove_reference_t<decltype(s)>::Entry e;
      for (int u = 0; u < 8; ++u) e.s[u] = (R)st[8 * k + u];
      s.cache[keys[k] & KEY_MASK50] = e;
    }
    return 0;
  });
}
int orc_get_cache(void* p, int cap, int* abc, double* st) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    std::vector<uint64_t> ks;
    for (auto& kv : s.cache) ks.push_back(kv.first);
    std::sort(ks.begin(), ks.end());
    int n = (int)ks.size();
    for (int k = 0; k < n && k < cap; ++k) {
      uint64_t key = ks[k];
      abc[3 * k] = (int)(key >> 26); abc[3 * k + 1] = (int)((key >> 2) & 0xFFFFFF); abc[3 * k + 2] = (int)(key & 3);
      const auto& e = s.cache[key];
      for (int u = 0; u < 8; ++u) st[8 * k + u] = e.s[u];
    }
    return n;
  });
}
int orc_set_cache(void* p, int n, const int* abc, const double* st) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    using R = std::remove_reference_t<decltype(s.dt)>;
    s.cache.clear();
    for (int k = 0; k < n; ++k) {
      typename std::remove_reference_t<decltype(s)>::Entry e;
      for (int u = 0; u < 8; ++u) e.s[u] = (R)st[8 * k + u];
      s.cache[pair_key(abc[3 * k], abc[3 * k + 1], abc[3 * k + 2])] = e;
    }
    return 0;
  });
}
int orc_get_colors(void* p, int* color) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    for (int i = 0; i < s.nb; ++i) color[i] = s.color[i];
    return s.n_colors;
  });
}
int orc_set_colors(void* p, const int* color, int n_colors, int dirty) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    for (int i = 0; i < s.nb; ++i) s.color[i] = color[i];
    s.n_colors = n_colors;
    s.color_dirty = dirty;
    return 0;
  });
}
int orc_count_conflicts(void* p) { return dispatch((OrcHandle*)p, [&](auto& s) { return (int)s.conflicts(); }); }
// Broad/narrow-phase outputs of the last substep, in pair order.
int orc_get_pairs(void* p, int cap, int* pa, int* pb, int* overlap, int* sat_idx, int* count, float* nrm) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    int n = (int)s.pairs.size();
    for (int k = 0; k < n && k < cap; ++k) {
      const PairOut& o = s.pairs[k];
      pa[k] = o.a; pb[k] = o.b; overlap[k] = o.overlap; sat_idx[k] = o.overlap ? o.sat_idx : -1; count[k] = o.count;
      if (nrm) { nrm[3 * k] = o.overlap ? o.n.x : 0; nrm[3 * k + 1] = o.overlap ? o.n.y : 0; nrm[3 * k + 2] = o.overlap ? o.n.z : 0; }
    }
    return n;
  });
}
// Dynamic contacts of the last substep: (ref body, inc body, ordinal) per contact.
int orc_get_contacts(void* p, int cap, int* abc) {
  return dispatch((OrcHandle*)p, [&](auto& s) {
    int n = (int)s.pool.size();
    for (int k = 0; k < n && k < cap; ++k) {
      abc[3 * k] = s.ba[s.pool[k].n]; abc[3 * k + 1] = s.bb[s.pool[k].n]; abc[3 * k + 2] = s.pool[k].c;
    }
    return n;
  });
}

// Single-call known-answer probes (no scene): SAT and geom_stiffness_diag.
int orc_sat(const float* cA, const float* qA, const float* eA, const float* cB, const float* qB, const float* eB,
            int* sat_idx, float* n, float* depth) {
  PairOut o;
  V3<float> a{cA[0], cA[1], cA[2]}, b{cB[0], cB[1], cB[2]}, ea{eA[0], eA[1], eA[2]}, eb{eB[0], eB[1], eB[2]};
  sat(a, qmat(Q4<float>{qA[0], qA[1], qA[2], qA[3]}), ea, b, qmat(Q4<float>{qB[0], qB[1], qB[2], qB[3]}), eb, o);
  if (!o.overlap) return 0;
  *sat_idx = o.sat_idx; n[0] = o.n.x; n[1] = o.n.y; n[2] = o.n.z; *depth = o.depth;
  return 1;
}
void orc_geom_stiffness_diag(const double* n, const double* r, double* out) {
  V3<double> g = geom_stiffness_diag(V3<double>{n[0], n[1], n[2]}, V3<double>{r[0], r[1], r[2]});
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
}

}  // extern "C"
