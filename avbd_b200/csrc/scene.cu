// Scene build on the device: the static constraint groups of the floor
// blocks (solver_6dof.py:474-541, add_floor_contact_box: 8 corners, each a
// normal row and, with friction, two tangent rows; stored by the reference
// as 24 c_* rows per box, solver_6dof.py:1067-1129).
//
// The host sorts the blocks (and the few explicit groups, pins) by body and
// first row and hands each block its first group index; one thread per
// corner then writes the corner's group record.  A block whose half extents
// are its body's is an implicit corner (no stored offset: the kernels rebuild
// it from the body's half extents and the corner index, floor height in
// mat.w); any other block keeps an explicit offset, floor height in offa.w.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"

namespace avbd {

#define SCENE_INF __int_as_float(0x7f800000)

__global__ void k_floor_groups(const __grid_constant__ Dev d, int nblk, const int* blk_body, const float4* blk_he_fy,
                               const float4* blk_mat, const int* blk_row0, const int* blk_per, const int* blk_goff) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * nblk) return;
  int b = t >> 3, c = t & 7;
  int body = blk_body[b];
  float4 hf = blk_he_fy[b];  // half extents, floor y
  float4 m = blk_mat[b];     // mu, mu_s, stiffness
  int per = blk_per[b];
  int g = blk_goff[b] + c;
  bool three = per == 3;
  bool hard = !(m.z < SCENE_INF);
  float4 bhe = d.he[body];
  bool implicit = hf.x == bhe.x && hf.y == bhe.y && hf.z == bhe.z;
  int meta = make_meta(KIND_FLOOR, three, hard, 0);
  // the reference's loop order: sx outer, sy, sz inner; set bit = + sign
  float sx = (c & 4) ? 1.0f : -1.0f, sy = (c & 2) ? 1.0f : -1.0f, sz = (c & 1) ? 1.0f : -1.0f;
  float4 offa, mat;
  if (implicit) {
    meta |= META_IMPLICIT | (c << 6);
    offa = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    mat = make_float4(m.x, m.y, m.z, hf.w);
  } else {
    offa = make_float4(sx * hf.x, sy * hf.y, sz * hf.z, hf.w);
    mat = make_float4(m.x, m.y, m.z, SCENE_INF);
  }
  d.g_body[g] = make_int2(body, -1);
  d.g_meta[g] = meta;
  d.g_row0[g] = blk_row0[b] + c * per;
  d.g_offa[g] = offa;
  d.g_n[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  d.g_mat[g] = mat;
  d.g_flags[g] = three ? 7 : 1;
  d.g_lam[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  d.g_pen[g] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);  // solver_6dof.py:1121: penalties seeded to 1
}

cudaError_t launch_floor_groups(const Dev& d, int nblk, const int* blk_body, const float4* blk_he_fy,
                                const float4* blk_mat, const int* blk_row0, const int* blk_per, const int* blk_goff,
                                cudaStream_t st) {
  int n = 8 * nblk;
  k_floor_groups<<<(n + 255) / 256, 256, 0, st>>>(d, nblk, blk_body, blk_he_fy, blk_mat, blk_row0, blk_per, blk_goff);
  g_kernel_launches += 1;
  return cudaGetLastError();
}

}  // namespace avbd
