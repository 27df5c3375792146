// Explicit liquid viscosity (LinearizedImplicitEuler::stepVelocity with
// compute_viscosity on and implicit_viscosity off, LinearizedImplicitEuler.cpp:
// 272-306).
//
// 1. Liquid volume fractions (TwoDScene::estimateVolumeFractions,
//    TwoDScene.cpp:3535-3584, called by updateLiquidPhi :3353-3367) at the cell
//    centres and the x/y/z edge nodes of every active bucket: eight samples of
//    the cell-centred liquid phi, each interpolated trilinearly
//    (interpolateValue :3586-3621, default dx outside active buckets), turned
//    into the fraction of a cube with phi <= 0 by the twelve-tetrahedron rule
//    of VolumeFractions.cpp:101-162.  The reference adds the node offsets
//    (0.5, 0.5, 0.5) and so on to the node positions in world units, not
//    cells; this does the same.  Positions and the interpolation coordinate
//    use round-to-nearest intrinsics, so the floor() of the sample cell and
//    the trilinear weights are the reference's.
// 2. applyNodeViscosityExplicit (Viscosity.cpp:1780-2107): per face node, the
//    liquid-volume-weighted viscous stress divergence from a copy of the face
//    velocities, in the reference's order of terms, sub-stepped; then the rhs
//    is rebuilt from the new velocity (rhs = v * m).
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_kernels.cuh"

namespace wcg {

__device__ inline double v_add(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double v_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ inline double v_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double v_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ inline float v_add(float a, float b) { return __fadd_rn(a, b); }
__device__ inline float v_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ inline float v_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ inline float v_div(float a, float b) { return __fdiv_rn(a, b); }

template <typename R>
__device__ inline void v_sort4(R& a, R& b, R& c, R& d) {
  R t;
  if (a > b) { t = a; a = b; b = t; }
  if (c > d) { t = c; c = d; d = t; }
  if (a > c) { t = a; a = c; c = t; }
  if (b > d) { t = b; b = d; d = t; }
  if (b > c) { t = b; b = c; c = t; }
}

// fraction of a tetrahedron with phi <= 0 (sorted tet / prism cases)
template <typename R>
__device__ inline R v_tet(R p0, R p1, R p2, R p3) {
  v_sort4(p0, p1, p2, p3);
  if (p3 <= R(0)) return R(1);
  if (p2 <= R(0)) return R(1) - p3 * p3 * p3 / ((p3 - p2) * (p3 - p1) * (p3 - p0));
  if (p1 <= R(0)) {
    const R a = p0 / (p0 - p2), b = p0 / (p0 - p3), c = p1 / (p1 - p3), d = p1 / (p1 - p2);
    return a * b * (R(1) - d) + b * (R(1) - c) * d + c * d;
  }
  if (p0 <= R(0)) return p0 * p0 * p0 / ((p0 - p1) * (p0 - p2) * (p0 - p3));
  return R(0);
}

// fraction of a cube from its corner values (twelve tetrahedra, two twice)
template <typename R>
__device__ inline R v_cube(R p000, R p100, R p010, R p110, R p001, R p101, R p011, R p111) {
  return (v_tet(p000, p001, p101, p011) + v_tet(p000, p101, p100, p110) +
          v_tet(p000, p010, p011, p110) + v_tet(p101, p011, p111, p110) +
          R(2) * v_tet(p000, p011, p101, p110) + v_tet(p100, p101, p001, p111) +
          v_tet(p100, p001, p000, p010) + v_tet(p100, p110, p111, p010) +
          v_tet(p001, p111, p011, p010) + R(2) * v_tet(p100, p111, p001, p010)) /
         R(12);
}

// trilinear liquid phi at pos (cell-centred samples, default dx)
template <typename R>
__device__ inline R v_interp_phi(const GridDesc& g, const unsigned char* __restrict__ active,
                                 const R* __restrict__ lphi, const R* pos, const R* ori, R dx) {
  R bp[3], fr[3], buf[8];
  int bi[3];
  for (int a = 0; a < 3; ++a) {
    bp[a] = v_div(v_sub(pos[a], ori[a]), dx);
    bi[a] = (int)floor(bp[a]);
  }
  for (int t = 0; t < 2; ++t)
    for (int u = 0; u < 2; ++u)
      for (int r = 0; r < 2; ++r) {
        const int q0 = bi[0] + r, q1 = bi[1] + u, q2 = bi[2] + t;
        // C++ integer division (truncation) as the reference; q >= 0 here
        const int h0 = q0 / 4, h1 = q1 / 4, h2 = q2 / 4;
        R v = dx;
        if (h0 >= 0 && h0 < g.ni && h1 >= 0 && h1 < g.nj && h2 >= 0 && h2 < g.nk) {
          const long long b = ((long long)h2 * g.nj + h1) * g.ni + h0;
          if (active[b]) {
            const int l = (q2 - h2 * 4) * 16 + (q1 - h1 * 4) * 4 + (q0 - h0 * 4);
            v = lphi[b * 64 + l];
          }
        }
        buf[t * 4 + u * 2 + r] = v;
      }
  for (int a = 0; a < 3; ++a) fr[a] = v_sub(bp[a], (R)bi[a]);
  auto lerp = [](R v0, R v1, R f) { return v_add(v_mul(v_sub(R(1), f), v0), v_mul(f, v1)); };
  const R b0 = lerp(lerp(buf[0], buf[1], fr[0]), lerp(buf[2], buf[3], fr[0]), fr[1]);
  const R b1 = lerp(lerp(buf[4], buf[5], fr[0]), lerp(buf[6], buf[7], fr[0]), fr[1]);
  return lerp(b0, b1, fr[2]);
}

// Volume fractions of the cell centres and x/y/z edges of every active bucket,
// and with nfrac = 7 of the x/y/z faces too (implicit viscosity).
template <typename R>
__global__ void __launch_bounds__(64)
    k_volume_fractions(GridDesc g, const int* __restrict__ active_list,
                       const unsigned char* __restrict__ active, R* __restrict__ F,
                       long long fs, int nfrac) {
  const int b = active_list[blockIdx.x];
  const int l = threadIdx.x;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx, bs = (R)g.bs;
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const int IJK[3] = {I, J, K};
  R corner[3], ori[3];
  for (int a = 0; a < 3; ++a) {
    const int h = IJK[a] >> 2, lc = IJK[a] & 3;
    corner[a] = v_add(v_add(v_mul((R)h, bs), org[a]), v_mul((R)lc, dx));
    ori[a] = v_add(org[a], v_mul(R(0.5), dx));
  }
  const R o = v_mul(R(0.5), dx);
  const R* lphi = F + G_LPHI * fs;
  const R offs[7][3] = {{0.5, 0.5, 0.5}, {0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5},
                        {0, 0.5, 0.5}, {0.5, 0, 0.5}, {0.5, 0.5, 0}};
  const int outf[7] = {G_VFC, G_VFEX, G_VFEY, G_VFEZ, G_VFU, G_VFV, G_VFW};
  for (int f = 0; f < nfrac; ++f) {
    R c[3];
    for (int a = 0; a < 3; ++a) c[a] = v_add(corner[a], offs[f][a]);
    R ph[8];  // index x*4 + y*2 + z
    for (int x = 0; x < 2; ++x)
      for (int y = 0; y < 2; ++y)
        for (int z = 0; z < 2; ++z) {
          const R pos[3] = {x ? v_add(c[0], o) : v_add(c[0], -o), y ? v_add(c[1], o) : v_add(c[1], -o),
                            z ? v_add(c[2], o) : v_add(c[2], -o)};
          ph[x * 4 + y * 2 + z] = v_interp_phi<R>(g, active, lphi, pos, ori, dx);
        }
    F[outf[f] * fs + n] = v_cube<R>(ph[0], ph[4], ph[2], ph[6], ph[1], ph[5], ph[3], ph[7]);
  }
}

// value of field f at global node (I, J, K); default outside active buckets
template <typename R>
__device__ inline R v_get(const GridDesc& g, const unsigned char* __restrict__ active,
                          const R* __restrict__ f, int I, int J, int K, R def) {
  if (!in_grid(g, I, J, K)) return def;
  const long long b = bucket_of(g, I, J, K);
  if (!active[b]) return def;
  return f[node_linear(g, I, J, K)];
}

// One explicit viscosity step: dst (G_VSTAR..) from src (G_UTMP..).  Block:
// one active bucket, threads [0,64) x faces, [64,128) y, [128,192) z.
template <typename R>
__global__ void __launch_bounds__(192)
    k_viscosity_explicit(GridDesc g, const int* __restrict__ active_list,
                         const unsigned char* __restrict__ active, R* __restrict__ F,
                         long long fs, R factor) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R* src[3] = {F + G_UTMP * fs, F + (G_UTMP + 1) * fs, F + (G_UTMP + 2) * fs};
  const R* cvf = F + G_VFC * fs;
  const R* evf[3] = {F + G_VFEX * fs, F + G_VFEY * fs, F + G_VFEZ * fs};
  auto VN = [&](int fld, int di, int dj, int dk, R def) {
    return v_get<R>(g, active, src[fld], I + di, J + dj, K + dk, def);
  };
  auto VF = [&](const R* arr, int di, int dj, int dk) {
    return v_get<R>(g, active, arr, I + di, J + dj, K + dk, R(0));
  };
  const R cv = src[a][n];
  R v = cv;
  if (a == 0) {
    const R vol_left = VF(cvf, -1, 0, 0), vol_right = VF(cvf, 0, 0, 0);
    const R vol_back = VF(evf[1], 0, 0, 0), vol_front = VF(evf[1], 0, 0, 1);
    const R vol_bottom = VF(evf[2], 0, 0, 0), vol_top = VF(evf[2], 0, 1, 0);
    v += R(2) * factor * vol_right * (VN(0, 1, 0, 0, cv) - cv);
    v += R(2) * factor * vol_left * (VN(0, -1, 0, 0, cv) - cv);
    v += factor * vol_top * (VN(0, 0, 1, 0, cv) - cv);
    v += factor * vol_bottom * (VN(0, 0, -1, 0, cv) - cv);
    v += factor * vol_front * (VN(0, 0, 0, 1, cv) - cv);
    v += factor * vol_back * (VN(0, 0, 0, -1, cv) - cv);
    v += factor * vol_top * (VN(1, 0, 1, 0, R(0)) - VN(1, -1, 1, 0, R(0)));
    v += factor * vol_bottom * (VN(1, -1, 0, 0, R(0)) - VN(1, 0, 0, 0, R(0)));
    v += factor * vol_front * (VN(2, 0, 0, 1, R(0)) - VN(2, -1, 0, 1, R(0)));
    v += factor * vol_back * (VN(2, -1, 0, 0, R(0)) - VN(2, 0, 0, 0, R(0)));
  } else if (a == 1) {
    const R vol_bottom = VF(cvf, 0, -1, 0), vol_top = VF(cvf, 0, 0, 0);
    const R vol_back = VF(evf[0], 0, 0, 0), vol_front = VF(evf[0], 0, 0, 1);
    const R vol_left = VF(evf[2], 0, 0, 0), vol_right = VF(evf[2], 1, 0, 0);
    v += factor * vol_right * (VN(1, 1, 0, 0, cv) - cv);
    v += factor * vol_left * (VN(1, -1, 0, 0, cv) - cv);
    v += R(2) * factor * vol_top * (VN(1, 0, 1, 0, cv) - cv);
    v += R(2) * factor * vol_bottom * (VN(1, 0, -1, 0, cv) - cv);
    v += factor * vol_front * (VN(1, 0, 0, 1, cv) - cv);
    v += factor * vol_back * (VN(1, 0, 0, -1, cv) - cv);
    v += factor * vol_right * (VN(0, 1, 0, 0, R(0)) - VN(0, 1, -1, 0, R(0)));
    v += factor * vol_left * (VN(0, 0, -1, 0, R(0)) - VN(0, 0, 0, 0, R(0)));
    v += factor * vol_front * (VN(2, 0, 0, 1, R(0)) - VN(2, 0, -1, 1, R(0)));
    v += factor * vol_back * (VN(2, 0, -1, 0, R(0)) - VN(2, 0, 0, 0, R(0)));
  } else {
    const R vol_back = VF(cvf, 0, 0, -1), vol_front = VF(cvf, 0, 0, 0);
    const R vol_bottom = VF(evf[0], 0, 0, 0), vol_top = VF(evf[0], 0, 1, 0);
    const R vol_left = VF(evf[1], 0, 0, 0), vol_right = VF(evf[1], 1, 0, 0);
    v += factor * vol_right * (VN(2, 1, 0, 0, cv) - cv);
    v += factor * vol_left * (VN(2, -1, 0, 0, cv) - cv);
    v += factor * vol_top * (VN(2, 0, 1, 0, cv) - cv);
    v += factor * vol_bottom * (VN(2, 0, -1, 0, cv) - cv);
    v += R(2) * factor * vol_front * (VN(2, 0, 0, 1, cv) - cv);
    v += R(2) * factor * vol_back * (VN(2, 0, 0, -1, cv) - cv);
    v += factor * vol_right * (VN(0, 1, 0, 0, R(0)) - VN(0, 1, 0, -1, R(0)));
    v += factor * vol_left * (VN(0, 0, 0, -1, R(0)) - VN(0, 0, 0, 0, R(0)));
    v += factor * vol_top * (VN(1, 0, 1, 0, R(0)) - VN(1, 0, 1, -1, R(0)));
    v += factor * vol_bottom * (VN(1, 0, 0, -1, R(0)) - VN(1, 0, 0, 0, R(0)));
  }
  F[(G_VSTAR + a) * fs + n] = v;
}

// rhs = v* * m on every face of the active buckets (after the viscosity)
template <typename R>
__global__ void __launch_bounds__(192)
    k_rhs_from_vstar(const int* __restrict__ active_list, R* __restrict__ F, long long fs) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  F[(G_RHS + a) * fs + n] = F[(G_VSTAR + a) * fs + n] * F[(G_MASS + a) * fs + n];
}

// ---- implicit viscosity: stepImplicitViscosityDiagonalPCG
// (LinearizedImplicitEuler.cpp:2127-2172), constructViscosityMatrixRHS /
// updateViscosityRHS (Viscosity.cpp:169-1779), applyNodeViscosityImplicit
// (:101-167).  The faces that are fluid and touch liquid are the unknowns; the
// system is applied matrix-free,
//   (V_f + f sum_d w_d V_d) u - f sum_d w_d V_d u_d - f sum (cross terms) = V_f u_src,
// f = dt mu / (rho dx^2), w_d = 2 along the face's own axis and 1 across,
// with solid neighbour faces moved to the rhs, and solved by PCG with the
// diagonal as preconditioner.  Block: one active bucket, threads [0,64) x
// faces, [64,128) y, [128,192) z.

enum : unsigned char { VF_FLUID = 1, VF_DOF = 2 };

// block sum (MAX false) or maximum of non-negative values (MAX true) in a
// fixed order: warp shuffles, then the warps' results in warp order; the
// result is valid in thread 0
template <bool MAX>
__device__ inline double visc_block_reduce(double v, double* sm) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, v, o);
    v = MAX ? fmax(v, w) : v + w;
  }
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    r = sm[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = MAX ? fmax(r, sm[k]) : r + sm[k];
  }
  return r;
}

// field offsets (in face-field triples of gcap) inside Context::visc
enum : int { VS_X = 0, VS_R = 3, VS_P = 6, VS_Q = 9, VS_D = 12, kNumViscFields = 15 };

// liquid volumes around a face of axis a, order +x, -x, +y, -y, +z, -z: the
// cell centres along a, the edges across the other two axes
template <typename R>
__device__ inline void visc_face_vols(const GridDesc& g, const unsigned char* __restrict__ active,
                                      const R* __restrict__ F, long long fs, int a, int I,
                                      int J, int K, R vol[6]) {
  for (int d = 0; d < 6; ++d) {
    const int ax = d >> 1;
    const bool up = !(d & 1);
    int o[3] = {0, 0, 0};
    const R* f;
    if (ax == a) {
      f = F + G_VFC * fs;
      if (!up) o[a] = -1;
    } else {
      f = F + (G_VFEX + (3 - a - ax)) * fs;
      if (up) o[ax] = 1;
    }
    vol[d] = v_get<R>(g, active, f, I + o[0], J + o[1], K + o[2], R(0));
  }
}

// face of axis b at (I, J, K) + the offset of entry t of the cross pair
// across direction d (ax = d >> 1) of a face of axis a
__device__ inline void visc_cross_face(int a, int d, int t, int I, int J, int K, int q[3]) {
  const int ax = d >> 1;
  q[0] = I;
  q[1] = J;
  q[2] = K;
  if (!(d & 1)) q[ax] += 1;
  if (t == 1) q[a] -= 1;
}

__device__ inline bool visc_node(const GridDesc& g, const unsigned char* __restrict__ active,
                                 int I, int J, int K, long long& m) {
  if (!in_grid(g, I, J, K) || !active[bucket_of(g, I, J, K)]) return false;
  m = node_linear(g, I, J, K);
  return true;
}

// face flags: fluid when the solid phi at the centres of its two cells (those
// in active buckets) does not sum below zero (updateSolidPhi
// TwoDScene.cpp:7972-8056); an unknown when fluid with a positive own, cell or
// edge liquid volume
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_flags(GridDesc g, const int* __restrict__ active_list,
                 const unsigned char* __restrict__ active, const R* __restrict__ F, long long fs,
                 Walls walls, unsigned char* __restrict__ flags) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  double sphi = 0.0;
  for (int t = 0; t < 2; ++t) {
    const int ci = I - (a == 0 && t == 0), cj = J - (a == 1 && t == 0), ck = K - (a == 2 && t == 0);
    long long m;
    if (!visc_node(g, active, ci, cj, ck, m)) continue;
    sphi += wall_phi(walls, coord<double>(g.ox, g.bs, g.dx, ci, 0.5),
                     coord<double>(g.oy, g.bs, g.dx, cj, 0.5),
                     coord<double>(g.oz, g.bs, g.dx, ck, 0.5), 3.0 * g.bs);
  }
  const bool fluid = !(sphi < 0.0);
  bool dof = false;
  if (fluid) {
    R vol[6];
    visc_face_vols<R>(g, active, F, fs, a, I, J, K, vol);
    dof = F[(G_VFU + a) * fs + n] > R(0);
    for (int d = 0; d < 6; ++d) dof = dof || vol[d] > R(0);
  }
  flags[a * fs + n] = (unsigned char)((fluid ? VF_FLUID : 0) | (dof ? VF_DOF : 0));
}

// rhs (into r) and diagonal of the unknowns, from the source velocity u_src
// (G_VSTAR), in the reference's order of terms; x = p = 0; partial[block] =
// max |rhs| over the block
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_rhs(GridDesc g, const int* __restrict__ active_list,
               const unsigned char* __restrict__ active, const R* __restrict__ F, long long fs,
               const unsigned char* __restrict__ flags, R factor, R* __restrict__ V,
               double* __restrict__ partial) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const long long fn = a * fs + n;
  R rhs = 0, diag = 0;
  if (flags[fn] & VF_DOF) {
    const R* src = F + G_VSTAR * fs;
    const R volu = F[(G_VFU + a) * fs + n];
    rhs = volu * src[a * fs + n];
    diag = volu;
    R vol[6];
    visc_face_vols<R>(g, active, F, fs, a, I, J, K, vol);
    for (int d = 0; d < 6; ++d) {
      if (!(vol[d] > R(0))) continue;
      const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
      long long m;
      if (!visc_node(g, active, I + (ax == 0) * sg, J + (ax == 1) * sg, K + (ax == 2) * sg, m))
        continue;
      const R w = ax == a ? R(2) : R(1);
      diag += w * factor * vol[d];
      if (!(flags[a * fs + m] & VF_FLUID)) rhs -= -w * src[a * fs + m] * factor * vol[d];
    }
    for (int d = 0; d < 6; ++d) {
      const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
      if (ax == a || !(vol[d] > R(0))) continue;
      for (int t = 0; t < 2; ++t) {
        int q[3];
        visc_cross_face(a, d, t, I, J, K, q);
        long long m;
        if (!visc_node(g, active, q[0], q[1], q[2], m)) continue;
        const R c = (t == 0 ? R(-1) : R(1)) * (R)sg;
        if (!(flags[ax * fs + m] & VF_FLUID)) rhs -= c * src[ax * fs + m] * factor * vol[d];
      }
    }
  }
  V[(VS_X + a) * fs + n] = R(0);
  V[(VS_R + a) * fs + n] = rhs;
  V[(VS_P + a) * fs + n] = R(0);
  V[(VS_D + a) * fs + n] = diag;
  __shared__ double sm[8];
  const double m = visc_block_reduce<true>(fabs((double)rhs), sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// q = A p over the unknowns; partial[block] = sum p.q
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_apply(GridDesc g, const int* __restrict__ active_list,
                 const unsigned char* __restrict__ active, const R* __restrict__ F, long long fs,
                 const unsigned char* __restrict__ flags, R factor, R* __restrict__ V,
                 double* __restrict__ partial) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R* P = V + VS_P * fs;
  double pq = 0.0;
  R q = 0;
  if (flags[a * fs + n] & VF_DOF) {
    const R p0 = P[a * fs + n];
    q = V[(VS_D + a) * fs + n] * p0;
    R vol[6];
    visc_face_vols<R>(g, active, F, fs, a, I, J, K, vol);
    for (int d = 0; d < 6; ++d) {
      if (!(vol[d] > R(0))) continue;
      const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
      long long m;
      if (!visc_node(g, active, I + (ax == 0) * sg, J + (ax == 1) * sg, K + (ax == 2) * sg, m))
        continue;
      if (flags[a * fs + m] & VF_DOF) {
        const R w = ax == a ? R(2) : R(1);
        q += -w * factor * vol[d] * P[a * fs + m];
      }
    }
    for (int d = 0; d < 6; ++d) {
      const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
      if (ax == a || !(vol[d] > R(0))) continue;
      for (int t = 0; t < 2; ++t) {
        int qq[3];
        visc_cross_face(a, d, t, I, J, K, qq);
        long long m;
        if (!visc_node(g, active, qq[0], qq[1], qq[2], m)) continue;
        if (flags[ax * fs + m] & VF_DOF) {
          const R c = (t == 0 ? R(-1) : R(1)) * (R)sg;
          q += c * factor * vol[d] * P[ax * fs + m];
        }
      }
    }
    pq = (double)p0 * (double)q;
  }
  V[(VS_Q + a) * fs + n] = q;
  __shared__ double sm[8];
  const double s = visc_block_reduce<false>(pq, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// x += alpha p, r -= alpha q with alpha = rho / (p.q) (device scalars);
// partial[block] = max |r|
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_update(const int* __restrict__ active_list, long long fs,
                  const unsigned char* __restrict__ flags, R* __restrict__ V,
                  const double* __restrict__ dsc, int rho_slot, int pq_slot,
                  double* __restrict__ partial) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  const double pqv = dsc[pq_slot];
  const R alpha = (R)(pqv != 0.0 ? dsc[rho_slot] / pqv : 0.0);
  double rm = 0.0;
  if (flags[a * fs + n] & VF_DOF) {
    V[(VS_X + a) * fs + n] += alpha * V[(VS_P + a) * fs + n];
    const R r = V[(VS_R + a) * fs + n] - alpha * V[(VS_Q + a) * fs + n];
    V[(VS_R + a) * fs + n] = r;
    rm = fabs((double)r);
  }
  __shared__ double sm[8];
  const double m = visc_block_reduce<true>(rm, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// partial[block] = sum r.z, z = r / diag (0 where the diagonal is 0)
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_zdot(const int* __restrict__ active_list, long long fs,
                const unsigned char* __restrict__ flags, const R* __restrict__ V,
                double* __restrict__ partial) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  double rz = 0.0;
  if (flags[a * fs + n] & VF_DOF) {
    const R d = V[(VS_D + a) * fs + n];
    const R r = V[(VS_R + a) * fs + n];
    if (d != R(0)) rz = (double)r * (double)(r / d);
  }
  __shared__ double sm[8];
  const double s = visc_block_reduce<false>(rz, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// p = z + beta p, beta = rho_new / rho (device scalars; beta 0 on the first)
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_dir(const int* __restrict__ active_list, long long fs,
               const unsigned char* __restrict__ flags, R* __restrict__ V,
               const double* __restrict__ dsc, int new_slot, int old_slot, int first) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  if (!(flags[a * fs + n] & VF_DOF)) return;
  const R beta = first ? R(0) : (R)(dsc[new_slot] / dsc[old_slot]);
  const R d = V[(VS_D + a) * fs + n];
  const R z = d != R(0) ? V[(VS_R + a) * fs + n] / d : R(0);
  V[(VS_P + a) * fs + n] = z + beta * V[(VS_P + a) * fs + n];
}

// applyNodeViscosityImplicit's write-back: unknowns take the solution, other
// fluid faces keep their value, solid faces the (static) solid velocity
template <typename R>
__global__ void __launch_bounds__(192)
    k_visc_writeback(const int* __restrict__ active_list, long long fs,
                     const unsigned char* __restrict__ flags, const R* __restrict__ V,
                     R* __restrict__ F, int zero_solution) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  const unsigned char f = flags[a * fs + n];
  R* u = F + (G_VSTAR + a) * fs;
  if (f & VF_FLUID) {
    if (f & VF_DOF) u[n] = zero_solution ? R(0) : V[(VS_X + a) * fs + n];
  } else {
    u[n] = R(0);
  }
}

}  // namespace wcg
