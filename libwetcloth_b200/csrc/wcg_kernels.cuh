// Kernels of the fluid step, templated on the arithmetic type R (double for
// the FP64 form, float for the mixed-precision form).  Every kernel cites the
// reference routine whose arithmetic it restates.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"

namespace wcg {

// ---- precision-specific rounding helpers ------------------------------------
__device__ inline double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ inline double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ inline float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ inline float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ inline float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ inline float div_rn(float a, float b) { return __fdiv_rn(a, b); }

template <typename R>
__device__ inline R coord(R origin, R bs, R dx, int node, R offset) {
  const int h = node >> 2;
  const int l = node & 3;
  R c = add_rn(mul_rn((R)h, bs), origin);
  c = add_rn(c, mul_rn((R)l, dx));
  return add_rn(c, mul_rn(offset, dx));
}

// Stencil base node of one axis, as TwoDScene::findNodes
// (TwoDScene.cpp:3692-3715): local = (x - corner)/dx with
// corner = (handle*bs + origin) + offset*dx; base = handle*4 + floor(local)
// + (frac(local) > 0.5 ? 0 : -1).
template <typename R>
__device__ inline int stencil_base(R x, R origin, R bs, R dx, int handle,
                                   R offset) {
  R corner = add_rn(mul_rn((R)handle, bs), origin);
  corner = add_rn(corner, mul_rn(offset, dx));
  const R lp = div_rn(sub_rn(x, corner), dx);
  const R fl = floor(lp);
  const R fr = sub_rn(lp, fl);
  return handle * 4 + (int)fl + (fr > R(0.5) ? 0 : -1);
}

struct DeltaRange {
  int lo[3];
  int hi[3];
};

// packed per-particle stencil offsets: delta_a = base(offset 0) - base(offset
// 0.5) on axis a, stored as delta+4 in 4 bits per axis.
__device__ inline int unpack_delta(int packed, int axis) {
  return ((packed >> (4 * axis)) & 15) - 4;
}

// ---- particle pass: buckets, stencil bases, activation, cell counts ---------
// Sorter::sort key (Sorter.h:126-140, TwoDScene::rebucketizeParticles
// :1694-1699), findNodes activation (TwoDScene.cpp:3683-3760) for the u, v, w,
// solid-phi and pressure stencils of every (soft) liquid particle.
template <typename R>
__global__ void k_particle_prepass(GridDesc g, const R* __restrict__ P,
                                   long long pcap, long long np,
                                   long long* __restrict__ key,
                                   int* __restrict__ delta,
                                   int* __restrict__ pbucket,
                                   unsigned char* __restrict__ active_pre,
                                   int* __restrict__ cell_count,
                                   int* __restrict__ drange, int* err,
                                   const R* __restrict__ surf = nullptr) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < np;
  int d[3] = {0, 0, 0};
  int dmin[3] = {1 << 20, 1 << 20, 1 << 20}, dmax[3] = {-(1 << 20), -(1 << 20), -(1 << 20)};
  if (live) {
    const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
    const int nbk[3] = {g.ni, g.nj, g.nk};
    const R bs = (R)g.bs, dx = (R)g.dx;
    int b0[3], b5[3], bh[3];
    for (int a = 0; a < 3; ++a) {
      const R x = P[(PX + a) * pcap + i];
      int h = (int)floor(div_rn(sub_rn(x, org[a]), bs));
      h = h < 0 ? 0 : (h > nbk[a] - 1 ? nbk[a] - 1 : h);
      bh[a] = h;
      b0[a] = stencil_base<R>(x, org[a], bs, dx, h, R(0));
      b5[a] = stencil_base<R>(x, org[a], bs, dx, h, R(0.5));
    }
    pbucket[i] = (bh[2] * g.nj + bh[1]) * g.ni + bh[0];
    int packed = 0;
    for (int a = 0; a < 3; ++a) {
      d[a] = b0[a] - b5[a];
      dmin[a] = dmax[a] = d[a];
      const int dc = d[a] < -4 ? -4 : (d[a] > 11 ? 11 : d[a]);
      packed |= (dc + 4) << (4 * a);
    }
    delta[i] = packed;
    const int KX = b5[0] + 1, KY = b5[1] + 1, KZ = b5[2] + 1;
    if (!in_grid(g, KX, KY, KZ)) {
      record_error(err, kErrIndex);
      key[i] = -1;
    } else {
      const long long k = node_linear(g, KX, KY, KZ);
      key[i] = k;
      atomicAdd(&cell_count[k], 1);
    }
    // activation of the buckets under the five 3x3x3 stencils, by soft
    // particles only (isSoft :697: surfels activate nothing)
    const int nt = (surf == nullptr || surf[i] == R(0)) ? 5 : 0;
    for (int t = 0; t < nt; ++t) {
      // offsets: u(0,.5,.5) v(.5,0,.5) w(.5,.5,0) solid-phi(0,0,0) p(.5,.5,.5)
      int lo[3];
      for (int a = 0; a < 3; ++a) {
        const bool zero = (t == 3) || (t == a);
        lo[a] = zero ? b0[a] : b5[a];
      }
      const int bx0 = lo[0] >> 2, bx1 = (lo[0] + 2) >> 2;
      const int by0 = lo[1] >> 2, by1 = (lo[1] + 2) >> 2;
      const int bz0 = lo[2] >> 2, bz1 = (lo[2] + 2) >> 2;
      for (int bz = bz0; bz <= bz1; ++bz)
        for (int by = by0; by <= by1; ++by)
          for (int bx = bx0; bx <= bx1; ++bx) {
            if (bx < 0 || by < 0 || bz < 0 || bx >= g.ni || by >= g.nj ||
                bz >= g.nk) {
              record_error(err, kErrIndex);
              continue;
            }
            const long long b = ((long long)bz * g.nj + by) * g.ni + bx;
            if (!active_pre[b]) active_pre[b] = 1;
          }
    }
  }
  // stencil-offset range: one atomic per warp and axis
  for (int a = 0; a < 3; ++a) {
    const int mn = __reduce_min_sync(0xffffffffu, dmin[a]);
    const int mx = __reduce_max_sync(0xffffffffu, dmax[a]);
    if ((threadIdx.x & 31) == 0) {
      if (mn < (1 << 20)) atomicMin(&drange[a], mn);
      if (mx > -(1 << 20)) atomicMax(&drange[3 + a], mx);
    }
  }
}

// expandFluidNodesMarked(1) (TwoDScene.cpp:5021-5064): a bucket becomes active
// if any of its 26 neighbours was active before the pass.
__global__ void k_dilate(GridDesc g, const unsigned char* __restrict__ pre,
                         unsigned char* __restrict__ act) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= g.nb) return;
  const int bk = (int)(b / ((long long)g.ni * g.nj));
  const int rem = (int)(b - (long long)bk * g.ni * g.nj);
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  unsigned char a = pre[b];
  for (int t = -1; t <= 1 && !a; ++t)
    for (int s = -1; s <= 1 && !a; ++s)
      for (int r = -1; r <= 1 && !a; ++r) {
        const int x = bi + r, y = bj + s, z = bk + t;
        if (x < 0 || y < 0 || z < 0 || x >= g.ni || y >= g.nj || z >= g.nk)
          continue;
        if (pre[((long long)z * g.nj + y) * g.ni + x]) a = 1;
      }
  act[b] = a;
}

__global__ void k_flag_to_int(const unsigned char* __restrict__ f, long long n,
                              int* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = f[i] ? 1 : 0;
}

__global__ void k_compact(const unsigned char* __restrict__ f,
                          const int* __restrict__ pos, long long n,
                          int* __restrict__ list) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && f[i]) list[pos[i]] = (int)i;
}

// active buckets bucketed by wave index bi+bj+bk (wavefront order)
__global__ void k_wave_count(GridDesc g, const int* __restrict__ active_list,
                             long long nact, int* __restrict__ wave_count) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nact) return;
  const int b = active_list[e];
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  atomicAdd(&wave_count[bi + bj + bk], 1);
}

__global__ void k_wave_scatter(GridDesc g, const int* __restrict__ active_list,
                               long long nact, int* __restrict__ wave_cursor,
                               int* __restrict__ wave_list) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nact) return;
  const int b = active_list[e];
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int slot = atomicAdd(&wave_cursor[bi + bj + bk], 1);
  wave_list[slot] = b;
}

// ---- counting sort by key node ---------------------------------------------
__global__ void k_sort_scatter(const long long* __restrict__ key, long long np,
                               const int* __restrict__ start,
                               int* __restrict__ cursor, int* __restrict__ perm) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const long long k = key[i];
  if (k < 0) return;
  const int slot = start[k] + atomicAdd(&cursor[k], 1);
  perm[slot] = (int)i;
}

// Order each cell's particles by original index so the sorted order (and
// with it every floating-point sum) is deterministic.
__global__ void k_sort_cells(const int* __restrict__ start, long long nnode,
                             const int* __restrict__ pid, int* __restrict__ perm) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nnode) return;
  const int s0 = start[c], s1 = start[c + 1];
  for (int a = s0 + 1; a < s1; ++a) {
    const int v = perm[a];
    const int kv = pid[v];
    int b = a - 1;
    while (b >= s0 && pid[perm[b]] > kv) {
      perm[b + 1] = perm[b];
      --b;
    }
    perm[b + 1] = v;
  }
}

template <typename R>
__global__ void k_gather_particles(const int* __restrict__ perm, long long np,
                                   long long pcap, const R* __restrict__ src,
                                   R* __restrict__ dst,
                                   const int* __restrict__ pid_src,
                                   int* __restrict__ pid_dst,
                                   const long long* __restrict__ key_src,
                                   long long* __restrict__ key_dst,
                                   const int* __restrict__ delta_src,
                                   int* __restrict__ delta_dst,
                                   const int* __restrict__ pb_src,
                                   int* __restrict__ pb_dst) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const int i = perm[s];
#pragma unroll
  for (int c = 0; c < kNumPCols; ++c) dst[c * pcap + s] = src[c * pcap + i];
  pid_dst[s] = pid_src[i];
  key_dst[s] = key_src[i];
  delta_dst[s] = delta_src[i];
  pb_dst[s] = pb_src[i];
}

// ---- P2G: gather per node ---------------------------------------------------
// mapParticleNodesAPIC (TwoDScene.cpp:6609-6919), liquid branch:
//   p_f += (v_a + C.row(a).(x_n - x_p)) * m * w;  m_f += m * w;  V_f += V * w
//   u_f = p_f / m_f if m_f > 1e-20; psi = 0; sat = clamp(V_f/max(1e-20,dV),0,1)
// updateLiquidPhi (TwoDScene.cpp:3286-3345) at cell centres and
// mapParticleSaturationPsiNodes (:5952-5992).  Each node sums the particles
// whose stencil contains it (exactly the reference's per-node pair lists,
// buildNodeParticlePairs :2257-2355), visiting them in key-cell order, so the
// result is deterministic and needs no atomics.
// Block: one active bucket; threads [0,64) u-faces, [64,128) v-faces,
// [128,192) w-faces, [192,256) cell centres.
template <typename R>
__global__ void __launch_bounds__(256)
    k_p2g(GridDesc g, const int* __restrict__ active_list,
          const unsigned char* __restrict__ active, const R* __restrict__ P,
          long long pcap, const int* __restrict__ start,
          const int* __restrict__ delta, DeltaRange dr, R* __restrict__ F,
          long long fstride, Walls walls, int raw_satp, int have_liquid) {
  const int b = active_list[blockIdx.x];
  const int type = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const int IJK[3] = {I, J, K};
  const R* px = P + PX * pcap;
  const R* py = P + PY * pcap;
  const R* pz = P + PZ * pcap;
  const R dV = dx * dx * dx;

  if (type < 3) {
    const int a = type;
    R np_[3];
    for (int q = 0; q < 3; ++q)
      np_[q] = coord<R>(org[q], bs, dx, IJK[q], q == a ? R(0) : R(0.5));
    int lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
      if (q == a) {
        lo[q] = IJK[q] - 1 - dr.hi[q];
        hi[q] = IJK[q] + 1 - dr.lo[q];
      } else {
        lo[q] = IJK[q] - 1;
        hi[q] = IJK[q] + 1;
      }
      lo[q] = lo[q] < 0 ? 0 : lo[q];
    }
    hi[0] = hi[0] > g.NI - 1 ? g.NI - 1 : hi[0];
    hi[1] = hi[1] > g.NJ - 1 ? g.NJ - 1 : hi[1];
    hi[2] = hi[2] > g.NK - 1 ? g.NK - 1 : hi[2];
    const R* va = P + (VX + a) * pcap;
    const R* c0 = P + (C00 + 3 * a) * pcap;
    const R* c1 = P + (C00 + 3 * a + 1) * pcap;
    const R* c2 = P + (C00 + 3 * a + 2) * pcap;
    const R* pm = P + PM * pcap;
    const R* pv = P + PV * pcap;
    R mom = 0, mass = 0, vol = 0;
    for (int KZ = lo[2]; KZ <= hi[2]; ++KZ)
      for (int KY = lo[1]; KY <= hi[1]; ++KY)
        for (int KX = lo[0]; KX <= hi[0]; ++KX) {
          const long long c = node_linear(g, KX, KY, KZ);
          const int s1 = start[c + 1];
          const int Ka = a == 0 ? KX : (a == 1 ? KY : KZ);
          for (int s = start[c]; s < s1; ++s) {
            const int base = Ka - 1 + unpack_delta(delta[s], a);
            const int off = IJK[a] - base;
            if (off < 0 || off > 2) continue;
            const R x = px[s], y = py[s], z = pz[s];
            const R w = quad_kernel<R>((x - np_[0]) * invh) *
                        quad_kernel<R>((y - np_[1]) * invh) *
                        quad_kernel<R>((z - np_[2]) * invh);
            if (!(w > R(0))) continue;
            const R m = pm[s];
            const R vel = va[s] + (c0[s] * (np_[0] - x) + c1[s] * (np_[1] - y)) +
                          c2[s] * (np_[2] - z);
            mom += vel * m * w;
            mass += m * w;
            vol += pv[s] * w;
          }
        }
    F[(G_MASS + a) * fstride + n] = mass;
    F[(G_VEL + a) * fstride + n] = mass > R(1e-20) ? mom / mass : R(0);
    F[(G_VOL + a) * fstride + n] = vol;
    const R den = dV > R(1e-20) ? dV : R(1e-20);
    F[(G_SAT + a) * fstride + n] = clamp01<R>(vol / den);
  } else {
    // cell centre: liquid level set + saturation; corner: solid phi
    R np_[3];
    for (int q = 0; q < 3; ++q) np_[q] = coord<R>(org[q], bs, dx, IJK[q], R(0.5));
    const R* pr = P + PR * pcap;
    const R* pv = P + PV * pcap;
    const R rmin = dx * (R)kLiquidPhiRadius;
    R phi = R(3) * bs;
    R vliq = 0;
    const int lo0 = I - 1 < 0 ? 0 : I - 1, hi0 = I + 1 > g.NI - 1 ? g.NI - 1 : I + 1;
    const int lo1 = J - 1 < 0 ? 0 : J - 1, hi1 = J + 1 > g.NJ - 1 ? g.NJ - 1 : J + 1;
    const int lo2 = K - 1 < 0 ? 0 : K - 1, hi2 = K + 1 > g.NK - 1 ? g.NK - 1 : K + 1;
    for (int KZ = lo2; KZ <= hi2; ++KZ)
      for (int KY = lo1; KY <= hi1; ++KY)
        for (int KX = lo0; KX <= hi0; ++KX) {
          const long long c = node_linear(g, KX, KY, KZ);
          const int s1 = start[c + 1];
          for (int s = start[c]; s < s1; ++s) {
            const R x = px[s], y = py[s], z = pz[s];
            const R ddx = x - np_[0], ddy = y - np_[1], ddz = z - np_[2];
            const R r = pr[s];
            const R d = sqrt((ddx * ddx + ddy * ddy) + ddz * ddz) -
                        (rmin > r ? rmin : r);
            phi = d < phi ? d : phi;
            const R w = quad_kernel<R>(ddx * invh) * quad_kernel<R>(ddy * invh) *
                        quad_kernel<R>(ddz * invh);
            if (w > R(0)) vliq += pv[s] * w;
          }
        }
    const double three_bs = 3.0 * g.bs;
    const double sphi_c = wall_phi(walls, (double)np_[0], (double)np_[1],
                                   (double)np_[2], three_bs);
    // updateLiquidPhi returns before the wall rule when there is no liquid
    // particle (TwoDScene.cpp:3303)
    if (have_liquid && sphi_c < 0.0) phi = R(-0.5) * dx;
    F[G_LPHI * fstride + n] = phi;
    const R den = dV > R(1e-20) ? dV : R(1e-20);
    // with elasto particles k_p2g_elasto completes sat_p from the raw sum
    F[G_SATP * fstride + n] = raw_satp ? vliq : clamp01<R>(vliq / den);
    // solid phi at the corner node (TwoDScene::updateSolidPhi :7940-7960)
    const double cx = (double)coord<R>(org[0], bs, dx, I, R(0));
    const double cy = (double)coord<R>(org[1], bs, dx, J, R(0));
    const double cz = (double)coord<R>(org[2], bs, dx, K, R(0));
    F[G_SPHI * fstride + n] = (R)wall_phi(walls, cx, cy, cz, three_bs);
  }
}

// ---- P2G as a particle scatter into bucket halo tiles -----------------------
// The same sums as k_p2g (mapParticleNodesAPIC TwoDScene.cpp:6609-6919 liquid
// branch, updateLiquidPhi :3286-3345, mapParticleSaturationPsiNodes
// :5952-5992), computed particle by particle instead of node by node, so each
// particle's per-axis weights are evaluated once.
//
// Halo tile of bucket B: every node the stencils of B's particles reach.  A
// particle with key cell c (the p-stencil centre) and stencil offsets delta in
// {0, 1} reaches cell-centre nodes c-1..c+1 on each axis and, for the face of
// axis a, nodes c-1+delta_a..c+1+delta_a on axis a.  Over c in [4B, 4B+3] that
// is [4B-1, 4B+4] (6 nodes) per axis and [4B-1, 4B+5] (7) on the face's own
// axis.  Tile layout (R values): for each face axis a, mass, momentum and
// volume (kHaloF each); then the cell-centre volume and liquid phi (kHaloC).
constexpr int kHaloF = 7 * 6 * 6;
constexpr int kHaloC = 6 * 6 * 6;
constexpr int kTileVals = 9 * kHaloF + 2 * kHaloC;

// index of halo node (x, y, z) (offsets from 4B - 1) in a face-a tile
__device__ inline int halo_face(int a, int x, int y, int z) {
  const int nx = a == 0 ? 7 : 6, ny = a == 1 ? 7 : 6;
  return (z * ny + y) * nx + x;
}
__device__ inline int halo_centre(int x, int y, int z) { return (z * 6 + y) * 6 + x; }

// Scatter: one warp per active bucket (WPB warps per block, each with its own
// tile).  The bucket's particles (key cells in the bucket: one contiguous run
// of the sorted arrays) are visited one at a time in sorted order; lane l < 27
// is stencil slot (l % 3, l / 3 % 3, l / 9) of the visited particle, so the 27
// lanes write 27 distinct nodes per node type and the warp adds into its tile
// without atomics, every node receiving its contributions in sorted-particle
// order: deterministic.  Lanes 0..17 evaluate the particle's 18 per-axis
// weights (3 axes x offsets 0 and 1/2 x 3 nodes) once; the slot lanes take
// theirs by shuffle.  Requires stencil offsets in {0, 1} (checked on the host).
template <typename R, int WPB>
__global__ void __launch_bounds__(32 * WPB)
    k_p2g_scatter(GridDesc g, const int* __restrict__ active_list, long long n_active,
                  const R* __restrict__ P, long long pcap, const int* __restrict__ start,
                  const long long* __restrict__ key, const int* __restrict__ delta,
                  R* __restrict__ halo) {
  __shared__ R tiles[WPB][kTileVals];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long ai = (long long)blockIdx.x * WPB + wid;
  if (ai >= n_active) return;
  const int b = active_list[ai];
  const long long n0 = (long long)b * 64;
  const int p0 = start[n0], p1 = start[n0 + 64];
  if (p1 <= p0) return;  // no particles: the merge skips this bucket
  R* T = tiles[wid];
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const R rmin = dx * (R)kLiquidPhiRadius;
  const R three_bs = R(3) * bs;
  for (int e = lane; e < kTileVals; e += 32) T[e] = e < 9 * kHaloF + kHaloC ? R(0) : three_bs;
  __syncwarp();
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  // weight lane (lane < 18): axis, offset (0 or 1/2), stencil node
  const int wq = lane / 6, wo = (lane / 3) & 1, wn = lane % 3;
  const R worg = wq == 0 ? (R)g.ox : (wq == 1 ? (R)g.oy : (R)g.oz);
  const int wb4 = 4 * (wq == 0 ? bi : (wq == 1 ? bj : bk));
  // slot lane (lane < 27)
  const int si = lane % 3, sj = (lane / 3) % 3, sk = lane / 9;
  const bool slot = lane < 27;
  R* Tc = T + 9 * kHaloF;
  R* Tphi = Tc + kHaloC;
  for (int s0 = p0; s0 < p1; s0 += 32) {
    const int s = s0 + lane;
    R mine[kNumPCols];
    int mdl = 0, mkl = 0;
    if (s < p1) {
#pragma unroll
      for (int c = 0; c < kNumPCols; ++c) mine[c] = P[c * pcap + s];
      mdl = delta[s];
      mkl = (int)(key[s] & 63);
    } else {
#pragma unroll
      for (int c = 0; c < kNumPCols; ++c) mine[c] = R(0);
    }
    const int cnt = min(32, p1 - s0);
    for (int q = 0; q < cnt; ++q) {
      R pc[kNumPCols];
#pragma unroll
      for (int c = 0; c < kNumPCols; ++c) pc[c] = __shfl_sync(full, mine[c], q);
      const int dl = __shfl_sync(full, mdl, q);
      const int kl = __shfl_sync(full, mkl, q);
      const int cl0 = kl & 3, cl1 = (kl >> 2) & 3, cl2 = kl >> 4;  // key cell in the bucket
      R wv = R(0), dv = R(0);
      if (lane < 18) {
        const int clq = wq == 0 ? cl0 : (wq == 1 ? cl1 : cl2);
        const int node = wb4 + clq - 1 + (wo == 0 ? unpack_delta(dl, wq) : 0) + wn;
        const R np = coord<R>(worg, bs, dx, node, wo ? R(0.5) : R(0));
        dv = (wq == 0 ? pc[PX] : (wq == 1 ? pc[PY] : pc[PZ])) - np;
        wv = quad_kernel<R>(dv * invh);
      }
      const R w0x = __shfl_sync(full, wv, si), w5x = __shfl_sync(full, wv, 3 + si);
      const R w0y = __shfl_sync(full, wv, 6 + sj), w5y = __shfl_sync(full, wv, 9 + sj);
      const R w0z = __shfl_sync(full, wv, 12 + sk), w5z = __shfl_sync(full, wv, 15 + sk);
      const R d0x = __shfl_sync(full, dv, si), d5x = __shfl_sync(full, dv, 3 + si);
      const R d0y = __shfl_sync(full, dv, 6 + sj), d5y = __shfl_sync(full, dv, 9 + sj);
      const R d0z = __shfl_sync(full, dv, 12 + sk), d5z = __shfl_sync(full, dv, 15 + sk);
      if (slot) {
        // halo coordinates of this slot's cell-centre node: (c - 1 + s) - (4B - 1)
        const int hx = cl0 + si, hy = cl1 + sj, hz = cl2 + sk;
        const R m = pc[PM], vol = pc[PV];
        // faces: offset 0 on the face's own axis; x_n - x_p = -(x_p - x_n)
        // (a zero weight adds +-0 to each sum, which leaves it unchanged:
        // the same sums as k_p2g's skip of non-positive weights)
        {
          const R w = (w0x * w5y) * w5z;
          const R vel = pc[VX] + (pc[C00] * (-d0x) + pc[C01] * (-d5y)) + pc[C02] * (-d5z);
          const int t = halo_face(0, hx + unpack_delta(dl, 0), hy, hz);
          T[t] += m * w;
          T[kHaloF + t] += vel * m * w;
          T[2 * kHaloF + t] += vol * w;
        }
        {
          const R w = (w5x * w0y) * w5z;
          const R vel = pc[VY] + (pc[C10] * (-d5x) + pc[C11] * (-d0y)) + pc[C12] * (-d5z);
          const int t = halo_face(1, hx, hy + unpack_delta(dl, 1), hz);
          T[3 * kHaloF + t] += m * w;
          T[4 * kHaloF + t] += vel * m * w;
          T[5 * kHaloF + t] += vol * w;
        }
        {
          const R w = (w5x * w5y) * w0z;
          const R vel = pc[VZ] + (pc[C20] * (-d5x) + pc[C21] * (-d5y)) + pc[C22] * (-d0z);
          const int t = halo_face(2, hx, hy, hz + unpack_delta(dl, 2));
          T[6 * kHaloF + t] += m * w;
          T[7 * kHaloF + t] += vel * m * w;
          T[8 * kHaloF + t] += vol * w;
        }
        // cell centre: liquid level set over every particle of the 27 key
        // cells around the node, liquid volume over the positive weights
        {
          const int t = halo_centre(hx, hy, hz);
          const R r = pc[PR];
          const R d = sqrt((d5x * d5x + d5y * d5y) + d5z * d5z) - (rmin > r ? rmin : r);
          if (d < Tphi[t]) Tphi[t] = d;
          const R w = (w5x * w5y) * w5z;
          Tc[t] += vol * w;
        }
      }
      __syncwarp();
    }
  }
  R* H = halo + (long long)b * kTileVals;
  for (int e = lane; e < kTileVals; e += 32) H[e] = T[e];
}

// Merge: one block per active bucket, threads [0,64) u-faces, [64,128)
// v-faces, [128,192) w-faces, [192,256) cell centres (k_p2g's layout and
// outputs).  A node sums the tiles of the buckets whose halo holds it (at
// most two per axis: its own and, near the bucket's faces, the neighbour's),
// in a fixed (z, y, x) order of those buckets; the liquid phi is their
// minimum.  Buckets without particles have no tile and are skipped.
//
// The same block also writes the solid face weights (k_solid_weights'
// updateSolidWeights, TwoDScene.cpp:1871-1962) from the corner solid phi of
// the bucket's 5 x 5 x 5 corner nodes, evaluated once into shared memory
// (corners in missing buckets read 0.5 dx, as k_solid_weights reads them).
template <typename R>
__global__ void __launch_bounds__(256)
    k_p2g_merge(GridDesc g, const int* __restrict__ active_list,
                const unsigned char* __restrict__ active, const int* __restrict__ start,
                const R* __restrict__ halo, R* __restrict__ F, long long fstride, Walls walls,
                int raw_satp, int have_liquid) {
  __shared__ R corner[5][5][5];
  const int b = active_list[blockIdx.x];
  const int type = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int li = l & 3, lj = (l >> 2) & 3, lk = l >> 4;
  const int I = bi * 4 + li, J = bj * 4 + lj, K = bk * 4 + lk;
  const long long n = (long long)b * 64 + l;
  {
    const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
    const R bs = (R)g.bs, dx = (R)g.dx;
    const double three_bs = 3.0 * g.bs;
    for (int e = threadIdx.x; e < 125; e += blockDim.x) {
      const int ci = bi * 4 + e % 5, cj = bj * 4 + (e / 5) % 5, ck = bk * 4 + e / 25;
      R v = R(0.5) * dx;
      if (in_grid(g, ci, cj, ck) && active[bucket_of(g, ci, cj, ck)]) {
        const double cx = (double)coord<R>(org[0], bs, dx, ci, R(0));
        const double cy = (double)coord<R>(org[1], bs, dx, cj, R(0));
        const double cz = (double)coord<R>(org[2], bs, dx, ck, R(0));
        v = (R)wall_phi(walls, cx, cy, cz, three_bs);
      }
      corner[e / 25][(e / 5) % 5][e % 5] = v;
    }
    __syncthreads();
    if (type < 3) {
      R phi[4];
      for (int r = 0; r < 2; ++r)
        for (int s2 = 0; s2 < 2; ++s2) {
          int ci = li, cj = lj, ck = lk;
          if (type == 0) { cj += s2; ck += r; }
          else if (type == 1) { ci += r; ck += s2; }
          else { ci += r; cj += s2; }
          phi[r * 2 + s2] = corner[ck][cj][ci];
        }
      F[(G_WEIGHT + type) * fstride + n] =
          clamp01<R>(R(1) - fraction_inside4<R>(phi[0], phi[1], phi[2], phi[3]));
    }
  }
  const int bq[3] = {bi, bj, bk};
  const int nq[3] = {g.ni, g.nj, g.nk};
  const int L[3] = {li, lj, lk};
  // neighbour range per axis: bucket B-1 holds local node i when i + 5 < extent,
  // B+1 when i == 3
  int lo[3], hi[3];
  for (int q = 0; q < 3; ++q) {
    const int ext = (type < 3 && q == type) ? 7 : 6;
    lo[q] = (L[q] + 5 < ext && bq[q] > 0) ? -1 : 0;
    hi[q] = (L[q] == 3 && bq[q] + 1 < nq[q]) ? 1 : 0;
  }
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R dV = dx * dx * dx;
  const R den = dV > R(1e-20) ? dV : R(1e-20);
  if (type < 3) {
    const int a = type;
    R mass = 0, mom = 0, vol = 0;
    for (int dz = lo[2]; dz <= hi[2]; ++dz)
      for (int dy = lo[1]; dy <= hi[1]; ++dy)
        for (int dxb = lo[0]; dxb <= hi[0]; ++dxb) {
          const long long sb = ((long long)(bk + dz) * g.nj + (bj + dy)) * g.ni + (bi + dxb);
          if (start[sb * 64 + 64] <= start[sb * 64]) continue;
          const int t = halo_face(a, li + 1 - 4 * dxb, lj + 1 - 4 * dy, lk + 1 - 4 * dz);
          const R* H = halo + sb * kTileVals + 3 * a * kHaloF;
          mass += H[t];
          mom += H[kHaloF + t];
          vol += H[2 * kHaloF + t];
        }
    F[(G_MASS + a) * fstride + n] = mass;
    F[(G_VEL + a) * fstride + n] = mass > R(1e-20) ? mom / mass : R(0);
    F[(G_VOL + a) * fstride + n] = vol;
    F[(G_SAT + a) * fstride + n] = clamp01<R>(vol / den);
  } else {
    R phi = R(3) * bs;
    R vliq = 0;
    for (int dz = lo[2]; dz <= hi[2]; ++dz)
      for (int dy = lo[1]; dy <= hi[1]; ++dy)
        for (int dxb = lo[0]; dxb <= hi[0]; ++dxb) {
          const long long sb = ((long long)(bk + dz) * g.nj + (bj + dy)) * g.ni + (bi + dxb);
          if (start[sb * 64 + 64] <= start[sb * 64]) continue;
          const int t = halo_centre(li + 1 - 4 * dxb, lj + 1 - 4 * dy, lk + 1 - 4 * dz);
          const R* H = halo + sb * kTileVals + 9 * kHaloF;
          vliq += H[t];
          const R p = H[kHaloC + t];
          phi = p < phi ? p : phi;
        }
    const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
    R np_[3];
    const int IJK[3] = {I, J, K};
    for (int q = 0; q < 3; ++q) np_[q] = coord<R>(org[q], bs, dx, IJK[q], R(0.5));
    const double three_bs = 3.0 * g.bs;
    const double sphi_c = wall_phi(walls, (double)np_[0], (double)np_[1], (double)np_[2],
                                   three_bs);
    if (have_liquid && sphi_c < 0.0) phi = R(-0.5) * dx;
    F[G_LPHI * fstride + n] = phi;
    F[G_SATP * fstride + n] = raw_satp ? vliq : clamp01<R>(vliq / den);
    // solid phi at the corner node (TwoDScene::updateSolidPhi :7940-7960): the
    // bucket's own corner, active by definition
    F[G_SPHI * fstride + n] = corner[lk][lj][li];
  }
}

// Solid face weights: updateSolidWeights (TwoDScene.cpp:1871-1962); corner
// phis of missing corner nodes (outside the grid or in an inactive bucket)
// default to 0.5*dx.  Corner ordering per connectSolidPhiNodes (:4433-4596).
template <typename R>
__global__ void __launch_bounds__(192)
    k_solid_weights(GridDesc g, const int* __restrict__ active_list,
                    const unsigned char* __restrict__ active,
                    R* __restrict__ F, long long fstride, Walls walls) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const double three_bs = 3.0 * g.bs;
  R phi[4];
  for (int r = 0; r < 2; ++r)
    for (int s = 0; s < 2; ++s) {
      int ci = I, cj = J, ck = K;
      if (a == 0) { cj += s; ck += r; }
      else if (a == 1) { ci += r; ck += s; }
      else { ci += r; cj += s; }
      R v = R(0.5) * dx;
      if (in_grid(g, ci, cj, ck) && active[bucket_of(g, ci, cj, ck)]) {
        const double cx = (double)coord<R>(org[0], bs, dx, ci, R(0));
        const double cy = (double)coord<R>(org[1], bs, dx, cj, R(0));
        const double cz = (double)coord<R>(org[2], bs, dx, ck, R(0));
        v = (R)wall_phi(walls, cx, cy, cz, three_bs);
      }
      phi[r * 2 + s] = v;
    }
  F[(G_WEIGHT + a) * fstride + n] =
      clamp01<R>(R(1) - fraction_inside4<R>(phi[0], phi[1], phi[2], phi[3]));
}

// stepVelocity for liquid nodes (LinearizedImplicitEuler.cpp:224-337):
// constructNodeForce (:548-667) with SimpleGravityForce::addLiquidGradEToNode
// (SimpleGravityForce.cpp:25-52, coeff -dt) and the node momentum;
// constructHDV/constructInvMDV/constructPsiSF (:846-1149) with no solid
// (drag 0, Q_s = 1, inv_C = 1/m_f or 1); performLocalSolve (:128-170).
// mathutils::get_rotated_pore_coeff_* (MathUtilities.h:792-818) in closed
// form: the row sum along `axis` of (2 - sf) I + (2 sf - 1) n n^T, n = o/|o|;
// 0 for a zero orientation.
__device__ inline double pore_coeff(double o0, double o1, double o2, double sf, int axis) {
  const double n2 = (o0 * o0 + o1 * o1) + o2 * o2;
  if (!(n2 > 0.0)) return 0.0;
  const double oa = axis == 0 ? o0 : (axis == 1 ? o1 : o2);
  return (2.0 - sf) + (2.0 * sf - 1.0) * oa * ((o0 + o1) + o2) / n2;
}

// TwoDScene::getDragCoeffWithOrientation (TwoDScene.cpp:4042-4097), liquid,
// use_drag and use_nonlinear_drag on, yarn diameter 0.01, Yazdchi power 1.6;
// the rotated coefficient (mathutils::get_rotated_drag_*) is the row sum
// c_xy + (c_z - c_xy) n_axis (n_x + n_y + n_z).
__device__ inline double drag_coeff(double psi, double sat, double dv, double o0, double o1,
                                    double o2, double sf, int axis, double mu, double rho) {
  const double n2 = (o0 * o0 + o1 * o1) + o2 * o2;
  if (psi == 0.0 || sat == 0.0 || n2 < 1e-20) return 0.0;
  const double ergun = 0.1428869017, di = 0.01, yp = 1.6;
  const double lp = -log(psi);
  double ka = (lp - 1.476 + 2.0 * psi - 0.5 * psi * psi) / (16.0 * psi) * di * di;
  double kb = (lp - 1.476 + 2.0 * psi - 1.774 * psi * psi + 4.078 * pow(psi, 3.0)) /
              (32.0 * psi) * di * di;
  ka = fmax(1e-20, ka);
  kb = fmax(1e-20, kb);
  const double inertial = ergun * pow(di, yp - 1.0) * pow(mu, 1.0 - yp);
  const double flow = pow(rho * fabs(dv), yp);
  const double den = pow(1.0 - psi, 1.5);
  const double ca = fmin(1e63, mu / ka + inertial / (den * sqrt(ka)) * flow);
  const double cb = fmin(1e63, mu / kb + inertial / (den * sqrt(kb)) * flow);
  const double cxy = ca * (1.0 - sf) + cb * sf;
  const double cz = ca * sf + cb * (1.0 - sf);
  const double oa = axis == 0 ? o0 : (axis == 1 ? o1 : o2);
  return cxy + (cz - cxy) * oa * ((o0 + o1) + o2) / n2;
}

// With elasto particles (EF != null): the pore-pressure gradient term of
// pressure::computePorePressureGrads (Pressure.cpp:26-110) on the liquid rhs,
// constructHDV's drag between the P2G liquid and solid velocities
// (drag_by_air off: damped mass = solid mass), Q = hdV/(m_s + hdV), inv_C =
// 1/(m_f + Q m_s), psi_fs = (1 - psi) inv_C m_f (inv_Cs = 0 without the solid
// solve); Q goes to EF[E_Q].
template <typename R>
__global__ void __launch_bounds__(192)
    k_predict(GridDesc g, const int* __restrict__ active_list, R* __restrict__ F,
              long long fstride, R gx, R gy, R gz, R dt, R* __restrict__ EF,
              const unsigned char* __restrict__ active, double drag_mu, double rho) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const long long n = (long long)b * 64 + l;
  const R grav = a == 0 ? gx : (a == 1 ? gy : gz);
  const R m = F[(G_MASS + a) * fstride + n];
  const R u = F[(G_VEL + a) * fstride + n];
  R rhs = R(0) - (m * grav) * (-dt);
  if (EF) {
    const R vf = F[(G_VOL + a) * fstride + n];
    const R w = F[(G_WEIGHT + a) * fstride + n];
    if (vf > R(0) && w > R(0)) {
      const int bk = b / (g.ni * g.nj);
      const int rem = b - bk * g.ni * g.nj;
      const int bj = rem / g.ni;
      const int bi = rem - bj * g.ni;
      const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
      const int lI = I - (a == 0), lJ = J - (a == 1), lK = K - (a == 2);
      const R pp0 = in_grid(g, lI, lJ, lK) && active[bucket_of(g, lI, lJ, lK)]
                        ? EF[E_PORE * fstride + node_linear(g, lI, lJ, lK)]
                        : R(0);
      const R pp1 = EF[E_PORE * fstride + n];
      const R grad = (pp1 - pp0) / (R)g.dx;
      const R coeff = (R)pore_coeff((double)EF[(E_ORI + 3 * a) * fstride + n],
                                    (double)EF[(E_ORI + 3 * a + 1) * fstride + n],
                                    (double)EF[(E_ORI + 3 * a + 2) * fstride + n],
                                    (double)EF[(E_SF + a) * fstride + n], a);
      rhs += grad * vf * dt * F[(G_SAT + a) * fstride + n] * w * coeff;
    }
  }
  rhs += m * u;
  const bool heavy = m > R(1e-20);
  R invC = heavy ? R(1) / m : R(1);
  R psifs = invC * m;
  if (EF) {
    const R ms = EF[(E_MASS + a) * fstride + n], vs = EF[(E_VOL + a) * fstride + n];
    const R psi = EF[(E_PSI + a) * fstride + n];
    const double dc = drag_coeff(
        (double)psi, (double)F[(G_SAT + a) * fstride + n],
        (double)(u - EF[(E_VEL + a) * fstride + n]), (double)EF[(E_ORI + 3 * a) * fstride + n],
        (double)EF[(E_ORI + 3 * a + 1) * fstride + n],
        (double)EF[(E_ORI + 3 * a + 2) * fstride + n], (double)EF[(E_SF + a) * fstride + n], a,
        drag_mu, rho);
    const R hdV = dt * (R)dc * (vs + F[(G_VOL + a) * fstride + n]);
    const R msh = ms + hdV;
    const R Q = msh > R(1e-20) ? hdV / msh : R(1);
    const R C = m + Q * ms;
    invC = C > R(1e-20) ? R(1) / C : R(1);
    psifs = ((R(1) - psi) * invC + psi * R(0) * Q) * m;
    EF[(E_Q + a) * fstride + n] = Q;
  }
  F[(G_RHS + a) * fstride + n] = rhs;
  F[(G_INVC + a) * fstride + n] = invC;
  F[(G_VSTAR + a) * fstride + n] = heavy ? rhs / m : rhs;
  F[(G_PSIFS + a) * fstride + n] = psifs;
}

// Pressure system (pressure::solveNodePressure, Core/Pressure.cpp:350-791):
// DOF iff liquid phi < 0 and some existing face has solid weight > 0; per face
// rhs += -/+ ((u* psi_fs) w)/dx; if w > 0, term = (w dt/dx^2)(inv_C V_f); a
// liquid neighbour couples (diag += term, off = -term), an air neighbour adds
// term/max(fraction_inside(phi_c,phi_n), 0.01) to the diagonal.  Face order
// left, right, bottom, top, near, far.  Couplings are stored at the lower cell
// (A_x[c] = A(c, c+x)), giving a matrix-free symmetric 7-point operator.
template <typename R>
__global__ void __launch_bounds__(64)
    k_assemble(GridDesc g, const int* __restrict__ active_list,
               const unsigned char* __restrict__ active, R* __restrict__ F,
               long long fstride, unsigned char* __restrict__ dof, R dt,
               const R* __restrict__ EF) {
  const int b = active_list[blockIdx.x];
  const int l = threadIdx.x;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx;
  const R coeff = dt / (dx * dx);
  const R phic = F[G_LPHI * fstride + n];
  // faces: axis, face node, neighbour cell, sign of the rhs term
  const int fI[6] = {I, I + 1, I, I, I, I};
  const int fJ[6] = {J, J, J, J + 1, J, J};
  const int fK[6] = {K, K, K, K, K, K + 1};
  const int cI[6] = {I - 1, I + 1, I, I, I, I};
  const int cJ[6] = {J, J, J - 1, J + 1, J, J};
  const int cK[6] = {K, K, K, K, K - 1, K + 1};
  bool exists[6];
  long long fn[6];
  bool open = false;
  for (int f = 0; f < 6; ++f) {
    exists[f] = in_grid(g, fI[f], fJ[f], fK[f]) &&
                active[bucket_of(g, fI[f], fJ[f], fK[f])];
    fn[f] = exists[f] ? node_linear(g, fI[f], fJ[f], fK[f]) : -1;
    if (exists[f] && F[(G_WEIGHT + (f >> 1)) * fstride + fn[f]] > R(0)) open = true;
  }
  const bool isdof = (phic < R(0)) && open;
  // dof byte: bit0 DOF, bits1-3 a +x/+y/+z coupling entry exists, bit4 a
  // diagonal entry exists (entries can hold an exact zero when V_f == 0, and
  // the reference's sparse matrix still stores them).
  int flags = isdof ? 1 : 0;
  R diag = 0, rhs = 0, off[3] = {0, 0, 0};
  if (isdof) {
    for (int f = 0; f < 6; ++f) {
      if (!exists[f]) continue;
      const int a = f >> 1;
      const long long q = fn[f];
      const R w = F[(G_WEIGHT + a) * fstride + q];
      const R t = ((F[(G_VSTAR + a) * fstride + q] * F[(G_PSIFS + a) * fstride + q]) * w) / dx;
      if (f & 1) rhs -= t; else rhs += t;
      if (w > R(0)) {
        // with elasto: (1 - psi) inv_C (V_f + V_s Q) (+ psi inv_Cs (...), inv_Cs = 0)
        const R term =
            EF ? (w * coeff) * ((R(1) - EF[(E_PSI + a) * fstride + q]) * F[(G_INVC + a) * fstride + q] *
                                (F[(G_VOL + a) * fstride + q] +
                                 EF[(E_VOL + a) * fstride + q] * EF[(E_Q + a) * fstride + q]))
               : (w * coeff) * (F[(G_INVC + a) * fstride + q] * F[(G_VOL + a) * fstride + q]);
        if (in_grid(g, cI[f], cJ[f], cK[f]) &&
            active[bucket_of(g, cI[f], cJ[f], cK[f])]) {
          const R phin = F[G_LPHI * fstride + node_linear(g, cI[f], cJ[f], cK[f])];
          flags |= 16;
          if (phin < R(0)) {
            diag += term;
            if (f & 1) {
              off[a] = -term;
              flags |= 2 << a;
            }
          } else {
            R theta = fraction_inside2<R>(phic, phin);
            theta = theta > R(kThetaCriterion) ? theta : R(kThetaCriterion);
            diag += term / theta;
          }
        }
      }
    }
  }
  dof[n] = (unsigned char)flags;
  F[G_ADIAG * fstride + n] = diag;
  F[G_AX * fstride + n] = off[0];
  F[G_AY * fstride + n] = off[1];
  F[G_AZ * fstride + n] = off[2];
  F[G_B * fstride + n] = rhs;
}

// applyPressureGradsFluidRHS (Pressure.cpp:1137-1314) then performInvLocalSolve
// (LinearizedImplicitEuler.cpp:65-98): valid iff w > 0 and a side cell is
// liquid; rhs -= ((p_r - p_l)/(dx theta)) dt V_f;  u = rhs inv_C.
template <typename R>
__global__ void __launch_bounds__(192)
    k_apply_pressure(GridDesc g, const int* __restrict__ active_list,
                     const unsigned char* __restrict__ active, R* __restrict__ F,
                     long long fstride, unsigned char* __restrict__ valid, R dt,
                     const R* __restrict__ EF) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx;
  R rhs = F[(G_RHS + a) * fstride + n];
  // addSolidDragRHS (LinearizedImplicitEuler.cpp:689-717) with the P2G solid velocity
  const R Q = EF ? EF[(E_Q + a) * fstride + n] : R(0);
  if (EF) rhs += Q * EF[(E_MASS + a) * fstride + n] * EF[(E_VEL + a) * fstride + n];
  unsigned char v = 0;
  const R w = F[(G_WEIGHT + a) * fstride + n];
  if (w > R(0)) {
    const int lI = I - (a == 0), lJ = J - (a == 1), lK = K - (a == 2);
    const bool hl = in_grid(g, lI, lJ, lK) && active[bucket_of(g, lI, lJ, lK)];
    const bool hr = in_grid(g, I, J, K);  // the cell shares the face's bucket
    const long long nl = hl ? node_linear(g, lI, lJ, lK) : -1;
    const R phil = hl ? F[G_LPHI * fstride + nl] : R(0);
    const R phir = hr ? F[G_LPHI * fstride + n] : R(0);
    if (phil < R(0) || phir < R(0)) {
      R theta = 1;
      if (phir >= R(0) || phil >= R(0)) {
        theta = fraction_inside2<R>(phil, phir);
        theta = theta > R(kThetaCriterion) ? theta : R(kThetaCriterion);
      }
      R pg = 0;
      if (hl) pg -= F[G_PRESSURE * fstride + nl];
      if (hr) pg += F[G_PRESSURE * fstride + n];
      pg /= (dx * theta);
      const R term = EF ? pg * dt * (F[(G_VOL + a) * fstride + n] + EF[(E_VOL + a) * fstride + n] * Q)
                        : pg * dt * F[(G_VOL + a) * fstride + n];
      rhs -= term;
      v = 1;
    }
  }
  F[(G_RHS + a) * fstride + n] = rhs;
  F[(G_U + a) * fstride + n] = rhs * F[(G_INVC + a) * fstride + n];
  valid[a * fstride + n] = v;
}

// One layer of pressure::extrapolate (Pressure.cpp:1826-1903): an invalid face
// takes the mean of its valid 6-neighbours (order -x,+x,-y,+y,-z,+z) from the
// previous layer.
template <typename R>
__global__ void __launch_bounds__(192)
    k_extrapolate(GridDesc g, const int* __restrict__ active_list,
                  const unsigned char* __restrict__ active,
                  const R* __restrict__ uin, R* __restrict__ uout,
                  const unsigned char* __restrict__ vin,
                  unsigned char* __restrict__ vout, long long fstride) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R* ui = uin + a * fstride;
  const unsigned char* vi = vin + a * fstride;
  R out = ui[n];
  unsigned char vv = vi[n];
  if (!vv) {
    R sum = 0;
    int count = 0;
    const int dI[6] = {-1, 1, 0, 0, 0, 0};
    const int dJ[6] = {0, 0, -1, 1, 0, 0};
    const int dK[6] = {0, 0, 0, 0, -1, 1};
    for (int r = 0; r < 6; ++r) {
      const int x = I + dI[r], y = J + dJ[r], z = K + dK[r];
      if (!in_grid(g, x, y, z) || !active[bucket_of(g, x, y, z)]) continue;
      const long long q = node_linear(g, x, y, z);
      if (!vi[q]) continue;
      sum += ui[q];
      ++count;
    }
    if (count > 0) {
      out = sum / (R)count;
      vv = 1;
    }
  }
  uout[a * fstride + n] = out;
  vout[a * fstride + n] = vv;
}

// constrainLiquidVelocity (TwoDScene.cpp:1827-1869): faces fully inside the
// solid (weight 0) blend towards the (static, zero) solid velocity.
template <typename R>
__global__ void __launch_bounds__(192)
    k_constrain(const int* __restrict__ active_list, R* __restrict__ F,
                long long fstride, R friction) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  if (F[(G_WEIGHT + a) * fstride + n] == R(0)) {
    const R u = F[(G_U + a) * fstride + n];
    const R us = R(0);
    F[(G_U + a) * fstride + n] = (R(1) - friction) * u + friction * us;
  }
}

// The solid phi a liquid particle sees through its solid-phi stencil (offset
// 0 on every axis: base = key node - 1 + stencil offset), with the weights
// m_particle_weights(., 3) of updateParticleWeights (TwoDScene.cpp:2113-2127)
// taken at xw, the position the sub-step's weights were computed at:
//   phi = sum phi_n w_n,   grad = sum phi_n iD w_n (x_n - pos),   iD = 4/h^2,
// grad normalised when its norm exceeds 1e-20 (solidProjection :1786-1811,
// correctLiquidParticles :2030-2050); nodes of inactive buckets read 3 dx.
// Returns the norm of the unnormalised gradient.
template <typename R>
__device__ inline R solid_sample(const GridDesc& g, const unsigned char* __restrict__ active,
                                 const R* __restrict__ F, long long fstride, const int kp[3],
                                 int dl, const R xw[3], const R pos[3], R& phi_out, R grad[3]) {
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const R iD = R(4) / (dx * dx);
  int base[3];
  R c[3][3], w[3][3];
  for (int q = 0; q < 3; ++q) {
    base[q] = kp[q] + unpack_delta(dl, q);
    for (int t = 0; t < 3; ++t) {
      c[q][t] = coord<R>(org[q], bs, dx, base[q] + t, R(0));
      w[q][t] = quad_kernel<R>((xw[q] - c[q][t]) * invh);
    }
  }
  const R* S = F + G_SPHI * fstride;
  R phi = 0, g0 = 0, g1 = 0, g2 = 0;
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const int NI_ = base[0] + i, NJ_ = base[1] + j, NK_ = base[2] + k;
        const bool on = in_grid(g, NI_, NJ_, NK_) && active[bucket_of(g, NI_, NJ_, NK_)];
        const R ph = on ? S[node_linear(g, NI_, NJ_, NK_)] : R(3) * dx;
        const R wn = w[0][i] * w[1][j] * w[2][k];
        phi += ph * wn;
        const R cc = ph * iD * wn;
        g0 += cc * (c[0][i] - pos[0]);
        g1 += cc * (c[1][j] - pos[1]);
        g2 += cc * (c[2][k] - pos[2]);
      }
  const R nrm = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
  if (nrm > R(1e-20)) {
    g0 /= nrm;
    g1 /= nrm;
    g2 /= nrm;
  }
  phi_out = phi;
  grad[0] = g0;
  grad[1] = g1;
  grad[2] = g2;
  return nrm;
}

// x += v dt followed by TwoDScene::solidProjection (TwoDScene.cpp:1776-1821)
// of a liquid particle: with the solid phi extrapolated by the step,
// phi_now = phi + grad . v dt, a particle with phi_now < 0 moves by
// -phi_now grad.  xw: the position the sub-step's weights were taken at.
template <typename R>
__device__ inline void advect_project(const GridDesc& g, const unsigned char* __restrict__ active,
                                      const R* __restrict__ F, long long fstride,
                                      const int kp[3], int dl, const R xw[3], const R x[3],
                                      const R v[3], R dt, R out[3]) {
  R pos[3], d[3];
  for (int q = 0; q < 3; ++q) {
    d[q] = v[q] * dt;
    pos[q] = x[q] + d[q];
  }
  R phi, gr[3];
  solid_sample<R>(g, active, F, fstride, kp, dl, xw, pos, phi, gr);
  const R phi_now = phi + (gr[0] * d[0] + gr[1] * d[1] + gr[2] * d[2]);
  if (phi_now < R(0))
    for (int q = 0; q < 3; ++q) pos[q] -= phi_now * gr[q];
  for (int q = 0; q < 3; ++q) out[q] = pos[q];
}

// G2P of one liquid particle (mapNodeParticlesAPIC TwoDScene.cpp:6936-7000
// liquid branch) over its own 27-node face stencils, nodes of inactive
// buckets skipped:
//   v_a = sum u w;  C.row(a) = flip * sum u w (x_n - x_p) 4/h^2.
// The weights are taken at xw (the positions the sub-step's weights were
// computed at, before any particle correction), x_n - x_p from the current
// position x.  friction >= 0 applies constrainLiquidVelocity to each face
// value read (u (1 - friction) where the solid weight is 0); -1 reads U as is.
template <typename R>
__device__ inline void g2p_gather(const GridDesc& g, const unsigned char* __restrict__ active,
                                  const R* __restrict__ F, long long fstride, const int kp[3],
                                  int dl, const R xw[3], const R x[3], R flip, R friction,
                                  R v[3], R C[9]) {
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const R invD = R(4) / (dx * dx);
  for (int a = 0; a < 3; ++a) {
    int base[3];
    for (int q = 0; q < 3; ++q) base[q] = kp[q] + (q == a ? unpack_delta(dl, a) : 0);
    // per-axis node coordinates and weights
    R cx[3], cy[3], cz[3], wx[3], wy[3], wz[3];
    for (int t = 0; t < 3; ++t) {
      cx[t] = coord<R>(org[0], bs, dx, base[0] + t, a == 0 ? R(0) : R(0.5));
      cy[t] = coord<R>(org[1], bs, dx, base[1] + t, a == 1 ? R(0) : R(0.5));
      cz[t] = coord<R>(org[2], bs, dx, base[2] + t, a == 2 ? R(0) : R(0.5));
      wx[t] = quad_kernel<R>((xw[0] - cx[t]) * invh);
      wy[t] = quad_kernel<R>((xw[1] - cy[t]) * invh);
      wz[t] = quad_kernel<R>((xw[2] - cz[t]) * invh);
    }
    R fv = 0, b0 = 0, b1 = 0, b2 = 0;
    const R* U = F + (G_U + a) * fstride;
    const R* W = F + (G_WEIGHT + a) * fstride;
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          const int NI_ = base[0] + i, NJ_ = base[1] + j, NK_ = base[2] + k;
          if (!in_grid(g, NI_, NJ_, NK_) || !active[bucket_of(g, NI_, NJ_, NK_)])
            continue;
          const long long nn = node_linear(g, NI_, NJ_, NK_);
          R un = U[nn];
          if (friction >= R(0) && W[nn] == R(0)) un = (R(1) - friction) * un + friction * R(0);
          const R w = wx[i] * wy[j] * wz[k];
          const R uw = un * w;
          fv += uw;
          b0 += uw * (cx[i] - x[0]) * invD;
          b1 += uw * (cy[j] - x[1]) * invD;
          b2 += uw * (cz[k] - x[2]) * invD;
        }
    v[a] = fv;
    C[a * 3 + 0] = b0 * flip;
    C[a * 3 + 1] = b1 * flip;
    C[a * 3 + 2] = b2 * flip;
  }
}

// G2P + advection + solid projection (mapNodeParticlesAPIC, then
// SceneStepper::advectScene SceneStepper.cpp:17-41 and
// TwoDScene::solidProjection :1776-1821).  XW: positions before the particle
// correction (3 columns, stride pcap), or null when no correction ran.
template <typename R>
__global__ void __launch_bounds__(128)
    k_g2p(GridDesc g, const unsigned char* __restrict__ active, R* __restrict__ P,
          long long pcap, long long np, const long long* __restrict__ key,
          const int* __restrict__ delta, const R* __restrict__ F,
          long long fstride, R flip, R dt, int advect, const R* __restrict__ XW) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const R x[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
  R xw[3] = {x[0], x[1], x[2]};
  if (XW)
    for (int q = 0; q < 3; ++q) xw[q] = XW[q * pcap + s];
  const long long kn = key[s];
  if (kn < 0) return;
  int KI, KJ, KK;
  node_ijk(g, kn, KI, KJ, KK);
  const int kp[3] = {KI - 1, KJ - 1, KK - 1};
  const int dl = delta[s];
  R v[3], C[9];
  g2p_gather<R>(g, active, F, fstride, kp, dl, xw, x, flip, R(-1), v, C);
  for (int a = 0; a < 3; ++a) P[(VX + a) * pcap + s] = v[a];
  for (int q = 0; q < 9; ++q) P[(C00 + q) * pcap + s] = C[q];
  if (advect) {
    R xn[3];
    advect_project<R>(g, active, F, fstride, kp, dl, xw, x, v, dt, xn);
    for (int q = 0; q < 3; ++q) P[(PX + q) * pcap + s] = xn[q];
  }
}

// ---- G2P from a staged bucket neighbourhood ---------------------------------
// k_g2p's arithmetic with every node value read from shared memory: one block
// per active bucket stages the nodes its particles' stencils reach (the face
// velocities u, v, w over the P2G halo extents, and the corner solid phi over
// [4B-1, 4B+5] on each axis) once, then each thread advances particles of the
// bucket.  Nodes of inactive buckets stage 0 for the velocities (k_g2p skips
// them: the same sums) and 3 dx for the solid phi (solid_sample's value).
// Requires stencil offsets in {0, 1} (checked on the host).
constexpr int kCornerHalo = 7 * 7 * 7;
constexpr int kG2PTile = 3 * kHaloF + kCornerHalo;

template <typename R>
__global__ void __launch_bounds__(128)
    k_g2p_tile(GridDesc g, const int* __restrict__ active_list,
               const unsigned char* __restrict__ active, R* __restrict__ P, long long pcap,
               const int* __restrict__ start, const long long* __restrict__ key,
               const int* __restrict__ delta, const R* __restrict__ F, long long fstride,
               R flip, R dt, int advect, const R* __restrict__ XW) {
  __shared__ R T[kG2PTile];
  const int b = active_list[blockIdx.x];
  const long long n0 = (long long)b * 64;
  const int p0 = start[n0], p1 = start[n0 + 64];
  if (p1 <= p0) return;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int h0[3] = {4 * bi - 1, 4 * bj - 1, 4 * bk - 1};
  const R dx = (R)g.dx;
  for (int e = threadIdx.x; e < kG2PTile; e += blockDim.x) {
    int a, x, y, z;
    if (e < 3 * kHaloF) {
      a = e / kHaloF;
      const int r = e - a * kHaloF;
      const int nx = a == 0 ? 7 : 6, ny = a == 1 ? 7 : 6;
      x = r % nx;
      y = (r / nx) % ny;
      z = r / (nx * ny);
    } else {
      a = 3;
      const int r = e - 3 * kHaloF;
      x = r % 7;
      y = (r / 7) % 7;
      z = r / 49;
    }
    const int NI_ = h0[0] + x, NJ_ = h0[1] + y, NK_ = h0[2] + z;
    const bool on = in_grid(g, NI_, NJ_, NK_) && active[bucket_of(g, NI_, NJ_, NK_)];
    R val;
    if (a < 3)
      val = on ? F[(G_U + a) * fstride + node_linear(g, NI_, NJ_, NK_)] : R(0);
    else
      val = on ? F[G_SPHI * fstride + node_linear(g, NI_, NJ_, NK_)] : R(3) * dx;
    T[e] = val;
  }
  __syncthreads();
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs;
  const R invh = R(1) / dx;
  const R invD = R(4) / (dx * dx);
  for (int s = p0 + threadIdx.x; s < p1; s += blockDim.x) {
    const R x[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
    R xw[3] = {x[0], x[1], x[2]};
    if (XW)
      for (int q = 0; q < 3; ++q) xw[q] = XW[q * pcap + s];
    const int kl = (int)(key[s] & 63);
    const int cl[3] = {kl & 3, (kl >> 2) & 3, kl >> 4};
    const int dl = delta[s];
    R v[3], C[9];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // stencil node 0 on each axis: halo coordinate and global node index
      int hb[3];
      R cx[3], cy[3], cz[3], wx[3], wy[3], wz[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) hb[q] = cl[q] + (q == a ? unpack_delta(dl, a) : 0);
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        cx[t] = coord<R>(org[0], bs, dx, h0[0] + hb[0] + t, a == 0 ? R(0) : R(0.5));
        cy[t] = coord<R>(org[1], bs, dx, h0[1] + hb[1] + t, a == 1 ? R(0) : R(0.5));
        cz[t] = coord<R>(org[2], bs, dx, h0[2] + hb[2] + t, a == 2 ? R(0) : R(0.5));
        wx[t] = quad_kernel<R>((xw[0] - cx[t]) * invh);
        wy[t] = quad_kernel<R>((xw[1] - cy[t]) * invh);
        wz[t] = quad_kernel<R>((xw[2] - cz[t]) * invh);
      }
      const R* U = T + a * kHaloF;
      R fv = 0, b0 = 0, b1 = 0, b2 = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const R un = U[halo_face(a, hb[0] + i, hb[1] + j, hb[2] + k)];
            const R w = wx[i] * wy[j] * wz[k];
            const R uw = un * w;
            fv += uw;
            b0 += uw * (cx[i] - x[0]) * invD;
            b1 += uw * (cy[j] - x[1]) * invD;
            b2 += uw * (cz[k] - x[2]) * invD;
          }
      v[a] = fv;
      C[a * 3 + 0] = b0 * flip;
      C[a * 3 + 1] = b1 * flip;
      C[a * 3 + 2] = b2 * flip;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) P[(VX + a) * pcap + s] = v[a];
#pragma unroll
    for (int q = 0; q < 9; ++q) P[(C00 + q) * pcap + s] = C[q];
    if (!advect) continue;
    // advect_project with solid_sample over the staged corner phi
    R pos[3], d[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      d[q] = v[q] * dt;
      pos[q] = x[q] + d[q];
    }
    int hc[3];
    R sc[3][3], sw[3][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      hc[q] = cl[q] + unpack_delta(dl, q);
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        sc[q][t] = coord<R>(org[q], bs, dx, h0[q] + hc[q] + t, R(0));
        sw[q][t] = quad_kernel<R>((xw[q] - sc[q][t]) * invh);
      }
    }
    const R* S = T + 3 * kHaloF;
    R phi = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const R ph = S[((hc[2] + k) * 7 + (hc[1] + j)) * 7 + (hc[0] + i)];
          const R wn = sw[0][i] * sw[1][j] * sw[2][k];
          phi += ph * wn;
          const R cc = ph * invD * wn;
          g0 += cc * (sc[0][i] - pos[0]);
          g1 += cc * (sc[1][j] - pos[1]);
          g2 += cc * (sc[2][k] - pos[2]);
        }
    const R nrm = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
    if (nrm > R(1e-20)) {
      g0 /= nrm;
      g1 /= nrm;
      g2 /= nrm;
    }
    const R phi_now = phi + (g0 * d[0] + g1 * d[1] + g2 * d[2]);
    if (phi_now < R(0)) {
      pos[0] -= phi_now * g0;
      pos[1] -= phi_now * g1;
      pos[2] -= phi_now * g2;
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) P[(PX + q) * pcap + s] = pos[q];
  }
}

// advection + solid projection alone (after a separate G2P)
template <typename R>
__global__ void k_advect(GridDesc g, const unsigned char* __restrict__ active, R* __restrict__ P,
                         long long pcap, long long np, const long long* __restrict__ key,
                         const int* __restrict__ delta, const R* __restrict__ F,
                         long long fstride, R dt, const R* __restrict__ XW) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const R x[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
  const R v[3] = {P[VX * pcap + s], P[VY * pcap + s], P[VZ * pcap + s]};
  R xw[3] = {x[0], x[1], x[2]};
  if (XW)
    for (int q = 0; q < 3; ++q) xw[q] = XW[q * pcap + s];
  const long long kn = key[s];
  if (kn < 0) {
    for (int q = 0; q < 3; ++q) P[(PX + q) * pcap + s] = x[q] + v[q] * dt;
    return;
  }
  int KI, KJ, KK;
  node_ijk(g, kn, KI, KJ, KK);
  const int kp[3] = {KI - 1, KJ - 1, KK - 1};
  R xn[3];
  advect_project<R>(g, active, F, fstride, kp, delta[s], xw, x, v, dt, xn);
  for (int q = 0; q < 3; ++q) P[(PX + q) * pcap + s] = xn[q];
}

}  // namespace wcg
