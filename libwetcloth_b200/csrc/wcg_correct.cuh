// Particle correction: TwoDScene::correctLiquidParticles (TwoDScene.cpp:1967-2061),
// the Ando-style relaxation that pushes liquid particles apart, in a
// deterministic, seeded form.
//
// The reference sorts the liquid particles into the cells of the grid
// (grid_num_cells of rebucketizeParticles :1662-1669, key cell
// floor((x - origin)/dx) clamped, ties by index), then visits the cells in
// the 8 colours of Sorter::for_each_bucket_particles_colored (Sorter.h:403-437:
// z parity outermost, then y, then x), each cell's particles in index order,
// moving the particles of the chosen subset (index % step == selector) while
// reading the positions as they are being moved.  Cells of one colour are two
// apart, so no cell of a colour reads a cell another cell of the same colour
// writes: one thread per cell of the colour reproduces the serial order
// exactly, and a launch per colour orders the colours.
//
// The reference draws the selector with rand() and pushes coincident pairs
// (closer than 1e-4 re) by re * scalarRand(0, 1), neither reproducible; here
// the selector comes from a seeded SplitMix64 stream (Steele, Lea and Flood,
// OOPSLA 2014) and the push from SplitMix64 of the pair's indices.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_kernels.cuh"

namespace wcg {

__host__ __device__ inline unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// uniform [0, 1) for the coincident pair (i, j), component c
__device__ inline double pair_unit(int i, int j, int c) {
  const unsigned long long key = ((unsigned long long)(unsigned)i << 34) ^
                                 ((unsigned long long)(unsigned)j << 2) ^ (unsigned long long)c;
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

struct CellGrid {
  int n[3];         // grid_num_cells per axis
  double org[3];    // m_grid_mincorner
  double dx;
};

// correction cell of each particle (clamped), counted per cell
template <typename R>
__global__ void k_corr_cells(const R* __restrict__ P, long long pcap, long long np, CellGrid cg,
                             long long* __restrict__ cell, int* __restrict__ count) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  int c[3];
  for (int a = 0; a < 3; ++a) {
    const double x = (double)P[(PX + a) * pcap + s];
    int v = (int)floor((x - cg.org[a]) / cg.dx);
    v = v < 0 ? 0 : (v > cg.n[a] - 1 ? cg.n[a] - 1 : v);
    c[a] = v;
  }
  const long long id = ((long long)c[2] * cg.n[1] + c[1]) * cg.n[0] + c[0];
  cell[s] = id;
  atomicAdd(&count[id], 1);
}

// One colour (cx, cy, cz parities) of the correction: a thread per cell.
template <typename R>
__global__ void __launch_bounds__(128)
    k_correct(GridDesc g, CellGrid cg, int cx, int cy, int cz, R* P, long long pcap,
              const int* __restrict__ pid, const int* __restrict__ list,
              const int* __restrict__ start, const long long* __restrict__ key,
              const int* __restrict__ delta, const unsigned char* __restrict__ active,
              const R* __restrict__ F, long long fstride, const R* __restrict__ XW, int selector,
              int step, R coeff, R mult, R dt) {
  const int sn0 = (cg.n[0] + 1) / 2, sn1 = (cg.n[1] + 1) / 2, sn2 = (cg.n[2] + 1) / 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)sn0 * sn1 * sn2) return;
  const int sk = (int)(t / ((long long)sn0 * sn1));
  const int sj = (int)((t - (long long)sk * sn0 * sn1) / sn0);
  const int si = (int)(t - (long long)sk * sn0 * sn1 - (long long)sj * sn0);
  const int ci = si * 2 + cx, cj = sj * 2 + cy, ck = sk * 2 + cz;
  if (ci >= cg.n[0] || cj >= cg.n[1] || ck >= cg.n[2]) return;
  const long long cell = ((long long)ck * cg.n[1] + cj) * cg.n[0] + ci;
  const int q0 = start[cell], q1 = start[cell + 1];
  for (int q = q0; q < q1; ++q) {
    const int s = list[q];
    const int i = pid[s];
    if (i % step != selector) continue;
    const long long kn = key[s];
    if (kn < 0) continue;
    const R pos[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
    const R ri = P[PR * pcap + s];
    R spring[3] = {0, 0, 0};
    // neighbours of the 27 cells, x outermost (Sorter.h:352-371)
    for (int x = ci - 1; x <= ci + 1; ++x)
      for (int y = cj - 1; y <= cj + 1; ++y)
        for (int z = ck - 1; z <= ck + 1; ++z) {
          if (x < 0 || x > cg.n[0] - 1 || y < 0 || y > cg.n[1] - 1 || z < 0 || z > cg.n[2] - 1)
            continue;
          const long long nb = ((long long)z * cg.n[1] + y) * cg.n[0] + x;
          const int r1 = start[nb + 1];
          for (int r = start[nb]; r < r1; ++r) {
            const int s2 = list[r];
            if (s2 == s) continue;
            const R d[3] = {pos[0] - P[PX * pcap + s2], pos[1] - P[PY * pcap + s2],
                            pos[2] - P[PZ * pcap + s2]};
            const R re = sqrt(ri * P[PR * pcap + s2]) * mult;
            const R dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (dist > re) continue;
            // mathutils::smooth_kernel (MathUtilities.h:412)
            const R k3 = pow(R(1) - dist * dist / (re * re), R(3));
            const R w = coeff * (k3 > R(0) ? k3 : R(0));
            if (w == R(0)) continue;
            if (dist > R(1e-4) * re) {
              for (int a = 0; a < 3; ++a) spring[a] += w * d[a] / dist * re;
            } else {
              const int j = pid[s2];
              for (int a = 0; a < 3; ++a) spring[a] += re * (R)pair_unit(i, j, a);
            }
          }
        }
    R buf[3], dp[3];
    for (int a = 0; a < 3; ++a) {
      dp[a] = spring[a] * dt;
      buf[a] = pos[a] + dp[a];
    }
    int KI, KJ, KK;
    node_ijk(g, kn, KI, KJ, KK);
    const int kp[3] = {KI - 1, KJ - 1, KK - 1};
    const R xw[3] = {XW[0 * pcap + s], XW[1 * pcap + s], XW[2 * pcap + s]};
    R phi, gr[3];
    solid_sample<R>(g, active, F, fstride, kp, delta[s], xw, pos, phi, gr);
    const R phi_now = phi + (gr[0] * dp[0] + gr[1] * dp[1] + gr[2] * dp[2]);
    if (phi_now < R(0))
      for (int a = 0; a < 3; ++a) buf[a] -= phi_now * gr[a];
    for (int a = 0; a < 3; ++a) P[(PX + a) * pcap + s] = buf[a];
  }
}

// correctLiquidParticles at correction_strength 0 (TwoDScene.cpp:1967-2061):
// every spring weight is 0, so a selected particle (original index % step ==
// selector) only moves out of the solid -- phi_now = phi, and by -phi grad
// when phi < 0 -- and reads nothing but its own position and the grid, so a
// thread per particle gives the reference's result whatever the order.  XW
// receives every particle's position before the pass (G2P keeps its weights).
template <typename R>
__global__ void k_correct_project(GridDesc g, R* __restrict__ P, long long pcap, long long np,
                                  const int* __restrict__ pid, const long long* __restrict__ key,
                                  const int* __restrict__ delta,
                                  const unsigned char* __restrict__ active,
                                  const R* __restrict__ F, long long fstride,
                                  R* __restrict__ XW, int selector, int step) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const R pos[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
  for (int a = 0; a < 3; ++a) XW[a * pcap + s] = pos[a];
  if (pid[s] % step != selector) return;
  const long long kn = key[s];
  if (kn < 0) return;
  int KI, KJ, KK;
  node_ijk(g, kn, KI, KJ, KK);
  const int kp[3] = {KI - 1, KJ - 1, KK - 1};
  R phi, gr[3];
  solid_sample<R>(g, active, F, fstride, kp, delta[s], pos, pos, phi, gr);
  const R phi_now = phi + (gr[0] * R(0) + gr[1] * R(0) + gr[2] * R(0));
  if (phi_now < R(0))
    for (int a = 0; a < 3; ++a) P[(PX + a) * pcap + s] = pos[a] - phi_now * gr[a];
}

}  // namespace wcg
