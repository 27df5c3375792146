// Warp-tile wavefronts for the MIC(0) factorisation and triangular solves.
//
// One warp owns a tile of 8x4x8 cells (2x1x2 buckets); lane (pj, pk) owns the
// 8-cell x-pencil (i, pj, pk).  At intra-tile step s the lane handles cell
// i = s - pj - pk (reversed for the backward solve): its x-neighbour is its own
// previous result, its y- and z-neighbours are the results lanes (pj-1, pk) and
// (pj, pk-1) produced one step earlier, read with warp shuffles.  Per-cell
// operands live in shift registers consumed front-first, so the 18 intra-tile
// hyperplanes need neither shared memory nor block barriers.  Tiles are handed
// out by an atomic ticket in wave order (ti+tj+tk); a tile stages its static
// operands, waits (bounded) on the completion flags of its three upstream tiles,
// fetches their face values from L2 and publishes its own flag when done.
//
// Arithmetic per cell follows PCGSolver.h:97-239 as restated in wcg_pcg.cuh.
#pragma once

#include "wcg_pcg.cuh"

namespace wcg {

constexpr int WX = 8, WY = 4, WZ = 8;  // warp tile (cells)
constexpr unsigned kFull = 0xffffffffu;

// node index of cell (I, J, K) if it is a DOF, else -1
__device__ inline long long dof_node(const GridDesc& g, int I, int J, int K,
                                     const unsigned char* active,
                                     const unsigned char* dof) {
  if (!in_grid(g, I, J, K)) return -1;
  const long long b = bucket_of(g, I, J, K);
  if (!active[b]) return -1;
  const long long n = b * 64 + (((K & 3) << 4) | ((J & 3) << 2) | (I & 3));
  return dof[n] ? n : -1;
}

template <typename R>
__device__ inline R ld_or0(const R* p, long long n) {
  return n >= 0 ? p[n] : R(0);
}

template <typename R>
__device__ inline R ldcg_or0(const R* p, long long n) {
  return n >= 0 ? __ldcg(p + n) : R(0);
}

// shift an 8-entry register array one slot towards the front
template <typename R>
__device__ inline void shift8(R (&a)[8]) {
#pragma unroll
  for (int k = 0; k < 7; ++k) a[k] = a[k + 1];
  a[7] = R(0);
}

template <typename R, int MODE>
__global__ void __launch_bounds__(32)
    k_wsweep(const SweepArgs<R> a) {
  const GridDesc& g = a.g;
  if (*(const int*)(a.sc + S_DONE)) return;
  const int lane = threadIdx.x;
  int t = 0;
  if (lane == 0) t = atomicAdd(a.ticket, 1);
  t = __shfl_sync(kFull, t, 0);
  if (t >= a.ntiles) return;
  const int tl = MODE == kBackward ? a.tile_list[a.ntiles - 1 - t] : a.tile_list[t];
  const int tk = tl / (a.nti * a.ntj);
  const int trem = tl - tk * a.nti * a.ntj;
  const int tj = trem / a.nti;
  const int ti = trem - tj * a.nti;
  const int pj = lane & 3, pk = lane >> 2;
  const int I0 = ti * WX, J = tj * WY + pj, K = tk * WZ + pk;
  const R* F = a.F;
  const long long fs = a.fs;
  const bool back = MODE == kBackward;

  // own cells, in processing order (backward: i = 7 .. 0)
  long long nd[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int i = back ? 7 - e : e;
    nd[e] = dof_node(g, I0 + i, J, K, a.active, a.dof);
  }

  R c0[8], c1[8], c2[8], c3[8], c4[8];  // per-cell operands (see per mode)
  R hy[8], hz[8];                        // face values of the y/z upstream tile
  double rmax = 0;
  // ---- stage static operands ----
  if (MODE == kFactor) {
    // c0 = A_diag, c1..c3 = own A_x, A_y, A_z
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      c0[e] = ld_or0(F + G_ADIAG * fs, nd[e]);
      c1[e] = ld_or0(F + G_AX * fs, nd[e]);
      c2[e] = ld_or0(F + G_AY * fs, nd[e]);
      c3[e] = ld_or0(F + G_AZ * fs, nd[e]);
      c4[e] = R(0);
    }
  } else if (MODE == kForward) {
    // c0 = r (after the fused update), c1 = invdiag, c2 = own S_x, c3 = S_y of
    // the y-lower cell, c4 = S_z of the z-lower cell
    const R al = a.update ? (R)a.sc[S_ALPHA] : R(0);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const long long n = nd[e];
      R rv = ld_or0(a.in, n);
      if (a.update && n >= 0) {
        a.x[n] = a.x[n] + al * a.s[n];
        rv = rv - al * a.q[n];
        a.r[n] = rv;
        const double av = fabs((double)rv);
        rmax = av > rmax ? av : rmax;
      }
      c0[e] = rv;
      c1[e] = ld_or0(F + G_INVDIAG * fs, n);
      c2[e] = ld_or0(F + G_SX * fs, n);
      c3[e] = ld_or0(F + G_SY * fs, n);
      c4[e] = ld_or0(F + G_SZ * fs, n);
    }
  } else {
    // c0 = y, c1 = invdiag, c2..c4 = own S_x, S_y, S_z
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const long long n = nd[e];
      c0[e] = ld_or0(a.in, n);
      c1[e] = ld_or0(F + G_INVDIAG * fs, n);
      c2[e] = ld_or0(F + G_SX * fs, n);
      c3[e] = ld_or0(F + G_SY * fs, n);
      c4[e] = ld_or0(F + G_SZ * fs, n);
    }
  }
  // couplings of the y/z-lower cells (forward) come from the neighbour lanes or
  // the upstream tile; the factor needs all three A's of each lower neighbour
  R ym[3][8], zm[3][8];
  const int dj = back ? 1 : -1;
  const bool ybound = back ? pj == WY - 1 : pj == 0;
  const bool zbound = back ? pk == WZ - 1 : pk == 0;
  long long hyn[8], hzn[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int i = back ? 7 - e : e;
    hyn[e] = ybound ? dof_node(g, I0 + i, J + dj, K, a.active, a.dof) : -1;
    hzn[e] = zbound ? dof_node(g, I0 + i, J, K + dj, a.active, a.dof) : -1;
  }
  if (MODE == kFactor) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const R y0 = __shfl_up_sync(kFull, c1[e], 1), y1 = __shfl_up_sync(kFull, c2[e], 1),
              y2 = __shfl_up_sync(kFull, c3[e], 1);
      const R z0 = __shfl_up_sync(kFull, c1[e], 4), z1 = __shfl_up_sync(kFull, c2[e], 4),
              z2 = __shfl_up_sync(kFull, c3[e], 4);
      ym[0][e] = ybound ? ld_or0(F + G_AX * fs, hyn[e]) : y0;
      ym[1][e] = ybound ? ld_or0(F + G_AY * fs, hyn[e]) : y1;
      ym[2][e] = ybound ? ld_or0(F + G_AZ * fs, hyn[e]) : y2;
      zm[0][e] = zbound ? ld_or0(F + G_AX * fs, hzn[e]) : z0;
      zm[1][e] = zbound ? ld_or0(F + G_AY * fs, hzn[e]) : z1;
      zm[2][e] = zbound ? ld_or0(F + G_AZ * fs, hzn[e]) : z2;
    }
  } else if (MODE == kForward) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const R ys = __shfl_up_sync(kFull, c3[e], 1);
      const R zs = __shfl_up_sync(kFull, c4[e], 4);
      ym[0][e] = ybound ? ld_or0(F + G_SY * fs, hyn[e]) : ys;
      zm[0][e] = zbound ? ld_or0(F + G_SZ * fs, hzn[e]) : zs;
    }
  }
  // x-neighbour across the tile face (static part)
  const long long hxn = dof_node(g, back ? I0 + WX : I0 - 1, J, K, a.active, a.dof);
  R hxA0 = 0, hxA1 = 0, hxA2 = 0;
  if (MODE == kFactor) {
    hxA0 = ld_or0(F + G_AX * fs, hxn);
    hxA1 = ld_or0(F + G_AY * fs, hxn);
    hxA2 = ld_or0(F + G_AZ * fs, hxn);
  } else if (MODE == kForward) {
    hxA0 = ld_or0(F + G_SX * fs, hxn);
  }

  // ---- wait for the upstream tiles ----
  if (lane < 3) {
    const int st = back ? 1 : -1;
    const int x = ti + (lane == 0 ? st : 0), y = tj + (lane == 1 ? st : 0),
              z = tk + (lane == 2 ? st : 0);
    if (x >= 0 && y >= 0 && z >= 0 && x < a.nti && y < a.ntj && z < a.ntk) {
      const long long ut = ((long long)z * a.ntj + y) * a.nti + x;
      if (a.tile_active[ut]) wait_tile(a.flags + ut, a.epoch, a.err);
    }
  }
  __syncwarp();
  // ---- face values of the upstream tiles ----
  const R* dyn = MODE == kFactor ? (const R*)(F + G_INVDIAG * fs) : (const R*)a.out;
  const R hx = ldcg_or0(dyn, hxn);
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    hy[e] = ldcg_or0(dyn, hyn[e]);
    hz[e] = ldcg_or0(dyn, hzn[e]);
  }

  // ---- intra-tile wavefront ----
  const int d = back ? (WY - 1 - pj) + (WZ - 1 - pk) : pj + pk;
  R res[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) res[e] = R(0);
  R prev = R(0);    // this lane's result of the previous step
  R xv = hx;        // x-neighbour value (own previous cell)
  R xa0 = hxA0, xa1 = hxA1, xa2 = hxA2;  // x-neighbour couplings (factor/forward)
#pragma unroll
  for (int s = 0; s < WX + WY + WZ - 2; ++s) {
    const R uy = back ? __shfl_down_sync(kFull, prev, 1) : __shfl_up_sync(kFull, prev, 1);
    const R uz = back ? __shfl_down_sync(kFull, prev, 4) : __shfl_up_sync(kFull, prev, 4);
    R out = R(0);
    if (s >= d && s < d + 8) {
      const R vy = ybound ? hy[0] : uy;
      const R vz = zbound ? hz[0] : uz;
      if (MODE == kFactor) {
        const R adiag = c0[0];
        R dd = adiag;
        R iv = R(0);
        if (adiag != R(0)) {
          // lower neighbours in the reference's interior column order -z, -y, -x
          if (vz != R(0)) {
            const R L = zm[2][0] * vz;
            const R miss = zm[0][0] * vz + zm[1][0] * vz;
            dd = dd - L * L;
            dd = dd - (a.omega * L) * miss;
          }
          if (vy != R(0)) {
            const R L = ym[1][0] * vy;
            const R miss = ym[0][0] * vy + ym[2][0] * vy;
            dd = dd - L * L;
            dd = dd - (a.omega * L) * miss;
          }
          if (xv != R(0)) {
            const R L = xa0 * xv;
            const R miss = xa1 * xv + xa2 * xv;
            dd = dd - L * L;
            dd = dd - (a.omega * L) * miss;
          }
          const R piv = dd < a.min_ratio * adiag ? adiag : dd;
          iv = R(1) / sqrt(piv);
        }
        out = iv;
        xa0 = c1[0];
        xa1 = c2[0];
        xa2 = c3[0];
      } else if (MODE == kForward) {
        R v = c0[0];
        v -= zm[0][0] * vz;
        v -= ym[0][0] * vy;
        v -= xa0 * xv;
        out = v * c1[0];
        xa0 = c2[0];
      } else {
        R v = c0[0];
        v -= c2[0] * xv;
        v -= c3[0] * vy;
        v -= c4[0] * vz;
        out = v * c1[0];
      }
      xv = out;
#pragma unroll
      for (int e = 0; e < 7; ++e) res[e] = res[e + 1];
      res[7] = out;
      shift8(c0);
      shift8(c1);
      shift8(c2);
      shift8(c3);
      shift8(c4);
      shift8(hy);
      shift8(hz);
      if (MODE == kFactor) {
        shift8(ym[0]); shift8(ym[1]); shift8(ym[2]);
        shift8(zm[0]); shift8(zm[1]); shift8(zm[2]);
      } else if (MODE == kForward) {
        shift8(ym[0]);
        shift8(zm[0]);
      }
    }
    prev = out;
  }

  // ---- write back (res[e] = result of the e-th processed cell) ----
  double dsum = 0;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const long long n = nd[e];
    if (n < 0) continue;
    if (MODE == kFactor) {
      const R iv = res[e];
      a.F[G_INVDIAG * fs + n] = iv;
      a.F[G_SX * fs + n] = F[G_AX * fs + n] * iv;
      a.F[G_SY * fs + n] = F[G_AY * fs + n] * iv;
      a.F[G_SZ * fs + n] = F[G_AZ * fs + n] * iv;
    } else {
      a.out[n] = res[e];
      if (MODE == kBackward && a.part) dsum += (double)res[e] * (double)a.r[n];
    }
  }
  if (MODE == kForward && a.update && a.part) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double v = __shfl_xor_sync(kFull, rmax, o);
      rmax = v > rmax ? v : rmax;
    }
    if (lane == 0) a.part[tl] = rmax;
  }
  if (MODE == kBackward && a.part) {
    // fixed butterfly order: deterministic
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(kFull, dsum, o);
    if (lane == 0) a.part[tl] = dsum;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) st_release_gpu(a.flags + tl, a.epoch);
}

// MIC(0) factorisation on the same warp tiles, operands in shared memory
// (indexed [cell e][lane]; the factor runs once per solve, so it trades the
// register shift pipeline of k_wsweep for a smaller footprint).
template <typename R>
__global__ void __launch_bounds__(32)
    k_wfactor(const SweepArgs<R> a) {
  __shared__ R sA[4][8][32];     // A_diag, A_x, A_y, A_z of own cells
  __shared__ R sYA[3][8][32];    // A_x, A_y, A_z of the y-lower face cells (pj == 0)
  __shared__ R sZA[3][8][32];    // ... of the z-lower face cells (pk == 0)
  __shared__ R sHv[2][8][32];    // invdiag of the y-/z-lower face cells
  __shared__ R sV[8][32];        // own invdiag results
  const GridDesc& g = a.g;
  const int lane = threadIdx.x;
  int t = 0;
  if (lane == 0) t = atomicAdd(a.ticket, 1);
  t = __shfl_sync(kFull, t, 0);
  if (t >= a.ntiles) return;
  const int tl = a.tile_list[t];
  const int tk = tl / (a.nti * a.ntj);
  const int trem = tl - tk * a.nti * a.ntj;
  const int tj = trem / a.nti;
  const int ti = trem - tj * a.nti;
  const int pj = lane & 3, pk = lane >> 2;
  const int I0 = ti * WX, J = tj * WY + pj, K = tk * WZ + pk;
  const R* F = a.F;
  const long long fs = a.fs;
  for (int e = 0; e < 8; ++e) {
    const long long n = dof_node(g, I0 + e, J, K, a.active, a.dof);
    sA[0][e][lane] = ld_or0(F + G_ADIAG * fs, n);
    sA[1][e][lane] = ld_or0(F + G_AX * fs, n);
    sA[2][e][lane] = ld_or0(F + G_AY * fs, n);
    sA[3][e][lane] = ld_or0(F + G_AZ * fs, n);
    const long long yn = pj == 0 ? dof_node(g, I0 + e, J - 1, K, a.active, a.dof) : -1;
    const long long zn = pk == 0 ? dof_node(g, I0 + e, J, K - 1, a.active, a.dof) : -1;
    for (int c = 0; c < 3; ++c) {
      sYA[c][e][lane] = ld_or0(F + (G_AX + c) * fs, yn);
      sZA[c][e][lane] = ld_or0(F + (G_AX + c) * fs, zn);
    }
    sV[e][lane] = R(0);
  }
  const long long hxn = dof_node(g, I0 - 1, J, K, a.active, a.dof);
  const R hxA0 = ld_or0(F + G_AX * fs, hxn), hxA1 = ld_or0(F + G_AY * fs, hxn),
          hxA2 = ld_or0(F + G_AZ * fs, hxn);
  if (lane < 3) {
    const int x = ti - (lane == 0), y = tj - (lane == 1), z = tk - (lane == 2);
    if (x >= 0 && y >= 0 && z >= 0) {
      const long long ut = ((long long)z * a.ntj + y) * a.nti + x;
      if (a.tile_active[ut]) wait_tile(a.flags + ut, a.epoch, a.err);
    }
  }
  __syncwarp();
  const R* INV = F + G_INVDIAG * fs;
  const R hx = ldcg_or0(INV, hxn);
  for (int e = 0; e < 8; ++e) {
    const long long yn = pj == 0 ? dof_node(g, I0 + e, J - 1, K, a.active, a.dof) : -1;
    const long long zn = pk == 0 ? dof_node(g, I0 + e, J, K - 1, a.active, a.dof) : -1;
    sHv[0][e][lane] = ldcg_or0(INV, yn);
    sHv[1][e][lane] = ldcg_or0(INV, zn);
  }
  __syncwarp();
  const int d = pj + pk;
  for (int s = 0; s < WX + WY + WZ - 2; ++s) {
    const int e = s - d;
    if (e >= 0 && e < 8) {
      const R adiag = sA[0][e][lane];
      R dd = adiag;
      R iv = R(0);
      if (adiag != R(0)) {
        // lower neighbours in the reference's interior column order -z, -y, -x
        R vz, z0, z1, z2;
        if (pk > 0) { vz = sV[e][lane - 4]; z0 = sA[1][e][lane - 4]; z1 = sA[2][e][lane - 4]; z2 = sA[3][e][lane - 4]; }
        else { vz = sHv[1][e][lane]; z0 = sZA[0][e][lane]; z1 = sZA[1][e][lane]; z2 = sZA[2][e][lane]; }
        if (vz != R(0)) {
          const R L = z2 * vz;
          const R miss = z0 * vz + z1 * vz;
          dd = dd - L * L;
          dd = dd - (a.omega * L) * miss;
        }
        R vy, y0, y1, y2;
        if (pj > 0) { vy = sV[e][lane - 1]; y0 = sA[1][e][lane - 1]; y1 = sA[2][e][lane - 1]; y2 = sA[3][e][lane - 1]; }
        else { vy = sHv[0][e][lane]; y0 = sYA[0][e][lane]; y1 = sYA[1][e][lane]; y2 = sYA[2][e][lane]; }
        if (vy != R(0)) {
          const R L = y1 * vy;
          const R miss = y0 * vy + y2 * vy;
          dd = dd - L * L;
          dd = dd - (a.omega * L) * miss;
        }
        R vx, x0, x1, x2;
        if (e > 0) { vx = sV[e - 1][lane]; x0 = sA[1][e - 1][lane]; x1 = sA[2][e - 1][lane]; x2 = sA[3][e - 1][lane]; }
        else { vx = hx; x0 = hxA0; x1 = hxA1; x2 = hxA2; }
        if (vx != R(0)) {
          const R L = x0 * vx;
          const R miss = x1 * vx + x2 * vx;
          dd = dd - L * L;
          dd = dd - (a.omega * L) * miss;
        }
        const R piv = dd < a.min_ratio * adiag ? adiag : dd;
        iv = R(1) / sqrt(piv);
      }
      sV[e][lane] = iv;
    }
    __syncwarp();
  }
  for (int e = 0; e < 8; ++e) {
    const long long n = dof_node(g, I0 + e, J, K, a.active, a.dof);
    if (n < 0) continue;
    const R iv = sV[e][lane];
    a.F[G_INVDIAG * fs + n] = iv;
    a.F[G_SX * fs + n] = sA[1][e][lane] * iv;
    a.F[G_SY * fs + n] = sA[2][e][lane] * iv;
    a.F[G_SZ * fs + n] = sA[3][e][lane] * iv;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) st_release_gpu(a.flags + tl, a.epoch);
}

// tiles of 2x1x2 buckets containing an active bucket
__global__ void k_wtile_active(GridDesc g, int nti, int ntj, int ntk,
                               const unsigned char* __restrict__ active,
                               unsigned char* __restrict__ tact) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nt = (long long)nti * ntj * ntk;
  if (t >= nt) return;
  const int tk = (int)(t / ((long long)nti * ntj));
  const int rem = (int)(t - (long long)tk * nti * ntj);
  const int tj = rem / nti;
  const int ti = rem - tj * nti;
  unsigned char any = 0;
  for (int m = 0; m < 4; ++m) {
    const int bi = ti * 2 + (m & 1), bj = tj, bk = tk * 2 + (m >> 1);
    if (bi < g.ni && bj < g.nj && bk < g.nk &&
        active[((long long)bk * g.nj + bj) * g.ni + bi])
      any = 1;
  }
  tact[t] = any;
}

}  // namespace wcg
