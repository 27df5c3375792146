// Multigrid-preconditioned CG: the reference's default pressure solver.
//
// Restates AMGPCGSolveSparse (libWetCloth/Core/AlgebraicMultigrid.h:248-361)
// with the levels of levelGen::generateLevelsGalerkinCoarseningSparse
// (GeometricLevelGen.h:125-249) and the V-cycle of amgVCycleCompressed
// (AlgebraicMultigrid.h:170-237):
//  * level l + 1 aggregates 2 x 2 x 2 cells of level l (cell (i, j, k) -> (i/2,
//    j/2, k/2)); prolongation P puts 1 on every DOF child, restriction
//    R = 0.125 P^T, and A_{l+1} = 0.5 R A_l P = P^T A_l P / 16.  Aggregating a
//    7-point operator keeps it 7-point: the diagonal of an aggregate is 1/16 of
//    its children's diagonals plus twice their internal couplings, and its
//    coupling to the next aggregate along an axis is 1/16 of the couplings that
//    cross the face.  Levels are added while a level has more than 4096 DOFs.
//  * the smoother is red-black Gauss-Seidel (RBGS_with_pattern, :103-166):
//    cells with (i + j + k) odd first, then even, x = (b - sum_offdiag) / diag;
//    4 sweeps before restriction and after prolongation, 200 on the coarsest
//    level; restriction b_{l+1} = R (b_l - A_l x_l), prolongation x_l += P x_{l+1}.
//  * the preconditioner is one V-cycle from x = 0.
// Every level is stored densely over its box of cells (i + ni (j + nj k)),
// with the diagonal and the couplings to the +x, +y, +z neighbour per cell and
// a DOF mask; cells that are not DOFs hold zeros.  Each colour of a sweep is one
// fully parallel launch.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_pcg.cuh"

namespace wcg {

template <typename R>
struct MgLevel {
  int ni, nj, nk;
  int n;                    // ni * nj * nk
  R* d;                     // diagonal
  R* ax;                    // coupling to the +x neighbour
  R* ay;
  R* az;
  R* x;                     // level solution
  R* b;                     // level rhs
  unsigned char* m;         // DOF mask
};

constexpr int kMgThreads = 256;
constexpr int kMgBlocks = 1184;  // 8 x 148 SMs
constexpr int kMgCoarseThreads = 1024;

__device__ inline void mg_ijk(int idx, int ni, int nj, int& i, int& j, int& k) {
  k = idx / (ni * nj);
  const int r = idx - k * ni * nj;
  j = r / ni;
  i = r - j * ni;
}

// sum of A(row, col) x(col) over the six neighbours, order -z -y -x +x +y +z
template <typename R>
__device__ inline R mg_offdiag(const MgLevel<R>& L, const R* __restrict__ x, int idx, int i,
                               int j, int k) {
  const int sj = L.ni, sk = L.ni * L.nj;
  R s = R(0);
  if (k > 0) s += L.az[idx - sk] * x[idx - sk];
  if (j > 0) s += L.ay[idx - sj] * x[idx - sj];
  if (i > 0) s += L.ax[idx - 1] * x[idx - 1];
  if (i + 1 < L.ni) s += L.ax[idx] * x[idx + 1];
  if (j + 1 < L.nj) s += L.ay[idx] * x[idx + sj];
  if (k + 1 < L.nk) s += L.az[idx] * x[idx + sk];
  return s;
}

// Level 0 from the assembled bucket-major system: diagonal, couplings between
// two DOF cells, rhs and mask over the whole grid of cells.
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_gather0(GridDesc g, const unsigned char* __restrict__ active,
                 const unsigned char* __restrict__ dof, const R* __restrict__ F, long long fs,
                 MgLevel<R> L, R* __restrict__ rhs) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < L.n; idx += gridDim.x * blockDim.x) {
    int I, J, K;
    mg_ijk(idx, L.ni, L.nj, I, J, K);
    R d = 0, cx = 0, cy = 0, cz = 0, bv = 0;
    unsigned char msk = 0;
    if (active[bucket_of(g, I, J, K)]) {
      const long long n = node_linear(g, I, J, K);
      if (dof[n] & 1) {
        msk = 1;
        d = F[G_ADIAG * fs + n];
        bv = F[G_B * fs + n];
        R c[3];
        for (int a = 0; a < 3; ++a) {
          const int Q[3] = {I + (a == 0), J + (a == 1), K + (a == 2)};
          c[a] = R(0);
          if (in_grid(g, Q[0], Q[1], Q[2]) && active[bucket_of(g, Q[0], Q[1], Q[2])] &&
              (dof[node_linear(g, Q[0], Q[1], Q[2])] & 1))
            c[a] = F[(G_AX + a) * fs + n];
        }
        cx = c[0]; cy = c[1]; cz = c[2];
      }
    }
    L.d[idx] = d; L.ax[idx] = cx; L.ay[idx] = cy; L.az[idx] = cz;
    L.m[idx] = msk;
    L.x[idx] = R(0);
    rhs[idx] = bv;
  }
}

// Galerkin coarse level c = P^T f P / 16 over 2x2x2 aggregates; partial[block]
// = number of coarse DOFs.
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_coarsen(MgLevel<R> f, MgLevel<R> c, double* __restrict__ partial) {
  __shared__ double sm[kMgThreads];
  double cnt = 0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < c.n; idx += gridDim.x * blockDim.x) {
    int I, J, K;
    mg_ijk(idx, c.ni, c.nj, I, J, K);
    R dsum = 0, sx = 0, sy = 0, sz = 0;
    unsigned char msk = 0;
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
          if (i >= f.ni || j >= f.nj || k >= f.nk) continue;
          const int e = i + f.ni * (j + f.nj * k);
          if (!f.m[e]) continue;
          msk = 1;
          dsum += f.d[e];
          // couplings inside the aggregate count twice (A_ij and A_ji)
          if (di == 0 && i + 1 < f.ni) dsum += R(2) * f.ax[e];
          if (dj == 0 && j + 1 < f.nj) dsum += R(2) * f.ay[e];
          if (dk == 0 && k + 1 < f.nk) dsum += R(2) * f.az[e];
          // couplings across the + faces of the aggregate
          if (di == 1) sx += f.ax[e];
          if (dj == 1) sy += f.ay[e];
          if (dk == 1) sz += f.az[e];
        }
    const R s16 = R(0.0625);
    c.d[idx] = dsum * s16;
    c.ax[idx] = sx * s16;
    c.ay[idx] = sy * s16;
    c.az[idx] = sz * s16;
    c.m[idx] = msk;
    c.x[idx] = R(0);
    c.b[idx] = R(0);
    cnt += msk ? 1.0 : 0.0;
  }
  cnt = block_sum<double>(cnt, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = cnt;
}

// One colour of a red-black Gauss-Seidel sweep: parity 1 = cells with
// (i + j + k) odd (RBGS_with_pattern's first pass), 0 = even.
template <typename R>
__global__ void __launch_bounds__(kMgThreads) k_mg_smooth(MgLevel<R> L, int parity) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < L.n; idx += gridDim.x * blockDim.x) {
    if (!L.m[idx]) continue;
    int i, j, k;
    mg_ijk(idx, L.ni, L.nj, i, j, k);
    if (((i + j + k) & 1) != parity) continue;
    const R s = mg_offdiag(L, L.x, idx, i, j, k);
    const R d = L.d[idx];
    L.x[idx] = d != R(0) ? (L.b[idx] - s) / d : R(0);
  }
}

// The coarsest level: `iters` red-black sweeps in one CTA (the level is small;
// the barrier orders the colours).
template <typename R>
__global__ void __launch_bounds__(kMgCoarseThreads) k_mg_coarsest(MgLevel<R> L, int iters) {
  for (int it = 0; it < iters; ++it)
    for (int parity = 1; parity >= 0; --parity) {
      for (int idx = threadIdx.x; idx < L.n; idx += blockDim.x) {
        if (!L.m[idx]) continue;
        int i, j, k;
        mg_ijk(idx, L.ni, L.nj, i, j, k);
        if (((i + j + k) & 1) != parity) continue;
        const R s = mg_offdiag(L, L.x, idx, i, j, k);
        const R d = L.d[idx];
        L.x[idx] = d != R(0) ? (L.b[idx] - s) / d : R(0);
      }
      __syncthreads();
    }
}

// b_c = R (b_f - A_f x_f) = 0.125 * (sum of the fine residuals of the DOF
// children); x_c = 0.
template <typename R>
__global__ void __launch_bounds__(kMgThreads) k_mg_restrict(MgLevel<R> f, MgLevel<R> c) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < c.n; idx += gridDim.x * blockDim.x) {
    int I, J, K;
    mg_ijk(idx, c.ni, c.nj, I, J, K);
    R acc = 0;
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
          if (i >= f.ni || j >= f.nj || k >= f.nk) continue;
          const int e = i + f.ni * (j + f.nj * k);
          if (!f.m[e]) continue;
          const R r = f.b[e] - (f.d[e] * f.x[e] + mg_offdiag(f, f.x, e, i, j, k));
          acc += R(0.125) * r;
        }
    c.b[idx] = acc;
    c.x[idx] = R(0);
  }
}

// x_f += P x_c
template <typename R>
__global__ void __launch_bounds__(kMgThreads) k_mg_prolong(MgLevel<R> c, MgLevel<R> f) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < f.n; idx += gridDim.x * blockDim.x) {
    if (!f.m[idx]) continue;
    int i, j, k;
    mg_ijk(idx, f.ni, f.nj, i, j, k);
    f.x[idx] += c.x[(i >> 1) + c.ni * ((j >> 1) + c.nj * (k >> 1))];
  }
}

// ---- PCG on level 0 (AMGPCGSolveSparse's loop) ----------------------------
// q = A s, partial[block] = s.q
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_spmv(MgLevel<R> L, const R* __restrict__ s, R* __restrict__ q,
              const double* __restrict__ sc, double* __restrict__ partial) {
  __shared__ double sm[kMgThreads];
  double acc = 0;
  if (!*(const int*)(sc + S_DONE)) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < L.n; idx += gridDim.x * blockDim.x) {
      R v = R(0);
      if (L.m[idx]) {
        int i, j, k;
        mg_ijk(idx, L.ni, L.nj, i, j, k);
        v = L.d[idx] * s[idx] + mg_offdiag(L, s, idx, i, j, k);
      }
      q[idx] = v;
      acc += (double)s[idx] * (double)v;
    }
  }
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// x += alpha s, r -= alpha q, partial[block] = max |r|
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_update(int n, const R* __restrict__ s, const R* __restrict__ q, R* __restrict__ x,
                R* __restrict__ r, const double* __restrict__ sc, double* __restrict__ partial) {
  __shared__ double sm[kMgThreads];
  double m = 0;
  if (!*(const int*)(sc + S_DONE)) {
    const R al = (R)sc[S_ALPHA];
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
      x[idx] = x[idx] + al * s[idx];
      const R rv = r[idx] - al * q[idx];
      r[idx] = rv;
      const double av = fabs((double)rv);
      m = av > m ? av : m;
    }
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// partial[block] = z.r
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_dot(int n, const R* __restrict__ a, const R* __restrict__ b,
             double* __restrict__ partial) {
  __shared__ double sm[kMgThreads];
  double acc = 0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x)
    acc += (double)a[idx] * (double)b[idx];
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// s = z + beta s
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_direction(int n, const R* __restrict__ z, R* __restrict__ s,
                   const double* __restrict__ sc) {
  const R be = (R)sc[S_BETA];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x)
    s[idx] = z[idx] + be * s[idx];
}

// FP64 residual r64 = b - A x64 (coefficients promoted); partial max |r64|
template <typename R>
__global__ void __launch_bounds__(kMgThreads)
    k_mg_residual64(MgLevel<R> L, const R* __restrict__ b, const double* __restrict__ x,
                    double* __restrict__ r, double* __restrict__ partial) {
  __shared__ double sm[kMgThreads];
  double m = 0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < L.n; idx += gridDim.x * blockDim.x) {
    double rv = 0;
    if (L.m[idx]) {
      int i, j, k;
      mg_ijk(idx, L.ni, L.nj, i, j, k);
      const int sj = L.ni, sk = L.ni * L.nj;
      double s = (double)L.d[idx] * x[idx];
      if (k > 0) s += (double)L.az[idx - sk] * x[idx - sk];
      if (j > 0) s += (double)L.ay[idx - sj] * x[idx - sj];
      if (i > 0) s += (double)L.ax[idx - 1] * x[idx - 1];
      if (i + 1 < L.ni) s += (double)L.ax[idx] * x[idx + 1];
      if (j + 1 < L.nj) s += (double)L.ay[idx] * x[idx + sj];
      if (k + 1 < L.nk) s += (double)L.az[idx] * x[idx + sk];
      rv = (double)b[idx] - s;
    }
    r[idx] = rv;
    const double av = fabs(rv);
    m = av > m ? av : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// pressure of every active node from the level-0 solution (0 off the DOFs)
template <typename R>
__global__ void k_mg_scatter_pressure(GridDesc g, const int* __restrict__ active_list,
                                      long long nent, const unsigned char* __restrict__ dof,
                                      const R* __restrict__ x32, const double* __restrict__ x64,
                                      R* __restrict__ p) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    R v = R(0);
    if (dof[n] & 1) {
      int I, J, K;
      node_ijk(g, n, I, J, K);
      const int idx = I + g.NI * (J + g.NJ * K);
      v = x64 ? (R)x64[idx] : x32[idx];
    }
    p[n] = v;
  }
}

}  // namespace wcg
