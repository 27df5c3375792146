// MIC(0)-preconditioned conjugate gradient on the matrix-free 7-point
// pressure operator.
//
// Factorisation and triangular solves restate robertbridson's
// factor_modified_incomplete_cholesky0 / solve_lower /
// solve_lower_transpose_in_place (libWetCloth/Core/PCGSolver/PCGSolver.h:
// 97-239) for the structure the pressure assembly produces: with the
// reference's bucket-major DOF numbering every -x/-y/-z neighbour precedes a
// cell and every +x/+y/+z neighbour follows it, and no fill-in position of
// MIC(0) on a 7-point stencil is itself a stencil entry, so for DOF j
//   d_j = A_jj - sum_{k in {j-z,j-y,j-x}} [ L_jk^2 + omega L_jk sum_{i in
//         upper(k), i != j} L_ik ],   L_ik = A_ik / sqrt(d_k'),
//   d_k' = d_k unless d_k < min_ratio A_kk (then A_kk); 1/sqrt(d_k') stored,
// and S_a[k] = A(k, k+e_a) / sqrt(d_k') (the reference's scaled column entry
// factor.value) is kept per cell for both triangular solves.
//
// The dependency graph is the i+j+k hyperplane order.  The GPU walks it in
// tiles of 8x8x8 cells (2x2x2 buckets): tiles are handed out by an atomic
// ticket in wave order (ti+tj+tk); a tile stages all its own static data in
// shared memory first, then spins (bounded) on the completion flags of its
// three upstream tiles, fetches their face values, and sweeps its 22 intra-tile
// hyperplanes with one thread per x-pencil entirely in shared memory.  The
// forward sweep also applies the PCG update x += alpha s, r -= alpha q and the
// residual norm; the backward sweep also forms z.r.  Iterations are
// launched in batches with convergence tested on the device.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"

namespace wcg {

constexpr long long kSpinLimit = 1ll << 20;  // bounded spin (well under a second)
constexpr int kTile = 8;                      // cells per tile edge
constexpr int kTileCells = kTile * kTile * kTile;
constexpr int kSweepThreads = kTile * kTile;  // one thread per x-pencil

// device scalar slots of the PCG state (dscalars)
enum PcgSlot : int {
  S_RHO = 20, S_SQ = 21, S_ALPHA = 22, S_RES = 23, S_BETA = 24, S_TOL = 25,
  S_ITER = 26, S_MAXIT = 27, S_DONE = 28  // S_DONE holds an int
};

__device__ inline int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ inline void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// wait for an upstream tile (bounded); returns false on timeout
__device__ inline bool wait_tile(const int* flag, int epoch, int* err) {
  long long it = 0;
  while (ld_acquire_gpu(flag) < epoch) {
    if (++it > kSpinLimit) {
      record_error(err, kErrWaitTimeout);
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

template <typename T>
__device__ inline T block_sum(T v, T* sm) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  const T r = sm[0];
  __syncthreads();
  return r;
}

template <typename T>
__device__ inline T block_max(T v, T* sm) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      sm[threadIdx.x] = sm[threadIdx.x] > sm[threadIdx.x + o] ? sm[threadIdx.x] : sm[threadIdx.x + o];
    __syncthreads();
  }
  const T r = sm[0];
  __syncthreads();
  return r;
}

enum WaveMode : int { kFactor = 0, kForward = 1, kBackward = 2 };

template <typename R>
struct SweepArgs {
  GridDesc g;
  int nti, ntj, ntk;
  const int* tile_list;
  int ntiles;
  int* ticket;
  int* flags;
  int epoch;
  const unsigned char* active;
  const unsigned char* tile_active;  // tiles that publish a completion flag
  const unsigned char* dof;
  R* F;
  long long fs;
  const R* in;     // forward: r; backward: y
  R* out;          // forward: y; backward: z
  R* r;            // forward with update: r (updated in place); backward: r for z.r
  R* x;            // forward with update
  const R* s;
  const R* q;
  double* sc;      // device scalars
  int update;      // forward: apply the PCG x/r update first
  double* part;    // per-tile partial (indexed by tile id): forward max|r|, backward z.r
  R omega, min_ratio;
  int* err;
};

// global node of tile-local cell (i,j,k) of tile (ti,tj,tk), -1 if absent
__device__ inline long long tile_node(const GridDesc& g, int ti, int tj, int tk,
                                      int i, int j, int k, const unsigned char* active) {
  const int I = ti * kTile + i, J = tj * kTile + j, K = tk * kTile + k;
  if (!in_grid(g, I, J, K)) return -1;
  const long long b = bucket_of(g, I, J, K);
  if (!active[b]) return -1;
  return b * 64 + (((K & 3) << 4) | ((J & 3) << 2) | (I & 3));
}

template <typename R, int MODE>
__global__ void __launch_bounds__(kSweepThreads)
    k_sweep(const SweepArgs<R> a) {
  __shared__ int s_tile;
  __shared__ R val[kTileCells];   // wavefront value (y, z or invdiag)
  __shared__ R rin[kTileCells];   // rhs of the sweep (r, y) or A_diag
  __shared__ R inv[kTileCells];   // invdiag (sweeps) ; unused (factor)
  __shared__ R sx[kTileCells], sy[kTileCells], sz[kTileCells];  // S (sweeps) or A (factor)
  __shared__ unsigned char dm[kTileCells];
  __shared__ R hv[3][kTile * kTile];   // neighbour face values
  __shared__ R ha[3][3][kTile * kTile];  // neighbour face couplings (factor: all 3 axes)
  __shared__ double red[kSweepThreads];
  const GridDesc& g = a.g;
  if (*(const int*)(a.sc + S_DONE)) return;
  const int tid = threadIdx.x;
  if (tid == 0) s_tile = atomicAdd(a.ticket, 1);
  __syncthreads();
  const int t = s_tile;
  if (t >= a.ntiles) return;
  const int tl = MODE == kBackward ? a.tile_list[a.ntiles - 1 - t] : a.tile_list[t];
  const int tk = tl / (a.nti * a.ntj);
  const int trem = tl - tk * a.nti * a.ntj;
  const int tj = trem / a.nti;
  const int ti = trem - tj * a.nti;
  const R* F = a.F;
  const long long fs = a.fs;

  // ---- stage own cells (bucket-major coalesced loads) ----
  double rmax = 0;
  const double alpha = (MODE == kForward && a.update) ? a.sc[S_ALPHA] : 0.0;
  for (int m = 0; m < 8; ++m) {
    const int bx = m & 1, by = (m >> 1) & 1, bz = m >> 2;
    const int li = tid & 3, lj = (tid >> 2) & 3, lk = tid >> 4;
    const int i = bx * 4 + li, j = by * 4 + lj, k = bz * 4 + lk;
    const int c = (k * kTile + j) * kTile + i;
    const long long n = tile_node(g, ti, tj, tk, i, j, k, a.active);
    const bool d = n >= 0 && a.dof[n];
    dm[c] = d ? 1 : 0;
    val[c] = R(0);
    if (!d) {
      rin[c] = R(0);
      inv[c] = R(0);
      sx[c] = sy[c] = sz[c] = R(0);
      continue;
    }
    if (MODE == kFactor) {
      rin[c] = F[G_ADIAG * fs + n];
      sx[c] = F[G_AX * fs + n];
      sy[c] = F[G_AY * fs + n];
      sz[c] = F[G_AZ * fs + n];
      inv[c] = R(0);
    } else {
      inv[c] = F[G_INVDIAG * fs + n];
      sx[c] = F[G_SX * fs + n];
      sy[c] = F[G_SY * fs + n];
      sz[c] = F[G_SZ * fs + n];
      if (MODE == kForward) {
        R rv = a.in[n];
        if (a.update) {
          const R al = (R)alpha;
          a.x[n] = a.x[n] + al * a.s[n];
          rv = rv - al * a.q[n];
          a.r[n] = rv;
          const double av = fabs((double)rv);
          rmax = av > rmax ? av : rmax;
        }
        rin[c] = rv;
      } else {
        rin[c] = a.in[n];
      }
    }
  }
  // ---- stage static data of the neighbour faces ----
  // face f: 0 -> x, 1 -> y, 2 -> z; slot p = (u, v) in the face
  const int fu = tid & 7, fv = tid >> 3;
  const int side = MODE == kBackward ? kTile : -1;
  long long hn[3];
  for (int f = 0; f < 3; ++f) {
    int i, j, k;
    if (f == 0) { i = side; j = fu; k = fv; }
    else if (f == 1) { i = fu; j = side; k = fv; }
    else { i = fu; j = fv; k = side; }
    long long n = tile_node(g, ti, tj, tk, i, j, k, a.active);
    if (n >= 0 && !a.dof[n]) n = -1;
    hn[f] = n;
    hv[f][tid] = R(0);
    if (MODE == kFactor) {
      ha[f][0][tid] = n >= 0 ? F[G_AX * fs + n] : R(0);
      ha[f][1][tid] = n >= 0 ? F[G_AY * fs + n] : R(0);
      ha[f][2][tid] = n >= 0 ? F[G_AZ * fs + n] : R(0);
    } else if (MODE == kForward) {
      const int gf = f == 0 ? G_SX : (f == 1 ? G_SY : G_SZ);
      ha[f][0][tid] = n >= 0 ? F[gf * fs + n] : R(0);
    }
  }
  // ---- wait for the upstream tiles ----
  if (tid < 3) {
    const int st = MODE == kBackward ? 1 : -1;
    const int x = ti + (tid == 0 ? st : 0), y = tj + (tid == 1 ? st : 0),
              z = tk + (tid == 2 ? st : 0);
    if (x >= 0 && y >= 0 && z >= 0 && x < a.nti && y < a.ntj && z < a.ntk) {
      const long long ut = ((long long)z * a.ntj + y) * a.nti + x;
      // only tiles holding an active bucket are launched and publish a flag
      if (a.tile_active[ut]) wait_tile(a.flags + ut, a.epoch, a.err);
    }
  }
  __syncthreads();
  // ---- neighbour face values ----
  for (int f = 0; f < 3; ++f) {
    const long long n = hn[f];
    if (n < 0) continue;
    if (MODE == kFactor) hv[f][tid] = __ldcg(F + G_INVDIAG * fs + n);
    else hv[f][tid] = __ldcg(a.out + n);
  }
  __syncthreads();
  // ---- intra-tile wavefront: thread = x-pencil (pj, pk) ----
  const int pj = tid & 7, pk = tid >> 3;
  for (int s = 0; s < 3 * kTile - 2; ++s) {
    const int i = MODE == kBackward ? (kTile - 1) - (s - ((kTile - 1 - pj) + (kTile - 1 - pk)))
                                    : s - pj - pk;
    const bool live = MODE == kBackward ? (s - ((kTile - 1 - pj) + (kTile - 1 - pk))) >= 0 &&
                                              (s - ((kTile - 1 - pj) + (kTile - 1 - pk))) < kTile
                                        : (i >= 0 && i < kTile);
    if (live) {
      const int c = (pk * kTile + pj) * kTile + i;
      if (dm[c]) {
        if (MODE == kFactor) {
          const R adiag = rin[c];
          R d = adiag;
          R iv = R(0);
          if (adiag != R(0)) {
            // lower neighbours in the reference's interior column order -z, -y, -x
            for (int ax = 2; ax >= 0; --ax) {
              R ik, cx, cy, cz;
              if (ax == 0) {
                if (i > 0) { ik = val[c - 1]; cx = sx[c - 1]; cy = sy[c - 1]; cz = sz[c - 1]; }
                else { const int p = pk * 8 + pj; ik = hv[0][p]; cx = ha[0][0][p]; cy = ha[0][1][p]; cz = ha[0][2][p]; }
              } else if (ax == 1) {
                if (pj > 0) { ik = val[c - 8]; cx = sx[c - 8]; cy = sy[c - 8]; cz = sz[c - 8]; }
                else { const int p = pk * 8 + i; ik = hv[1][p]; cx = ha[1][0][p]; cy = ha[1][1][p]; cz = ha[1][2][p]; }
              } else {
                if (pk > 0) { ik = val[c - 64]; cx = sx[c - 64]; cy = sy[c - 64]; cz = sz[c - 64]; }
                else { const int p = pj * 8 + i; ik = hv[2][p]; cx = ha[2][0][p]; cy = ha[2][1][p]; cz = ha[2][2][p]; }
              }
              if (ik == R(0)) continue;  // absent or null column
              const R L = (ax == 0 ? cx : (ax == 1 ? cy : cz)) * ik;
              const R miss = ax == 0 ? (cy * ik + cz * ik)
                                     : (ax == 1 ? (cx * ik + cz * ik) : (cx * ik + cy * ik));
              d = d - L * L;
              d = d - (a.omega * L) * miss;
            }
            const R piv = d < a.min_ratio * adiag ? adiag : d;
            iv = R(1) / sqrt(piv);
          }
          val[c] = iv;
        } else if (MODE == kForward) {
          R v = rin[c];
          const R zm = pk > 0 ? val[c - 64] : hv[2][pj * 8 + i];
          const R Lz = pk > 0 ? sz[c - 64] : ha[2][0][pj * 8 + i];
          const R ym = pj > 0 ? val[c - 8] : hv[1][pk * 8 + i];
          const R Ly = pj > 0 ? sy[c - 8] : ha[1][0][pk * 8 + i];
          const R xm = i > 0 ? val[c - 1] : hv[0][pk * 8 + pj];
          const R Lx = i > 0 ? sx[c - 1] : ha[0][0][pk * 8 + pj];
          v -= Lz * zm;
          v -= Ly * ym;
          v -= Lx * xm;
          val[c] = v * inv[c];
        } else {
          R v = rin[c];
          const R xp = i < kTile - 1 ? val[c + 1] : hv[0][pk * 8 + pj];
          const R yp = pj < kTile - 1 ? val[c + 8] : hv[1][pk * 8 + i];
          const R zp = pk < kTile - 1 ? val[c + 64] : hv[2][pj * 8 + i];
          v -= sx[c] * xp;
          v -= sy[c] * yp;
          v -= sz[c] * zp;
          val[c] = v * inv[c];
        }
      }
    }
    __syncthreads();
  }
  // ---- write back (coalesced), partials ----
  double dsum = 0;
  for (int m = 0; m < 8; ++m) {
    const int bx = m & 1, by = (m >> 1) & 1, bz = m >> 2;
    const int li = tid & 3, lj = (tid >> 2) & 3, lk = tid >> 4;
    const int i = bx * 4 + li, j = by * 4 + lj, k = bz * 4 + lk;
    const int c = (k * kTile + j) * kTile + i;
    if (!dm[c]) continue;
    const long long n = tile_node(g, ti, tj, tk, i, j, k, a.active);
    if (MODE == kFactor) {
      const R iv = val[c];
      a.F[G_INVDIAG * fs + n] = iv;
      a.F[G_SX * fs + n] = sx[c] * iv;
      a.F[G_SY * fs + n] = sy[c] * iv;
      a.F[G_SZ * fs + n] = sz[c] * iv;
    } else {
      a.out[n] = val[c];
      if (MODE == kBackward && a.part) dsum += (double)val[c] * (double)a.r[n];
    }
  }
  if (MODE == kForward && a.update && a.part) {
    const double m = block_max<double>(rmax, red);
    if (tid == 0) a.part[tl] = m;
  }
  if (MODE == kBackward && a.part) {
    const double sm = block_sum<double>(dsum, red);
    if (tid == 0) a.part[tl] = sm;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release_gpu(a.flags + tl, a.epoch);
}

// ---- vector kernels over the active buckets ---------------------------------
// Each active bucket is 64 consecutive nodes; e indexes (active bucket, node).
__device__ inline long long active_node(const int* active_list, long long e) {
  return (long long)active_list[e >> 6] * 64 + (e & 63);
}

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

// partial[blockIdx] = sum a*b over DOFs (FP64 accumulation)
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_dot_partial(const int* __restrict__ active_list, long long nent,
                  const unsigned char* __restrict__ dof, const R* __restrict__ a,
                  const R* __restrict__ b, double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    if (dof[n]) s += (double)a[n] * (double)b[n];
  }
  s = block_sum<double>(s, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// out = sum of partials (fixed order)
__global__ void k_reduce_sum(const double* __restrict__ partial, int n,
                             double* __restrict__ out) {
  __shared__ double sm[kRedThreads];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  s = block_sum<double>(s, sm);
  if (threadIdx.x == 0) *out = s;
}

template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_absmax_partial(const int* __restrict__ active_list, long long nent,
                     const unsigned char* __restrict__ dof,
                     const R* __restrict__ a, double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double m = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    if (dof[n]) {
      const double v = fabs((double)a[n]);
      m = v > m ? v : m;
    }
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// partial[block] = number of DOFs (as double, exact below 2^53)
__global__ void __launch_bounds__(kRedThreads)
    k_count_dof(const int* __restrict__ active_list, long long nent,
                const unsigned char* __restrict__ dof, double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x)
    if (dof[active_node(active_list, e)]) s += 1.0;
  s = block_sum<double>(s, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_reduce_max(const double* __restrict__ partial, int n,
                             double* __restrict__ out) {
  __shared__ double sm[kRedThreads];
  double m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = partial[i] > m ? partial[i] : m;
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) *out = m;
}

// s_new = z + beta s_old (recomputed at all 7 stencil points), q = A s_new,
// partial[block] = sum s_new.q.  PCG direction update fused into the SpMV.
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_spmv_s(GridDesc g, const int* __restrict__ active_list, long long nent,
             const unsigned char* __restrict__ active,
             const unsigned char* __restrict__ dof, const R* __restrict__ F,
             long long fstride, const R* __restrict__ z, const R* __restrict__ sold,
             R* __restrict__ snew, R* __restrict__ q, const double* __restrict__ sc,
             double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  const R be = (R)sc[S_BETA];
  double acc = 0;
  const R* AD = F + G_ADIAG * fstride;
  const R* AX = F + G_AX * fstride;
  const R* AY = F + G_AY * fstride;
  const R* AZ = F + G_AZ * fstride;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    if (!dof[n]) continue;
    int I, J, K;
    node_ijk(g, n, I, J, K);
    R r = 0;
    // row order of the reference's sorted row for interior cells
    if (K > 0) {
      const long long m = node_linear(g, I, J, K - 1);
      if (active[m >> 6] && dof[m]) r += AZ[m] * (z[m] + be * sold[m]);
    }
    if (J > 0) {
      const long long m = node_linear(g, I, J - 1, K);
      if (active[m >> 6] && dof[m]) r += AY[m] * (z[m] + be * sold[m]);
    }
    if (I > 0) {
      const long long m = node_linear(g, I - 1, J, K);
      if (active[m >> 6] && dof[m]) r += AX[m] * (z[m] + be * sold[m]);
    }
    const R sn = z[n] + be * sold[n];
    r += AD[n] * sn;
    if (I + 1 < g.NI) {
      const long long m = node_linear(g, I + 1, J, K);
      if (active[m >> 6] && dof[m]) r += AX[n] * (z[m] + be * sold[m]);
    }
    if (J + 1 < g.NJ) {
      const long long m = node_linear(g, I, J + 1, K);
      if (active[m >> 6] && dof[m]) r += AY[n] * (z[m] + be * sold[m]);
    }
    if (K + 1 < g.NK) {
      const long long m = node_linear(g, I, J, K + 1);
      if (active[m >> 6] && dof[m]) r += AZ[n] * (z[m] + be * sold[m]);
    }
    snew[n] = sn;
    q[n] = r;
    acc += (double)sn * (double)r;
  }
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// alpha = rho / sum(partials)
// The three per-iteration reductions, as block bodies: a kernel of their own
// (k_red_*) or the last block of the kernel that wrote the partials
// (last_block).  Partials are summed thread-strided, then by the block tree,
// so both forms give the same bits.
__device__ inline void red_alpha_body(const double* partial, int n, double* sc, double* sm) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += __ldcg(partial + i);
  s = block_sum<double>(s, sm);
  if (threadIdx.x == 0) {
    sc[S_SQ] = s;
    sc[S_ALPHA] = sc[S_RHO] / s;
  }
}

__device__ inline void red_conv_body(const double* partial, int n, double* sc, double* sm) {
  double m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = __ldcg(partial + i);
    m = v > m ? v : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) {
    sc[S_RES] = m;
    sc[S_ITER] += 1.0;
    if (m <= sc[S_TOL]) *(int*)(sc + S_DONE) = 1;
    else if (sc[S_ITER] >= sc[S_MAXIT]) *(int*)(sc + S_DONE) = 2;
  }
}

__device__ inline void red_beta_body(const double* partial, int n, double* sc, double* sm,
                                     int init) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += __ldcg(partial + i);
  s = block_sum<double>(s, sm);
  if (threadIdx.x == 0) {
    if (init) {
      sc[S_BETA] = 0.0;
    } else {
      sc[S_BETA] = s / sc[S_RHO];
    }
    sc[S_RHO] = s;
  }
}

// True in the block that reaches the counter last (every block calls it
// once, after writing its partial); that block resets the counter for the
// next launch.  The fences order the partials before the count and the
// count before the last block's reads.
__device__ inline bool last_block(int* ctr, int nblocks) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int k = atomicAdd(ctr, 1);
    s_last = k == nblocks - 1 ? 1 : 0;
    if (s_last) {
      atomicExch(ctr, 0);
      __threadfence();
    }
  }
  __syncthreads();
  return s_last != 0;
}

__global__ void k_red_alpha(const double* __restrict__ partial, int n, double* sc) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  red_alpha_body(partial, n, sc, sm);
}

// res = max(partials); stop (done = 1) when res <= tol, or (done = 2) when
// the iteration budget is spent (PCGSolver::solve, PCGSolver.h:282-307)
__global__ void k_red_conv(const double* __restrict__ partial, int n, double* sc) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  red_conv_body(partial, n, sc, sm);
}

// rho_new = sum(partials); beta = rho_new / rho; rho = rho_new.  With init,
// only rho is set (the first direction is s = z).
__global__ void k_red_beta(const double* __restrict__ partial, int n, double* sc, int init) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  red_beta_body(partial, n, sc, sm, init);
}

template <typename R>
__global__ void k_copy_dof(const int* __restrict__ active_list, long long nent,
                           const unsigned char* __restrict__ dof,
                           const R* __restrict__ a, R* __restrict__ b) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    b[n] = dof[n] ? a[n] : R(0);
  }
}

// tiles of 2x2x2 buckets containing an active bucket
__global__ void k_tile_active(GridDesc g, int nti, int ntj, int ntk,
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
  for (int m = 0; m < 8; ++m) {
    const int bi = ti * 2 + (m & 1), bj = tj * 2 + ((m >> 1) & 1), bk = tk * 2 + (m >> 2);
    if (bi < g.ni && bj < g.nj && bk < g.nk &&
        active[((long long)bk * g.nj + bj) * g.ni + bi])
      any = 1;
  }
  tact[t] = any;
}

__global__ void k_tile_wave_count(int nti, int ntj, const int* __restrict__ list,
                                  long long n, int* __restrict__ count) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int t = list[e];
  const int tk = t / (nti * ntj);
  const int rem = t - tk * nti * ntj;
  const int tj = rem / nti;
  const int ti = rem - tj * nti;
  atomicAdd(&count[ti + tj + tk], 1);
}

__global__ void k_tile_wave_scatter(int nti, int ntj, const int* __restrict__ list,
                                    long long n, int* __restrict__ cursor,
                                    int* __restrict__ out) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int t = list[e];
  const int tk = t / (nti * ntj);
  const int rem = t - tk * nti * ntj;
  const int tj = rem / nti;
  const int ti = rem - tj * nti;
  out[atomicAdd(&cursor[ti + tj + tk], 1)] = t;
}

}  // namespace wcg
