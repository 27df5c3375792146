// MIC(0)-preconditioned CG on a general sparse symmetric matrix given in CSR
// form: the call shape of robertbridson::PCGSolver<double>::solve
// (libWetCloth/Core/PCGSolver/PCGSolver.h:260-308), which the reference calls
// on assembled SparseMatrix objects (the implicit viscosity solve,
// Core/Viscosity.cpp:112-116; the pressure system re-solved with MIC(0)).
//
// Everything numeric runs on the GPU:
//   * structure: the factor's columns are the upper parts of the matrix rows
//     (factor_modified_incomplete_cholesky0 copies them, PCGSolver.h:106-117),
//     their transpose lists for each column the earlier columns that update
//     it, and two level schedules (forward: a row after every earlier column
//     that updates it; backward: a row after every later row in its column)
//     come from iterated frontier kernels;
//   * the factorisation, one launch per forward level: each column gathers
//     the eliminations of its earlier columns in ascending column order, with
//     the reference's dropped-entry rule ("missing", modification 0.97) and
//     its pivot test (ratio 0.25), so every entry sees the reference's
//     sequence of subtractions (PCGSolver.h:142-204);
//   * the triangular solves, one launch per level, each row gathering its
//     terms in the order solve_lower / solve_lower_transpose_in_place apply
//     them (:211-239);
//   * the PCG iteration of PCGSolver::solve with its infinity-norm stop.
// Products and sums are rounded separately (_rn intrinsics), as the
// reference's compiled code evaluates them.  Dot products are deterministic
// block reductions; their summation order is not Eigen's, so the iterates
// agree with the reference's to rounding, not bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/wetcloth_gpu.h"
#include "wcg_context.h"
#include "wcg_scan.cuh"

namespace wcg {
namespace {

constexpr double kOmega = 0.97;     // modification parameter (PCGSolver.h:100)
constexpr double kMinRatio = 0.25;  // min_diagonal_ratio (:101)
constexpr int kThreads = 256;
constexpr int kDotBlocks = 296;     // 2 per SM of a B200

inline unsigned nblocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

struct Mem {
  void* p = nullptr;
  ~Mem() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
  template <typename T>
  T* as() const { return (T*)p; }
};

#define CSR_TRY(x)                       \
  do {                                   \
    cudaError_t e_ = (x);                \
    if (e_ != cudaSuccess) return e_;    \
  } while (0)

// rows must list strictly ascending columns in [0, n); counts the upper
// entries of each row (the factor's column) and takes the diagonal
__global__ void k_csr_rows(int n, const int* __restrict__ rowstart, const int* __restrict__ col,
                           const double* __restrict__ val, int* __restrict__ ucount,
                           double* __restrict__ adiag, int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = rowstart[i], e = rowstart[i + 1];
  if (e < s) {
    atomicExch(bad, 1);
    ucount[i] = 0;
    adiag[i] = 0.0;
    return;
  }
  int prev = -1, cnt = 0;
  double d = 0.0;
  for (int p = s; p < e; ++p) {
    const int c = col[p];
    if (c < 0 || c >= n || c <= prev) atomicExch(bad, 1);
    prev = c;
    if (c > i) ++cnt;
    else if (c == i) d = val[p];
  }
  ucount[i] = cnt;
  adiag[i] = d;
}

// factor column k = the entries of row k right of the diagonal, in row order
__global__ void k_csr_upper(int n, const int* __restrict__ rowstart, const int* __restrict__ col,
                            const double* __restrict__ val, const int* __restrict__ ustart,
                            int* __restrict__ urow, double* __restrict__ uval,
                            int* __restrict__ tcount) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int q = ustart[k];
  for (int p = rowstart[k]; p < rowstart[k + 1]; ++p) {
    const int c = col[p];
    if (c <= k) continue;
    urow[q] = c;
    uval[q] = val[p];
    ++q;
    atomicAdd(&tcount[c], 1);
  }
}

// for each column j: the earlier columns k holding row j, with the position
// of that entry
__global__ void k_csr_transpose(int n, const int* __restrict__ ustart,
                                const int* __restrict__ urow, const int* __restrict__ tstart,
                                int* __restrict__ tcur, int* __restrict__ tk,
                                int* __restrict__ tp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  for (int p = ustart[k]; p < ustart[k + 1]; ++p) {
    const int j = urow[p];
    const int q = tstart[j] + atomicAdd(&tcur[j], 1);
    tk[q] = k;
    tp[q] = p;
  }
}

// ascending column order inside each transpose list (insertion sort)
__global__ void k_csr_sort_transpose(int n, const int* __restrict__ tstart, int* __restrict__ tk,
                                     int* __restrict__ tp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int s = tstart[j], e = tstart[j + 1];
  for (int a = s + 1; a < e; ++a) {
    const int k = tk[a], p = tp[a];
    int b = a - 1;
    while (b >= s && tk[b] > k) {
      tk[b + 1] = tk[b];
      tp[b + 1] = tp[b];
      --b;
    }
    tk[b + 1] = k;
    tp[b + 1] = p;
  }
}

// frontier t of the forward schedule: rows whose updating columns all sit on
// earlier levels
__global__ void k_csr_level_fwd(int n, const int* __restrict__ tstart, const int* __restrict__ tk,
                                int* lev, int t, int* assigned) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || lev[i] >= 0) return;
  for (int q = tstart[i]; q < tstart[i + 1]; ++q) {
    const int l = ((volatile int*)lev)[tk[q]];
    if (l < 0 || l >= t) return;
  }
  lev[i] = t;
  atomicAdd(assigned, 1);
}

// frontier t of the backward schedule: rows whose column entries (later
// rows) all sit on earlier levels
__global__ void k_csr_level_bwd(int n, const int* __restrict__ ustart, const int* __restrict__ urow,
                                int* lev, int t, int* assigned) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || lev[i] >= 0) return;
  for (int p = ustart[i]; p < ustart[i + 1]; ++p) {
    const int l = ((volatile int*)lev)[urow[p]];
    if (l < 0 || l >= t) return;
  }
  lev[i] = t;
  atomicAdd(assigned, 1);
}

__global__ void k_csr_level_count(int n, const int* __restrict__ lev, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&cnt[lev[i]], 1);
}

__global__ void k_csr_level_scatter(int n, const int* __restrict__ lev,
                                    const int* __restrict__ start, int* __restrict__ cur,
                                    int* __restrict__ rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rows[start[lev[i]] + atomicAdd(&cur[lev[i]], 1)] = i;
}

// factor_modified_incomplete_cholesky0 (PCGSolver.h:142-204) for the columns
// of one level: column j applies the eliminations of the earlier columns k
// that hold row j in ascending k (the order in which the reference's column
// loop reaches j), then takes its pivot and scales itself.
__global__ void k_csr_factor_level(const int* __restrict__ rows, int cnt,
                                   const int* __restrict__ rowstart, const int* __restrict__ col,
                                   const int* __restrict__ ustart, const int* __restrict__ urow,
                                   double* __restrict__ uval, const int* __restrict__ tstart,
                                   const int* __restrict__ tk, const int* __restrict__ tp,
                                   const double* __restrict__ adiag, double* __restrict__ invdiag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int j = rows[t];
  double d = adiag[j];
  const int ej = ustart[j + 1];
  for (int q = tstart[j]; q < tstart[j + 1]; ++q) {
    const int k = tk[q];
    if (adiag[k] == 0.0) continue;  // null row/column: skipped (:144)
    const double mult = uval[tp[q]];
    double missing = 0.0;
    int a = ustart[k];
    const int ek = ustart[k + 1];
    // dropped entries above the diagonal of column j: rows of column k below
    // j that row j of the matrix does not hold
    int b = rowstart[j];
    const int eb = rowstart[j + 1];
    while (a < ek && urow[a] < j) {
      while (b < eb) {
        const int c = col[b];
        if (c < urow[a]) {
          ++b;
        } else if (c == urow[a]) {
          break;
        } else {
          missing = __dadd_rn(missing, uval[a]);
          break;
        }
      }
      ++a;
    }
    if (a < ek && urow[a] == j) d = __dsub_rn(d, __dmul_rn(mult, uval[a]));
    ++a;
    // entries below the diagonal of column j, or dropped into missing
    int bb = ustart[j];
    while (a < ek && bb < ej) {
      if (urow[bb] < urow[a]) {
        ++bb;
      } else if (urow[bb] == urow[a]) {
        uval[bb] = __dsub_rn(uval[bb], __dmul_rn(mult, uval[a]));
        ++a;
        ++bb;
      } else {
        missing = __dadd_rn(missing, uval[a]);
        ++a;
      }
    }
    while (a < ek) {
      missing = __dadd_rn(missing, uval[a]);
      ++a;
    }
    d = __dsub_rn(d, __dmul_rn(__dmul_rn(kOmega, mult), missing));
  }
  if (adiag[j] == 0.0) {
    invdiag[j] = d;
    return;
  }
  const double piv = d < __dmul_rn(kMinRatio, adiag[j]) ? adiag[j] : d;
  const double inv = __ddiv_rn(1.0, __dsqrt_rn(piv));
  for (int p = ustart[j]; p < ej; ++p) uval[p] = __dmul_rn(uval[p], inv);
  invdiag[j] = inv;
}

// solve_lower (PCGSolver.h:211-222) for the rows of one forward level
__global__ void k_csr_lower_level(const int* __restrict__ rows, int cnt,
                                  const int* __restrict__ tstart, const int* __restrict__ tk,
                                  const int* __restrict__ tp, const double* __restrict__ uval,
                                  const double* __restrict__ invdiag,
                                  const double* __restrict__ rhs, double* __restrict__ y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int r = rows[t];
  double acc = rhs[r];
  for (int q = tstart[r]; q < tstart[r + 1]; ++q)
    acc = __dsub_rn(acc, __dmul_rn(uval[tp[q]], y[tk[q]]));
  y[r] = __dmul_rn(acc, invdiag[r]);
}

// solve_lower_transpose_in_place (:226-239) for the rows of one backward level
__global__ void k_csr_upper_level(const int* __restrict__ rows, int cnt,
                                  const int* __restrict__ ustart, const int* __restrict__ urow,
                                  const double* __restrict__ uval,
                                  const double* __restrict__ invdiag, double* __restrict__ x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int i = rows[t];
  double acc = x[i];
  for (int p = ustart[i]; p < ustart[i + 1]; ++p)
    acc = __dsub_rn(acc, __dmul_rn(uval[p], x[urow[p]]));
  x[i] = __dmul_rn(acc, invdiag[i]);
}

// multiply(FixedSparseMatrix, x, result) (SparseMatrix.h:299-320)
__global__ void k_csr_spmv(int n, const int* __restrict__ rowstart, const int* __restrict__ col,
                           const double* __restrict__ val, const double* __restrict__ x,
                           double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  for (int p = rowstart[i]; p < rowstart[i + 1]; ++p)
    acc = __dadd_rn(acc, __dmul_rn(val[p], x[col[p]]));
  out[i] = acc;
}

// per-block partial of sum a_i b_i (fixed grid, fixed order: deterministic)
__global__ void k_csr_dot_part(int n, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ part) {
  __shared__ double sm[kThreads];
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc = __dadd_rn(acc, __dmul_rn(a[i], b[i]));
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] = __dadd_rn(sm[threadIdx.x], sm[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// per-block partial of max |a_i|
__global__ void k_csr_absmax_part(int n, const double* __restrict__ a, double* __restrict__ part) {
  __shared__ double sm[kThreads];
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = fabs(a[i]);
    m = (v > m || v != v) ? v : m;  // NaN propagates
  }
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = sm[threadIdx.x + s];
      if (o > sm[threadIdx.x] || o != o) sm[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// sc[slot] = sum (or max) of the partials, in block order
__global__ void k_csr_finish(const double* __restrict__ part, int nparts, double* sc, int slot,
                             int is_max) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc = 0.0;
  for (int b = 0; b < nparts; ++b) {
    const double v = part[b];
    if (is_max)
      acc = (v > acc || v != v) ? v : acc;
    else
      acc = __dadd_rn(acc, v);
  }
  sc[slot] = acc;
}

// scalar slots
enum : int { SC_RHO = 0, SC_SZ, SC_RES, SC_RHONEW, SC_ALPHA, SC_BETA, kNumSc = 8 };

__global__ void k_csr_alpha(double* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc[SC_ALPHA] = __ddiv_rn(sc[SC_RHO], sc[SC_SZ]);
}

__global__ void k_csr_beta(double* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    sc[SC_BETA] = __ddiv_rn(sc[SC_RHONEW], sc[SC_RHO]);
    sc[SC_RHO] = sc[SC_RHONEW];
  }
}

// result += s * alpha;  r += z * (-alpha)  (BLAS::add_scaled, BLASWrapper.h:52-56)
__global__ void k_csr_update_xr(int n, const double* __restrict__ s, const double* __restrict__ z,
                                double* __restrict__ x, double* __restrict__ r,
                                const double* __restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double alpha = sc[SC_ALPHA];
  x[i] = __dadd_rn(x[i], __dmul_rn(s[i], alpha));
  r[i] = __dadd_rn(r[i], __dmul_rn(z[i], -alpha));
}

// z += s * beta (then the host swaps s and z)
__global__ void k_csr_update_z(int n, const double* __restrict__ s, double* __restrict__ z,
                               const double* __restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = __dadd_rn(z[i], __dmul_rn(s[i], sc[SC_BETA]));
}

struct Levels {
  std::vector<int> start;  // host copy of the level offsets
  Mem rows;                // rows ordered by level
};

// iterated frontier: level t holds the rows whose dependencies all sit on
// levels below t; every step assigns at least the lowest unassigned row
template <bool kForward>
cudaError_t make_levels(int n, const int* dep_start, const int* dep_list, Levels& L,
                        cudaStream_t st) {
  Mem lev, cnt, cur, assigned;
  CSR_TRY(lev.alloc((size_t)n * sizeof(int)));
  CSR_TRY(assigned.alloc(sizeof(int)));
  CSR_TRY(cudaMemsetAsync(lev.p, 0xff, (size_t)n * sizeof(int), st));
  CSR_TRY(cudaMemsetAsync(assigned.p, 0, sizeof(int), st));
  int total = 0, t = 0;
  while (total < n) {
    if (kForward)
      k_csr_level_fwd<<<nblocks(n), kThreads, 0, st>>>(n, dep_start, dep_list, lev.as<int>(), t,
                                                       assigned.as<int>());
    else
      k_csr_level_bwd<<<nblocks(n), kThreads, 0, st>>>(n, dep_start, dep_list, lev.as<int>(), t,
                                                       assigned.as<int>());
    CSR_TRY(cudaGetLastError());
    int now = 0;
    CSR_TRY(cudaMemcpyAsync(&now, assigned.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CSR_TRY(cudaStreamSynchronize(st));
    if (now == total) return cudaErrorInvalidValue;  // cannot happen for a triangular order
    total = now;
    ++t;
  }
  const int nlev = t;
  CSR_TRY(cnt.alloc((size_t)(nlev + 1) * sizeof(int)));
  CSR_TRY(cur.alloc((size_t)nlev * sizeof(int)));
  CSR_TRY(cudaMemsetAsync(cnt.p, 0, (size_t)(nlev + 1) * sizeof(int), st));
  CSR_TRY(cudaMemsetAsync(cur.p, 0, (size_t)nlev * sizeof(int), st));
  k_csr_level_count<<<nblocks(n), kThreads, 0, st>>>(n, lev.as<int>(), cnt.as<int>());
  std::vector<int> c(nlev);
  CSR_TRY(cudaMemcpyAsync(c.data(), cnt.p, (size_t)nlev * sizeof(int), cudaMemcpyDeviceToHost, st));
  CSR_TRY(cudaStreamSynchronize(st));
  L.start.assign(nlev + 1, 0);
  for (int l = 0; l < nlev; ++l) L.start[l + 1] = L.start[l] + c[l];
  CSR_TRY(cudaMemcpyAsync(cnt.p, L.start.data(), (size_t)(nlev + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  CSR_TRY(L.rows.alloc((size_t)n * sizeof(int)));
  k_csr_level_scatter<<<nblocks(n), kThreads, 0, st>>>(n, lev.as<int>(), cnt.as<int>(),
                                                       cur.as<int>(), L.rows.as<int>());
  CSR_TRY(cudaGetLastError());
  return cudaStreamSynchronize(st);
}

struct Solver {
  int n = 0;
  cudaStream_t st = nullptr;
  Mem rowstart, col, val, adiag, invdiag, ustart, urow, uval, tstart, tk, tp;
  Levels fwd, bwd;
  Mem vx, vr, vz, vs, part, sc;

  void precondition(double* in, double* out) {
    for (size_t l = 0; l + 1 < fwd.start.size(); ++l) {
      const int cnt = fwd.start[l + 1] - fwd.start[l];
      k_csr_lower_level<<<nblocks(cnt), kThreads, 0, st>>>(
          fwd.rows.as<int>() + fwd.start[l], cnt, tstart.as<int>(), tk.as<int>(), tp.as<int>(),
          uval.as<double>(), invdiag.as<double>(), in, out);
    }
    for (size_t l = 0; l + 1 < bwd.start.size(); ++l) {
      const int cnt = bwd.start[l + 1] - bwd.start[l];
      k_csr_upper_level<<<nblocks(cnt), kThreads, 0, st>>>(
          bwd.rows.as<int>() + bwd.start[l], cnt, ustart.as<int>(), urow.as<int>(),
          uval.as<double>(), invdiag.as<double>(), out);
    }
  }
  void dot(const double* a, const double* b, int slot) {
    k_csr_dot_part<<<kDotBlocks, kThreads, 0, st>>>(n, a, b, part.as<double>());
    k_csr_finish<<<1, 1, 0, st>>>(part.as<double>(), kDotBlocks, sc.as<double>(), slot, 0);
  }
  void absmax(const double* a, int slot) {
    k_csr_absmax_part<<<kDotBlocks, kThreads, 0, st>>>(n, a, part.as<double>());
    k_csr_finish<<<1, 1, 0, st>>>(part.as<double>(), kDotBlocks, sc.as<double>(), slot, 1);
  }
  cudaError_t read(int slot, double* out) {
    CSR_TRY(cudaMemcpyAsync(out, sc.as<double>() + slot, sizeof(double), cudaMemcpyDeviceToHost, st));
    return cudaStreamSynchronize(st);
  }
};

// 0: converged, 1: not converged (iteration limit or rho 0/NaN), 2: bad matrix
cudaError_t csr_solve(const int* h_rowstart, const int* h_col, const double* h_val, int n,
                      const double* h_rhs, double* h_x, double tolerance_factor, int maxiter,
                      double* residual_out, int* iters_out, int* outcome) {
  Solver S;
  S.n = n;
  CSR_TRY(cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{S.st};
  cudaStream_t st = S.st;
  const int nnz = h_rowstart[n] - h_rowstart[0];
  CSR_TRY(S.rowstart.alloc((size_t)(n + 1) * sizeof(int)));
  CSR_TRY(S.col.alloc((size_t)nnz * sizeof(int)));
  CSR_TRY(S.val.alloc((size_t)nnz * sizeof(double)));
  // rowstart relative to its first entry
  std::vector<int> rs(h_rowstart, h_rowstart + n + 1);
  const int base = rs[0];
  for (int& v : rs) v -= base;
  CSR_TRY(cudaMemcpyAsync(S.rowstart.p, rs.data(), (size_t)(n + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  CSR_TRY(cudaMemcpyAsync(S.col.p, h_col + base, (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, st));
  CSR_TRY(cudaMemcpyAsync(S.val.p, h_val + base, (size_t)nnz * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  Mem ucount, bad, tcount, tcur;
  CSR_TRY(ucount.alloc((size_t)(n + 1) * sizeof(int)));
  CSR_TRY(S.adiag.alloc((size_t)n * sizeof(double)));
  CSR_TRY(S.invdiag.alloc((size_t)n * sizeof(double)));
  CSR_TRY(bad.alloc(sizeof(int)));
  CSR_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
  k_csr_rows<<<nblocks(n), kThreads, 0, st>>>(n, S.rowstart.as<int>(), S.col.as<int>(),
                                              S.val.as<double>(), ucount.as<int>(),
                                              S.adiag.as<double>(), bad.as<int>());
  int hbad = 0;
  CSR_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSR_TRY(cudaStreamSynchronize(st));
  if (hbad) {
    *outcome = 2;
    return cudaSuccess;
  }
  // factor columns (upper parts of the rows) and their transpose
  Mem tmp;
  CSR_TRY(tmp.alloc((size_t)((n + 1 + kScanTile - 1) / kScanTile + 1) * sizeof(int)));
  CSR_TRY(S.ustart.alloc((size_t)(n + 1) * sizeof(int)));
  exclusive_scan<int, int>(ucount.as<int>(), n, S.ustart.as<int>(), tmp.as<int>(),
                           S.ustart.as<int>() + n, st);
  int nu = 0;
  CSR_TRY(cudaMemcpyAsync(&nu, S.ustart.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSR_TRY(cudaStreamSynchronize(st));
  CSR_TRY(S.urow.alloc((size_t)nu * sizeof(int)));
  CSR_TRY(S.uval.alloc((size_t)nu * sizeof(double)));
  CSR_TRY(tcount.alloc((size_t)(n + 1) * sizeof(int)));
  CSR_TRY(tcur.alloc((size_t)n * sizeof(int)));
  CSR_TRY(cudaMemsetAsync(tcount.p, 0, (size_t)(n + 1) * sizeof(int), st));
  CSR_TRY(cudaMemsetAsync(tcur.p, 0, (size_t)n * sizeof(int), st));
  k_csr_upper<<<nblocks(n), kThreads, 0, st>>>(n, S.rowstart.as<int>(), S.col.as<int>(),
                                               S.val.as<double>(), S.ustart.as<int>(),
                                               S.urow.as<int>(), S.uval.as<double>(),
                                               tcount.as<int>());
  CSR_TRY(S.tstart.alloc((size_t)(n + 1) * sizeof(int)));
  exclusive_scan<int, int>(tcount.as<int>(), n, S.tstart.as<int>(), tmp.as<int>(),
                           S.tstart.as<int>() + n, st);
  CSR_TRY(S.tk.alloc((size_t)nu * sizeof(int)));
  CSR_TRY(S.tp.alloc((size_t)nu * sizeof(int)));
  k_csr_transpose<<<nblocks(n), kThreads, 0, st>>>(n, S.ustart.as<int>(), S.urow.as<int>(),
                                                   S.tstart.as<int>(), tcur.as<int>(),
                                                   S.tk.as<int>(), S.tp.as<int>());
  k_csr_sort_transpose<<<nblocks(n), kThreads, 0, st>>>(n, S.tstart.as<int>(), S.tk.as<int>(),
                                                        S.tp.as<int>());
  CSR_TRY(cudaGetLastError());
  CSR_TRY((make_levels<true>(n, S.tstart.as<int>(), S.tk.as<int>(), S.fwd, st)));
  CSR_TRY((make_levels<false>(n, S.ustart.as<int>(), S.urow.as<int>(), S.bwd, st)));

  // PCG vectors
  const size_t vb = (size_t)n * sizeof(double);
  CSR_TRY(S.vx.alloc(vb));
  CSR_TRY(S.vr.alloc(vb));
  CSR_TRY(S.vz.alloc(vb));
  CSR_TRY(S.vs.alloc(vb));
  CSR_TRY(S.part.alloc(kDotBlocks * sizeof(double)));
  CSR_TRY(S.sc.alloc(kNumSc * sizeof(double)));
  double* x = S.vx.as<double>();
  double* r = S.vr.as<double>();
  double* z = S.vz.as<double>();
  double* s = S.vs.as<double>();
  CSR_TRY(cudaMemsetAsync(x, 0, vb, st));
  CSR_TRY(cudaMemcpyAsync(r, h_rhs, vb, cudaMemcpyHostToDevice, st));
  int iters = 0;
  bool ok = false;
  double res = 0.0;
  S.absmax(r, SC_RES);
  CSR_TRY(S.read(SC_RES, &res));
  if (res < 1e-30) {
    ok = true;
  } else {
    const double tf = tolerance_factor < 1e-30 ? 1e-30 : tolerance_factor;
    const double tol = tf * res;
    // the factorisation, level by level
    for (size_t l = 0; l + 1 < S.fwd.start.size(); ++l) {
      const int cnt = S.fwd.start[l + 1] - S.fwd.start[l];
      k_csr_factor_level<<<nblocks(cnt), kThreads, 0, st>>>(
          S.fwd.rows.as<int>() + S.fwd.start[l], cnt, S.rowstart.as<int>(), S.col.as<int>(),
          S.ustart.as<int>(), S.urow.as<int>(), S.uval.as<double>(), S.tstart.as<int>(),
          S.tk.as<int>(), S.tp.as<int>(), S.adiag.as<double>(), S.invdiag.as<double>());
    }
    CSR_TRY(cudaGetLastError());
    S.precondition(r, z);
    S.dot(z, r, SC_RHO);
    double rho = 0.0;
    CSR_TRY(S.read(SC_RHO, &rho));
    if (!(rho == 0.0 || rho != rho)) {
      CSR_TRY(cudaMemcpyAsync(s, z, vb, cudaMemcpyDeviceToDevice, st));
      int it = 0;
      for (; it < maxiter; ++it) {
        k_csr_spmv<<<nblocks(n), kThreads, 0, st>>>(n, S.rowstart.as<int>(), S.col.as<int>(),
                                                    S.val.as<double>(), s, z);
        S.dot(s, z, SC_SZ);
        k_csr_alpha<<<1, 1, 0, st>>>(S.sc.as<double>());
        k_csr_update_xr<<<nblocks(n), kThreads, 0, st>>>(n, s, z, x, r, S.sc.as<double>());
        S.absmax(r, SC_RES);
        CSR_TRY(cudaGetLastError());
        CSR_TRY(S.read(SC_RES, &res));
        if (res <= tol) {
          iters = it + 1;
          ok = true;
          break;
        }
        S.precondition(r, z);
        S.dot(z, r, SC_RHONEW);
        k_csr_beta<<<1, 1, 0, st>>>(S.sc.as<double>());
        k_csr_update_z<<<nblocks(n), kThreads, 0, st>>>(n, s, z, S.sc.as<double>());
        std::swap(s, z);
      }
      if (!ok) iters = it;
    }
  }
  CSR_TRY(cudaMemcpyAsync(h_x, x, vb, cudaMemcpyDeviceToHost, st));
  CSR_TRY(cudaStreamSynchronize(st));
  CSR_TRY(cudaGetLastError());
  *residual_out = res;
  *iters_out = iters;
  *outcome = ok ? 0 : 1;
  return cudaSuccess;
}

}  // namespace
}  // namespace wcg

extern "C" int wcg_pcg_solve_csr(const int* rowstart, const int* col, const double* val, int n,
                                 const double* rhs, double* x, double tolerance_factor,
                                 int max_iterations, double* residual_out, int* iterations_out) {
  if (n < 0) return wcg::set_last_error(WCG_ERR_ARG, "wcg_pcg_solve_csr: negative size");
  if (n > 0 && (!rowstart || !col || !val || !rhs || !x))
    return wcg::set_last_error(WCG_ERR_ARG, "wcg_pcg_solve_csr: null array");
  if (!residual_out || !iterations_out)
    return wcg::set_last_error(WCG_ERR_ARG, "wcg_pcg_solve_csr: null output");
  if (max_iterations < 0)
    return wcg::set_last_error(WCG_ERR_ARG, "wcg_pcg_solve_csr: negative iteration limit");
  *residual_out = 0.0;
  *iterations_out = 0;
  if (n == 0) return WCG_OK;
  if (rowstart[n] < rowstart[0])
    return wcg::set_last_error(WCG_ERR_ARG, "wcg_pcg_solve_csr: rowstart decreases");
  int outcome = 0;
  const cudaError_t e = wcg::csr_solve(rowstart, col, val, n, rhs, x, tolerance_factor,
                                       max_iterations, residual_out, iterations_out, &outcome);
  if (e != cudaSuccess)
    return wcg::set_last_error(WCG_ERR_CUDA, std::string("wcg_pcg_solve_csr: ") +
                                                 cudaGetErrorString(e));
  if (outcome == 2)
    return wcg::set_last_error(WCG_ERR_ARG,
                               "wcg_pcg_solve_csr: rows must hold strictly ascending columns "
                               "in [0, n) and rowstart must not decrease");
  if (outcome == 1)
    return wcg::set_last_error(WCG_ERR_NOT_CONVERGED,
                               "wcg_pcg_solve_csr: iteration limit reached or rho was 0/NaN");
  return WCG_OK;
}
