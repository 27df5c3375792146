// Allocation-free variant of the pressure solve (wcg_pressure_solve_noalloc).
//
// Some callers cannot call cudaMalloc at all: a host simulator that owns and
// pre-reserves every byte of device memory, a process running under a strict
// memory budget or pool, or code that must not allocate between frames.  This
// entry point runs the same FP64 MIC(0)-PCG as wcg_project_fine on a system the
// caller has already assembled, and takes every byte of solver scratch (PCG
// vectors, MIC(0) factor, wavefront tile lists and flags, reduction partials)
// from one file-scope __device__ array.  That array is part of the module, so
// every GPU that loads libwcgpu.so holds it (about 17 MB) until the process
// exits.
//
// Limits and sharing: at most kNoAllocMaxBuckets buckets (4x4x4 cells each,
// 131072 cells).  All calls on a device share the array and it keeps the last
// call's contents; every field that must start at zero is cleared per call.
// Calls whose GPU work overlaps (concurrent streams or threads on one device)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/wetcloth_gpu.h"
#include "wcg_context.h"

namespace {

constexpr long long kNoAllocMaxBuckets = 2048;
constexpr long long kNoAllocMaxCells = kNoAllocMaxBuckets * 64;
constexpr long long kFirstField = wcg::G_ADIAG;  // solver fields G_ADIAG..G_SZ
constexpr long long kNumFields = wcg::G_SZ - wcg::G_ADIAG + 1;
constexpr long long kMaxTiles = kNoAllocMaxBuckets;  // 2x2x2-bucket tiles <= buckets
constexpr long long kIntTmp = 2 * kNoAllocMaxBuckets + 64;
constexpr long long kWaveInts = 4096;
constexpr long long kPartials = 8192;  // reduction partials (>= 8 per block of 592)

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// byte offsets inside the scratch array
constexpr size_t kOffFields = 0;
constexpr size_t kOffActive = align256(kOffFields + kNumFields * kNoAllocMaxCells * sizeof(double));
constexpr size_t kOffActiveList = align256(kOffActive + kNoAllocMaxBuckets);
constexpr size_t kOffTmp = align256(kOffActiveList + kNoAllocMaxBuckets * sizeof(int));
constexpr size_t kOffTileActive = align256(kOffTmp + kIntTmp * sizeof(int));
constexpr size_t kOffTileFlag = align256(kOffTileActive + kMaxTiles);
constexpr size_t kOffWaveList = align256(kOffTileFlag + kMaxTiles * sizeof(int));
constexpr size_t kOffTilePart = align256(kOffWaveList + kMaxTiles * sizeof(int));
constexpr size_t kOffWaveCount = align256(kOffTilePart + kMaxTiles * sizeof(double));
constexpr size_t kOffPartials = align256(kOffWaveCount + kWaveInts * sizeof(int));
constexpr size_t kOffScalars = align256(kOffPartials + kPartials * sizeof(double));
constexpr size_t kOffTicket = align256(kOffScalars + 64 * sizeof(double));
constexpr size_t kOffErr = align256(kOffTicket + 16 * sizeof(int));
constexpr size_t kScratchBytes = align256(kOffErr + sizeof(int));

}  // namespace

// The scratch.  In host code this name is only a host-side stand-in; the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_wcg_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mutex;
void* g_scratch_addr[64] = {nullptr};

int noalloc_fail(int code, const std::string& m) { return wcg::set_last_error(code, m); }

}  // namespace

extern "C" int wcg_pressure_solve_noalloc(int ni, int nj, int nk, const unsigned char* dof,
                                          const double* a_diag, const double* a_x,
                                          const double* a_y, const double* a_z,
                                          const double* rhs, double* pressure,
                                          double criterion, int maxiters, void* stream,
                                          int* iters_out, double* residual_out) {
  if (ni <= 0 || nj <= 0 || nk <= 0)
    return noalloc_fail(WCG_ERR_ARG, "grid dimensions must be positive");
  const long long nb = (long long)ni * nj * nk;
  if (nb > kNoAllocMaxBuckets)
    return noalloc_fail(WCG_ERR_ARG,
                        "grid of " + std::to_string(nb) + " buckets exceeds the " +
                            std::to_string(kNoAllocMaxBuckets) +
                            "-bucket (131072-cell) limit of the allocation-free solver");
  if (!dof || !a_diag || !a_x || !a_y || !a_z || !rhs || !pressure)
    return noalloc_fail(WCG_ERR_ARG, "null device array");
  if (!(criterion > 0) || maxiters < 0)
    return noalloc_fail(WCG_ERR_ARG, "criterion must be > 0 and maxiters >= 0");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return noalloc_fail(WCG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  void* base = nullptr;
  {
    // once per device, with that device current: the device address of the
    // scratch array (the symbol itself is not a device address in host code)
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_wcg_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        return noalloc_fail(WCG_ERR_CUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    base = g_scratch_addr[dev];
  }
  unsigned char* S = (unsigned char*)base;
  const cudaStream_t st = (cudaStream_t)stream;

  wcg::Context c;
  c.stream = st;
  c.device = dev;
  c.prm.criterion = criterion;
  c.prm.maxiters = maxiters;
  c.prm.precision = 0;
  wcg::GridDesc& g = c.g;
  g.ni = ni; g.nj = nj; g.nk = nk;
  g.NI = ni * 4; g.NJ = nj * 4; g.NK = nk * 4;
  g.nb = nb;
  g.nnode = nb * 64;
  g.ox = g.oy = g.oz = 0.0;
  g.bs = 4.0;
  g.dx = 1.0;
  c.have_grid = true;
  // field base chosen so that field G_ADIAG starts at the scratch fields
  c.gcap = kNoAllocMaxCells;
  double* fields = (double*)(S + kOffFields);
  c.gfield.p = (void*)(fields - kFirstField * c.gcap);
  c.gfield.bytes = 0;  // views into the scratch: never grown or freed
  c.gdof.p = (void*)dof;
  c.active.p = S + kOffActive;
  c.active_list.p = S + kOffActiveList;
  c.cell_cursor.p = S + kOffTmp;
  c.tile_active.p = S + kOffTileActive;
  c.tile_flag.p = S + kOffTileFlag;
  c.wave_list.p = S + kOffWaveList;
  c.tile_part.p = S + kOffTilePart;
  c.wave_count.p = S + kOffWaveCount;
  c.scratch.p = S + kOffPartials;
  c.dscalars.p = S + kOffScalars;
  c.ticket.p = S + kOffTicket;
  c.derr.p = S + kOffErr;

  // clear the state that must start at zero; copy in the system
  const size_t cells = (size_t)g.nnode * sizeof(double);
  double* F = (double*)c.gfield.p;
  cudaError_t ce = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (ce == cudaSuccess) ce = x;
  };
  chk(cudaMemsetAsync(S + kOffTileFlag, 0, kMaxTiles * sizeof(int), st));
  chk(cudaMemsetAsync(S + kOffErr, 0, sizeof(int), st));
  chk(cudaMemcpyAsync(F + wcg::G_ADIAG * c.gcap, a_diag, cells, cudaMemcpyDeviceToDevice, st));
  chk(cudaMemcpyAsync(F + wcg::G_AX * c.gcap, a_x, cells, cudaMemcpyDeviceToDevice, st));
  chk(cudaMemcpyAsync(F + wcg::G_AY * c.gcap, a_y, cells, cudaMemcpyDeviceToDevice, st));
  chk(cudaMemcpyAsync(F + wcg::G_AZ * c.gcap, a_z, cells, cudaMemcpyDeviceToDevice, st));
  chk(cudaMemcpyAsync(F + wcg::G_B * c.gcap, rhs, cells, cudaMemcpyDeviceToDevice, st));
  if (ce != cudaSuccess)
    return noalloc_fail(WCG_ERR_CUDA, std::string("set-up: ") + cudaGetErrorString(ce));
  int iters = 0, conv = 0;
  double res = 0, bnorm = 0;
  ce = wcg::prepared_solve_fp64(c, pressure, &iters, &res, &conv, &bnorm);
  if (ce != cudaSuccess)
    return noalloc_fail(WCG_ERR_CUDA, std::string("solve: ") + cudaGetErrorString(ce));
  int herr = 0;
  ce = cudaMemcpyAsync(&herr, c.derr.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess)
    return noalloc_fail(WCG_ERR_CUDA, std::string("status: ") + cudaGetErrorString(ce));
  if (iters_out) *iters_out = iters;
  if (residual_out) *residual_out = res;
  if (herr)
    return noalloc_fail(WCG_ERR_DEVICE, "device error code " + std::to_string(herr));
  if (!conv)
    return noalloc_fail(WCG_ERR_NOT_CONVERGED, "pressure PCG did not converge");
  return WCG_OK;
}
