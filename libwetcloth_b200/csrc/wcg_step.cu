// Host orchestration of the fluid step: one function per reference call,
// dispatching on the precision of the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "wcg_context.h"
#include "wcg_kernels.cuh"
#include "wcg_pcg.cuh"
#include "wcg_wsweep.cuh"
#include "wcg_pencil.cuh"
#include "wcg_mg.cuh"
#include "wcg_visc.cuh"
#include "wcg_elasto.cuh"
#include "wcg_adjoint.cuh"
#include "wcg_correct.cuh"
#include "wcg_merge.cuh"
#include "wcg_scan.cuh"

namespace wcg {

#define WCG_TRY(x)                          \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

cudaError_t DevBuf::ensure(size_t n) {
  if (n <= bytes && p) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(&p, n);
  if (e == cudaSuccess) bytes = n;
  return e;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

static inline unsigned nblk(long long n, int t) {
  return (unsigned)((n + t - 1) / t);
}

cudaError_t ctx_init(Context& c) {
  WCG_TRY(cudaGetDevice(&c.device));
  WCG_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  WCG_TRY(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_store, cudaEventDisableTiming));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_d2h, cudaEventDisableTiming));
  WCG_TRY(cudaStreamCreateWithFlags(&c.in_stream, cudaStreamNonBlocking));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_staged, cudaEventDisableTiming));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_loaded, cudaEventDisableTiming));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_ss_ready, cudaEventDisableTiming));
  WCG_TRY(cudaEventCreateWithFlags(&c.ev_ss_done, cudaEventDisableTiming));
  WCG_TRY(cudaMallocHost((void**)&c.hscalars, 64 * sizeof(double)));
  WCG_TRY(cudaHostAlloc((void**)&c.hmap, kReadSmallBytes, cudaHostAllocMapped));
  WCG_TRY(cudaHostGetDevicePointer((void**)&c.hmap_dev, c.hmap, 0));
  WCG_TRY(c.dscalars.ensure(64 * sizeof(double)));
  WCG_TRY(c.derr.ensure(sizeof(int)));
  WCG_TRY(c.ticket.ensure(16 * sizeof(int)));
  WCG_TRY(cudaMemsetAsync(c.derr.p, 0, sizeof(int), c.stream));
  WCG_TRY(cudaMemsetAsync(c.dscalars.p, 0, 64 * sizeof(double), c.stream));
  return cudaStreamSynchronize(c.stream);
}

void ctx_free(Context& c) {
  DevBuf* bufs[] = {&c.pbuf[0], &c.pbuf[1], &c.pid[0], &c.pid[1], &c.pkey,
                    &c.pdelta, &c.pbucket, &c.perm, &c.hostorder,
                    &c.ebuf[0], &c.ebuf[1], &c.epid[0], &c.epid[1], &c.ekey, &c.edelta,
                    &c.ebucket, &c.eperm, &c.estage, &c.ecell_start, &c.efield,
                    &c.active_pre, &c.active, &c.cell_start, &c.cell_cursor,
                    &c.gfield, &c.gvalid, &c.gdof, &c.wave_list, &c.wave_count,
                    &c.tile_flag, &c.tile_active, &c.tile_part, &c.active_list, &c.p2g_halo,
                    &c.rx64, &c.rr64, &c.rb64,
                    &c.pl, &c.pl64, &c.pl_edge, &c.pl_order, &c.pl_corder, &c.pl_corder2,
                    &c.pl_part,
                    &c.mg, &c.mg_mask, &c.mg_vec,
                    &c.adj, &c.adjp, &c.adjmask, &c.adjstage, &c.adjvisc, &c.adjxc, &c.adjam,
                    &c.visc, &c.viscflag, &c.dstage, &c.ustage,
                    &c.xw, &c.corr_start, &c.corr_cursor, &c.corr_list, &c.mwork,
                    &c.split_rank, &c.split_pat, &c.split_rot,
                    &c.scratch, &c.dscalars, &c.derr, &c.ticket};
  for (DevBuf* b : bufs) b->release();
  if (c.hscalars) cudaFreeHost(c.hscalars);
  c.hscalars = nullptr;
  if (c.hmap) cudaFreeHost(c.hmap);
  c.hmap = c.hmap_dev = nullptr;
  for (Context::ProfRec& r : c.prof_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  c.prof_recs.clear();
  for (cudaEvent_t e : c.prof_pool) cudaEventDestroy(e);
  c.prof_pool.clear();
  if (c.copy_stream) {
    cudaStreamSynchronize(c.copy_stream);
    cudaStreamDestroy(c.copy_stream);
  }
  c.copy_stream = nullptr;
  if (c.in_stream) {
    cudaStreamSynchronize(c.in_stream);
    cudaStreamDestroy(c.in_stream);
  }
  c.in_stream = nullptr;
  if (c.ev_staged) cudaEventDestroy(c.ev_staged);
  if (c.ev_loaded) cudaEventDestroy(c.ev_loaded);
  c.ev_staged = c.ev_loaded = nullptr;
  if (c.ev_ss_ready) cudaEventDestroy(c.ev_ss_ready);
  if (c.ev_ss_done) cudaEventDestroy(c.ev_ss_done);
  c.ev_ss_ready = c.ev_ss_done = nullptr;
  if (c.ev_store) cudaEventDestroy(c.ev_store);
  if (c.ev_d2h) cudaEventDestroy(c.ev_d2h);
  c.ev_store = c.ev_d2h = nullptr;
  if (c.stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
}

ProfScope::ProfScope(Context& cc, int category) : c(cc), cat(category), l0(cc.launches) {
  if (!c.prof_on) return;
  if (c.prof_pool.empty()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c.prof_pool.push_back(e);
  }
  a = c.prof_pool.back();
  c.prof_pool.pop_back();
  cudaEventRecord(a, c.stream);
}

ProfScope::~ProfScope() {
  if (!c.prof_on || !a) return;
  cudaEvent_t b;
  if (c.prof_pool.empty()) {
    cudaEventCreate(&b);
  } else {
    b = c.prof_pool.back();
    c.prof_pool.pop_back();
  }
  cudaEventRecord(b, c.stream);
  c.prof_recs.push_back({cat, (int)(c.launches - l0), a, b});
}

__global__ void k_read_words(const unsigned* __restrict__ src, unsigned* __restrict__ dst,
                             int nwords) {
  for (int i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = src[i];
}

cudaError_t read_small(Context& c, const void* d, size_t bytes, void* h) {
  if (bytes == 0) return cudaSuccess;
  if (!c.hmap || !c.hmap_dev) {
    // a context without the mapped words (the allocation-free solve builds
    // its context from caller memory and allocates nothing): a plain copy
    WCG_TRY(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c.stream));
    return cudaStreamSynchronize(c.stream);
  }
  if (bytes % 4 != 0 || bytes > kReadSmallBytes || ((size_t)d & 3) != 0)
    return cudaErrorInvalidValue;
  ++c.launches, k_read_words<<<1, 128, 0, c.stream>>>(static_cast<const unsigned*>(d),
                                                       c.hmap_dev, (int)(bytes / 4));
  WCG_TRY(cudaGetLastError());
  WCG_TRY(cudaStreamSynchronize(c.stream));
  std::memcpy(h, c.hmap, bytes);
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// particles

// device word set by an upload that brought a liquid particle without fluid
// volume (cleared when the sub-step removes such particles)
static int* empty_word(Context& c) { return (int*)(c.dscalars.as<double>() + 52); }

template <typename R>
__global__ void k_load_particles(long long n, long long pcap, const double* x3,
                                 const double* v3, const double* C9,
                                 const double* m, const double* vol,
                                 const double* rad, R* P, int* pid, int* err,
                                 int* empty) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool bad = !(m[i] >= 0.0) || !(vol[i] >= 0.0) || !(rad[i] >= 0.0);
  // removeEmptyParticles drops liquid particles below 1e-20 of fluid volume
  // at the start of every sub-step (TwoDScene.cpp:1717-1721)
  if (vol[i] < 1e-20) *empty = 1;
  for (int a = 0; a < 3; ++a) {
    const double x = x3[i * 3 + a], v = v3[i * 3 + a];
    bad = bad || !isfinite(x) || !isfinite(v);
    P[(PX + a) * pcap + i] = (R)x;
    P[(VX + a) * pcap + i] = (R)v;
  }
  if (bad && err) record_error(err, kErrInput);
  for (int q = 0; q < 9; ++q) P[(C00 + q) * pcap + i] = C9 ? (R)C9[i * 9 + q] : R(0);
  P[PM * pcap + i] = (R)m[i];
  P[PV * pcap + i] = (R)vol[i];
  P[PR * pcap + i] = (R)rad[i];
  pid[i] = (int)i;
}

// scatter sorted state back to original particle order: x3 at out[0, 3n),
// v3 at out[3n, 6n), C9 at out[6n, 15n), each in the caller's layout so the
// copies out are contiguous
template <typename R>
__global__ void k_store_particles(long long n, long long pcap, const R* P,
                                  const int* pid, double* out) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long long i = pid[s];
  for (int a = 0; a < 3; ++a) {
    out[i * 3 + a] = (double)P[(PX + a) * pcap + s];
    out[3 * n + i * 3 + a] = (double)P[(VX + a) * pcap + s];
  }
  for (int q = 0; q < 9; ++q) out[6 * n + i * 9 + q] = (double)P[(C00 + q) * pcap + s];
}

// positions in the reference's m_x layout (x, y, z, twist = 0 per particle) and
// radii, original particle order
template <typename R>
__global__ void k_store_positions(long long n, long long pcap, const R* P, const int* pid,
                                  double* x4, double* rad) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long long i = pid[s];
  for (int a = 0; a < 3; ++a) x4[i * 4 + a] = (double)P[(PX + a) * pcap + s];
  x4[i * 4 + 3] = 0.0;
  rad[i] = (double)P[PR * pcap + s];
}

// replace positions (reference m_x layout, original order) of the sorted state
template <typename R>
__global__ void k_set_positions(long long n, long long pcap, R* P, const int* pid,
                                const double* x4) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long long i = pid[s];
  for (int a = 0; a < 3; ++a) P[(PX + a) * pcap + s] = (R)x4[i * 4 + a];
}

cudaError_t upload_particles(Context& c, long long n, const double* x3,
                             const double* v3, const double* C9,
                             const double* mass, const double* vol,
                             const double* radius, bool device_ptrs) {
  const int rb = c.real_bytes();
  if (n > c.pcap) {
    const long long cap = n;
    for (int k = 0; k < 2; ++k) {
      WCG_TRY(c.pbuf[k].ensure((size_t)kNumPCols * cap * rb));
      WCG_TRY(c.pid[k].ensure((size_t)cap * sizeof(int)));
    }
    WCG_TRY(c.pkey.ensure((size_t)2 * cap * sizeof(long long)));
    WCG_TRY(c.pdelta.ensure((size_t)2 * cap * sizeof(int)));
    WCG_TRY(c.pbucket.ensure((size_t)2 * cap * sizeof(int)));
    WCG_TRY(c.perm.ensure((size_t)cap * sizeof(int)));
    WCG_TRY(c.hostorder.ensure((size_t)cap * 15 * sizeof(double)));
    c.pcap = cap;
  }
  c.np = n;
  c.cur = 0;
  c.buckets_valid = false;
  if (n == 0) return cudaSuccess;
  // stage host arrays into the scratch copy (device side, doubles)
  double* stage = c.hostorder.as<double>();
  const double* dx3 = x3;
  const double* dv3 = v3;
  const double* dC9 = C9;
  const double* dm = mass;
  const double* dvol = vol;
  const double* drad = radius;
  if (!device_ptrs) {
    double* s = stage;
    WCG_TRY(cudaMemcpyAsync(s, x3, n * 3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    dx3 = s; s += n * 3;
    WCG_TRY(cudaMemcpyAsync(s, v3, n * 3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    dv3 = s; s += n * 3;
    if (C9) {
      WCG_TRY(cudaMemcpyAsync(s, C9, n * 9 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
      dC9 = s; s += n * 9;
    }
    // mass/vol/radius reuse the pkey buffer (3n doubles fit in 2n int64 + ...)
    double* t = (double*)c.pkey.p;
    WCG_TRY(cudaMemcpyAsync(t, mass, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    WCG_TRY(cudaMemcpyAsync(t + n, vol, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    // radius goes to the delta+bucket buffers viewed as doubles
    double* t2 = (double*)c.pdelta.p;
    WCG_TRY(cudaMemcpyAsync(t2, radius, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    dm = t;
    dvol = t + n;
    drad = t2;
  }
  if (c.prm.precision == 0)
    ++c.launches, k_load_particles<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, dx3, dv3, dC9, dm, dvol, drad, c.pbuf[0].as<double>(),
        c.pid[0].as<int>(), c.derr.as<int>(), empty_word(c));
  else
    ++c.launches, k_load_particles<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, dx3, dv3, dC9, dm, dvol, drad, c.pbuf[0].as<float>(),
        c.pid[0].as<int>(), c.derr.as<int>(), empty_word(c));
  c.maybe_empty = true;
  WCG_TRY(cudaGetLastError());
  return cudaStreamSynchronize(c.stream);
}

cudaError_t download_particles(Context& c, double* x3, double* v3, double* C9,
                               bool device_ptrs) {
  const long long n = c.np;
  if (n == 0) return cudaSuccess;
  double* st = c.hostorder.as<double>();
  if (c.prm.precision == 0)
    ++c.launches, k_store_particles<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<double>(), c.pid[c.cur].as<int>(), st);
  else
    ++c.launches, k_store_particles<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<float>(), c.pid[c.cur].as<int>(), st);
  WCG_TRY(cudaGetLastError());
  const cudaMemcpyKind kind =
      device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (x3)
    WCG_TRY(cudaMemcpyAsync(x3, st, n * 3 * sizeof(double), kind, c.stream));
  if (v3)
    WCG_TRY(cudaMemcpyAsync(v3, st + 3 * n, n * 3 * sizeof(double), kind, c.stream));
  if (C9)
    WCG_TRY(cudaMemcpyAsync(C9, st + 6 * n, n * 9 * sizeof(double), kind, c.stream));
  return cudaStreamSynchronize(c.stream);
}

cudaError_t download_particles_async(Context& c, double* x3, double* v3, double* C9) {
  const long long n = c.np;
  if (n == 0) return cudaSuccess;
  WCG_TRY(c.dstage.ensure((size_t)15 * n * sizeof(double)));
  double* st = c.dstage.as<double>();
  // the previous asynchronous download must have read dstage out
  WCG_TRY(cudaStreamWaitEvent(c.stream, c.ev_d2h, 0));
  if (c.prm.precision == 0)
    ++c.launches, k_store_particles<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<double>(), c.pid[c.cur].as<int>(), st);
  else
    ++c.launches, k_store_particles<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<float>(), c.pid[c.cur].as<int>(), st);
  WCG_TRY(cudaGetLastError());
  WCG_TRY(cudaEventRecord(c.ev_store, c.stream));
  WCG_TRY(cudaStreamWaitEvent(c.copy_stream, c.ev_store, 0));
  if (x3)
    WCG_TRY(cudaMemcpyAsync(x3, st, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c.copy_stream));
  if (v3)
    WCG_TRY(cudaMemcpyAsync(v3, st + 3 * n, n * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                            c.copy_stream));
  if (C9)
    WCG_TRY(cudaMemcpyAsync(C9, st + 6 * n, n * 9 * sizeof(double), cudaMemcpyDeviceToHost,
                            c.copy_stream));
  return cudaEventRecord(c.ev_d2h, c.copy_stream);
}

cudaError_t synchronize(Context& c) {
  WCG_TRY(cudaStreamSynchronize(c.stream));
  WCG_TRY(cudaStreamSynchronize(c.in_stream));
  return cudaStreamSynchronize(c.copy_stream);
}

cudaError_t stage_particles_async(Context& c, long long n, const double* x3, const double* v3,
                                  const double* C9, const double* mass, const double* vol,
                                  const double* radius) {
  WCG_TRY(c.ustage.ensure((size_t)18 * std::max(n, 1LL) * sizeof(double)));
  double* u = c.ustage.as<double>();
  // the previously staged set must have been loaded
  WCG_TRY(cudaStreamWaitEvent(c.in_stream, c.ev_loaded, 0));
  const cudaMemcpyKind k = cudaMemcpyHostToDevice;
  WCG_TRY(cudaMemcpyAsync(u, x3, n * 3 * sizeof(double), k, c.in_stream));
  WCG_TRY(cudaMemcpyAsync(u + 3 * n, v3, n * 3 * sizeof(double), k, c.in_stream));
  if (C9) WCG_TRY(cudaMemcpyAsync(u + 6 * n, C9, n * 9 * sizeof(double), k, c.in_stream));
  WCG_TRY(cudaMemcpyAsync(u + 15 * n, mass, n * sizeof(double), k, c.in_stream));
  WCG_TRY(cudaMemcpyAsync(u + 16 * n, vol, n * sizeof(double), k, c.in_stream));
  WCG_TRY(cudaMemcpyAsync(u + 17 * n, radius, n * sizeof(double), k, c.in_stream));
  WCG_TRY(cudaEventRecord(c.ev_staged, c.in_stream));
  c.staged_n = n;
  c.staged_C = C9 != nullptr;
  return cudaSuccess;
}

cudaError_t load_staged(Context& c) {
  const long long n = c.staged_n;
  const double* u = c.ustage.as<double>();
  WCG_TRY(cudaStreamWaitEvent(c.stream, c.ev_staged, 0));
  // device-pointer upload from the staging buffer (grows the arrays as needed)
  WCG_TRY(upload_particles(c, n, u, u + 3 * n, c.staged_C ? u + 6 * n : nullptr, u + 15 * n,
                           u + 16 * n, u + 17 * n, true));
  WCG_TRY(cudaEventRecord(c.ev_loaded, c.stream));
  c.staged_n = -1;
  return cudaSuccess;
}

cudaError_t download_positions(Context& c, double* x4, double* radius) {
  const long long n = c.np;
  if (n == 0) return cudaSuccess;
  double* st = c.hostorder.as<double>();
  if (c.prm.precision == 0)
    ++c.launches, k_store_positions<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<double>(), c.pid[c.cur].as<int>(), st, st + 4 * n);
  else
    ++c.launches, k_store_positions<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<float>(), c.pid[c.cur].as<int>(), st, st + 4 * n);
  WCG_TRY(cudaGetLastError());
  WCG_TRY(cudaMemcpyAsync(x4, st, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (radius)
    WCG_TRY(cudaMemcpyAsync(radius, st + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
  return cudaStreamSynchronize(c.stream);
}

cudaError_t upload_positions(Context& c, const double* x4) {
  const long long n = c.np;
  if (n == 0) return cudaSuccess;
  double* st = c.hostorder.as<double>();
  WCG_TRY(cudaMemcpyAsync(st, x4, n * 4 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  if (c.prm.precision == 0)
    ++c.launches, k_set_positions<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<double>(), c.pid[c.cur].as<int>(), st);
  else
    ++c.launches, k_set_positions<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.pcap, c.pbuf[c.cur].as<float>(), c.pid[c.cur].as<int>(), st);
  WCG_TRY(cudaGetLastError());
  // positions changed: the grid of the old positions no longer applies
  c.have_grid = false;
  return cudaStreamSynchronize(c.stream);
}

// Elasto particles: the host packs the reference's per-particle members into
// kNumECols double columns (m(a) + m_fluid(a) summed in double, as the
// reference's P2G does), one copy, one conversion kernel.
cudaError_t upload_elasto(Context& c, long long n, const double* x4, const double* v4,
                          const double* B9, const double* m4, const double* fm4,
                          const double* rest_vol, const double* rest_vf,
                          const double* fluid_vol, const double* shape_factor,
                          const double* orient3, const int* surfel) {
  const int rb = c.real_bytes();
  if (n > c.ecap) {
    const long long cap = n;
    for (int k = 0; k < 2; ++k) {
      WCG_TRY(c.ebuf[k].ensure((size_t)kNumECols * cap * rb));
      WCG_TRY(c.epid[k].ensure((size_t)cap * sizeof(int)));
    }
    WCG_TRY(c.ekey.ensure((size_t)2 * cap * sizeof(long long)));
    WCG_TRY(c.edelta.ensure((size_t)2 * cap * sizeof(int)));
    WCG_TRY(c.ebucket.ensure((size_t)2 * cap * sizeof(int)));
    WCG_TRY(c.eperm.ensure((size_t)cap * sizeof(int)));
    WCG_TRY(c.estage.ensure((size_t)kNumECols * cap * sizeof(double)));
    c.ecap = cap;
  }
  c.ne = n;
  c.ecur = 0;
  c.have_grid = false;
  if (n == 0) return cudaSuccess;
  std::vector<double> h((size_t)kNumECols * n);
  auto col = [&](int k) { return h.data() + (size_t)k * n; };
  for (long long i = 0; i < n; ++i) {
    for (int a = 0; a < 4; ++a) {
      col(EX + a)[i] = x4[i * 4 + a];
      col(EVX + a)[i] = v4[i * 4 + a];
    }
    for (int q = 0; q < 9; ++q) col(EB00 + q)[i] = B9[i * 9 + q];
    for (int a = 0; a < 3; ++a) {
      col(EM0 + a)[i] = m4[i * 4 + a] + fm4[i * 4 + a];
      col(EOX + a)[i] = orient3[i * 3 + a];
    }
    col(ERV)[i] = rest_vol[i];
    col(ERF)[i] = rest_vf[i];
    col(EFV)[i] = fluid_vol[i];
    col(ESF)[i] = shape_factor[i];
    col(ESURF)[i] = surfel[i] ? 1.0 : 0.0;
  }
  double* st = c.estage.as<double>();
  WCG_TRY(cudaMemcpyAsync(st, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                          c.stream));
  if (c.prm.precision == 0)
    ++c.launches, k_load_elasto<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, st, c.ebuf[0].as<double>(), c.epid[0].as<int>());
  else
    ++c.launches, k_load_elasto<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, st, c.ebuf[0].as<float>(), c.epid[0].as<int>());
  WCG_TRY(cudaGetLastError());
  return cudaStreamSynchronize(c.stream);
}

cudaError_t download_elasto(Context& c, double* x4, double* v4, double* B9) {
  const long long n = c.ne;
  if (n == 0) return cudaSuccess;
  double* st = c.estage.as<double>();
  if (c.prm.precision == 0)
    ++c.launches, k_store_elasto<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, c.ebuf[c.ecur].as<double>(), c.epid[c.ecur].as<int>(), st, st + 4 * n,
        st + 8 * n);
  else
    ++c.launches, k_store_elasto<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, c.ebuf[c.ecur].as<float>(), c.epid[c.ecur].as<int>(), st, st + 4 * n,
        st + 8 * n);
  WCG_TRY(cudaGetLastError());
  if (x4) WCG_TRY(cudaMemcpyAsync(x4, st, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (v4)
    WCG_TRY(cudaMemcpyAsync(v4, st + 4 * n, n * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
  if (B9)
    WCG_TRY(cudaMemcpyAsync(B9, st + 8 * n, n * 9 * sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
  return cudaStreamSynchronize(c.stream);
}

cudaError_t upload_elasto_positions(Context& c, const double* x4) {
  const long long n = c.ne;
  if (n == 0) return cudaSuccess;
  double* st = c.estage.as<double>();
  WCG_TRY(cudaMemcpyAsync(st, x4, n * 4 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  if (c.prm.precision == 0)
    ++c.launches, k_set_elasto_positions<double><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, c.ebuf[c.ecur].as<double>(), c.epid[c.ecur].as<int>(), st);
  else
    ++c.launches, k_set_elasto_positions<float><<<nblk(n, 256), 256, 0, c.stream>>>(
        n, c.ecap, c.ebuf[c.ecur].as<float>(), c.epid[c.ecur].as<int>(), st);
  WCG_TRY(cudaGetLastError());
  c.have_grid = false;
  return cudaStreamSynchronize(c.stream);
}

// ---------------------------------------------------------------------------
// bounding box
template <typename R>
__global__ void k_minmax(const R* __restrict__ P, long long pcap, long long n,
                         double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double mn[3] = {1e20, 1e20, 1e20}, mx[3] = {-1e20, -1e20, -1e20};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    for (int a = 0; a < 3; ++a) {
      const double v = (double)P[(PX + a) * pcap + i];
      mn[a] = v < mn[a] ? v : mn[a];
      mx[a] = v > mx[a] ? v : mx[a];
    }
  for (int a = 0; a < 3; ++a) {
    const double lo = -block_max<double>(-mn[a], sm);
    const double hi = block_max<double>(mx[a], sm);
    if (threadIdx.x == 0) {
      partial[blockIdx.x * 6 + a] = lo;
      partial[blockIdx.x * 6 + 3 + a] = hi;
    }
  }
}

__global__ void k_minmax_final(const double* __restrict__ partial, int nb,
                               double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double r[6] = {1e20, 1e20, 1e20, -1e20, -1e20, -1e20};
  for (int b = 0; b < nb; ++b)
    for (int a = 0; a < 3; ++a) {
      r[a] = partial[b * 6 + a] < r[a] ? partial[b * 6 + a] : r[a];
      r[3 + a] = partial[b * 6 + 3 + a] > r[3 + a] ? partial[b * 6 + 3 + a] : r[3 + a];
    }
  for (int k = 0; k < 6; ++k) out[k] = r[k];
}

// max over particles of |v|^2 (TwoDScene::getMaxFluidVelocity :4180-4188)
template <typename R>
__global__ void k_maxvel2(const R* __restrict__ P, long long pcap, long long n,
                          double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double vx = P[VX * pcap + i], vy = P[VY * pcap + i], vz = P[VZ * pcap + i];
    const double s = (vx * vx + vy * vy) + vz * vz;
    m = s > m ? s : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

static cudaError_t ensure_scratch(Context& c, size_t bytes) {
  return c.scratch.ensure(std::max(bytes, (size_t)(kRedBlocks * 8 * sizeof(double))));
}

template <typename R>
static cudaError_t build_grid_t(Context& c) {
  ProfScope prof(c, P_GRID);
  c.xw_valid = false;  // the weights now follow the current positions
  const long long n = c.np;
  R* P = c.pbuf[c.cur].as<R>();
  WCG_TRY(ensure_scratch(c, (size_t)kRedBlocks * 12 * sizeof(double)));
  double* part = c.scratch.as<double>();
  double* dsc = c.dscalars.as<double>();
  const long long ne = c.ne;
  R* EP = ne > 0 ? c.ebuf[c.ecur].as<R>() : nullptr;
  // 1. bounding box over all particles, elasto included
  //    (TwoDScene::updateParticleBoundingBox :1588-1612)
  ++c.launches, k_minmax<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(P, c.pcap, n, part);
  if (ne > 0)
    ++c.launches, k_minmax<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(EP, c.ecap, ne,
                                                                      part + kRedBlocks * 6);
  ++c.launches, k_minmax_final<<<1, 32, 0, c.stream>>>(part, ne > 0 ? 2 * kRedBlocks : kRedBlocks,
                                                        dsc);
  WCG_TRY(read_small(c, dsc, 6 * sizeof(double), c.hscalars));
  double bbmin[3] = {1e20, 1e20, 1e20}, bbmax[3] = {-1e20, -1e20, -1e20};
  if (n + ne > 0)
    for (int a = 0; a < 3; ++a) {
      bbmin[a] = c.hscalars[a];
      bbmax[a] = c.hscalars[3 + a];
    }
  const double cell = c.prm.dx;
  const double bs = cell * 4.0;  // bucket size (numcells = 4)
  const double d2 = bs * 2.0;
  for (int a = 0; a < 3; ++a) {
    c.bbx_min[a] = std::floor(bbmin[a] / d2) * d2;
    c.bbx_max[a] = std::ceil(bbmax[a] / d2) * d2;
  }
  // 2. TwoDScene::rebucketizeParticles (:1657-1710)
  const double extra = 3.0;
  int nbk[3];
  double org[3];
  for (int a = 0; a < 3; ++a) {
    const double content = (c.bbx_max[a] - c.bbx_min[a]) + bs * extra * 2.0;
    const int cells = std::max(1, (int)std::ceil(content / cell));
    const double gsize = (double)cells * cell;
    org[a] = c.bbx_min[a] - bs * extra;
    nbk[a] = std::max(1, (int)std::ceil(gsize / bs));
  }
  GridDesc& g = c.g;
  g.ni = nbk[0]; g.nj = nbk[1]; g.nk = nbk[2];
  g.NI = g.ni * 4; g.NJ = g.nj * 4; g.NK = g.nk * 4;
  g.nb = (long long)g.ni * g.nj * g.nk;
  g.nnode = g.nb * 64;
  g.ox = org[0]; g.oy = org[1]; g.oz = org[2];
  g.bs = bs;
  g.dx = cell;
  c.have_grid = true;
  const int rb = c.real_bytes();
  // 3. storage
  if (g.nnode > c.gcap) {
    const long long cap = g.nnode + g.nnode / 8;
    WCG_TRY(c.gfield.ensure((size_t)kNumGFields * cap * rb));
    WCG_TRY(c.gvalid.ensure((size_t)6 * cap));
    WCG_TRY(c.gdof.ensure((size_t)cap));
    WCG_TRY(c.cell_start.ensure((size_t)(cap + 1) * sizeof(int)));
    WCG_TRY(c.cell_cursor.ensure((size_t)(cap + cap / 64 + 64) * sizeof(int)));
    if (c.prm.precision != 0) {
      WCG_TRY(c.rx64.ensure((size_t)cap * sizeof(double)));
      WCG_TRY(c.rr64.ensure((size_t)cap * sizeof(double)));
      WCG_TRY(c.rb64.ensure((size_t)cap * sizeof(double)));
    }
    c.gcap = cap;
  }
  if (ne > 0 && c.efcap < c.gcap) {
    WCG_TRY(c.efield.ensure((size_t)kNumEFields * c.gcap * rb));
    WCG_TRY(c.ecell_start.ensure((size_t)(c.gcap + 1) * sizeof(int)));
    c.efcap = c.gcap;
  }
  const long long bcap = c.gcap / 64 + 1;
  if ((size_t)bcap > c.active.bytes) {
    WCG_TRY(c.active_pre.ensure((size_t)bcap));
    WCG_TRY(c.active.ensure((size_t)bcap));
    WCG_TRY(c.active_list.ensure((size_t)bcap * sizeof(int)));
  }
  // wavefront tiles: 8x8x8 cells (2x2x2 buckets) or 8x4x8 (2x1x2)
  c.nti = (g.ni + 1) / 2;
  c.ntj = c.sweep_variant == 1 ? g.nj : (g.nj + 1) / 2;
  c.ntk = (g.nk + 1) / 2;
  const long long ntot = (long long)c.nti * c.ntj * c.ntk;
  if ((size_t)ntot * sizeof(int) > c.tile_flag.bytes) {
    const long long tcap = ntot + ntot / 4 + 64;
    WCG_TRY(c.tile_flag.ensure((size_t)tcap * sizeof(int)));
    WCG_TRY(cudaMemsetAsync(c.tile_flag.p, 0, c.tile_flag.bytes, c.stream));
    WCG_TRY(c.tile_active.ensure((size_t)tcap));
    WCG_TRY(c.wave_list.ensure((size_t)tcap * sizeof(int)));
    WCG_TRY(c.tile_part.ensure((size_t)tcap * sizeof(double)));
  }
  const int nwave = c.nti + c.ntj + c.ntk;
  WCG_TRY(c.wave_count.ensure((size_t)(2 * (nwave + 2)) * sizeof(int)));
  const long long scan_tiles = (std::max(g.nnode + 1, (long long)n) + kScanTile - 1) / kScanTile + 1;
  WCG_TRY(ensure_scratch(c, (size_t)scan_tiles * sizeof(long long) + 64));
  part = c.scratch.as<double>();
  // 4. particle pass
  int* drange = (int*)(dsc + 8);
  {
    int init[6] = {1 << 20, 1 << 20, 1 << 20, -(1 << 20), -(1 << 20), -(1 << 20)};
    WCG_TRY(cudaMemcpyAsync(drange, init, sizeof(init), cudaMemcpyHostToDevice, c.stream));
  }
  WCG_TRY(cudaMemsetAsync(c.active_pre.p, 0, g.nb, c.stream));
  int* cstart = c.cell_start.as<int>();
  WCG_TRY(cudaMemsetAsync(cstart, 0, (g.nnode + 1) * sizeof(int), c.stream));
  const int half = c.cur;
  long long* key_cur = c.pkey.as<long long>() + half * c.pcap;
  int* delta_cur = c.pdelta.as<int>() + half * c.pcap;
  int* pb_cur = c.pbucket.as<int>() + half * c.pcap;
  if (n > 0)
    ++c.launches, k_particle_prepass<R><<<nblk(n, 256), 256, 0, c.stream>>>(
        g, P, c.pcap, n, key_cur, delta_cur, pb_cur, c.active_pre.as<unsigned char>(),
        cstart, drange, c.derr.as<int>());
  int* ecstart = c.ecell_start.as<int>();
  long long* ekey_cur = c.ekey.as<long long>() + c.ecur * c.ecap;
  int* edelta_cur = c.edelta.as<int>() + c.ecur * c.ecap;
  if (ne > 0) {
    WCG_TRY(cudaMemsetAsync(ecstart, 0, (g.nnode + 1) * sizeof(int), c.stream));
    ++c.launches, k_particle_prepass<R><<<nblk(ne, 256), 256, 0, c.stream>>>(
        g, EP, c.ecap, ne, ekey_cur, edelta_cur, c.ebucket.as<int>() + c.ecur * c.ecap,
        c.active_pre.as<unsigned char>(), ecstart, drange, c.derr.as<int>(), EP + ESURF * c.ecap);
  }
  WCG_TRY(cudaGetLastError());
  // 5. dilation
  ++c.launches, k_dilate<<<nblk(g.nb, 256), 256, 0, c.stream>>>(g, c.active_pre.as<unsigned char>(),
                                                  c.active.as<unsigned char>());
  // 6. active list
  int* tmpi = c.cell_cursor.as<int>();
  ++c.launches, k_flag_to_int<<<nblk(g.nb, 256), 256, 0, c.stream>>>(c.active.as<unsigned char>(), g.nb, tmpi);
  int* dtotal = (int*)(dsc + 16);
  exclusive_scan<int, int>(tmpi, g.nb, tmpi, (int*)part, dtotal, c.stream);
  ++c.launches, k_compact<<<nblk(g.nb, 256), 256, 0, c.stream>>>(c.active.as<unsigned char>(), tmpi, g.nb,
                                                   c.active_list.as<int>());
  // tiles (2x2x2 buckets) with an active bucket, compacted into tile_part as ints
  int* ttmp = tmpi + g.nb + 1;
  int* tlist = (int*)c.tile_part.p;
  if (c.sweep_variant == 1)
    ++c.launches, k_wtile_active<<<nblk(ntot, 256), 256, 0, c.stream>>>(
        g, c.nti, c.ntj, c.ntk, c.active.as<unsigned char>(), c.tile_active.as<unsigned char>());
  else
    ++c.launches, k_tile_active<<<nblk(ntot, 256), 256, 0, c.stream>>>(
        g, c.nti, c.ntj, c.ntk, c.active.as<unsigned char>(), c.tile_active.as<unsigned char>());
  ++c.launches, k_flag_to_int<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      c.tile_active.as<unsigned char>(), ntot, ttmp);
  exclusive_scan<int, int>(ttmp, ntot, ttmp, (int*)part, dtotal + 1, c.stream);
  ++c.launches, k_compact<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      c.tile_active.as<unsigned char>(), ttmp, ntot, tlist);
  WCG_TRY(read_small(c, dsc + 8, 9 * sizeof(double), c.hscalars + 8));
  {
    const int* hr = (const int*)(c.hscalars + 8);
    c.n_active = *(const int*)(c.hscalars + 16);
    c.n_tiles = *((const int*)(c.hscalars + 16) + 1);
    c.stats.nactive = c.n_active;
    for (int k = 0; k < 6; ++k) c.drange_h[k] = n + ne > 0 ? hr[k] : (k < 3 ? 0 : 1);
  }
  // 7. wave ordering of the active tiles (ti+tj+tk)
  int* wcount = c.wave_count.as<int>();
  int* wcursor = wcount + (nwave + 2);
  WCG_TRY(cudaMemsetAsync(wcount, 0, (nwave + 2) * sizeof(int), c.stream));
  if (c.n_tiles > 0) {
    ++c.launches, k_tile_wave_count<<<nblk(c.n_tiles, 256), 256, 0, c.stream>>>(
        c.nti, c.ntj, tlist, c.n_tiles, wcount);
    exclusive_scan<int, int>(wcount, nwave + 1, wcursor, (int*)part, nullptr, c.stream);
    ++c.launches, k_tile_wave_scatter<<<nblk(c.n_tiles, 256), 256, 0, c.stream>>>(
        c.nti, c.ntj, tlist, c.n_tiles, wcursor, c.wave_list.as<int>());
  }
  // per-tile partials are indexed by tile id and reduced over all tiles in
  // index order (deterministic whatever order a wave's tiles were listed in)
  c.n_tiles_total = ntot;
  WCG_TRY(cudaMemsetAsync(c.tile_part.p, 0, ntot * sizeof(double), c.stream));
  // 8. counting sort by key node, deterministic within a cell
  exclusive_scan<int, int>(cstart, g.nnode, cstart, (int*)part, cstart + g.nnode, c.stream);
  WCG_TRY(cudaMemsetAsync(tmpi, 0, g.nnode * sizeof(int), c.stream));
  if (n > 0) {
    ++c.launches, k_sort_scatter<<<nblk(n, 256), 256, 0, c.stream>>>(key_cur, n, cstart, tmpi,
                                                       c.perm.as<int>());
    ++c.launches, k_sort_cells<<<nblk(g.nnode, 256), 256, 0, c.stream>>>(cstart, g.nnode,
                                                           c.pid[c.cur].as<int>(),
                                                           c.perm.as<int>());
    const int nxt = c.cur ^ 1;
    ++c.launches, k_gather_particles<R><<<nblk(n, 256), 256, 0, c.stream>>>(
        c.perm.as<int>(), n, c.pcap, P, c.pbuf[nxt].as<R>(), c.pid[c.cur].as<int>(),
        c.pid[nxt].as<int>(), key_cur, c.pkey.as<long long>() + nxt * c.pcap, delta_cur,
        c.pdelta.as<int>() + nxt * c.pcap, pb_cur, c.pbucket.as<int>() + nxt * c.pcap);
    c.cur = nxt;
  }
  // the same counting sort for the elasto particles
  if (ne > 0) {
    exclusive_scan<int, int>(ecstart, g.nnode, ecstart, (int*)part, ecstart + g.nnode, c.stream);
    WCG_TRY(cudaMemsetAsync(tmpi, 0, g.nnode * sizeof(int), c.stream));
    ++c.launches, k_sort_scatter<<<nblk(ne, 256), 256, 0, c.stream>>>(ekey_cur, ne, ecstart, tmpi,
                                                                     c.eperm.as<int>());
    ++c.launches, k_sort_cells<<<nblk(g.nnode, 256), 256, 0, c.stream>>>(
        ecstart, g.nnode, c.epid[c.ecur].as<int>(), c.eperm.as<int>());
    const int nxt = c.ecur ^ 1;
    ++c.launches, k_gather_elasto<R><<<nblk(ne, 256), 256, 0, c.stream>>>(
        c.eperm.as<int>(), ne, c.ecap, EP, c.ebuf[nxt].as<R>(), c.epid[c.ecur].as<int>(),
        c.epid[nxt].as<int>(), ekey_cur, c.ekey.as<long long>() + nxt * c.ecap, edelta_cur,
        c.edelta.as<int>() + nxt * c.ecap);
    // bucket indices move with their particles (host-side key listings)
    ++c.launches, k_permute_int<<<nblk(ne, 256), 256, 0, c.stream>>>(
        c.eperm.as<int>(), ne, c.ebucket.as<int>() + c.ecur * c.ecap,
        c.ebucket.as<int>() + nxt * c.ecap);
    c.ecur = nxt;
  }
  c.buckets_valid = true;
  WCG_TRY(cudaGetLastError());
  return cudaSuccess;
}

cudaError_t build_grid(Context& c) {
  return c.prm.precision == 0 ? build_grid_t<double>(c) : build_grid_t<float>(c);
}

// node fields of the elasto particles, or null for a liquid-only scene
template <typename R>
static R* elasto_fields(Context& c) {
  return c.ne > 0 && c.efcap >= c.gcap ? c.efield.as<R>() : nullptr;
}

// LiquidInfo::viscosity as the drag reads it: the liquid viscosity when the
// viscosity term is on, else the scene's drag viscosity (8.9e-3 by default)
static double drag_viscosity(const Context& c) {
  return c.prm.viscosity > 0.0 ? c.prm.viscosity : c.prm.drag_viscosity;
}

static Walls make_walls(const Context& c) {
  Walls w;
  w.cx = c.prm.box_center[0]; w.cy = c.prm.box_center[1]; w.cz = c.prm.box_center[2];
  w.ex = c.prm.box_half[0]; w.ey = c.prm.box_half[1]; w.ez = c.prm.box_half[2];
  w.radius = c.prm.box_radius;
  w.sign = -1.0;
  w.enabled = c.prm.walls;
  return w;
}

// The bucket-tile transfers (k_p2g_scatter + k_p2g_merge, k_g2p_tile) cover
// stencil offsets in {0, 1}, which is every particle inside the grid; anything
// else, or WCG_TRANSFERS=gather, takes the per-node gather P2G and the
// per-particle global G2P.
static bool tiled_transfers(const Context& c) {
  if (c.xfer_mode == 1) return false;
  for (int a = 0; a < 3; ++a)
    if (c.drange_h[a] < 0 || c.drange_h[3 + a] > 1) return false;
  return true;
}

template <typename R>
static cudaError_t map_particles_to_grid_t(Context& c) {
  if (c.n_active == 0) return cudaSuccess;
  ProfScope prof(c, P_P2G);
  DeltaRange dr;
  for (int a = 0; a < 3; ++a) {
    dr.lo[a] = c.drange_h[a];
    dr.hi[a] = c.drange_h[3 + a];
  }
  R* F = c.gfield.as<R>();
  const Walls w = make_walls(c);
  const bool elasto = c.ne > 0;
  if (tiled_transfers(c)) {
    constexpr int wpb = sizeof(R) == 4 ? 4 : 2;  // warps (buckets) per block: 43 KB of tiles
    WCG_TRY(c.p2g_halo.ensure((size_t)c.g.nb * kTileVals * sizeof(R)));
    ++c.launches, k_p2g_scatter<R, wpb><<<(unsigned)((c.n_active + wpb - 1) / wpb), 32 * wpb, 0,
                                          c.stream>>>(
        c.g, c.active_list.as<int>(), c.n_active, c.pbuf[c.cur].as<R>(), c.pcap,
        c.cell_start.as<int>(), c.pkey.as<long long>() + c.cur * c.pcap,
        c.pdelta.as<int>() + c.cur * c.pcap, c.p2g_halo.as<R>());
    // the merge writes the solid face weights too
    ++c.launches, k_p2g_merge<R><<<(unsigned)c.n_active, 256, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), c.cell_start.as<int>(),
        c.p2g_halo.as<R>(), F, c.gcap, w, elasto ? 1 : 0, c.np > 0 ? 1 : 0);
  } else {
    ++c.launches, k_p2g<R><<<(unsigned)c.n_active, 256, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), c.pbuf[c.cur].as<R>(),
        c.pcap, c.cell_start.as<int>(), c.pdelta.as<int>() + c.cur * c.pcap, dr, F, c.gcap, w,
        elasto ? 1 : 0, c.np > 0 ? 1 : 0);
  }
  // solid phase of the same P2G, sat/psi/pore pressure with elasto volumes;
  // LiquidInfo surf_tension_coeff 72.8, rest_contact_angle 40.8 deg,
  // pore_radius 0.005 (App/TwoDSceneXMLParser.cpp:1851-1904 defaults)
  if (elasto)
    ++c.launches, k_p2g_elasto<R><<<(unsigned)c.n_active, 256, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), c.ebuf[c.ecur].as<R>(), c.ecap,
        c.ecell_start.as<int>(), c.edelta.as<int>() + c.ecur * c.ecap, dr, F, c.gcap,
        c.efield.as<R>(), 72.8, std::cos(40.8 / 180.0 * M_PI), 0.005);
  if (!tiled_transfers(c))
    ++c.launches, k_solid_weights<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), F, c.gcap, w);
  // liquid volume fractions for the viscosity (updateLiquidPhi :3353-3367)
  if (c.prm.viscosity > 0.0 && c.np > 0)
    ++c.launches, k_volume_fractions<R><<<(unsigned)c.n_active, 64, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), F, c.gcap,
        c.prm.viscosity_implicit ? 7 : 4);
  return cudaGetLastError();
}

cudaError_t map_particles_to_grid(Context& c) {
  return c.prm.precision == 0 ? map_particles_to_grid_t<double>(c)
                              : map_particles_to_grid_t<float>(c);
}

static cudaError_t fetch(Context& c, const double* d, int k, double* h);

// One implicit viscosity sub-step on G_VSTAR (stepImplicitViscosityDiagonalPCG
// LinearizedImplicitEuler.cpp:2127-2172 with the PCG stop rule of
// robertbridson::PCGSolver::solve PCGSolver.h:261-330: ||r||_inf <=
// criterion ||b||_inf; the diagonal preconditions).  Device scalars 40-43:
// max |r|, p.q and rho (two slots).
template <typename R>
static cudaError_t viscosity_implicit_t(Context& c, double dt) {
  const unsigned nb = (unsigned)c.n_active;
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  R* F = c.gfield.as<R>();
  WCG_TRY(c.visc.ensure((size_t)kNumViscFields * c.gcap * sizeof(R)));
  WCG_TRY(c.viscflag.ensure((size_t)3 * c.gcap));
  WCG_TRY(ensure_scratch(c, (size_t)c.n_active * sizeof(double) + 64));
  double* part = c.scratch.as<double>();
  double* dsc = c.dscalars.as<double>();
  R* V = c.visc.as<R>();
  unsigned char* fl = c.viscflag.as<unsigned char>();
  const double dx = c.prm.dx;
  const R factor = (R)(dt / (dx * dx) * c.prm.viscosity / c.prm.liquid_density);
  const int kRmax = 40, kPq = 41, kRho0 = 42;
  ++c.launches, k_visc_flags<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap, make_walls(c), fl);
  ++c.launches, k_visc_rhs<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap, fl, factor, V, part);
  ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, (int)nb, dsc + kRmax);
  double bmax = 0;
  WCG_TRY(fetch(c, dsc + kRmax, 1, &bmax));
  c.stats.visc_iters = 0;
  c.stats.visc_residual = bmax;
  if (bmax < 1e-30) {
    ++c.launches, k_visc_writeback<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, F, 1);
    return cudaGetLastError();
  }
  const double tol = std::max(c.prm.viscosity_criterion, 1e-30) * bmax;
  int cur = 0;
  ++c.launches, k_visc_zdot<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, part);
  ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, (int)nb, dsc + kRho0);
  double rho = 0;
  WCG_TRY(fetch(c, dsc + kRho0, 1, &rho));
  if (rho == 0.0 || rho != rho) {
    c.stats.visc_converged = 0;
    return cudaSuccess;  // the reference stops the program here
  }
  ++c.launches, k_visc_dir<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, dsc, kRho0, kRho0, 1);
  bool done = false;
  double rmax = bmax;
  for (int it = 0; it < c.prm.maxiters && !done; ++it) {
    ++c.launches, k_visc_apply<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap, fl, factor,
                                                             V, part);
    ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, (int)nb, dsc + kPq);
    ++c.launches, k_visc_update<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, dsc,
                                                              kRho0 + cur, kPq, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, (int)nb, dsc + kRmax);
    WCG_TRY(fetch(c, dsc + kRmax, 1, &rmax));
    c.stats.visc_iters = it + 1;
    if (rmax <= tol) {
      done = true;
      break;
    }
    const int nxt = cur ^ 1;
    ++c.launches, k_visc_zdot<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, part);
    ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, (int)nb, dsc + kRho0 + nxt);
    ++c.launches, k_visc_dir<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, dsc, kRho0 + nxt,
                                                           kRho0 + cur, 0);
    cur = nxt;
  }
  c.stats.visc_residual = rmax;
  if (!done) c.stats.visc_converged = 0;
  ++c.launches, k_visc_writeback<R><<<nb, 192, 0, c.stream>>>(al, c.gcap, fl, V, F, 0);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t step_velocity_t(Context& c, double dt) {
  if (c.n_active == 0) return cudaSuccess;
  ProfScope prof(c, P_GRIDOPS);
  ++c.launches, k_predict<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
      c.g, c.active_list.as<int>(), c.gfield.as<R>(), c.gcap, (R)c.prm.gravity[0],
      (R)c.prm.gravity[1], (R)c.prm.gravity[2], (R)dt, elasto_fields<R>(c),
      c.active.as<unsigned char>(), drag_viscosity(c), c.prm.liquid_density);
  // viscosity sub-steps (explicit, or implicit solves), then rhs = v * m
  // (stepVelocity :272-306)
  if (c.prm.viscosity > 0.0) {
    R* F = c.gfield.as<R>();
    const int ns = c.prm.viscosity_substeps > 0 ? c.prm.viscosity_substeps : 1;
    const double sub_dt = dt / (double)ns;
    const double dx = c.prm.dx;
    const R factor = (R)(sub_dt / (dx * dx) * c.prm.viscosity / c.prm.liquid_density);
    c.stats.visc_converged = 1;
    for (int it = 0; it < ns; ++it) {
      if (c.prm.viscosity_implicit) {
        WCG_TRY(viscosity_implicit_t<R>(c, sub_dt));
        continue;
      }
      WCG_TRY(cudaMemcpyAsync(F + G_UTMP * c.gcap, F + G_VSTAR * c.gcap,
                              3 * c.gcap * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
      ++c.launches, k_viscosity_explicit<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
          c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), F, c.gcap, factor);
    }
    ++c.launches, k_rhs_from_vstar<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.active_list.as<int>(), F, c.gcap);
  }
  return cudaGetLastError();
}

cudaError_t step_velocity(Context& c, double dt) {
  return c.prm.precision == 0 ? step_velocity_t<double>(c, dt)
                              : step_velocity_t<float>(c, dt);
}

// ---------------------------------------------------------------------------
// PCG
template <typename R>
static SweepArgs<R> sweep_args(Context& c) {
  SweepArgs<R> a{};
  a.g = c.g;
  a.nti = c.nti;
  a.ntj = c.ntj;
  a.ntk = c.ntk;
  a.tile_list = c.wave_list.as<int>();
  a.ntiles = (int)c.n_tiles;
  a.ticket = c.ticket.as<int>();
  a.flags = c.tile_flag.as<int>();
  a.active = c.active.as<unsigned char>();
  a.tile_active = c.tile_active.as<unsigned char>();
  a.dof = c.gdof.as<unsigned char>();
  a.F = c.gfield.as<R>();
  a.fs = c.gcap;
  a.sc = c.dscalars.as<double>();
  a.omega = (R)0.97;
  a.min_ratio = (R)0.25;
  a.err = c.derr.as<int>();
  return a;
}

// one wavefront launch (factorisation, forward or backward sweep)
template <typename R>
static cudaError_t sweep(Context& c, int mode, SweepArgs<R> a) {
  if (c.n_tiles == 0) return cudaSuccess;
  ProfScope prof(c, mode == kFactor ? P_MICFACTOR : P_MICSWEEP);
  a.epoch = ++c.tile_epoch;
  WCG_TRY(cudaMemsetAsync(c.ticket.p, 0, sizeof(int), c.stream));
  const unsigned nt = (unsigned)c.n_tiles;
  if (c.sweep_variant == 1) {
    if (mode == kFactor) ++c.launches, k_wfactor<R><<<nt, 32, 0, c.stream>>>(a);
    else if (mode == kForward) ++c.launches, k_wsweep<R, kForward><<<nt, 32, 0, c.stream>>>(a);
    else ++c.launches, k_wsweep<R, kBackward><<<nt, 32, 0, c.stream>>>(a);
  } else {
    if (mode == kFactor) ++c.launches, k_sweep<R, kFactor><<<nt, kSweepThreads, 0, c.stream>>>(a);
    else if (mode == kForward) ++c.launches, k_sweep<R, kForward><<<nt, kSweepThreads, 0, c.stream>>>(a);
    else ++c.launches, k_sweep<R, kBackward><<<nt, kSweepThreads, 0, c.stream>>>(a);
  }
  return cudaGetLastError();
}

template <typename R>
static void dot(Context& c, const R* a, const R* b, double* out) {
  ProfScope prof(c, P_PCGVEC);
  const long long nent = c.n_active * 64;
  double* part = c.scratch.as<double>();
  ++c.launches, k_dot_partial<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
      c.active_list.as<int>(), nent, c.gdof.as<unsigned char>(), a, b, part);
  ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, out);
}

template <typename R>
static void absmax(Context& c, const R* a, double* out) {
  ProfScope prof(c, P_PCGVEC);
  const long long nent = c.n_active * 64;
  double* part = c.scratch.as<double>();
  ++c.launches, k_absmax_partial<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
      c.active_list.as<int>(), nent, c.gdof.as<unsigned char>(), a, part);
  ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, out);
}

static cudaError_t fetch(Context& c, const double* d, int k, double* h) {
  return read_small(c, d, (size_t)k * sizeof(double), h);
}

static cudaError_t set_scalars(Context& c, int slot, const double* v, int k) {
  return cudaMemcpyAsync(c.dscalars.as<double>() + slot, v, k * sizeof(double),
                         cudaMemcpyHostToDevice, c.stream);
}

// Inner MIC(0)-PCG (PCGSolver<T>::solve, PCGSolver.h:260-308) on the system
// already assembled and factored: solves A x = r0 from x = 0 (x must be zero
// on entry), r is overwritten with the residual.  tol_abs is the absolute
// infinity-norm target.  Convergence is tested on the device after every
// iteration; the host checks every c.pcg_batch iterations (the launches of a
// batch after convergence return at once, so results do not depend on it).
template <typename R>
static cudaError_t pcg_inner(Context& c, R* r, R* x, double tol_abs, int maxiters,
                             int* iters, int* conv, double* res) {
  R* F = c.gfield.as<R>();
  R* z = F + G_Z * c.gcap;
  R* s0 = F + G_S * c.gcap;
  R* s1 = F + G_S2 * c.gcap;
  R* q = F + G_Q * c.gcap;
  R* y = F + G_Y * c.gcap;
  double* sc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  double* tpart = c.tile_part.as<double>();
  const long long nent = c.n_active * 64;
  const int* al = c.active_list.as<int>();
  const unsigned char* dof = c.gdof.as<unsigned char>();
  *iters = 0;
  *conv = 0;
  *res = 0;
  if (maxiters <= 0) return cudaSuccess;
  {
    const double init[9] = {0.0, 0.0, 0.0, 0.0, 0.0, tol_abs, 0.0, (double)maxiters, 0.0};
    WCG_TRY(set_scalars(c, S_RHO, init, 9));  // clears S_DONE too
  }
  WCG_TRY(cudaMemsetAsync(s0, 0, c.gcap * sizeof(R), c.stream));
  WCG_TRY(cudaMemsetAsync(s1, 0, c.gcap * sizeof(R), c.stream));
  // z = M^-1 r, rho = z.r
  SweepArgs<R> fa = sweep_args<R>(c);
  fa.in = r;
  fa.out = y;
  fa.update = 0;
  fa.part = nullptr;
  WCG_TRY(sweep<R>(c, kForward, fa));
  SweepArgs<R> ba = sweep_args<R>(c);
  ba.in = y;
  ba.out = z;
  ba.r = r;
  ba.part = tpart;
  WCG_TRY(sweep<R>(c, kBackward, ba));
  {
    ProfScope prof(c, P_PCGVEC);
    ++c.launches, k_red_beta<<<1, kRedThreads, 0, c.stream>>>(tpart, (int)c.n_tiles_total, sc, 1);
  }
  double h[9];
  WCG_TRY(fetch(c, sc + S_RHO, 1, h));
  if (h[0] == 0 || h[0] != h[0]) return cudaSuccess;  // PCGSolver.h:276-279
  // forward sweeps with the fused x/r update
  fa.update = 1;
  fa.r = r;
  fa.x = x;
  fa.q = q;
  fa.part = tpart;
  R* sold = s0;
  R* snew = s1;
  for (;;) {
    for (int b = 0; b < c.pcg_batch; ++b) {
      {
        ProfScope prof(c, P_PCGVEC);
        ++c.launches, k_spmv_s<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
            c.g, al, nent, c.active.as<unsigned char>(), dof, F, c.gcap, z, sold, snew, q, sc,
            part);
        ++c.launches, k_red_alpha<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, sc);
      }
      fa.s = snew;
      WCG_TRY(sweep<R>(c, kForward, fa));
      {
        ProfScope prof(c, P_PCGVEC);
        ++c.launches, k_red_conv<<<1, kRedThreads, 0, c.stream>>>(tpart, (int)c.n_tiles_total, sc);
      }
      WCG_TRY(sweep<R>(c, kBackward, ba));
      {
        ProfScope prof(c, P_PCGVEC);
        ++c.launches, k_red_beta<<<1, kRedThreads, 0, c.stream>>>(tpart, (int)c.n_tiles_total, sc, 0);
      }
      R* t = sold;
      sold = snew;
      snew = t;
    }
    WCG_TRY(fetch(c, sc + S_RES, 6, h));  // res, beta, tol, iter, maxit, done
    const int done = *(const int*)&h[5];
    *res = h[0];
    *iters = (int)h[3];
    if (done) {
      *conv = done == 1 ? 1 : 0;
      break;
    }
  }
  return cudaGetLastError();
}

// FP64 residual r64 = b64 - A x64 with the (promoted) assembled coefficients
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_residual64(GridDesc g, const int* __restrict__ active_list, long long nent,
                 const unsigned char* __restrict__ active,
                 const unsigned char* __restrict__ dof, const R* __restrict__ F,
                 long long fstride, const double* __restrict__ b,
                 const double* __restrict__ x, double* __restrict__ r,
                 double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double m = 0;
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
    double acc = (double)AD[n] * x[n];
    if (I > 0) { const long long q = node_linear(g, I - 1, J, K); if (active[q >> 6] && dof[q]) acc += (double)AX[q] * x[q]; }
    if (J > 0) { const long long q = node_linear(g, I, J - 1, K); if (active[q >> 6] && dof[q]) acc += (double)AY[q] * x[q]; }
    if (K > 0) { const long long q = node_linear(g, I, J, K - 1); if (active[q >> 6] && dof[q]) acc += (double)AZ[q] * x[q]; }
    if (I + 1 < g.NI) { const long long q = node_linear(g, I + 1, J, K); if (active[q >> 6] && dof[q]) acc += (double)AX[n] * x[q]; }
    if (J + 1 < g.NJ) { const long long q = node_linear(g, I, J + 1, K); if (active[q >> 6] && dof[q]) acc += (double)AY[n] * x[q]; }
    if (K + 1 < g.NK) { const long long q = node_linear(g, I, J, K + 1); if (active[q >> 6] && dof[q]) acc += (double)AZ[n] * x[q]; }
    const double rv = b[n] - acc;
    r[n] = rv;
    const double av = fabs(rv);
    m = av > m ? av : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

template <typename R>
__global__ void k_promote(const int* __restrict__ active_list, long long nent,
                          const unsigned char* __restrict__ dof, const R* __restrict__ a,
                          double* __restrict__ o) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    o[n] = dof[n] ? (double)a[n] : 0.0;
  }
}

// r32 = r64 * scale; used to hand the FP64 residual to the FP32 inner solve
template <typename R>
__global__ void k_demote_scaled(const int* __restrict__ active_list, long long nent,
                                const unsigned char* __restrict__ dof,
                                const double* __restrict__ a, const double* __restrict__ sc,
                                R* __restrict__ o, R* __restrict__ x) {
  const double scale = 1.0 / sc[0];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    o[n] = dof[n] ? (R)(a[n] * scale) : R(0);
    x[n] = R(0);
  }
}

// x64 += e32 * norm
template <typename R>
__global__ void k_accumulate(const int* __restrict__ active_list, long long nent,
                             const unsigned char* __restrict__ dof,
                             const R* __restrict__ e32, const double* __restrict__ sc,
                             double* __restrict__ x) {
  const double s = sc[0];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    if (dof[n]) x[n] += (double)e32[n] * s;
  }
}

template <typename R>
__global__ void k_store_pressure(const int* __restrict__ active_list, long long nent,
                                 const unsigned char* __restrict__ dof,
                                 const R* __restrict__ x32, const double* __restrict__ x64,
                                 R* __restrict__ p) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    p[n] = dof[n] ? (x64 ? (R)x64[n] : x32[n]) : R(0);
  }
}

// ---------------------------------------------------------------------------
// Pressure solve in the pencil layout (wcg_pencil.cuh)

// Lay out the DOF box [lo, hi] (grid cells, inclusive) and allocate the arrays.
template <typename R>
static cudaError_t pl_setup(Context& c, const int* lo, const int* hi) {
  PencilGeom G{};
  int ext[3];
  for (int a = 0; a < 3; ++a) {
    G.lo[a] = lo[a];
    ext[a] = hi[a] - lo[a] + 1;
  }
  G.ax_s = 0;
  for (int a = 1; a < 3; ++a)
    if (ext[a] > ext[G.ax_s]) G.ax_s = a;
  G.ax_a = G.ax_s == 0 ? 1 : 0;
  G.ax_c = G.ax_s == 2 ? 1 : 2;
  G.Ls = ext[G.ax_s];
  G.NA = ext[G.ax_a];
  G.NC = ext[G.ax_c];
  G.nPA = (G.NA + kPatch - 1) / kPatch;
  G.nPC = (G.NC + kPatch - 1) / kPatch;
  G.R = G.Ls + 2 * (kPatch - 1);
  G.npatch = (long long)G.nPA * G.nPC;
  G.len = G.npatch * G.R * kPatchLines;
  const bool same_shape = c.plg.npatch == G.npatch && c.plg.nPA == G.nPA;
  c.plg = G;
  if (G.len > c.pl_cap) {
    c.pl_cap = G.len;
    WCG_TRY(c.pl.ensure((size_t)kNumPlFields * G.len * sizeof(R)));
    if (c.prm.precision != 0) WCG_TRY(c.pl64.ensure((size_t)kNumPl64Fields * G.len * sizeof(double)));
  }
  // edge words: 2 faces x Ls x 16 entries x (2 values x words per value)
  const size_t edge_bytes = (size_t)G.npatch * 2 * G.Ls * kPatch * 2 * (sizeof(R) / 4) * 8;
  if (edge_bytes > c.pl_edge.bytes) {
    WCG_TRY(c.pl_edge.ensure(edge_bytes));
    // tags of a fresh buffer must not match any epoch (epochs start at 1)
    WCG_TRY(cudaMemsetAsync(c.pl_edge.p, 0, c.pl_edge.bytes, c.stream));
  }
  WCG_TRY(c.pl_part.ensure(
      (size_t)std::max<long long>(G.npatch, std::max(kPlBlocks, kPlSpmvBlocks32)) * sizeof(double)));
  if (!same_shape || c.pl_order_h.size() != (size_t)G.npatch) {
    // patches in wave order PAi + PCi
    c.pl_order_h.resize(G.npatch);
    int k = 0;
    for (int w = 0; w <= G.nPA + G.nPC - 2; ++w)
      for (int pc = 0; pc < G.nPC; ++pc) {
        const int pa = w - pc;
        if (pa >= 0 && pa < G.nPA) c.pl_order_h[k++] = pc * G.nPA + pa;
      }
    WCG_TRY(c.pl_order.ensure((size_t)G.npatch * sizeof(int)));
    WCG_TRY(cudaMemcpyAsync(c.pl_order.p, c.pl_order_h.data(), G.npatch * sizeof(int),
                            cudaMemcpyHostToDevice, c.stream));
  }
  // The cluster's extent along c.  Chosen (sweep_cluster 0): a cluster that
  // tiles the patches along c exactly, so no CTA idles, at most 9 CTAs in
  // FP32 (two CTAs per SM fit) and 3 in FP64 (one per SM).  At 256^3 (9
  // patches along c, ms per sweep launch): FP32 plain 0.461, 3 0.436, 8
  // 0.423, 9 0.415, 16 0.521; FP64 plain 0.594, 3 0.550, 8 0.721, 9 0.638.
  // On small boxes they cost more than they save (the 64^3 dam break, 2
  // patches along c: 7.4 ms per step in 2-CTA clusters, 7.0 ms plain).
  // Given: used where the box has more patches along c than half a cluster.
  if (c.sweep_cluster == 0) {
    c.pl_cc = 1;
    const int fp32[] = {9, 8}, fp64[] = {3};
    const int* cand = c.prm.precision != 0 ? fp32 : fp64;
    const int ncand = c.prm.precision != 0 ? 2 : 1;
    if (G.nPC >= 6)
      for (int k = 0; k < ncand; ++k)
        if (G.nPC % cand[k] == 0) {
          c.pl_cc = cand[k];
          break;
        }
    if (c.pl_cc == 1 && c.prm.precision != 0 && G.nPC >= 6) c.pl_cc = 8;
  } else {
    c.pl_cc = G.nPC > c.sweep_cluster / 2 ? c.sweep_cluster : 1;
  }
  // the cluster orders are rebuilt only when the patch grid or the cluster
  // shape changes (a pageable upload waits for the stream)
  const long long okey = ((long long)G.nPA << 40) | ((long long)G.nPC << 16) |
                         ((long long)c.pl_cc << 8) | c.sweep_cluster_a;
  if (c.sweep_cluster_a > 1 && okey != c.pl_corder2_key) {
    // tiles of pl_cc c-patches by sweep_cluster_a a-patches, in wave order
    const int CC = c.pl_cc, CA = c.sweep_cluster_a;
    const int nTA = (G.nPA + CA - 1) / CA, nTC = (G.nPC + CC - 1) / CC;
    std::vector<int>& co = c.pl_corder2_h;
    co.clear();
    for (int w = 0; w <= nTA + nTC - 2; ++w)
      for (int tc = 0; tc < nTC; ++tc) {
        const int ta = w - tc;
        if (ta >= 0 && ta < nTA) co.push_back(tc * nTA + ta);
      }
    WCG_TRY(c.pl_corder2.ensure(co.size() * sizeof(int)));
    WCG_TRY(cudaMemcpyAsync(c.pl_corder2.p, co.data(), co.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c.stream));
    c.pl_corder2_key = okey;
  }
  if (c.pl_cc > 1 && okey != c.pl_corder_key) {
    // cluster columns (PAi, PCc) of pl_cc c-patches, in wave order
    const int CL = c.pl_cc;
    const int nPCc = (G.nPC + CL - 1) / CL;
    std::vector<int>& co = c.pl_corder_h;
    co.clear();
    for (int w = 0; w <= G.nPA + nPCc - 2; ++w)
      for (int pc = 0; pc < nPCc; ++pc) {
        const int pa = w - pc;
        if (pa >= 0 && pa < G.nPA) co.push_back(pc * G.nPA + pa);
      }
    WCG_TRY(c.pl_corder.ensure(co.size() * sizeof(int)));
    WCG_TRY(cudaMemcpyAsync(c.pl_corder.p, co.data(), co.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c.stream));
    c.pl_corder_key = okey;
  }
  // every array starts at zero (rows and lines outside the box stay zero)
  WCG_TRY(cudaMemsetAsync(c.pl.p, 0, (size_t)kNumPlFields * G.len * sizeof(R), c.stream));
  c.pl_tickets = 0;
  // the sweep ticket and the done counters of the SpMV and the sweeps
  WCG_TRY(cudaMemsetAsync(c.ticket.as<int>() + 1, 0, 3 * sizeof(int), c.stream));
  return cudaSuccess;
}

template <typename R>
static R* pl_field(Context& c, int f) {
  return c.pl.as<R>() + (size_t)f * c.plg.len;
}

template <typename R>
static PencilSweepArgs<R> pl_args(Context& c) {
  PencilSweepArgs<R> a{};
  a.G = c.plg;
  a.order = c.pl_order.as<int>();
  a.ticket = c.ticket.as<int>() + 1;
  a.edge = c.pl_edge.as<u64>();
  a.AD = pl_field<R>(c, PL_AD);
  a.AS = pl_field<R>(c, PL_AS);
  a.AA = pl_field<R>(c, PL_AA);
  a.AC = pl_field<R>(c, PL_AC);
  a.coef = pl_field<R>(c, PL_COEF);
  a.sc = c.dscalars.as<double>();
  a.omega = (R)0.97;
  a.min_ratio = (R)0.25;
  a.err = c.derr.as<int>();
  a.spin_limit = c.spin_limit;
  a.stale_patch = c.stale_patch < 0 ? -1 : (int)std::min<long long>(c.stale_patch,
                                                                     c.plg.npatch - 1);
  return a;
}

// dynamic shared memory a cluster sweep may use (the kernel's static
// arrays take under 8 KB of the 227 KB per CTA)
constexpr size_t kSweepSmemMax = 216 * 1024;

template <typename R, int MODE, bool UPD, int CC, int CA>
static cudaError_t pl_sweep_cl(Context& c, PencilSweepArgs<R> a) {
  constexpr int CL = CC * CA;
  ProfScope prof(c, MODE == kFactor ? P_MICFACTOR : P_MICSWEEP);
  const PencilGeom& G = c.plg;
  const int nTA = (G.nPA + CA - 1) / CA, nTC = (G.nPC + CC - 1) / CC;
  const int nunits = CL > 1 ? nTA * nTC : (int)G.npatch;
  a.epoch = (unsigned)(++c.tile_epoch);
  a.ticket_base = c.pl_tickets;
  c.pl_tickets += nunits;
  const size_t smem = CL > 1 ? sweep_cluster_smem<R>(MODE, UPD, G.Ls, CC, CA)
                             : sweep_dyn_smem<R>(MODE, UPD);
  // function attributes are per device: set once per instantiation and
  // device (the batch may step contexts of several devices from several
  // threads; setting them twice is harmless)
  static std::atomic<unsigned long long> attr_set{0};
  const unsigned long long dbit = 1ull << (c.device & 63);
  if (!(attr_set.load(std::memory_order_acquire) & dbit)) {
    WCG_TRY(cudaFuncSetAttribute(k_pencil_sweep<R, MODE, UPD, CC, CA>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(CL > 1 ? kSweepSmemMax : smem)));
    if (CL > 8)
      WCG_TRY(cudaFuncSetAttribute(k_pencil_sweep<R, MODE, UPD, CC, CA>,
                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr_set.fetch_or(dbit, std::memory_order_release);
  }
  if (CL == 1) {
    ++c.launches, k_pencil_sweep<R, MODE, UPD, 1, 1><<<(unsigned)G.npatch, kPatchLines, smem,
                                                       c.stream>>>(a);
    return cudaGetLastError();
  }
  a.order = CA > 1 ? c.pl_corder2.as<int>() : c.pl_corder.as<int>();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nunits * CL));
  cfg.blockDim = dim3(kPatchLines);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ++c.launches;
  return cudaLaunchKernelEx(&cfg, k_pencil_sweep<R, MODE, UPD, CC, CA>, a);
}

// The cluster forms need the edge buffers of a patch (Ls x 16 tagged entries
// per clustered face) in shared memory; when they do not fit, a 2-D cluster
// falls back to its c-clusters and those to the plain form.
template <typename R, int MODE, bool UPD>
static cudaError_t pl_sweep(Context& c, PencilSweepArgs<R> a) {
  const int CC = c.pl_cc, CA = c.sweep_cluster_a;
  const int Ls = c.plg.Ls;
  if (CA > 1 && sweep_cluster_smem<R>(MODE, UPD, Ls, CC, CA) <= kSweepSmemMax) {
    if (CC == 1 && CA == 4) return pl_sweep_cl<R, MODE, UPD, 1, 4>(c, a);
    if (CC == 1 && CA == 8) return pl_sweep_cl<R, MODE, UPD, 1, 8>(c, a);
    if (CC == 2 && CA == 4) return pl_sweep_cl<R, MODE, UPD, 2, 4>(c, a);
    if (CC == 2 && CA == 8) return pl_sweep_cl<R, MODE, UPD, 2, 8>(c, a);
    if (CC == 4 && CA == 4) return pl_sweep_cl<R, MODE, UPD, 4, 4>(c, a);
  }
  if (CC > 1 && sweep_cluster_smem<R>(MODE, UPD, Ls, CC, 1) <= kSweepSmemMax) {
    if (CC == 2) return pl_sweep_cl<R, MODE, UPD, 2, 1>(c, a);
    if (CC == 4) return pl_sweep_cl<R, MODE, UPD, 4, 1>(c, a);
    if (CC == 3) return pl_sweep_cl<R, MODE, UPD, 3, 1>(c, a);
    if (CC == 8) return pl_sweep_cl<R, MODE, UPD, 8, 1>(c, a);
    if (CC == 9) return pl_sweep_cl<R, MODE, UPD, 9, 1>(c, a);
    if (CC == 16) return pl_sweep_cl<R, MODE, UPD, 16, 1>(c, a);
  }
  return pl_sweep_cl<R, MODE, UPD, 1, 1>(c, a);
}

// ---------------------------------------------------------------------------
// The shared solve of a batch (no reference counterpart: the reference steps
// one scene per process).  Every context of a batch step that reaches the
// iterations of its pressure solve hands them to the batch's coordinator
// thread and waits; the coordinator runs the iterations of all waiting solves
// of one precision as one launch per kernel (SpMV, forward sweep, backward
// sweep), chunks of kSharedChunk iterations, reads every solve's status once
// per chunk, releases the converged ones and admits new ones between chunks.
// Each solve's arithmetic, block counts and partial sums are those it has
// alone, so results are bit-identical.

constexpr int kSharedChunk = 8;

struct SolveReq {
  Context* c = nullptr;
  int prec = 0;  // 0: FP64, 1: FP32
  PencilSweepArgs<double> fa64{}, ba64{};
  PencilSweepArgs<float> fa32{}, ba32{};
  PlSpmvArgs<double> sa64{};
  PlSpmvArgs<float> sa32{};
  int npatch = 0, nspmv = 0;
  int launched = 0;  // iterations launched so far
  bool finished = false;
  cudaError_t cerr = cudaSuccess;
  double status[6] = {};
};

struct SharedSolve {
  int device = 0;
  std::atomic<int> max_patches{INT_MAX};  // larger solves iterate alone
  cudaStream_t stream = nullptr;
  std::mutex m;
  std::condition_variable cv;       // the coordinator: requests or stop
  std::condition_variable cv_done;  // the requesters: a request finished
  std::vector<SolveReq*> queue, active;
  bool stop = false;
  std::thread th;
  DevBuf dtab;                    // argument tables, block offsets, status
  unsigned char* hpin = nullptr;  // their pinned host image
  size_t hpin_bytes = 0;
  std::atomic<long long> launches{0};
};

static size_t ss_align(size_t b) { return (b + 255) & ~(size_t)255; }

template <typename R>
static PencilSweepArgs<R>& ss_fa(SolveReq& q);
template <>
PencilSweepArgs<double>& ss_fa<double>(SolveReq& q) { return q.fa64; }
template <>
PencilSweepArgs<float>& ss_fa<float>(SolveReq& q) { return q.fa32; }
template <typename R>
static PencilSweepArgs<R>& ss_ba(SolveReq& q);
template <>
PencilSweepArgs<double>& ss_ba<double>(SolveReq& q) { return q.ba64; }
template <>
PencilSweepArgs<float>& ss_ba<float>(SolveReq& q) { return q.ba32; }
template <typename R>
static PlSpmvArgs<R>& ss_sa(SolveReq& q);
template <>
PlSpmvArgs<double>& ss_sa<double>(SolveReq& q) { return q.sa64; }
template <>
PlSpmvArgs<float>& ss_sa<float>(SolveReq& q) { return q.sa32; }

// One chunk of kSharedChunk iterations over the solves L (one precision).
template <typename R>
static cudaError_t ss_chunk(SharedSolve& S, const std::vector<SolveReq*>& L) {
  const int n = (int)L.size();
  const size_t o_sa = 0;
  const size_t o_fa = o_sa + ss_align(n * sizeof(PlSpmvArgs<R>));
  const size_t o_ba = o_fa + ss_align(n * sizeof(PencilSweepArgs<R>));
  const size_t o_f1 = o_ba + ss_align(n * sizeof(PencilSweepArgs<R>));
  const size_t o_f2 = o_f1 + ss_align((n + 1) * sizeof(int));
  const size_t o_sc = o_f2 + ss_align((n + 1) * sizeof(int));
  const size_t o_st = o_sc + ss_align(n * sizeof(double*));
  const size_t bytes = o_st + ss_align(6 * n * sizeof(double));
  WCG_TRY(S.dtab.ensure(bytes));
  if (bytes > S.hpin_bytes) {
    if (S.hpin) cudaFreeHost(S.hpin);
    S.hpin = nullptr;
    S.hpin_bytes = 0;
    WCG_TRY(cudaMallocHost((void**)&S.hpin, bytes));
    S.hpin_bytes = bytes;
  }
  auto* sa = reinterpret_cast<PlSpmvArgs<R>*>(S.hpin + o_sa);
  auto* fa = reinterpret_cast<PencilSweepArgs<R>*>(S.hpin + o_fa);
  auto* ba = reinterpret_cast<PencilSweepArgs<R>*>(S.hpin + o_ba);
  int* f1 = reinterpret_cast<int*>(S.hpin + o_f1);
  int* f2 = reinterpret_cast<int*>(S.hpin + o_f2);
  double** scs = reinterpret_cast<double**>(S.hpin + o_sc);
  long long n1 = 0, n2 = 0;
  for (int i = 0; i < n; ++i) {
    SolveReq& q = *L[(size_t)i];
    Context& c = *q.c;
    sa[i] = ss_sa<R>(q);
    sa[i].parity = q.launched & 1;
    fa[i] = ss_fa<R>(q);
    ba[i] = ss_ba<R>(q);
    // launch k of the chunk (forward 2b, backward 2b + 1) adds k to these
    fa[i].epoch = ba[i].epoch = (unsigned)(c.tile_epoch + 1);
    fa[i].ticket_base = ba[i].ticket_base = c.pl_tickets;
    f1[i] = (int)n1;
    f2[i] = (int)n2;
    n1 += q.nspmv;
    n2 += q.npatch;
    scs[i] = c.dscalars.as<double>();
  }
  if (n1 > INT_MAX || n2 > INT_MAX) return cudaErrorInvalidValue;
  f1[n] = (int)n1;
  f2[n] = (int)n2;
  unsigned char* d = S.dtab.as<unsigned char>();
  WCG_TRY(cudaMemcpyAsync(d, S.hpin, o_st, cudaMemcpyHostToDevice, S.stream));
  const auto* dsa = reinterpret_cast<const PlSpmvArgs<R>*>(d + o_sa);
  const auto* dfa = reinterpret_cast<const PencilSweepArgs<R>*>(d + o_fa);
  const auto* dba = reinterpret_cast<const PencilSweepArgs<R>*>(d + o_ba);
  const int* df1 = reinterpret_cast<const int*>(d + o_f1);
  const int* df2 = reinterpret_cast<const int*>(d + o_f2);
  double* const* dsc = reinterpret_cast<double* const*>(d + o_sc);
  double* dst = reinterpret_cast<double*>(d + o_st);
  const size_t smf = sweep_dyn_smem<R>(kForward, true), smb = sweep_dyn_smem<R>(kBackward, false);
  static std::atomic<unsigned long long> attr_set{0};
  const unsigned long long dbit = 1ull << (S.device & 63);
  if (!(attr_set.load(std::memory_order_acquire) & dbit)) {
    WCG_TRY(cudaFuncSetAttribute(k_pencil_sweep_batch<R, kForward, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
    WCG_TRY(cudaFuncSetAttribute(k_pencil_sweep_batch<R, kBackward, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb));
    attr_set.fetch_or(dbit, std::memory_order_release);
  }
  for (int b = 0; b < kSharedChunk; ++b) {
    k_pl_spmv_batch<R><<<(unsigned)n1, kRedThreads, 0, S.stream>>>(dsa, df1, n, b);
    k_pencil_sweep_batch<R, kForward, true><<<(unsigned)n2, kPatchLines, smf, S.stream>>>(
        dfa, df2, n, 2 * b);
    k_pencil_sweep_batch<R, kBackward, false><<<(unsigned)n2, kPatchLines, smb, S.stream>>>(
        dba, df2, n, 2 * b + 1);
  }
  k_pl_batch_status<<<(unsigned)((6 * n + 255) / 256), 256, 0, S.stream>>>(dsc, n, dst);
  WCG_TRY(cudaGetLastError());
  S.launches += 3 * kSharedChunk + 1;
  double* hst = reinterpret_cast<double*>(S.hpin + o_st);
  WCG_TRY(cudaMemcpyAsync(hst, dst, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  WCG_TRY(cudaStreamSynchronize(S.stream));
  for (int i = 0; i < n; ++i) {
    SolveReq& q = *L[(size_t)i];
    Context& c = *q.c;
    c.tile_epoch += 2 * kSharedChunk;
    c.pl_tickets += 2 * kSharedChunk * q.npatch;
    q.launched += kSharedChunk;
    std::memcpy(q.status, hst + 6 * i, sizeof(q.status));
  }
  return cudaSuccess;
}

static bool ss_done(const SolveReq& q) {
  int done = 0;
  std::memcpy(&done, &q.status[5], sizeof(int));
  return done != 0;
}

static void ss_loop(SharedSolve* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->m);
  for (;;) {
    S->cv.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->active.empty(); });
    if (S->active.empty() && S->queue.empty()) break;  // stop
    for (SolveReq* q : S->queue) {
      // the chunk's launches follow the solve's own work on its stream
      const cudaError_t e = cudaStreamWaitEvent(S->stream, q->c->ev_ss_ready, 0);
      if (e != cudaSuccess) q->cerr = e;
      S->active.push_back(q);
    }
    S->queue.clear();
    std::vector<SolveReq*> act = S->active;
    lk.unlock();
    std::vector<SolveReq*> L64, L32;
    for (SolveReq* q : act)
      if (q->cerr == cudaSuccess) (q->prec == 0 ? L64 : L32).push_back(q);
    cudaError_t e = cudaSuccess;
    if (!L64.empty()) e = ss_chunk<double>(*S, L64);
    if (e == cudaSuccess && !L32.empty()) e = ss_chunk<float>(*S, L32);
    lk.lock();
    std::vector<SolveReq*> keep;
    for (SolveReq* q : act) {
      if (e != cudaSuccess && q->cerr == cudaSuccess) q->cerr = e;
      if (q->cerr != cudaSuccess || ss_done(*q)) {
        // the solve's stream waits for its last iterations
        const cudaError_t r = cudaEventRecord(q->c->ev_ss_done, S->stream);
        if (r != cudaSuccess && q->cerr == cudaSuccess) q->cerr = r;
        q->finished = true;
      } else {
        keep.push_back(q);
      }
    }
    S->active.swap(keep);
    S->cv_done.notify_all();
  }
}

// Called by a context in its pressure solve: waits until the coordinator
// has run the solve's iterations to convergence (or the iteration limit).
static cudaError_t shared_solve_run(SharedSolve& S, SolveReq& q) {
  std::unique_lock<std::mutex> lk(S.m);
  S.queue.push_back(&q);
  S.cv.notify_one();
  S.cv_done.wait(lk, [&] { return q.finished; });
  return q.cerr;
}

SharedSolve* shared_solve_create(int device, std::string* err) {
  SharedSolve* S = new SharedSolve();
  S->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    if (err) *err = cudaGetErrorString(e);
    delete S;
    return nullptr;
  }
  S->th = std::thread(ss_loop, S);
  return S;
}

void shared_solve_destroy(SharedSolve* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->m);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->th.joinable()) S->th.join();
  cudaSetDevice(S->device);
  if (S->stream) {
    cudaStreamSynchronize(S->stream);
    cudaStreamDestroy(S->stream);
  }
  S->dtab.release();
  if (S->hpin) cudaFreeHost(S->hpin);
  delete S;
}

long long shared_solve_launches(const SharedSolve* S) { return S ? S->launches.load() : 0; }

void shared_solve_set_limit(SharedSolve* S, int max_patches) {
  if (S) S->max_patches = max_patches;
}

// PCGSolver<T>::solve (PCGSolver.h:260-308) in the pencil layout on the
// factored system: A x = r from x = 0; r is overwritten with the residual.
template <typename R>
static cudaError_t pl_pcg(Context& c, R* r, R* x, double tol_abs, int maxiters, int* iters,
                          int* conv, double* res) {
  const PencilGeom& G = c.plg;
  R* z = pl_field<R>(c, PL_Z);
  R* s0 = pl_field<R>(c, PL_S0);
  R* s1 = pl_field<R>(c, PL_S1);
  R* q = pl_field<R>(c, PL_Q);
  R* y = pl_field<R>(c, PL_Y);
  double* sc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  double* ppart = c.pl_part.as<double>();
  const int np = (int)G.npatch;
  *iters = 0;
  *conv = 0;
  *res = 0;
  if (maxiters <= 0) return cudaSuccess;
  {
    const double init[9] = {0.0, 0.0, 0.0, 0.0, 0.0, tol_abs, 0.0, (double)maxiters, 0.0};
    WCG_TRY(set_scalars(c, S_RHO, init, 9));  // clears S_DONE too
  }
  WCG_TRY(cudaMemsetAsync(s0, 0, G.len * sizeof(R), c.stream));
  // z = M^-1 r, rho = z.r
  PencilSweepArgs<R> fa = pl_args<R>(c);
  fa.in = r;
  fa.out = y;
  WCG_TRY((pl_sweep<R, kForward, false>(c, fa)));
  PencilSweepArgs<R> ba = pl_args<R>(c);
  ba.in = y;
  ba.out = z;
  ba.r = r;
  ba.part = ppart;
  // the sweeps' last CTAs reduce their partials (z.r and beta; max|r| and the
  // stop test), in place of separate reduction launches
  int* const done_ctr = c.ticket.as<int>() + 3;
  ba.done_ctr = done_ctr;
  ba.npart = np;
  ba.red_init = 1;
  WCG_TRY((pl_sweep<R, kBackward, false>(c, ba)));
  ba.red_init = 0;
  double h[9];
  WCG_TRY(fetch(c, sc + S_RHO, 1, h));
  if (h[0] == 0 || h[0] != h[0]) return cudaSuccess;  // PCGSolver.h:276-279
  fa.r = r;
  fa.q = q;
  fa.part = ppart;
  fa.done_ctr = done_ctr;
  fa.npart = np;
  R* sold = s0;
  R* snew = s1;
  const R* AD = pl_field<R>(c, PL_AD);
  const R* AS = pl_field<R>(c, PL_AS);
  const R* AA = pl_field<R>(c, PL_AA);
  const R* AC = pl_field<R>(c, PL_AC);
  // the streamed SpMV: chunks of consecutive rows of one patch per block,
  // about four blocks of resident capacity (kPlSpmvBlocks32) in all
  const int nchunk = (int)std::min<long long>(
      G.R, std::max<long long>(1, (4 * kPlSpmvBlocks32 + G.npatch - 1) / G.npatch));
  const int rows_per_chunk = (G.R + nchunk - 1) / nchunk;
  const int spmv_blocks = (int)(G.npatch * nchunk);
  const int rows_blocks = pl_spmv_blocks(G);
  WCG_TRY(ensure_scratch(c, (size_t)std::max(spmv_blocks, rows_blocks) * sizeof(double)));
  part = c.scratch.as<double>();
  if (c.shared_solve && c.spmv_rows && G.npatch <= c.shared_solve->max_patches.load()) {
    // the iterations run in the batch's shared launches
    SolveReq req;
    req.c = &c;
    req.prec = c.prm.precision == 0 ? 0 : 1;
    ss_fa<R>(req) = fa;
    ss_ba<R>(req) = ba;
    PlSpmvArgs<R>& sa = ss_sa<R>(req);
    sa.G = G;
    sa.AD = AD;
    sa.AS = AS;
    sa.AA = AA;
    sa.AC = AC;
    sa.z = z;
    sa.s0 = s0;
    sa.s1 = s1;
    sa.q = q;
    sa.x = x;
    sa.sc = sc;
    sa.part = part;
    sa.done_ctr = c.ticket.as<int>() + 2;
    req.npatch = (int)G.npatch;
    req.nspmv = rows_blocks;
    WCG_TRY(cudaEventRecord(c.ev_ss_ready, c.stream));
    WCG_TRY(shared_solve_run(*c.shared_solve, req));
    WCG_TRY(cudaStreamWaitEvent(c.stream, c.ev_ss_done, 0));
    int done = 0;
    std::memcpy(&done, &req.status[5], sizeof(int));
    *res = req.status[0];
    *iters = (int)req.status[3];
    *conv = done == 1 ? 1 : 0;
  } else {
  for (;;) {
    for (int b = 0; b < c.pcg_batch; ++b) {
      {
        ProfScope prof(c, P_PCGVEC);
        if (c.spmv_rows) {  // its last block forms alpha
          ++c.launches, k_pl_spmv_s<R><<<rows_blocks, kRedThreads, 0, c.stream>>>(
              G, AD, AS, AA, AC, z, sold, snew, q, x, sc, part, c.ticket.as<int>() + 2);
        } else {
          ++c.launches, k_pl_spmv_stream<R><<<spmv_blocks, kRedThreads, 0, c.stream>>>(
              G, rows_per_chunk, nchunk, AD, AS, AA, AC, z, sold, snew, q, x, sc, part);
          ++c.launches, k_red_alpha<<<1, kRedThreads, 0, c.stream>>>(part, spmv_blocks, sc);
        }
      }
      WCG_TRY((pl_sweep<R, kForward, true>(c, fa)));
      WCG_TRY((pl_sweep<R, kBackward, false>(c, ba)));
      R* t = sold;
      sold = snew;
      snew = t;
    }
    WCG_TRY(fetch(c, sc + S_RES, 6, h));  // res, beta, tol, iter, maxit, done
    const int done = *(const int*)&h[5];
    *res = h[0];
    *iters = (int)h[3];
    if (done) {
      *conv = done == 1 ? 1 : 0;
      break;
    }
  }
  }
  // x += alpha s of the last iteration (iteration i searched along s1 for even
  // i, s0 for odd i; later launches of the batch returned early)
  if (*iters > 0) {
    ProfScope prof(c, P_PCGVEC);
    const R* slast = ((*iters - 1) & 1) == 0 ? s1 : s0;
    ++c.launches, k_pl_axpy<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(G.len, sc, slast, x);
  }
  return cudaGetLastError();
}

// project_fine's solve in the pencil layout, from the assembled bucket-major
// system to the bucket-major pressure field.
template <typename R>
static cudaError_t pl_project(Context& c, double bnorm, const int* lo, const int* hi) {
  R* F = c.gfield.as<R>();
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  const unsigned char* dof = c.gdof.as<unsigned char>();
  const long long nent = c.n_active * 64;
  double* dsc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  const double tol = c.prm.criterion * bnorm;
  WCG_TRY(pl_setup<R>(c, lo, hi));
  const PencilGeom& G = c.plg;
  {
    ProfScope prof(c, P_PCGVEC);
    ++c.launches, k_pl_gather<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(
        G, c.g, act, dof, F, c.gcap, pl_field<R>(c, PL_AD), pl_field<R>(c, PL_AS),
        pl_field<R>(c, PL_AA), pl_field<R>(c, PL_AC), pl_field<R>(c, PL_B));
  }
  WCG_TRY(cudaGetLastError());
  // MIC(0) factor (PCGSolver::form_preconditioner)
  {
    const double zero = 0.0;
    WCG_TRY(set_scalars(c, S_DONE, &zero, 1));
  }
  WCG_TRY((pl_sweep<R, kFactor, false>(c, pl_args<R>(c))));
  R* r = pl_field<R>(c, PL_R);
  R* x = pl_field<R>(c, PL_X);
  const R* b = pl_field<R>(c, PL_B);
  R* pressure = F + G_PRESSURE * c.gcap;
  if (c.prm.precision == 0) {
    WCG_TRY(cudaMemcpyAsync(r, b, G.len * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
    int iters = 0, conv = 0;
    double res = bnorm;
    WCG_TRY(pl_pcg<R>(c, r, x, tol, c.prm.maxiters, &iters, &conv, &res));
    c.stats.pcg_iters = iters;
    c.stats.converged = conv;
    c.stats.residual = res;
    ++c.launches, k_pl_scatter_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
        G, c.g, al, nent, dof, x, nullptr, pressure);
    return cudaGetLastError();
  }
  // mixed precision: FP32 inner PCG, FP64 residual and solution
  double* x64 = c.pl64.as<double>() + (size_t)PL64_X * G.len;
  double* r64 = c.pl64.as<double>() + (size_t)PL64_R * G.len;
  WCG_TRY(cudaMemsetAsync(x64, 0, G.len * sizeof(double), c.stream));
  ++c.launches, k_pl_promote<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(G.len, b, r64);
  double res = bnorm;
  double h[1];
  int total = 0, k = 0;
  bool conv = false;
  const double inner_rel = c.prm.refine_inner_tol > 0 ? c.prm.refine_inner_tol : 0.0;
  for (k = 0; k <= c.prm.max_refinements; ++k) {
    if (res <= tol) {
      conv = true;
      break;
    }
    if (total >= c.prm.maxiters || k == c.prm.max_refinements) break;
    // scaled residual (||r32||_inf == 1) into r, x = 0
    WCG_TRY(cudaMemcpyAsync(dsc + 5, &res, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    {
      ProfScope prof(c, P_REFINE);
      ++c.launches, k_pl_demote<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(G.len, r64, dsc + 5, r, x);
    }
    const double want = std::max(inner_rel, 0.5 * tol / res);
    int iters = 0, ic = 0;
    double ires = 0;
    WCG_TRY(pl_pcg<R>(c, r, x, want, c.prm.maxiters - total, &iters, &ic, &ires));
    total += iters;
    part = c.scratch.as<double>();  // the inner solve may have grown the scratch buffer
    ProfScope prof3(c, P_REFINE);
    ++c.launches, k_pl_accumulate<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(G.len, x, dsc + 5, x64);
    ++c.launches, k_pl_residual64<R><<<kPlBlocks, kRedThreads, 0, c.stream>>>(
        G, pl_field<R>(c, PL_AD), pl_field<R>(c, PL_AS), pl_field<R>(c, PL_AA),
        pl_field<R>(c, PL_AC), b, x64, r64, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, kPlBlocks, dsc + 6);
    WCG_TRY(fetch(c, dsc + 6, 1, h));
    res = h[0];
    if (iters == 0) break;
  }
  c.stats.pcg_iters = total;
  c.stats.refinements = k;
  c.stats.converged = conv ? 1 : 0;
  c.stats.residual = res;
  ++c.launches, k_pl_scatter_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
      G, c.g, al, nent, dof, x, x64, pressure);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Multigrid-PCG (wcg_mg.cuh): AMGPCGSolveSparse, AlgebraicMultigrid.h:248-361

constexpr int kMgMaxLevels = 24;
constexpr int kMgPreSweeps = 4;      // amgVCycleCompressed: RBGS(.., 4)
constexpr int kMgCoarseSweeps = 200; // RBGS(.., 200) on the coarsest level
constexpr int kMgMaxCoarseDofs = 4096;

static int mg_blocks(long long n) {
  const long long b = (n + kMgThreads - 1) / kMgThreads;
  return (int)std::max<long long>(1, std::min<long long>(b, kMgBlocks));
}

template <typename R>
static MgLevel<R> mg_level(Context& c, int l) {
  const Context::MgDims& d = c.mg_dims[l];
  R* base = c.mg.as<R>() + d.off * 6;
  MgLevel<R> L;
  L.ni = d.ni; L.nj = d.nj; L.nk = d.nk; L.n = d.n;
  L.d = base;
  L.ax = base + d.n;
  L.ay = base + 2 * (long long)d.n;
  L.az = base + 3 * (long long)d.n;
  L.x = base + 4 * (long long)d.n;
  L.b = base + 5 * (long long)d.n;
  L.m = c.mg_mask.as<unsigned char>() + d.off;
  return L;
}

// Level 0 over the grid of cells; coarse levels while a level has more than
// 4096 DOFs (generateLevelsGalerkinCoarseningSparse, GeometricLevelGen.h:192-236).
// rhs receives the assembled rhs in the level-0 layout.
template <typename R>
static cudaError_t mg_setup(Context& c, long long ndof0) {
  const GridDesc& g = c.g;
  // dims of every possible level, then the allocation
  std::vector<Context::MgDims> dims;
  long long off = 0;
  int ni = g.NI, nj = g.NJ, nk = g.NK;
  for (int l = 0; l < kMgMaxLevels; ++l) {
    Context::MgDims d{ni, nj, nk, ni * nj * nk, off};
    dims.push_back(d);
    off += d.n;
    if (ni == 1 && nj == 1 && nk == 1) break;
    ni = (ni + 1) / 2; nj = (nj + 1) / 2; nk = (nk + 1) / 2;
  }
  WCG_TRY(c.mg.ensure((size_t)off * 6 * sizeof(R)));
  WCG_TRY(c.mg_mask.ensure((size_t)off));
  const long long n0 = dims[0].n;
  WCG_TRY(c.mg_vec.ensure((size_t)n0 * 5 * sizeof(R)));
  c.mg_dims = dims;
  R* F = c.gfield.as<R>();
  R* rhs = c.mg_vec.as<R>();
  MgLevel<R> L0 = mg_level<R>(c, 0);
  {
    ProfScope prof(c, P_PCGVEC);
    ++c.launches, k_mg_gather0<R><<<mg_blocks(n0), kMgThreads, 0, c.stream>>>(
        g, c.active.as<unsigned char>(), c.gdof.as<unsigned char>(), F, c.gcap, L0, rhs);
  }
  long long unknowns = ndof0;
  int nlev = 1;
  double* part = c.scratch.as<double>();
  double* dsc = c.dscalars.as<double>();
  while (unknowns > kMgMaxCoarseDofs && nlev < (int)dims.size()) {
    MgLevel<R> f = mg_level<R>(c, nlev - 1), cl = mg_level<R>(c, nlev);
    const int nb = std::min(mg_blocks(cl.n), kRedBlocks);
    {
      ProfScope prof(c, P_PCGVEC);
      ++c.launches, k_mg_coarsen<R><<<nb, kMgThreads, 0, c.stream>>>(f, cl, part);
      ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, nb, dsc + 7);
    }
    double h = 0;
    WCG_TRY(fetch(c, dsc + 7, 1, &h));
    unknowns = (long long)h;
    ++nlev;
    if (cl.ni == 1 && cl.nj == 1 && cl.nk == 1) break;
  }
  c.mg_dims.resize(nlev);
  return cudaGetLastError();
}

// z = one V-cycle from z = 0 on A z = r (amgPrecondCompressed /
// amgVCycleCompressed); r and z are level-0 vectors
template <typename R>
static cudaError_t mg_vcycle(Context& c, R* z, R* r) {
  ProfScope prof(c, P_MICSWEEP);
  const int nlev = (int)c.mg_dims.size();
  MgLevel<R> L[kMgMaxLevels];
  for (int l = 0; l < nlev; ++l) L[l] = mg_level<R>(c, l);
  L[0].x = z;
  L[0].b = r;
  WCG_TRY(cudaMemsetAsync(z, 0, (size_t)L[0].n * sizeof(R), c.stream));
  auto smooth = [&](int l, int sweeps) {
    const int nb = mg_blocks(L[l].n);
    for (int it = 0; it < sweeps; ++it) {
      ++c.launches, k_mg_smooth<R><<<nb, kMgThreads, 0, c.stream>>>(L[l], 1);
      ++c.launches, k_mg_smooth<R><<<nb, kMgThreads, 0, c.stream>>>(L[l], 0);
    }
  };
  for (int l = 0; l + 1 < nlev; ++l) {
    smooth(l, kMgPreSweeps);
    ++c.launches, k_mg_restrict<R><<<mg_blocks(L[l + 1].n), kMgThreads, 0, c.stream>>>(L[l], L[l + 1]);
  }
  ++c.launches, k_mg_coarsest<R><<<1, kMgCoarseThreads, 0, c.stream>>>(L[nlev - 1], kMgCoarseSweeps);
  for (int l = nlev - 2; l >= 0; --l) {
    ++c.launches, k_mg_prolong<R><<<mg_blocks(L[l].n), kMgThreads, 0, c.stream>>>(L[l + 1], L[l]);
    smooth(l, kMgPreSweeps);
  }
  return cudaGetLastError();
}

// AMGPCGSolveSparse's CG loop on level 0: A x = r from x = 0 (r is overwritten
// with the residual); stops when ||r||_inf <= tol_abs
template <typename R>
static cudaError_t mg_pcg(Context& c, R* r, R* x, double tol_abs, int maxiters, int* iters,
                          int* conv, double* res) {
  MgLevel<R> L0 = mg_level<R>(c, 0);
  const int n = L0.n;
  R* base = c.mg_vec.as<R>();
  R* s = base + 2 * (long long)n;
  R* q = base + 3 * (long long)n;
  R* z = base + 4 * (long long)n;
  double* sc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  const int nb = std::min(mg_blocks(n), kRedBlocks);
  *iters = 0;
  *conv = 0;
  *res = 0;
  if (maxiters <= 0) return cudaSuccess;
  {
    const double init[9] = {0.0, 0.0, 0.0, 0.0, 0.0, tol_abs, 0.0, (double)maxiters, 0.0};
    WCG_TRY(set_scalars(c, S_RHO, init, 9));
  }
  WCG_TRY(cudaMemsetAsync(x, 0, (size_t)n * sizeof(R), c.stream));
  WCG_TRY(mg_vcycle<R>(c, z, r));
  {
    ProfScope prof(c, P_PCGVEC);
    ++c.launches, k_mg_dot<R><<<nb, kMgThreads, 0, c.stream>>>(n, z, r, part);
    ++c.launches, k_red_beta<<<1, kRedThreads, 0, c.stream>>>(part, nb, sc, 1);
  }
  double h[6];
  WCG_TRY(fetch(c, sc + S_RHO, 1, h));
  if (h[0] == 0 || h[0] != h[0]) return cudaSuccess;  // AlgebraicMultigrid.h:301-314
  WCG_TRY(cudaMemcpyAsync(s, z, (size_t)n * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
  for (;;) {
    {
      ProfScope prof(c, P_PCGVEC);
      ++c.launches, k_mg_spmv<R><<<nb, kMgThreads, 0, c.stream>>>(L0, s, q, sc, part);
      ++c.launches, k_red_alpha<<<1, kRedThreads, 0, c.stream>>>(part, nb, sc);
      ++c.launches, k_mg_update<R><<<nb, kMgThreads, 0, c.stream>>>(n, s, q, x, r, sc, part);
      ++c.launches, k_red_conv<<<1, kRedThreads, 0, c.stream>>>(part, nb, sc);
    }
    WCG_TRY(fetch(c, sc + S_RES, 6, h));  // res, beta, tol, iter, maxit, done
    const int done = *(const int*)&h[5];
    *res = h[0];
    *iters = (int)h[3];
    if (done) {
      *conv = done == 1 ? 1 : 0;
      break;
    }
    WCG_TRY(mg_vcycle<R>(c, z, r));
    ProfScope prof(c, P_PCGVEC);
    ++c.launches, k_mg_dot<R><<<nb, kMgThreads, 0, c.stream>>>(n, z, r, part);
    ++c.launches, k_red_beta<<<1, kRedThreads, 0, c.stream>>>(part, nb, sc, 0);
    ++c.launches, k_mg_direction<R><<<nb, kMgThreads, 0, c.stream>>>(n, z, s, sc);
  }
  return cudaGetLastError();
}

// project_fine's solve with multigrid-PCG, from the assembled bucket-major
// system to the bucket-major pressure field
template <typename R>
static cudaError_t mg_project(Context& c, double bnorm) {
  R* F = c.gfield.as<R>();
  const int* al = c.active_list.as<int>();
  const unsigned char* dof = c.gdof.as<unsigned char>();
  const long long nent = c.n_active * 64;
  double* dsc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  const double tol = c.prm.criterion * bnorm;
  WCG_TRY(mg_setup<R>(c, c.stats.ndof));
  MgLevel<R> L0 = mg_level<R>(c, 0);
  const int n = L0.n;
  // level-0 vectors in mg_vec: rhs, r, s, q, z; the solution x takes the
  // level-0 b array, which the V-cycle does not use (its level-0 rhs is r)
  R* rhs = c.mg_vec.as<R>();
  R* r = rhs + n;
  R* x = L0.b;
  R* pressure = F + G_PRESSURE * c.gcap;
  const int nb = std::min(mg_blocks(n), kRedBlocks);
  if (c.prm.precision == 0) {
    WCG_TRY(cudaMemcpyAsync(r, rhs, (size_t)n * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
    int iters = 0, conv = 0;
    double res = bnorm;
    WCG_TRY(mg_pcg<R>(c, r, x, tol, c.prm.maxiters, &iters, &conv, &res));
    c.stats.pcg_iters = iters;
    c.stats.converged = conv;
    c.stats.residual = res;
    ++c.launches, k_mg_scatter_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
        c.g, al, nent, dof, x, nullptr, pressure);
    return cudaGetLastError();
  }
  // mixed precision: FP32 multigrid-PCG, FP64 residual and solution
  WCG_TRY(c.rx64.ensure((size_t)n * sizeof(double)));
  WCG_TRY(c.rr64.ensure((size_t)n * sizeof(double)));
  double* x64 = c.rx64.as<double>();
  double* r64 = c.rr64.as<double>();
  WCG_TRY(cudaMemsetAsync(x64, 0, (size_t)n * sizeof(double), c.stream));
  ++c.launches, k_pl_promote<R><<<nb, kMgThreads, 0, c.stream>>>(n, rhs, r64);
  double res = bnorm;
  double h[1];
  int total = 0, k = 0;
  bool conv = false;
  const double inner_rel = c.prm.refine_inner_tol > 0 ? c.prm.refine_inner_tol : 0.0;
  for (k = 0; k <= c.prm.max_refinements; ++k) {
    if (res <= tol) {
      conv = true;
      break;
    }
    if (total >= c.prm.maxiters || k == c.prm.max_refinements) break;
    WCG_TRY(cudaMemcpyAsync(dsc + 5, &res, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    {
      ProfScope prof(c, P_REFINE);
      ++c.launches, k_pl_demote<R><<<nb, kMgThreads, 0, c.stream>>>(n, r64, dsc + 5, r, x);
    }
    const double want = std::max(inner_rel, 0.5 * tol / res);
    int iters = 0, ic = 0;
    double ires = 0;
    WCG_TRY(mg_pcg<R>(c, r, x, want, c.prm.maxiters - total, &iters, &ic, &ires));
    total += iters;
    part = c.scratch.as<double>();  // the inner solve may have grown the scratch buffer
    ProfScope prof3(c, P_REFINE);
    ++c.launches, k_pl_accumulate<R><<<nb, kMgThreads, 0, c.stream>>>(n, x, dsc + 5, x64);
    ++c.launches, k_mg_residual64<R><<<nb, kMgThreads, 0, c.stream>>>(L0, rhs, x64, r64, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, nb, dsc + 6);
    WCG_TRY(fetch(c, dsc + 6, 1, h));
    res = h[0];
    if (iters == 0) break;
  }
  c.stats.pcg_iters = total;
  c.stats.refinements = k;
  c.stats.converged = conv ? 1 : 0;
  c.stats.residual = res;
  ++c.launches, k_mg_scatter_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
      c.g, al, nent, dof, x, x64, pressure);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t solve_assembled_t(Context& c);

template <typename R>
static cudaError_t project_fine_t(Context& c, double dt) {
  c.stats.pcg_iters = 0;
  c.stats.refinements = 0;
  c.stats.residual = 0;
  c.stats.rhs_norm = 0;
  c.stats.converged = 1;
  if (c.n_active == 0) return cudaSuccess;
  R* F = c.gfield.as<R>();
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  unsigned char* dof = c.gdof.as<unsigned char>();
  {
    ProfScope prof(c, P_GRIDOPS);
    ++c.launches, k_assemble<R><<<(unsigned)c.n_active, 64, 0, c.stream>>>(c.g, al, act, F, c.gcap, dof, (R)dt,
                                                                            elasto_fields<R>(c));
  }
  WCG_TRY(cudaGetLastError());
  return solve_assembled_t<R>(c);
}

// The pressure solve of projectFine on the system in the context's fields
// (G_ADIAG, G_AX/AY/AZ, DOF flags, rhs G_B, zero off the DOFs); the solution
// goes to G_PRESSURE.
template <typename R>
static cudaError_t solve_assembled_t(Context& c) {
  c.stats.pcg_iters = 0;
  c.stats.refinements = 0;
  c.stats.residual = 0;
  c.stats.rhs_norm = 0;
  c.stats.converged = 1;
  if (c.n_active == 0) return cudaSuccess;
  R* F = c.gfield.as<R>();
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  unsigned char* dof = c.gdof.as<unsigned char>();
  const long long nent = c.n_active * 64;
  double* dsc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  R* r = F + G_R * c.gcap;
  R* x = F + G_X * c.gcap;
  const R* b = F + G_B * c.gcap;
  double h[4];
  // ||b||_inf, the number of DOFs and their bounding box
  absmax<R>(c, b, dsc + 4);
  int* dbox = (int*)(dsc + 32);
  {
    ProfScope prof(c, P_PCGVEC);
    const int init[6] = {1 << 30, 1 << 30, 1 << 30, -1, -1, -1};
    WCG_TRY(cudaMemcpyAsync(dbox, init, sizeof(init), cudaMemcpyHostToDevice, c.stream));
    ++c.launches, k_dof_box<<<kRedBlocks, kRedThreads, 0, c.stream>>>(c.g, al, nent, dof, dbox, part);
    ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, dsc + 5);
  }
  WCG_TRY(read_small(c, dsc + 4, 31 * sizeof(double), c.hscalars + 4));
  h[0] = c.hscalars[4];
  h[1] = c.hscalars[5];
  int box[6];
  std::memcpy(box, c.hscalars + 32, sizeof(box));
  const double bnorm = h[0];
  c.stats.rhs_norm = bnorm;
  c.stats.ndof = (long long)h[1];
  if (bnorm < 1e-30) {
    // PCGSolver::solve returns x = 0 after zero iterations (PCGSolver.h:268-272)
    WCG_TRY(cudaMemsetAsync(F + G_PRESSURE * c.gcap, 0, c.gcap * sizeof(R), c.stream));
    return cudaGetLastError();
  }
  if (c.prm.solver == 1) return mg_project<R>(c, bnorm);
  if (c.pcg_layout == 0) return pl_project<R>(c, bnorm, box, box + 3);
  const double tol = c.prm.criterion * bnorm;
  // MIC(0) factor (PCGSolver::form_preconditioner)
  {
    const double zero = 0.0;
    WCG_TRY(set_scalars(c, S_DONE, &zero, 1));
  }
  WCG_TRY(sweep<R>(c, kFactor, sweep_args<R>(c)));
  WCG_TRY(cudaMemsetAsync(x, 0, c.gcap * sizeof(R), c.stream));
  if (c.prm.precision == 0) {
    {
      ProfScope prof(c, P_PCGVEC);
      ++c.launches, k_copy_dof<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, b, r);
    }
    int iters = 0, conv = 0;
    double res = bnorm;
    WCG_TRY(pcg_inner<R>(c, r, x, tol, c.prm.maxiters, &iters, &conv, &res));
    c.stats.pcg_iters = iters;
    c.stats.converged = conv;
    c.stats.residual = res;
    ++c.launches, k_store_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, x, nullptr,
                                                                  F + G_PRESSURE * c.gcap);
    return cudaGetLastError();
  }
  // mixed precision: FP32 inner PCG, FP64 residual and solution
  double* x64 = c.rx64.as<double>();
  double* r64 = c.rr64.as<double>();
  double* b64 = c.rb64.as<double>();
  WCG_TRY(cudaMemsetAsync(x64, 0, c.gcap * sizeof(double), c.stream));
  ++c.launches, k_promote<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, b, b64);
  ++c.launches, k_promote<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, b, r64);
  double res = bnorm;
  int total = 0, k = 0;
  bool conv = false;
  // inner target: the remaining factor to the final tolerance (or a fixed
  // relative reduction when refine_inner_tol > 0)
  const double inner_rel = c.prm.refine_inner_tol > 0 ? c.prm.refine_inner_tol : 0.0;
  for (k = 0; k <= c.prm.max_refinements; ++k) {
    if (res <= tol) {
      conv = true;
      break;
    }
    if (total >= c.prm.maxiters || k == c.prm.max_refinements) break;
    // scaled residual (||r32||_inf == 1) into r, x = 0
    WCG_TRY(cudaMemcpyAsync(dsc + 5, &res, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    {
      ProfScope prof(c, P_REFINE);
      ++c.launches, k_demote_scaled<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
          al, nent, dof, r64, dsc + 5, r, x);
    }
    const double want = std::max(inner_rel, 0.5 * tol / res);
    int iters = 0, ic = 0;
    double ires = 0;
    WCG_TRY(pcg_inner<R>(c, r, x, want, c.prm.maxiters - total, &iters, &ic, &ires));
    total += iters;
    part = c.scratch.as<double>();  // the inner solve may have grown the scratch buffer
    ProfScope prof3(c, P_REFINE);
    ++c.launches, k_accumulate<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, x, dsc + 5, x64);
    ++c.launches, k_residual64<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
        c.g, al, nent, act, dof, F, c.gcap, b64, x64, r64, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, dsc + 6);
    WCG_TRY(fetch(c, dsc + 6, 1, h));
    res = h[0];
    if (iters == 0) break;
  }
  c.stats.pcg_iters = total;
  c.stats.refinements = k;
  c.stats.converged = conv ? 1 : 0;
  c.stats.residual = res;
  ++c.launches, k_store_pressure<R><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, x, x64,
                                                                F + G_PRESSURE * c.gcap);
  return cudaGetLastError();
}

cudaError_t project_fine(Context& c, double dt) {
  return c.prm.precision == 0 ? project_fine_t<double>(c, dt) : project_fine_t<float>(c, dt);
}

template <typename R>
static cudaError_t apply_pressure_t(Context& c, double dt) {
  if (c.n_active == 0) return cudaSuccess;
  ProfScope prof(c, P_GRIDOPS);
  R* F = c.gfield.as<R>();
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  unsigned char* valid = c.gvalid.as<unsigned char>();
  unsigned char* vtmp = valid + 3 * c.gcap;
  ++c.launches, k_apply_pressure<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap,
                                                                  valid, (R)dt, elasto_fields<R>(c));
  R* U = F + G_U * c.gcap;
  R* UT = F + G_UTMP * c.gcap;
  ++c.launches, k_extrapolate<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(c.g, al, act, U, UT, valid,
                                                               vtmp, c.gcap);
  ++c.launches, k_extrapolate<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(c.g, al, act, UT, U, vtmp,
                                                               valid, c.gcap);
  return cudaGetLastError();
}

cudaError_t apply_pressure_and_extrapolate(Context& c, double dt) {
  return c.prm.precision == 0 ? apply_pressure_t<double>(c, dt)
                              : apply_pressure_t<float>(c, dt);
}

cudaError_t constrain_liquid_velocity(Context& c) {
  if (c.n_active == 0) return cudaSuccess;
  ProfScope prof(c, P_GRIDOPS);
  if (c.prm.precision == 0)
    ++c.launches, k_constrain<double><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.active_list.as<int>(), c.gfield.as<double>(), c.gcap,
        c.prm.liquid_boundary_friction);
  else
    ++c.launches, k_constrain<float><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.active_list.as<int>(), c.gfield.as<float>(), c.gcap,
        (float)c.prm.liquid_boundary_friction);
  return cudaGetLastError();
}

template <typename R>
static void elasto_g2p_t(Context& c, double dt, bool g2p, bool advect) {
  ++c.launches, k_g2p_elasto<R><<<nblk(c.ne, 128), 128, 0, c.stream>>>(
      c.g, c.active.as<unsigned char>(), c.ebuf[c.ecur].as<R>(), c.ecap, c.ne,
      c.ekey.as<long long>() + c.ecur * c.ecap, c.edelta.as<int>() + c.ecur * c.ecap,
      c.efield.as<R>(), c.gcap, (R)c.prm.elasto_flip, (R)c.prm.elasto_flip_asym,
      (R)c.prm.elasto_advect, (R)dt, g2p ? 1 : 0, advect ? 1 : 0);
}

template <typename R>
static cudaError_t g2p_t(Context& c, double dt, bool advect) {
  if (c.np + c.ne == 0) return cudaSuccess;
  ProfScope prof(c, P_G2P);
  if (c.np > 0) {
    if (tiled_transfers(c))
      ++c.launches, k_g2p_tile<R><<<(unsigned)c.n_active, 128, 0, c.stream>>>(
          c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), c.pbuf[c.cur].as<R>(),
          c.pcap, c.cell_start.as<int>(), c.pkey.as<long long>() + c.cur * c.pcap,
          c.pdelta.as<int>() + c.cur * c.pcap, c.gfield.as<R>(), c.gcap, (R)c.prm.flip_coeff,
          (R)dt, advect ? 1 : 0, c.xw_valid ? c.xw.as<R>() : nullptr);
    else
      ++c.launches, k_g2p<R><<<nblk(c.np, 128), 128, 0, c.stream>>>(
          c.g, c.active.as<unsigned char>(), c.pbuf[c.cur].as<R>(), c.pcap, c.np,
          c.pkey.as<long long>() + c.cur * c.pcap, c.pdelta.as<int>() + c.cur * c.pcap,
          c.gfield.as<R>(), c.gcap, (R)c.prm.flip_coeff, (R)dt, advect ? 1 : 0,
          c.xw_valid ? c.xw.as<R>() : nullptr);
  }
  if (c.ne > 0) elasto_g2p_t<R>(c, dt, true, advect);
  return cudaGetLastError();
}

cudaError_t map_grid_to_particles_and_advect(Context& c, double dt, bool advect) {
  return c.prm.precision == 0 ? g2p_t<double>(c, dt, advect) : g2p_t<float>(c, dt, advect);
}

template <typename R>
static void advect_liquid_t(Context& c, double dt) {
  ++c.launches, k_advect<R><<<nblk(c.np, 128), 128, 0, c.stream>>>(
      c.g, c.active.as<unsigned char>(), c.pbuf[c.cur].as<R>(), c.pcap, c.np,
      c.pkey.as<long long>() + c.cur * c.pcap, c.pdelta.as<int>() + c.cur * c.pcap,
      c.gfield.as<R>(), c.gcap, (R)dt, c.xw_valid ? c.xw.as<R>() : nullptr);
}

cudaError_t advect_only(Context& c, double dt) {
  if (c.np + c.ne == 0) return cudaSuccess;
  ProfScope prof(c, P_G2P);
  if (c.np > 0) {
    if (c.prm.precision == 0)
      advect_liquid_t<double>(c, dt);
    else
      advect_liquid_t<float>(c, dt);
  }
  if (c.ne > 0) {
    if (c.prm.precision == 0)
      elasto_g2p_t<double>(c, dt, false, true);
    else
      elasto_g2p_t<float>(c, dt, false, true);
  }
  return cudaGetLastError();
}

// WetClothCore::stepSystem sub-stepping (WetClothCore.cpp:50-62)
cudaError_t num_substeps(Context& c, double dt, int* n) {
  WCG_TRY(ensure_scratch(c, 0));
  ProfScope prof(c, P_OTHER);
  double* part = c.scratch.as<double>();
  double* dsc = c.dscalars.as<double>();
  if (c.np > 0) {
    if (c.prm.precision == 0)
      ++c.launches, k_maxvel2<double><<<kRedBlocks, kRedThreads, 0, c.stream>>>(c.pbuf[c.cur].as<double>(),
                                                                 c.pcap, c.np, part);
    else
      ++c.launches, k_maxvel2<float><<<kRedBlocks, kRedThreads, 0, c.stream>>>(c.pbuf[c.cur].as<float>(),
                                                                c.pcap, c.np, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, dsc + 7);
  } else {
    WCG_TRY(cudaMemsetAsync(dsc + 7, 0, sizeof(double), c.stream));
  }
  double h;
  WCG_TRY(fetch(c, dsc + 7, 1, &h));
  const double max_fluid_vel = std::sqrt(h);
  double he = 0.0;
  if (c.ne > 0) {
    if (c.prm.precision == 0)
      ++c.launches, k_maxvel2_elasto<double><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
          c.ebuf[c.ecur].as<double>(), c.ecap, c.ne, part);
    else
      ++c.launches, k_maxvel2_elasto<float><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
          c.ebuf[c.ecur].as<float>(), c.ecap, c.ne, part);
    ++c.launches, k_reduce_max<<<1, kRedThreads, 0, c.stream>>>(part, kRedBlocks, dsc + 7);
    WCG_TRY(fetch(c, dsc + 7, 1, &he));
  }
  const double max_elasto_vel = std::sqrt(he);
  const double cell = c.prm.dx;
  const double max_elasto_dt = std::min(cell / std::max(1e-63, max_elasto_vel) / 3.0, 1.0 / 30.0);
  const double max_fluid_dt = std::min(cell / std::max(1e-63, max_fluid_vel) * 3.0, 1.0 / 30.0);
  const double max_dt = std::min(max_elasto_dt, max_fluid_dt);
  *n = std::max(1, (int)std::ceil(dt / max_dt));
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Solve of a caller-assembled system on a context whose buffers were set up
// by the caller (used by the allocation-free entry point in wcg_noalloc.cu).
// Every bucket counts as active; the DOF mask selects the unknowns.  FP64,
// the same MIC(0)-PCG as project_fine.
cudaError_t prepared_solve_fp64(Context& c, double* out, int* iters, double* res,
                                int* converged, double* rhs_norm) {
  const GridDesc& g = c.g;
  double* F = c.gfield.as<double>();
  double* dsc = c.dscalars.as<double>();
  double* part = c.scratch.as<double>();
  int* tmpi = c.cell_cursor.as<int>();
  unsigned char* act = c.active.as<unsigned char>();
  *iters = 0;
  *res = 0;
  *converged = 1;
  *rhs_norm = 0;
  // all buckets active, list = 0..nb-1
  WCG_TRY(cudaMemsetAsync(act, 1, g.nb, c.stream));
  ++c.launches, k_flag_to_int<<<nblk(g.nb, 256), 256, 0, c.stream>>>(act, g.nb, tmpi);
  exclusive_scan<int, int>(tmpi, g.nb, tmpi, (int*)part, (int*)(dsc + 16), c.stream);
  ++c.launches, k_compact<<<nblk(g.nb, 256), 256, 0, c.stream>>>(act, tmpi, g.nb,
                                                                 c.active_list.as<int>());
  c.n_active = g.nb;
  // wavefront tiles (8x8x8 cells) ordered by wave
  c.sweep_variant = 0;
  c.nti = (g.ni + 1) / 2;
  c.ntj = (g.nj + 1) / 2;
  c.ntk = (g.nk + 1) / 2;
  const long long ntot = (long long)c.nti * c.ntj * c.ntk;
  const int nwave = c.nti + c.ntj + c.ntk;
  int* ttmp = tmpi + g.nb + 1;
  int* tlist = (int*)c.tile_part.p;
  ++c.launches, k_tile_active<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      g, c.nti, c.ntj, c.ntk, act, c.tile_active.as<unsigned char>());
  ++c.launches, k_flag_to_int<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      c.tile_active.as<unsigned char>(), ntot, ttmp);
  exclusive_scan<int, int>(ttmp, ntot, ttmp, (int*)part, (int*)(dsc + 16) + 1, c.stream);
  ++c.launches, k_compact<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      c.tile_active.as<unsigned char>(), ttmp, ntot, tlist);
  int* wcount = c.wave_count.as<int>();
  int* wcursor = wcount + (nwave + 2);
  WCG_TRY(cudaMemsetAsync(wcount, 0, (nwave + 2) * sizeof(int), c.stream));
  ++c.launches, k_tile_wave_count<<<nblk(ntot, 256), 256, 0, c.stream>>>(c.nti, c.ntj, tlist,
                                                                         ntot, wcount);
  exclusive_scan<int, int>(wcount, nwave + 1, wcursor, (int*)part, nullptr, c.stream);
  ++c.launches, k_tile_wave_scatter<<<nblk(ntot, 256), 256, 0, c.stream>>>(
      c.nti, c.ntj, tlist, ntot, wcursor, c.wave_list.as<int>());
  c.n_tiles = ntot;
  c.n_tiles_total = ntot;
  WCG_TRY(cudaMemsetAsync(c.tile_part.p, 0, ntot * sizeof(double), c.stream));
  WCG_TRY(cudaGetLastError());
  // the solve (project_fine_t minus assembly)
  const int* al = c.active_list.as<int>();
  const unsigned char* dof = c.gdof.as<unsigned char>();
  const long long nent = c.n_active * 64;
  double h[2];
  absmax<double>(c, F + G_B * c.gcap, dsc + 4);
  WCG_TRY(fetch(c, dsc + 4, 1, h));
  const double bnorm = h[0];
  *rhs_norm = bnorm;
  if (bnorm < 1e-30) {
    WCG_TRY(cudaMemsetAsync(out, 0, g.nnode * sizeof(double), c.stream));
    return cudaStreamSynchronize(c.stream);
  }
  {
    const double zero = 0.0;
    WCG_TRY(set_scalars(c, S_DONE, &zero, 1));
  }
  WCG_TRY(sweep<double>(c, kFactor, sweep_args<double>(c)));
  double* r = F + G_R * c.gcap;
  double* x = F + G_X * c.gcap;
  WCG_TRY(cudaMemsetAsync(x, 0, g.nnode * sizeof(double), c.stream));
  ++c.launches, k_copy_dof<double><<<kRedBlocks, kRedThreads, 0, c.stream>>>(
      al, nent, dof, F + G_B * c.gcap, r);
  int conv = 0;
  WCG_TRY(pcg_inner<double>(c, r, x, c.prm.criterion * bnorm, c.prm.maxiters, iters, &conv, res));
  *converged = conv;
  ++c.launches, k_copy_dof<double><<<kRedBlocks, kRedThreads, 0, c.stream>>>(al, nent, dof, x, out);
  WCG_TRY(cudaGetLastError());
  return cudaStreamSynchronize(c.stream);
}

template <typename R>
static cudaError_t substep_vjp_t(Context& c, double dt, const double* vbar, const double* Cbar,
                                 const double* xbar, double* vbar0, double* Cbar0,
                                 double* xbar0, double* mubar) {
  const long long np = c.np;
  const int rb = c.real_bytes();
  const bool visc = c.prm.viscosity > 0.0;
  const int ns = visc ? std::max(1, c.prm.viscosity_substeps) : 0;
  if (mubar) *mubar = 0.0;
  // forward recompute at the checkpoint: grid, fields, matrix, masks (the
  // particle state is not touched); with the viscosity, the velocity before
  // each explicit sub-step is kept for the reverse pass
  WCG_TRY(build_grid(c));
  WCG_TRY(map_particles_to_grid(c));
  const R factor = visc ? (R)(dt / ns / (c.prm.dx * c.prm.dx) * c.prm.viscosity /
                              c.prm.liquid_density)
                        : R(0);
  if (!visc) {
    WCG_TRY(step_velocity(c, dt));
  } else if (c.n_active > 0) {
    R* F = c.gfield.as<R>();
    WCG_TRY(c.adjvisc.ensure((size_t)(ns + 1) * 3 * c.gcap * rb));
    R* VK = c.adjvisc.as<R>();
    ++c.launches, k_predict<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.g, c.active_list.as<int>(), F, c.gcap, (R)c.prm.gravity[0], (R)c.prm.gravity[1],
        (R)c.prm.gravity[2], (R)dt, elasto_fields<R>(c), c.active.as<unsigned char>(),
        drag_viscosity(c), c.prm.liquid_density);
    for (int it = 0; it < ns; ++it) {
      WCG_TRY(cudaMemcpyAsync(VK + (size_t)it * 3 * c.gcap, F + G_VSTAR * c.gcap,
                              3 * c.gcap * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
      WCG_TRY(cudaMemcpyAsync(F + G_UTMP * c.gcap, F + G_VSTAR * c.gcap, 3 * c.gcap * sizeof(R),
                              cudaMemcpyDeviceToDevice, c.stream));
      ++c.launches, k_viscosity_explicit<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
          c.g, c.active_list.as<int>(), c.active.as<unsigned char>(), F, c.gcap, factor);
    }
    WCG_TRY(cudaMemcpyAsync(VK + (size_t)ns * 3 * c.gcap, F + G_VSTAR * c.gcap,
                            3 * c.gcap * sizeof(R), cudaMemcpyDeviceToDevice, c.stream));
    ++c.launches, k_rhs_from_vstar<R><<<(unsigned)c.n_active, 192, 0, c.stream>>>(
        c.active_list.as<int>(), F, c.gcap);
  }
  WCG_TRY(project_fine(c, dt));
  WCG_TRY(apply_pressure_and_extrapolate(c, dt));
  if (np == 0 || c.n_active == 0) {
    std::fill(vbar0, vbar0 + 3 * np, 0.0);
    std::fill(Cbar0, Cbar0 + 9 * np, 0.0);
    if (xbar0) std::copy(xbar, xbar + 3 * np, xbar0);
    return cudaSuccess;
  }
  WCG_TRY(c.adj.ensure((size_t)kNumAdjFields * c.gcap * rb));
  WCG_TRY(c.adjmask.ensure((size_t)3 * c.gcap));
  WCG_TRY(c.adjp.ensure((size_t)15 * c.pcap * rb));  // B (12 columns), XB (3)
  WCG_TRY(c.adjstage.ensure((size_t)18 * np * sizeof(double)));
  double* st = c.adjstage.as<double>();
  WCG_TRY(cudaMemcpyAsync(st, vbar, 3 * np * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  WCG_TRY(cudaMemcpyAsync(st + 3 * np, Cbar, 9 * np * sizeof(double), cudaMemcpyHostToDevice,
                          c.stream));
  WCG_TRY(cudaMemcpyAsync(st + 12 * np, xbar, 3 * np * sizeof(double), cudaMemcpyHostToDevice,
                          c.stream));
  R* F = c.gfield.as<R>();
  R* AG = c.adj.as<R>();
  R* B = c.adjp.as<R>();
  R* XB = xbar0 ? B + 12 * c.pcap : nullptr;
  const int* al = c.active_list.as<int>();
  const unsigned char* act = c.active.as<unsigned char>();
  const unsigned char* dof = c.gdof.as<unsigned char>();
  unsigned char* vtmp = c.gvalid.as<unsigned char>() + 3 * c.gcap;  // layer-1 output mask
  unsigned char* v0 = c.adjmask.as<unsigned char>();
  const unsigned nb = (unsigned)c.n_active;
  DeltaRange dr;
  for (int a = 0; a < 3; ++a) {
    dr.lo[a] = c.drange_h[a];
    dr.hi[a] = c.drange_h[3 + a];
  }
  // the positions G2P and the advection see: the particle correction of this
  // sub-step (the next selector of the seeded stream; at strength 0 only its
  // projection out of the solid) on the recomputed grid, into XC, the
  // particle state restored after it
  const R* XC = nullptr;
  {
    R* P = c.pbuf[c.cur].as<R>();
    const int sel = correction_selector(c.prm.correction_seed, c.corr_count,
                                        c.prm.correction_step);
    WCG_TRY(correct_liquid_particles(c, dt, sel));  // x -> xw, P positions -> x_c
    WCG_TRY(c.adjxc.ensure((size_t)3 * c.pcap * rb));
    WCG_TRY(cudaMemcpyAsync(c.adjxc.p, P + PX * c.pcap, 3 * c.pcap * sizeof(R),
                            cudaMemcpyDeviceToDevice, c.stream));
    WCG_TRY(cudaMemcpyAsync(P + PX * c.pcap, c.xw.p, 3 * c.pcap * sizeof(R),
                            cudaMemcpyDeviceToDevice, c.stream));
    c.xw_valid = false;
    XC = c.adjxc.as<R>();
  }
  ++c.launches, k_adj_load<R><<<nblk(np, 128), 128, 0, c.stream>>>(
      c.g, act, c.pbuf[c.cur].as<R>(), c.pcap, np, c.pkey.as<long long>() + c.cur * c.pcap,
      c.pdelta.as<int>() + c.cur * c.pcap, F, c.gcap, (R)c.prm.flip_coeff,
      (R)c.prm.liquid_boundary_friction, c.pid[c.cur].as<int>(), st, st + 3 * np,
      st + 12 * np, dt, B, XC, XB);
  ++c.launches, k_adj_g2p<R><<<nb, 192, 0, c.stream>>>(
      c.g, al, c.pbuf[c.cur].as<R>(), c.pcap, c.cell_start.as<int>(),
      c.pdelta.as<int>() + c.cur * c.pcap, dr, B, F, c.gcap, AG, (R)c.prm.flip_coeff,
      (R)c.prm.liquid_boundary_friction, XC);
  // extrapolation layers in reverse: layer 2 read the layer-1 output mask,
  // layer 1 the validity after the pressure gradient
  ++c.launches, k_adj_extrapolate<R><<<nb, 192, 0, c.stream>>>(
      c.g, al, act, AG + A_UBAR * c.gcap, AG + A_UTMP * c.gcap, vtmp, c.gcap);
  ++c.launches, k_adj_valid0<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap, v0);
  ++c.launches, k_adj_extrapolate<R><<<nb, 192, 0, c.stream>>>(
      c.g, al, act, AG + A_UTMP * c.gcap, AG + A_UBAR * c.gcap, v0, c.gcap);
  ++c.launches, k_adj_apply<R><<<nb, 64, 0, c.stream>>>(c.g, al, act, dof, AG, F, c.gcap, (R)dt);
  WCG_TRY(cudaGetLastError());
  if (xbar0)  // the forward pressure, for the ghost-fluid fractions' part
    WCG_TRY(cudaMemcpyAsync(AG + A_PF * c.gcap, F + G_PRESSURE * c.gcap, c.gcap * sizeof(R),
                            cudaMemcpyDeviceToDevice, c.stream));
  WCG_TRY(solve_assembled_t<R>(c));  // A lambda = p-bar, A symmetric
  int* AM = nullptr;
  if (xbar0) {
    WCG_TRY(c.adjam.ensure((size_t)c.gcap * sizeof(int)));
    AM = c.adjam.as<int>();
    ++c.launches, k_adj_theta<R><<<nb, 64, 0, c.stream>>>(
        c.g, al, act, dof, F, c.gcap, AG, (R)dt, c.pbuf[c.cur].as<R>(), c.pcap,
        c.cell_start.as<int>(), make_walls(c), c.np > 0 ? 1 : 0, AM);
  }
  ++c.launches, k_adj_div<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, dof, F, c.gcap, AG,
                                                        visc ? 1 : 0);
  if (visc) {
    // explicit viscosity steps in reverse: mu-bar += <v-bar_{k+1}, v_{k+1} - v_k> / mu,
    // v-bar_k = v-bar_{k+1} + f K^T v-bar_{k+1}
    const R* VK = c.adjvisc.as<R>();
    WCG_TRY(ensure_scratch(c, (size_t)c.n_active * sizeof(double) + 64));
    double* part = c.scratch.as<double>();
    double* dsc = c.dscalars.as<double>();
    double musum = 0.0;
    R* cur = AG + A_VSBAR * c.gcap;
    R* tmp = AG + A_UTMP * c.gcap;
    for (int it = ns - 1; it >= 0; --it) {
      ++c.launches, k_adj_mu_dot<R><<<nb, 192, 0, c.stream>>>(
          al, cur, VK + (size_t)(it + 1) * 3 * c.gcap, VK + (size_t)it * 3 * c.gcap, c.gcap, part);
      ++c.launches, k_reduce_sum<<<1, kRedThreads, 0, c.stream>>>(part, (int)c.n_active, dsc + 7);
      double h = 0;
      WCG_TRY(fetch(c, dsc + 7, 1, &h));
      musum += h;
      ++c.launches, k_adj_viscosity<R><<<nb, 192, 0, c.stream>>>(c.g, al, act, F, c.gcap, cur, tmp,
                                                                  factor);
      std::swap(cur, tmp);
    }
    if (cur != AG + A_VSBAR * c.gcap)
      WCG_TRY(cudaMemcpyAsync(AG + A_VSBAR * c.gcap, cur, 3 * c.gcap * sizeof(R),
                              cudaMemcpyDeviceToDevice, c.stream));
    if (mubar) *mubar = musum / c.prm.viscosity;
  }
  ++c.launches, k_adj_p2g<R><<<nblk(np, 128), 128, 0, c.stream>>>(
      c.g, act, c.pbuf[c.cur].as<R>(), c.pcap, np, c.pid[c.cur].as<int>(),
      c.pkey.as<long long>() + c.cur * c.pcap, c.pdelta.as<int>() + c.cur * c.pcap, F, AG,
      c.gcap, st, st + 3 * np, XB, st + 15 * np, AM);
  WCG_TRY(cudaGetLastError());
  WCG_TRY(cudaMemcpyAsync(vbar0, st, 3 * np * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  WCG_TRY(cudaMemcpyAsync(Cbar0, st + 3 * np, 9 * np * sizeof(double), cudaMemcpyDeviceToHost,
                          c.stream));
  if (xbar0)
    WCG_TRY(cudaMemcpyAsync(xbar0, st + 15 * np, 3 * np * sizeof(double),
                            cudaMemcpyDeviceToHost, c.stream));
  return cudaStreamSynchronize(c.stream);
}

cudaError_t substep_vjp(Context& c, double dt, const double* vbar, const double* Cbar,
                        const double* xbar, double* vbar0, double* Cbar0, double* xbar0,
                        double* mubar) {
  return c.prm.precision == 0
             ? substep_vjp_t<double>(c, dt, vbar, Cbar, xbar, vbar0, Cbar0, xbar0, mubar)
             : substep_vjp_t<float>(c, dt, vbar, Cbar, xbar, vbar0, Cbar0, xbar0, mubar);
}

int correction_selector(unsigned long long seed, unsigned long long k, int step) {
  return (int)(splitmix64(seed ^ splitmix64(k)) % (unsigned long long)(step > 0 ? step : 1));
}

template <typename R>
static cudaError_t correct_liquid_t(Context& c, double dt, int selector) {
  const long long n = c.np;
  if (n == 0 || c.n_active == 0) return cudaSuccess;
  ProfScope prof(c, P_OTHER);
  R* P = c.pbuf[c.cur].as<R>();
  // positions before the correction: G2P keeps their weights
  WCG_TRY(c.xw.ensure((size_t)3 * c.pcap * sizeof(R)));
  if (!(c.prm.correction_strength > 0.0)) {
    // strength 0: the selected particles are only projected out of the solid
    const int step = c.prm.correction_step > 0 ? c.prm.correction_step : 1;
    ++c.launches, k_correct_project<R><<<nblk(n, 256), 256, 0, c.stream>>>(
        c.g, P, c.pcap, n, c.pid[c.cur].as<int>(), c.pkey.as<long long>() + c.cur * c.pcap,
        c.pdelta.as<int>() + c.cur * c.pcap, c.active.as<unsigned char>(), c.gfield.as<R>(),
        c.gcap, c.xw.as<R>(), selector, step);
    c.xw_valid = true;
    return cudaGetLastError();
  }
  WCG_TRY(cudaMemcpyAsync(c.xw.p, P + PX * c.pcap, 3 * c.pcap * sizeof(R),
                          cudaMemcpyDeviceToDevice, c.stream));
  c.xw_valid = true;
  // the cells of rebucketizeParticles (grid_num_cells, TwoDScene.cpp:1662-1669)
  CellGrid cg;
  const double org[3] = {c.g.ox, c.g.oy, c.g.oz};
  long long ncell = 1;
  for (int a = 0; a < 3; ++a) {
    const double content = (c.bbx_max[a] - c.bbx_min[a]) + c.g.bs * 3.0 * 2.0;
    cg.n[a] = std::max(1, (int)std::ceil(content / c.prm.dx));
    cg.org[a] = org[a];
    ncell *= cg.n[a];
  }
  cg.dx = c.prm.dx;
  WCG_TRY(c.corr_start.ensure((size_t)(ncell + 1) * sizeof(int)));
  WCG_TRY(c.corr_cursor.ensure((size_t)ncell * sizeof(int)));
  WCG_TRY(c.corr_list.ensure((size_t)n * sizeof(int)));
  const long long scan_tiles = (std::max(ncell + 1, n) + kScanTile - 1) / kScanTile + 1;
  WCG_TRY(ensure_scratch(c, (size_t)scan_tiles * sizeof(long long) + 64));
  int* start = c.corr_start.as<int>();
  int* cursor = c.corr_cursor.as<int>();
  int* list = c.corr_list.as<int>();
  long long* cell = c.pkey.as<long long>() + (c.cur ^ 1) * c.pcap;  // free half
  const int* pid = c.pid[c.cur].as<int>();
  WCG_TRY(cudaMemsetAsync(start, 0, (size_t)(ncell + 1) * sizeof(int), c.stream));
  WCG_TRY(cudaMemsetAsync(cursor, 0, (size_t)ncell * sizeof(int), c.stream));
  ++c.launches, k_corr_cells<R><<<nblk(n, 256), 256, 0, c.stream>>>(P, c.pcap, n, cg, cell, start);
  exclusive_scan<int, int>(start, ncell, start, c.scratch.as<int>(), start + ncell, c.stream);
  ++c.launches, k_sort_scatter<<<nblk(n, 256), 256, 0, c.stream>>>(cell, n, start, cursor, list);
  ++c.launches, k_sort_cells<<<nblk(ncell, 256), 256, 0, c.stream>>>(start, ncell, pid, list);
  const long long ncol = (long long)((cg.n[0] + 1) / 2) * ((cg.n[1] + 1) / 2) * ((cg.n[2] + 1) / 2);
  const int step = c.prm.correction_step > 0 ? c.prm.correction_step : 1;
  for (int t = 0; t < 2; ++t)
    for (int u = 0; u < 2; ++u)
      for (int r = 0; r < 2; ++r)
        ++c.launches, k_correct<R><<<nblk(ncol, 128), 128, 0, c.stream>>>(
            c.g, cg, r, u, t, P, c.pcap, pid, list, start,
            c.pkey.as<long long>() + c.cur * c.pcap, c.pdelta.as<int>() + c.cur * c.pcap,
            c.active.as<unsigned char>(), c.gfield.as<R>(), c.gcap, c.xw.as<R>(), selector, step,
            (R)(c.prm.correction_strength / dt), (R)c.prm.correction_multiplier, (R)dt);
  return cudaGetLastError();
}

cudaError_t correct_liquid_particles(Context& c, double dt, int selector) {
  return c.prm.precision == 0 ? correct_liquid_t<double>(c, dt, selector)
                              : correct_liquid_t<float>(c, dt, selector);
}

void merge_draws(unsigned long long seed, unsigned long long k, int step, int* selector,
                 int* perm) {
  unsigned long long z = splitmix64(seed ^ splitmix64(k ^ 0x6d657267652d6b65ull));
  *selector = (int)(z % (unsigned long long)(step > 0 ? step : 1));
  for (int q = 0; q < 3; ++q) {
    int* pq = perm + 3 * q;
    pq[0] = 0;
    pq[1] = 1;
    pq[2] = 2;
    for (int i = 2; i >= 1; --i) {  // mathutils::fisherYates (MathUtilities.h:238-245)
      z = splitmix64(z);
      const int j = (int)(z % (unsigned long long)(i + 1));
      const int t = pq[i];
      pq[i] = pq[j];
      pq[j] = t;
    }
  }
}

// removeEmptyParticles (TwoDScene.cpp:1713-1745) on flagged slots: alive_slot
// holds 0/1 per slot (scanned in place here), alive_pid the same per original
// index; hole_rank, high_rank and holes take n ints each, corr_cursor and
// corr_list n each.  The holes below K (the survivor count) take the
// survivors at K and above in descending order; the slots are compacted and
// the original indices renumbered.
template <typename R>
static cudaError_t remove_flagged_t(Context& c, long long n, int* alive_slot, int* alive_pid,
                                    int* hole_rank, int* high_rank, int* holes,
                                    long long* removed) {
  const long long cap = c.pcap;
  R* P = c.pbuf[c.cur].as<R>();
  const int* pid = c.pid[c.cur].as<int>();
  const int* pb = c.pbucket.as<int>() + c.cur * c.pcap;
  int* cursor = c.corr_cursor.as<int>();
  int* list = c.corr_list.as<int>();
  int* dtot = (int*)(c.dscalars.as<double>() + 48);
  exclusive_scan<int, int>(alive_slot, n, alive_slot, c.scratch.as<int>(), dtot, c.stream);
  int K = 0;
  WCG_TRY(read_small(c, dtot, sizeof(int), &K));
  c.have_grid = false;  // volumes, masses and radii changed
  c.xw_valid = false;
  if (K == n) return cudaGetLastError();
  ++c.launches, k_merge_flags<<<nblk(n, 256), 256, 0, c.stream>>>(n, K, alive_pid, hole_rank,
                                                                   high_rank);
  exclusive_scan<int, int>(hole_rank, n, hole_rank, c.scratch.as<int>(), dtot, c.stream);
  exclusive_scan<int, int>(high_rank, n, high_rank, c.scratch.as<int>(), dtot + 1, c.stream);
  ++c.launches, k_merge_holes<<<nblk(n, 256), 256, 0, c.stream>>>(n, K, alive_pid, hole_rank, holes);
  int counts[2] = {0, 0};
  // surviving slots: alive_slot now holds their ranks; the flags come back
  // from alive_pid through pid
  ++c.launches, k_merge_alive_slots<<<nblk(n, 256), 256, 0, c.stream>>>(n, pid, alive_pid, cursor);
  ++c.launches, k_merge_compact<<<nblk(n, 256), 256, 0, c.stream>>>(n, cursor, alive_slot, list);
  WCG_TRY(read_small(c, dtot, 2 * sizeof(int), counts));  // (the two kernels leave dtot)
  const int nxt = c.cur ^ 1;
  ++c.launches, k_gather_particles<R><<<nblk(K, 256), 256, 0, c.stream>>>(
      list, K, cap, P, c.pbuf[nxt].as<R>(), pid, c.pid[nxt].as<int>(),
      c.pkey.as<long long>() + c.cur * cap, c.pkey.as<long long>() + nxt * cap,
      c.pdelta.as<int>() + c.cur * cap, c.pdelta.as<int>() + nxt * cap, pb,
      c.pbucket.as<int>() + nxt * cap);
  ++c.launches, k_merge_repid<<<nblk(K, 256), 256, 0, c.stream>>>(
      K, list, pid, high_rank, holes, counts[1], c.pid[nxt].as<int>());
  WCG_TRY(cudaGetLastError());
  c.cur = nxt;
  *removed = n - K;
  c.np = K;
  c.have_grid = false;
  c.xw_valid = false;
  // removeEmptyParticles re-sorts the bucket lists from the current positions
  // after a removal (TwoDScene.cpp:1734-1743): a merge later in the sub-step
  // re-buckets the survivors before it pairs them
  c.buckets_valid = false;
  return cudaStreamSynchronize(c.stream);
}

template <typename R>
static cudaError_t merge_liquid_t(Context& c, int selector, const int* perm, long long* removed) {
  *removed = 0;
  const long long n = c.np;
  if (n == 0 || c.g.nb == 0) return cudaSuccess;
  ProfScope prof(c, P_OTHER);
  const int rb = c.real_bytes();
  const long long cap = c.pcap;
  // mwork: cls, removed (bytes), gvol, gmom (Reals), five int arrays
  const size_t off_g = ((size_t)2 * cap + 15) / 16 * 16;
  const size_t off_i = off_g + ((size_t)4 * cap * rb + 15) / 16 * 16;
  WCG_TRY(c.mwork.ensure(off_i + (size_t)5 * cap * sizeof(int) + 64));
  unsigned char* cls = c.mwork.as<unsigned char>();
  unsigned char* rem = cls + cap;
  R* gvol = (R*)(c.mwork.as<unsigned char>() + off_g);
  R* gmom = gvol + cap;
  int* iw = (int*)(c.mwork.as<unsigned char>() + off_i);
  int* alive_slot = iw;
  int* alive_pid = iw + cap;
  int* hole_rank = iw + 2 * cap;
  int* high_rank = iw + 3 * cap;
  int* holes = iw + 4 * cap;
  const long long nb = c.g.nb;
  WCG_TRY(c.corr_start.ensure((size_t)(nb + 2) * sizeof(int)));
  WCG_TRY(c.corr_cursor.ensure((size_t)std::max(nb, n) * sizeof(int)));
  WCG_TRY(c.corr_list.ensure((size_t)n * sizeof(int)));
  const long long scan_tiles = (std::max(nb + 1, n) + kScanTile - 1) / kScanTile + 1;
  WCG_TRY(ensure_scratch(c, (size_t)scan_tiles * sizeof(long long) + 64));
  int* start = c.corr_start.as<int>();
  int* cursor = c.corr_cursor.as<int>();
  int* list = c.corr_list.as<int>();
  R* P = c.pbuf[c.cur].as<R>();
  const int* pid = c.pid[c.cur].as<int>();
  const int* pb = c.pbucket.as<int>() + c.cur * c.pcap;
  long long* key = c.pkey.as<long long>() + (c.cur ^ 1) * c.pcap;  // free half
  // particles uploaded since the last grid build: their buckets in that
  // build's bucket grid, from the current positions
  if (!c.buckets_valid) {
    ++c.launches, k_rebucket<R><<<nblk(n, 256), 256, 0, c.stream>>>(
        P, c.pcap, n, c.g, c.pbucket.as<int>() + c.cur * c.pcap);
    c.buckets_valid = true;
  }
  const double rad_fine = 1.0 / std::sqrt(3.0) * c.prm.dx * c.prm.cell_multiplier;
  const double vf = 4.0 / 3.0 * M_PI * rad_fine * rad_fine * rad_fine;
  // 1. classes and the bucket lists (index order inside a bucket)
  WCG_TRY(cudaMemsetAsync(start, 0, (size_t)(nb + 1) * sizeof(int), c.stream));
  WCG_TRY(cudaMemsetAsync(cursor, 0, (size_t)nb * sizeof(int), c.stream));
  ++c.launches, k_merge_setup<R><<<nblk(n, 256), 256, 0, c.stream>>>(
      P, cap, n, pb, nb, vf, cls, rem, gvol, gmom, key, start);
  exclusive_scan<int, int>(start, nb, start, c.scratch.as<int>(), start + nb, c.stream);
  ++c.launches, k_sort_scatter<<<nblk(n, 256), 256, 0, c.stream>>>(key, n, start, cursor, list);
  ++c.launches, k_sort_cells<<<nblk(nb, 256), 256, 0, c.stream>>>(start, nb, pid, list);
  // 2. the 27 colours in the drawn order
  MergeArgs A;
  A.g = c.g;
  A.selector = selector;
  A.step = c.prm.correction_step > 0 ? c.prm.correction_step : 1;
  A.ne = (int)c.ne;
  A.vf = vf;
  A.should_rad = rad_fine * 2.0;
  A.pid = pid;
  A.list = list;
  A.start = start;
  const long long ncol = (long long)((c.g.ni + 2) / 3) * ((c.g.nj + 2) / 3) * ((c.g.nk + 2) / 3);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int d = 0; d < 3; ++d)
        ++c.launches, k_merge<R><<<nblk(ncol, 128), 128, 0, c.stream>>>(
            A, perm[6 + d], perm[3 + b], perm[a], P, cap, cls, rem, gvol, gmom);
  // 3. gather and update, alive flags
  ++c.launches, k_merge_gather<R><<<nblk(n, 256), 256, 0, c.stream>>>(
      P, cap, n, pid, rem, gvol, gmom, c.prm.liquid_density, alive_slot, alive_pid);
  return remove_flagged_t<R>(c, n, alive_slot, alive_pid, hole_rank, high_rank, holes, removed);
}

template <typename R>
static cudaError_t terminate_liquid_t(Context& c, long long* removed) {
  *removed = 0;
  const long long n = c.np;
  if (n == 0) return cudaSuccess;
  ProfScope prof(c, P_OTHER);
  const long long cap = c.pcap;
  WCG_TRY(c.mwork.ensure((size_t)5 * cap * sizeof(int) + 64));
  int* iw = c.mwork.as<int>();
  WCG_TRY(c.corr_cursor.ensure((size_t)n * sizeof(int)));
  WCG_TRY(c.corr_list.ensure((size_t)n * sizeof(int)));
  const long long scan_tiles = (n + kScanTile - 1) / kScanTile + 1;
  WCG_TRY(ensure_scratch(c, (size_t)scan_tiles * sizeof(long long) + 64));
  TermSet t = c.term;
  if (!c.prm.terminator) t.n = 0;
  ++c.launches, k_terminate<R><<<nblk(n, 256), 256, 0, c.stream>>>(
      c.pbuf[c.cur].as<R>(), cap, n, c.pid[c.cur].as<int>(), t, 3.0 * 4.0 * c.prm.dx, iw,
      iw + cap);
  return remove_flagged_t<R>(c, n, iw, iw + cap, iw + 2 * cap, iw + 3 * cap, iw + 4 * cap,
                             removed);
}

cudaError_t terminate_liquid_particles(Context& c, long long* removed) {
  return c.prm.precision == 0 ? terminate_liquid_t<double>(c, removed)
                              : terminate_liquid_t<float>(c, removed);
}

unsigned long long split_key(unsigned long long seed, unsigned long long k) {
  return splitmix64(seed ^ splitmix64(k ^ 0x73706c69742d6b65ull));
}

// grows the particle capacity to cap, keeping the state of the current half
// (columns, original indices); the other buffers are re-sized empty
static cudaError_t grow_particles(Context& c, long long cap) {
  if (cap <= c.pcap) return cudaSuccess;
  const int rb = c.real_bytes();
  const long long n = c.np;
  DevBuf nb, np_;
  WCG_TRY(nb.ensure((size_t)kNumPCols * cap * rb));
  WCG_TRY(np_.ensure((size_t)cap * sizeof(int)));
  for (int col = 0; col < kNumPCols; ++col)
    WCG_TRY(cudaMemcpyAsync((char*)nb.p + (size_t)col * cap * rb,
                            (const char*)c.pbuf[c.cur].p + (size_t)col * c.pcap * rb,
                            (size_t)n * rb, cudaMemcpyDeviceToDevice, c.stream));
  WCG_TRY(cudaMemcpyAsync(np_.p, c.pid[c.cur].p, (size_t)n * sizeof(int),
                          cudaMemcpyDeviceToDevice, c.stream));
  WCG_TRY(cudaStreamSynchronize(c.stream));
  c.pbuf[c.cur].release();
  c.pid[c.cur].release();
  c.pbuf[c.cur] = nb;
  c.pid[c.cur] = np_;
  const int o = c.cur ^ 1;
  WCG_TRY(c.pbuf[o].ensure((size_t)kNumPCols * cap * rb));
  WCG_TRY(c.pid[o].ensure((size_t)cap * sizeof(int)));
  // keys, offsets and buckets are rebuilt by the next grid build
  WCG_TRY(c.pkey.ensure((size_t)2 * cap * sizeof(long long)));
  WCG_TRY(c.pdelta.ensure((size_t)2 * cap * sizeof(int)));
  WCG_TRY(c.pbucket.ensure((size_t)2 * cap * sizeof(int)));
  WCG_TRY(c.perm.ensure((size_t)cap * sizeof(int)));
  WCG_TRY(c.hostorder.ensure((size_t)cap * 15 * sizeof(double)));
  c.pcap = cap;
  return cudaSuccess;
}

// Children per particle (add_slot, by slot) and their exclusive offsets by
// original index (off_pid); with `nparents`, also the rank of every splitting
// parent by original index (split_rank).  Returns the child total in *total.
template <typename R>
static cudaError_t split_count_t(Context& c, int* total, long long* nparents) {
  const long long n = c.np;
  const double rad_fine = 1.0 / std::sqrt(3.0) * c.prm.dx * c.prm.cell_multiplier;
  const double vf = 4.0 / 3.0 * M_PI * rad_fine * rad_fine * rad_fine;
  WCG_TRY(c.corr_cursor.ensure((size_t)(n + 1) * sizeof(int)));
  WCG_TRY(c.corr_list.ensure((size_t)(n + 1) * sizeof(int)));
  const long long scan_tiles = (n + 1 + kScanTile - 1) / kScanTile + 1;
  WCG_TRY(ensure_scratch(c, (size_t)scan_tiles * sizeof(long long) + 64));
  if (nparents) WCG_TRY(c.split_rank.ensure((size_t)(n + 1) * sizeof(int)));
  int* add_slot = c.corr_cursor.as<int>();
  int* off_pid = c.corr_list.as<int>();
  int* dtot = (int*)(c.dscalars.as<double>() + 50);
  ++c.launches, k_split_count<R><<<nblk(n, 256), 256, 0, c.stream>>>(
      c.pbuf[c.cur].as<R>(), c.pcap, n, c.pid[c.cur].as<int>(), vf, add_slot, off_pid);
  if (nparents) {
    int* rank = c.split_rank.as<int>();
    ++c.launches, k_split_parent_flag<<<nblk(n, 256), 256, 0, c.stream>>>(n, off_pid, rank);
    exclusive_scan<int, int>(rank, n, rank, c.scratch.as<int>(), dtot + 1, c.stream);
  }
  exclusive_scan<int, int>(off_pid, n, off_pid, c.scratch.as<int>(), dtot, c.stream);
  int tot[2] = {0, 0};
  WCG_TRY(read_small(c, dtot, sizeof(tot), tot));
  *total = tot[0];
  if (nparents) *nparents = tot[1];
  return cudaGetLastError();
}

template <typename R>
static cudaError_t split_liquid_t(Context& c, unsigned long long key, long long* added,
                                  const double* pattern = nullptr, const double* rot = nullptr,
                                  long long nparents = 0) {
  *added = 0;
  const long long n = c.np;
  if (n == 0) return nparents == 0 ? cudaSuccess : cudaErrorInvalidValue;
  ProfScope prof(c, P_OTHER);
  int total = 0;
  long long have = 0;
  WCG_TRY(split_count_t<R>(c, &total, pattern ? &have : nullptr));
  // a rotation per splitting parent, no more and no fewer
  if (pattern && have != nparents) return cudaErrorInvalidValue;
  if (total == 0) return cudaSuccess;
  if (n + total > 2000000000ll) return cudaErrorInvalidValue;
  if (pattern) {
    WCG_TRY(c.split_pat.ensure((size_t)kSplitPatternLen * sizeof(double)));
    WCG_TRY(c.split_rot.ensure((size_t)nparents * 9 * sizeof(double)));
    WCG_TRY(cudaMemcpyAsync(c.split_pat.p, pattern, (size_t)kSplitPatternLen * sizeof(double),
                            cudaMemcpyHostToDevice, c.stream));
    WCG_TRY(cudaMemcpyAsync(c.split_rot.p, rot, (size_t)nparents * 9 * sizeof(double),
                            cudaMemcpyHostToDevice, c.stream));
  }
  WCG_TRY(grow_particles(c, n + total));
  int* add_slot = c.corr_cursor.as<int>();
  int* off_pid = c.corr_list.as<int>();
  ++c.launches, k_split<R><<<nblk(n, 128), 128, 0, c.stream>>>(
      c.pbuf[c.cur].as<R>(), c.pcap, n, c.pid[c.cur].as<int>(), add_slot, off_pid, key,
      c.prm.liquid_density, pattern ? c.split_pat.as<double>() : nullptr,
      pattern ? c.split_rot.as<double>() : nullptr, pattern ? c.split_rank.as<int>() : nullptr);
  c.np = n + total;
  c.have_grid = false;
  c.xw_valid = false;
  if (c.g.nb > 0) {
    ++c.launches, k_rebucket<R><<<nblk(c.np, 256), 256, 0, c.stream>>>(
        c.pbuf[c.cur].as<R>(), c.pcap, c.np, c.g, c.pbucket.as<int>() + c.cur * c.pcap);
    c.buckets_valid = true;
  }
  *added = total;
  WCG_TRY(cudaGetLastError());
  return cudaStreamSynchronize(c.stream);
}

cudaError_t split_liquid_particles(Context& c, unsigned long long key, long long* added) {
  return c.prm.precision == 0 ? split_liquid_t<double>(c, key, added)
                              : split_liquid_t<float>(c, key, added);
}

cudaError_t split_liquid_parents(Context& c, long long* nparents) {
  *nparents = 0;
  if (c.np == 0) return cudaSuccess;
  int total = 0;
  return c.prm.precision == 0 ? split_count_t<double>(c, &total, nparents)
                              : split_count_t<float>(c, &total, nparents);
}

cudaError_t split_liquid_particles_with(Context& c, const double* pattern, const double* rot,
                                        long long nparents, long long* added) {
  return c.prm.precision == 0
             ? split_liquid_t<double>(c, 0, added, pattern, rot, nparents)
             : split_liquid_t<float>(c, 0, added, pattern, rot, nparents);
}

cudaError_t merge_liquid_particles(Context& c, int selector, const int* perm, long long* removed) {
  return c.prm.precision == 0 ? merge_liquid_t<double>(c, selector, perm, removed)
                              : merge_liquid_t<float>(c, selector, perm, removed);
}

cudaError_t substep(Context& c, double dt) {
  // terminateParticles (WetClothCore.cpp:97) ahead of the particle maintenance;
  // its removeEmptyParticles also runs without a terminator, and then only
  // matters after an upload that brought particles without fluid volume
  bool run_term = c.prm.terminator != 0;
  if (!run_term && c.maybe_empty && c.np > 0) {
    int flag = 0;
    WCG_TRY(cudaMemcpyAsync(&flag, empty_word(c), sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    WCG_TRY(cudaStreamSynchronize(c.stream));
    run_term = flag != 0;
  }
  if (run_term && c.np > 0) {
    long long rem = 0;
    WCG_TRY(terminate_liquid_particles(c, &rem));
  }
  if (c.maybe_empty) {
    WCG_TRY(cudaMemsetAsync(empty_word(c), 0, sizeof(int), c.stream));
    c.maybe_empty = false;
  }
  // updateOptiVolume, splitLiquidParticles, mergeLiquidParticles
  // (WetClothCore.cpp:97-110): the merge works on the buckets of the previous
  // sub-step's grid build, re-sorted by a split that added particles
  if (c.prm.particle_split && c.np > 0) {
    long long added = 0;
    WCG_TRY(split_liquid_particles(c, split_key(c.prm.split_seed, c.split_count++), &added));
  }
  if (c.prm.particle_merge && c.np > 0 && c.g.nb > 0) {
    int sel = 0, perm[9];
    merge_draws(c.prm.merge_seed, c.merge_count++, c.prm.correction_step, &sel, perm);
    long long removed = 0;
    WCG_TRY(merge_liquid_particles(c, sel, perm, &removed));
    c.merged_removed = removed;
  }
  WCG_TRY(build_grid(c));
  WCG_TRY(map_particles_to_grid(c));
  WCG_TRY(step_velocity(c, dt));
  WCG_TRY(project_fine(c, dt));
  WCG_TRY(apply_pressure_and_extrapolate(c, dt));
  WCG_TRY(constrain_liquid_velocity(c));
  // correctLiquidParticles (WetClothCore.cpp:242) in every sub-step, subset
  // from the seeded stream (at strength 0 it only projects the subset out of
  // the solid)
  if (c.np > 0) {
    const int sel = correction_selector(c.prm.correction_seed, c.corr_count++,
                                        c.prm.correction_step);
    WCG_TRY(correct_liquid_particles(c, dt, sel));
  }
  WCG_TRY(map_grid_to_particles_and_advect(c, dt, true));
  return cudaSuccess;
}

}  // namespace wcg
