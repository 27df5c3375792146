// Many independent scenes stepped together.
//
// Each scene is its own wcg_ctx with its own stream; a batch steps them from a
// small pool of host threads that take scenes from a shared queue, largest
// first.  The kernels of different scenes then overlap on the GPU: small
// scenes leave most SMs idle and their launches are short, so running several
// at once fills the machine.  The thread count is chosen by
// wcg_batch_autotune, which times one batch step per candidate, and each
// scene's launch schedule (the sweep clusters' shape, the PCG iterations per
// host check) by wcg_batch_autotune_schedules, from the device time of each
// scene's step under each candidate.  With the shared solve on
// (wcg_batch_set_shared_solve), the PCG iterations of all scenes waiting in
// their pressure solve run as one launch per kernel from a coordinator
// thread (wcg_step.cu), in place of one launch per scene.  Results are those
// of stepping each scene alone (the same arithmetic on the same data; the
// schedules and the shared solve do not change them).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <string>
#include <thread>
#include <vector>

#include "wcg_context.h"
#include "../../include/wetcloth_gpu.h"

struct wcg_batch {
  std::vector<wcg_ctx*> scenes;
  std::vector<int> order;  // largest particle count first
  int nthreads = 1;
  std::vector<int> device;      // per scene, taken at creation
  std::vector<cudaEvent_t> ev;  // per scene: start, end of a timed step (created on first use)
  wcg::SharedSolve* ss = nullptr;  // the shared solve, when on
  long long ss_launches = 0;       // launches of shared solves turned off since
  int ss_limit = INT_MAX;          // patches of the largest solve that joins
};

namespace {

int fail(int code, const std::string& msg) { return wcg::set_last_error(code, msg); }

// One batch step: every scene takes nsteps calls of wcg_step with its dt.
// Returns the first hard error; WCG_ERR_NOT_CONVERGED (which the reference
// treats as a warning) only if no hard error occurred.
// With `timed`, each scene's steps are bracketed by its two events.
int run_batch(wcg_batch* b, const double* dt, int nsteps, int nthreads, int* status,
              bool timed = false) {
  const int n = (int)b->scenes.size();
  std::atomic<int> next(0);
  std::vector<int> st((size_t)n, WCG_OK);
  std::vector<std::string> msg((size_t)n);
  auto worker = [&]() {
    int dev = -1;
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) break;
      const int i = b->order[k];
      wcg_ctx* ctx = b->scenes[i];
      if (ctx->c.device != dev) {
        cudaSetDevice(ctx->c.device);
        dev = ctx->c.device;
      }
      cudaStream_t strm = (cudaStream_t)wcg_stream(ctx);
      if (timed) cudaEventRecord(b->ev[2 * i], strm);
      for (int s = 0; s < nsteps; ++s) {
        int sub = 0;
        const int r = wcg_step(ctx, dt[i], &sub);
        if (r == WCG_OK) continue;
        if (r == WCG_ERR_NOT_CONVERGED) {
          st[i] = r;
          continue;
        }
        st[i] = r;
        msg[i] = wcg_last_error();
        break;
      }
      if (timed) cudaEventRecord(b->ev[2 * i + 1], strm);
    }
  };
  // the scenes' solves join the shared launches for this step only (a
  // scene stepped on its own afterwards solves alone)
  for (int i = 0; i < n; ++i) b->scenes[i]->c.shared_solve = b->ss;
  const int nt = std::max(1, std::min(nthreads, n));
  std::vector<std::thread> pool;
  pool.reserve((size_t)nt - 1);
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (std::thread& t : pool) t.join();
  for (int i = 0; i < n; ++i) b->scenes[i]->c.shared_solve = nullptr;
  int first = WCG_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = st[i];
    if (st[i] != WCG_OK && st[i] != WCG_ERR_NOT_CONVERGED && first == WCG_OK) {
      first = st[i];
      fail(st[i], "scene " + std::to_string(i) + ": " + msg[i]);
    }
  }
  if (first != WCG_OK) return first;
  for (int i = 0; i < n; ++i)
    if (st[i] == WCG_ERR_NOT_CONVERGED)
      return fail(WCG_ERR_NOT_CONVERGED, "scene " + std::to_string(i) + " did not converge");
  return WCG_OK;
}

}  // namespace

extern "C" {

int wcg_batch_create(int n, wcg_ctx* const* scenes, wcg_batch** out) {
  if (!out || n <= 0 || !scenes) return fail(WCG_ERR_ARG, "need scenes and an output pointer");
  for (int i = 0; i < n; ++i)
    if (!scenes[i]) return fail(WCG_ERR_ARG, "null scene in batch");
  wcg_batch* b = new wcg_batch();
  b->scenes.assign(scenes, scenes + n);
  for (int i = 0; i < n; ++i) b->device.push_back(scenes[i]->c.device);
  b->order.resize((size_t)n);
  for (int i = 0; i < n; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    return b->scenes[x]->c.np + b->scenes[x]->c.ne > b->scenes[y]->c.np + b->scenes[y]->c.ne;
  });
  b->nthreads = std::min(n, 8);
  *out = b;
  return WCG_OK;
}

int wcg_batch_destroy(wcg_batch* b) {
  if (!b) return WCG_OK;
  // the scenes may already be destroyed: only the batch's own records are used
  wcg::shared_solve_destroy(b->ss);
  for (size_t i = 0; i < b->ev.size(); ++i) {
    cudaSetDevice(b->device[i / 2]);
    cudaEventDestroy(b->ev[i]);
  }
  delete b;
  return WCG_OK;
}

int wcg_batch_step(wcg_batch* b, const double* dt, int nsteps, int* status) {
  if (!b || !dt || nsteps < 0) return fail(WCG_ERR_ARG, "bad batch step arguments");
  for (size_t i = 0; i < b->scenes.size(); ++i)
    if (!(dt[i] > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  return run_batch(b, dt, nsteps, b->nthreads, status);
}

int wcg_batch_set_threads(wcg_batch* b, int nthreads) {
  if (!b || nthreads < 1) return fail(WCG_ERR_ARG, "thread count must be >= 1");
  b->nthreads = nthreads;
  return WCG_OK;
}

int wcg_batch_threads(const wcg_batch* b) { return b ? b->nthreads : -1; }

int wcg_batch_set_shared_solve(wcg_batch* b, int on) {
  if (!b) return fail(WCG_ERR_ARG, "null batch");
  if (!on) {
    b->ss_launches += wcg::shared_solve_launches(b->ss);
    wcg::shared_solve_destroy(b->ss);
    b->ss = nullptr;
    return WCG_OK;
  }
  if (b->ss) return WCG_OK;
  for (int d : b->device)
    if (d != b->device[0])
      return fail(WCG_ERR_ARG, "the shared solve needs every scene on one device");
  std::string err;
  b->ss = wcg::shared_solve_create(b->device[0], &err);
  if (!b->ss) return fail(WCG_ERR_CUDA, "shared solve: " + err);
  wcg::shared_solve_set_limit(b->ss, b->ss_limit);
  return WCG_OK;
}

int wcg_batch_set_shared_solve_limit(wcg_batch* b, int max_patches) {
  if (!b) return fail(WCG_ERR_ARG, "null batch");
  if (max_patches < 1) return fail(WCG_ERR_ARG, "max_patches must be >= 1");
  b->ss_limit = max_patches;
  wcg::shared_solve_set_limit(b->ss, max_patches);
  return WCG_OK;
}

long long wcg_batch_shared_launches(const wcg_batch* b) {
  return b ? b->ss_launches + wcg::shared_solve_launches(b->ss) : -1;
}

// Times one batch step for each candidate thread count (each trial advances
// every scene by one step) and keeps the fastest.
int wcg_batch_autotune(wcg_batch* b, const double* dt, const int* candidates, int ncand,
                       double* ms_out) {
  if (!b || !dt || !candidates || ncand <= 0) return fail(WCG_ERR_ARG, "bad autotune arguments");
  double best = 1e300;
  int best_t = b->nthreads;
  for (int k = 0; k < ncand; ++k) {
    if (candidates[k] < 1) return fail(WCG_ERR_ARG, "thread count must be >= 1");
    const auto t0 = std::chrono::steady_clock::now();
    const int r = run_batch(b, dt, 1, candidates[k], nullptr);
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (r != WCG_OK && r != WCG_ERR_NOT_CONVERGED) return r;
    if (ms_out) ms_out[k] = ms;
    if (ms < best) {
      best = ms;
      best_t = candidates[k];
    }
  }
  b->nthreads = best_t;
  return WCG_OK;
}

// Each candidate in turn: every scene takes it, the batch steps `trials`
// times with each scene's step timed on its stream; a scene keeps the
// candidate with its smallest time.
int wcg_batch_autotune_schedules(wcg_batch* b, const double* dt, const wcg_schedule* cand,
                                 int ncand, int trials, double* ms_out, int* chosen_out) {
  if (!b || !dt || !cand || ncand <= 0 || trials < 1)
    return fail(WCG_ERR_ARG, "bad schedule autotune arguments");
  const int n = (int)b->scenes.size();
  for (int i = 0; i < n; ++i)
    if (!(dt[i] > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  std::vector<wcg_schedule> keep((size_t)n);
  for (int i = 0; i < n; ++i) wcg_get_schedule(b->scenes[i], &keep[(size_t)i]);
  // every candidate must be accepted by every scene before any trial runs
  for (int k = 0; k < ncand; ++k)
    for (int i = 0; i < n; ++i) {
      const int r = wcg_set_schedule(b->scenes[i], &cand[k]);
      wcg_set_schedule(b->scenes[i], &keep[(size_t)i]);
      if (r != WCG_OK) return r;
    }
  if (b->ev.empty()) {
    b->ev.resize((size_t)2 * n);
    for (int i = 0; i < 2 * n; ++i) {
      cudaSetDevice(b->device[(size_t)i / 2]);
      if (cudaEventCreate(&b->ev[(size_t)i]) != cudaSuccess) {
        b->ev.resize((size_t)i);
        return fail(WCG_ERR_CUDA, "cudaEventCreate failed");
      }
    }
  }
  std::vector<double> best((size_t)n * ncand, 1e300);
  for (int k = 0; k < ncand; ++k) {
    for (int i = 0; i < n; ++i) wcg_set_schedule(b->scenes[i], &cand[k]);
    for (int t = 0; t < trials; ++t) {
      const int r = run_batch(b, dt, 1, b->nthreads, nullptr, true);
      if (r != WCG_OK && r != WCG_ERR_NOT_CONVERGED) {
        for (int i = 0; i < n; ++i) wcg_set_schedule(b->scenes[i], &keep[(size_t)i]);
        return r;
      }
      for (int i = 0; i < n; ++i) {
        cudaSetDevice(b->device[(size_t)i]);
        float ms = 0.f;
        if (cudaEventSynchronize(b->ev[2 * i + 1]) != cudaSuccess ||
            cudaEventElapsedTime(&ms, b->ev[2 * i], b->ev[2 * i + 1]) != cudaSuccess)
          return fail(WCG_ERR_CUDA, "timing a scene's step failed");
        double& m = best[(size_t)i * ncand + k];
        m = std::min(m, (double)ms);
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    int kb = 0;
    for (int k = 1; k < ncand; ++k)
      if (best[(size_t)i * ncand + k] < best[(size_t)i * ncand + kb]) kb = k;
    wcg_set_schedule(b->scenes[i], &cand[kb]);
    if (chosen_out) chosen_out[i] = kb;
  }
  if (ms_out) std::copy(best.begin(), best.end(), ms_out);
  return WCG_OK;
}

}  // extern "C"
