// MIC(0)-PCG in the skewed pencil layout.
//
// The pressure unknowns of one solve (the bounding box of the DOF cells) are
// copied once into a layout built for the triangular sweeps.  One grid axis is
// the stream axis s (the longest extent of the box); the other two (a, c) are
// cut into patches of 16 x 16 lines.  Line (al, cl) of a patch is skewed by
// d = al + cl rows: cell (s, a, c) sits at row t = s + d of its patch, and
// element (patch, t, line) is stored at ((patch * R + t) * 256 + line) with
// line = al + 16 cl and R = Ls + 30 rows.  Rows outside a line's range and
// lines outside the box hold zeros.
//
// In this layout every MIC(0) hyperplane dependency is one row back (one row
// forward for the backward sweep):
//   (s-1, a, c): row t-1 of the same line
//   (s, a-1, c): row t-1 of line - 1
//   (s, a, c-1): row t-1 of line - 16
// so a CTA of 256 threads (one per line) walks its patch row by row, one
// barrier per row, every load and store a coalesced row, rows prefetched kPre
// ahead in registers.  The factor is stored interleaved per cell
// {1/sqrt(d'), S_s, S_a, S_c} so a sweep reads it with one vector load.  Values
// crossing a patch edge go through a global buffer of tagged 64-bit words,
// (epoch << 32 | 32 data bits), one word per 32 bits of payload: the consumer
// re-reads its word until the tag equals the launch's epoch, so no fence or
// flag is needed and a patch waits only for the rows it reads.
// Patches are handed out by an atomic ticket in wave order (PAi + PCi), so a
// patch's upstream patches always started before it.
//
// The arithmetic is that of the tile sweeps in wcg_pcg.cuh (restating
// robertbridson's factor_modified_incomplete_cholesky0 / solve_lower /
// solve_lower_transpose_in_place, libWetCloth/Core/PCGSolver/PCGSolver.h:
// 97-239): per DOF j, d_j = A_jj - sum over the three lower neighbours k of
// [L^2 + omega L miss], L = A(k, j) / sqrt(d_k'), miss = the other two upper
// couplings of k over sqrt(d_k'); forward y_j = (r_j - sum S_k y_k) / sqrt(d_j');
// backward z_j = (y_j - sum S_j z_k) / sqrt(d_j').  The lower neighbours are
// taken in the order c, a, s (z, y, x when s is x).
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_pcg.cuh"

namespace wcg {

constexpr int kPatch = 16;                    // lines per patch edge
constexpr int kPatchLines = kPatch * kPatch;  // threads of a sweep CTA
constexpr int kPre = 4;                       // rows of edge words prefetched ahead
constexpr int kPlBlocks = 592;                // streaming kernels: 4 x 148 SMs
// the fused SpMV in FP32 (32 registers): 8 resident CTAs per SM, so twice the
// loads in flight of the other streaming kernels
constexpr int kPlSpmvBlocks32 = 1184;
static_assert(kRedThreads == kPatchLines, "streaming kernels walk one row per block");

__host__ __device__ inline long long pl_index(const PencilGeom& G, long long p, int t, int l) {
  return (p * G.R + t) * kPatchLines + l;
}

// ---- tagged edge words -----------------------------------------------------------
typedef unsigned long long u64;

__device__ inline u64 ld_relaxed_u64(const u64* p) {
  u64 v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

__device__ inline void st_relaxed_u64(u64* p, u64 v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v));
}

template <typename R>
struct TagWords;
template <>
struct TagWords<float> {
  static constexpr int W = 1;
  __device__ static void pack(float v, unsigned tag, u64* w) {
    w[0] = ((u64)tag << 32) | (u64)__float_as_uint(v);
  }
  __device__ static float unpack(const u64* w) { return __uint_as_float((unsigned)w[0]); }
};
template <>
struct TagWords<double> {
  static constexpr int W = 2;
  __device__ static void pack(double v, unsigned tag, u64* w) {
    const u64 b = (u64)__double_as_longlong(v);
    w[0] = ((u64)tag << 32) | (b & 0xffffffffull);
    w[1] = ((u64)tag << 32) | (b >> 32);
  }
  __device__ static double unpack(const u64* w) {
    return __longlong_as_double((long long)((w[1] << 32) | (w[0] & 0xffffffffull)));
  }
};

// ---- bulk row copies into shared memory (cp.async.bulk + mbarrier) ---------
__device__ inline unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ inline void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ inline void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ inline bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// global -> shared, 16-byte aligned addresses, bytes a multiple of 16
__device__ inline void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ inline unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of an mbarrier wait (2 s)

// ---- thread-block clusters: distributed shared memory -----------------------
__device__ inline unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// every thread of every CTA of the cluster; release/acquire orders the shared
// memory each CTA wrote before it against the reads after it
__device__ inline void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// address of the same shared variable in CTA `rank` of the cluster
__device__ inline unsigned cluster_map(unsigned local, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ inline unsigned ld_cluster_u32(unsigned addr) {
  unsigned v;
  asm volatile("ld.relaxed.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
__device__ inline void st_cluster_u64(unsigned addr, u64 v) {
  asm volatile("st.relaxed.cluster.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}
// a word of this CTA's shared memory that peers of the cluster write
__device__ inline u64 ld_own_u64(unsigned addr) {
  u64 v;
  asm volatile("ld.relaxed.cluster.shared::cta.u64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
  return v;
}

// Stages of the shared-memory row ring of a sweep.
template <typename R>
struct SweepStages {
  static constexpr int D = sizeof(R) == 4 ? 8 : 6;
};
// Arrays staged per row: factor A_d, A_s, A_a, A_c; forward r, coef x4 (, q);
// backward y, coef x4, r.
__host__ __device__ constexpr int sweep_nf(int mode, bool upd) {
  return mode == 0 ? 4 : (mode == 1 ? (upd ? 6 : 5) : 6);
}
template <typename R>
__host__ __device__ constexpr size_t sweep_dyn_smem(int mode, bool upd) {
  return (size_t)SweepStages<R>::D * sweep_nf(mode, upd) * 256 * sizeof(R) +
         (size_t)SweepStages<R>::D * 8;
}
// With clusters the c-face edge words of the patch upstream in the same
// cluster land in this CTA's shared memory: Ls x 16 entries, 16-byte aligned
// after the ring and its mbarriers.
template <typename R>
__host__ __device__ constexpr size_t sweep_cedge_off(int mode, bool upd) {
  return (sweep_dyn_smem<R>(mode, upd) + 15) / 16 * 16;
}
template <typename R>
__host__ __device__ constexpr size_t sweep_cedge_bytes(int mode, int Ls) {
  return (size_t)Ls * 16 * (mode == 0 ? 2 : 1) * (sizeof(R) / 4) * 8;
}
// dynamic shared memory of a cluster sweep: the ring, then the edge words of
// the clustered faces
template <typename R>
__host__ __device__ constexpr size_t sweep_cluster_smem(int mode, bool upd, int Ls, int cc,
                                                        int ca) {
  return sweep_cedge_off<R>(mode, upd) + (cc > 1 ? sweep_cedge_bytes<R>(mode, Ls) : 0) +
         (ca > 1 ? sweep_cedge_bytes<R>(mode, Ls) : 0);
}
// the a-face words of a 2-D cluster, after the c-face ones (when present)
template <typename R>
__host__ __device__ constexpr size_t sweep_aedge_off(int mode, bool upd, int Ls, bool cfaces) {
  return sweep_cedge_off<R>(mode, upd) + (cfaces ? sweep_cedge_bytes<R>(mode, Ls) : 0);
}

// Words of the edge buffer: entry (producer patch, side, s, k), EW words each.
// side 0: the a-face (k = cl), side 1: the c-face (k = al).
__device__ inline long long edge_word(const PencilGeom& G, long long p, int side, int s, int k,
                                      int EW) {
  return (((p * 2 + side) * G.Ls + s) * kPatch + k) * EW;
}

// The MIC(0) factor of a cell, interleaved: {1/sqrt(d'), S_s, S_a, S_c}.
__device__ inline void ld_coef(const float* p, float* c) {
  const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
  c[0] = t.x; c[1] = t.y; c[2] = t.z; c[3] = t.w;
}
__device__ inline void ld_coef(const double* p, double* c) {
  const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  c[0] = a.x; c[1] = a.y; c[2] = b.x; c[3] = b.y;
}
__device__ inline void st_coef(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ inline void st_coef(double* p, double a, double b, double c, double d) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
  reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
}

template <typename R>
struct PencilSweepArgs {
  PencilGeom G;
  const int* order;   // patches in wave order
  int* ticket;
  int ticket_base;    // tickets already handed out this solve
  unsigned epoch;     // tag of this launch's edge words
  u64* edge;
  // factorisation input
  const R* AD;
  const R* AS;
  const R* AA;
  const R* AC;
  R* coef;      // factor: 4 per cell {1/sqrt(d'), S_s, S_a, S_c}
  // sweeps
  const R* in;  // forward: r; backward: y
  R* out;       // forward: y; backward: z
  R* r;         // forward (update): r updated in place; backward: r for z.r
  const R* q;   // forward (update)
  double* sc;            // device scalars (the last CTA of a reducing sweep writes them)
  double* part;  // per-patch partial: forward max|r|, backward z.r
  R omega, min_ratio;
  int* err;
  int* done_ctr;         // with part: the last CTA reduces the partials (forward with
                         // update: max|r| and the stop test; backward: z.r and beta)
  int red_init;          // backward: the first z.r of a solve (beta = 0)
  int npart;             // partials (patches)
  long long spin_limit;  // polls of an edge word before the wait gives up
  int stale_patch;       // failure-path test: this patch waits for a tag nothing
                         // writes (-1: none)
};

// MODE: kFactor, kForward, kBackward.  UPD: the forward sweep first applies
// r -= alpha q (and reports max|r|); the matching x += alpha s is applied by
// the next SpMV (k_pl_spmv_s) or, after the last iteration, by k_pl_axpy.
//
// One thread per line, tid = al + 16 cl, warp w holding cl = 2w and 2w + 1;
// the CTA advances one row per step with one barrier.  The a-neighbour and the
// c-neighbour inside the warp come by shuffle of the previous step's outputs,
// the c-neighbour in the adjacent warp through shared memory, and values across
// the patch faces through the tagged edge words.
//
// CL > 1: launched in clusters of CL CTAs along c.  The patches of a cluster
// are one cluster column of CL consecutive c-patches; a c-face neighbour in
// the same cluster writes its tagged words straight into this CTA's shared
// memory (st.shared::cluster), which takes the global round trip off those
// hops.  Tickets are handed out per cluster in wave order, so every upstream
// cluster started earlier.  The cluster syncs after the edge buffers are
// cleared and before any CTA exits, so no CTA writes into a peer that has not
// started or has already left.
//
// CA > 1 as well: clusters of CC x CA CTAs, a tile of CC c-patches by CA
// a-patches (rank = ra + CA rc); a-face neighbours inside the tile exchange
// through shared memory the same way (their words after the c-face ones).
//
// The body takes the launch's CTA count (nblocks) as an argument so a launch
// over several solves (k_pencil_sweep_batch) can run it per solve.
template <typename R, int MODE, bool UPD, int CC, int CA>
__device__ __forceinline__ void pencil_sweep_run(const PencilSweepArgs<R>& A, int nblocks) {
  constexpr int CL = CC * CA;
  constexpr bool BWD = MODE == kBackward;
  constexpr int PW = MODE == kFactor ? 2 : 1;  // values sent across an edge
  constexpr int TW = TagWords<R>::W;
  constexpr int EW = PW * TW;
  // prefetched per cell: factor A_d, A_s, A_a, A_c; forward in, coef[4] (, q);
  // backward in, coef[4], r
  constexpr int NF = sweep_nf(MODE, UPD);
  static_assert(kFactor == 0 && kForward == 1 && kBackward == 2, "mode numbering");
  constexpr int RS = BWD ? -kPatchLines : kPatchLines;  // element step per row
  constexpr int NW = kPatchLines / 32;
  constexpr int D = SweepStages<R>::D;             // rows in flight
  constexpr int SLOT = NF * kPatchLines;            // Reals per staged row
  __shared__ int s_ticket;
  __shared__ R xc[2][NW][kPatch][PW];
  __shared__ double red[kPatchLines];
  extern __shared__ __align__(128) unsigned char dsm[];  // D slots, then D mbarriers
  R* const ring = reinterpret_cast<R*>(dsm);
  const unsigned bar0 = smem_u32(dsm + (size_t)D * SLOT * sizeof(R));
  const PencilGeom& G = A.G;
  const int tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  // one ticket per patch (per cluster with CL > 1), taken even by a launch
  // that returns at once, so the counter stays in step with the host's base
  const int crank = CL > 1 ? (int)cluster_rank() : 0;
  if (tid == 0 && crank == 0) s_ticket = atomicAdd(A.ticket, 1) - A.ticket_base;
  // set by an earlier launch, so uniform: the whole cluster returns before
  // any cross-CTA access
  if (*(const int*)(A.sc + S_DONE)) return;
  for (int i = tid; i < 2 * NW * kPatch * PW; i += kPatchLines) (&xc[0][0][0][0])[i] = R(0);
  u64* const cedge = CC > 1 ? reinterpret_cast<u64*>(dsm + sweep_cedge_off<R>(MODE, UPD)) : nullptr;
  u64* const aedge =
      CA > 1 ? reinterpret_cast<u64*>(dsm + sweep_aedge_off<R>(MODE, UPD, G.Ls, CC > 1)) : nullptr;
  if (CC > 1)
    for (int i = tid; i < G.Ls * kPatch * EW; i += kPatchLines) cedge[i] = 0ull;
  if (CA > 1)
    for (int i = tid; i < G.Ls * kPatch * EW; i += kPatchLines) aedge[i] = 0ull;
  if (CL > 1)
    cluster_sync();
  else
    __syncthreads();
  const int tk = CL > 1 ? (int)ld_cluster_u32(cluster_map(smem_u32(&s_ticket), 0)) : s_ticket;
  const int nTA = (G.nPA + CA - 1) / CA;
  const int nunits = CL > 1 ? nTA * ((G.nPC + CC - 1) / CC) : (int)G.npatch;
  const int ra = crank % CA, rc = crank / CA;
  bool run = true;
  if (tk < 0 || tk >= nunits) {
    if (tid == 0) record_error(A.err, kErrIndex);
    run = false;
  }
  int p = 0, PAi = 0, PCi = 0;
  if (run) {
    const int unit = BWD ? A.order[nunits - 1 - tk] : A.order[tk];
    PAi = CL > 1 ? (unit % nTA) * CA + ra : unit % G.nPA;
    PCi = CL > 1 ? (unit / nTA) * CC + rc : unit / G.nPA;
    run = PCi < G.nPC && PAi < G.nPA;  // the last tiles may reach past the box
    p = PCi * G.nPA + PAi;
  }
  if (run) {
  const int al = tid & (kPatch - 1), cl = tid / kPatch;
  const bool line = PAi * kPatch + al < G.NA && PCi * kPatch + cl < G.NC;
  const int dl = al + cl;
  const int Ls = G.Ls, NR = G.R;
  const int u0 = BWD ? (NR - Ls) - dl : dl;  // first live step
  int up_a = -1, up_c = -1;
  bool pub_a, pub_c;
  if (!BWD) {
    if (al == 0 && PAi > 0) up_a = p - 1;
    if (cl == 0 && PCi > 0) up_c = p - G.nPA;
    pub_a = al == kPatch - 1 && PAi + 1 < G.nPA;
    pub_c = cl == kPatch - 1 && PCi + 1 < G.nPC;
  } else {
    if (al == kPatch - 1 && PAi + 1 < G.nPA) up_a = p + 1;
    if (cl == kPatch - 1 && PCi + 1 < G.nPC) up_c = p + G.nPA;
    pub_a = al == 0 && PAi > 0;
    pub_c = cl == 0 && PCi > 0;
  }
  if (!line) up_a = up_c = -1;
  // c-face neighbours in the same cluster exchange through shared memory
  const bool c_loc = CC > 1 && up_c >= 0 && (BWD ? rc < CC - 1 : rc > 0);
  const bool c_rem = CC > 1 && pub_c && (BWD ? rc > 0 : rc < CC - 1);
  const bool a_loc = CA > 1 && up_a >= 0 && (BWD ? ra < CA - 1 : ra > 0);
  const bool a_rem = CA > 1 && pub_a && (BWD ? ra > 0 : ra < CA - 1);
  if (c_loc) up_c = -1;
  if (c_rem) pub_c = false;
  if (a_loc) up_a = -1;
  if (a_rem) pub_a = false;
  const unsigned cedge_own = CC > 1 ? smem_u32(cedge) : 0u;
  const unsigned cedge_dst = c_rem ? cluster_map(cedge_own, BWD ? crank - CA : crank + CA) : 0u;
  const unsigned aedge_own = CA > 1 ? smem_u32(aedge) : 0u;
  const unsigned aedge_dst = a_rem ? cluster_map(aedge_own, BWD ? crank - 1 : crank + 1) : 0u;
  const bool a_edge = al == (BWD ? kPatch - 1 : 0);  // no in-warp a source
  const bool c_prod = BWD ? lane < 16 : lane >= 16;  // half read by the next warp
  const int w_src = BWD ? w + 1 : w - 1;
  const bool has_wsrc = BWD ? w + 1 < NW : w > 0;
  constexpr int ES = kPatch * EW;  // words between consecutive s of one entry
  const u64* ea_src = up_a >= 0 ? A.edge + edge_word(G, up_a, 0, 0, cl, EW) : nullptr;
  const u64* ec_src = up_c >= 0 ? A.edge + edge_word(G, up_c, 1, 0, al, EW) : nullptr;
  u64* ea_dst = pub_a ? A.edge + edge_word(G, p, 0, 0, cl, EW) : nullptr;
  u64* ec_dst = pub_c ? A.edge + edge_word(G, p, 1, 0, al, EW) : nullptr;
  const unsigned ep = A.epoch;
  // the tag this patch waits for: the launch's, except on the patch a
  // failure-path test marks, whose waits then run into their limit
  const unsigned ep_want = p == A.stale_patch ? (ep ^ 0x80000000u) : ep;
  const long long spin_limit = A.spin_limit;
  const R al_r = (MODE == kForward && UPD) ? (R)A.sc[S_ALPHA] : R(0);
  const R omega = A.omega, min_ratio = A.min_ratio;
  // per-thread base pointers (patch and line applied); rows by 32-bit offset
  const long long pb = (long long)p * NR * kPatchLines + tid;
  R* __restrict__ pcoef = A.coef + 4 * pb;
  R* __restrict__ o_out = MODE == kFactor ? nullptr : A.out + pb;
  R* __restrict__ o_r = (MODE == kForward && UPD) ? A.r + pb : nullptr;
  const int off0 = BWD ? (NR - 1) * kPatchLines : 0;
  auto s_at = [&](int u) { return BWD ? (NR - 1 - u) - dl : u - dl; };
  auto live_at = [&](int u) { return line && (unsigned)(u - u0) < (unsigned)Ls; };
  // Rows outside a line's range hold zeros, so whole rows are staged and every
  // cell is computed (zeros stay zeros); only the edge words need liveness.
  // Thread 0 copies whole rows (one bulk copy per array) D rows ahead into a
  // ring slot; the slot layout is [first array][coef x4 or A_s, A_a, A_c][q/r].
  const long long pbase = (long long)p * NR * kPatchLines;
  auto issue = [&](int u) {
    const int j = u % D;
    const unsigned bar = bar0 + 8 * j;
    const unsigned dst = smem_u32(ring + (size_t)j * SLOT);
    const long long rb = pbase + (long long)(BWD ? NR - 1 - u : u) * kPatchLines;
    constexpr unsigned RB = kPatchLines * sizeof(R);
    mbar_expect_tx(bar, NF * RB);
    if (MODE == kFactor) {
      bulk_g2s(dst, A.AD + rb, RB, bar);
      bulk_g2s(dst + RB, A.AS + rb, RB, bar);
      bulk_g2s(dst + 2 * RB, A.AA + rb, RB, bar);
      bulk_g2s(dst + 3 * RB, A.AC + rb, RB, bar);
    } else {
      bulk_g2s(dst, A.in + rb, RB, bar);
      bulk_g2s(dst + RB, A.coef + 4 * rb, 4 * RB, bar);
      if (NF == 6) bulk_g2s(dst + 5 * RB, (MODE == kForward ? A.q : A.r) + rb, RB, bar);
    }
  };
  bool gave_up = false;
  auto mwait = [&](int u) {
    const unsigned bar = bar0 + 8 * (u % D);
    const unsigned par = (unsigned)(u / D) & 1u;
    if (mbar_try_wait(bar, par)) return;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, par)) {
      if (gave_up || global_ns() - t0 > kWaitNs) {
        if (!gave_up) record_error(A.err, kErrWaitTimeout);
        gave_up = true;
        return;
      }
    }
  };
  if (tid == 0) {
    for (int j = 0; j < D; ++j) mbar_init(bar0 + 8 * j, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int u = 0; u < D && u < NR; ++u) issue(u);

  u64 epa[kPre][EW], epc[kPre][EW];
#pragma unroll
  for (int v = 0; v < kPre; ++v) {
    const bool lv = v < NR && live_at(v);
    const int sv = s_at(v);
#pragma unroll
    for (int k = 0; k < EW; ++k) {
      epa[v][k] = (lv && ea_src) ? ld_relaxed_u64(ea_src + sv * ES + k) : 0ull;
      epc[v][k] = (lv && ec_src) ? ld_relaxed_u64(ec_src + sv * ES + k) : 0ull;
    }
  }
  R carry[PW], prev_a[PW], prev_c[PW];
#pragma unroll
  for (int k = 0; k < PW; ++k) carry[k] = prev_a[k] = prev_c[k] = R(0);
  R rmax = 0;
  double dsum = 0;
  // complete an edge entry: re-read words whose tag is stale (bounded)
  auto ewait = [&](u64* wd, const u64* src) {
#pragma unroll
    for (int k = 0; k < EW; ++k) {
      if ((unsigned)(wd[k] >> 32) == ep_want) continue;
      long long it = 0;
      do {
        if (gave_up || ++it > spin_limit) {
          if (!gave_up) record_error(A.err, kErrWaitTimeout);
          gave_up = true;
          wd[k] = (u64)ep << 32;
          break;
        }
        wd[k] = ld_relaxed_u64(src + k);
      } while ((unsigned)(wd[k] >> 32) != ep_want);
    }
  };

  for (int ub = 0; ub < NR; ub += kPre) {
#pragma unroll
    for (int v = 0; v < kPre; ++v) {
      const int u = ub + v;
      if (u >= NR) break;  // uniform over the CTA
      const int off = off0 + u * RS;
      const int cur = u & 1, nxt = cur ^ 1;
      // neighbour inputs of step u = outputs of step u - 1
      R in_a[PW], in_c[PW];
#pragma unroll
      for (int k = 0; k < PW; ++k) {
        in_a[k] = BWD ? __shfl_down_sync(0xffffffffu, prev_a[k], 1)
                      : __shfl_up_sync(0xffffffffu, prev_a[k], 1);
        in_c[k] = BWD ? __shfl_down_sync(0xffffffffu, prev_c[k], 16)
                      : __shfl_up_sync(0xffffffffu, prev_c[k], 16);
        if (a_edge) in_a[k] = R(0);
        if (!c_prod) in_c[k] = has_wsrc ? xc[cur][w_src][al][k] : R(0);
      }
      const bool live = live_at(u);
      const int s = s_at(u);
      if (live && ea_src) {
        ewait(epa[v], ea_src + s * ES);
#pragma unroll
        for (int k = 0; k < PW; ++k) in_a[k] = TagWords<R>::unpack(epa[v] + k * TW);
      }
      if (live && ec_src) {
        ewait(epc[v], ec_src + s * ES);
#pragma unroll
        for (int k = 0; k < PW; ++k) in_c[k] = TagWords<R>::unpack(epc[v] + k * TW);
      }
      if (CA > 1 && live && a_loc) {
        u64 wd[EW];
        const unsigned a0 = aedge_own + (unsigned)((s * kPatch + cl) * EW) * 8u;
#pragma unroll
        for (int k = 0; k < EW; ++k) {
          wd[k] = ld_own_u64(a0 + 8u * k);
          long long it = 0;
          while ((unsigned)(wd[k] >> 32) != ep_want) {
            if (gave_up || ++it > spin_limit) {
              if (!gave_up) record_error(A.err, kErrWaitTimeout);
              gave_up = true;
              break;
            }
            wd[k] = ld_own_u64(a0 + 8u * k);
          }
        }
#pragma unroll
        for (int k = 0; k < PW; ++k) in_a[k] = TagWords<R>::unpack(wd + k * TW);
      }
      if (CC > 1 && live && c_loc) {
        u64 wd[EW];
        const unsigned a0 = cedge_own + (unsigned)((s * kPatch + al) * EW) * 8u;
#pragma unroll
        for (int k = 0; k < EW; ++k) {
          wd[k] = ld_own_u64(a0 + 8u * k);
          long long it = 0;
          while ((unsigned)(wd[k] >> 32) != ep_want) {
            if (gave_up || ++it > spin_limit) {
              if (!gave_up) record_error(A.err, kErrWaitTimeout);
              gave_up = true;
              break;
            }
            wd[k] = ld_own_u64(a0 + 8u * k);
          }
        }
#pragma unroll
        for (int k = 0; k < PW; ++k) in_c[k] = TagWords<R>::unpack(wd + k * TW);
      }
      // this row's inputs from the ring
      R f[NF];
      mwait(u);
      {
        const R* S = ring + (size_t)(u % D) * SLOT;
        f[0] = S[tid];
        if (MODE == kFactor) {
          f[1] = S[kPatchLines + tid];
          f[2] = S[2 * kPatchLines + tid];
          f[3] = S[3 * kPatchLines + tid];
        } else {
          const R* cf = S + kPatchLines + 4 * tid;
          f[1] = cf[0]; f[2] = cf[1]; f[3] = cf[2]; f[4] = cf[3];
          if (NF == 6) f[5] = S[5 * kPatchLines + tid];
        }
      }
      R out_s[PW], out_a[PW], out_c[PW];
      if (MODE == kFactor) {
        const R ad = f[0];
        R d = ad;
        R iv = R(0);
        if (ad != R(0)) {
          d = d - in_c[0] * in_c[0];
          d = d - (omega * in_c[0]) * in_c[1];
          d = d - in_a[0] * in_a[0];
          d = d - (omega * in_a[0]) * in_a[1];
          d = d - carry[0] * carry[0];
          d = d - (omega * carry[0]) * carry[1];
          const R piv = d < min_ratio * ad ? ad : d;
          iv = R(1) / sqrt(piv);
        }
        const R ss = f[1] * iv, sa = f[2] * iv, scv = f[3] * iv;
        st_coef(pcoef + 4 * off, iv, ss, sa, scv);
        out_s[0] = ss; out_s[1] = sa + scv;
        out_a[0] = sa; out_a[1] = ss + scv;
        out_c[0] = scv; out_c[1] = ss + sa;
      } else if (MODE == kForward) {
        R rv = f[0];
        if (UPD) {
          rv = rv - al_r * f[5];
          o_r[off] = rv;
          const R av = fabs(rv);
          rmax = av > rmax ? av : rmax;
        }
        R vv = rv;
        vv -= in_c[0];
        vv -= in_a[0];
        vv -= carry[0];
        const R y = vv * f[1];
        o_out[off] = y;
        out_s[0] = f[2] * y;
        out_a[0] = f[3] * y;
        out_c[0] = f[4] * y;
      } else {
        R vv = f[0];
        vv -= f[2] * carry[0];
        vv -= f[3] * in_a[0];
        vv -= f[4] * in_c[0];
        const R z = vv * f[1];
        o_out[off] = z;
        dsum += (double)z * (double)f[5];
        out_s[0] = out_a[0] = out_c[0] = z;
      }
      if (live && ea_dst) {
        u64 wd[EW];
#pragma unroll
        for (int k = 0; k < PW; ++k) TagWords<R>::pack(out_a[k], ep, wd + k * TW);
#pragma unroll
        for (int k = 0; k < EW; ++k) st_relaxed_u64(ea_dst + s * ES + k, wd[k]);
      }
      if (live && ec_dst) {
        u64 wd[EW];
#pragma unroll
        for (int k = 0; k < PW; ++k) TagWords<R>::pack(out_c[k], ep, wd + k * TW);
#pragma unroll
        for (int k = 0; k < EW; ++k) st_relaxed_u64(ec_dst + s * ES + k, wd[k]);
      }
      if (CC > 1 && live && c_rem) {
        u64 wd[EW];
#pragma unroll
        for (int k = 0; k < PW; ++k) TagWords<R>::pack(out_c[k], ep, wd + k * TW);
        const unsigned a0 = cedge_dst + (unsigned)((s * kPatch + al) * EW) * 8u;
#pragma unroll
        for (int k = 0; k < EW; ++k) st_cluster_u64(a0 + 8u * k, wd[k]);
      }
      if (CA > 1 && live && a_rem) {
        u64 wd[EW];
#pragma unroll
        for (int k = 0; k < PW; ++k) TagWords<R>::pack(out_a[k], ep, wd + k * TW);
        const unsigned a0 = aedge_dst + (unsigned)((s * kPatch + cl) * EW) * 8u;
#pragma unroll
        for (int k = 0; k < EW; ++k) st_cluster_u64(a0 + 8u * k, wd[k]);
      }
#pragma unroll
      for (int k = 0; k < PW; ++k) {
        if (c_prod) xc[nxt][w][al][k] = out_c[k];
        prev_a[k] = out_a[k];
        prev_c[k] = out_c[k];
        carry[k] = out_s[k];
      }
      // edge words of step u + kPre
      {
        const int un = u + kPre;
        const bool lv = un < NR && live_at(un);
        const int sn = s_at(un);
#pragma unroll
        for (int k = 0; k < EW; ++k) {
          if (lv && ea_src) epa[v][k] = ld_relaxed_u64(ea_src + sn * ES + k);
          if (lv && ec_src) epc[v][k] = ld_relaxed_u64(ec_src + sn * ES + k);
        }
      }
      // Every thread passed row u - 1's barrier, so slot (u - 1) % D is free:
      // refill it with row u - 1 + D, before this row's barrier, from a lane
      // that waits on no c-face edge word in this direction.  (Refills
      // issued by thread 0 after each row's barrier -- of slot u % D, or of
      // slot (u - 1) % D -- gave solves that differed from run to run at 256
      // patches; this order repeats bit for bit.)
      if (tid == (BWD ? 31 : kPatchLines - 1) && u >= 1 && u - 1 + D < NR) issue(u - 1 + D);
      __syncthreads();
    }
  }
  if (gave_up) {
    // a wait gave up: give the copies still in flight into the ring time to
    // land (bounded) before the CTA exits
    for (int u = NR - D > 0 ? NR - D : 0; u < NR; ++u) {
      const unsigned bar = bar0 + 8 * (u % D);
      const unsigned par = (unsigned)(u / D) & 1u;
      const unsigned long long t0 = global_ns();
      while (!mbar_try_wait(bar, par) && global_ns() - t0 < kWaitNs) {
      }
    }
  }
  if (MODE == kForward && UPD && A.part) {
    const double m = block_max<double>((double)rmax, red);
    if (tid == 0) A.part[p] = m;
  }
  if (MODE == kBackward && A.part) {
    const double sm = block_sum<double>(dsum, red);
    if (tid == 0) A.part[p] = sm;
  }
  }  // run
  // every CTA counts, running or not; the last one reduces the partials
  if (A.done_ctr && A.part && ((MODE == kForward && UPD) || MODE == kBackward) &&
      last_block(A.done_ctr, nblocks)) {
    if (MODE == kForward)
      red_conv_body(A.part, A.npart, A.sc, red);
    else
      red_beta_body(A.part, A.npart, A.sc, red, A.red_init);
  }
  if (CL > 1) cluster_sync();
}

template <typename R, int MODE, bool UPD, int CC, int CA>
__global__ void __launch_bounds__(kPatchLines, 1)
    k_pencil_sweep(const PencilSweepArgs<R> A) {
  pencil_sweep_run<R, MODE, UPD, CC, CA>(A, (int)gridDim.x);
}

// The solve of block b in a launch over several solves: first[] holds each
// solve's first block (first[n] = the grid), so b lies in [first[s],
// first[s + 1]).
__device__ inline int batch_solve_of(const int* __restrict__ first, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(first + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One sweep launch over several solves (the shared solve of a batch of
// scenes): solve s owns first[s + 1] - first[s] CTAs (its patches, plain
// form) and its arguments come from tab[s].  Launch k of a chunk advances
// each solve's edge-word epoch by k and its ticket base by k launches of its
// patches, as k separate launches would.
template <typename R, int MODE, bool UPD>
__global__ void __launch_bounds__(kPatchLines, 1)
    k_pencil_sweep_batch(const PencilSweepArgs<R>* __restrict__ tab, const int* __restrict__ first,
                         int nsolve, int k) {
  const int s = batch_solve_of(first, nsolve, (int)blockIdx.x);
  PencilSweepArgs<R> A = tab[s];
  const int nb = __ldg(first + s + 1) - __ldg(first + s);
  A.epoch += (unsigned)k;
  A.ticket_base += k * nb;
  pencil_sweep_run<R, MODE, UPD, 1, 1>(A, nb);
}

// x += alpha s (the update of the last PCG iteration, which no SpMV follows)
template <typename R>
__global__ void k_pl_axpy(long long len, const double* __restrict__ sc, const R* __restrict__ s,
                          R* __restrict__ x) {
  const R al = (R)sc[S_ALPHA];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len;
       e += (long long)gridDim.x * blockDim.x)
    x[e] = x[e] + al * s[e];
}

// ---- streaming kernels over the pencil layout --------------------------------
// Element e -> (patch, row, line) and the cell's position in the box.
struct PlCell {
  long long p;
  int t, l, al, cl, PAi, PCi, s;
  bool live;
};

// Cell of line l in row `row` (= patch * R + t) of the layout; 32-bit math
// (npatch * R stays far below 2^31).
__device__ inline PlCell pl_cell(const PencilGeom& G, int row, int l) {
  PlCell c;
  const int p = row / G.R;
  c.p = p;
  c.t = row - p * G.R;
  c.l = l;
  c.al = l & (kPatch - 1);
  c.cl = l / kPatch;
  c.PAi = p % G.nPA;
  c.PCi = p / G.nPA;
  c.s = c.t - c.al - c.cl;
  c.live = c.s >= 0 && c.s < G.Ls && c.PAi * kPatch + c.al < G.NA &&
           c.PCi * kPatch + c.cl < G.NC;
  return c;
}

// Indices of the six neighbours of a live cell (-1 where the box ends).
struct PlNbr {
  long long ms, ps, ma, pa, mc, pc;
};

__device__ inline PlNbr pl_nbr(const PencilGeom& G, const PlCell& c, long long e) {
  PlNbr n;
  n.ms = c.s > 0 ? e - kPatchLines : -1;
  n.ps = c.s + 1 < G.Ls ? e + kPatchLines : -1;
  if (c.al > 0) n.ma = e - kPatchLines - 1;
  else n.ma = c.PAi > 0 ? pl_index(G, c.p - 1, c.t + kPatch - 1, c.l + kPatch - 1) : -1;
  if (c.al < kPatch - 1) n.pa = e + kPatchLines + 1;
  else n.pa = c.PAi + 1 < G.nPA ? pl_index(G, c.p + 1, c.t - (kPatch - 1), c.l - (kPatch - 1)) : -1;
  if (c.cl > 0) n.mc = e - kPatchLines - kPatch;
  else n.mc = c.PCi > 0 ? pl_index(G, c.p - G.nPA, c.t + kPatch - 1,
                                    c.l + kPatch * (kPatch - 1)) : -1;
  if (c.cl < kPatch - 1) n.pc = e + kPatchLines + kPatch;
  else n.pc = c.PCi + 1 < G.nPC ? pl_index(G, c.p + G.nPA, c.t - (kPatch - 1),
                                            c.l - kPatch * (kPatch - 1)) : -1;
  return n;
}

// s_new = z + beta s_old (at all 7 stencil points), q = A s_new,
// partial[block] = sum s_new.q.  Row order of the reference's sorted row for
// interior cells: -c, -a, -s, diagonal, +s, +a, +c.
//
// The previous iteration's x += alpha s_old is applied here too (alpha is
// still the previous iteration's when this kernel runs; 0 before the first).
//
// Block bid of nblk: the arithmetic of k_pl_spmv_s (below) for one solve of a
// launch over several solves (k_pl_spmv_batch).
template <typename R>
__device__ __forceinline__ void pl_spmv_run(
    const PencilGeom& G, const R* __restrict__ AD, const R* __restrict__ AS,
    const R* __restrict__ AA, const R* __restrict__ AC, const R* __restrict__ z,
    const R* __restrict__ sold, R* __restrict__ snew, R* __restrict__ q, R* __restrict__ x,
    double* __restrict__ sc, double* __restrict__ partial, int* __restrict__ done_ctr, int bid,
    int nblk) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  const R be = (R)sc[S_BETA];
  const R al = (R)sc[S_ALPHA];
  double acc = 0;
  const int nrow = (int)(G.npatch * G.R);
  for (int row = bid; row < nrow; row += nblk) {
    const long long e = (long long)row * kPatchLines + threadIdx.x;
    const PlCell c = pl_cell(G, row, threadIdx.x);
    if (!c.live) continue;
    const PlNbr n = pl_nbr(G, c, e);
    R r = 0;
    if (n.mc >= 0) r += AC[n.mc] * (z[n.mc] + be * sold[n.mc]);
    if (n.ma >= 0) r += AA[n.ma] * (z[n.ma] + be * sold[n.ma]);
    if (n.ms >= 0) r += AS[n.ms] * (z[n.ms] + be * sold[n.ms]);
    const R so = sold[e];
    x[e] = x[e] + al * so;
    const R sn = z[e] + be * so;
    r += AD[e] * sn;
    if (n.ps >= 0) r += AS[e] * (z[n.ps] + be * sold[n.ps]);
    if (n.pa >= 0) r += AA[e] * (z[n.pa] + be * sold[n.pa]);
    if (n.pc >= 0) r += AC[e] * (z[n.pc] + be * sold[n.pc]);
    snew[e] = sn;
    q[e] = r;
    acc += (double)sn * (double)r;
  }
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[bid] = acc;
  // the last block: alpha = rho / s.q (k_red_alpha's body)
  if (done_ctr && last_block(done_ctr, nblk)) red_alpha_body(partial, nblk, sc, sm);
}

// (written out rather than through pl_spmv_run: the launch alone ran about
// 10 % slower through the shared body)
template <typename R>
__global__ void __launch_bounds__(kRedThreads, sizeof(R) == 4 ? 8 : 4)
    k_pl_spmv_s(PencilGeom G, const R* __restrict__ AD, const R* __restrict__ AS,
                const R* __restrict__ AA, const R* __restrict__ AC, const R* __restrict__ z,
                const R* __restrict__ sold, R* __restrict__ snew, R* __restrict__ q,
                R* __restrict__ x, double* __restrict__ sc,
                double* __restrict__ partial, int* __restrict__ done_ctr) {
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  const R be = (R)sc[S_BETA];
  const R al = (R)sc[S_ALPHA];
  double acc = 0;
  const int nrow = (int)(G.npatch * G.R);
  for (int row = blockIdx.x; row < nrow; row += gridDim.x) {
    const long long e = (long long)row * kPatchLines + threadIdx.x;
    const PlCell c = pl_cell(G, row, threadIdx.x);
    if (!c.live) continue;
    const PlNbr n = pl_nbr(G, c, e);
    R r = 0;
    if (n.mc >= 0) r += AC[n.mc] * (z[n.mc] + be * sold[n.mc]);
    if (n.ma >= 0) r += AA[n.ma] * (z[n.ma] + be * sold[n.ma]);
    if (n.ms >= 0) r += AS[n.ms] * (z[n.ms] + be * sold[n.ms]);
    const R so = sold[e];
    x[e] = x[e] + al * so;
    const R sn = z[e] + be * so;
    r += AD[e] * sn;
    if (n.ps >= 0) r += AS[e] * (z[n.ps] + be * sold[n.ps]);
    if (n.pa >= 0) r += AA[e] * (z[n.pa] + be * sold[n.pa]);
    if (n.pc >= 0) r += AC[e] * (z[n.pc] + be * sold[n.pc]);
    snew[e] = sn;
    q[e] = r;
    acc += (double)sn * (double)r;
  }
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
  // the last block: alpha = rho / s.q (k_red_alpha's body)
  if (done_ctr && last_block(done_ctr, (int)gridDim.x))
    red_alpha_body(partial, (int)gridDim.x, sc, sm);
}

// Blocks of k_pl_spmv_s for a layout: about four rows per block, at most the
// resident capacity (kPlSpmvBlocks32).  The partial sums of s.q follow the
// block count, so a solve alone and in a launch over several solves use this
// same count and give the same bits.
__host__ __device__ inline int pl_spmv_blocks(const PencilGeom& G) {
  const long long nrow = G.npatch * G.R;
  const long long b = (nrow + 3) / 4;
  return (int)(b < 1 ? 1 : (b > kPlSpmvBlocks32 ? kPlSpmvBlocks32 : b));
}

// One SpMV launch over several solves: solve s owns first[s + 1] - first[s]
// blocks; iteration it of a chunk takes s_old / s_new from s0 / s1 by the
// solve's iteration parity.
template <typename R>
struct PlSpmvArgs {
  PencilGeom G;
  const R* AD;
  const R* AS;
  const R* AA;
  const R* AC;
  const R* z;
  R* s0;
  R* s1;
  R* q;
  R* x;
  double* sc;
  double* part;
  int* done_ctr;
  int parity;  // iterations the solve ran before the chunk, mod 2
};

template <typename R>
__global__ void __launch_bounds__(kRedThreads, sizeof(R) == 4 ? 6 : 3)
    k_pl_spmv_batch(const PlSpmvArgs<R>* __restrict__ tab, const int* __restrict__ first,
                    int nsolve, int it) {
  const int s = batch_solve_of(first, nsolve, (int)blockIdx.x);
  const PlSpmvArgs<R>& a = tab[s];
  const int b0 = __ldg(first + s);
  const bool odd = ((a.parity + it) & 1) != 0;
  pl_spmv_run<R>(a.G, a.AD, a.AS, a.AA, a.AC, a.z, odd ? a.s1 : a.s0, odd ? a.s0 : a.s1, a.q,
                 a.x, a.sc, a.part, a.done_ctr, (int)blockIdx.x - b0, __ldg(first + s + 1) - b0);
}

// status[6 s + j] = sc_s[S_RES + j] (residual, beta, tolerance, iteration,
// iteration limit, done) for each solve of a chunk
__global__ void k_pl_batch_status(double* const* __restrict__ scs, int nsolve,
                                  double* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * nsolve) status[i] = __ldcg(scs[i / 6] + S_RES + i % 6);
}

// k_pl_spmv_s's arithmetic, streamed: block (patch p, chunk k) walks rows
// [t0, t1) of one patch in order, one thread per line.  s_new of rows t - 1,
// t and t + 1 sits in a ring of three shared-memory rows and the couplings
// A_s, A_a, A_c of row t - 1 in a second ring, so every in-patch neighbour
// (one row back or ahead, the same line, line -+1 or line -+16) is read from
// shared memory and each value is loaded from global memory once; only the
// neighbours across a patch face (lines at a = 0 / 15, c = 0 / 15) are read
// from global memory as k_pl_spmv_s reads them.  Terms are summed in the same
// order as k_pl_spmv_s, missing neighbours skipped.  partial[block] = s_new.q
// over the chunk (blocks ordered patch-major, then chunk).
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_pl_spmv_stream(PencilGeom G, int rows_per_chunk, int nchunk, const R* __restrict__ AD,
                     const R* __restrict__ AS, const R* __restrict__ AA,
                     const R* __restrict__ AC, const R* __restrict__ z,
                     const R* __restrict__ sold, R* __restrict__ snew, R* __restrict__ q,
                     R* __restrict__ x, const double* __restrict__ sc,
                     double* __restrict__ partial) {
  __shared__ R ring[3][kPatchLines];
  __shared__ R cs[2][kPatchLines], ca[2][kPatchLines], cc[2][kPatchLines];
  __shared__ double sm[kRedThreads];
  if (*(const int*)(sc + S_DONE)) return;
  const R be = (R)sc[S_BETA];
  const R al = (R)sc[S_ALPHA];
  const int l = threadIdx.x;
  const int p = blockIdx.x / nchunk;
  const int k = blockIdx.x - p * nchunk;
  const int t0 = k * rows_per_chunk;
  const int t1 = min(G.R, t0 + rows_per_chunk);
  double acc = 0;
  if (t0 < t1) {
    const long long base = (long long)p * G.R * kPatchLines + l;
    // s_new and the couplings of row t0 - 1 (zero before the first row)
    if (t0 > 0) {
      const long long e = base + (long long)(t0 - 1) * kPatchLines;
      ring[(t0 + 2) % 3][l] = z[e] + be * sold[e];
      cs[(t0 + 1) & 1][l] = AS[e];
      ca[(t0 + 1) & 1][l] = AA[e];
      cc[(t0 + 1) & 1][l] = AC[e];
    } else {
      ring[2][l] = R(0);
      cs[1][l] = ca[1][l] = cc[1][l] = R(0);
    }
    // row t's own values and row t + 1's z, s_old, held one row ahead in
    // registers so the loads of the next row overlap this row's work
    long long e0 = base + (long long)t0 * kPatchLines;
    R nz = z[e0], ns = sold[e0];
    ring[t0 % 3][l] = nz + be * ns;
    R ad = AD[e0], as = AS[e0], aa = AA[e0], ac = AC[e0], so = ns, xv = x[e0];
    if (t0 + 1 < G.R) {
      nz = z[e0 + kPatchLines];
      ns = sold[e0 + kPatchLines];
    }
    for (int t = t0; t < t1; ++t) {
      const long long e = base + (long long)t * kPatchLines;
      if (t + 1 < G.R) ring[(t + 1) % 3][l] = nz + be * ns;
      cs[t & 1][l] = as;
      ca[t & 1][l] = aa;
      cc[t & 1][l] = ac;
      const R ns1 = ns;
      // prefetch: row t + 1's own values, row t + 2's z and s_old
      R ad_n = 0, as_n = 0, aa_n = 0, ac_n = 0, xv_n = 0;
      if (t + 1 < t1) {
        ad_n = AD[e + kPatchLines];
        as_n = AS[e + kPatchLines];
        aa_n = AA[e + kPatchLines];
        ac_n = AC[e + kPatchLines];
        xv_n = x[e + kPatchLines];
        if (t + 2 < G.R) {
          nz = z[e + 2 * kPatchLines];
          ns = sold[e + 2 * kPatchLines];
        }
      }
      __syncthreads();
      const PlCell c = pl_cell(G, p * G.R + t, l);
      if (c.live) {
        const R* sm1 = ring[(t + 2) % 3];
        const R* s0 = ring[t % 3];
        const R* sp1 = ring[(t + 1) % 3];
        const int pr = (t + 1) & 1;  // coupling ring slot of row t - 1
        R r = 0;
        // -c
        if (c.cl > 0) {
          r += cc[pr][l - kPatch] * sm1[l - kPatch];
        } else if (c.PCi > 0) {
          const long long n = pl_index(G, p - G.nPA, t + kPatch - 1, l + kPatch * (kPatch - 1));
          r += AC[n] * (z[n] + be * sold[n]);
        }
        // -a
        if (c.al > 0) {
          r += ca[pr][l - 1] * sm1[l - 1];
        } else if (c.PAi > 0) {
          const long long n = pl_index(G, p - 1, t + kPatch - 1, l + kPatch - 1);
          r += AA[n] * (z[n] + be * sold[n]);
        }
        // -s
        if (c.s > 0) r += cs[pr][l] * sm1[l];
        x[e] = xv + al * so;
        const R sn = s0[l];
        r += ad * sn;
        // +s
        if (c.s + 1 < G.Ls) r += as * sp1[l];
        // +a
        if (c.al < kPatch - 1) {
          r += aa * sp1[l + 1];
        } else if (c.PAi + 1 < G.nPA) {
          const long long n = pl_index(G, p + 1, t - (kPatch - 1), l - (kPatch - 1));
          r += aa * (z[n] + be * sold[n]);
        }
        // +c
        if (c.cl < kPatch - 1) {
          r += ac * sp1[l + kPatch];
        } else if (c.PCi + 1 < G.nPC) {
          const long long n = pl_index(G, p + G.nPA, t - (kPatch - 1), l - kPatch * (kPatch - 1));
          r += ac * (z[n] + be * sold[n]);
        }
        snew[e] = sn;
        q[e] = r;
        acc += (double)sn * (double)r;
      }
      ad = ad_n;
      as = as_n;
      aa = aa_n;
      ac = ac_n;
      xv = xv_n;
      so = ns1;
      __syncthreads();
    }
  }
  acc = block_sum<double>(acc, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// FP64 residual r64 = b - A x64 with the coefficients promoted; partial max|r64|
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_pl_residual64(PencilGeom G, const R* __restrict__ AD, const R* __restrict__ AS,
                    const R* __restrict__ AA, const R* __restrict__ AC,
                    const R* __restrict__ b, const double* __restrict__ x,
                    double* __restrict__ r, double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double m = 0;
  const int nrow = (int)(G.npatch * G.R);
  for (int row = blockIdx.x; row < nrow; row += gridDim.x) {
    const long long e = (long long)row * kPatchLines + threadIdx.x;
    const PlCell c = pl_cell(G, row, threadIdx.x);
    if (!c.live) continue;
    const PlNbr n = pl_nbr(G, c, e);
    double acc = (double)AD[e] * x[e];
    if (n.ms >= 0) acc += (double)AS[n.ms] * x[n.ms];
    if (n.ma >= 0) acc += (double)AA[n.ma] * x[n.ma];
    if (n.mc >= 0) acc += (double)AC[n.mc] * x[n.mc];
    if (n.ps >= 0) acc += (double)AS[e] * x[n.ps];
    if (n.pa >= 0) acc += (double)AA[e] * x[n.pa];
    if (n.pc >= 0) acc += (double)AC[e] * x[n.pc];
    const double rv = (double)b[e] - acc;
    r[e] = rv;
    const double av = fabs(rv);
    m = av > m ? av : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// r32 = r64 / res, x32 = 0 (inner solve of one refinement)
template <typename R>
__global__ void k_pl_demote(long long len, const double* __restrict__ r64,
                            const double* __restrict__ sc, R* __restrict__ r,
                            R* __restrict__ x) {
  const double scale = 1.0 / sc[0];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len;
       e += (long long)gridDim.x * blockDim.x) {
    r[e] = (R)(r64[e] * scale);
    x[e] = R(0);
  }
}

// x64 += x32 * res
template <typename R>
__global__ void k_pl_accumulate(long long len, const R* __restrict__ x,
                                const double* __restrict__ sc, double* __restrict__ x64) {
  const double s = sc[0];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len;
       e += (long long)gridDim.x * blockDim.x)
    x64[e] += (double)x[e] * s;
}

// r64 = b (promoted)
template <typename R>
__global__ void k_pl_promote(long long len, const R* __restrict__ b, double* __restrict__ o) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len;
       e += (long long)gridDim.x * blockDim.x)
    o[e] = (double)b[e];
}

// The DOF box: block-reduced min/max of the DOF cell coordinates into
// bbox[0..5] (min x,y,z, max x,y,z) and the DOF count into partial[block].
__global__ void __launch_bounds__(kRedThreads)
    k_dof_box(GridDesc g, const int* __restrict__ active_list, long long nent,
              const unsigned char* __restrict__ dof, int* __restrict__ bbox,
              double* __restrict__ partial) {
  __shared__ int smn[3][kRedThreads / 32], smx[3][kRedThreads / 32];
  __shared__ double sm[kRedThreads];
  int mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
  double cnt = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    if (!(dof[n] & 1)) continue;
    int I, J, K;
    node_ijk(g, n, I, J, K);
    const int v[3] = {I, J, K};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = v[a] < mn[a] ? v[a] : mn[a];
      mx[a] = v[a] > mx[a] ? v[a] : mx[a];
    }
    cnt += 1.0;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int wmn = __reduce_min_sync(0xffffffffu, mn[a]);
    const int wmx = __reduce_max_sync(0xffffffffu, mx[a]);
    if (lane == 0) { smn[a][wid] = wmn; smx[a][wid] = wmx; }
  }
  cnt = block_sum<double>(cnt, sm);  // contains __syncthreads
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = cnt;
    for (int a = 0; a < 3; ++a) {
      int bmn = 1 << 30, bmx = -1;
      for (int w = 0; w < kRedThreads / 32; ++w) {
        bmn = smn[a][w] < bmn ? smn[a][w] : bmn;
        bmx = smx[a][w] > bmx ? smx[a][w] : bmx;
      }
      if (bmx >= 0) {
        atomicMin(bbox + a, bmn);
        atomicMax(bbox + 3 + a, bmx);
      }
    }
  }
}

// Gather the assembled system into the pencil layout.  Couplings are kept
// only between two DOF cells (the reference's matrix has no other entries).
template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_pl_gather(PencilGeom G, GridDesc g, const unsigned char* __restrict__ active,
                const unsigned char* __restrict__ dof, const R* __restrict__ F,
                long long fs, R* __restrict__ AD, R* __restrict__ AS, R* __restrict__ AA,
                R* __restrict__ AC, R* __restrict__ B) {
  const int nrow = (int)(G.npatch * G.R);
  for (int row = blockIdx.x; row < nrow; row += gridDim.x) {
    const long long e = (long long)row * kPatchLines + threadIdx.x;
    const PlCell c = pl_cell(G, row, threadIdx.x);
    R ad = 0, as = 0, aa = 0, ac = 0, bv = 0;
    if (c.live) {
      int P[3];
      P[G.ax_s] = G.lo[G.ax_s] + c.s;
      P[G.ax_a] = G.lo[G.ax_a] + c.PAi * kPatch + c.al;
      P[G.ax_c] = G.lo[G.ax_c] + c.PCi * kPatch + c.cl;
      if (in_grid(g, P[0], P[1], P[2]) && active[bucket_of(g, P[0], P[1], P[2])]) {
        const long long n = node_linear(g, P[0], P[1], P[2]);
        if (dof[n] & 1) {
          ad = F[G_ADIAG * fs + n];
          bv = F[G_B * fs + n];
          const int axes[3] = {G.ax_s, G.ax_a, G.ax_c};
          R cpl[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            int Q[3] = {P[0], P[1], P[2]};
            Q[axes[k]] += 1;
            cpl[k] = R(0);
            if (in_grid(g, Q[0], Q[1], Q[2]) && active[bucket_of(g, Q[0], Q[1], Q[2])] &&
                (dof[node_linear(g, Q[0], Q[1], Q[2])] & 1))
              cpl[k] = F[(G_AX + axes[k]) * fs + n];
          }
          as = cpl[0]; aa = cpl[1]; ac = cpl[2];
        }
      }
    }
    AD[e] = ad; AS[e] = as; AA[e] = aa; AC[e] = ac; B[e] = bv;
  }
}

// pressure of every active node from the pencil solution (0 off the DOFs)
template <typename R>
__global__ void k_pl_scatter_pressure(PencilGeom G, GridDesc g, const int* __restrict__ active_list,
                                      long long nent, const unsigned char* __restrict__ dof,
                                      const R* __restrict__ x32, const double* __restrict__ x64,
                                      R* __restrict__ p) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const long long n = active_node(active_list, e);
    R v = R(0);
    if (dof[n] & 1) {
      int P[3];
      node_ijk(g, n, P[0], P[1], P[2]);
      const int s = P[G.ax_s] - G.lo[G.ax_s];
      const int a = P[G.ax_a] - G.lo[G.ax_a];
      const int c = P[G.ax_c] - G.lo[G.ax_c];
      const int PAi = a / kPatch, al = a - PAi * kPatch;
      const int PCi = c / kPatch, cl = c - PCi * kPatch;
      const long long idx = pl_index(G, (long long)PCi * G.nPA + PAi, s + al + cl, al + kPatch * cl);
      v = x64 ? (R)x64[idx] : x32[idx];
    }
    p[n] = v;
  }
}

}  // namespace wcg
