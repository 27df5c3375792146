// Particle merge: TwoDScene::updateOptiVolume / relabelLiquidParticles
// (TwoDScene.cpp:2484-2505), mergeLiquidParticles (:2510-2666) and
// removeEmptyParticles (:1713-1745), in a deterministic, seeded form.
//
// The reference visits the buckets of its last sort (the previous grid build)
// in the 27 colours of Sorter::for_each_bucket_particles_colored_randomized
// (Sorter.h:439-480, numcolors 3) and each bucket's particles in index order.
// Buckets of one colour are three apart, so the 27-bucket neighbourhoods a
// colour reads and writes do not overlap: one thread per bucket of the colour
// reproduces the serial order, and a launch per colour orders the colours.
// The subset selector and the colour order are rand() draws in the reference;
// here they are arguments (wcg_merge_draws gives the seeded stream).
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_correct.cuh"
#include "wcg_kernels.cuh"

namespace wcg {

// particle classes of relabelLiquidParticles (TwoDScene.h:31)
enum : unsigned char { PCL_NONE = 0, PCL_S, PCL_s, PCL_o, PCL_l, PCL_L };

template <typename R>
__device__ inline unsigned char particle_class(R vol, double vf) {
  const double mrel = (double)vol / vf;
  return mrel < 0.5 ? PCL_S : mrel <= 0.9 ? PCL_s : mrel <= 1.1 ? PCL_o : mrel <= 2.0 ? PCL_l : PCL_L;
}

// classes, the bucket of the last build as a sort key, cleared merge sums;
// count per bucket
template <typename R>
__global__ void k_merge_setup(const R* __restrict__ P, long long pcap, long long np,
                              const int* __restrict__ pbucket, long long nb, double vf,
                              unsigned char* __restrict__ cls, unsigned char* __restrict__ removed,
                              R* __restrict__ gvol, R* __restrict__ gmom,
                              long long* __restrict__ key, int* __restrict__ count) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  cls[s] = particle_class<R>(P[PV * pcap + s], vf);
  removed[s] = 0;
  gvol[s] = R(0);
  for (int a = 0; a < 3; ++a) gmom[a * pcap + s] = R(0);
  const int b = pbucket[s];
  if (b < 0 || b >= nb) {
    key[s] = -1;
    return;
  }
  key[s] = b;
  atomicAdd(&count[b], 1);
}

struct MergeArgs {
  GridDesc g;        // bucket grid of the last build
  int selector, step, ne;
  double vf, should_rad;
  const int* pid;
  const int* list;   // slots by bucket, index order inside a bucket
  const int* start;  // per bucket, nb + 1
};

// one colour (cr, cs, ct) of the merge: a thread per bucket of the colour
template <typename R>
__global__ void __launch_bounds__(128)
    k_merge(MergeArgs A, int cr, int cs, int ct, R* P, long long pcap, unsigned char* cls,
            unsigned char* removed, R* gvol, R* gmom) {
  const GridDesc& g = A.g;
  const int sn0 = (g.ni + 2) / 3, sn1 = (g.nj + 2) / 3, sn2 = (g.nk + 2) / 3;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)sn0 * sn1 * sn2) return;
  const int sk = (int)(t / ((long long)sn0 * sn1));
  const int sj = (int)((t - (long long)sk * sn0 * sn1) / sn0);
  const int si = (int)(t - (long long)sk * sn0 * sn1 - (long long)sj * sn0);
  const int i = si * 3 + cr, j = sj * 3 + cs, k = sk * 3 + ct;
  if (i >= g.ni || j >= g.nj || k >= g.nk) return;
  const long long b = ((long long)k * g.nj + j) * g.ni + i;
  const int q1 = A.start[b + 1];
  for (int q = A.start[b]; q < q1; ++q) {
    const int s = A.list[q];
    const unsigned char c0 = cls[s];
    if (c0 != PCL_S && c0 != PCL_l) continue;
    if ((A.ne + A.pid[s]) % A.step != A.selector) continue;
    const bool small = c0 == PCL_S;
    const R vol0 = P[PV * pcap + s];
    const R full_vol = vol0 + gvol[s];
    if (!small && full_vol < R(1e-20)) continue;
    const R mrel = full_vol / (R)A.vf;
    if (small && mrel >= R(0.5)) {
      cls[s] = PCL_s;
      continue;
    }
    if (!small && mrel > R(2)) {
      cls[s] = PCL_L;
      continue;
    }
    const R px = P[PX * pcap + s], py = P[PY * pcap + s], pz = P[PZ * pcap + s];
    // partners in the 27 buckets around (x outermost, Sorter.h:352-371),
    // counted first, then served with the same test
    int npart = 0;
    for (int pass = 0; pass < 2; ++pass) {
      R dvol = 0, dm[3] = {0, 0, 0};
      if (pass == 1) {
        if (npart == 0) break;
        const R invN = R(1) / (R)npart;
        R f;
        if (small) {
          dvol = full_vol * invN;
          f = invN;
        } else {
          const R ex_vol = full_vol - (R)A.vf;
          dvol = ex_vol * invN;
          f = dvol / full_vol;
        }
        for (int a = 0; a < 3; ++a) dm[a] = (P[(VX + a) * pcap + s] * vol0 + gmom[a * pcap + s]) * f;
      }
      for (int x = i - 1; x <= i + 1; ++x)
        for (int y = j - 1; y <= j + 1; ++y)
          for (int z = k - 1; z <= k + 1; ++z) {
            if (x < 0 || x > g.ni - 1 || y < 0 || y > g.nj - 1 || z < 0 || z > g.nk - 1) continue;
            const long long nbk = ((long long)z * g.nj + y) * g.ni + x;
            const int r1 = A.start[nbk + 1];
            for (int r = A.start[nbk]; r < r1; ++r) {
              const int n = A.list[r];
              if (n == s || removed[n]) continue;
              const unsigned char c2 = cls[n];
              if (small ? !(c2 == PCL_S || c2 == PCL_s || c2 == PCL_o) : c2 != PCL_s) continue;
              if (P[PV * pcap + n] + gvol[n] > (R)A.vf) continue;
              const R d0 = px - P[PX * pcap + n], d1 = py - P[PY * pcap + n],
                      d2 = pz - P[PZ * pcap + n];
              const R dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
              if (!(dist < (R)A.should_rad)) continue;
              if (pass == 0) {
                ++npart;
              } else {
                gvol[n] += dvol;
                for (int a = 0; a < 3; ++a) gmom[a * pcap + n] += dm[a];
              }
            }
          }
    }
    if (npart == 0) continue;
    if (small) {
      removed[s] = 1;
      P[PV * pcap + s] = R(0);
      gvol[s] = R(0);
      for (int a = 0; a < 3; ++a) gmom[a * pcap + s] = R(0);
    } else {
      const R scaling = (R)A.vf / full_vol;
      const R rad_scaling = pow(scaling, R(1) / R(3));
      P[PV * pcap + s] = vol0 * scaling;
      P[PM * pcap + s] = P[PM * pcap + s] * scaling;
      P[PR * pcap + s] = P[PR * pcap + s] * rad_scaling;
      cls[s] = PCL_o;
    }
  }
}

// gather and update (TwoDScene.cpp:2649-2666); then alive flags by original
// index (fluid volume >= 1e-20, removeEmptyParticles' test)
template <typename R>
__global__ void k_merge_gather(R* __restrict__ P, long long pcap, long long np,
                               const int* __restrict__ pid, const unsigned char* __restrict__ removed,
                               const R* __restrict__ gvol, const R* __restrict__ gmom, double rho,
                               int* __restrict__ alive_slot, int* __restrict__ alive_pid) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  if (!removed[s] && gvol[s] != R(0)) {
    const R vol = P[PV * pcap + s];
    R fm[3];
    for (int a = 0; a < 3; ++a) fm[a] = P[(VX + a) * pcap + s] * vol + gmom[a * pcap + s];
    const R full_vol = vol + gvol[s];
    const R full_rad = pow(full_vol * R(0.75) / R(M_PI), R(1) / R(3));
    const R inv = R(1) / full_vol;
    P[PV * pcap + s] = full_vol;
    for (int a = 0; a < 3; ++a) P[(VX + a) * pcap + s] = fm[a] * inv;
    P[PM * pcap + s] = full_vol * (R)rho;
    P[PR * pcap + s] = full_rad;
  }
  const int al = P[PV * pcap + s] < R(1e-20) ? 0 : 1;
  alive_slot[s] = al;
  alive_pid[pid[s]] = al;
}

// TwoDScene::terminateParticles (TwoDScene.cpp:1756-1771): a liquid particle
// where the terminator shapes' phi (the running minimum of computePhiVel over
// the terminator groups) is negative loses its fluid volume; every particle
// without volume (below 1e-20, removeEmptyParticles) is flagged for removal
template <typename R>
__global__ void k_terminate(R* __restrict__ P, long long pcap, long long np,
                            const int* __restrict__ pid, const TermSet term, double three_bs,
                            int* __restrict__ alive_slot, int* __restrict__ alive_pid) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  if (term.n > 0 && term_phi(term, (double)P[PX * pcap + s], (double)P[(PX + 1) * pcap + s],
                             (double)P[(PX + 2) * pcap + s], three_bs) < 0.0)
    P[PV * pcap + s] = R(0);
  const int al = P[PV * pcap + s] < R(1e-20) ? 0 : 1;
  alive_slot[s] = al;
  alive_pid[pid[s]] = al;
}

// the swap-with-last removal as a map of original indices: the holes below
// K (the survivor count) in ascending order take the survivors at K and
// above in descending order.  hole_flag / high_flag per original index.
__global__ void k_merge_flags(long long np, long long K, const int* __restrict__ alive_pid,
                              int* __restrict__ hole_flag, int* __restrict__ high_flag) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int al = alive_pid[i];
  hole_flag[i] = (i < K && !al) ? 1 : 0;
  high_flag[i] = (i >= K && al) ? 1 : 0;
}

__global__ void k_merge_holes(long long np, long long K, const int* __restrict__ alive_pid,
                              const int* __restrict__ hole_rank, int* __restrict__ holes) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np || i >= K || alive_pid[i]) return;
  holes[hole_rank[i]] = (int)i;
}

// new original index of each surviving slot after compaction (perm: slot ->
// old slot); nhigh = survivors at K and above
__global__ void k_merge_repid(long long K, const int* __restrict__ perm,
                              const int* __restrict__ pid_old, const int* __restrict__ high_rank,
                              const int* __restrict__ holes, int nhigh, int* __restrict__ pid_new) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= K) return;
  const int i = pid_old[perm[s]];
  pid_new[s] = i < K ? i : holes[nhigh - 1 - high_rank[i]];
}

// alive flag per slot again (the slot array was scanned in place)
__global__ void k_merge_alive_slots(long long np, const int* __restrict__ pid,
                                    const int* __restrict__ alive_pid, int* __restrict__ out) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  out[s] = alive_pid[pid[s]];
}

// surviving slots in order
__global__ void k_merge_compact(long long np, const int* __restrict__ alive_slot,
                                const int* __restrict__ rank, int* __restrict__ perm) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np || !alive_slot[s]) return;
  perm[rank[s]] = (int)s;
}

// ---- particle split: TwoDScene::splitLiquidParticles (TwoDScene.cpp:2362-2480)

// point i of n on the unit sphere (spherical Fibonacci lattice)
__host__ __device__ inline void sphere_point(int n, int i, double* p) {
  const double y = 1.0 - (2.0 * i + 1.0) / (double)n;
  const double r = sqrt(1.0 - y * y);
  const double phi = (double)i * 2.3999632297286533;
  p[0] = r * cos(phi);
  p[1] = y;
  p[2] = r * sin(phi);
}

// rotation of a split parent: a uniform random unit quaternion (Shoemake,
// Graphics Gems III, 1992) from SplitMix64 draws of key
__host__ __device__ inline void split_rotation(unsigned long long key, double* Q) {
  unsigned long long z = splitmix64(key);
  const double u1 = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  z = splitmix64(z);
  const double u2 = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  z = splitmix64(z);
  const double u3 = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  const double a = sqrt(1.0 - u1), b = sqrt(u1);
  const double tp = 6.283185307179586;
  const double w = a * sin(tp * u2), x = a * cos(tp * u2), y = b * sin(tp * u3),
               zq = b * cos(tp * u3);
  Q[0] = 1.0 - 2.0 * (y * y + zq * zq);
  Q[1] = 2.0 * (x * y - zq * w);
  Q[2] = 2.0 * (x * zq + y * w);
  Q[3] = 2.0 * (x * y + zq * w);
  Q[4] = 1.0 - 2.0 * (x * x + zq * zq);
  Q[5] = 2.0 * (y * zq - x * w);
  Q[6] = 2.0 * (x * zq - y * w);
  Q[7] = 2.0 * (y * zq + x * w);
  Q[8] = 1.0 - 2.0 * (x * x + y * y);
}

// children per large particle, n = min(ceil(V / V_fine), 32), by slot and by
// original index
template <typename R>
__global__ void k_split_count(const R* __restrict__ P, long long pcap, long long np,
                              const int* __restrict__ pid, double vf, int* __restrict__ add_slot,
                              int* __restrict__ add_pid) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const R vol = P[PV * pcap + s];
  int add = 0;
  if (particle_class<R>(vol, vf) == PCL_L) {
    int n = (int)ceil((double)vol / vf);
    n = n > 32 ? 32 : n;
    add = n > 1 ? n - 1 : 0;
  }
  add_slot[s] = add;
  add_pid[pid[s]] = add;
}

// the parent moves to centre + p_0 s and takes volume V/n; its children are
// appended at np + (exclusive sum of the children of lower original index)
//
// With `pattern` given, the children sit as the reference places them: the
// caller's sphere-pattern table (points of n = 2..32, 3n doubles each,
// concatenated; TwoDScene::m_sphere_pattern) and one caller rotation per
// splitting parent (row-major, parents ranked by original index in
// `rank_pid`; the Q of the QR decomposition of the reference's
// Matrix3s::Random(), TwoDScene.cpp:2390-2402).
template <typename R>
__global__ void k_split(R* P, long long pcap, long long np, int* pid,
                        const int* __restrict__ add_slot, const int* __restrict__ off_pid,
                        unsigned long long key, double rho,
                        const double* __restrict__ pattern = nullptr,
                        const double* __restrict__ rot = nullptr,
                        const int* __restrict__ rank_pid = nullptr) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const int add = add_slot[s];
  if (add == 0) return;
  const int f = pid[s];
  const int n = add + 1;
  const double c[3] = {(double)P[PX * pcap + s], (double)P[PY * pcap + s],
                       (double)P[PZ * pcap + s]};
  const double rad = (double)P[PR * pcap + s];
  const double new_vol = (double)P[PV * pcap + s] / (double)n;
  const double new_rad = pow(new_vol / M_PI * 0.75, 1.0 / 3.0);
  const double splat = (new_rad > rad - new_rad ? new_rad : rad - new_rad) * 0.75;
  double Q[9];
  const double* pat = pattern ? pattern + 3 * ((n - 1) * n / 2 - 1) : nullptr;
  if (pattern)
    for (int r = 0; r < 9; ++r) Q[r] = rot[(long long)rank_pid[f] * 9 + r];
  else
    split_rotation(splitmix64(key ^ (unsigned long long)f), Q);
  const long long base = np + off_pid[f];
  for (int i = 1; i < n; ++i) {
    double pt[3];
    if (pat) {
      pt[0] = pat[3 * i];
      pt[1] = pat[3 * i + 1];
      pt[2] = pat[3 * i + 2];
    } else {
      sphere_point(n, i, pt);
    }
    const long long q = base + i - 1;
    for (int a = 0; a < 3; ++a) {
      const double rq = Q[a * 3] * pt[0] + Q[a * 3 + 1] * pt[1] + Q[a * 3 + 2] * pt[2];
      P[(PX + a) * pcap + q] = (R)(c[a] + rq * splat);
      P[(VX + a) * pcap + q] = P[(VX + a) * pcap + s];
    }
    for (int r = 0; r < 9; ++r) P[(C00 + r) * pcap + q] = R(0);
    P[PM * pcap + q] = (R)(new_vol * rho);
    P[PV * pcap + q] = (R)new_vol;
    P[PR * pcap + q] = (R)new_rad;
    pid[q] = (int)q;
  }
  double p0[3];
  if (pat) {
    p0[0] = pat[0];
    p0[1] = pat[1];
    p0[2] = pat[2];
  } else {
    sphere_point(n, 0, p0);
  }
  for (int a = 0; a < 3; ++a) P[(PX + a) * pcap + s] = (R)(c[a] + p0[a] * splat);
  P[PR * pcap + s] = (R)new_rad;
  P[PV * pcap + s] = (R)new_vol;
  P[PM * pcap + s] = (R)(new_vol * rho);
}

// 1 for a splitting parent (by original index), for the ranks of k_split
__global__ void k_split_parent_flag(long long np, const int* __restrict__ add_pid,
                                    int* __restrict__ flag) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < np) flag[i] = add_pid[i] > 0 ? 1 : 0;
}

// bucket of every particle's current position in the last build's bucket grid
// (the re-sort at the end of splitLiquidParticles, TwoDScene.cpp:2471-2478)
template <typename R>
__global__ void k_rebucket(const R* __restrict__ P, long long pcap, long long np, GridDesc g,
                           int* __restrict__ pbucket) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const int nbk[3] = {g.ni, g.nj, g.nk};
  int h[3];
  for (int a = 0; a < 3; ++a) {
    int v = (int)floor(div_rn(sub_rn(P[(PX + a) * pcap + s], org[a]), (R)g.bs));
    h[a] = v < 0 ? 0 : (v > nbk[a] - 1 ? nbk[a] - 1 : v);
  }
  pbucket[s] = (h[2] * g.nj + h[1]) * g.ni + h[0];
}

}  // namespace wcg
