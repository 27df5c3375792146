// Elasto (cloth / yarn) particle transfers: the !isFluid branches of
// TwoDScene::mapParticleNodesAPIC (TwoDScene.cpp:6686-6699, :6774-6787,
// :6862-6875), mapParticleSaturationPsiNodes (:5952-5992),
// updatePorePressureNodes (:5933-5950), mapNodeParticlesAPIC (:7023-7088) and
// SceneStepper::advectScene (SceneStepper.cpp:17-41).
//
// Elasto particles live in their own SoA (ECol), sorted by key cell like the
// liquid ones, so the liquid kernels are untouched and a liquid-only scene
// pays nothing.  The node sums are gathers in fixed particle order, as in
// k_p2g: deterministic, no atomics.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_kernels.cuh"
#include "wcg_pcg.cuh"

namespace wcg {

// Elasto SoA from the host-packed double columns (column-major, n per column).
template <typename R>
__global__ void k_load_elasto(long long n, long long ecap, const double* __restrict__ src,
                              R* __restrict__ E, int* __restrict__ pid) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll 4
  for (int c = 0; c < kNumECols; ++c) E[c * ecap + i] = (R)src[c * n + i];
  pid[i] = (int)i;
}

template <typename R>
__global__ void k_gather_elasto(const int* __restrict__ perm, long long n, long long ecap,
                                const R* __restrict__ src, R* __restrict__ dst,
                                const int* __restrict__ pid_src, int* __restrict__ pid_dst,
                                const long long* __restrict__ key_src,
                                long long* __restrict__ key_dst,
                                const int* __restrict__ delta_src, int* __restrict__ delta_dst) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = perm[s];
#pragma unroll 4
  for (int c = 0; c < kNumECols; ++c) dst[c * ecap + s] = src[c * ecap + i];
  pid_dst[s] = pid_src[i];
  key_dst[s] = key_src[i];
  delta_dst[s] = delta_src[i];
}

__global__ void k_permute_int(const int* __restrict__ perm, long long n,
                              const int* __restrict__ src, int* __restrict__ dst) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) dst[s] = src[perm[s]];
}

// Sorted state back to the reference's layouts, original order.
template <typename R>
__global__ void k_store_elasto(long long n, long long ecap, const R* __restrict__ E,
                               const int* __restrict__ pid, double* __restrict__ x4,
                               double* __restrict__ v4, double* __restrict__ B9) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long long i = pid[s];
  for (int a = 0; a < 4; ++a) {
    x4[i * 4 + a] = (double)E[(EX + a) * ecap + s];
    v4[i * 4 + a] = (double)E[(EVX + a) * ecap + s];
  }
  for (int q = 0; q < 9; ++q) B9[i * 9 + q] = (double)E[(EB00 + q) * ecap + s];
}

// positions (twist included) from the reference's m_x layout, original order
template <typename R>
__global__ void k_set_elasto_positions(long long n, long long ecap, R* __restrict__ E,
                                       const int* __restrict__ pid,
                                       const double* __restrict__ x4) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long long i = pid[s];
  for (int a = 0; a < 4; ++a) E[(EX + a) * ecap + s] = (R)x4[i * 4 + a];
}

// max |v|^2 over soft elasto particles (TwoDScene::getMaxVelocity :4171-4178)
template <typename R>
__global__ void k_maxvel2_elasto(const R* __restrict__ E, long long ecap, long long n,
                                 double* __restrict__ partial) {
  __shared__ double sm[kRedThreads];
  double m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (E[ESURF * ecap + i] != R(0)) continue;
    const double vx = E[EVX * ecap + i], vy = E[EVY * ecap + i], vz = E[EVZ * ecap + i];
    const double s = (vx * vx + vy * vy) + vz * vz;
    m = s > m ? s : m;
  }
  m = block_max<double>(m, sm);
  if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

// ---- P2G, solid phase -------------------------------------------------------
// Per face node, over the elasto particles whose stencil holds it:
//   p += (v_a + B.row(a).(x_n - x_p)) (m_a + m_fluid_a) w;  m += (m_a + m_fluid_a) w
// and, for particles that are not surfels,
//   V_s += (V_rest phi_rest) w;  V_fe += V_fluid w;  sf += shape_factor w;
//   rw += w;  o += orientation w.
// Then vel = p/m (m > 1e-20), vol = V_s + V_fe, psi = clamp(V_s/dV),
// sat = clamp((V_f + V_fe)/max(1e-20, dV - V_s)) with the liquid V_f that
// k_p2g left in G_VOL, sf /= rw (rw > 1e-20), o /= |o| (|o| > 1e-20).
// Per cell centre (mapParticleSaturationPsiNodes, surfels skipped):
//   V_l += V_fluid w;  V_s += V_rest w phi_rest;  psi_p = clamp(V_s/dV),
//   sat_p = clamp((V_l,liquid + V_l)/max(1e-20, dV - V_s)) with the liquid sum
//   k_p2g left in G_SATP; pore pressure = capillary(psi_p) (1 - sat_p),
//   capillary(psi) = psi/(1-psi) * sigma * cos(theta) / r_pore
//   (getCapillaryPressure :563-570).
// Block: one active bucket; threads [0,64) u, [64,128) v, [128,192) w faces,
// [192,256) cell centres.
template <typename R>
__global__ void __launch_bounds__(256)
    k_p2g_elasto(GridDesc g, const int* __restrict__ active_list, const R* __restrict__ E,
                 long long ecap, const int* __restrict__ start, const int* __restrict__ delta,
                 DeltaRange dr, R* __restrict__ F, long long fstride, R* __restrict__ EF,
                 double surf_tension, double cos_contact, double pore_radius) {
  const int b = active_list[blockIdx.x];
  const int type = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const int IJK[3] = {I, J, K};
  const R* px = E + EX * ecap;
  const R* py = E + EY * ecap;
  const R* pz = E + EZ * ecap;
  const R* surf = E + ESURF * ecap;
  const R* rv = E + ERV * ecap;
  const R* rf = E + ERF * ecap;
  const R* fv = E + EFV * ecap;
  const R dV = dx * dx * dx;

  if (type < 3) {
    const int a = type;
    R np_[3];
    for (int q = 0; q < 3; ++q)
      np_[q] = coord<R>(org[q], bs, dx, IJK[q], q == a ? R(0) : R(0.5));
    int lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
      if (q == a) {
        lo[q] = IJK[q] - 1 - dr.hi[q];
        hi[q] = IJK[q] + 1 - dr.lo[q];
      } else {
        lo[q] = IJK[q] - 1;
        hi[q] = IJK[q] + 1;
      }
      lo[q] = lo[q] < 0 ? 0 : lo[q];
    }
    hi[0] = hi[0] > g.NI - 1 ? g.NI - 1 : hi[0];
    hi[1] = hi[1] > g.NJ - 1 ? g.NJ - 1 : hi[1];
    hi[2] = hi[2] > g.NK - 1 ? g.NK - 1 : hi[2];
    const R* va = E + (EVX + a) * ecap;
    const R* b0 = E + (EB00 + 3 * a) * ecap;
    const R* b1 = E + (EB00 + 3 * a + 1) * ecap;
    const R* b2 = E + (EB00 + 3 * a + 2) * ecap;
    const R* ma = E + (EM0 + a) * ecap;
    const R* sf = E + ESF * ecap;
    const R* ox = E + EOX * ecap;
    const R* oy = E + EOY * ecap;
    const R* oz = E + EOZ * ecap;
    R mom = 0, mass = 0, vs = 0, vfe = 0, shp = 0, shw = 0, o0 = 0, o1 = 0, o2 = 0;
    for (int KZ = lo[2]; KZ <= hi[2]; ++KZ)
      for (int KY = lo[1]; KY <= hi[1]; ++KY)
        for (int KX = lo[0]; KX <= hi[0]; ++KX) {
          const long long c = node_linear(g, KX, KY, KZ);
          const int s1 = start[c + 1];
          const int Ka = a == 0 ? KX : (a == 1 ? KY : KZ);
          for (int s = start[c]; s < s1; ++s) {
            const int base = Ka - 1 + unpack_delta(delta[s], a);
            const int off = IJK[a] - base;
            if (off < 0 || off > 2) continue;
            const R x = px[s], y = py[s], z = pz[s];
            const R w = quad_kernel<R>((x - np_[0]) * invh) *
                        quad_kernel<R>((y - np_[1]) * invh) *
                        quad_kernel<R>((z - np_[2]) * invh);
            if (!(w > R(0))) continue;
            const R m = ma[s];
            const R vel = va[s] + (b0[s] * (np_[0] - x) + b1[s] * (np_[1] - y)) +
                          b2[s] * (np_[2] - z);
            mom += vel * m * w;
            mass += m * w;
            if (surf[s] == R(0)) {
              vs += rv[s] * rf[s] * w;
              vfe += fv[s] * w;
              shp += sf[s] * w;
              shw += w;
              o0 += ox[s] * w;
              o1 += oy[s] * w;
              o2 += oz[s] * w;
            }
          }
        }
    EF[(E_MASS + a) * fstride + n] = mass;
    EF[(E_VEL + a) * fstride + n] = mass > R(1e-20) ? mom / mass : R(0);
    EF[(E_VOL + a) * fstride + n] = vs + vfe;
    EF[(E_PSI + a) * fstride + n] = clamp01<R>(vs / dV);
    const R vf = F[(G_VOL + a) * fstride + n];
    const R room = dV - vs;
    F[(G_SAT + a) * fstride + n] = clamp01<R>((vf + vfe) / (room > R(1e-20) ? room : R(1e-20)));
    EF[(E_SF + a) * fstride + n] = shw > R(1e-20) ? shp / shw : shp;
    const R len = sqrt((o0 * o0 + o1 * o1) + o2 * o2);
    if (len > R(1e-20)) {
      o0 /= len;
      o1 /= len;
      o2 /= len;
    }
    EF[(E_ORI + 3 * a) * fstride + n] = o0;
    EF[(E_ORI + 3 * a + 1) * fstride + n] = o1;
    EF[(E_ORI + 3 * a + 2) * fstride + n] = o2;
  } else {
    R np_[3];
    for (int q = 0; q < 3; ++q) np_[q] = coord<R>(org[q], bs, dx, IJK[q], R(0.5));
    R vl = 0, vs = 0;
    const int lo0 = I - 1 < 0 ? 0 : I - 1, hi0 = I + 1 > g.NI - 1 ? g.NI - 1 : I + 1;
    const int lo1 = J - 1 < 0 ? 0 : J - 1, hi1 = J + 1 > g.NJ - 1 ? g.NJ - 1 : J + 1;
    const int lo2 = K - 1 < 0 ? 0 : K - 1, hi2 = K + 1 > g.NK - 1 ? g.NK - 1 : K + 1;
    for (int KZ = lo2; KZ <= hi2; ++KZ)
      for (int KY = lo1; KY <= hi1; ++KY)
        for (int KX = lo0; KX <= hi0; ++KX) {
          const long long c = node_linear(g, KX, KY, KZ);
          const int s1 = start[c + 1];
          for (int s = start[c]; s < s1; ++s) {
            if (surf[s] != R(0)) continue;
            const R w = quad_kernel<R>((px[s] - np_[0]) * invh) *
                        quad_kernel<R>((py[s] - np_[1]) * invh) *
                        quad_kernel<R>((pz[s] - np_[2]) * invh);
            if (!(w > R(0))) continue;
            vl += fv[s] * w;
            vs += rv[s] * w * rf[s];
          }
        }
    const R vliq = F[G_SATP * fstride + n];  // raw liquid sum from k_p2g
    const R psi = clamp01<R>(vs / dV);
    const R room = dV - vs;
    const R sat = clamp01<R>((vliq + vl) / (room > R(1e-20) ? room : R(1e-20)));
    F[G_SATP * fstride + n] = sat;
    EF[E_PSIP * fstride + n] = psi;
    double cp = 0.0;
    const double ps = (double)psi;
    if (!(1.0 - ps < 1e-20 || pore_radius < 1e-20))
      cp = ps / (1. - ps) * surf_tension * cos_contact / pore_radius;
    EF[E_PORE * fstride + n] = (R)(cp * (1.0 - (double)sat));
  }
}

// ---- G2P, solid phase, and advection ----------------------------------------
// For elasto particles that are not surfels, over the particle's own face
// stencils (nodes of inactive buckets skipped):
//   v_a = sum u_s w;  B.row(a) = sum u_s w (x_n - x_p) 4/h^2;
//   v (twist included) *= elasto_advect_coeff;
//   B = ((f + g) B + (f - g) B^T) / 2, f = elasto_flip_coeff,
//   g = elasto_flip_asym_coeff.
// The reference assigns that blend into m_B's own block, which Eigen
// evaluates coefficient by coefficient in column-major order: an entry above
// the diagonal reads the already blended entry below it.  The same order is
// kept here.  Surfels keep v and B.  With advect, every elasto particle then
// moves x += v dt, twist included.
template <typename R>
__global__ void __launch_bounds__(128)
    k_g2p_elasto(GridDesc g, const unsigned char* __restrict__ active, R* __restrict__ E,
                 long long ecap, long long n, const long long* __restrict__ key,
                 const int* __restrict__ delta, const R* __restrict__ EF, long long fstride,
                 R flip, R asym, R advect_coeff, R dt, int g2p, int advect) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  // the key (and stencil offsets) exist only once a grid was built
  const long long kn = g2p ? key[s] : 0;
  if (kn < 0) return;
  const R x = E[EX * ecap + s], y = E[EY * ecap + s], z = E[EZ * ecap + s];
  if (g2p && E[ESURF * ecap + s] == R(0)) {
    const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
    const R bs = (R)g.bs, dx = (R)g.dx;
    const R invh = R(1) / dx;
    const R invD = R(4) / (dx * dx);
    int KI, KJ, KK;
    node_ijk(g, kn, KI, KJ, KK);
    const int kp[3] = {KI - 1, KJ - 1, KK - 1};
    const int dl = delta[s];
    R v[3], B[9];
    for (int a = 0; a < 3; ++a) {
      int base[3];
      for (int q = 0; q < 3; ++q) base[q] = kp[q] + (q == a ? unpack_delta(dl, a) : 0);
      R cx[3], cy[3], cz[3], wx[3], wy[3], wz[3];
      for (int t = 0; t < 3; ++t) {
        cx[t] = coord<R>(org[0], bs, dx, base[0] + t, a == 0 ? R(0) : R(0.5));
        cy[t] = coord<R>(org[1], bs, dx, base[1] + t, a == 1 ? R(0) : R(0.5));
        cz[t] = coord<R>(org[2], bs, dx, base[2] + t, a == 2 ? R(0) : R(0.5));
        wx[t] = quad_kernel<R>((x - cx[t]) * invh);
        wy[t] = quad_kernel<R>((y - cy[t]) * invh);
        wz[t] = quad_kernel<R>((z - cz[t]) * invh);
      }
      R fv = 0, b0 = 0, b1 = 0, b2 = 0;
      const R* U = EF + (E_VEL + a) * fstride;
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            const int NI_ = base[0] + i, NJ_ = base[1] + j, NK_ = base[2] + k;
            if (!in_grid(g, NI_, NJ_, NK_) || !active[bucket_of(g, NI_, NJ_, NK_)]) continue;
            const R un = U[node_linear(g, NI_, NJ_, NK_)];
            const R w = wx[i] * wy[j] * wz[k];
            const R uw = un * w;
            fv += uw;
            b0 += uw * (cx[i] - x) * invD;
            b1 += uw * (cy[j] - y) * invD;
            b2 += uw * (cz[k] - z) * invD;
          }
      v[a] = fv;
      B[a * 3 + 0] = b0;
      B[a * 3 + 1] = b1;
      B[a * 3 + 2] = b2;
    }
    for (int a = 0; a < 3; ++a) E[(EVX + a) * ecap + s] = v[a] * advect_coeff;
    E[EVT * ecap + s] = E[EVT * ecap + s] * advect_coeff;
    const R c1 = flip + asym, c2 = flip - asym;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) B[i * 3 + j] = (c1 * B[i * 3 + j] + c2 * B[j * 3 + i]) * R(0.5);
    for (int q = 0; q < 9; ++q) E[(EB00 + q) * ecap + s] = B[q];
  }
  if (advect) {
    E[EX * ecap + s] = x + E[EVX * ecap + s] * dt;
    E[EY * ecap + s] = y + E[EVY * ecap + s] * dt;
    E[EZ * ecap + s] = z + E[EVZ * ecap + s] * dt;
    E[ETH * ecap + s] = E[ETH * ecap + s] + E[EVT * ecap + s] * dt;
  }
}

}  // namespace wcg
