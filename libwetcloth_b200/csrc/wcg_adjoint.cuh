// Reverse mode of one liquid sub-step with the particle positions held fixed.
//
// With x fixed, the grid (activation, weights, liquid phi, DOFs, solid
// weights, the matrix) is fixed too, and the sub-step is affine in the
// particles' velocities v and affine matrices C:
//   P2G          mom = sum m w (v + C d),  u_f = mom / m_node   (m_node > 1e-20)
//   stepVelocity v* = u_f + g dt           (heavy nodes; light nodes constant)
//   assembly     b(c) = sum_faces +-(v* psi_fs w) / dx
//   solve        A p = b
//   apply        u = v* - s (p_r - p_l),   s = dt V_f inv_C / (dx theta) on valid faces
//   extrapolate  two layers of neighbour means into invalid faces
//   constrain    u *= (1 - friction) on faces with solid weight 0
//   G2P          v' = sum u w,  C' = flip sum u w d 4/h^2,  x' = x + v' dt
// (d = x_node - x_particle).  The kernels below apply the transposes in reverse
// order; A is symmetric, so the adjoint solve reuses the forward solver on the
// same matrix.  After G2P come advection and the solid projection of the
// particles that end inside the solid (piecewise smooth in v'; k_adj_load).
// The positions' own cotangent x-bar0 = d(loss)/d(x) at the start of the
// sub-step follows the weights' dependence on x (quadratic B-spline weights,
// TwoDScene::updateParticleWeights TwoDScene.cpp:2084-2174, and the APIC
// offsets d) through P2G and G2P, plus the identity part of the advection.
// The grid's discrete structure (activation, DOFs, valid faces, heavy nodes),
// the liquid phi of the ghost-fluid fractions, the solid weights and the
// solid projections are held at their recomputed values.  Uniform density
// makes V_f inv_C = 1/rho on every heavy face, so the pressure system itself
// does not move with x.  Every sum is a gather in fixed order.
#pragma once

#include <cuda_runtime.h>

#include "wcg_common.cuh"
#include "wcg_context.h"
#include "wcg_kernels.cuh"

namespace wcg {

// d/dr of quad_kernel (MathUtilities.h:416): -2r inside |r| < 1/2,
// -(3/2 - |r|) sign(r) on 1/2 <= |r| < 3/2, 0 outside.
template <typename R>
__device__ inline R quad_kernel_d(R r) {
  const R d = fabs(r);
  if (d < R(0.5)) return R(-2) * r;
  if (d < R(1.5)) return r > R(0) ? -(R(1.5) - d) : (R(1.5) - d);
  return R(0);
}

// Adjoint grid fields (adj buffer, gcap each).
// A_PF: the forward pressure (kept across the adjoint solve); A_PHIB: the
// cotangent of the cell-centred liquid phi through the ghost-fluid fractions.
enum AdjField : int {
  A_UBAR = 0, A_UTMP = 3, A_VSBAR = 6, A_PF = 9, A_PHIB = 10, kNumAdjFields = 11
};

// Original-order cotangents of (v', C', x') into sorted-order columns:
// Cb = C-bar, vb = v-bar + dt d-bar, where d-bar is the cotangent of the step
// d = v' dt through advection and TwoDScene::solidProjection
// (TwoDScene.cpp:1776-1821).  A projected particle (phi_now < 0) ends at
//   x' = x + d - phi_now g,  phi_now = phi + g . d,  g = G / |G|,
//   G = sum phi_n iD w_n (x_n - x - d),  dG/dd = -iD phi I,
// so with M = I - g g^T and s = -iD phi / |G| (M = I, s = -iD phi when |G|
// is at most 1e-20 and G is used unnormalised)
//   d-bar = x-bar - (g + s M d)(g . x-bar) - phi_now s M x-bar;
// any other particle has d-bar = x-bar.  v' is recomputed by G2P from the
// face velocities with constrainLiquidVelocity applied on the fly (friction).
// A projected particle's x-cotangent also follows phi's and G's weights at x
// and pos = x + d (see the block below); the particle correction before G2P
// is taken as the identity in x.
//
// With XB: XB = x-bar + G2P's x-part (sorted order, 3 columns), from
//   v'_a = sum w u_a,  C'_aq = f sum w u_a d_q  (f = flip 4/h^2, d = x_n - x_c):
//   x-bar += sum_a sum_n u_a [(vb_a + f sum_q Cb_aq d_q) grad w - f w Cb_a.]
// with vb and Cb the cotangents just formed (grad w from the weights' x).
template <typename R>
__global__ void __launch_bounds__(128)
    k_adj_load(GridDesc g, const unsigned char* __restrict__ active, const R* __restrict__ P,
               long long pcap, long long np, const long long* __restrict__ key,
               const int* __restrict__ delta, const R* __restrict__ F, long long fstride,
               R flip, R friction, const int* __restrict__ pid,
               const double* __restrict__ vbar, const double* __restrict__ Cbar,
               const double* __restrict__ xbar, double dt, R* __restrict__ B,
               const R* __restrict__ XC, R* __restrict__ XB) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const long long i = pid[s];
  double db[3] = {xbar[i * 3 + 0], xbar[i * 3 + 1], xbar[i * 3 + 2]};
  const long long kn = key[s];
  R xg[3] = {R(0), R(0), R(0)};
  if (kn >= 0) {
    const R x[3] = {P[PX * pcap + s], P[PY * pcap + s], P[PZ * pcap + s]};
    // the corrected position (the particle correction ran before G2P), or x
    const R xc[3] = {XC ? XC[s] : x[0], XC ? XC[pcap + s] : x[1], XC ? XC[2 * pcap + s] : x[2]};
    int KI, KJ, KK;
    node_ijk(g, kn, KI, KJ, KK);
    const int kp[3] = {KI - 1, KJ - 1, KK - 1};
    const int dl = delta[s];
    R v[3], C[9];
    g2p_gather<R>(g, active, F, fstride, kp, dl, x, xc, flip, friction, v, C);
    R d[3], pos[3];
    for (int q = 0; q < 3; ++q) {
      d[q] = v[q] * (R)dt;
      pos[q] = xc[q] + d[q];
    }
    R phi, gr[3];
    const R nrm = solid_sample<R>(g, active, F, fstride, kp, dl, x, pos, phi, gr);
    const double phi_now = (double)phi + ((double)gr[0] * d[0] + (double)gr[1] * d[1] +
                                          (double)gr[2] * d[2]);
    if (phi_now < 0.0) {
      const double iD = 4.0 / (g.dx * g.dx);
      const bool unit = nrm > R(1e-20);
      const double sc = unit ? -iD * (double)phi / (double)nrm : -iD * (double)phi;
      const double gx = gr[0] * db[0] + gr[1] * db[1] + gr[2] * db[2];
      const double gd = gr[0] * (double)d[0] + gr[1] * (double)d[1] + gr[2] * (double)d[2];
      double out[3];
      for (int q = 0; q < 3; ++q) {
        const double Md = unit ? (double)d[q] - gr[q] * gd : (double)d[q];
        const double Mx = unit ? db[q] - gr[q] * gx : db[q];
        out[q] = db[q] - ((double)gr[q] + sc * Md) * gx - phi_now * sc * Mx;
      }
      if (XB) {
        // the projected particle's own x (the weights of phi and G at x, and
        // pos = x + d): x-bar_c = d-bar + (g - J) (g . x-bar)
        //   - K^T M_s (d (g . x-bar) + phi_now x-bar),
        // J = sum phi_n grad w_n, K^T v = sum phi_n iD ((x_n - pos) . v) grad w_n,
        // M_s = (I - g g^T) / |G| (I when G is used unnormalised)
        double vv[3];
        for (int q = 0; q < 3; ++q) vv[q] = (double)d[q] * gx + phi_now * db[q];
        if (unit) {
          const double gv = gr[0] * vv[0] + gr[1] * vv[1] + gr[2] * vv[2];
          for (int q = 0; q < 3; ++q) vv[q] = (vv[q] - gr[q] * gv) / (double)nrm;
        }
        const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
        const R bs = (R)g.bs, dxr = (R)g.dx;
        const R invh = R(1) / dxr;
        int base[3];
        R cn[3][3], wn[3][3], dn[3][3];
        for (int q = 0; q < 3; ++q) {
          base[q] = kp[q] + unpack_delta(dl, q);
          for (int t = 0; t < 3; ++t) {
            cn[q][t] = coord<R>(org[q], bs, dxr, base[q] + t, R(0));
            wn[q][t] = quad_kernel<R>((x[q] - cn[q][t]) * invh);
            dn[q][t] = quad_kernel_d<R>((x[q] - cn[q][t]) * invh) * invh;
          }
        }
        const R* S = F + G_SPHI * fstride;
        double J[3] = {0, 0, 0}, Kv[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < 3; ++j)
            for (int ii = 0; ii < 3; ++ii) {
              const int NI_ = base[0] + ii, NJ_ = base[1] + j, NK_ = base[2] + k;
              const bool on = in_grid(g, NI_, NJ_, NK_) && active[bucket_of(g, NI_, NJ_, NK_)];
              const double ph = on ? (double)S[node_linear(g, NI_, NJ_, NK_)] : 3.0 * g.dx;
              const double gw[3] = {(double)(dn[0][ii] * wn[1][j] * wn[2][k]),
                                    (double)(wn[0][ii] * dn[1][j] * wn[2][k]),
                                    (double)(wn[0][ii] * wn[1][j] * dn[2][k])};
              const double pv = ((double)cn[0][ii] - (double)pos[0]) * vv[0] +
                                ((double)cn[1][j] - (double)pos[1]) * vv[1] +
                                ((double)cn[2][k] - (double)pos[2]) * vv[2];
              for (int q = 0; q < 3; ++q) {
                J[q] += ph * gw[q];
                Kv[q] += ph * iD * pv * gw[q];
              }
            }
        for (int q = 0; q < 3; ++q)
          xg[q] += (R)(out[q] + ((double)gr[q] - J[q]) * gx - Kv[q] - db[q]);
      }
      for (int q = 0; q < 3; ++q) db[q] = out[q];
    }
    if (XB) {
      const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
      const R bs = (R)g.bs, dx = (R)g.dx;
      const R invh = R(1) / dx;
      const R fi = flip * (R(4) / (dx * dx));
      for (int a = 0; a < 3; ++a) {
        const R vb = (R)(vbar[i * 3 + a] + dt * db[a]);
        const R cb[3] = {(R)Cbar[i * 9 + a * 3], (R)Cbar[i * 9 + a * 3 + 1],
                         (R)Cbar[i * 9 + a * 3 + 2]};
        int base[3];
        for (int q = 0; q < 3; ++q) base[q] = kp[q] + (q == a ? unpack_delta(dl, a) : 0);
        R cx[3], cy[3], cz[3], wx[3], wy[3], wz[3], gx[3], gy[3], gz[3];
        for (int t = 0; t < 3; ++t) {
          cx[t] = coord<R>(org[0], bs, dx, base[0] + t, a == 0 ? R(0) : R(0.5));
          cy[t] = coord<R>(org[1], bs, dx, base[1] + t, a == 1 ? R(0) : R(0.5));
          cz[t] = coord<R>(org[2], bs, dx, base[2] + t, a == 2 ? R(0) : R(0.5));
          wx[t] = quad_kernel<R>((x[0] - cx[t]) * invh);
          wy[t] = quad_kernel<R>((x[1] - cy[t]) * invh);
          wz[t] = quad_kernel<R>((x[2] - cz[t]) * invh);
          gx[t] = quad_kernel_d<R>((x[0] - cx[t]) * invh) * invh;
          gy[t] = quad_kernel_d<R>((x[1] - cy[t]) * invh) * invh;
          gz[t] = quad_kernel_d<R>((x[2] - cz[t]) * invh) * invh;
        }
        const R* U = F + (G_U + a) * fstride;
        const R* W = F + (G_WEIGHT + a) * fstride;
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < 3; ++j)
            for (int ii = 0; ii < 3; ++ii) {
              const int NI_ = base[0] + ii, NJ_ = base[1] + j, NK_ = base[2] + k;
              if (!in_grid(g, NI_, NJ_, NK_) || !active[bucket_of(g, NI_, NJ_, NK_)]) continue;
              const long long nn = node_linear(g, NI_, NJ_, NK_);
              R un = U[nn];
              if (W[nn] == R(0)) un = (R(1) - friction) * un;
              const R w = wx[ii] * wy[j] * wz[k];
              const R cd = (cb[0] * (cx[ii] - xc[0]) + cb[1] * (cy[j] - xc[1])) +
                           cb[2] * (cz[k] - xc[2]);
              const R t = un * (vb + fi * cd);
              const R uw = un * fi * w;
              xg[0] += t * (gx[ii] * wy[j] * wz[k]) - uw * cb[0];
              xg[1] += t * (wx[ii] * gy[j] * wz[k]) - uw * cb[1];
              xg[2] += t * (wx[ii] * wy[j] * gz[k]) - uw * cb[2];
            }
      }
    }
  }
  for (int a = 0; a < 3; ++a) B[a * pcap + s] = (R)(vbar[i * 3 + a] + dt * db[a]);
  for (int q = 0; q < 9; ++q) B[(3 + q) * pcap + s] = (R)Cbar[i * 9 + q];
  if (XB)
    for (int q = 0; q < 3; ++q) XB[q * pcap + s] = (R)xbar[i * 3 + q] + xg[q];
}

// G2P^T and constrain^T: per face node, over the particles whose stencil
// holds it (the k_p2g neighbourhood),
//   u-bar = sum w (vb_a + flip 4/h^2 sum_q Cb_aq d_q),
// then u-bar *= 1 - friction where the solid weight is 0.
template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_g2p(GridDesc g, const int* __restrict__ active_list, const R* __restrict__ P,
              long long pcap, const int* __restrict__ start, const int* __restrict__ delta,
              DeltaRange dr, const R* __restrict__ B, const R* __restrict__ F, long long fstride,
              R* __restrict__ AG, R flip, R friction, const R* __restrict__ XC) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
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
  const R invD = R(4) / (dx * dx);
  const int IJK[3] = {I, J, K};
  R np_[3];
  for (int q = 0; q < 3; ++q) np_[q] = coord<R>(org[q], bs, dx, IJK[q], q == a ? R(0) : R(0.5));
  int lo[3], hi[3];
  for (int q = 0; q < 3; ++q) {
    lo[q] = q == a ? IJK[q] - 1 - dr.hi[q] : IJK[q] - 1;
    hi[q] = q == a ? IJK[q] + 1 - dr.lo[q] : IJK[q] + 1;
    lo[q] = lo[q] < 0 ? 0 : lo[q];
  }
  hi[0] = hi[0] > g.NI - 1 ? g.NI - 1 : hi[0];
  hi[1] = hi[1] > g.NJ - 1 ? g.NJ - 1 : hi[1];
  hi[2] = hi[2] > g.NK - 1 ? g.NK - 1 : hi[2];
  const R* px = P + PX * pcap;
  const R* py = P + PY * pcap;
  const R* pz = P + PZ * pcap;
  const R* vb = B + a * pcap;
  const R* c0 = B + (3 + 3 * a) * pcap;
  const R* c1 = B + (3 + 3 * a + 1) * pcap;
  const R* c2 = B + (3 + 3 * a + 2) * pcap;
  const R fi = flip * invD;
  R acc = 0;
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
          const R w = quad_kernel<R>((x - np_[0]) * invh) * quad_kernel<R>((y - np_[1]) * invh) *
                      quad_kernel<R>((z - np_[2]) * invh);
          // x_n - x_p from the corrected position when the step corrects
          const R xc = XC ? XC[s] : x, yc = XC ? XC[pcap + s] : y, zc = XC ? XC[2 * pcap + s] : z;
          const R cd = (c0[s] * (np_[0] - xc) + c1[s] * (np_[1] - yc)) + c2[s] * (np_[2] - zc);
          acc += w * (vb[s] + fi * cd);
        }
      }
  if (F[(G_WEIGHT + a) * fstride + n] == R(0)) acc *= R(1) - friction;
  AG[(A_UBAR + a) * fstride + n] = acc;
}

// Validity after applyPressureGradsFluidRHS (k_apply_pressure): solid weight
// > 0 and a liquid cell on either side.
template <typename R>
__device__ inline bool adj_face_valid(const GridDesc& g, const unsigned char* active,
                                      const R* F, long long fstride, int a, int I, int J, int K,
                                      long long n, R* theta) {
  if (!(F[(G_WEIGHT + a) * fstride + n] > R(0))) return false;
  const int lI = I - (a == 0), lJ = J - (a == 1), lK = K - (a == 2);
  const bool hl = in_grid(g, lI, lJ, lK) && active[bucket_of(g, lI, lJ, lK)];
  const R phil = hl ? F[G_LPHI * fstride + node_linear(g, lI, lJ, lK)] : R(0);
  const R phir = F[G_LPHI * fstride + n];
  if (!(phil < R(0) || phir < R(0))) return false;
  R t = 1;
  if (phir >= R(0) || phil >= R(0)) {
    t = fraction_inside2<R>(phil, phir);
    t = t > R(kThetaCriterion) ? t : R(kThetaCriterion);
  }
  *theta = t;
  return true;
}

template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_valid0(GridDesc g, const int* __restrict__ active_list,
                 const unsigned char* __restrict__ active, const R* __restrict__ F,
                 long long fstride, unsigned char* __restrict__ mask) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  R t;
  mask[a * fstride + n] = adj_face_valid<R>(g, active, F, fstride, a, I, J, K, n, &t) ? 1 : 0;
}

// extrapolate^T for one layer whose input validity is vin:
//   in-bar(q) = out-bar(q)             if q valid or q had no valid neighbour
//             + sum over invalid neighbours n of q with count(n) > 0 of
//               out-bar(n) / count(n)  (q valid)
template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_extrapolate(GridDesc g, const int* __restrict__ active_list,
                      const unsigned char* __restrict__ active, const R* __restrict__ obar,
                      R* __restrict__ ibar, const unsigned char* __restrict__ vin,
                      long long fstride) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R* ob = obar + a * fstride;
  const unsigned char* vi = vin + a * fstride;
  const int dI[6] = {-1, 1, 0, 0, 0, 0};
  const int dJ[6] = {0, 0, -1, 1, 0, 0};
  const int dK[6] = {0, 0, 0, 0, -1, 1};
  // number of valid neighbours of the face (I, J, K) as the forward layer counts them
  auto count_at = [&](int x0, int y0, int z0) {
    int cnt = 0;
    for (int r = 0; r < 6; ++r) {
      const int x = x0 + dI[r], y = y0 + dJ[r], z = z0 + dK[r];
      if (!in_grid(g, x, y, z) || !active[bucket_of(g, x, y, z)]) continue;
      if (vi[node_linear(g, x, y, z)]) ++cnt;
    }
    return cnt;
  };
  R acc = 0;
  if (vi[n] || count_at(I, J, K) == 0) acc = ob[n];
  if (vi[n]) {
    for (int r = 0; r < 6; ++r) {
      const int x = I + dI[r], y = J + dJ[r], z = K + dK[r];
      if (!in_grid(g, x, y, z) || !active[bucket_of(g, x, y, z)]) continue;
      const long long q = node_linear(g, x, y, z);
      if (vi[q]) continue;
      const int cnt = count_at(x, y, z);
      if (cnt > 0) acc += ob[q] / (R)cnt;
    }
  }
  ibar[a * fstride + n] = acc;
}

// apply^T to the cells: p-bar(c) = sum over valid faces f of c of -+ s_f u-bar_f
// (the face above c along an axis has c as its left cell: +s; the face at c
// has c as its right cell: -s), kept on the DOFs; written to G_B as the rhs
// of the adjoint solve.
template <typename R>
__global__ void __launch_bounds__(64)
    k_adj_apply(GridDesc g, const int* __restrict__ active_list,
                const unsigned char* __restrict__ active, const unsigned char* __restrict__ dof,
                const R* __restrict__ AG, R* __restrict__ F, long long fstride, R dt) {
  const int b = active_list[blockIdx.x];
  const int l = threadIdx.x;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx;
  R acc = 0;
  if (dof[n] & 1) {
    for (int a = 0; a < 3; ++a) {
      // face at the cell (the cell is its right side)
      R t;
      if (adj_face_valid<R>(g, active, F, fstride, a, I, J, K, n, &t)) {
        const R s = ((dt * F[(G_VOL + a) * fstride + n]) * F[(G_INVC + a) * fstride + n]) / (dx * t);
        acc -= s * AG[(A_UBAR + a) * fstride + n];
      }
      // face above the cell (the cell is its left side)
      const int uI = I + (a == 0), uJ = J + (a == 1), uK = K + (a == 2);
      if (in_grid(g, uI, uJ, uK) && active[bucket_of(g, uI, uJ, uK)]) {
        const long long u = node_linear(g, uI, uJ, uK);
        if (adj_face_valid<R>(g, active, F, fstride, a, uI, uJ, uK, u, &t)) {
          const R s = ((dt * F[(G_VOL + a) * fstride + u]) * F[(G_INVC + a) * fstride + u]) / (dx * t);
          acc += s * AG[(A_UBAR + a) * fstride + u];
        }
      }
    }
  }
  F[G_B * fstride + n] = acc;
}

// assembly^T plus the identity part of apply: per face,
//   v*-bar = u-bar + (psi_fs w / dx) (lambda(cell at the face) - lambda(cell below))
// over the DOF cells (lambda = the adjoint solve's solution in G_PRESSURE).
// With the viscosity on, the rhs the pressure step starts from is v* m (not
// the predictor's rhs), so u depends on v* through m inv_C (1 on heavy nodes,
// m on light ones): rhs_from_vstar scales the identity part by it.
template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_div(GridDesc g, const int* __restrict__ active_list,
              const unsigned char* __restrict__ active, const unsigned char* __restrict__ dof,
              const R* __restrict__ F, long long fstride, R* __restrict__ AG,
              int rhs_from_vstar) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx;
  R lam = 0;
  if (dof[n] & 1) lam += F[G_PRESSURE * fstride + n];
  const int lI = I - (a == 0), lJ = J - (a == 1), lK = K - (a == 2);
  if (in_grid(g, lI, lJ, lK) && active[bucket_of(g, lI, lJ, lK)]) {
    const long long c = node_linear(g, lI, lJ, lK);
    if (dof[c] & 1) lam -= F[G_PRESSURE * fstride + c];
  }
  const R k = (F[(G_PSIFS + a) * fstride + n] * F[(G_WEIGHT + a) * fstride + n]) / dx;
  R ub = AG[(A_UBAR + a) * fstride + n];
  if (rhs_from_vstar) ub *= F[(G_MASS + a) * fstride + n] * F[(G_INVC + a) * fstride + n];
  AG[(A_VSBAR + a) * fstride + n] = ub + k * lam;
}

// The ghost-fluid fraction's part of the position cotangent.  On a face with
// solid weight w > 0 between a liquid cell (phi < 0) and an air cell the
// fraction theta = phi_neg / (phi_neg - phi_pos) (fraction_inside,
// MathUtilities.h:286-293; clamped below at 0.01, Pressure.cpp:20) enters
//   the apply step   u = inv_C (rhs - dt V_f (p_r - p_l) / (dx theta)), and
//   the matrix       diag(liquid cell) += w dt inv_C V_f / (dx^2 theta)
// (k_apply_pressure, k_assemble).  With u-bar the cotangent of u, lambda the
// adjoint solve's solution and p the forward pressure:
//   theta-bar = u-bar s (p_r - p_l) / theta + lambda_L p_L term / theta^2,
// s = dt V_f inv_C / (dx theta); nothing where theta is clamped.  Per cell,
//   phi-bar = sum over its six faces of theta-bar d(theta)/d(phi_cell),
// and, where phi-bar is nonzero, the particle that sets the cell's phi
// (updateLiquidPhi TwoDScene.cpp:3286-3376: phi = min over the particles of
// the 27 cells around of |x_c - x_p| - max(0.883644 dx, r_p); none where the
// wall rule or no particle sets it) goes to AM (sorted index, or -1).
template <typename R>
__global__ void __launch_bounds__(64)
    k_adj_theta(GridDesc g, const int* __restrict__ active_list,
                const unsigned char* __restrict__ active, const unsigned char* __restrict__ dof,
                const R* __restrict__ F, long long fstride, R* __restrict__ AG, R dt,
                const R* __restrict__ P, long long pcap, const int* __restrict__ start,
                Walls walls, int have_liquid, int* __restrict__ AM) {
  const int b = active_list[blockIdx.x];
  const int l = threadIdx.x;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long n = (long long)b * 64 + l;
  const R dx = (R)g.dx;
  const R phic = F[G_LPHI * fstride + n];
  const R* PF = AG + A_PF * fstride;
  R phib = 0;
  for (int f = 0; f < 6; ++f) {
    const int a = f >> 1;
    const bool upper = f & 1;
    // the face node and the neighbour cell across it
    const int qI = I + (upper && a == 0), qJ = J + (upper && a == 1), qK = K + (upper && a == 2);
    const int mI = upper ? qI : I - (a == 0), mJ = upper ? qJ : J - (a == 1),
              mK = upper ? qK : K - (a == 2);
    if (!in_grid(g, qI, qJ, qK) || !active[bucket_of(g, qI, qJ, qK)]) continue;
    const long long q = node_linear(g, qI, qJ, qK);
    const R w = F[(G_WEIGHT + a) * fstride + q];
    if (!(w > R(0))) continue;
    const bool hm = in_grid(g, mI, mJ, mK) && active[bucket_of(g, mI, mJ, mK)];
    const long long m = hm ? node_linear(g, mI, mJ, mK) : -1;
    const R phim = hm ? F[G_LPHI * fstride + m] : R(0);
    const R phil = upper ? phic : phim, phir = upper ? phim : phic;
    if (!(phil < R(0) || phir < R(0))) continue;
    if (phil < R(0) && phir < R(0)) continue;  // theta = 1
    if (!upper && !hm) continue;                // a missing left cell is no particle's phi
    const R neg = phil < R(0) ? phil : phir, pos = phil < R(0) ? phir : phil;
    const R den = neg - pos;
    const R theta = neg / den;
    if (!(theta > R(kThetaCriterion))) continue;
    const R V = F[(G_VOL + a) * fstride + q], invC = F[(G_INVC + a) * fstride + q];
    const R pl = upper ? PF[n] : (hm ? PF[m] : R(0));
    const R pr = upper ? PF[m] : PF[n];
    const R sc = ((dt * V) * invC) / (dx * theta);
    R tb = AG[(A_UBAR + a) * fstride + q] * sc * (pr - pl) / theta;
    // the liquid side's diagonal, when it is a DOF and the air cell exists
    const long long L = phil < R(0) ? (upper ? n : m) : (upper ? m : n);
    if (hm && (dof[L] & 1)) {
      const R term = (w * (dt / (dx * dx))) * (invC * V);
      tb += F[G_PRESSURE * fstride + L] * PF[L] * term / (theta * theta);
    }
    // d(theta)/d(phi) of this cell
    const bool cneg = phic < R(0);
    phib += tb * (cneg ? -pos / (den * den) : neg / (den * den));
  }
  AG[A_PHIB * fstride + n] = phib;
  int am = -1;
  if (phib != R(0)) {
    const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
    const R bs = (R)g.bs;
    R np_[3];
    const int IJK[3] = {I, J, K};
    for (int q = 0; q < 3; ++q) np_[q] = coord<R>(org[q], bs, dx, IJK[q], R(0.5));
    const double sphi = wall_phi(walls, (double)np_[0], (double)np_[1], (double)np_[2],
                                 3.0 * g.bs);
    if (!(have_liquid && sphi < 0.0)) {
      const R rmin = dx * (R)kLiquidPhiRadius;
      R best = R(3) * bs;
      for (int KZ = (K > 0 ? K - 1 : 0); KZ <= (K + 1 < g.NK ? K + 1 : g.NK - 1); ++KZ)
        for (int KY = (J > 0 ? J - 1 : 0); KY <= (J + 1 < g.NJ ? J + 1 : g.NJ - 1); ++KY)
          for (int KX = (I > 0 ? I - 1 : 0); KX <= (I + 1 < g.NI ? I + 1 : g.NI - 1); ++KX) {
            const long long c = node_linear(g, KX, KY, KZ);
            for (int s = start[c]; s < start[c + 1]; ++s) {
              const R ddx = P[PX * pcap + s] - np_[0], ddy = P[PY * pcap + s] - np_[1],
                      ddz = P[PZ * pcap + s] - np_[2];
              const R r = P[PR * pcap + s];
              const R d = sqrt((ddx * ddx + ddy * ddy) + ddz * ddz) - (rmin > r ? rmin : r);
              if (d < best) {
                best = d;
                am = s;
              }
            }
          }
    }
  }
  AM[n] = am;
}

// stepVelocity^T and P2G^T per particle over its own face stencils (nodes of
// inactive buckets skipped): mom-bar = v*-bar / m_node on heavy nodes,
//   v-bar_a = sum m w mom-bar,  C-bar_aq = sum m w mom-bar d_q;
// results in original particle order.  With XB (the x-bar of the later stages,
// sorted order) the weights' part of u_f = mom / m_node is added,
//   x-bar += sum_a sum_n (m / m_node) v*-bar [(phi_a - u_f) grad w - w C_a.],
//   phi_a = v_a + C_a. d  (m-bar and mom-bar of the same node combined),
// and x-bar0 written in original order.
template <typename R>
__global__ void __launch_bounds__(128)
    k_adj_p2g(GridDesc g, const unsigned char* __restrict__ active, const R* __restrict__ P,
              long long pcap, long long np, const int* __restrict__ pid,
              const long long* __restrict__ key, const int* __restrict__ delta,
              const R* __restrict__ F, const R* __restrict__ AG, long long fstride,
              double* __restrict__ vbar0, double* __restrict__ Cbar0,
              const R* __restrict__ XB, double* __restrict__ xbar0,
              const int* __restrict__ AM) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const long long i = pid[s];
  const long long kn = key[s];
  if (kn < 0) {
    if (XB)
      for (int q = 0; q < 3; ++q) xbar0[i * 3 + q] = (double)XB[q * pcap + s];
    return;
  }
  const R org[3] = {(R)g.ox, (R)g.oy, (R)g.oz};
  const R bs = (R)g.bs, dx = (R)g.dx;
  const R invh = R(1) / dx;
  const R x = P[PX * pcap + s], y = P[PY * pcap + s], z = P[PZ * pcap + s];
  const R m = P[PM * pcap + s];
  int KI, KJ, KK;
  node_ijk(g, kn, KI, KJ, KK);
  const int kp[3] = {KI - 1, KJ - 1, KK - 1};
  const int dl = delta[s];
  R xg[3] = {R(0), R(0), R(0)};
  for (int a = 0; a < 3; ++a) {
    int base[3];
    for (int q = 0; q < 3; ++q) base[q] = kp[q] + (q == a ? unpack_delta(dl, a) : 0);
    R cx[3], cy[3], cz[3], wx[3], wy[3], wz[3], gx[3], gy[3], gz[3];
    for (int t = 0; t < 3; ++t) {
      cx[t] = coord<R>(org[0], bs, dx, base[0] + t, a == 0 ? R(0) : R(0.5));
      cy[t] = coord<R>(org[1], bs, dx, base[1] + t, a == 1 ? R(0) : R(0.5));
      cz[t] = coord<R>(org[2], bs, dx, base[2] + t, a == 2 ? R(0) : R(0.5));
      wx[t] = quad_kernel<R>((x - cx[t]) * invh);
      wy[t] = quad_kernel<R>((y - cy[t]) * invh);
      wz[t] = quad_kernel<R>((z - cz[t]) * invh);
      gx[t] = quad_kernel_d<R>((x - cx[t]) * invh) * invh;
      gy[t] = quad_kernel_d<R>((y - cy[t]) * invh) * invh;
      gz[t] = quad_kernel_d<R>((z - cz[t]) * invh) * invh;
    }
    const R* VS = AG + (A_VSBAR + a) * fstride;
    const R* MS = F + (G_MASS + a) * fstride;
    const R* UF = F + (G_VEL + a) * fstride;
    const R va = P[(VX + a) * pcap + s];
    const R ca[3] = {P[(C00 + 3 * a) * pcap + s], P[(C00 + 3 * a + 1) * pcap + s],
                     P[(C00 + 3 * a + 2) * pcap + s]};
    R vb = 0, b0 = 0, b1 = 0, b2 = 0;
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j)
        for (int ii = 0; ii < 3; ++ii) {
          const int NI_ = base[0] + ii, NJ_ = base[1] + j, NK_ = base[2] + k;
          if (!in_grid(g, NI_, NJ_, NK_) || !active[bucket_of(g, NI_, NJ_, NK_)]) continue;
          const long long nn = node_linear(g, NI_, NJ_, NK_);
          const R mn = MS[nn];
          if (!(mn > R(1e-20))) continue;
          const R w = wx[ii] * wy[j] * wz[k];
          const R mw = (m * w) * (VS[nn] / mn);
          vb += mw;
          b0 += mw * (cx[ii] - x);
          b1 += mw * (cy[j] - y);
          b2 += mw * (cz[k] - z);
          if (XB) {
            const R r = m * (VS[nn] / mn);
            const R phi = va + (ca[0] * (cx[ii] - x) + ca[1] * (cy[j] - y)) + ca[2] * (cz[k] - z);
            const R t = r * (phi - UF[nn]);
            const R rw = r * w;
            xg[0] += t * (gx[ii] * wy[j] * wz[k]) - rw * ca[0];
            xg[1] += t * (wx[ii] * gy[j] * wz[k]) - rw * ca[1];
            xg[2] += t * (wx[ii] * wy[j] * gz[k]) - rw * ca[2];
          }
        }
    vbar0[i * 3 + a] = (double)vb;
    Cbar0[i * 9 + a * 3 + 0] = (double)b0;
    Cbar0[i * 9 + a * 3 + 1] = (double)b1;
    Cbar0[i * 9 + a * 3 + 2] = (double)b2;
  }
  if (XB && AM) {
    // the liquid phi of the cells this particle sets: d(phi)/dx = (x - x_c) / |x - x_c|
    const R* PB = AG + A_PHIB * fstride;
    for (int KZ = (KK > 0 ? KK - 1 : 0); KZ <= (KK + 1 < g.NK ? KK + 1 : g.NK - 1); ++KZ)
      for (int KY = (KJ > 0 ? KJ - 1 : 0); KY <= (KJ + 1 < g.NJ ? KJ + 1 : g.NJ - 1); ++KY)
        for (int KX = (KI > 0 ? KI - 1 : 0); KX <= (KI + 1 < g.NI ? KI + 1 : g.NI - 1); ++KX) {
          if (!active[bucket_of(g, KX, KY, KZ)]) continue;
          const long long c = node_linear(g, KX, KY, KZ);
          if (AM[c] != (int)s) continue;
          const R ex = x - coord<R>(org[0], bs, dx, KX, R(0.5));
          const R ey = y - coord<R>(org[1], bs, dx, KY, R(0.5));
          const R ez = z - coord<R>(org[2], bs, dx, KZ, R(0.5));
          const R dist = sqrt((ex * ex + ey * ey) + ez * ez);
          if (!(dist > R(0))) continue;
          const R pb = PB[c] / dist;
          xg[0] += pb * ex;
          xg[1] += pb * ey;
          xg[2] += pb * ez;
        }
  }
  if (XB)
    for (int q = 0; q < 3; ++q) xbar0[i * 3 + q] = (double)XB[q * pcap + s] + (double)xg[q];
}

// ---- explicit viscosity (k_viscosity_explicit) ------------------------------
// One explicit step is v_out = v_in + f K v_in with f = sub_dt mu / (rho dx^2).
// Per output component a, K has six same-component neighbour terms
// c_t (v_a(n + o_t) - v_a(n)) (present when n + o_t is in an active bucket)
// and eight cross terms +-c (v_b(n + o)) (zero outside active buckets).  The
// coefficients c are volume fractions at fixed offsets from n (times 2 on the
// component's own axis).  The table below lists, per component: the six
// coefficient sources {field, offset} in the order (+x, -x, +y, -y, +z, -z)
// with their multipliers, and the cross terms {component, offset, sign,
// coefficient}; it restates k_viscosity_explicit term by term.
struct VCoef { signed char field, di, dj, dk; };   // field 0 centre, 1..3 x/y/z edge
struct VCross { signed char comp, di, dj, dk, sign, coef; };
__constant__ VCoef kVCoef[3][6] = {
    {{0, 0, 0, 0}, {0, -1, 0, 0}, {3, 0, 1, 0}, {3, 0, 0, 0}, {2, 0, 0, 1}, {2, 0, 0, 0}},
    {{3, 1, 0, 0}, {3, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, -1, 0}, {1, 0, 0, 1}, {1, 0, 0, 0}},
    {{2, 1, 0, 0}, {2, 0, 0, 0}, {1, 0, 1, 0}, {1, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, -1}}};
__constant__ signed char kVMult[3][6] = {{2, 2, 1, 1, 1, 1}, {1, 1, 2, 2, 1, 1}, {1, 1, 1, 1, 2, 2}};
__constant__ VCross kVCross[3][8] = {
    {{1, 0, 1, 0, 1, 2}, {1, -1, 1, 0, -1, 2}, {1, -1, 0, 0, 1, 3}, {1, 0, 0, 0, -1, 3},
     {2, 0, 0, 1, 1, 4}, {2, -1, 0, 1, -1, 4}, {2, -1, 0, 0, 1, 5}, {2, 0, 0, 0, -1, 5}},
    {{0, 1, 0, 0, 1, 0}, {0, 1, -1, 0, -1, 0}, {0, 0, -1, 0, 1, 1}, {0, 0, 0, 0, -1, 1},
     {2, 0, 0, 1, 1, 4}, {2, 0, -1, 1, -1, 4}, {2, 0, -1, 0, 1, 5}, {2, 0, 0, 0, -1, 5}},
    {{0, 1, 0, 0, 1, 0}, {0, 1, 0, -1, -1, 0}, {0, 0, 0, -1, 1, 1}, {0, 0, 0, 0, -1, 1},
     {1, 0, 1, 0, 1, 2}, {1, 0, 1, -1, -1, 2}, {1, 0, 0, -1, 1, 3}, {1, 0, 0, 0, -1, 3}}};
__constant__ signed char kVDir[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                                        {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

template <typename R>
__device__ inline R v_coef(const GridDesc& g, const unsigned char* active, const R* F,
                           long long fs, int a, int t, int I, int J, int K) {
  const VCoef c = kVCoef[a][t];
  const int fld = c.field == 0 ? G_VFC : G_VFEX + c.field - 1;
  return (R)kVMult[a][t] *
         v_get<R>(g, active, F + (long long)fld * fs, I + c.di, J + c.dj, K + c.dk, R(0));
}

template <typename R>
__device__ inline bool v_live(const GridDesc& g, const unsigned char* active, int I, int J, int K) {
  return in_grid(g, I, J, K) && active[bucket_of(g, I, J, K)];
}

// K^T: in-bar(a, m) = out-bar(a, m) + f [sum of the terms of every output
// (b, n) that read (a, m)]; written to ib (3 fields).
template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_viscosity(GridDesc g, const int* __restrict__ active_list,
                    const unsigned char* __restrict__ active, const R* __restrict__ F,
                    long long fs, const R* __restrict__ ob, R* __restrict__ ib, R factor) {
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const int l = threadIdx.x & 63;
  const int bk = b / (g.ni * g.nj);
  const int rem = b - bk * g.ni * g.nj;
  const int bj = rem / g.ni;
  const int bi = rem - bj * g.ni;
  const int I = bi * 4 + (l & 3), J = bj * 4 + ((l >> 2) & 3), K = bk * 4 + (l >> 4);
  const long long m = (long long)b * 64 + l;
  const R* oa = ob + a * fs;
  R acc = 0;
  for (int t = 0; t < 6; ++t) {
    const int di = kVDir[t][0], dj = kVDir[t][1], dk = kVDir[t][2];
    // the output at m itself: its own part of the term toward m + o_t
    if (v_live<R>(g, active, I + di, J + dj, K + dk))
      acc -= v_coef<R>(g, active, F, fs, a, t, I, J, K) * oa[m];
    // the output at n = m - o_t whose term reads m
    const int nI = I - di, nJ = J - dj, nK = K - dk;
    if (v_live<R>(g, active, nI, nJ, nK))
      acc += v_coef<R>(g, active, F, fs, a, t, nI, nJ, nK) * oa[node_linear(g, nI, nJ, nK)];
  }
  for (int c = 0; c < 3; ++c) {
    if (c == a) continue;
    for (int t = 0; t < 8; ++t) {
      const VCross x = kVCross[c][t];
      if (x.comp != a) continue;
      // output (c, n) reads (a, n + o) = (a, m)
      const int nI = I - x.di, nJ = J - x.dj, nK = K - x.dk;
      if (!v_live<R>(g, active, nI, nJ, nK)) continue;
      const R cf = v_coef<R>(g, active, F, fs, c, x.coef, nI, nJ, nK) / (R)kVMult[c][x.coef];
      acc += (R)x.sign * cf * ob[c * fs + node_linear(g, nI, nJ, nK)];
    }
  }
  ib[a * fs + m] = oa[m] + factor * acc;
}

// <out-bar, v_out - v_in> over the faces of the active buckets, per block
// (the viscosity cotangent: each explicit step's increment is linear in mu)
template <typename R>
__global__ void __launch_bounds__(192)
    k_adj_mu_dot(const int* __restrict__ active_list, const R* __restrict__ ob,
                 const R* __restrict__ vout, const R* __restrict__ vin, long long fs,
                 double* __restrict__ part) {
  __shared__ double sm[192];
  const int b = active_list[blockIdx.x];
  const int a = threadIdx.x >> 6;
  const long long n = (long long)b * 64 + (threadIdx.x & 63);
  sm[threadIdx.x] = (double)ob[a * fs + n] * ((double)vout[a * fs + n] - (double)vin[a * fs + n]);
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < 192; ++k) s += sm[k];
    part[blockIdx.x] = s;
  }
}

}  // namespace wcg
