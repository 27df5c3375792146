// Shared device definitions for the libWetCloth fluid-step hot path on sm_100a.
//
// Grid layout (the reference's own node layout, libWetCloth/Core/Sorter.h:63,
// TwoDScene.cpp:3746): buckets of 4x4x4 cells, bucket index
// b = bk*ni*nj + bj*ni + bi, local node index l = lk*16 + lj*4 + li, linear node
// index b*64 + l.  Every node kind (u/v/w faces, cell centres, corners) uses the
// same index space.  Storage is dense over all buckets; only buckets flagged
// active carry meaningful values (inactive buckets have no nodes in the
// reference, TwoDScene.cpp:303-308).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wcg {

constexpr int kNodesPerSide = 4;
constexpr int kNodesPerBucket = 64;
constexpr double kThetaCriterion = 0.01;   // Core/Pressure.cpp:20
constexpr double kLiquidPhiRadius = 0.883644;  // Core/TwoDScene.cpp:3328

// Scene-wide grid description (plain values; passed by value to kernels).
struct GridDesc {
  int ni, nj, nk;       // buckets per axis
  int NI, NJ, NK;       // nodes per axis (= 4 * buckets)
  long long nb;         // number of buckets
  long long nnode;      // nb * 64
  double ox, oy, oz;    // m_grid_mincorner == m_bucket_mincorner
  double bs;            // bucket size
  double dx;            // cell size = bs / 4
};

// Error codes recorded by kernels into a device word (first error wins).
enum DeviceError : int {
  kErrNone = 0,
  kErrWaitTimeout = 1,   // a wavefront dependency wait gave up
  kErrIndex = 2,         // an index fell outside its buffer (skipped)
  kErrInput = 3,         // a staged particle had a non-finite position or velocity,
                         // or a negative or NaN mass, volume or radius
};

__host__ __device__ inline long long node_linear(const GridDesc& g, int I,
                                                 int J, int K) {
  const long long b = ((long long)(K >> 2) * g.nj + (J >> 2)) * g.ni + (I >> 2);
  return b * 64 + (((K & 3) << 4) | ((J & 3) << 2) | (I & 3));
}

__host__ __device__ inline bool in_grid(const GridDesc& g, int I, int J, int K) {
  return I >= 0 && J >= 0 && K >= 0 && I < g.NI && J < g.NJ && K < g.NK;
}

__host__ __device__ inline long long bucket_of(const GridDesc& g, int I, int J,
                                               int K) {
  return ((long long)(K >> 2) * g.nj + (J >> 2)) * g.ni + (I >> 2);
}

__device__ inline void node_ijk(const GridDesc& g, long long n, int& I, int& J,
                                int& K) {
  const long long b = n >> 6;
  const int l = (int)(n & 63);
  const long long bk = b / ((long long)g.ni * g.nj);
  const long long rem = b - bk * (long long)g.ni * g.nj;
  const int bj = (int)(rem / g.ni);
  const int bi = (int)(rem - (long long)bj * g.ni);
  I = bi * 4 + (l & 3);
  J = bj * 4 + ((l >> 2) & 3);
  K = (int)bk * 4 + (l >> 4);
}

// Node position exactly as TwoDScene::getNodePos{X,Y,Z,P,SolidPhi} computes it
// for an active bucket (TwoDScene.cpp:3776-3813, generateNodes :3870-3876):
//   ((handle*bs + origin) + local*dx) + offset*dx, each step rounded separately.
// The _rn intrinsics stop nvcc contracting these into FMAs, so stencil indices
// and activation masks come out bit-identical to the reference's.
__device__ inline double node_coord(double origin, double bs, double dx,
                                    int node, double offset) {
  const int h = node >> 2;
  const int l = node & 3;
  double c = __dadd_rn(__dmul_rn((double)h, bs), origin);
  c = __dadd_rn(c, __dmul_rn((double)l, dx));
  return __dadd_rn(c, __dmul_rn(offset, dx));
}

// Quadratic B-spline (MathUtilities.h:416-424).
template <typename R>
__device__ inline R quad_kernel(R x) {
  const R d = fabs(x);
  if (d < R(0.5)) return R(0.75) - d * d;
  if (d < R(1.5)) return R(0.5) * (R(1.5) - d) * (R(1.5) - d);
  return R(0);
}

// fraction_inside for a segment (MathUtilities.h:286-293).
template <typename R>
__host__ __device__ inline R fraction_inside2(R phi_left, R phi_right) {
  if (phi_left < 0 && phi_right < 0) return R(1);
  if (phi_left < 0 && phi_right >= 0) return phi_left / (phi_left - phi_right);
  if (phi_left >= 0 && phi_right < 0) return phi_right / (phi_right - phi_left);
  return R(0);
}

// fraction_inside for a square given its corner values (bl, br, tl, tr), the
// marching-squares area of MathUtilities.h:301-376.
template <typename R>
__host__ __device__ inline R fraction_inside4(R bl, R br, R tl, R tr) {
  const int inside = (bl < 0) + (tl < 0) + (br < 0) + (tr < 0);
  R l[4] = {bl, br, tr, tl};
  auto cycle = [&]() {
    const R t = l[0];
    l[0] = l[1];
    l[1] = l[2];
    l[2] = l[3];
    l[3] = t;
  };
  if (inside == 4) return R(1);
  if (inside == 3) {
    while (l[0] < 0) cycle();
    const R s0 = R(1) - fraction_inside2(l[0], l[3]);
    const R s1 = R(1) - fraction_inside2(l[0], l[1]);
    return R(1) - R(0.5) * s0 * s1;
  }
  if (inside == 2) {
    while (l[0] >= 0 || !(l[1] < 0 || l[2] < 0)) cycle();
    if (l[1] < 0) {
      const R sl = fraction_inside2(l[0], l[3]);
      const R sr = fraction_inside2(l[1], l[2]);
      return R(0.5) * (sl + sr);
    }
    const R mid = R(0.25) * (l[0] + l[1] + l[2] + l[3]);
    if (mid < 0) {
      R area = 0;
      const R s1 = R(1) - fraction_inside2(l[0], l[3]);
      const R s3 = R(1) - fraction_inside2(l[2], l[3]);
      area += R(0.5) * s1 * s3;
      const R s2 = R(1) - fraction_inside2(l[2], l[1]);
      const R s0 = R(1) - fraction_inside2(l[0], l[1]);
      area += R(0.5) * s0 * s2;
      return R(1) - area;
    }
    R area = 0;
    const R s0 = fraction_inside2(l[0], l[1]);
    const R s1 = fraction_inside2(l[0], l[3]);
    area += R(0.5) * s0 * s1;
    const R s2 = fraction_inside2(l[2], l[1]);
    const R s3 = fraction_inside2(l[2], l[3]);
    area += R(0.5) * s2 * s3;
    return area;
  }
  if (inside == 1) {
    while (l[0] >= 0) cycle();
    const R s0 = fraction_inside2(l[0], l[3]);
    const R s1 = fraction_inside2(l[0], l[1]);
    return R(0.5) * s0 * s1;
  }
  return R(0);
}

template <typename R>
__host__ __device__ inline R clamp01(R a) {
  return a < R(0) ? R(0) : (a > R(1) ? R(1) : a);
}

// Solid walls: a box distance field with the fluid inside (DFT_BOX, usage
// DFU_SOLID, inside=true), combined as TwoDScene::computePhiVel
// (TwoDScene.cpp:5427-5448: running minimum starting at 3*bucket_size) over a
// DistanceFieldOperator union (DistanceFields.cpp:866-880, starting at 1e20).
// The identity-rotation quaternion sandwich of DistanceFieldObject::compute_phi
// (DistanceFields.cpp:607-615) is exactly ((p - c) + c); the box SDF is
// box_phi (DistanceFields.cpp:68-78).  Static walls have zero velocity.
struct Walls {
  double cx, cy, cz;
  double ex, ey, ez;
  double radius;
  double sign;   // -1 for "inside" boxes
  int enabled;
};

// Terminator shapes (DistanceFieldObject::compute_phi, DistanceFields.cpp:
// 601-660; the SDFs sphere_phi, capsule_phi, box_phi, cylinder_phi :32-114).
// Products and sums in the reference's order, rounded one by one.
constexpr int kMaxTermShapes = 16;
struct TermShape {
  int type;        // 0 box, 1 sphere, 2 capsule, 3 cylinder
  double sign;     // -1 for inside objects
  double c[3];
  double q[4];     // rotation w, x, y, z
  double par[4];
};
struct TermSet {
  int n;
  TermShape s[kMaxTermShapes];
};

__host__ __device__ inline double rn_add(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ inline double rn_sub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
__host__ __device__ inline double rn_mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

// Eigen's quaternion product (w, x, y, z), terms left to right
__device__ inline void quat_mul(const double a[4], const double b[4], double o[4]) {
  o[0] = rn_sub(rn_sub(rn_sub(rn_mul(a[0], b[0]), rn_mul(a[1], b[1])), rn_mul(a[2], b[2])),
                rn_mul(a[3], b[3]));
  o[1] = rn_sub(rn_add(rn_add(rn_mul(a[0], b[1]), rn_mul(a[1], b[0])), rn_mul(a[2], b[3])),
                rn_mul(a[3], b[2]));
  o[2] = rn_sub(rn_add(rn_add(rn_mul(a[0], b[2]), rn_mul(a[2], b[0])), rn_mul(a[3], b[1])),
                rn_mul(a[1], b[3]));
  o[3] = rn_sub(rn_add(rn_add(rn_mul(a[0], b[3]), rn_mul(a[3], b[0])), rn_mul(a[1], b[2])),
                rn_mul(a[2], b[1]));
}

// the position in the object's frame: conj(q) (0, p - c) conj(q)^-1 + c
__device__ inline void term_frame(const TermShape& t, const double p[3], double r[3]) {
  const double iq[4] = {t.q[0], -t.q[1], -t.q[2], -t.q[3]};
  const double p0[4] = {0.0, rn_sub(p[0], t.c[0]), rn_sub(p[1], t.c[1]), rn_sub(p[2], t.c[2])};
  // squaredNorm over the coefficients (x, y, z, w) in halves
  const double n2 = rn_add(rn_add(rn_mul(iq[1], iq[1]), rn_mul(iq[2], iq[2])),
                           rn_add(rn_mul(iq[3], iq[3]), rn_mul(iq[0], iq[0])));
  const double inv[4] = {iq[0] / n2, -iq[1] / n2, -iq[2] / n2, -iq[3] / n2};
  double a[4], b[4];
  quat_mul(iq, p0, a);
  quat_mul(a, inv, b);
  for (int k = 0; k < 3; ++k) r[k] = rn_add(b[k + 1], t.c[k]);
}

__device__ inline double norm3(double x, double y, double z) {
  return sqrt(rn_add(rn_add(rn_mul(x, x), rn_mul(y, y)), rn_mul(z, z)));
}

__device__ inline double term_shape_phi(const TermShape& t, const double p[3]) {
  double phi = 0.0;
  if (t.type == 1) {  // sphere
    phi = rn_sub(norm3(rn_sub(p[0], t.c[0]), rn_sub(p[1], t.c[1]), rn_sub(p[2], t.c[2])),
                 t.par[0]);
  } else {
    double r[3];
    term_frame(t, p, r);
    if (t.type == 0) {  // box
      double d[3], da[3];
      for (int k = 0; k < 3; ++k) {
        d[k] = rn_sub(fabs(rn_sub(r[k], t.c[k])), t.par[k]);
        da[k] = d[k] > 0.0 ? d[k] : 0.0;
      }
      double m = d[0] > d[1] ? d[0] : d[1];
      m = m > d[2] ? m : d[2];
      m = m < 0.0 ? m : 0.0;
      phi = rn_sub(rn_add(m, norm3(da[0], da[1], da[2])), t.par[3]);
    } else if (t.type == 2) {  // capsule along x
      const double hl = t.par[1];
      const double pa[3] = {rn_sub(r[0], rn_sub(t.c[0], hl)), rn_sub(r[1], t.c[1]),
                            rn_sub(r[2], t.c[2])};
      const double ba0 = rn_mul(2.0, hl);
      // pa . ba with ba = (2 hl, 0, 0), then / (4 hl hl), clamped to [0, 1]
      const double dot = rn_add(rn_add(rn_mul(pa[0], ba0), rn_mul(pa[1], 0.0)),
                                rn_mul(pa[2], 0.0));
      double h = dot / rn_mul(rn_mul(4.0, hl), hl);
      h = h < 0.0 ? 0.0 : (h > 1.0 ? 1.0 : h);
      phi = rn_sub(norm3(rn_sub(pa[0], rn_mul(ba0, h)), rn_sub(pa[1], rn_mul(0.0, h)),
                         rn_sub(pa[2], rn_mul(0.0, h))),
                   t.par[0]);
    } else {  // cylinder along y
      const double q0 = rn_sub(r[0], t.c[0]), q1 = rn_sub(r[1], t.c[1]), q2 = rn_sub(r[2], t.c[2]);
      const double d0 =
          rn_add(rn_sub(sqrt(rn_add(rn_mul(q0, q0), rn_mul(q2, q2))), t.par[0]), t.par[1]);
      const double d1 = rn_sub(fabs(q1), t.par[2]);
      double m = d0 > d1 ? d0 : d1;
      m = m < 0.0 ? m : 0.0;
      const double e0 = d0 > 0.0 ? d0 : 0.0, e1 = d1 > 0.0 ? d1 : 0.0;
      phi = rn_sub(rn_add(m, sqrt(rn_add(rn_mul(e0, e0), rn_mul(e1, e1)))), t.par[1]);
    }
  }
  return t.sign * phi;
}

// TwoDScene::computePhiVel over the terminator groups: the running minimum
// from 3 bucket sizes of each group's union (from 1e20)
__device__ inline double term_phi(const TermSet& T, double px, double py, double pz,
                                  double three_bs) {
  const double p[3] = {px, py, pz};
  double u = 1e20;
  for (int k = 0; k < T.n; ++k) {
    const double f = term_shape_phi(T.s[k], p);
    u = f < u ? f : u;
  }
  return u < three_bs ? u : three_bs;
}

__device__ inline double wall_phi(const Walls& w, double px, double py,
                                  double pz, double three_bs) {
  if (!w.enabled) return three_bs;
  const double rx = __dadd_rn(__dsub_rn(px, w.cx), w.cx);
  const double ry = __dadd_rn(__dsub_rn(py, w.cy), w.cy);
  const double rz = __dadd_rn(__dsub_rn(pz, w.cz), w.cz);
  const double dx = __dsub_rn(fabs(__dsub_rn(rx, w.cx)), w.ex);
  const double dy = __dsub_rn(fabs(__dsub_rn(ry, w.cy)), w.ey);
  const double dz = __dsub_rn(fabs(__dsub_rn(rz, w.cz)), w.ez);
  const double ax = dx > 0.0 ? dx : 0.0;
  const double ay = dy > 0.0 ? dy : 0.0;
  const double az = dz > 0.0 ? dz : 0.0;
  double m = dx > dy ? dx : dy;
  m = m > dz ? m : dz;
  m = m < 0.0 ? m : 0.0;
  const double s =
      __dadd_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)), __dmul_rn(az, az));
  const double box = __dsub_rn(__dadd_rn(m, __dsqrt_rn(s)), w.radius);
  const double phi = w.sign * box;
  double out = 1e20;
  if (phi < out) out = phi;
  return out < three_bs ? out : three_bs;
}

__device__ inline void record_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

}  // namespace wcg
