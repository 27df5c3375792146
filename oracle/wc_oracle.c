/*
 * wc_oracle.c -- CPU restatement of libWetCloth's liquid fluid-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for libwcgpu (tests,
 * __graft_entry__.smoke and bench.py's CPU-baseline leg may use it); no
 * product code links it.  It restates, in plain C99 and serially, the
 * algorithm of the reference for a liquid-only scene with box walls, in the
 * reference's own orders (sort keys, 27-colour bucket traversal, per-node
 * particle lists, sorted sparse rows, column-oriented MIC(0)), and is pinned
 * against the compiled reference (oracle/_ref) by the CPU tests and the
 * golden fixtures under tests/golden/.
 *
 * Every function cites the reference routine (file:line under
 * libWetCloth/Core/) it restates.  Node fields are stored densely over all
 * buckets (bucket * 64 + k*16 + j*4 + i); inactive buckets read back as NaN.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NN 4          /* nodes per bucket side (bucketinfo numcells) */
#define NPB 64        /* nodes per bucket */

typedef struct {
  double dx, g[3], rho, flip, friction, bc[3], bh[3], br, criterion;
  int maxiters, mic;
  double visc;       /* LiquidInfo::viscosity; 0: compute_viscosity off */
  int visc_substeps; /* LinearizedImplicitEuler::m_viscosity_substeps */
  int visc_implicit; /* LiquidInfo::implicit_viscosity */
  double visc_criterion; /* LinearizedImplicitEuler::m_viscous_criterion */
  double e_flip, e_asym, e_advect; /* elasto_flip_coeff, _asym_coeff, elasto_advect_coeff */
  double drag_mu;  /* LiquidInfo::viscosity as the drag reads it (also when compute_viscosity is off) */
  /* LiquidInfo correction_strength (0: correctLiquidParticles off),
   * correction_step, correction_multiplier */
  double corr_strength, corr_mult;
  int corr_step;
  double cell_mult; /* LiquidInfo::particle_cell_multiplier */
  int merge_on;     /* relabel + mergeLiquidParticles before each sub-step */
  int split_on;     /* relabel + splitLiquidParticles before each sub-step */
  /* one terminator box (DFT_BOX, DFU_TERMINATOR, in a distance-field group of
   * its own): centre, half extents, radius, sign (-1: inside=true) */
  int term_on;
  double tc[3], th[3], tr, tsign;
  /* terminator shapes (wco_set_terminators): when nshape > 0 they replace
   * the box above */
  int nshape;
  int stype[16];
  double ssign[16], sc[16][3], sq[16][4], spar[16][4];
} Params;

typedef struct {
  char name[32];
  int is_int;
  long long n;
  double* f;
  long long* i;
} Snap;

typedef struct {
  /* CSR list of (particle, slot) pairs per node */
  int* start; /* nnode + 1 */
  int* pid;
  int* slot;
} Pairs;

typedef struct {
  Params p;
  int np;  /* all particles: [0, ne) elasto, then liquid (TwoDScene::isFluid :6921) */
  int ne;
  double *x, *v, *C, *m, *vol, *rad;  /* particle state (x3, v3, C9) */
  /* elasto particles only (liquid entries are 0): m(a) + m_fluid(a) per axis,
   * m_rest_vol, m_rest_volume_fraction, m_shape_factor, m_orientation (3),
   * twist angle and twist velocity (4th components of m_x, m_v), surfel flag */
  double *em, *rvol, *rvf, *sf, *ori, *xt, *vt;
  unsigned char* surf;
  /* grid */
  double bbmin[3], bbmax[3], org[3], bs;
  int ni, nj, nk;
  long long nb, nnode;
  uint64_t* keys;
  int* sup; /* 2 per bucket */
  unsigned char *act;
  int* base; /* np * 15: u, v, w, sphi, p stencil base (global node ijk) */
  unsigned char* inside;
  double *wu, *wv, *ww, *wp; /* np * 27 */
  Pairs pu, pv, pw, pp;
  /* node fields */
  double *mass[3], *vel[3], *vol_f[3], *sat[3], *psi[3], *wgt[3], *svel[3];
  /* elasto P2G: m_node_mass, m_node_vel, m_node_vol, m_node_shape_factor,
   * m_node_orientation (3 per node) */
  double *emass[3], *evel[3], *evol[3], *esf[3], *eori[3];
  double *sat_p, *psi_p, *pore_p, *lphi, *sphi, *pressure;
  double *vf_c, *vf_e[3];  /* liquid volume fractions: cell centres, x/y/z edges */
  double* vf_f[3];         /* ... at x/y/z faces (implicit viscosity) */
  int visc_iters, visc_ndof; /* last implicit viscosity solve */
  double visc_res;
  double *rhs[3], *vstar[3], *invC[3], *psifs[3], *psisf[3], *mshdvm[3], *mfhdvm[3];
  unsigned char* valid[3];
  /* pressure system */
  long long* dofidx;
  int ndof;
  int *rowstart, *col;
  double* val;
  double* b;
  int last_iters;
  double last_res;
  double timers[12];
  double* xw;  /* positions the sub-step's stencil weights were taken at (x3) */
  uint64_t corr_seed, corr_count; /* selector stream of the particle correction */
  int corr_sel_once;              /* >= 0: selector of the next correction */
  unsigned char* cls;             /* m_classifier of the liquid particles */
  uint64_t merge_seed, merge_count; /* draw stream of the merge */
  uint64_t split_seed, split_count; /* draw stream of the split */
  Snap snaps[256];
  int nsnaps;
} Scene;

/* ---------------------------------------------------------------------- */
static void snap_put_f(Scene* s, const char* name, const double* a, long long n) {
  Snap* t = NULL;
  for (int k = 0; k < s->nsnaps; ++k)
    if (!strcmp(s->snaps[k].name, name)) t = &s->snaps[k];
  if (!t) {
    t = &s->snaps[s->nsnaps++];
    memset(t, 0, sizeof(*t));
    strncpy(t->name, name, 31);
  }
  free(t->f);
  free(t->i);
  t->i = NULL;
  t->is_int = 0;
  t->n = n;
  t->f = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  memcpy(t->f, a, sizeof(double) * n);
}

static void snap_put_i(Scene* s, const char* name, const long long* a, long long n) {
  Snap* t = NULL;
  for (int k = 0; k < s->nsnaps; ++k)
    if (!strcmp(s->snaps[k].name, name)) t = &s->snaps[k];
  if (!t) {
    t = &s->snaps[s->nsnaps++];
    memset(t, 0, sizeof(*t));
    strncpy(t->name, name, 31);
  }
  free(t->f);
  free(t->i);
  t->f = NULL;
  t->is_int = 1;
  t->n = n;
  t->i = (long long*)malloc(sizeof(long long) * (n > 0 ? n : 1));
  memcpy(t->i, a, sizeof(long long) * n);
}

/* dense node field, NaN in inactive buckets */
static void snap_node(Scene* s, const char* name, const double* a) {
  double* t = (double*)malloc(sizeof(double) * s->nnode);
  for (long long n = 0; n < s->nnode; ++n) t[n] = s->act[n >> 6] ? a[n] : NAN;
  snap_put_f(s, name, t, s->nnode);
  free(t);
}

/* ---------------------------------------------------------------------- */
static inline long long bucket_index(const Scene* s, int i, int j, int k) {
  return ((long long)k * s->nj + j) * s->ni + i;
}

/* global node (I,J,K) -> dense index; -1 outside the grid */
static inline long long node_of(const Scene* s, int I, int J, int K) {
  if (I < 0 || J < 0 || K < 0 || I >= s->ni * NN || J >= s->nj * NN || K >= s->nk * NN)
    return -1;
  return bucket_index(s, I / NN, J / NN, K / NN) * NPB + (K % NN) * 16 + (J % NN) * 4 + (I % NN);
}

static inline int node_active(const Scene* s, long long n) { return n >= 0 && s->act[n >> 6]; }

/* TwoDScene::getNodePos{X,Y,Z,P,SolidPhi} for an active bucket
 * (TwoDScene.cpp:3776-3813 with generateNodes :3870-3876):
 * m_node_pos = (handle*bs + origin) + local*dx, then + offset*dx;
 * for an inactive bucket nodePosFromBucket (:2064-2078). */
static double node_coord(const Scene* s, int a, int I, double off) {
  const int h = I >= 0 ? I / NN : (I - NN + 1) / NN;
  const int l = I - h * NN;
  double c = (double)h * s->bs + s->org[a];
  c = c + (double)l * s->p.dx;
  return c + off * s->p.dx;
}

static double node_coord_inactive(const Scene* s, int a, int I, double off) {
  const int h = I >= 0 ? I / NN : (I - NN + 1) / NN;
  const int l = I - h * NN;
  const double corner = s->org[a] + (double)h * s->bs;
  return corner + ((double)l + off) * s->p.dx;
}

/* quad_kernel, MathUtilities.h:416-424 */
static double quad_kernel(double x) {
  const double d = fabs(x);
  if (d < 0.5) return 0.75 - d * d;
  if (d < 1.5) return 0.5 * (1.5 - d) * (1.5 - d);
  return 0.0;
}

/* fraction_inside (2 values), MathUtilities.h:286-293 */
static double frac_in2(double l, double r) {
  if (l < 0 && r < 0) return 1;
  if (l < 0 && r >= 0) return l / (l - r);
  if (l >= 0 && r < 0) return r / (r - l);
  return 0;
}

static void cycle4(double* a) {
  const double t = a[0];
  a[0] = a[1];
  a[1] = a[2];
  a[2] = a[3];
  a[3] = t;
}

/* fraction_inside (4 corners), MathUtilities.h:301-376 */
static double frac_in4(double bl, double br, double tl, double tr) {
  const int inside = (bl < 0) + (tl < 0) + (br < 0) + (tr < 0);
  double l[4] = {bl, br, tr, tl};
  if (inside == 4) return 1.;
  if (inside == 3) {
    while (l[0] < 0) cycle4(l);
    const double s0 = 1. - frac_in2(l[0], l[3]);
    const double s1 = 1. - frac_in2(l[0], l[1]);
    return 1. - 0.5 * s0 * s1;
  }
  if (inside == 2) {
    while (l[0] >= 0 || !(l[1] < 0 || l[2] < 0)) cycle4(l);
    if (l[1] < 0) return 0.5 * (frac_in2(l[0], l[3]) + frac_in2(l[1], l[2]));
    if (0.25 * (l[0] + l[1] + l[2] + l[3]) < 0) {
      double area = 0.;
      area += 0.5 * (1. - frac_in2(l[0], l[3])) * (1. - frac_in2(l[2], l[3]));
      area += 0.5 * (1 - frac_in2(l[0], l[1])) * (1 - frac_in2(l[2], l[1]));
      return 1. - area;
    }
    double area = 0.;
    area += 0.5 * frac_in2(l[0], l[1]) * frac_in2(l[0], l[3]);
    area += 0.5 * frac_in2(l[2], l[1]) * frac_in2(l[2], l[3]);
    return area;
  }
  if (inside == 1) {
    while (l[0] >= 0) cycle4(l);
    return 0.5 * frac_in2(l[0], l[3]) * frac_in2(l[0], l[1]);
  }
  return 0;
}

static double clampd(double a, double lo, double hi) { return a < lo ? lo : (a > hi ? hi : a); }

/* Solid walls: DistanceFieldObject DFT_BOX, inside (sign -1)
 * (DistanceFields.cpp:68-78, :607-615) under a DFT_UNION operator
 * (:866-880, start 1e20) and TwoDScene::computePhiVel (TwoDScene.cpp:5427-5448,
 * running minimum from 3*bucket_size).  Static: velocity 0. */
static double wall_phi(const Scene* s, double px, double py, double pz) {
  const double p[3] = {px, py, pz};
  double d[3], da[3];
  for (int a = 0; a < 3; ++a) {
    const double rp = (p[a] - s->p.bc[a]) + s->p.bc[a];
    d[a] = fabs(rp - s->p.bc[a]) - s->p.bh[a];
    da[a] = d[a] > 0.0 ? d[a] : 0.0;
  }
  double m = d[0] > d[1] ? d[0] : d[1];
  m = m > d[2] ? m : d[2];
  m = m < 0.0 ? m : 0.0;
  const double box = m + sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]) - s->p.br;
  const double phi = -1.0 * box;
  double u = 1e20;
  if (phi < u) u = phi;
  double r = 3.0 * s->bs;
  if (u < r) r = u;
  return r;
}

/* The terminator: the same box distance field with usage DFU_TERMINATOR in
 * its own group, whose DFT_UNION operator votes the terminator usage
 * (DistanceFieldOperator::vote_usage, DistanceFields.cpp:922-938), read by
 * computePhiVel through the terminator selector (TwoDScene.cpp:1757-1759). */
/* Eigen's quaternion product (w, x, y, z), Quaternion.h quat_product */
static void quat_mul(const double a[4], const double b[4], double o[4]) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] + a[2] * b[0] + a[3] * b[1] - a[1] * b[3];
  o[3] = a[0] * b[3] + a[3] * b[0] + a[1] * b[2] - a[2] * b[1];
}

/* DistanceFieldObject::compute_phi (DistanceFields.cpp:601-660) of shape k,
 * with the SDFs of DistanceFields.cpp:32-114; the frame change is
 * conj(q) (0, p - c) conj(q)^-1 + c */
static double shape_phi(const Scene* s, int k, const double p[3]) {
  const double* c = s->p.sc[k];
  const double* par = s->p.spar[k];
  const int type = s->p.stype[k];
  double phi;
  if (type == 1) {
    const double d0 = p[0] - c[0], d1 = p[1] - c[1], d2 = p[2] - c[2];
    phi = sqrt(d0 * d0 + d1 * d1 + d2 * d2) - par[0];
  } else {
    const double* q = s->p.sq[k];
    const double iq[4] = {q[0], -q[1], -q[2], -q[3]};
    const double p0[4] = {0.0, p[0] - c[0], p[1] - c[1], p[2] - c[2]};
    const double n2 = (iq[1] * iq[1] + iq[2] * iq[2]) + (iq[3] * iq[3] + iq[0] * iq[0]);
    const double inv[4] = {iq[0] / n2, -iq[1] / n2, -iq[2] / n2, -iq[3] / n2};
    double a[4], b[4], r[3];
    quat_mul(iq, p0, a);
    quat_mul(a, inv, b);
    for (int j = 0; j < 3; ++j) r[j] = b[j + 1] + c[j];
    if (type == 0) { /* box_phi */
      double d[3], da[3];
      for (int j = 0; j < 3; ++j) {
        d[j] = fabs(r[j] - c[j]) - par[j];
        da[j] = d[j] > 0.0 ? d[j] : 0.0;
      }
      double m = d[0] > d[1] ? d[0] : d[1];
      m = m > d[2] ? m : d[2];
      m = m < 0.0 ? m : 0.0;
      phi = m + sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]) - par[3];
    } else if (type == 2) { /* capsule_phi, axis x */
      const double hl = par[1];
      const double pa[3] = {r[0] - (c[0] - hl), r[1] - c[1], r[2] - c[2]};
      const double ba0 = 2.0 * hl;
      const double dot = pa[0] * ba0 + pa[1] * 0.0 + pa[2] * 0.0;
      double h = dot / (4.0 * hl * hl);
      h = h < 0.0 ? 0.0 : (h > 1.0 ? 1.0 : h);
      const double e0 = pa[0] - ba0 * h, e1 = pa[1] - 0.0 * h, e2 = pa[2] - 0.0 * h;
      phi = sqrt(e0 * e0 + e1 * e1 + e2 * e2) - par[0];
    } else { /* cylinder_phi, axis y */
      const double q0 = r[0] - c[0], q1 = r[1] - c[1], q2 = r[2] - c[2];
      const double d0 = sqrt(q0 * q0 + q2 * q2) - par[0] + par[1];
      const double d1 = fabs(q1) - par[2];
      double m = d0 > d1 ? d0 : d1;
      m = m < 0.0 ? m : 0.0;
      const double e0 = d0 > 0.0 ? d0 : 0.0, e1 = d1 > 0.0 ? d1 : 0.0;
      phi = m + sqrt(e0 * e0 + e1 * e1) - par[1];
    }
  }
  return s->p.ssign[k] * phi;
}

static double term_phi(const Scene* s, double px, double py, double pz) {
  if (s->p.nshape > 0) {
    const double p[3] = {px, py, pz};
    double u = 1e20;
    for (int k = 0; k < s->p.nshape; ++k) {
      const double f = shape_phi(s, k, p);
      if (f < u) u = f;
    }
    const double r = 3.0 * s->bs;
    return u < r ? u : r;
  }
  const double p[3] = {px, py, pz};
  double d[3], da[3];
  for (int a = 0; a < 3; ++a) {
    const double rp = (p[a] - s->p.tc[a]) + s->p.tc[a];
    d[a] = fabs(rp - s->p.tc[a]) - s->p.th[a];
    da[a] = d[a] > 0.0 ? d[a] : 0.0;
  }
  double m = d[0] > d[1] ? d[0] : d[1];
  m = m > d[2] ? m : d[2];
  m = m < 0.0 ? m : 0.0;
  const double box = m + sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]) - s->p.tr;
  const double phi = s->p.tsign * box;
  double u = 1e20;
  if (phi < u) u = phi;
  double r = 3.0 * s->bs;
  if (u < r) r = u;
  return r;
}

/* ---------------------------------------------------------------------- */
/* TwoDScene::updateParticleBoundingBox (TwoDScene.cpp:1588-1612) and
 * rebucketizeParticles (:1657-1710) */
static void build_grid(Scene* s) {
  double mn[3] = {1e20, 1e20, 1e20}, mx[3] = {-1e20, -1e20, -1e20};
  for (int i = 0; i < s->np; ++i)
    for (int a = 0; a < 3; ++a) {
      const double v = s->x[i * 3 + a];
      if (v < mn[a]) mn[a] = v;
      if (v > mx[a]) mx[a] = v;
    }
  const double d2 = s->bs * 2.0;
  int nbk[3];
  for (int a = 0; a < 3; ++a) {
    s->bbmin[a] = floor(mn[a] / d2) * d2;
    s->bbmax[a] = ceil(mx[a] / d2) * d2;
    const double content = (s->bbmax[a] - s->bbmin[a]) + s->bs * 3.0 * 2.0;
    int cells = (int)ceil(content / s->p.dx);
    if (cells < 1) cells = 1;
    const double gsize = (double)cells * s->p.dx;
    s->org[a] = s->bbmin[a] - s->bs * 3.0;
    nbk[a] = (int)ceil(gsize / s->bs);
    if (nbk[a] < 1) nbk[a] = 1;
  }
  s->ni = nbk[0];
  s->nj = nbk[1];
  s->nk = nbk[2];
  s->nb = (long long)s->ni * s->nj * s->nk;
  s->nnode = s->nb * NPB;
}

static int cmp_u64(const void* a, const void* b) {
  const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* Sorter::sort (Sorter.h:126-163) */
static void sort_particles(Scene* s) {
  free(s->keys);
  free(s->sup);
  s->keys = (uint64_t*)malloc(sizeof(uint64_t) * (s->np > 0 ? s->np : 1));
  s->sup = (int*)calloc((size_t)s->nb * 2, sizeof(int));
  const int nbk[3] = {s->ni, s->nj, s->nk};
  for (int p = 0; p < s->np; ++p) {
    int h[3];
    for (int a = 0; a < 3; ++a) {
      h[a] = (int)floor((s->x[p * 3 + a] - s->org[a]) / s->bs);
      if (h[a] < 0) h[a] = 0;
      if (h[a] > nbk[a] - 1) h[a] = nbk[a] - 1;
    }
    s->keys[p] = ((uint64_t)bucket_index(s, h[0], h[1], h[2]) << 32) | (uint64_t)p;
  }
  qsort(s->keys, s->np, sizeof(uint64_t), cmp_u64);
  for (int q = 0; q < s->np; ++q) {
    const unsigned b = (unsigned)(s->keys[q] >> 32);
    const unsigned bp = q > 0 ? (unsigned)(s->keys[q - 1] >> 32) : 0xffffffffu;
    const unsigned bn = q + 1 < s->np ? (unsigned)(s->keys[q + 1] >> 32) : 0xffffffffu;
    if (b != bp) s->sup[b * 2] = q;
    if (b != bn) s->sup[b * 2 + 1] = q + 1;
  }
}

/* TwoDScene::findNodes (TwoDScene.cpp:3683-3760): stencil base per axis and
 * bucket activation; resampleNodes (:5069-5119) runs it for the u, v, w,
 * solid-phi and pressure offsets, then expandFluidNodesMarked(1)
 * (:5021-5064) and markInsideOut (:447-490). */
static void resample_nodes(Scene* s) {
  free(s->act);
  free(s->base);
  free(s->inside);
  s->act = (unsigned char*)calloc((size_t)s->nb, 1);
  s->base = (int*)malloc(sizeof(int) * 15 * (s->np > 0 ? s->np : 1));
  s->inside = (unsigned char*)malloc(s->np > 0 ? s->np : 1);
  static const double offs[5][3] = {{0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0},
                                    {0.0, 0.0, 0.0}, {0.5, 0.5, 0.5}};
  for (int q = 0; q < s->np; ++q) {
    const int p = (int)(s->keys[q] & 0xffffffffu);
    const long long b = (long long)(s->keys[q] >> 32);
    const int bk = (int)(b / ((long long)s->ni * s->nj));
    const int bj = (int)((b - (long long)bk * s->ni * s->nj) / s->ni);
    const int bi = (int)(b - ((long long)bk * s->ni * s->nj + (long long)bj * s->ni));
    const int bh[3] = {bi, bj, bk};
    for (int t = 0; t < 5; ++t) {
      int lo[3];
      for (int a = 0; a < 3; ++a) {
        const double corner = ((double)bh[a] * s->bs + s->org[a]) + offs[t][a] * s->p.dx;
        const double local = (s->x[p * 3 + a] - corner) / s->p.dx;
        const double fl = floor(local);
        const double fr = local - fl;
        lo[a] = bh[a] * NN + (int)fl + (fr > 0.5 ? 0 : -1);
        s->base[p * 15 + t * 3 + a] = lo[a];
      }
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            const int I = lo[0] + i, J = lo[1] + j, K = lo[2] + k;
            const int hi = I >= 0 ? I / NN : -1, hj = J >= 0 ? J / NN : -1, hk = K >= 0 ? K / NN : -1;
            if (hi < 0 || hj < 0 || hk < 0 || hi >= s->ni || hj >= s->nj || hk >= s->nk) continue;
            /* only soft particles (not surfels) activate (isSoft :697) */
            if (!s->surf[p]) s->act[bucket_index(s, hi, hj, hk)] = 1;
          }
    }
  }
  unsigned char* pre = (unsigned char*)malloc((size_t)s->nb);
  memcpy(pre, s->act, (size_t)s->nb);
  for (int k = 0; k < s->nk; ++k)
    for (int j = 0; j < s->nj; ++j)
      for (int i = 0; i < s->ni; ++i) {
        const long long b = bucket_index(s, i, j, k);
        if (pre[b]) continue;
        int any = 0;
        for (int t = -1; t <= 1 && !any; ++t)
          for (int u = -1; u <= 1 && !any; ++u)
            for (int r = -1; r <= 1 && !any; ++r) {
              if (!t && !u && !r) continue;
              const int x = i + r, y = j + u, z = k + t;
              if (x < 0 || y < 0 || z < 0 || x >= s->ni || y >= s->nj || z >= s->nk) continue;
              if (pre[bucket_index(s, x, y, z)]) any = 1;
            }
        if (any) s->act[b] = 1;
      }
  free(pre);
  for (int p = 0; p < s->np; ++p) {
    int comp = 0, uncomp = 0;
    for (int t = 0; t < 3; ++t)
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            const long long n = node_of(s, s->base[p * 15 + t * 3] + i, s->base[p * 15 + t * 3 + 1] + j,
                                        s->base[p * 15 + t * 3 + 2] + k);
            if (node_active(s, n)) comp = 1;
            else uncomp = 1;
          }
    s->inside[p] = comp ? (uncomp ? 1 : 2) : 0;
  }
}

/* getNodePos* of stencil node: active bucket formula or nodePosFromBucket */
static void stencil_node_pos(const Scene* s, int I, int J, int K, const double* off, double* np) {
  const long long n = node_of(s, I, J, K);
  const int a = node_active(s, n);
  np[0] = a ? node_coord(s, 0, I, off[0]) : node_coord_inactive(s, 0, I, off[0]);
  np[1] = a ? node_coord(s, 1, J, off[1]) : node_coord_inactive(s, 1, J, off[1]);
  np[2] = a ? node_coord(s, 2, K, off[2]) : node_coord_inactive(s, 2, K, off[2]);
}

/* TwoDScene::updateParticleWeights (TwoDScene.cpp:2084-2174):
 * w = N_kernel<2>((x_p - x_n)/h) for the 27 nodes of each stencil */
static void compute_weights(Scene* s) {
  static const double offs[4][3] = {{0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0},
                                    {0.5, 0.5, 0.5}};
  double* W[4] = {s->wu, s->wv, s->ww, s->wp};
  free(s->xw);
  s->xw = (double*)malloc(sizeof(double) * 3 * (size_t)(s->np > 0 ? s->np : 1));
  memcpy(s->xw, s->x, sizeof(double) * 3 * (size_t)s->np);
  const int tmap[4] = {0, 1, 2, 4};
  const double h = s->p.dx;
  for (int p = 0; p < s->np; ++p) {
    if (s->inside[p] == 0) continue;
    for (int t = 0; t < 4; ++t) {
      const int* lo = &s->base[p * 15 + tmap[t] * 3];
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            double np[3];
            stencil_node_pos(s, lo[0] + i, lo[1] + j, lo[2] + k, offs[t], np);
            const double dxv[3] = {(s->x[p * 3] - np[0]) / h, (s->x[p * 3 + 1] - np[1]) / h,
                                   (s->x[p * 3 + 2] - np[2]) / h};
            W[t][p * 27 + k * 9 + j * 3 + i] =
                quad_kernel(dxv[0]) * quad_kernel(dxv[1]) * quad_kernel(dxv[2]);
          }
    }
  }
}

/* TwoDScene::buildNodeParticlePairs (TwoDScene.cpp:2257-2355): per-node
 * (particle, slot) lists, appended in the 27-colour bucket traversal of
 * Sorter::for_each_bucket_particles_colored (Sorter.h:403-437, numcolors 3). */
static void build_pairs(Scene* s, Pairs* P, const double* W, int t) {
  free(P->start);
  free(P->pid);
  free(P->slot);
  P->start = (int*)calloc((size_t)s->nnode + 1, sizeof(int));
  int* cursor = (int*)calloc((size_t)s->nnode, sizeof(int));
  const int nc = 3;
  const int sni = (s->ni + nc - 1) / nc, snj = (s->nj + nc - 1) / nc, snk = (s->nk + nc - 1) / nc;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      for (long long n = 0; n < s->nnode; ++n) P->start[n + 1] += P->start[n];
      const int tot = P->start[s->nnode];
      P->pid = (int*)malloc(sizeof(int) * (tot > 0 ? tot : 1));
      P->slot = (int*)malloc(sizeof(int) * (tot > 0 ? tot : 1));
    }
    for (int ct = 0; ct < nc; ++ct)
      for (int cs = 0; cs < nc; ++cs)
        for (int cr = 0; cr < nc; ++cr)
          for (long long sb = 0; sb < (long long)sni * snj * snk; ++sb) {
            const int sk = (int)(sb / ((long long)sni * snj));
            const int sj = (int)((sb - (long long)sk * sni * snj) / sni);
            const int si = (int)(sb - (long long)sk * sni * snj - (long long)sj * sni);
            const int k = sk * nc + ct, j = sj * nc + cs, i = si * nc + cr;
            if (k >= s->nk || j >= s->nj || i >= s->ni) continue;
            const long long b = bucket_index(s, i, j, k);
            if (!s->act[b]) continue;
            for (int q = s->sup[b * 2]; q < s->sup[b * 2 + 1]; ++q) {
              const int p = (int)(s->keys[q] & 0xffffffffu);
              const int* lo = &s->base[p * 15 + t * 3];
              for (int sl = 0; sl < 27; ++sl) {
                const int di = sl % 3, dj = (sl / 3) % 3, dk = sl / 9;
                const long long n = node_of(s, lo[0] + di, lo[1] + dj, lo[2] + dk);
                if (!node_active(s, n) || !(W[p * 27 + sl] > 0.0)) continue;
                if (pass == 0) {
                  P->start[n + 1]++;
                } else {
                  const int at = P->start[n] + cursor[n]++;
                  P->pid[at] = p;
                  P->slot[at] = sl;
                }
              }
            }
          }
  }
  free(cursor);
}

/* TwoDScene::mapParticleNodesAPIC (TwoDScene.cpp:6609-6919), both branches:
 * elasto particles (p < ne) add (m + m_fluid) and their momentum to the solid
 * phase and, unless surfels, their solid volume (m_rest_vol x rest volume
 * fraction), held liquid volume, shape factor and orientation; liquid
 * particles add to the liquid phase. */
static void p2g(Scene* s) {
  const double dV = s->p.dx * s->p.dx * s->p.dx;
  Pairs* PP[3] = {&s->pu, &s->pv, &s->pw};
  double* W[3] = {s->wu, s->wv, s->ww};
  for (int a = 0; a < 3; ++a) {
    for (long long n = 0; n < s->nnode; ++n) {
      s->mass[a][n] = s->vel[a][n] = s->vol_f[a][n] = 0;
      s->psi[a][n] = s->sat[a][n] = 0;
      s->emass[a][n] = s->evel[a][n] = s->evol[a][n] = s->esf[a][n] = 0;
      s->eori[a][n * 3] = s->eori[a][n * 3 + 1] = s->eori[a][n * 3 + 2] = 0;
      if (!s->act[n >> 6]) continue;
      const int I = (int)((n >> 6) % s->ni) * NN + (int)(n & 3);
      const long long bb = n >> 6;
      const int bk = (int)(bb / ((long long)s->ni * s->nj));
      const int bj = (int)((bb - (long long)bk * s->ni * s->nj) / s->ni);
      const int J = bj * NN + (int)((n >> 2) & 3), K = bk * NN + (int)(n >> 4 & 3);
      const double off[3] = {a == 0 ? 0.0 : 0.5, a == 1 ? 0.0 : 0.5, a == 2 ? 0.0 : 0.5};
      const double np[3] = {node_coord(s, 0, I, off[0]), node_coord(s, 1, J, off[1]),
                            node_coord(s, 2, K, off[2])};
      double ps = 0, ms = 0, vs = 0, pf = 0, mf = 0, vf = 0, vfe = 0, shp = 0, shw = 0;
      double o[3] = {0, 0, 0};
      for (int e = PP[a]->start[n]; e < PP[a]->start[n + 1]; ++e) {
        const int p = PP[a]->pid[e];
        const double w = W[a][p * 27 + PP[a]->slot[e]];
        const double* C = &s->C[p * 9 + a * 3];
        const double dot = (C[0] * (np[0] - s->x[p * 3]) + C[1] * (np[1] - s->x[p * 3 + 1])) +
                           C[2] * (np[2] - s->x[p * 3 + 2]);
        const double vel = s->v[p * 3 + a] + dot;
        if (p < s->ne) {
          const double mm = s->em[p * 3 + a];
          ps += vel * mm * w;
          ms += mm * w;
          if (!s->surf[p]) {
            vs += s->rvol[p] * s->rvf[p] * w;
            vfe += s->vol[p] * w;
            shp += s->sf[p] * w;
            shw += w;
            for (int q = 0; q < 3; ++q) o[q] += s->ori[p * 3 + q] * w;
          }
        } else {
          pf += vel * s->m[p] * w;
          mf += s->m[p] * w;
          vf += s->vol[p] * w;
        }
      }
      if (ms > 1e-20) s->evel[a][n] = ps / ms;
      if (mf > 1e-20) s->vel[a][n] = pf / mf;
      if (shw > 1e-20) shp /= shw;
      s->emass[a][n] = ms;
      s->evol[a][n] = vs + vfe;
      s->mass[a][n] = mf;
      s->vol_f[a][n] = vf;
      s->psi[a][n] = clampd(vs / dV, 0.0, 1.0);
      s->sat[a][n] = clampd((vf + vfe) / fmax(1e-20, dV - vs), 0.0, 1.0);
      /* Vector3s::norm, then orientation /= norm (Eigen: per component) */
      const double lo = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      if (lo > 1e-20)
        for (int q = 0; q < 3; ++q) o[q] /= lo;
      for (int q = 0; q < 3; ++q) s->eori[a][n * 3 + q] = o[q];
      s->esf[a][n] = shp;
    }
  }
}

/* updateLiquidPhi (TwoDScene.cpp:3286-3345) */
static void liquid_phi(Scene* s) {
  const double dx = s->p.dx;
  for (long long n = 0; n < s->nnode; ++n) {
    s->lphi[n] = 3.0 * s->bs;
    s->pressure[n] = 0.0;
  }
  if (s->np == s->ne) return;  /* no liquid particles: nothing else (:3303) */
  const int nc = 3;
  const int sni = (s->ni + nc - 1) / nc, snj = (s->nj + nc - 1) / nc, snk = (s->nk + nc - 1) / nc;
  const double off[3] = {0.5, 0.5, 0.5};
  for (int ct = 0; ct < nc; ++ct)
    for (int cs = 0; cs < nc; ++cs)
      for (int cr = 0; cr < nc; ++cr)
        for (long long sb = 0; sb < (long long)sni * snj * snk; ++sb) {
          const int sk = (int)(sb / ((long long)sni * snj));
          const int sj = (int)((sb - (long long)sk * sni * snj) / sni);
          const int si = (int)(sb - (long long)sk * sni * snj - (long long)sj * sni);
          const int k = sk * nc + ct, j = sj * nc + cs, i = si * nc + cr;
          if (k >= s->nk || j >= s->nj || i >= s->ni) continue;
          const long long b = bucket_index(s, i, j, k);
          for (int q = s->sup[b * 2]; q < s->sup[b * 2 + 1]; ++q) {
            const int p = (int)(s->keys[q] & 0xffffffffu);
            if (p < s->ne) continue;  /* liquid particles only (:3309) */
            const int* lo = &s->base[p * 15 + 12];
            for (int sl = 0; sl < 27; ++sl) {
              const int I = lo[0] + sl % 3, J = lo[1] + (sl / 3) % 3, K = lo[2] + sl / 9;
              const long long n = node_of(s, I, J, K);
              if (!node_active(s, n)) continue;
              double np[3];
              stencil_node_pos(s, I, J, K, off, np);
              const double d0 = s->x[p * 3] - np[0], d1 = s->x[p * 3 + 1] - np[1],
                           d2 = s->x[p * 3 + 2] - np[2];
              const double r = fmax(dx * 0.883644, s->rad[p]);
              const double phi = sqrt(d0 * d0 + d1 * d1 + d2 * d2) - r;
              if (phi < s->lphi[n]) s->lphi[n] = phi;
            }
          }
        }
  for (long long n = 0; n < s->nnode; ++n) {
    if (!s->act[n >> 6]) continue;
    const long long bb = n >> 6;
    const int bk = (int)(bb / ((long long)s->ni * s->nj));
    const int bj = (int)((bb - (long long)bk * s->ni * s->nj) / s->ni);
    const int bi = (int)(bb - (long long)bk * s->ni * s->nj - (long long)bj * s->ni);
    const int I = bi * NN + (int)(n & 3), J = bj * NN + (int)((n >> 2) & 3), K = bk * NN + (int)((n >> 4) & 3);
    const double np[3] = {node_coord(s, 0, I, 0.5), node_coord(s, 1, J, 0.5), node_coord(s, 2, K, 0.5)};
    if (wall_phi(s, np[0], np[1], np[2]) < 0.0) s->lphi[n] = -0.5 * dx;
  }
}

static void node_ijk(const Scene* s, long long n, int* I, int* J, int* K) {
  const long long bb = n >> 6;
  const int bk = (int)(bb / ((long long)s->ni * s->nj));
  const int bj = (int)((bb - (long long)bk * s->ni * s->nj) / s->ni);
  const int bi = (int)(bb - (long long)bk * s->ni * s->nj - (long long)bj * s->ni);
  *I = bi * NN + (int)(n & 3);
  *J = bj * NN + (int)((n >> 2) & 3);
  *K = bk * NN + (int)((n >> 4) & 3);
}

/* updateSolidPhi (TwoDScene.cpp:7940-7967) and updateSolidWeights
 * (:1871-1962; corner order of connectSolidPhiNodes :4433-4596) */
static void solid_phi_and_weights(Scene* s) {
  for (long long n = 0; n < s->nnode; ++n) {
    s->sphi[n] = 0;
    for (int a = 0; a < 3; ++a) s->svel[a][n] = 0;
    if (!s->act[n >> 6]) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    s->sphi[n] = wall_phi(s, node_coord(s, 0, I, 0.0), node_coord(s, 1, J, 0.0), node_coord(s, 2, K, 0.0));
  }
  for (long long n = 0; n < s->nnode; ++n) {
    for (int a = 0; a < 3; ++a) s->wgt[a][n] = 0;
    if (!s->act[n >> 6]) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    for (int a = 0; a < 3; ++a) {
      double phi[4];
      for (int r = 0; r < 2; ++r)
        for (int t = 0; t < 2; ++t) {
          int ci = I, cj = J, ck = K;
          if (a == 0) { cj += t; ck += r; }
          else if (a == 1) { ci += r; ck += t; }
          else { ci += r; cj += t; }
          const long long q = node_of(s, ci, cj, ck);
          phi[r * 2 + t] = node_active(s, q) ? s->sphi[q] : 0.5 * s->p.dx;
        }
      s->wgt[a][n] = clampd(1.0 - frac_in4(phi[0], phi[1], phi[2], phi[3]), 0.0, 1.0);
    }
  }
}

/* mapParticleSaturationPsiNodes (TwoDScene.cpp:5952-5992) and
 * updatePorePressureNodes (:5933-5950, getCapillaryPressure :563-571) */
static void sat_psi_p(Scene* s) {
  const double dV = s->p.dx * s->p.dx * s->p.dx;
  const double pore_radius = 0.005, stc = 72.8, angle = 40.8 / 180.0 * M_PI;
  for (long long n = 0; n < s->nnode; ++n) {
    double vl = 0, vs = 0;
    for (int e = s->pp.start[n]; e < s->pp.start[n + 1]; ++e) {
      const int p = s->pp.pid[e];
      if (s->surf[p]) continue;
      const double w = s->wp[p * 27 + s->pp.slot[e]];
      vl += s->vol[p] * w;
      vs += s->rvol[p] * w * s->rvf[p];  /* 0 for liquid particles */
    }
    s->psi_p[n] = clampd(vs / dV, 0.0, 1.0);
    s->sat_p[n] = clampd(vl / fmax(1e-20, dV - vs), 0.0, 1.0);
    double cp = 0.0;
    const double psi = s->psi_p[n];
    if (!(1.0 - psi < 1e-20 || pore_radius < 1e-20))
      cp = (psi / (1. - psi)) * stc * cos(angle) / pore_radius;
    s->pore_p[n] = cp * (1.0 - s->sat_p[n]);
  }
}

/* mathutils::get_rotated_pore_coeff_{x,y,z} (MathUtilities.h:792-818): the
 * row sum along `axis` of (2 - sf) I + (2 sf - 1) n n^T, n = o/|o|, written in
 * closed form; 0 when the orientation is zero, as the reference's quotient by
 * max(1e-63, |o|^2) gives. */
static double pore_coeff(const double* o, double sf, int axis) {
  const double n2 = (o[0] * o[0] + o[1] * o[1]) + o[2] * o[2];
  if (!(n2 > 0.0)) return 0.0;
  return (2.0 - sf) + (2.0 * sf - 1.0) * o[axis] * ((o[0] + o[1]) + o[2]) / n2;
}

/* TwoDScene::getDragCoeffWithOrientation (TwoDScene.cpp:4042-4097) for the
 * liquid (material 0) with use_drag and use_nonlinear_drag on: permeabilities
 * k_a, k_b of the yarn packing at solid fraction psi, the Ergun/Yazdchi
 * coefficients c_a, c_b, the transversely isotropic tensor (c_xy, c_xy, c_z)
 * about the node orientation, and its row sum along `axis`
 * (mathutils::get_rotated_drag_*, MathUtilities.h:819-878), written as
 * c_xy + (c_z - c_xy) n_axis (n_x + n_y + n_z).  Yarn diameter 0.01,
 * Yazdchi power 1.6 (the LiquidInfo defaults of loadLiquidInfo). */
static double drag_coeff(const Scene* s, double psi, double sat, double dv, const double* o,
                         double sf, int axis) {
  const double n2 = (o[0] * o[0] + o[1] * o[1]) + o[2] * o[2];
  if (psi == 0.0 || sat == 0.0 || n2 < 1e-20) return 0.0;
  const double ergun = 0.1428869017, di = 0.01, yp = 1.6;
  const double mu = s->p.drag_mu, rho = s->p.rho;
  const double lp = -log(psi);
  double ka = (lp - 1.476 + 2.0 * psi - 0.5 * psi * psi) / (16.0 * psi) * di * di;
  double kb = (lp - 1.476 + 2.0 * psi - 1.774 * psi * psi + 4.078 * pow(psi, 3.0)) /
              (32.0 * psi) * di * di;
  ka = fmax(1e-20, ka);
  kb = fmax(1e-20, kb);
  const double inertial = ergun * pow(di, yp - 1.0) * pow(mu, 1.0 - yp);
  const double flow = pow(rho * fabs(dv), yp);
  const double den = pow(1.0 - psi, 1.5);
  const double ca = fmin(1e63, mu / ka + inertial / (den * sqrt(ka)) * flow);
  const double cb = fmin(1e63, mu / kb + inertial / (den * sqrt(kb)) * flow);
  const double cxy = ca * (1.0 - sf) + cb * sf;
  const double cz = ca * sf + cb * (1.0 - sf);
  return cxy + (cz - cxy) * o[axis] * ((o[0] + o[1]) + o[2]) / n2;
}

/* LinearizedImplicitEuler::stepVelocity for liquid nodes
 * (LinearizedImplicitEuler.cpp:224-337): constructNodeForce (:548-667),
 * SimpleGravityForce::addLiquidGradEToNode (SimpleGravityForce.cpp:25-52),
 * pressure::computePorePressureGrads (Pressure.cpp:26-110, orientation 0),
 * constructHDV (:846-965, no drag), constructInvMDV (:1109-1148),
 * performLocalSolve (:128-170), acceptVelocity (:2176-2212),
 * constructPsiSF (:1052-1107). */
/* ---- explicit viscosity ------------------------------------------------ */
/* mathutils::sort of four values (MathUtilities.h:959-965) */
static void sort4(double* a, double* b, double* c, double* d) {
  double t;
#define SWP(u, v) if (*u > *v) { t = *u; *u = *v; *v = t; }
  SWP(a, b) SWP(c, d) SWP(a, c) SWP(b, d) SWP(b, c)
#undef SWP
}

/* volume_fraction of a tetrahedron (VolumeFractions.cpp:101-127): the
 * fraction with phi <= 0 by the sorted tet/prism cases */
static double vf_tet(double p0, double p1, double p2, double p3) {
  sort4(&p0, &p1, &p2, &p3);
  if (p3 <= 0) return 1;
  if (p2 <= 0) return 1 - p3 * p3 * p3 / ((p3 - p2) * (p3 - p1) * (p3 - p0));
  if (p1 <= 0) {
    const double a = p0 / (p0 - p2), b = p0 / (p0 - p3), c = p1 / (p1 - p3), d = p1 / (p1 - p2);
    return a * b * (1 - d) + b * (1 - c) * d + c * d;
  }
  if (p0 <= 0) return p0 * p0 * p0 / ((p0 - p1) * (p0 - p2) * (p0 - p3));
  return 0;
}

/* volume_fraction of a cube from its corner values, as twelve tetrahedra
 * (two of them counted twice) (VolumeFractions.cpp:129-162) */
static double vf_cube(double p000, double p100, double p010, double p110, double p001,
                      double p101, double p011, double p111) {
  return (vf_tet(p000, p001, p101, p011) + vf_tet(p000, p101, p100, p110) +
          vf_tet(p000, p010, p011, p110) + vf_tet(p101, p011, p111, p110) +
          2 * vf_tet(p000, p011, p101, p110) + vf_tet(p100, p101, p001, p111) +
          vf_tet(p100, p001, p000, p010) + vf_tet(p100, p110, p111, p010) +
          vf_tet(p001, p111, p011, p010) + 2 * vf_tet(p100, p111, p001, p010)) /
         12;
}

/* TwoDScene::interpolateValue (TwoDScene.cpp:3586-3621) of the cell-centred
 * liquid phi, default dx outside the grid or in inactive buckets */
static double interp_lphi(const Scene* s, const double* pos) {
  const double dx = s->p.dx;
  double bp[3], fr[3], buf[8];
  int bi[3];
  for (int a = 0; a < 3; ++a) {
    const double ori = s->org[a] + 0.5 * dx;
    bp[a] = (pos[a] - ori) / dx;
    bi[a] = (int)floor(bp[a]);
  }
  for (int t = 0; t < 2; ++t)
    for (int u = 0; u < 2; ++u)
      for (int r = 0; r < 2; ++r) {
        const int q[3] = {bi[0] + r, bi[1] + u, bi[2] + t};
        const int h[3] = {q[0] / NN, q[1] / NN, q[2] / NN};
        double v = dx;
        if (h[0] >= 0 && h[0] < s->ni && h[1] >= 0 && h[1] < s->nj && h[2] >= 0 && h[2] < s->nk) {
          const long long b = bucket_index(s, h[0], h[1], h[2]);
          if (s->act[b]) {
            const int l = (q[2] - h[2] * NN) * NN * NN + (q[1] - h[1] * NN) * NN + (q[0] - h[0] * NN);
            v = s->lphi[b * NPB + l];
          }
        }
        buf[t * 4 + u * 2 + r] = v;
      }
  for (int a = 0; a < 3; ++a) fr[a] = bp[a] - (double)bi[a];
#define LERP(v0, v1, f) ((1 - (f)) * (v0) + (f) * (v1))
  const double b0 = LERP(LERP(buf[0], buf[1], fr[0]), LERP(buf[2], buf[3], fr[0]), fr[1]);
  const double b1 = LERP(LERP(buf[4], buf[5], fr[0]), LERP(buf[6], buf[7], fr[0]), fr[1]);
  return LERP(b0, b1, fr[2]);
#undef LERP
}

/* TwoDScene::estimateVolumeFractions (TwoDScene.cpp:3535-3584) for the node
 * offsets of updateLiquidPhi (:3353-3367).  The reference adds the offset to
 * the node position in world units, not cells, and so does this. */
static void volume_fractions(Scene* s) {
  const double dx = s->p.dx;
  const double offs[7][3] = {{0.5, 0.5, 0.5}, {0.5, 0.0, 0.0}, {0.0, 0.5, 0.0}, {0.0, 0.0, 0.5},
                             {0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0}};
  double* out[7] = {s->vf_c, s->vf_e[0], s->vf_e[1], s->vf_e[2], s->vf_f[0], s->vf_f[1], s->vf_f[2]};
  const int nf = s->p.visc_implicit ? 7 : 4;
  for (long long n = 0; n < s->nnode; ++n) {
    for (int f = 0; f < nf; ++f) out[f][n] = 0.0;
    if (!s->act[n >> 6]) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    const double corner[3] = {node_coord(s, 0, I, 0.0), node_coord(s, 1, J, 0.0),
                              node_coord(s, 2, K, 0.0)};
    const double o = 0.5 * dx;
    for (int f = 0; f < nf; ++f) {
      const double c[3] = {corner[0] + offs[f][0], corner[1] + offs[f][1], corner[2] + offs[f][2]};
      double ph[8];
      for (int z = 0; z < 2; ++z)
        for (int y = 0; y < 2; ++y)
          for (int x = 0; x < 2; ++x) {
            const double pos[3] = {c[0] + (x ? o : -o), c[1] + (y ? o : -o), c[2] + (z ? o : -o)};
            ph[x * 4 + y * 2 + z] = interp_lphi(s, pos);
          }
      /* ph index x*4 + y*2 + z holds phi_xyz */
      out[f][n] = vf_cube(ph[0], ph[4], ph[2], ph[6], ph[1], ph[5], ph[3], ph[7]);
    }
  }
}

/* viscosity::get_value (Viscosity.cpp:27-55): node value of a field at global
 * node (I, J, K), default outside the grid or in an inactive bucket */
static double vget(const Scene* s, const double* f, int I, int J, int K, double def) {
  const long long n = node_of(s, I, J, K);
  if (!node_active(s, n)) return def;
  return f[n];
}

/* applyNodeViscosityExplicit (Viscosity.cpp:1780-2107): one explicit step of
 * the liquid-volume-weighted viscous stress divergence on the face
 * velocities, src -> dst, in the reference's order of terms. */
static void viscosity_explicit(Scene* s, double* const* src, double* const* dst, double dt) {
  const double dx = s->p.dx;
  const double factor = dt / (dx * dx) * s->p.visc / s->p.rho;
  const double* cvf = s->vf_c;
  const double* const* evf = (const double* const*)s->vf_e;
  for (long long n = 0; n < s->nnode; ++n) {
    if (!s->act[n >> 6]) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    for (int a = 0; a < 3; ++a) {
      /* axes: a (normal), and for the cross terms the reference's naming */
      double v = src[a][n];
      const double cv = v;
#define VN(fld, di, dj, dk, def) vget(s, src[fld], I + (di), J + (dj), K + (dk), def)
#define VF(arr, di, dj, dk) vget(s, arr, I + (di), J + (dj), K + (dk), 0.0)
      if (a == 0) {
        const double vol_left = VF(cvf, -1, 0, 0), vol_right = VF(cvf, 0, 0, 0);
        const double vol_back = VF(evf[1], 0, 0, 0), vol_front = VF(evf[1], 0, 0, 1);
        const double vol_bottom = VF(evf[2], 0, 0, 0), vol_top = VF(evf[2], 0, 1, 0);
        v += 2.0 * factor * vol_right * (VN(0, 1, 0, 0, cv) - cv);
        v += 2.0 * factor * vol_left * (VN(0, -1, 0, 0, cv) - cv);
        v += factor * vol_top * (VN(0, 0, 1, 0, cv) - cv);
        v += factor * vol_bottom * (VN(0, 0, -1, 0, cv) - cv);
        v += factor * vol_front * (VN(0, 0, 0, 1, cv) - cv);
        v += factor * vol_back * (VN(0, 0, 0, -1, cv) - cv);
        v += factor * vol_top * (VN(1, 0, 1, 0, 0.0) - VN(1, -1, 1, 0, 0.0));
        v += factor * vol_bottom * (VN(1, -1, 0, 0, 0.0) - VN(1, 0, 0, 0, 0.0));
        v += factor * vol_front * (VN(2, 0, 0, 1, 0.0) - VN(2, -1, 0, 1, 0.0));
        v += factor * vol_back * (VN(2, -1, 0, 0, 0.0) - VN(2, 0, 0, 0, 0.0));
      } else if (a == 1) {
        const double vol_bottom = VF(cvf, 0, -1, 0), vol_top = VF(cvf, 0, 0, 0);
        const double vol_back = VF(evf[0], 0, 0, 0), vol_front = VF(evf[0], 0, 0, 1);
        const double vol_left = VF(evf[2], 0, 0, 0), vol_right = VF(evf[2], 1, 0, 0);
        v += factor * vol_right * (VN(1, 1, 0, 0, cv) - cv);
        v += factor * vol_left * (VN(1, -1, 0, 0, cv) - cv);
        v += 2.0 * factor * vol_top * (VN(1, 0, 1, 0, cv) - cv);
        v += 2.0 * factor * vol_bottom * (VN(1, 0, -1, 0, cv) - cv);
        v += factor * vol_front * (VN(1, 0, 0, 1, cv) - cv);
        v += factor * vol_back * (VN(1, 0, 0, -1, cv) - cv);
        v += factor * vol_right * (VN(0, 1, 0, 0, 0.0) - VN(0, 1, -1, 0, 0.0));
        v += factor * vol_left * (VN(0, 0, -1, 0, 0.0) - VN(0, 0, 0, 0, 0.0));
        v += factor * vol_front * (VN(2, 0, 0, 1, 0.0) - VN(2, 0, -1, 1, 0.0));
        v += factor * vol_back * (VN(2, 0, -1, 0, 0.0) - VN(2, 0, 0, 0, 0.0));
      } else {
        const double vol_back = VF(cvf, 0, 0, -1), vol_front = VF(cvf, 0, 0, 0);
        const double vol_bottom = VF(evf[0], 0, 0, 0), vol_top = VF(evf[0], 0, 1, 0);
        const double vol_left = VF(evf[1], 0, 0, 0), vol_right = VF(evf[1], 1, 0, 0);
        v += factor * vol_right * (VN(2, 1, 0, 0, cv) - cv);
        v += factor * vol_left * (VN(2, -1, 0, 0, cv) - cv);
        v += factor * vol_top * (VN(2, 0, 1, 0, cv) - cv);
        v += factor * vol_bottom * (VN(2, 0, -1, 0, cv) - cv);
        v += 2.0 * factor * vol_front * (VN(2, 0, 0, 1, cv) - cv);
        v += 2.0 * factor * vol_back * (VN(2, 0, 0, -1, cv) - cv);
        v += factor * vol_right * (VN(0, 1, 0, 0, 0.0) - VN(0, 1, 0, -1, 0.0));
        v += factor * vol_left * (VN(0, 0, 0, -1, 0.0) - VN(0, 0, 0, 0, 0.0));
        v += factor * vol_top * (VN(1, 0, 1, 0, 0.0) - VN(1, 0, 1, -1, 0.0));
        v += factor * vol_bottom * (VN(1, 0, 0, -1, 0.0) - VN(1, 0, 0, 0, 0.0));
      }
#undef VN
#undef VF
      dst[a][n] = v;
    }
  }
}

int wco_pcg_solve(int n, const int* rs, const int* col, const double* val, const double* rhs,
                  double* result, double tol_factor, int maxiters, double omega,
                  double min_ratio, double* residual_out, int* iters_out);

/* node state of a face for the viscosity (updateSolidPhi, TwoDScene.cpp:7972-8056):
 * solid when the solid phi at the centres of its two cells (those in active
 * buckets) sums below zero, fluid otherwise */
static int face_is_fluid(const Scene* s, int a, int I, int J, int K) {
  double sphi = 0.0;
  for (int t = 0; t < 2; ++t) {
    const int ci = I - (a == 0 && t == 0), cj = J - (a == 1 && t == 0), ck = K - (a == 2 && t == 0);
    if (!node_active(s, node_of(s, ci, cj, ck))) continue;
    sphi += wall_phi(s, node_coord(s, 0, ci, 0.5), node_coord(s, 1, cj, 0.5), node_coord(s, 2, ck, 0.5));
  }
  return !(sphi < 0.0);
}

/* the liquid volume weights around a face of axis a, in the reference's
 * order right, left, top, bottom, front, back (+x, -x, +y, -y, +z, -z): the
 * cell centres along a, the edges across the other two axes
 * (constructViscosityMatrixRHS :1130-1151 and its y/z counterparts) */
static void face_vols(const Scene* s, int a, int I, int J, int K, double vol[6]) {
  for (int d = 0; d < 6; ++d) {
    const int ax = d >> 1, up = !(d & 1);
    int o[3] = {0, 0, 0};
    const double* f;
    if (ax == a) {
      f = s->vf_c;
      if (!up) o[a] = -1;
    } else {
      f = s->vf_e[3 - a - ax];
      if (up) o[ax] = 1;
    }
    vol[d] = vget(s, f, I + o[0], J + o[1], K + o[2], 0.0);
  }
}

typedef struct {
  int n;
  int col[16];
  double val[16];
} VRow;

static void vrow_add(VRow* r, int j, double v) {
  int k = 0;
  while (k < r->n && r->col[k] < j) ++k;
  if (k < r->n && r->col[k] == j) {
    r->val[k] += v;
    return;
  }
  for (int q = r->n; q > k; --q) {
    r->col[q] = r->col[q - 1];
    r->val[q] = r->val[q - 1];
  }
  r->col[k] = j;
  r->val[k] = v;
  ++r->n;
}

/* One implicit viscosity sub-step (constructViscosityMatrixRHS /
 * updateViscosityRHS Viscosity.cpp:169-1779, applyNodeViscosityImplicit
 * :101-167): the faces of axis x, then y, then z, bucket by bucket, that are
 * fluid and touch liquid (own, cell or edge volume fraction > 0) become
 * unknowns;
 *   (V_f + f sum_d w_d V_d) u - f sum_d w_d V_d u_d - f sum (cross terms) = V_f u_src,
 * f = dt mu / (rho dx^2), w_d = 2 along the face's own axis, 1 across;
 * neighbours that are solid faces move to the rhs with their source values.
 * Solved with robertbridson::PCGSolver (MIC(0) 0.97, minimum diagonal ratio
 * 0.1); fluid faces that are no unknown keep their value, other faces take
 * the solid velocity. */
static void viscosity_implicit(Scene* s, double* const* vel, double dt) {
  const double dx = s->p.dx;
  const double factor = dt / (dx * dx) * s->p.visc / s->p.rho;
  const long long nn = s->nnode;
  int* idx = (int*)malloc(sizeof(int) * 3 * (size_t)nn);
  unsigned char* fl = (unsigned char*)calloc(3 * (size_t)nn, 1);
  int ndof = 0;
  for (int a = 0; a < 3; ++a)
    for (long long n = 0; n < nn; ++n) {
      idx[a * nn + n] = -1;
      if (!s->act[n >> 6]) continue;
      int I, J, K;
      node_ijk(s, n, &I, &J, &K);
      fl[a * nn + n] = (unsigned char)face_is_fluid(s, a, I, J, K);
      if (!fl[a * nn + n]) continue;
      double vol[6];
      face_vols(s, a, I, J, K, vol);
      int any = s->vf_f[a][n] > 0.0;
      for (int d = 0; d < 6; ++d) any |= vol[d] > 0.0;
      if (any) idx[a * nn + n] = ndof++;
    }
  s->visc_ndof = ndof;
  s->visc_iters = 0;
  s->visc_res = 0.0;
  if (ndof == 0) {
    free(idx);
    free(fl);
    return;
  }
  VRow* rows = (VRow*)calloc((size_t)ndof, sizeof(VRow));
  double* rhs = (double*)malloc(sizeof(double) * (size_t)ndof);
  for (int a = 0; a < 3; ++a)
    for (long long n = 0; n < nn; ++n) {
      const int row = idx[a * nn + n];
      if (row < 0) continue;
      int I, J, K;
      node_ijk(s, n, &I, &J, &K);
      VRow* R = &rows[row];
      rhs[row] = s->vf_f[a][n] * vel[a][n];
      vrow_add(R, row, s->vf_f[a][n]);
      double vol[6];
      face_vols(s, a, I, J, K, vol);
      /* same-axis neighbours */
      for (int d = 0; d < 6; ++d) {
        if (!(vol[d] > 0.0)) continue;
        const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
        const int q[3] = {I + (ax == 0) * sg, J + (ax == 1) * sg, K + (ax == 2) * sg};
        const long long m = node_of(s, q[0], q[1], q[2]);
        if (!node_active(s, m)) continue;
        const double w = ax == a ? 2.0 : 1.0;
        vrow_add(R, row, w * factor * vol[d]);
        if (fl[a * nn + m])
          vrow_add(R, idx[a * nn + m], -w * factor * vol[d]);
        else
          rhs[row] -= -w * vel[a][m] * factor * vol[d];
      }
      /* cross terms: the two faces of axis ax on the edge across direction d */
      for (int d = 0; d < 6; ++d) {
        const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
        if (ax == a || !(vol[d] > 0.0)) continue;
        for (int t = 0; t < 2; ++t) {
          int q[3] = {I, J, K};
          if (sg > 0) q[ax] += 1;
          if (t == 1) q[a] -= 1;
          const long long m = node_of(s, q[0], q[1], q[2]);
          if (!node_active(s, m)) continue;
          const double c = (t == 0 ? -1.0 : 1.0) * (double)sg;
          if (fl[ax * nn + m])
            vrow_add(R, idx[ax * nn + m], c * factor * vol[d]);
          else
            rhs[row] -= c * vel[ax][m] * factor * vol[d];
        }
      }
    }
  int* rs = (int*)malloc(sizeof(int) * ((size_t)ndof + 1));
  rs[0] = 0;
  for (int r = 0; r < ndof; ++r) rs[r + 1] = rs[r] + rows[r].n;
  int* col = (int*)malloc(sizeof(int) * (size_t)rs[ndof]);
  double* val = (double*)malloc(sizeof(double) * (size_t)rs[ndof]);
  for (int r = 0; r < ndof; ++r)
    for (int k = 0; k < rows[r].n; ++k) {
      col[rs[r] + k] = rows[r].col[k];
      val[rs[r] + k] = rows[r].val[k];
    }
  double* soln = (double*)malloc(sizeof(double) * (size_t)ndof);
  wco_pcg_solve(ndof, rs, col, val, rhs, soln, s->p.visc_criterion, s->p.maxiters, 0.97, 0.1,
                &s->visc_res, &s->visc_iters);
  for (int a = 0; a < 3; ++a)
    for (long long n = 0; n < nn; ++n) {
      if (!s->act[n >> 6]) continue;
      if (fl[a * nn + n]) {
        if (idx[a * nn + n] >= 0) vel[a][n] = soln[idx[a * nn + n]];
      } else {
        vel[a][n] = s->svel[a][n];
      }
    }
  /* the system of this sub-step, in the reference's CSR order */
  {
    long long* t = (long long*)malloc(sizeof(long long) * ((size_t)rs[ndof] + (size_t)ndof + 1));
    for (int r = 0; r <= ndof; ++r) t[r] = rs[r];
    snap_put_i(s, "V_rowstart", t, ndof + 1);
    for (int k = 0; k < rs[ndof]; ++k) t[k] = col[k];
    snap_put_i(s, "V_col", t, rs[ndof]);
    free(t);
    snap_put_f(s, "V_val", val, rs[ndof]);
    snap_put_f(s, "V_rhs", rhs, ndof);
    snap_put_f(s, "V_soln", soln, ndof);
    double* vu = (double*)malloc(sizeof(double) * (size_t)ndof);
    for (int a = 0; a < 3; ++a)
      for (long long n = 0; n < nn; ++n)
        if (idx[a * nn + n] >= 0) vu[idx[a * nn + n]] = s->vf_f[a][n];
    snap_put_f(s, "V_volu", vu, ndof);
    free(vu);
    long long* vf = (long long*)malloc(sizeof(long long) * (size_t)ndof);
    for (int a = 0; a < 3; ++a)
      for (long long n = 0; n < nn; ++n)
        if (idx[a * nn + n] >= 0) vf[idx[a * nn + n]] = a * nn + n;
    snap_put_i(s, "V_face", vf, ndof);
    free(vf);
  }
  free(soln);
  free(val);
  free(col);
  free(rs);
  free(rhs);
  free(rows);
  free(idx);
  free(fl);
}

static void step_velocity(Scene* s, double dt) {
  for (int a = 0; a < 3; ++a)
    for (long long n = 0; n < s->nnode; ++n) {
      s->rhs[a][n] = s->vstar[a][n] = s->invC[a][n] = s->psifs[a][n] = s->psisf[a][n] = 0;
      s->mshdvm[a][n] = s->mfhdvm[a][n] = 0;
      if (!s->act[n >> 6]) continue;
      const double m = s->mass[a][n];
      double r = 0.0;
      r -= m * s->p.g[a] * (-dt);
      const double* ori = &s->eori[a][n * 3];
      if (s->vol_f[a][n] > 0.0 && s->wgt[a][n] > 0.0) {
        int I, J, K;
        node_ijk(s, n, &I, &J, &K);
        const long long l = node_of(s, I - (a == 0), J - (a == 1), K - (a == 2));
        const double pp0 = node_active(s, l) ? s->pore_p[l] : 0.0;
        const double pp1 = s->pore_p[n];
        const double grad = (pp1 - pp0) / s->p.dx;
        const double coeff = pore_coeff(ori, s->esf[a][n], a);
        r += grad * s->vol_f[a][n] * dt * s->sat[a][n] * s->wgt[a][n] * coeff;
      }
      r += m * s->vel[a][n];
      /* constructHDV (:846-1000, drag_by_air off: damped mass = solid mass) with
       * the P2G liquid and solid velocities; constructInvMDV (:1109-1148) */
      const double ms = s->emass[a][n], vs = s->evol[a][n], psi = s->psi[a][n];
      const double dc = drag_coeff(s, psi, s->sat[a][n], s->vel[a][n] - s->evel[a][n], ori,
                                   s->esf[a][n], a);
      const double hdV = dt * dc * (vs + s->vol_f[a][n]);
      const double mf = m + hdV, msh = ms + hdV;
      s->mfhdvm[a][n] = mf > 1e-20 ? hdV / mf : 1.0;
      s->mshdvm[a][n] = msh > 1e-20 ? hdV / msh : 1.0;
      const double C = m + s->mshdvm[a][n] * ms;
      s->invC[a][n] = C > 1e-20 ? 1.0 / C : 1.0;
      s->rhs[a][n] = r;
      s->vstar[a][n] = m > 1e-20 ? r / m : r;
      /* constructPsiSF (:1052-1107); inv_Cs stays 0 without the solid solve */
      const double invCs = 0.0;
      s->psifs[a][n] = ((1.0 - psi) * s->invC[a][n] + psi * invCs * s->mfhdvm[a][n]) * m;
      s->psisf[a][n] = (psi * invCs + (1.0 - psi) * s->invC[a][n] * s->mshdvm[a][n]) * ms;
    }
  /* explicit viscosity sub-steps, then the rhs from the new velocity
   * (LinearizedImplicitEuler::stepVelocity, LinearizedImplicitEuler.cpp:272-306) */
  if (s->p.visc > 0.0) {
    const int ns = s->p.visc_substeps > 0 ? s->p.visc_substeps : 1;
    const double sub_dt = dt / (double)ns;
    double* tmp[3];
    for (int a = 0; a < 3; ++a) tmp[a] = (double*)malloc(sizeof(double) * (size_t)s->nnode);
    for (int it = 0; it < ns; ++it) {
      if (s->p.visc_implicit) {
        /* stepImplicitViscosityDiagonalPCG (LinearizedImplicitEuler.cpp:2127-2172) */
        viscosity_implicit(s, s->vstar, sub_dt);
        continue;
      }
      for (int a = 0; a < 3; ++a) memcpy(tmp[a], s->vstar[a], sizeof(double) * (size_t)s->nnode);
      viscosity_explicit(s, tmp, s->vstar, sub_dt);
    }
    for (int a = 0; a < 3; ++a) {
      free(tmp[a]);
      for (long long n = 0; n < s->nnode; ++n)
        if (s->act[n >> 6]) s->rhs[a][n] = s->vstar[a][n] * s->mass[a][n];
    }
  }
}

/* robertbridson::SparseMatrix::add_to_element (SparseMatrix.h:64-80) on a
 * row stored as a small sorted array */
typedef struct {
  int n;
  int col[8];
  double val[8];
} Row;

static void row_add(Row* r, int j, double v) {
  int k = 0;
  for (; k < r->n; ++k) {
    if (r->col[k] == j) {
      r->val[k] += v;
      return;
    }
    if (r->col[k] > j) break;
  }
  for (int m = r->n; m > k; --m) {
    r->col[m] = r->col[m - 1];
    r->val[m] = r->val[m - 1];
  }
  r->col[k] = j;
  r->val[k] = v;
  r->n++;
}

/* pressure::solveNodePressure assembly (Pressure.cpp:350-791) */
static void assemble(Scene* s, double dt) {
  free(s->dofidx);
  s->dofidx = (long long*)malloc(sizeof(long long) * s->nnode);
  int k = 0;
  for (long long n = 0; n < s->nnode; ++n) {
    if (!s->act[n >> 6]) {
      s->dofidx[n] = -2;
      continue;
    }
    s->dofidx[n] = -1;
    if (!(s->lphi[n] < 0)) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    const long long f[6] = {n, node_of(s, I + 1, J, K), n, node_of(s, I, J + 1, K), n,
                            node_of(s, I, J, K + 1)};
    int open = 0;
    for (int q = 0; q < 6; ++q)
      if (node_active(s, f[q]) && s->wgt[q >> 1][f[q]] > 0) open = 1;
    if (open) s->dofidx[n] = k++;
  }
  s->ndof = k;
  Row* rows = (Row*)calloc(k > 0 ? k : 1, sizeof(Row));
  free(s->b);
  s->b = (double*)calloc(k > 0 ? k : 1, sizeof(double));
  const double dx = s->p.dx;
  const double coeff = dt / (dx * dx);
  for (long long n = 0; n < s->nnode; ++n) {
    const long long d = s->dofidx[n];
    if (d < 0) continue;
    int I, J, K;
    node_ijk(s, n, &I, &J, &K);
    const double cphi = s->lphi[n];
    /* left, right, bottom, top, near, far */
    for (int q = 0; q < 6; ++q) {
      const int a = q >> 1, up = q & 1;
      const long long f = up ? node_of(s, I + (a == 0), J + (a == 1), K + (a == 2)) : n;
      if (!node_active(s, f)) continue;
      const double w = s->wgt[a][f];
      /* the elasto velocity projectFine passes is m_node_v_plus, which stays
       * zero without the solid solve (LinearizedImplicitEuler.cpp:2511-2522) */
      const double ue = 0.0;
      const double t = ((s->vstar[a][f] * s->psifs[a][f] + ue * s->psisf[a][f]) * w +
                        s->svel[a][f] * (1.0 - w)) / dx;
      if (up) s->b[d] -= t; else s->b[d] += t;
      if (w > 0.0) {
        double term = w * coeff;
        const double psi = s->psi[a][f];
        const double invCs = 0.0, vs = s->evol[a][f];
        term *= (1.0 - psi) * s->invC[a][f] * (s->vol_f[a][f] + vs * s->mshdvm[a][f]) +
                psi * invCs * (vs + s->vol_f[a][f] * s->mfhdvm[a][f]);
        const long long c = up ? f : node_of(s, I - (a == 0), J - (a == 1), K - (a == 2));
        if (!node_active(s, c)) continue;
        const double nphi = s->lphi[c];
        if (nphi < 0.0) {
          const long long dn = s->dofidx[c];
          if (dn >= 0) {
            row_add(&rows[d], (int)d, term);
            row_add(&rows[d], (int)dn, -term);
          }
        } else {
          double theta = frac_in2(cphi, nphi);
          if (theta < 0.01) theta = 0.01;
          row_add(&rows[d], (int)d, term / theta);
        }
      }
    }
  }
  free(s->rowstart);
  free(s->col);
  free(s->val);
  s->rowstart = (int*)malloc(sizeof(int) * (k + 1));
  int nz = 0;
  for (int r = 0; r < k; ++r) nz += rows[r].n;
  s->col = (int*)malloc(sizeof(int) * (nz > 0 ? nz : 1));
  s->val = (double*)malloc(sizeof(double) * (nz > 0 ? nz : 1));
  nz = 0;
  for (int r = 0; r < k; ++r) {
    s->rowstart[r] = nz;
    for (int m = 0; m < rows[r].n; ++m) {
      s->col[nz] = rows[r].col[m];
      s->val[nz] = rows[r].val[m];
      ++nz;
    }
  }
  s->rowstart[k] = nz;
  free(rows);
}

/* ---------------------------------------------------------------------- */
/* MIC(0)-PCG: factor_modified_incomplete_cholesky0, solve_lower,
 * solve_lower_transpose_in_place and PCGSolver::solve
 * (PCGSolver/PCGSolver.h:97-308), on the CSR matrix (sorted rows). */
typedef struct {
  int n;
  double *invdiag, *adiag, *value;
  int *rowindex, *colstart;
} Factor;

static int row_has(const int* rs, const int* col, int j, int c) {
  for (int k = rs[j]; k < rs[j + 1]; ++k) {
    if (col[k] == c) return 1;
    if (col[k] > c) return 0;
  }
  return 0;
}

int wco_mic0_factor(int n, const int* rs, const int* col, const double* val, double omega,
                    double min_ratio, Factor* F) {
  F->n = n;
  F->invdiag = (double*)calloc(n > 0 ? n : 1, sizeof(double));
  F->adiag = (double*)calloc(n > 0 ? n : 1, sizeof(double));
  F->colstart = (int*)malloc(sizeof(int) * (n + 1));
  int nl = 0;
  for (int i = 0; i < n; ++i)
    for (int k = rs[i]; k < rs[i + 1]; ++k)
      if (col[k] > i) ++nl;
  F->value = (double*)malloc(sizeof(double) * (nl > 0 ? nl : 1));
  F->rowindex = (int*)malloc(sizeof(int) * (nl > 0 ? nl : 1));
  nl = 0;
  for (int i = 0; i < n; ++i) {
    F->colstart[i] = nl;
    for (int k = rs[i]; k < rs[i + 1]; ++k) {
      if (col[k] > i) {
        F->rowindex[nl] = col[k];
        F->value[nl] = val[k];
        ++nl;
      } else if (col[k] == i) {
        F->invdiag[i] = F->adiag[i] = val[k];
      }
    }
  }
  F->colstart[n] = nl;
  for (int k = 0; k < n; ++k) {
    if (F->adiag[k] == 0) continue;
    if (F->invdiag[k] < min_ratio * F->adiag[k])
      F->invdiag[k] = 1 / sqrt(F->adiag[k]);
    else
      F->invdiag[k] = 1 / sqrt(F->invdiag[k]);
    for (int p = F->colstart[k]; p < F->colstart[k + 1]; ++p) F->value[p] *= F->invdiag[k];
    for (int p = F->colstart[k]; p < F->colstart[k + 1]; ++p) {
      const int j = F->rowindex[p];
      const double mult = F->value[p];
      double missing = 0;
      int a = F->colstart[k];
      /* dropped entries above the diagonal of column j: row j of A lacks them */
      while (a < F->colstart[k + 1] && F->rowindex[a] < j) {
        if (!row_has(rs, col, j, F->rowindex[a])) missing += F->value[a];
        ++a;
      }
      if (a < F->colstart[k + 1] && F->rowindex[a] == j) F->invdiag[j] -= mult * F->value[a];
      ++a;
      int b = F->colstart[j];
      while (a < F->colstart[k + 1] && b < F->colstart[j + 1]) {
        if (F->rowindex[b] < F->rowindex[a]) {
          ++b;
        } else if (F->rowindex[b] == F->rowindex[a]) {
          F->value[b] -= mult * F->value[a];
          ++a;
          ++b;
        } else {
          missing += F->value[a];
          ++a;
        }
      }
      while (a < F->colstart[k + 1]) {
        missing += F->value[a];
        ++a;
      }
      F->invdiag[j] -= omega * mult * missing;
    }
  }
  return 0;
}

static void factor_free(Factor* F) {
  free(F->invdiag);
  free(F->adiag);
  free(F->value);
  free(F->rowindex);
  free(F->colstart);
}

static void apply_precond(const Factor* F, const double* x, double* out) {
  for (int i = 0; i < F->n; ++i) out[i] = x[i];
  for (int i = 0; i < F->n; ++i) {
    out[i] *= F->invdiag[i];
    for (int j = F->colstart[i]; j < F->colstart[i + 1]; ++j)
      out[F->rowindex[j]] -= F->value[j] * out[i];
  }
  for (int i = F->n - 1; i >= 0; --i) {
    for (int j = F->colstart[i]; j < F->colstart[i + 1]; ++j)
      out[i] -= F->value[j] * out[F->rowindex[j]];
    out[i] *= F->invdiag[i];
  }
}

static double dotv(const double* a, const double* b, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static double absmaxv(const double* a, int n) {
  double m = 0;
  for (int i = 0; i < n; ++i)
    if (fabs(a[i]) > m) m = fabs(a[i]);
  return m;
}

/* PCGSolver<double>::solve (PCGSolver.h:260-308); returns 1 on convergence */
int wco_pcg_solve(int n, const int* rs, const int* col, const double* val, const double* rhs,
                  double* result, double tol_factor, int maxiters, double omega,
                  double min_ratio, double* residual_out, int* iters_out) {
  for (int i = 0; i < n; ++i) result[i] = 0;
  double* r = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  double* z = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  double* sv = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) r[i] = rhs[i];
  int ok = 0;
  *residual_out = absmaxv(r, n);
  *iters_out = 0;
  if (*residual_out < 1e-30) {
    ok = 1;
    goto done;
  }
  {
    if (tol_factor < 1e-30) tol_factor = 1e-30;
    const double tol = tol_factor * *residual_out;
    Factor F;
    wco_mic0_factor(n, rs, col, val, omega, min_ratio, &F);
    apply_precond(&F, r, z);
    double rho = dotv(z, r, n);
    if (rho == 0 || rho != rho) {
      factor_free(&F);
      goto done;
    }
    for (int i = 0; i < n; ++i) sv[i] = z[i];
    int it;
    for (it = 0; it < maxiters; ++it) {
      for (int i = 0; i < n; ++i) {
        double acc = 0;
        for (int k = rs[i]; k < rs[i + 1]; ++k) acc += val[k] * sv[col[k]];
        z[i] = acc;
      }
      const double alpha = rho / dotv(sv, z, n);
      for (int i = 0; i < n; ++i) result[i] += alpha * sv[i];
      for (int i = 0; i < n; ++i) r[i] += -alpha * z[i];
      *residual_out = absmaxv(r, n);
      if (*residual_out <= tol) {
        *iters_out = it + 1;
        ok = 1;
        break;
      }
      apply_precond(&F, r, z);
      const double rho_new = dotv(z, r, n);
      const double beta = rho_new / rho;
      for (int i = 0; i < n; ++i) z[i] += beta * sv[i];
      double* t = sv;
      sv = z;
      z = t;
      rho = rho_new;
    }
    if (!ok) *iters_out = it;
    factor_free(&F);
  }
done:
  free(r);
  free(z);
  free(sv);
  return ok;
}

/* applyPressureGradsFluidRHS (Pressure.cpp:1137-1314), performInvLocalSolve
 * (LinearizedImplicitEuler.cpp:65-98), extrapolate (Pressure.cpp:1826-1903),
 * acceptVelocity and constrainLiquidVelocity (TwoDScene.cpp:1827-1869). */
static void apply_pressure(Scene* s, double dt) {
  const double dx = s->p.dx;
  double* u[3];
  for (int a = 0; a < 3; ++a) {
    u[a] = s->vel[a];  /* reused: the node fluid velocity after acceptVelocity */
    for (long long n = 0; n < s->nnode; ++n) {
      s->valid[a][n] = 0;
      if (!s->act[n >> 6]) continue;
      /* addSolidDragRHS (LinearizedImplicitEuler.cpp:689-717) */
      s->rhs[a][n] += s->mshdvm[a][n] * s->emass[a][n] * s->evel[a][n];
      if (s->wgt[a][n] > 0.) {
        int I, J, K;
        node_ijk(s, n, &I, &J, &K);
        const long long l = node_of(s, I - (a == 0), J - (a == 1), K - (a == 2));
        const int hl = node_active(s, l);
        const double lphi = hl ? s->lphi[l] : 0, rphi = s->lphi[n];
        if (lphi < 0.0 || rphi < 0.0) {
          double theta = 1.;
          if (rphi >= 0.0 || lphi >= 0.0) {
            theta = frac_in2(lphi, rphi);
            if (theta < 0.01) theta = 0.01;
          }
          double pg = 0;
          if (hl) pg -= s->pressure[l];
          pg += s->pressure[n];
          pg /= (dx * theta);
          const double term = pg * dt * (s->vol_f[a][n] + s->evol[a][n] * s->mshdvm[a][n]);
          s->rhs[a][n] -= term;
          s->valid[a][n] = 1;
        }
      }
      u[a][n] = s->rhs[a][n] * s->invC[a][n];
    }
    /* two layers of 6-neighbour averaging */
    double* cu = (double*)malloc(sizeof(double) * s->nnode);
    unsigned char* cv = (unsigned char*)malloc((size_t)s->nnode);
    for (int layer = 0; layer < 2; ++layer) {
      memcpy(cu, u[a], sizeof(double) * s->nnode);
      memcpy(cv, s->valid[a], (size_t)s->nnode);
      for (long long n = 0; n < s->nnode; ++n) {
        if (!s->act[n >> 6] || cv[n]) continue;
        int I, J, K;
        node_ijk(s, n, &I, &J, &K);
        static const int o[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        double sum = 0;
        int cnt = 0;
        for (int r = 0; r < 6; ++r) {
          const long long q = node_of(s, I + o[r][0], J + o[r][1], K + o[r][2]);
          if (!node_active(s, q) || !cv[q]) continue;
          sum += cu[q];
          ++cnt;
        }
        if (cnt > 0) {
          u[a][n] = sum / (double)cnt;
          s->valid[a][n] = 1;
        }
      }
    }
    free(cu);
    free(cv);
  }
}

static void constrain(Scene* s) {
  for (int a = 0; a < 3; ++a)
    for (long long n = 0; n < s->nnode; ++n) {
      if (!s->act[n >> 6]) continue;
      if (s->wgt[a][n] == 0.0)
        s->vel[a][n] = (1 - s->p.friction) * s->vel[a][n] + s->p.friction * s->svel[a][n];
    }
}

/* mapNodeParticlesAPIC (TwoDScene.cpp:6936-7090): liquid particles gather the
 * liquid face velocities into v and C (x flip_coeff); elasto particles other
 * than surfels gather the solid-phase velocities into v and B, then
 * v (twist included) *= elasto_advect_coeff and
 * B = ((f + g) B + (f - g) B^T) / 2 with f = elasto_flip_coeff,
 * g = elasto_flip_asym_coeff. */
static void g2p(Scene* s) {
  const double invD = 4.0 / (s->p.dx * s->p.dx);
  double* W[3] = {s->wu, s->wv, s->ww};
  for (int p = 0; p < s->np; ++p) {
    const int elasto = p < s->ne;
    if (elasto ? s->surf[p] : s->inside[p] == 0) continue;
    double fv[3] = {0, 0, 0}, B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int a = 0; a < 3; ++a) {
      const int* lo = &s->base[p * 15 + a * 3];
      const double off[3] = {a == 0 ? 0.0 : 0.5, a == 1 ? 0.0 : 0.5, a == 2 ? 0.0 : 0.5};
      const double* U = elasto ? s->evel[a] : s->vel[a];
      for (int sl = 0; sl < 27; ++sl) {
        const int I = lo[0] + sl % 3, J = lo[1] + (sl / 3) % 3, K = lo[2] + sl / 9;
        const long long n = node_of(s, I, J, K);
        if (!node_active(s, n)) continue;
        double np[3];
        stencil_node_pos(s, I, J, K, off, np);
        const double fnv = U[n];
        const double w = W[a][p * 27 + sl];
        fv[a] += fnv * w;
        for (int q = 0; q < 3; ++q) B[a * 3 + q] += fnv * w * (np[q] - s->x[p * 3 + q]) * invD;
      }
    }
    if (!elasto) {
      for (int a = 0; a < 3; ++a) s->v[p * 3 + a] = fv[a];
      for (int q = 0; q < 9; ++q) s->C[p * 9 + q] = B[q] * s->p.flip;
      continue;
    }
    const double ac = s->p.e_advect;
    for (int a = 0; a < 3; ++a) s->v[p * 3 + a] = fv[a] * ac;
    s->vt[p] *= ac;
    const double c1 = s->p.e_flip + s->p.e_asym, c2 = s->p.e_flip - s->p.e_asym;
    /* the reference assigns the blend into m_B's own block: Eigen evaluates
     * it coefficient by coefficient in column-major order, so entries above
     * the diagonal read the already blended entries below it */
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) B[i * 3 + j] = (c1 * B[i * 3 + j] + c2 * B[j * 3 + i]) * 0.5;
    for (int q = 0; q < 9; ++q) s->C[p * 9 + q] = B[q];
  }
}

/* SceneStepper::advectScene (SceneStepper.cpp:17-41): liquid x += v dt,
 * elasto x += v dt including the twist */
/* The solid phi seen by liquid particle p through its solid-phi stencil
 * (offset 0) with the weights m_particle_weights(., 3) of updateParticleWeights
 * (TwoDScene.cpp:2113-2127), i.e. taken at the position xw the sub-step's
 * weights were computed at:
 *   phi = sum phi_n w_n,  grad = sum phi_n iD w_n (x_n - pos),
 * grad normalised when its norm exceeds 1e-20; nodes of inactive buckets read
 * 3 dx (solidProjection :1786-1811, correctLiquidParticles :2030-2050). */
static void solid_sample(const Scene* s, int p, const double* xw, const double* pos,
                         double* phi_out, double* grad) {
  static const double off0[3] = {0.0, 0.0, 0.0};
  const double h = s->p.dx;
  const double iD = 4.0 / (h * h);
  const int* lo = &s->base[p * 15 + 9];
  double phi_ori = 0.0, g[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const int I = lo[0] + i, J = lo[1] + j, K = lo[2] + k;
        double np[3];
        stencil_node_pos(s, I, J, K, off0, np);
        const double w = quad_kernel((xw[0] - np[0]) / h) * quad_kernel((xw[1] - np[1]) / h) *
                         quad_kernel((xw[2] - np[2]) / h);
        const long long n = node_of(s, I, J, K);
        const double phi = node_active(s, n) ? s->sphi[n] : 3.0 * h;
        phi_ori += phi * w;
        const double c = phi * iD * w;
        for (int q = 0; q < 3; ++q) g[q] += c * (np[q] - pos[q]);
      }
  const double nrm = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if (nrm > 1e-20)
    for (int q = 0; q < 3; ++q) g[q] /= nrm;
  *phi_out = phi_ori;
  for (int q = 0; q < 3; ++q) grad[q] = g[q];
}

/* SceneStepper::advectScene (SceneStepper.cpp:17-41), then
 * TwoDScene::solidProjection (TwoDScene.cpp:1776-1821) of the liquid
 * particles: the solid phi extrapolated by the step just taken,
 * phi + grad . v dt, pushes a particle that ends inside back out along grad */
static void advect(Scene* s, double dt) {
  for (int p = 0; p < s->np; ++p) {
    for (int a = 0; a < 3; ++a) s->x[p * 3 + a] += s->v[p * 3 + a] * dt;
    if (p < s->ne) s->xt[p] += s->vt[p] * dt;
  }
  int projected = 0;
  for (int p = s->ne; p < s->np; ++p) {
    double* pos = &s->x[p * 3];
    double phi, g[3];
    solid_sample(s, p, &s->xw[p * 3], pos, &phi, g);
    const double d[3] = {s->v[p * 3] * dt, s->v[p * 3 + 1] * dt, s->v[p * 3 + 2] * dt};
    const double phi_now = phi + (g[0] * d[0] + g[1] * d[1] + g[2] * d[2]);
    if (phi_now < 0.0) {
      for (int q = 0; q < 3; ++q) pos[q] -= phi_now * g[q];
      ++projected;
    }
  }
  const long long pc = projected;
  snap_put_i(s, "projected", &pc, 1);
}

/* SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): the deterministic
 * stream that stands in for the reference's rand() and scalarRand */
static uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* correction selector of call k of a seeded stream */
int wco_correction_selector(uint64_t seed, uint64_t k, int step) {
  return (int)(splitmix64(seed ^ splitmix64(k)) % (uint64_t)(step > 0 ? step : 1));
}

/* uniform [0, 1) for the coincident-pair push of particles i, j (fluid
 * indices), component c */
static double pair_unit(int i, int j, int c) {
  const uint64_t key = ((uint64_t)(uint32_t)i << 34) ^ ((uint64_t)(uint32_t)j << 2) ^ (uint64_t)c;
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

/* TwoDScene::correctLiquidParticles (TwoDScene.cpp:1967-2061): Ando-style
 * relaxation of the liquid particles with fluid index i % step == selector.
 * Particles are sorted into the grid cells of rebucketizeParticles
 * (grid_num_cells :1662-1669; key cell floor((x - origin)/dx), clamped) and
 * visited in the 8-colour order of Sorter::for_each_bucket_particles_colored
 * (Sorter.h:403-437), each cell's particles in index order, reading the
 * positions as they are being moved.  Each pulls away from the neighbours of
 * the 27 cells around (Sorter.h:352-371 order: x outermost) within
 * re = sqrt(r_i r_j) * multiplier:
 *   spring += (strength/dt) smooth_kernel(d^2, re) (x_i - x_j) / d * re,
 * moves by spring dt and is projected out of the solid along the gradient of
 * the solid phi when phi + grad . (spring dt) < 0.  Pairs closer than
 * 1e-4 re get a push re * u with u uniform in [0, 1) per component: from
 * pair_unit here (scalarRand in the reference). */
static void correct_liquid(Scene* s, double dt, int selector) {
  const int nf = s->np - s->ne;
  if (nf == 0) return;
  const double dx = s->p.dx;
  const int step = s->p.corr_step > 0 ? s->p.corr_step : 1;
  int nc[3];
  for (int a = 0; a < 3; ++a) {
    const double content = (s->bbmax[a] - s->bbmin[a]) + s->bs * 3.0 * 2.0;
    nc[a] = (int)ceil(content / dx);
    if (nc[a] < 1) nc[a] = 1;
  }
  const long long ncell = (long long)nc[0] * nc[1] * nc[2];
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nf);
  for (int i = 0; i < nf; ++i) {
    const double* x = &s->x[(s->ne + i) * 3];
    int c[3];
    for (int a = 0; a < 3; ++a) {
      c[a] = (int)floor((x[a] - s->org[a]) / dx);
      if (c[a] < 0) c[a] = 0;
      if (c[a] > nc[a] - 1) c[a] = nc[a] - 1;
    }
    const uint64_t cell = ((uint64_t)c[2] * nc[1] + c[1]) * nc[0] + c[0];
    key[i] = (cell << 32) | (uint64_t)i;
  }
  qsort(key, nf, sizeof(uint64_t), cmp_u64);
  int* cs = (int*)calloc((size_t)ncell * 2, sizeof(int));
  for (int q = 0; q < nf; ++q) {
    const uint64_t b = key[q] >> 32;
    if (q == 0 || (key[q - 1] >> 32) != b) cs[b * 2] = q;
    if (q + 1 == nf || (key[q + 1] >> 32) != b) cs[b * 2 + 1] = q + 1;
  }
  const double coeff = s->p.corr_strength / dt;
  const int sn[3] = {(nc[0] + 1) / 2, (nc[1] + 1) / 2, (nc[2] + 1) / 2};
  for (int t = 0; t < 2; ++t)
    for (int u = 0; u < 2; ++u)
      for (int r = 0; r < 2; ++r)
        for (long long sb = 0; sb < (long long)sn[0] * sn[1] * sn[2]; ++sb) {
          const int sk = (int)(sb / ((long long)sn[0] * sn[1]));
          const int sj = (int)((sb - (long long)sk * sn[0] * sn[1]) / sn[0]);
          const int si = (int)(sb - (long long)sk * sn[0] * sn[1] - (long long)sj * sn[0]);
          const int ck = sk * 2 + t, cj = sj * 2 + u, ci = si * 2 + r;
          if (ck >= nc[2] || cj >= nc[1] || ci >= nc[0]) continue;
          const long long cell = ((long long)ck * nc[1] + cj) * nc[0] + ci;
          for (int q = cs[cell * 2]; q < cs[cell * 2 + 1]; ++q) {
            const int i = (int)(key[q] & 0xffffffffu);
            if (i % step != selector) continue;
            const int p = s->ne + i;
            double* pos = &s->x[p * 3];
            const double ri = s->rad[p];
            double spring[3] = {0.0, 0.0, 0.0};
            for (int x = ci - 1; x <= ci + 1; ++x)
              for (int y = cj - 1; y <= cj + 1; ++y)
                for (int z = ck - 1; z <= ck + 1; ++z) {
                  if (x < 0 || x > nc[0] - 1 || y < 0 || y > nc[1] - 1 || z < 0 || z > nc[2] - 1)
                    continue;
                  const long long nb = ((long long)z * nc[1] + y) * nc[0] + x;
                  for (int q2 = cs[nb * 2]; q2 < cs[nb * 2 + 1]; ++q2) {
                    const int j = (int)(key[q2] & 0xffffffffu);
                    if (j == i) continue;
                    const double* xn = &s->x[(s->ne + j) * 3];
                    const double re = sqrt(ri * s->rad[s->ne + j]) * s->p.corr_mult;
                    const double d[3] = {pos[0] - xn[0], pos[1] - xn[1], pos[2] - xn[2]};
                    const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    if (dist > re) continue;
                    const double sk3 = pow(1.0 - dist * dist / (re * re), 3.0);
                    const double w = coeff * (sk3 > 0.0 ? sk3 : 0.0);
                    if (w == 0.0) continue;
                    if (dist > 1e-4 * re) {
                      for (int a = 0; a < 3; ++a) spring[a] += w * d[a] / dist * re;
                    } else {
                      for (int a = 0; a < 3; ++a) spring[a] += re * pair_unit(i, j, a);
                    }
                  }
                }
            double buf[3];
            for (int a = 0; a < 3; ++a) buf[a] = pos[a] + spring[a] * dt;
            double phi, g[3];
            solid_sample(s, p, &s->xw[p * 3], pos, &phi, g);
            const double dp[3] = {spring[0] * dt, spring[1] * dt, spring[2] * dt};
            const double phi_now = phi + (g[0] * dp[0] + g[1] * dp[1] + g[2] * dp[2]);
            if (phi_now < 0.0)
              for (int a = 0; a < 3; ++a) buf[a] -= phi_now * g[a];
            for (int a = 0; a < 3; ++a) pos[a] = buf[a];
          }
        }
  free(cs);
  free(key);
}

static void snap_particles(Scene* s, const char* tag);

/* particle classes of relabelLiquidParticles (TwoDScene.h:31) */
enum { PCL_NONE = 0, PCL_S, PCL_s, PCL_o, PCL_l, PCL_L };

/* V_fine of relabelLiquidParticles / mergeLiquidParticles
 * (TwoDScene.cpp:2484-2489, 2518-2520) */
static double fine_volume(const Scene* s) {
  const double rad_fine = 1.0 / sqrt(3.0) * s->p.dx * s->p.cell_mult;
  return 4.0 / 3.0 * M_PI * rad_fine * rad_fine * rad_fine;
}

/* TwoDScene::relabelLiquidParticles (TwoDScene.cpp:2484-2505) */
static void relabel(Scene* s) {
  const double vf = fine_volume(s);
  free(s->cls);
  s->cls = (unsigned char*)calloc((size_t)(s->np > 0 ? s->np : 1), 1);
  for (int p = s->ne; p < s->np; ++p) {
    const double mrel = s->vol[p] / vf;
    s->cls[p] = mrel < 0.5 ? PCL_S : mrel <= 0.9 ? PCL_s : mrel <= 1.1 ? PCL_o
              : mrel <= 2.0 ? PCL_l : PCL_L;
  }
}

static void swap_d(double* a, int i, int j, int w) {
  for (int k = 0; k < w; ++k) {
    const double t = a[i * w + k];
    a[i * w + k] = a[j * w + k];
    a[j * w + k] = t;
  }
}

/* TwoDScene::removeEmptyParticles (TwoDScene.cpp:1713-1745): a liquid
 * particle with fluid volume below 1e-20 is swapped with the last one and
 * the count shrinks (swapParticles :176-208 on the liquid attributes) */
static int remove_empty(Scene* s) {
  int n = s->np;
  for (int i = s->ne; i < n;) {
    if (s->vol[i] < 1e-20) {
      --n;
      swap_d(s->x, i, n, 3);
      swap_d(s->v, i, n, 3);
      swap_d(s->C, i, n, 9);
      swap_d(s->m, i, n, 1);
      swap_d(s->vol, i, n, 1);
      swap_d(s->rad, i, n, 1);
      if (s->cls) {
        const unsigned char t = s->cls[i];
        s->cls[i] = s->cls[n];
        s->cls[n] = t;
      }
    } else {
      ++i;
    }
  }
  const int removed = s->np - n;
  s->np = n;
  return removed;
}

/* TwoDScene::mergeLiquidParticles (TwoDScene.cpp:2510-2666) after
 * updateOptiVolume's relabelling: the small (S) and the large-ish (l) liquid
 * particles of the subset index % step == selector, visited bucket by bucket
 * in the 27 colours of Sorter::for_each_bucket_particles_colored_randomized
 * (Sorter.h:439-480, numcolors 3, colour order perm_t x perm_s x perm_r), hand
 * their volume (S: all of it, then they are removed; l: the part above V_fine,
 * then they shrink to V_fine) and the matching momentum in equal parts to the
 * neighbours within 2 r_fine in the 27 buckets around (S: to S, s and o
 * particles; l: to s particles) holding no more than V_fine; then every
 * particle that gathered volume takes the volume-weighted mean velocity and
 * the radius of its new volume, empty particles are removed and all are
 * relabelled.  The bucket lists are those of the last grid build (the
 * reference merges before the step's rebucketizeParticles).  The reference
 * draws the selector and the three colour permutations with rand(); here
 * they are arguments. */
int wco_merge_liquid(Scene* s, int selector, const int* perm_t, const int* perm_s,
                     const int* perm_r) {
  if (!s->keys || s->np == s->ne) return 0;
  relabel(s);
  const double vf = fine_volume(s);
  const double rad_fine = 1.0 / sqrt(3.0) * s->p.dx * s->p.cell_mult;
  const double should_rad = rad_fine * 2.0;
  const int step = s->p.corr_step > 0 ? s->p.corr_step : 1;
  const int np = s->np;
  unsigned char* removed = (unsigned char*)calloc((size_t)np, 1);
  double* gvol = (double*)calloc((size_t)np, sizeof(double));
  double* gmom = (double*)calloc((size_t)np * 3, sizeof(double));
  const int nc = 3;
  const int sn[3] = {(s->ni + nc - 1) / nc, (s->nj + nc - 1) / nc, (s->nk + nc - 1) / nc};
  for (int a = 0; a < nc; ++a)
    for (int b = 0; b < nc; ++b)
      for (int c = 0; c < nc; ++c) {
        const int t = perm_t[a], u = perm_s[b], r = perm_r[c];
        for (long long sb = 0; sb < (long long)sn[0] * sn[1] * sn[2]; ++sb) {
          const int sk = (int)(sb / ((long long)sn[0] * sn[1]));
          const int sj = (int)((sb - (long long)sk * sn[0] * sn[1]) / sn[0]);
          const int si = (int)(sb - (long long)sk * sn[0] * sn[1] - (long long)sj * sn[0]);
          const int k = sk * nc + t, j = sj * nc + u, i = si * nc + r;
          if (k >= s->nk || j >= s->nj || i >= s->ni) continue;
          const long long bkt = bucket_index(s, i, j, k);
          for (int q = s->sup[bkt * 2]; q < s->sup[bkt * 2 + 1]; ++q) {
            const int p = (int)(s->keys[q] & 0xffffffffu);
            if (p < s->ne || (s->cls[p] != PCL_S && s->cls[p] != PCL_l)) continue;
            if (p % step != selector) continue;
            const int small = s->cls[p] == PCL_S;
            const double full_vol = s->vol[p] + gvol[p];
            if (!small && full_vol < 1e-20) continue;
            const double mrel = full_vol / vf;
            if (small && mrel >= 0.5) {
              s->cls[p] = PCL_s;
              continue;
            }
            if (!small && mrel > 2.0) {
              s->cls[p] = PCL_L;
              continue;
            }
            /* partners in the 27 buckets around, x outermost (Sorter.h:352-371);
             * counted first, then served, both with the same test */
            int npart = 0;
            for (int pass = 0; pass < 2; ++pass) {
              double dvol = 0.0, dmom[3] = {0.0, 0.0, 0.0};
              if (pass == 1) {
                if (npart == 0) break;
                const double invN = 1.0 / (double)npart;
                if (small) {
                  dvol = full_vol * invN;
                  for (int a2 = 0; a2 < 3; ++a2)
                    dmom[a2] = (s->v[p * 3 + a2] * s->vol[p] + gmom[p * 3 + a2]) * invN;
                } else {
                  const double ex_vol = full_vol - vf;
                  dvol = ex_vol * invN;
                  const double coeff = dvol / full_vol;
                  for (int a2 = 0; a2 < 3; ++a2)
                    dmom[a2] = (s->v[p * 3 + a2] * s->vol[p] + gmom[p * 3 + a2]) * coeff;
                }
              }
              for (int x = i - 1; x <= i + 1; ++x)
                for (int y = j - 1; y <= j + 1; ++y)
                  for (int z = k - 1; z <= k + 1; ++z) {
                    if (x < 0 || x > s->ni - 1 || y < 0 || y > s->nj - 1 || z < 0 ||
                        z > s->nk - 1)
                      continue;
                    const long long nb = bucket_index(s, x, y, z);
                    for (int q2 = s->sup[nb * 2]; q2 < s->sup[nb * 2 + 1]; ++q2) {
                      const int n = (int)(s->keys[q2] & 0xffffffffu);
                      if (n == p || n < s->ne || removed[n]) continue;
                      const int c2 = s->cls[n];
                      if (small ? !(c2 == PCL_S || c2 == PCL_s || c2 == PCL_o) : c2 != PCL_s)
                        continue;
                      const double neigh_vol = s->vol[n] + gvol[n];
                      if (neigh_vol > vf) continue;
                      const double d[3] = {s->x[p * 3] - s->x[n * 3], s->x[p * 3 + 1] - s->x[n * 3 + 1],
                                           s->x[p * 3 + 2] - s->x[n * 3 + 2]};
                      const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                      if (!(dist < should_rad)) continue;
                      if (pass == 0) {
                        ++npart;
                      } else {
                        gvol[n] += dvol;
                        for (int a2 = 0; a2 < 3; ++a2) gmom[n * 3 + a2] += dmom[a2];
                      }
                    }
                  }
            }
            if (npart == 0) continue;
            if (small) {
              removed[p] = 1;
              s->vol[p] = 0.0;
              gvol[p] = 0.0;
              for (int a2 = 0; a2 < 3; ++a2) gmom[p * 3 + a2] = 0.0;
            } else {
              const double scaling = vf / full_vol;
              const double rad_scaling = pow(scaling, 1.0 / 3.0);
              s->vol[p] *= scaling;
              s->m[p] *= scaling;
              s->rad[p] *= rad_scaling;
              s->cls[p] = PCL_o;
            }
          }
        }
      }
  /* gather and update (:2649-2666) */
  for (int p = s->ne; p < np; ++p) {
    if (removed[p] || gvol[p] == 0.0) continue;
    double fm[3];
    for (int a2 = 0; a2 < 3; ++a2) fm[a2] = s->v[p * 3 + a2] * s->vol[p] + gmom[p * 3 + a2];
    const double full_vol = s->vol[p] + gvol[p];
    const double full_rad = pow(full_vol * 0.75 / M_PI, 1.0 / 3.0);
    const double inv = 1.0 / full_vol;
    s->vol[p] = full_vol;
    for (int a2 = 0; a2 < 3; ++a2) s->v[p * 3 + a2] = fm[a2] * inv;
    s->m[p] = full_vol * s->p.rho;
    s->rad[p] = full_rad;
  }
  free(removed);
  free(gvol);
  free(gmom);
  const int nrem = remove_empty(s);
  relabel(s);
  {
    const int n = s->np;
    double* t = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    long long* c = (long long*)malloc(sizeof(long long) * (size_t)(n > 0 ? n : 1));
    snap_particles(s, "merge_");
    memcpy(t, s->vol, sizeof(double) * (size_t)n);
    snap_put_f(s, "merge_vol", t, n);
    memcpy(t, s->m, sizeof(double) * (size_t)n);
    snap_put_f(s, "merge_mass", t, n);
    memcpy(t, s->rad, sizeof(double) * (size_t)n);
    snap_put_f(s, "merge_radius", t, n);
    for (int p = 0; p < n; ++p) c[p] = s->cls[p];
    snap_put_i(s, "merge_class", c, n);
    free(t);
    free(c);
  }
  free(s->keys);
  s->keys = NULL;  /* the bucket lists no longer match the particles */
  return nrem;
}

/* the draws of merge call k of a seeded stream: selector, then three
 * Fisher-Yates permutations of {0, 1, 2} (mathutils::fisherYates,
 * MathUtilities.h:238-245, on SplitMix64 draws) */
void wco_merge_draws(uint64_t seed, uint64_t k, int step, int* selector, int* perm9) {
  uint64_t z = splitmix64(seed ^ splitmix64(k ^ 0x6d657267652d6b65ull));
  *selector = (int)(z % (uint64_t)(step > 0 ? step : 1));
  for (int q = 0; q < 3; ++q) {
    int* pq = perm9 + 3 * q;
    pq[0] = 0;
    pq[1] = 1;
    pq[2] = 2;
    for (int i = 2; i >= 1; --i) {
      z = splitmix64(z);
      const int j = (int)(z % (uint64_t)(i + 1));
      const int t = pq[i];
      pq[i] = pq[j];
      pq[j] = t;
    }
  }
}

/* merge before each sub-step with the seeded draws; LiquidInfo
 * particle_cell_multiplier */
void wco_set_merge(Scene* s, int on, uint64_t seed, double cell_mult) {
  s->p.merge_on = on;
  s->merge_seed = seed;
  s->merge_count = 0;
  s->p.cell_mult = cell_mult;
}

/* point i of n on the unit sphere (spherical Fibonacci lattice, golden angle
 * pi (3 - sqrt 5)): the children's pattern of the particle split */
static void sphere_point(int n, int i, double* p) {
  const double y = 1.0 - (2.0 * i + 1.0) / (double)n;
  const double r = sqrt(1.0 - y * y);
  const double phi = (double)i * 2.3999632297286533;
  p[0] = r * cos(phi);
  p[1] = y;
  p[2] = r * sin(phi);
}

/* rotation of a split parent: a uniform random unit quaternion (Shoemake,
 * Graphics Gems III, 1992) from SplitMix64 draws of key */
static void split_rotation(uint64_t key, double* Q) {
  uint64_t z = splitmix64(key);
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

/* the key of split call k of a seeded stream */
uint64_t wco_split_key(uint64_t seed, uint64_t k) {
  return splitmix64(seed ^ splitmix64(k ^ 0x73706c69742d6b65ull));
}

static double* grow_d(double* a, int w, int oldn, int newn) {
  double* b = (double*)calloc((size_t)w * (size_t)(newn > 0 ? newn : 1), sizeof(double));
  if (a) memcpy(b, a, sizeof(double) * (size_t)w * (size_t)oldn);
  free(a);
  return b;
}

/* TwoDScene::splitLiquidParticles (TwoDScene.cpp:2362-2480) after
 * updateOptiVolume's relabelling: every large (L) liquid particle splits
 * into n = min(ceil(V / V_fine), 32) particles of volume V/n and radius
 * (3 V / (4 pi n))^(1/3); the parent moves to centre + p_0 s and its n - 1
 * children, appended after all particles in the parents' index order, sit at
 * centre + Q p_i s, s = 0.75 max(r_new, r - r_new), with the parent's
 * velocity and a zero affine matrix.  The pattern p_i and the rotation Q are
 * this library's (sphere_point, split_rotation with the parent's key
 * splitmix64(key ^ fluid index)); the reference takes p_i from its
 * compiled pattern table and Q from Matrix3s::Random().  Returns the number
 * of particles added. */
int wco_split_liquid(Scene* s, uint64_t key) {
  if (s->np == s->ne) return 0;
  relabel(s);
  const double vf = fine_volume(s);
  const int np = s->np, nf = s->np - s->ne;
  int* add = (int*)calloc((size_t)nf, sizeof(int));
  int total = 0;
  for (int f = 0; f < nf; ++f) {
    const int p = s->ne + f;
    if (s->cls[p] != PCL_L) continue;
    int n = (int)ceil(s->vol[p] / vf);
    if (n > 32) n = 32;
    if (n <= 1) continue;
    add[f] = n - 1;
    total += n - 1;
  }
  if (total == 0) {
    free(add);
    return 0;
  }
  const int nn = np + total;
  s->x = grow_d(s->x, 3, np, nn);
  s->v = grow_d(s->v, 3, np, nn);
  s->C = grow_d(s->C, 9, np, nn);
  s->m = grow_d(s->m, 1, np, nn);
  s->vol = grow_d(s->vol, 1, np, nn);
  s->rad = grow_d(s->rad, 1, np, nn);
  if (s->em) {
    s->em = grow_d(s->em, 3, np, nn);
    s->rvol = grow_d(s->rvol, 1, np, nn);
    s->rvf = grow_d(s->rvf, 1, np, nn);
    s->sf = grow_d(s->sf, 1, np, nn);
    s->ori = grow_d(s->ori, 3, np, nn);
    s->xt = grow_d(s->xt, 1, np, nn);
    s->vt = grow_d(s->vt, 1, np, nn);
    unsigned char* su = (unsigned char*)calloc((size_t)nn, 1);
    memcpy(su, s->surf, (size_t)np);
    free(s->surf);
    s->surf = su;
  }
  int next = np;
  for (int f = 0; f < nf; ++f) {
    if (!add[f]) continue;
    const int p = s->ne + f;
    const int n = add[f] + 1;
    const double c[3] = {s->x[p * 3], s->x[p * 3 + 1], s->x[p * 3 + 2]};
    const double rad = s->rad[p];
    const double new_vol = s->vol[p] / (double)n;
    const double new_rad = pow(new_vol / M_PI * 0.75, 1.0 / 3.0);
    const double splat = (new_rad > rad - new_rad ? new_rad : rad - new_rad) * 0.75;
    double Q[9];
    split_rotation(splitmix64(key ^ (uint64_t)f), Q);
    for (int i = 1; i < n; ++i) {
      double pt[3];
      sphere_point(n, i, pt);
      const int q = next++;
      for (int a = 0; a < 3; ++a) {
        const double rq = Q[a * 3] * pt[0] + Q[a * 3 + 1] * pt[1] + Q[a * 3 + 2] * pt[2];
        s->x[q * 3 + a] = c[a] + rq * splat;
        s->v[q * 3 + a] = s->v[p * 3 + a];
      }
      for (int r = 0; r < 9; ++r) s->C[q * 9 + r] = 0.0;
      s->m[q] = new_vol * s->p.rho;
      s->vol[q] = new_vol;
      s->rad[q] = new_rad;
    }
    double p0[3];
    sphere_point(n, 0, p0);
    for (int a = 0; a < 3; ++a) s->x[p * 3 + a] = c[a] + p0[a] * splat;
    s->rad[p] = new_rad;
    s->vol[p] = new_vol;
    s->m[p] = new_vol * s->p.rho;
  }
  s->np = nn;
  free(add);
  relabel(s);
  free(s->keys);
  s->keys = NULL;
  {
    double* t = (double*)malloc(sizeof(double) * (size_t)nn);
    long long* c = (long long*)malloc(sizeof(long long) * (size_t)nn);
    snap_particles(s, "split_");
    memcpy(t, s->vol, sizeof(double) * (size_t)nn);
    snap_put_f(s, "split_vol", t, nn);
    memcpy(t, s->m, sizeof(double) * (size_t)nn);
    snap_put_f(s, "split_mass", t, nn);
    memcpy(t, s->rad, sizeof(double) * (size_t)nn);
    snap_put_f(s, "split_radius", t, nn);
    for (int p = 0; p < nn; ++p) c[p] = s->cls[p];
    snap_put_i(s, "split_class", c, nn);
    free(t);
    free(c);
  }
  return total;
}

/* TwoDScene::terminateParticles (TwoDScene.cpp:1756-1771): a liquid particle
 * where the terminator's phi is negative loses its fluid volume, then
 * removeEmptyParticles drops every liquid particle without volume.  Returns
 * the particles removed. */
int wco_terminate_liquid(Scene* s) {
  if (s->bs <= 0.0) s->bs = s->p.dx * NN;
  for (int i = s->ne; i < s->np; ++i)
    if (s->p.term_on && term_phi(s, s->x[i * 3], s->x[i * 3 + 1], s->x[i * 3 + 2]) < 0.0)
      s->vol[i] = 0.0;
  const int removed = remove_empty(s);
  snap_particles(s, "term_");
  /* removeEmptyParticles re-sorts the bucket lists after a removal
   * (TwoDScene.cpp:1734-1743) */
  if (removed > 0 && s->keys && s->nb > 0) sort_particles(s);
  return removed;
}

/* the terminator box (inside: 1 removes the particles that leave it, 0 the
 * ones that enter it) */
void wco_set_terminator(Scene* s, int on, const double* c, const double* h, double r,
                        int inside) {
  s->p.term_on = on;
  for (int a = 0; a < 3; ++a) {
    s->p.tc[a] = c[a];
    s->p.th[a] = h[a];
  }
  s->p.tr = r;
  s->p.tsign = inside ? -1.0 : 1.0;
}

/* terminator shapes: type (0 box, 1 sphere, 2 capsule, 3 cylinder), inside,
 * centre (3 each), rotation quaternion w x y z (4 each), parameters (4 each);
 * n = 0 removes them */
void wco_set_terminators(Scene* s, int n, const int* type, const int* inside,
                         const double* c, const double* q, const double* par) {
  s->p.nshape = n < 0 ? 0 : (n > 16 ? 16 : n);
  for (int k = 0; k < s->p.nshape; ++k) {
    s->p.stype[k] = type[k];
    s->p.ssign[k] = inside[k] ? -1.0 : 1.0;
    for (int j = 0; j < 3; ++j) s->p.sc[k][j] = c[3 * k + j];
    for (int j = 0; j < 4; ++j) {
      s->p.sq[k][j] = q[4 * k + j];
      s->p.spar[k][j] = par[4 * k + j];
    }
  }
  s->p.term_on = s->p.nshape > 0;
}

/* split before each sub-step with the seeded keys */
void wco_set_split(Scene* s, int on, uint64_t seed) {
  s->p.split_on = on;
  s->split_seed = seed;
  s->split_count = 0;
}

/* correctLiquidParticles with an explicit particle subset, outside a step */
void wco_correct_liquid(Scene* s, double dt, int selector) { correct_liquid(s, dt, selector); }

/* LiquidInfo correction_strength / _step / _multiplier and the seed of the
 * selector stream (strength 0: off) */
void wco_set_correction(Scene* s, double strength, int step, double mult, uint64_t seed) {
  s->p.corr_strength = strength;
  s->p.corr_step = step > 0 ? step : 1;
  s->p.corr_mult = mult;
  s->corr_seed = seed;
  s->corr_count = 0;
  s->corr_sel_once = -1;
}

/* the selector the next correction uses instead of the seeded stream's */
void wco_set_correction_selector(Scene* s, int selector) { s->corr_sel_once = selector; }

/* ---------------------------------------------------------------------- */
static void alloc_nodes(Scene* s) {
  const size_t n = (size_t)s->nnode;
  for (int a = 0; a < 3; ++a) {
    double** F[] = {&s->mass[a], &s->vel[a], &s->vol_f[a], &s->sat[a], &s->psi[a], &s->wgt[a],
                    &s->svel[a], &s->rhs[a], &s->vstar[a], &s->invC[a], &s->psifs[a],
                    &s->psisf[a], &s->mshdvm[a], &s->mfhdvm[a], &s->emass[a], &s->evel[a],
                    &s->evol[a], &s->esf[a]};
    for (size_t k = 0; k < sizeof(F) / sizeof(F[0]); ++k) {
      free(*F[k]);
      *F[k] = (double*)calloc(n, sizeof(double));
    }
    free(s->eori[a]);
    s->eori[a] = (double*)calloc(3 * n, sizeof(double));
    free(s->valid[a]);
    s->valid[a] = (unsigned char*)calloc(n, 1);
  }
  double** G[] = {&s->sat_p, &s->psi_p, &s->pore_p, &s->lphi, &s->sphi, &s->pressure,
                  &s->vf_c, &s->vf_e[0], &s->vf_e[1], &s->vf_e[2], &s->vf_f[0],
                  &s->vf_f[1], &s->vf_f[2]};
  for (size_t k = 0; k < sizeof(G) / sizeof(G[0]); ++k) {
    free(*G[k]);
    *G[k] = (double*)calloc(n, sizeof(double));
  }
  const size_t np = (size_t)(s->np > 0 ? s->np : 1);
  double** Wt[] = {&s->wu, &s->wv, &s->ww, &s->wp};
  for (int k = 0; k < 4; ++k) {
    free(*Wt[k]);
    *Wt[k] = (double*)calloc(np * 27, sizeof(double));
  }
}

static void snap_particles(Scene* s, const char* tag) {
  char nm[32];
  snprintf(nm, sizeof nm, "%sx", tag);
  snap_put_f(s, nm, s->x, (long long)s->np * 3);
  /* m_fluid_v and m_fB: liquid entries, zeros for elasto particles */
  double* fv = (double*)malloc(sizeof(double) * 3 * (size_t)(s->np > 0 ? s->np : 1));
  double* fb = (double*)malloc(sizeof(double) * 9 * (size_t)(s->np > 0 ? s->np : 1));
  for (int p = 0; p < s->np; ++p) {
    for (int a = 0; a < 3; ++a) fv[p * 3 + a] = p < s->ne ? 0.0 : s->v[p * 3 + a];
    for (int q = 0; q < 9; ++q) fb[p * 9 + q] = p < s->ne ? 0.0 : s->C[p * 9 + q];
  }
  snprintf(nm, sizeof nm, "%sv", tag);
  snap_put_f(s, nm, fv, (long long)s->np * 3);
  snprintf(nm, sizeof nm, "%sC", tag);
  snap_put_f(s, nm, fb, (long long)s->np * 9);
  free(fv);
  free(fb);
  /* m_x and m_v with their 4th (twist) components, m_B: elasto entries,
   * zeros for liquid particles */
  const size_t n = (size_t)(s->np > 0 ? s->np : 1);
  double* x4 = (double*)calloc(4 * n, sizeof(double));
  double* v4 = (double*)calloc(4 * n, sizeof(double));
  double* b9 = (double*)calloc(9 * n, sizeof(double));
  for (int p = 0; p < s->np; ++p) {
    for (int a = 0; a < 3; ++a) x4[p * 4 + a] = s->x[p * 3 + a];
    if (p >= s->ne) continue;
    x4[p * 4 + 3] = s->xt[p];
    for (int a = 0; a < 3; ++a) v4[p * 4 + a] = s->v[p * 3 + a];
    v4[p * 4 + 3] = s->vt[p];
    for (int q = 0; q < 9; ++q) b9[p * 9 + q] = s->C[p * 9 + q];
  }
  snprintf(nm, sizeof nm, "%sx4", tag);
  snap_put_f(s, nm, x4, (long long)s->np * 4);
  snprintf(nm, sizeof nm, "%sev4", tag);
  snap_put_f(s, nm, v4, (long long)s->np * 4);
  snprintf(nm, sizeof nm, "%seB", tag);
  snap_put_f(s, nm, b9, (long long)s->np * 9);
  free(x4);
  free(v4);
  free(b9);
}

/* grid, weights and P2G of a sub-step (WetClothCore.cpp:115-160) */
static void transfer_in(Scene* s, int snapshot) {
  build_grid(s);
  sort_particles(s);
  resample_nodes(s);
  alloc_nodes(s);
  if (snapshot) {
    const double org[3] = {s->org[0], s->org[1], s->org[2]};
    const double bbx[6] = {s->bbmin[0], s->bbmin[1], s->bbmin[2], s->bbmax[0], s->bbmax[1], s->bbmax[2]};
    const long long dims[3] = {s->ni, s->nj, s->nk};
    snap_put_f(s, "grid_origin", org, 3);
    snap_put_f(s, "bbx", bbx, 6);
    snap_put_i(s, "grid_dims", dims, 3);
    long long* t = (long long*)malloc(sizeof(long long) * (s->np + 2 * s->nb + 15 * (long long)s->np + s->nb + 2));
    for (int q = 0; q < s->np; ++q) t[q] = (long long)s->keys[q];
    snap_put_i(s, "array_idx", t, s->np);
    for (long long b = 0; b < 2 * s->nb; ++b) t[b] = s->sup[b];
    snap_put_i(s, "array_sup", t, 2 * s->nb);
    for (long long b = 0; b < s->nb; ++b) t[b] = s->act[b];
    snap_put_i(s, "active", t, s->nb);
    for (long long k = 0; k < 15 * (long long)s->np; ++k) t[k] = s->base[k];
    snap_put_i(s, "stencil_base", t, 15 * (long long)s->np);
    for (int q = 0; q < s->np; ++q) t[q] = s->inside[q];
    snap_put_i(s, "inside", t, s->np);
    free(t);
  }
  compute_weights(s);
  build_pairs(s, &s->pu, s->wu, 0);
  build_pairs(s, &s->pv, s->wv, 1);
  build_pairs(s, &s->pw, s->ww, 2);
  build_pairs(s, &s->pp, s->wp, 4);
  liquid_phi(s);
  if (s->p.visc > 0.0) volume_fractions(s);
  solid_phi_and_weights(s);
  p2g(s);
  sat_psi_p(s);
  if (snapshot) {
    static const char* xyz = "xyz";
    char nm[32];
    for (int a = 0; a < 3; ++a) {
      snprintf(nm, sizeof nm, "mass_fluid_%c", xyz[a]); snap_node(s, nm, s->mass[a]);
      snprintf(nm, sizeof nm, "vel_fluid_%c", xyz[a]); snap_node(s, nm, s->vel[a]);
      snprintf(nm, sizeof nm, "vol_fluid_%c", xyz[a]); snap_node(s, nm, s->vol_f[a]);
      if (s->p.visc > 0.0) {
        snprintf(nm, sizeof nm, "liquid_e%c_vf", xyz[a]); snap_node(s, nm, s->vf_e[a]);
        if (s->p.visc_implicit) {
          snprintf(nm, sizeof nm, "liquid_%c_vf", "uvw"[a]); snap_node(s, nm, s->vf_f[a]);
        }
      }
      snprintf(nm, sizeof nm, "sat_%c", xyz[a]); snap_node(s, nm, s->sat[a]);
      snprintf(nm, sizeof nm, "psi_%c", xyz[a]); snap_node(s, nm, s->psi[a]);
      snprintf(nm, sizeof nm, "solid_weight_%c", xyz[a]); snap_node(s, nm, s->wgt[a]);
      snprintf(nm, sizeof nm, "solid_vel_%c", xyz[a]); snap_node(s, nm, s->svel[a]);
      snprintf(nm, sizeof nm, "mass_%c", xyz[a]); snap_node(s, nm, s->emass[a]);
      snprintf(nm, sizeof nm, "vel_%c", xyz[a]); snap_node(s, nm, s->evel[a]);
      snprintf(nm, sizeof nm, "vol_%c", xyz[a]); snap_node(s, nm, s->evol[a]);
      snprintf(nm, sizeof nm, "shape_factor_%c", xyz[a]); snap_node(s, nm, s->esf[a]);
      snprintf(nm, sizeof nm, "orientation_%c", xyz[a]);
      double* t = (double*)malloc(sizeof(double) * 3 * (size_t)s->nnode);
      for (long long n = 0; n < s->nnode; ++n)
        for (int q = 0; q < 3; ++q) t[n * 3 + q] = s->act[n >> 6] ? s->eori[a][n * 3 + q] : NAN;
      snap_put_f(s, nm, t, 3 * s->nnode);
      free(t);
    }
    snap_node(s, "sat_p", s->sat_p);
    snap_node(s, "psi_p", s->psi_p);
    snap_node(s, "pore_pressure_p", s->pore_p);
    snap_node(s, "liquid_phi", s->lphi);
    if (s->p.visc > 0.0) snap_node(s, "liquid_c_vf", s->vf_c);
    snap_node(s, "solid_phi", s->sphi);
  }
}

/* particle correction, G2P and advection of a sub-step
 * (WetClothCore.cpp:241-262); G2P keeps the weights of the positions before
 * the correction and measures x_n - x_p from the corrected ones */
static void transfer_out(Scene* s, double dt, int snapshot, int correct) {
  /* correctLiquidParticles runs in every sub-step; at strength 0 its spring
   * weights vanish and it only projects its particle subset out of the solid */
  if (correct && s->np > s->ne) {
    int sel = s->corr_sel_once;
    if (sel < 0) sel = wco_correction_selector(s->corr_seed, s->corr_count, s->p.corr_step);
    s->corr_sel_once = -1;
    ++s->corr_count;
    correct_liquid(s, dt, sel);
    const long long sl = sel;
    snap_put_i(s, "correction_selector", &sl, 1);
    if (snapshot) snap_particles(s, "corr_");
  }
  g2p(s);
  if (snapshot) snap_particles(s, "g2p_");
  advect(s, dt);
  if (snapshot) snap_particles(s, "adv_");
}

/* one sub-step in WetClothCore::stepSystem order (WetClothCore.cpp:97-258) */
int wco_substep(Scene* s, double dt, int snapshot) {
  /* updateOptiVolume, splitLiquidParticles, mergeLiquidParticles
   * (WetClothCore.cpp:97-110); a split that adds particles re-sorts the
   * buckets (TwoDScene.cpp:2471-2478), so the merge after it sees the new
   * positions in the buckets of the last grid build */
  /* terminateParticles runs every sub-step; without a terminator its
   * removeEmptyParticles still drops liquid particles without fluid volume */
  int any_empty = 0;
  for (int i = s->ne; i < s->np && !any_empty; ++i) any_empty = s->vol[i] < 1e-20;
  if (s->p.term_on || any_empty) {
    const long long nrem = wco_terminate_liquid(s);
    snap_put_i(s, "terminate_removed", &nrem, 1);
  }
  if (s->p.split_on && s->np > s->ne) {
    const long long nadd = wco_split_liquid(s, wco_split_key(s->split_seed, s->split_count++));
    snap_put_i(s, "split_added", &nadd, 1);
    if (nadd > 0 && s->p.merge_on && s->nb > 0) sort_particles(s);
  }
  if (s->p.merge_on && s->keys && s->np > s->ne) {
    int sel, perm[9];
    wco_merge_draws(s->merge_seed, s->merge_count++, s->p.corr_step, &sel, perm);
    const long long nrem = wco_merge_liquid(s, sel, perm, perm + 3, perm + 6);
    snap_put_i(s, "merge_removed", &nrem, 1);
  }
  transfer_in(s, snapshot);
  step_velocity(s, dt);
  if (snapshot) {
    static const char* xyz = "xyz";
    char nm[32];
    for (int a = 0; a < 3; ++a) {
      snprintf(nm, sizeof nm, "v_star_%c", xyz[a]); snap_node(s, nm, s->vstar[a]);
      snprintf(nm, sizeof nm, "rhs_fluid_%c", xyz[a]); snap_node(s, nm, s->rhs[a]);
      snprintf(nm, sizeof nm, "inv_C_%c", xyz[a]); snap_node(s, nm, s->invC[a]);
      snprintf(nm, sizeof nm, "psi_fs_%c", xyz[a]); snap_node(s, nm, s->psifs[a]);
    }
  }
  /* acceptVelocity: the scene's node fluid velocity becomes u* */
  for (int a = 0; a < 3; ++a) memcpy(s->vel[a], s->vstar[a], sizeof(double) * s->nnode);
  assemble(s, dt);
  if (snapshot) {
    long long* rs = (long long*)malloc(sizeof(long long) * (s->ndof + 1));
    long long* cl = (long long*)malloc(sizeof(long long) * (s->rowstart[s->ndof] + 1));
    for (int r = 0; r <= s->ndof; ++r) rs[r] = s->rowstart[r];
    for (int k = 0; k < s->rowstart[s->ndof]; ++k) cl[k] = s->col[k];
    snap_put_i(s, "A_rowstart", rs, s->ndof + 1);
    snap_put_i(s, "A_col", cl, s->rowstart[s->ndof]);
    snap_put_f(s, "A_val", s->val, s->rowstart[s->ndof]);
    snap_put_f(s, "b", s->b, s->ndof);
    snap_put_i(s, "dof_index", s->dofidx, s->nnode);
    free(rs);
    free(cl);
  }
  double* res = (double*)calloc(s->ndof > 0 ? s->ndof : 1, sizeof(double));
  double rr = 0;
  int it = 0;
  if (s->ndof > 0)
    wco_pcg_solve(s->ndof, s->rowstart, s->col, s->val, s->b, res, s->p.criterion,
                  s->p.maxiters, 0.97, 0.25, &rr, &it);
  s->last_iters = it;
  s->last_res = rr;
  for (long long n = 0; n < s->nnode; ++n)
    if (s->dofidx[n] >= 0) s->pressure[n] = res[s->dofidx[n]];
  free(res);
  if (snapshot) snap_node(s, "pressure", s->pressure);
  apply_pressure(s, dt);
  if (snapshot) {
    static const char* xyz = "xyz";
    char nm[32];
    for (int a = 0; a < 3; ++a) {
      snprintf(nm, sizeof nm, "u_proj_%c", xyz[a]); snap_node(s, nm, s->vel[a]);
      long long* t = (long long*)malloc(sizeof(long long) * s->nnode);
      for (long long n = 0; n < s->nnode; ++n) t[n] = s->act[n >> 6] ? s->valid[a][n] : -1;
      snprintf(nm, sizeof nm, "valid_%c", xyz[a]);
      snap_put_i(s, nm, t, s->nnode);
      free(t);
    }
  }
  constrain(s);
  if (snapshot) {
    static const char* xyz = "xyz";
    char nm[32];
    for (int a = 0; a < 3; ++a) {
      snprintf(nm, sizeof nm, "u_final_%c", xyz[a]);
      snap_node(s, nm, s->vel[a]);
    }
  }
  transfer_out(s, dt, snapshot, 1);
  return 0;
}

/* the transfers alone: grid, P2G, then G2P straight from the P2G node
 * velocities and advection (no solve), snapshots as in a step */
int wco_transfer(Scene* s, double dt) {
  transfer_in(s, 1);
  transfer_out(s, dt, 1, 0);
  return 0;
}

/* WetClothCore::stepSystem CFL sub-stepping (WetClothCore.cpp:50-62) */
int wco_num_substeps(Scene* s, double dt) {
  double mv = 0.0;
  for (int p = s->ne; p < s->np; ++p) {
    const double q = s->v[p * 3] * s->v[p * 3] + s->v[p * 3 + 1] * s->v[p * 3 + 1] +
                     s->v[p * 3 + 2] * s->v[p * 3 + 2];
    if (q > mv) mv = q;
  }
  mv = sqrt(mv);
  /* getMaxVelocity (TwoDScene.cpp:4171-4178): soft elasto particles */
  double ev = 0.0;
  for (int p = 0; p < s->ne; ++p) {
    if (s->surf[p]) continue;
    const double q = s->v[p * 3] * s->v[p * 3] + s->v[p * 3 + 1] * s->v[p * 3 + 1] +
                     s->v[p * 3 + 2] * s->v[p * 3 + 2];
    if (q > ev) ev = q;
  }
  ev = sqrt(ev);
  const double dx = s->p.dx;
  double me = dx / (ev > 1e-63 ? ev : 1e-63) / 3.0;
  if (me > 1.0 / 30.0) me = 1.0 / 30.0;
  double mf = dx / (mv > 1e-63 ? mv : 1e-63) * 3.0;
  if (mf > 1.0 / 30.0) mf = 1.0 / 30.0;
  const double md = me < mf ? me : mf;
  int n = (int)ceil(dt / md);
  return n > 1 ? n : 1;
}

int wco_step(Scene* s, double dt, int snapshot) {
  const int n = wco_num_substeps(s, dt);
  for (int k = 0; k < n; ++k) wco_substep(s, dt / (double)n, snapshot);
  return n;
}

/* liquid viscosity (LiquidInfo::viscosity with compute_viscosity on, explicit)
 * and LinearizedImplicitEuler's viscosity sub-steps; mu = 0 turns it off */
/* LiquidInfo elasto_flip_coeff, elasto_flip_asym_coeff, elasto_advect_coeff */
void wco_set_elasto_coeffs(Scene* s, double flip, double asym, double advect) {
  s->p.e_flip = flip;
  s->p.e_asym = asym;
  s->p.e_advect = advect;
}

void wco_set_viscosity(Scene* s, double mu, int substeps) {
  s->p.visc = mu;
  s->p.visc_substeps = substeps > 0 ? substeps : 1;
  s->p.drag_mu = mu > 0.0 ? mu : 8.9e-3;
}

/* LiquidInfo::implicit_viscosity and the stepper's viscous criterion */
void wco_set_viscosity_implicit(Scene* s, int implicit, double criterion) {
  s->p.visc_implicit = implicit;
  s->p.visc_criterion = criterion;
}

/* iterations, residual and unknowns of the last implicit viscosity solve */
void wco_viscosity_stats(Scene* s, int* iters, double* res, int* ndof) {
  *iters = s->visc_iters;
  *res = s->visc_res;
  *ndof = s->visc_ndof;
}

Scene* wco_create(double dx, const double* g, double rho, double flip, double friction,
                  const double* bc, const double* bh, double br, double criterion,
                  int maxiters, int mic, int np, const double* x3, const double* v3,
                  const double* C9, const double* mass, const double* vol, const double* radius) {
  Scene* s = (Scene*)calloc(1, sizeof(Scene));
  s->p.dx = dx;
  for (int a = 0; a < 3; ++a) {
    s->p.g[a] = g[a];
    s->p.bc[a] = bc[a];
    s->p.bh[a] = bh[a];
  }
  s->p.rho = rho;
  s->p.flip = flip;
  s->p.friction = friction;
  s->p.br = br;
  s->p.criterion = criterion;
  s->p.maxiters = maxiters;
  s->p.mic = mic;
  s->p.e_flip = 0.95;
  s->p.e_asym = 1.0;
  s->p.e_advect = 1.0;
  s->p.drag_mu = 8.9e-3;
  s->p.corr_step = 8;
  s->p.corr_mult = 2.0;
  s->p.visc_criterion = 1e-6;
  s->p.cell_mult = 0.3535533906;
  s->corr_sel_once = -1;
  s->bs = dx * 4.0;
  s->np = np;
  const size_t n = (size_t)(np > 0 ? np : 1);
  s->x = (double*)malloc(sizeof(double) * 3 * n);
  s->v = (double*)malloc(sizeof(double) * 3 * n);
  s->C = (double*)calloc(9 * n, sizeof(double));
  s->m = (double*)malloc(sizeof(double) * n);
  s->vol = (double*)malloc(sizeof(double) * n);
  s->rad = (double*)malloc(sizeof(double) * n);
  memcpy(s->x, x3, sizeof(double) * 3 * np);
  memcpy(s->v, v3, sizeof(double) * 3 * np);
  if (C9) memcpy(s->C, C9, sizeof(double) * 9 * np);
  memcpy(s->m, mass, sizeof(double) * np);
  memcpy(s->vol, vol, sizeof(double) * np);
  memcpy(s->rad, radius, sizeof(double) * np);
  s->ne = 0;
  s->em = (double*)calloc(3 * n, sizeof(double));
  s->rvol = (double*)calloc(n, sizeof(double));
  s->rvf = (double*)calloc(n, sizeof(double));
  s->sf = (double*)calloc(n, sizeof(double));
  s->ori = (double*)calloc(3 * n, sizeof(double));
  s->xt = (double*)calloc(n, sizeof(double));
  s->vt = (double*)calloc(n, sizeof(double));
  s->surf = (unsigned char*)calloc(n, 1);
  return s;
}

/* grow a per-particle array of k values to ne + np particles, the old
 * (liquid) values moving behind ne zeroed elasto slots */
static double* prepend(double* a, int k, int ne, int np) {
  double* b = (double*)calloc((size_t)k * (ne + np > 0 ? ne + np : 1), sizeof(double));
  memcpy(b + (size_t)k * ne, a, sizeof(double) * k * np);
  free(a);
  return b;
}

/* Elasto (cloth/yarn) particles become particles [0, ne) ahead of the liquid
 * ones (TwoDScene::getNumElastoParticles :5212-5217).  Per particle: x4/v4
 * (position/velocity with the twist as 4th component), B9 (row-major m_B),
 * m4/fm4 (m_m, m_fluid_m; P2G uses m(a) + m_fluid(a)), m_rest_vol,
 * m_rest_volume_fraction, m_fluid_vol, m_shape_factor, m_orientation (3),
 * surfel flag (m_particle_to_surfel >= 0), radius. */
void wco_set_elasto(Scene* s, int ne, const double* x4, const double* v4, const double* B9,
                    const double* m4, const double* fm4, const double* rest_vol,
                    const double* rest_vf, const double* fluid_vol, const double* shape_factor,
                    const double* orient3, const int* surfel, const double* radius) {
  const int nl = s->np;
  s->x = prepend(s->x, 3, ne, nl);
  s->v = prepend(s->v, 3, ne, nl);
  s->C = prepend(s->C, 9, ne, nl);
  s->m = prepend(s->m, 1, ne, nl);
  s->vol = prepend(s->vol, 1, ne, nl);
  s->rad = prepend(s->rad, 1, ne, nl);
  s->em = prepend(s->em, 3, ne, nl);
  s->rvol = prepend(s->rvol, 1, ne, nl);
  s->rvf = prepend(s->rvf, 1, ne, nl);
  s->sf = prepend(s->sf, 1, ne, nl);
  s->ori = prepend(s->ori, 3, ne, nl);
  s->xt = prepend(s->xt, 1, ne, nl);
  s->vt = prepend(s->vt, 1, ne, nl);
  unsigned char* su = (unsigned char*)calloc((size_t)(ne + nl > 0 ? ne + nl : 1), 1);
  free(s->surf);
  s->surf = su;
  for (int p = 0; p < ne; ++p) {
    for (int a = 0; a < 3; ++a) {
      s->x[p * 3 + a] = x4[p * 4 + a];
      s->v[p * 3 + a] = v4[p * 4 + a];
      s->em[p * 3 + a] = m4[p * 4 + a] + fm4[p * 4 + a];
      s->ori[p * 3 + a] = orient3[p * 3 + a];
    }
    for (int q = 0; q < 9; ++q) s->C[p * 9 + q] = B9[p * 9 + q];
    s->xt[p] = x4[p * 4 + 3];
    s->vt[p] = v4[p * 4 + 3];
    s->m[p] = 0.0;
    s->vol[p] = fluid_vol[p];
    s->rad[p] = radius[p];
    s->rvol[p] = rest_vol[p];
    s->rvf[p] = rest_vf[p];
    s->sf[p] = shape_factor[p];
    s->surf[p] = surfel[p] ? 1 : 0;
  }
  s->ne = ne;
  s->np = ne + nl;
}

void wco_destroy(Scene* s) {
  if (!s) return;
  for (int k = 0; k < s->nsnaps; ++k) {
    free(s->snaps[k].f);
    free(s->snaps[k].i);
  }
  void* ptrs[] = {s->x, s->v, s->C, s->m, s->vol, s->rad, s->em, s->rvol, s->rvf, s->sf,
                  s->ori, s->xt, s->vt, s->surf, s->keys, s->sup, s->act, s->base,
                  s->inside, s->wu, s->wv, s->ww, s->wp, s->pu.start, s->pu.pid, s->pu.slot,
                  s->pv.start, s->pv.pid, s->pv.slot, s->pw.start, s->pw.pid, s->pw.slot,
                  s->pp.start, s->pp.pid, s->pp.slot, s->sat_p, s->psi_p, s->pore_p, s->lphi,
                  s->sphi, s->pressure, s->dofidx, s->rowstart, s->col, s->val, s->b, s->xw,
                  s->vf_c, s->vf_e[0], s->vf_e[1], s->vf_e[2], s->vf_f[0], s->vf_f[1], s->vf_f[2],
                  s->cls};
  for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
  for (int a = 0; a < 3; ++a) {
    void* q[] = {s->mass[a], s->vel[a], s->vol_f[a], s->sat[a], s->psi[a], s->wgt[a], s->svel[a],
                 s->rhs[a], s->vstar[a], s->invC[a], s->psifs[a], s->psisf[a], s->mshdvm[a],
                 s->mfhdvm[a], s->valid[a], s->emass[a], s->evel[a], s->evol[a], s->esf[a],
                 s->eori[a]};
    for (size_t k = 0; k < sizeof(q) / sizeof(q[0]); ++k) free(q[k]);
  }
  free(s);
}

long long wco_size(Scene* s, const char* name) {
  for (int k = 0; k < s->nsnaps; ++k)
    if (!strcmp(s->snaps[k].name, name)) return s->snaps[k].n;
  return -1;
}

/* the particle state (positions, velocities, affine matrices) under
 * tag + "x" / "v" / "C", without the per-stage snapshots of a step */
void wco_snap_state(Scene* s, const char* tag) { snap_particles(s, tag); }

int wco_get_f(Scene* s, const char* name, double* out) {
  for (int k = 0; k < s->nsnaps; ++k)
    if (!strcmp(s->snaps[k].name, name) && !s->snaps[k].is_int) {
      memcpy(out, s->snaps[k].f, sizeof(double) * s->snaps[k].n);
      return 0;
    }
  return -1;
}

int wco_get_i(Scene* s, const char* name, long long* out) {
  for (int k = 0; k < s->nsnaps; ++k)
    if (!strcmp(s->snaps[k].name, name) && s->snaps[k].is_int) {
      memcpy(out, s->snaps[k].i, sizeof(long long) * s->snaps[k].n);
      return 0;
    }
  return -1;
}

void wco_solver_stats(Scene* s, int* iters, double* res) {
  *iters = s->last_iters;
  *res = s->last_res;
}

int wco_num_particles(Scene* s) { return s->np; }
