// extern "C" surface of libwcgpu (declared in include/wetcloth_gpu.h).
#include <cuda_runtime.h>
#include <fstream>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/wetcloth_gpu.h"
#include "wcg_context.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_status(wcg::Context& c, cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    c.last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(WCG_ERR_CUDA, c.last_error);
  }
  return WCG_OK;
}

// check the device error word after a stage
int device_status(wcg::Context& c, const char* what) {
  int h = 0;
  const cudaError_t e = wcg::read_small(c, c.derr.p, sizeof(int), &h);
  if (e != cudaSuccess) return cuda_status(c, e, what);
  if (h != 0) {
    cudaMemsetAsync(c.derr.p, 0, sizeof(int), c.stream);
    cudaStreamSynchronize(c.stream);
    return fail(WCG_ERR_DEVICE, std::string(what) + ": device error code " +
                                    std::to_string(h) +
                                    (h == wcg::kErrWaitTimeout
                                         ? " (wavefront wait limit reached)"
                                         : h == wcg::kErrInput
                                               ? " (invalid particle input: non-finite position "
                                                 "or velocity, or negative mass/volume/radius)"
                                               : " (index out of range, access skipped)"));
  }
  return WCG_OK;
}

#define WCG_CHECK_CTX(ctx)                                        \
  do {                                                            \
    if (!(ctx)) return fail(WCG_ERR_ARG, "null context");         \
  } while (0)

#define WCG_CALL(ctx, expr, what)                                 \
  do {                                                            \
    int s_ = cuda_status((ctx)->c, (expr), (what));               \
    if (s_) return s_;                                            \
  } while (0)

struct FieldName {
  const char* name;
  int field;      // wcg::GField, kEBase + wcg::EField, or -1 for an all-zero field
  int ncomp = 1;  // values per node
};

// elasto node fields are numbered after the GField ones
constexpr int kEBase = 1000;

// P2G/step outputs that are identically zero for liquid-only scenes (no
// elasto particles, static walls): solid volume fraction psi, solid velocity,
// pore pressure.
const FieldName kFields[] = {
    {"mass_fluid_x", wcg::G_MASS}, {"mass_fluid_y", wcg::G_MASS + 1},
    {"mass_fluid_z", wcg::G_MASS + 2}, {"vel_fluid_x", wcg::G_VEL},
    {"vel_fluid_y", wcg::G_VEL + 1}, {"vel_fluid_z", wcg::G_VEL + 2},
    {"vol_fluid_x", wcg::G_VOL}, {"vol_fluid_y", wcg::G_VOL + 1},
    {"vol_fluid_z", wcg::G_VOL + 2}, {"sat_x", wcg::G_SAT},
    {"sat_y", wcg::G_SAT + 1}, {"sat_z", wcg::G_SAT + 2},
    {"psi_x", kEBase + wcg::E_PSI}, {"psi_y", kEBase + wcg::E_PSI + 1},
    {"psi_z", kEBase + wcg::E_PSI + 2},
    {"mass_x", kEBase + wcg::E_MASS}, {"mass_y", kEBase + wcg::E_MASS + 1},
    {"mass_z", kEBase + wcg::E_MASS + 2}, {"vel_x", kEBase + wcg::E_VEL},
    {"vel_y", kEBase + wcg::E_VEL + 1}, {"vel_z", kEBase + wcg::E_VEL + 2},
    {"vol_x", kEBase + wcg::E_VOL}, {"vol_y", kEBase + wcg::E_VOL + 1},
    {"vol_z", kEBase + wcg::E_VOL + 2}, {"shape_factor_x", kEBase + wcg::E_SF},
    {"shape_factor_y", kEBase + wcg::E_SF + 1}, {"shape_factor_z", kEBase + wcg::E_SF + 2},
    {"orientation_x", kEBase + wcg::E_ORI, 3}, {"orientation_y", kEBase + wcg::E_ORI + 3, 3},
    {"orientation_z", kEBase + wcg::E_ORI + 6, 3},
    {"solid_weight_x", wcg::G_WEIGHT}, {"solid_weight_y", wcg::G_WEIGHT + 1},
    {"solid_weight_z", wcg::G_WEIGHT + 2}, {"solid_vel_x", -1},
    {"solid_vel_y", -1}, {"solid_vel_z", -1},
    {"v_star_x", wcg::G_VSTAR}, {"v_star_y", wcg::G_VSTAR + 1},
    {"v_star_z", wcg::G_VSTAR + 2}, {"rhs_fluid_x", wcg::G_RHS},
    {"rhs_fluid_y", wcg::G_RHS + 1}, {"rhs_fluid_z", wcg::G_RHS + 2},
    {"inv_C_x", wcg::G_INVC}, {"inv_C_y", wcg::G_INVC + 1},
    {"inv_C_z", wcg::G_INVC + 2}, {"psi_fs_x", wcg::G_PSIFS},
    {"psi_fs_y", wcg::G_PSIFS + 1}, {"psi_fs_z", wcg::G_PSIFS + 2},
    {"u_x", wcg::G_U}, {"u_y", wcg::G_U + 1}, {"u_z", wcg::G_U + 2},
    {"liquid_phi", wcg::G_LPHI}, {"sat_p", wcg::G_SATP}, {"psi_p", kEBase + wcg::E_PSIP},
    {"pore_pressure_p", kEBase + wcg::E_PORE}, {"solid_phi", wcg::G_SPHI},
    {"pressure", wcg::G_PRESSURE}, {"A_diag", wcg::G_ADIAG},
    {"A_x", wcg::G_AX}, {"A_y", wcg::G_AY}, {"A_z", wcg::G_AZ},
    {"b_dense", wcg::G_B}, {"mic_invdiag", wcg::G_INVDIAG},
    {"liquid_c_vf", wcg::G_VFC}, {"liquid_ex_vf", wcg::G_VFEX},
    {"liquid_ey_vf", wcg::G_VFEY}, {"liquid_ez_vf", wcg::G_VFEZ},
    {"liquid_u_vf", wcg::G_VFU}, {"liquid_v_vf", wcg::G_VFV}, {"liquid_w_vf", wcg::G_VFW},
};

int lookup_field(const char* name, int* ncomp = nullptr) {
  for (const FieldName& f : kFields)
    if (!strcmp(f.name, name)) {
      if (ncomp) *ncomp = f.ncomp;
      return f.field;
    }
  return -2;
}

std::vector<unsigned char> host_active(wcg::Context& c) {
  std::vector<unsigned char> a((size_t)c.g.nb);
  if (c.g.nb)
    cudaMemcpy(a.data(), c.active.p, (size_t)c.g.nb, cudaMemcpyDeviceToHost);
  return a;
}

// raw field (converted to double) over all nodes; elasto fields are zero
// while the scene has no elasto particles
std::vector<double> host_field(wcg::Context& c, int field) {
  const long long nn = c.g.nnode;
  std::vector<double> out((size_t)nn, 0.0);
  if (field < 0 || nn == 0) return out;
  const bool ef = field >= kEBase;
  if (ef && (c.ne == 0 || c.efcap < c.gcap)) return out;
  const wcg::DevBuf& buf = ef ? c.efield : c.gfield;
  const size_t off = (size_t)(ef ? field - kEBase : field) * c.gcap;
  if (c.prm.precision == 0) {
    cudaMemcpy(out.data(), buf.as<double>() + off, nn * sizeof(double), cudaMemcpyDeviceToHost);
  } else {
    std::vector<float> f((size_t)nn);
    cudaMemcpy(f.data(), buf.as<float>() + off, nn * sizeof(float), cudaMemcpyDeviceToHost);
    for (long long i = 0; i < nn; ++i) out[i] = f[i];
  }
  return out;
}

std::vector<unsigned char> host_bytes(const void* dev, long long n) {
  std::vector<unsigned char> v((size_t)n);
  if (n) cudaMemcpy(v.data(), dev, (size_t)n, cudaMemcpyDeviceToHost);
  return v;
}

}  // namespace

int wcg::set_last_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

extern "C" {

const char* wcg_last_error(void) { return g_err.c_str(); }

void wcg_default_params(wcg_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->dx = 1.0 / 64.0;
  p->gravity[1] = -9.81;
  p->liquid_density = 1000.0;
  p->flip_coeff = 0.99;
  p->liquid_boundary_friction = 0.0;
  for (int a = 0; a < 3; ++a) {
    p->box_center[a] = 0.5;
    p->box_half[a] = 0.5;
  }
  p->box_radius = 0.0;
  p->walls = 1;
  p->criterion = 1e-6;
  p->maxiters = 1000;
  p->precision = WCG_FP64;
  // the first FP32 inner solve stops at 1e-5 and the FP64 refinement takes it
  // the rest of the way: at 256^3 about 5 % fewer PCG iterations than aiming
  // every inner solve at the criterion
  p->refine_inner_tol = 1e-5;
  p->max_refinements = 20;
  p->solver = WCG_SOLVER_MIC0;
  p->viscosity = 0.0;
  p->viscosity_substeps = 1;
  p->elasto_flip_coeff = 0.95;
  p->elasto_flip_asym_coeff = 1.0;
  p->elasto_advect_coeff = 1.0;
  p->drag_viscosity = 8.9e-3;
  p->correction_strength = 0.0;
  p->correction_step = 8;
  p->correction_multiplier = 2.0;
  p->correction_seed = 0;
  p->viscosity_implicit = 0;
  p->viscosity_criterion = 1e-6;
  p->particle_merge = 0;
  p->merge_seed = 0;
  p->particle_split = 0;
  p->split_seed = 0;
  p->terminator = 0;
  for (int a = 0; a < 3; ++a) {
    p->terminator_center[a] = 0.5;
    p->terminator_half[a] = 0.5;
  }
  p->terminator_radius = 0.0;
  p->terminator_inside = 1;
  p->particle_cell_multiplier = 0.3535533906;
}

int wcg_create(const wcg_params* params, wcg_ctx** out) {
  if (!params || !out) return fail(WCG_ERR_ARG, "null argument");
  if (!(params->dx > 0)) return fail(WCG_ERR_ARG, "dx must be positive");
  if (params->precision != WCG_FP64 && params->precision != WCG_FP32_REFINE)
    return fail(WCG_ERR_ARG, "precision must be WCG_FP64 or WCG_FP32_REFINE");
  if (params->maxiters < 0) return fail(WCG_ERR_ARG, "maxiters must be >= 0");
  if (params->solver != WCG_SOLVER_MIC0 && params->solver != WCG_SOLVER_MG)
    return fail(WCG_ERR_ARG, "solver must be WCG_SOLVER_MIC0 or WCG_SOLVER_MG");
  if (!(params->viscosity >= 0.0) || !std::isfinite(params->viscosity))
    return fail(WCG_ERR_ARG, "viscosity must be finite and >= 0");
  if (!std::isfinite(params->elasto_flip_coeff) || !std::isfinite(params->elasto_flip_asym_coeff) ||
      !std::isfinite(params->elasto_advect_coeff))
    return fail(WCG_ERR_ARG, "elasto coefficients must be finite");
  if (!(params->drag_viscosity > 0.0) || !std::isfinite(params->drag_viscosity))
    return fail(WCG_ERR_ARG, "drag_viscosity must be finite and > 0");
  if (!(params->particle_cell_multiplier > 0.0) || !std::isfinite(params->particle_cell_multiplier))
    return fail(WCG_ERR_ARG, "particle_cell_multiplier must be finite and > 0");
  if (!(params->viscosity_criterion > 0.0) || !std::isfinite(params->viscosity_criterion))
    return fail(WCG_ERR_ARG, "viscosity_criterion must be finite and > 0");
  if (!(params->correction_strength >= 0.0) || !std::isfinite(params->correction_strength) ||
      !std::isfinite(params->correction_multiplier) || params->correction_step < 1)
    return fail(WCG_ERR_ARG,
                "correction_strength must be finite and >= 0, correction_step >= 1, "
                "correction_multiplier finite");
  if (params->terminator) {
    bool ok = std::isfinite(params->terminator_radius) && params->terminator_radius >= 0.0;
    for (int a = 0; a < 3; ++a)
      ok = ok && std::isfinite(params->terminator_center[a]) &&
           std::isfinite(params->terminator_half[a]) && params->terminator_half[a] >= 0.0;
    if (!ok)
      return fail(WCG_ERR_ARG,
                  "terminator centre, half extents (>= 0) and radius (>= 0) must be finite");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(WCG_ERR_CUDA, "no CUDA device available");
  wcg_ctx* ctx = new wcg_ctx();
  wcg::Params& p = ctx->c.prm;
  p.dx = params->dx;
  for (int a = 0; a < 3; ++a) {
    p.gravity[a] = params->gravity[a];
    p.box_center[a] = params->box_center[a];
    p.box_half[a] = params->box_half[a];
  }
  p.liquid_density = params->liquid_density;
  p.flip_coeff = params->flip_coeff;
  p.liquid_boundary_friction = params->liquid_boundary_friction;
  p.box_radius = params->box_radius;
  p.walls = params->walls;
  p.criterion = params->criterion;
  p.maxiters = params->maxiters;
  p.precision = params->precision;
  p.refine_inner_tol = params->refine_inner_tol > 0 ? params->refine_inner_tol : 0.0;
  p.max_refinements = params->max_refinements > 0 ? params->max_refinements : 20;
  p.solver = params->solver;
  p.viscosity = params->viscosity;
  p.viscosity_substeps = params->viscosity_substeps > 0 ? params->viscosity_substeps : 1;
  p.elasto_flip = params->elasto_flip_coeff;
  p.elasto_flip_asym = params->elasto_flip_asym_coeff;
  p.elasto_advect = params->elasto_advect_coeff;
  p.drag_viscosity = params->drag_viscosity;
  p.correction_strength = params->correction_strength;
  p.correction_step = params->correction_step;
  p.correction_multiplier = params->correction_multiplier;
  p.correction_seed = params->correction_seed;
  p.viscosity_implicit = params->viscosity_implicit ? 1 : 0;
  p.particle_merge = params->particle_merge ? 1 : 0;
  p.merge_seed = params->merge_seed;
  p.particle_split = params->particle_split ? 1 : 0;
  p.split_seed = params->split_seed;
  p.terminator = params->terminator ? 1 : 0;
  for (int a = 0; a < 3; ++a) {
    p.term_center[a] = params->terminator_center[a];
    p.term_half[a] = params->terminator_half[a];
  }
  p.term_radius = params->terminator_radius;
  p.term_inside = params->terminator_inside ? 1 : 0;
  p.cell_multiplier = params->particle_cell_multiplier;
  p.viscosity_criterion = params->viscosity_criterion;
  // wavefront tile shape (performance knob; both compute identical results)
  if (const char* v = getenv("WCG_SWEEP_TILE")) ctx->c.sweep_variant = !strcmp(v, "warp") ? 1 : 0;
  // layout of the pressure solve (performance knob; same arithmetic)
  if (const char* v = getenv("WCG_PCG_LAYOUT")) ctx->c.pcg_layout = !strcmp(v, "tiles") ? 1 : 0;
  // transfer formulation: bucket tiles (default) or the global gathers
  if (const char* v = getenv("WCG_TRANSFERS")) ctx->c.xfer_mode = !strcmp(v, "gather") ? 1 : 0;
  // the PCG's SpMV: row-parallel (default) or patch-streamed (performance
  // knob; the dot products' partial sums are grouped differently)
  if (const char* v = getenv("WCG_SPMV")) ctx->c.spmv_rows = !strcmp(v, "stream") ? 0 : 1;
  // CTAs per thread-block cluster along c in the MIC(0) sweeps (1, 2, 3, 4,
  // 8, 9 or 16; performance knob, identical results).  Default 0: chosen per
  // solve from the patches along c (pl_setup).
  ctx->c.sweep_cluster = 0;
  if (const char* v = getenv("WCG_SWEEP_CLUSTER")) {
    const int k = atoi(v);
    ctx->c.sweep_cluster = (k == 2 || k == 3 || k == 4 || k == 8 || k == 9 || k == 16) ? k : 1;
  }
  // and along a: 2-D clusters of CC x CA CTAs (CA 4 or 8 with CC 1, 2 or 4;
  // CA 8 with CC 1 or 2), a-face neighbours through shared memory as well
  if (const char* v = getenv("WCG_SWEEP_CLUSTER_A")) {
    const int k = atoi(v), cc = ctx->c.sweep_cluster;
    const bool ok = (k == 4 && cc <= 4) || (k == 8 && cc <= 2);
    ctx->c.sweep_cluster_a = ok ? k : 1;
  }
  // the params' terminator box as the one terminator shape (identity rotation)
  if (p.terminator) {
    wcg::TermShape& t = ctx->c.term.s[0];
    t.type = 0;
    t.sign = p.term_inside ? -1.0 : 1.0;
    for (int a = 0; a < 3; ++a) {
      t.c[a] = p.term_center[a];
      t.par[a] = p.term_half[a];
    }
    t.par[3] = p.term_radius;
    t.q[0] = 1.0;
    t.q[1] = t.q[2] = t.q[3] = 0.0;
    ctx->c.term.n = 1;
  }
  cudaError_t e = wcg::ctx_init(ctx->c);
  if (e != cudaSuccess) {
    std::string m = std::string("context init: ") + cudaGetErrorString(e);
    wcg::ctx_free(ctx->c);
    delete ctx;
    return fail(WCG_ERR_CUDA, m);
  }
  *out = ctx;
  return WCG_OK;
}

int wcg_destroy(wcg_ctx* ctx) {
  if (!ctx) return WCG_OK;
  cudaStreamSynchronize(ctx->c.stream);
  wcg::ctx_free(ctx->c);
  delete ctx;
  return WCG_OK;
}

static int upload(wcg_ctx* ctx, long long n, const double* x3, const double* v3,
                  const double* C9, const double* mass, const double* vol,
                  const double* radius, bool dev) {
  WCG_CHECK_CTX(ctx);
  if (n < 0 || n > 2000000000ll) return fail(WCG_ERR_ARG, "particle count out of range");
  if (n > 0 && (!x3 || !v3 || !mass || !vol || !radius))
    return fail(WCG_ERR_ARG, "null particle array");
  if (!dev && n > 0) {
    for (long long i = 0; i < 3 * n; ++i)
      if (!std::isfinite(x3[i]) || !std::isfinite(v3[i]))
        return fail(WCG_ERR_ARG, "non-finite particle position or velocity");
    for (long long i = 0; i < n; ++i)
      if (!(mass[i] >= 0) || !(vol[i] >= 0) || !(radius[i] >= 0))
        return fail(WCG_ERR_ARG, "negative or NaN particle mass/volume/radius");
  }
  WCG_CALL(ctx, wcg::upload_particles(ctx->c, n, x3, v3, C9, mass, vol, radius, dev),
           "upload");
  ctx->c.have_grid = false;
  return WCG_OK;
}

int wcg_upload_liquid(wcg_ctx* ctx, long long n, const double* x3, const double* v3,
                      const double* C9, const double* mass, const double* vol,
                      const double* radius) {
  return upload(ctx, n, x3, v3, C9, mass, vol, radius, false);
}

int wcg_upload_liquid_device(wcg_ctx* ctx, long long n, const double* x3,
                             const double* v3, const double* C9, const double* mass,
                             const double* vol, const double* radius) {
  return upload(ctx, n, x3, v3, C9, mass, vol, radius, true);
}

int wcg_download_liquid(wcg_ctx* ctx, double* x3, double* v3, double* C9) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::download_particles(ctx->c, x3, v3, C9, false), "download");
  return WCG_OK;
}

int wcg_download_liquid_async(wcg_ctx* ctx, double* x3, double* v3, double* C9) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::download_particles_async(ctx->c, x3, v3, C9), "download (asynchronous)");
  return WCG_OK;
}

int wcg_stage_liquid_async(wcg_ctx* ctx, long long n, const double* x3, const double* v3,
                           const double* C9, const double* mass, const double* vol,
                           const double* radius) {
  WCG_CHECK_CTX(ctx);
  if (n < 0) return fail(WCG_ERR_ARG, "negative particle count");
  if (n > 0 && (!x3 || !v3 || !mass || !vol || !radius))
    return fail(WCG_ERR_ARG, "null particle array");
  if (n > INT_MAX) return fail(WCG_ERR_ARG, "more than 2^31 - 1 particles");
  WCG_CALL(ctx, wcg::stage_particles_async(ctx->c, n, x3, v3, C9, mass, vol, radius),
           "stage (asynchronous)");
  return WCG_OK;
}

int wcg_upload_staged(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  if (ctx->c.staged_n < 0) return fail(WCG_ERR_STATE, "no staged particle set");
  WCG_CALL(ctx, wcg::load_staged(ctx->c), "upload staged");
  ctx->c.have_grid = false;
  return WCG_OK;
}

int wcg_synchronize(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::synchronize(ctx->c), "synchronize");
  return WCG_OK;
}

int wcg_download_liquid_device(wcg_ctx* ctx, double* x3, double* v3, double* C9) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::download_particles(ctx->c, x3, v3, C9, true), "download");
  return WCG_OK;
}

long long wcg_num_particles(const wcg_ctx* ctx) { return ctx ? ctx->c.np : -1; }

int wcg_upload_elasto(wcg_ctx* ctx, long long n, const double* x4, const double* v4,
                      const double* B9, const double* m4, const double* fm4,
                      const double* rest_vol, const double* rest_vf, const double* fluid_vol,
                      const double* shape_factor, const double* orient3, const int* surfel) {
  WCG_CHECK_CTX(ctx);
  if (n < 0 || n > 2000000000ll) return fail(WCG_ERR_ARG, "particle count out of range");
  if (n > 0 && (!x4 || !v4 || !B9 || !m4 || !fm4 || !rest_vol || !rest_vf || !fluid_vol ||
                !shape_factor || !orient3 || !surfel))
    return fail(WCG_ERR_ARG, "null elasto particle array");
  for (long long i = 0; i < 4 * n; ++i)
    if (!std::isfinite(x4[i]) || !std::isfinite(v4[i]) || !std::isfinite(m4[i]) ||
        !std::isfinite(fm4[i]))
      return fail(WCG_ERR_ARG, "non-finite elasto position, velocity or mass");
  for (long long i = 0; i < 9 * n; ++i)
    if (!std::isfinite(B9[i])) return fail(WCG_ERR_ARG, "non-finite elasto affine matrix");
  for (long long i = 0; i < n; ++i) {
    if (!(rest_vol[i] >= 0) || !(fluid_vol[i] >= 0) || !(rest_vf[i] >= 0) ||
        !std::isfinite(rest_vol[i]) || !std::isfinite(fluid_vol[i]) ||
        !std::isfinite(rest_vf[i]) || !std::isfinite(shape_factor[i]))
      return fail(WCG_ERR_ARG, "negative or non-finite elasto volume attribute");
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(orient3[i * 3 + a]))
        return fail(WCG_ERR_ARG, "non-finite elasto orientation");
  }
  WCG_CALL(ctx, wcg::upload_elasto(ctx->c, n, x4, v4, B9, m4, fm4, rest_vol, rest_vf, fluid_vol,
                                   shape_factor, orient3, surfel),
           "upload elasto");
  return WCG_OK;
}

int wcg_download_elasto(wcg_ctx* ctx, double* x4, double* v4, double* B9) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::download_elasto(ctx->c, x4, v4, B9), "download elasto");
  return WCG_OK;
}

long long wcg_num_elasto(const wcg_ctx* ctx) { return ctx ? ctx->c.ne : -1; }

// ---- state I/O in the reference's file formats ------------------------------
// TwoDSceneSerializer::serializePositionOnly / serialize_pos_subprog
// (App/TwoDSceneSerializer.cpp:20-32, :161-170): an int byte count and m_x
// (x, y, z, twist per particle, doubles), then an int byte count and the
// Gauss-point matrix of the cloth (empty here).
int wcg_save_positions(wcg_ctx* ctx, const char* path) {
  WCG_CHECK_CTX(ctx);
  if (!path) return fail(WCG_ERR_ARG, "null path");
  // elasto particles first, as the reference numbers them
  const long long ne = ctx->c.ne, n = ne + ctx->c.np;
  if (n * 4 * (long long)sizeof(double) > 2147483647ll)
    return fail(WCG_ERR_ARG, "too many particles for the position file's int byte count");
  std::vector<double> x4((size_t)n * 4);
  if (ne > 0) WCG_CALL(ctx, wcg::download_elasto(ctx->c, x4.data(), nullptr, nullptr),
                       "save positions");
  if (ctx->c.np > 0)
    WCG_CALL(ctx, wcg::download_positions(ctx->c, x4.data() + 4 * ne, nullptr), "save positions");
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(WCG_ERR_ARG, std::string("cannot open ") + path);
  const int bytes = (int)(n * 4 * sizeof(double));
  const int gauss_bytes = 0;
  f.write((const char*)&bytes, sizeof(int));
  f.write((const char*)x4.data(), bytes);
  f.write((const char*)&gauss_bytes, sizeof(int));
  if (!f) return fail(WCG_ERR_ARG, std::string("write failed: ") + path);
  return WCG_OK;
}

// TwoDSceneSerializer::loadPosOnly (App/TwoDSceneSerializer.cpp:172-182): the
// particle count of the file must equal the context's.
int wcg_load_positions(wcg_ctx* ctx, const char* path) {
  WCG_CHECK_CTX(ctx);
  if (!path) return fail(WCG_ERR_ARG, "null path");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(WCG_ERR_ARG, std::string("cannot open ") + path);
  int bytes = -1;
  f.read((char*)&bytes, sizeof(int));
  const long long ne = ctx->c.ne, n = ne + ctx->c.np;
  if (!f || bytes != n * 4 * (long long)sizeof(double))
    return fail(WCG_ERR_ARG, "position file holds " + std::to_string(bytes) +
                                 " bytes, the scene needs " +
                                 std::to_string(n * 4 * (long long)sizeof(double)));
  std::vector<double> x4((size_t)n * 4);
  f.read((char*)x4.data(), bytes);
  int gauss_bytes = 0;
  f.read((char*)&gauss_bytes, sizeof(int));
  if (!f) return fail(WCG_ERR_ARG, std::string("truncated position file: ") + path);
  for (double v : x4)
    if (!std::isfinite(v)) return fail(WCG_ERR_ARG, "non-finite position in file");
  if (ne > 0)
    WCG_CALL(ctx, wcg::upload_elasto_positions(ctx->c, x4.data()), "load positions");
  if (ctx->c.np > 0)
    WCG_CALL(ctx, wcg::upload_positions(ctx->c, x4.data() + 4 * ne), "load positions");
  return WCG_OK;
}

// The fluid OBJ of serialize_subprog (App/TwoDSceneSerializer.cpp:40-47;
// updateFluid :242-255): "v x y z r" per fluid particle, 8 significant digits.
int wcg_write_fluid_obj(wcg_ctx* ctx, const char* path) {
  WCG_CHECK_CTX(ctx);
  if (!path) return fail(WCG_ERR_ARG, "null path");
  const long long n = ctx->c.np;
  std::vector<double> x4((size_t)n * 4), r((size_t)n);
  if (n > 0) WCG_CALL(ctx, wcg::download_positions(ctx->c, x4.data(), r.data()), "fluid obj");
  FILE* f = fopen(path, "w");
  if (!f) return fail(WCG_ERR_ARG, std::string("cannot open ") + path);
  for (long long i = 0; i < n; ++i)
    fprintf(f, "v %.8g %.8g %.8g %.8g\n", x4[i * 4], x4[i * 4 + 1], x4[i * 4 + 2], r[i]);
  const bool ok = fclose(f) == 0;
  if (!ok) return fail(WCG_ERR_ARG, std::string("write failed: ") + path);
  return WCG_OK;
}

int wcg_rebucketize_and_resample(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::build_grid(ctx->c), "rebucketize/resample");
  return device_status(ctx->c, "rebucketize/resample");
}

#define WCG_NEED_GRID(ctx)                                                     \
  do {                                                                         \
    if (!(ctx)->c.have_grid)                                                   \
      return fail(WCG_ERR_STATE, "no grid: call wcg_rebucketize_and_resample"); \
  } while (0)

// Calls without an elasto form refuse scenes with elasto particles.
#define WCG_NO_ELASTO(ctx, what)                                              \
  do {                                                                       \
    if ((ctx)->c.ne > 0)                                                     \
      return fail(WCG_ERR_UNSUPPORTED, std::string(what) +                   \
                                           ": not available with elasto particles"); \
  } while (0)

int wcg_map_particle_nodes(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  WCG_CALL(ctx, wcg::map_particles_to_grid(ctx->c), "mapParticleNodesAPIC");
  return device_status(ctx->c, "mapParticleNodesAPIC");
}

int wcg_step_velocity(wcg_ctx* ctx, double dt) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  WCG_CALL(ctx, wcg::step_velocity(ctx->c, dt), "stepVelocity");
  int s = device_status(ctx->c, "stepVelocity");
  if (s) return s;
  if (!ctx->c.stats.visc_converged)
    return fail(WCG_ERR_NOT_CONVERGED, "implicit viscosity PCG did not converge (residual " +
                                           std::to_string(ctx->c.stats.visc_residual) + ")");
  return WCG_OK;
}

int wcg_project_fine(wcg_ctx* ctx, double dt) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  WCG_CALL(ctx, wcg::project_fine(ctx->c, dt), "projectFine");
  int s = device_status(ctx->c, "projectFine");
  if (s) return s;
  if (!ctx->c.stats.converged)
    return fail(WCG_ERR_NOT_CONVERGED,
                "pressure PCG did not converge (residual " +
                    std::to_string(ctx->c.stats.residual) + ", iterations " +
                    std::to_string(ctx->c.stats.pcg_iters) + ")");
  return WCG_OK;
}

int wcg_apply_pressure_drag_fluid(wcg_ctx* ctx, double dt) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  WCG_CALL(ctx, wcg::apply_pressure_and_extrapolate(ctx->c, dt), "applyPressureDragFluid");
  return device_status(ctx->c, "applyPressureDragFluid");
}

int wcg_constrain_liquid_velocity(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  WCG_CALL(ctx, wcg::constrain_liquid_velocity(ctx->c), "constrainLiquidVelocity");
  return device_status(ctx->c, "constrainLiquidVelocity");
}

int wcg_map_node_particles(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  WCG_CALL(ctx, wcg::map_grid_to_particles_and_advect(ctx->c, 0.0, false),
           "mapNodeParticlesAPIC");
  return device_status(ctx->c, "mapNodeParticlesAPIC");
}

int wcg_correct_liquid_particles(wcg_ctx* ctx, double dt, int selector) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  const int step = ctx->c.prm.correction_step > 0 ? ctx->c.prm.correction_step : 1;
  if (selector < -1 || selector >= step)
    return fail(WCG_ERR_ARG, "selector must be -1 or lie in [0, correction_step)");
  // -1: the next subset of the context's seeded stream, as wcg_substep draws it
  if (selector < 0)
    selector = wcg::correction_selector(ctx->c.prm.correction_seed, ctx->c.corr_count++, step);
  WCG_CALL(ctx, wcg::correct_liquid_particles(ctx->c, dt, selector), "correctLiquidParticles");
  return device_status(ctx->c, "correctLiquidParticles");
}

static bool valid_perm3(const int* p) {
  return p[0] >= 0 && p[0] < 3 && p[1] >= 0 && p[1] < 3 && p[2] >= 0 && p[2] < 3 &&
         p[0] != p[1] && p[0] != p[2] && p[1] != p[2];
}

int wcg_merge_liquid_particles(wcg_ctx* ctx, int selector, const int* perm9,
                               long long* removed) {
  WCG_CHECK_CTX(ctx);
  if (!perm9) return fail(WCG_ERR_ARG, "null colour permutation");
  if (selector < 0 || selector >= ctx->c.prm.correction_step)
    return fail(WCG_ERR_ARG, "selector must lie in [0, correction_step)");
  for (int q = 0; q < 3; ++q)
    if (!valid_perm3(perm9 + 3 * q))
      return fail(WCG_ERR_ARG, "perm9 must hold three permutations of {0, 1, 2}");
  if (ctx->c.g.nb == 0) return fail(WCG_ERR_STATE, "no grid build to take the buckets from");
  long long rem = 0;
  WCG_CALL(ctx, wcg::merge_liquid_particles(ctx->c, selector, perm9, &rem),
           "mergeLiquidParticles");
  if (removed) *removed = rem;
  return device_status(ctx->c, "mergeLiquidParticles");
}

int wcg_split_liquid_particles(wcg_ctx* ctx, unsigned long long key, long long* added) {
  WCG_CHECK_CTX(ctx);
  long long add = 0;
  WCG_CALL(ctx, wcg::split_liquid_particles(ctx->c, key, &add), "splitLiquidParticles");
  if (added) *added = add;
  return device_status(ctx->c, "splitLiquidParticles");
}

int wcg_split_parents(wcg_ctx* ctx, long long* nparents) {
  WCG_CHECK_CTX(ctx);
  if (!nparents) return fail(WCG_ERR_ARG, "nparents must not be NULL");
  long long k = 0;
  WCG_CALL(ctx, wcg::split_liquid_parents(ctx->c, &k), "splitLiquidParticles");
  *nparents = k;
  return device_status(ctx->c, "splitLiquidParticles");
}

int wcg_split_liquid_particles_with(wcg_ctx* ctx, const double* pattern, const double* rot9,
                                    long long nparents, long long* added) {
  WCG_CHECK_CTX(ctx);
  if (!pattern || nparents < 0 || (nparents > 0 && !rot9))
    return fail(WCG_ERR_ARG, "a pattern table and nparents rotations are required");
  long long have = 0;
  WCG_CALL(ctx, wcg::split_liquid_parents(ctx->c, &have), "splitLiquidParticles");
  if (have != nparents)
    return fail(WCG_ERR_ARG, "nparents differs from the particles that split (" +
                                 std::to_string(have) + ")");
  long long add = 0;
  WCG_CALL(ctx, wcg::split_liquid_particles_with(ctx->c, pattern, rot9, nparents, &add),
           "splitLiquidParticles");
  if (added) *added = add;
  return device_status(ctx->c, "splitLiquidParticles");
}

int wcg_terminate_liquid_particles(wcg_ctx* ctx, long long* removed) {
  WCG_CHECK_CTX(ctx);
  long long rem = 0;
  WCG_CALL(ctx, wcg::terminate_liquid_particles(ctx->c, &rem), "terminateParticles");
  if (removed) *removed = rem;
  return device_status(ctx->c, "terminateParticles");
}

int wcg_set_terminators(wcg_ctx* ctx, int n, const wcg_shape* shapes) {
  WCG_CHECK_CTX(ctx);
  if (n < 0 || n > WCG_MAX_TERMINATOR_SHAPES || (n > 0 && !shapes))
    return fail(WCG_ERR_ARG, "between 0 and 16 terminator shapes");
  wcg::TermSet t{};
  for (int k = 0; k < n; ++k) {
    const wcg_shape& h = shapes[k];
    if (h.type < WCG_SHAPE_BOX || h.type > WCG_SHAPE_CYLINDER)
      return fail(WCG_ERR_ARG, "unknown terminator shape type");
    bool finite = true;
    for (int a = 0; a < 3; ++a) finite = finite && std::isfinite(h.center[a]);
    for (int a = 0; a < 4; ++a) finite = finite && std::isfinite(h.rot[a]) && std::isfinite(h.param[a]);
    const double q2 = h.rot[0] * h.rot[0] + h.rot[1] * h.rot[1] + h.rot[2] * h.rot[2] +
                      h.rot[3] * h.rot[3];
    if (!finite || !(q2 > 0.0)) return fail(WCG_ERR_ARG, "terminator shape not finite");
    wcg::TermShape& s = t.s[k];
    s.type = h.type;
    s.sign = h.inside ? -1.0 : 1.0;
    for (int a = 0; a < 3; ++a) s.c[a] = h.center[a];
    for (int a = 0; a < 4; ++a) {
      s.q[a] = h.rot[a];
      s.par[a] = h.param[a];
    }
  }
  t.n = n;
  ctx->c.term = t;
  ctx->c.prm.terminator = n > 0 ? 1 : 0;
  return WCG_OK;
}

int wcg_set_correction_count(wcg_ctx* ctx, unsigned long long k) {
  WCG_CHECK_CTX(ctx);
  ctx->c.corr_count = k;
  return WCG_OK;
}

unsigned long long wcg_correction_count(const wcg_ctx* ctx) { return ctx ? ctx->c.corr_count : 0; }

unsigned long long wcg_split_key(unsigned long long seed, unsigned long long k) {
  return wcg::split_key(seed, k);
}

int wcg_merge_draws(unsigned long long seed, unsigned long long k, int step, int* selector,
                    int* perm9) {
  if (!selector || !perm9 || step < 1) return fail(WCG_ERR_ARG, "bad merge draw arguments");
  wcg::merge_draws(seed, k, step, selector, perm9);
  return WCG_OK;
}

int wcg_correction_selector(unsigned long long seed, unsigned long long k, int step) {
  return wcg::correction_selector(seed, k, step);
}

int wcg_advect(wcg_ctx* ctx, double dt) {
  WCG_CHECK_CTX(ctx);
  WCG_CALL(ctx, wcg::advect_only(ctx->c, dt), "advectScene");
  ctx->c.have_grid = false;
  return device_status(ctx->c, "advectScene");
}

int wcg_substep(wcg_ctx* ctx, double dt) {
  WCG_CHECK_CTX(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  WCG_CALL(ctx, wcg::substep(ctx->c, dt), "substep");
  int s = device_status(ctx->c, "substep");
  if (s) return s;
  ctx->c.have_grid = false;
  if (!ctx->c.stats.converged)
    return fail(WCG_ERR_NOT_CONVERGED, "pressure PCG did not converge");
  if (!ctx->c.stats.visc_converged)
    return fail(WCG_ERR_NOT_CONVERGED, "implicit viscosity PCG did not converge");
  return WCG_OK;
}

int wcg_substep_vjp(wcg_ctx* ctx, double dt, const double* vbar3, const double* Cbar9,
                    const double* xbar3, double* vbar0, double* Cbar0, double* xbar0,
                    double* viscosity_bar) {
  WCG_CHECK_CTX(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  WCG_NO_ELASTO(ctx, "substep_vjp");
  if (ctx->c.prm.viscosity > 0.0 && ctx->c.prm.viscosity_implicit)
    return fail(WCG_ERR_UNSUPPORTED, "substep_vjp: not available with the implicit viscosity");
  if (ctx->c.prm.particle_merge || ctx->c.prm.particle_split || ctx->c.prm.terminator)
    return fail(WCG_ERR_UNSUPPORTED,
                "substep_vjp: not available with the particle merge, split or terminator on");
  const long long n = ctx->c.np;
  if (n > 0 && (!vbar3 || !Cbar9 || !xbar3 || !vbar0 || !Cbar0 || !xbar0))
    return fail(WCG_ERR_ARG, "null cotangent array");
  WCG_CALL(ctx, wcg::substep_vjp(ctx->c, dt, vbar3, Cbar9, xbar3, vbar0, Cbar0,
                                 ctx->c.adjoint_fixed_x ? nullptr : xbar0, viscosity_bar),
           "substep_vjp");
  int st = device_status(ctx->c, "substep_vjp");
  if (st) return st;
  if (ctx->c.adjoint_fixed_x)
    for (long long i = 0; i < 3 * n; ++i) xbar0[i] = xbar3[i];
  ctx->c.have_grid = true;
  if (!ctx->c.stats.converged)
    return fail(WCG_ERR_NOT_CONVERGED, "adjoint pressure solve did not converge");
  return WCG_OK;
}

int wcg_set_adjoint_positions(wcg_ctx* ctx, int differentiate) {
  WCG_CHECK_CTX(ctx);
  ctx->c.adjoint_fixed_x = differentiate ? 0 : 1;
  return WCG_OK;
}

int wcg_set_viscosity(wcg_ctx* ctx, double viscosity, int substeps) {
  WCG_CHECK_CTX(ctx);
  if (!(viscosity >= 0.0) || !std::isfinite(viscosity))
    return fail(WCG_ERR_ARG, "viscosity must be finite and >= 0");
  ctx->c.prm.viscosity = viscosity;
  ctx->c.prm.viscosity_substeps = substeps > 0 ? substeps : 1;
  return WCG_OK;
}

int wcg_set_schedule(wcg_ctx* ctx, const wcg_schedule* s) {
  WCG_CHECK_CTX(ctx);
  if (!s) return fail(WCG_ERR_ARG, "null schedule");
  const int cc = s->sweep_cluster, ca = s->sweep_cluster_a;
  if (!(cc == 0 || cc == 1 || cc == 2 || cc == 3 || cc == 4 || cc == 8 || cc == 9 || cc == 16))
    return fail(WCG_ERR_ARG, "sweep_cluster must be 0, 1, 2, 3, 4, 8, 9 or 16");
  if (!(ca == 1 || (ca == 4 && cc >= 1 && cc <= 4) || (ca == 8 && cc >= 1 && cc <= 2)))
    return fail(WCG_ERR_ARG, "sweep_cluster_a must be 1, 4 (sweep_cluster 1..4) or 8 "
                             "(sweep_cluster 1..2)");
  if (s->pcg_batch < 1 || s->pcg_batch > 64) return fail(WCG_ERR_ARG, "pcg_batch must lie in [1, 64]");
  ctx->c.sweep_cluster = cc;
  ctx->c.sweep_cluster_a = ca;
  ctx->c.pcg_batch = s->pcg_batch;
  return WCG_OK;
}

int wcg_get_schedule(const wcg_ctx* ctx, wcg_schedule* s) {
  if (!ctx || !s) return fail(WCG_ERR_ARG, "null argument");
  s->sweep_cluster = ctx->c.sweep_cluster;
  s->sweep_cluster_a = ctx->c.sweep_cluster_a;
  s->pcg_batch = ctx->c.pcg_batch;
  return WCG_OK;
}

int wcg_set_wait_limit(wcg_ctx* ctx, long long spin_limit, int stale_patch) {
  WCG_CHECK_CTX(ctx);
  if (spin_limit < 1 || spin_limit > (1ll << 40))
    return fail(WCG_ERR_ARG, "spin_limit must lie in [1, 2^40]");
  ctx->c.spin_limit = spin_limit;
  ctx->c.stale_patch = stale_patch < 0 ? -1 : stale_patch;
  return WCG_OK;
}

int wcg_num_substeps(wcg_ctx* ctx, double dt, int* n_out) {
  WCG_CHECK_CTX(ctx);
  if (!n_out || !(dt > 0)) return fail(WCG_ERR_ARG, "bad argument");
  WCG_CALL(ctx, wcg::num_substeps(ctx->c, dt, n_out), "num_substeps");
  return WCG_OK;
}

int wcg_step(wcg_ctx* ctx, double dt, int* substeps_out) {
  WCG_CHECK_CTX(ctx);
  if (!(dt > 0)) return fail(WCG_ERR_ARG, "dt must be positive");
  int n = 1;
  WCG_CALL(ctx, wcg::num_substeps(ctx->c, dt, &n), "num_substeps");
  // a staged upload is checked on the device: stop before stepping bad input
  if (int st = device_status(ctx->c, "particle upload")) return st;
  const double sub = dt / (double)n;
  int status = WCG_OK;
  for (int k = 0; k < n; ++k) {
    int s = wcg_substep(ctx, sub);
    if (s == WCG_ERR_NOT_CONVERGED) {
      status = s;  // the reference warns and continues (Pressure.cpp:803-811)
      continue;
    }
    if (s) return s;
  }
  ctx->c.stats.substeps = n;
  if (substeps_out) *substeps_out = n;
  return status;
}

int wcg_get_stats(const wcg_ctx* ctx, wcg_stats* out) {
  if (!ctx || !out) return fail(WCG_ERR_ARG, "null argument");
  const wcg::Stats& s = ctx->c.stats;
  out->substeps = s.substeps;
  out->pcg_iters = s.pcg_iters;
  out->refinements = s.refinements;
  out->converged = s.converged;
  out->residual = s.residual;
  out->rhs_norm = s.rhs_norm;
  out->ndof = s.ndof;
  out->nactive_buckets = s.nactive;
  out->visc_iters = s.visc_iters;
  out->visc_converged = s.visc_converged;
  out->visc_residual = s.visc_residual;
  return WCG_OK;
}

int wcg_grid_info(const wcg_ctx* ctx, int* dims, double* origin, double* bbx) {
  if (!ctx) return fail(WCG_ERR_ARG, "null context");
  if (!ctx->c.have_grid && ctx->c.g.nb == 0) return fail(WCG_ERR_STATE, "no grid");
  const wcg::GridDesc& g = ctx->c.g;
  if (dims) {
    dims[0] = g.ni;
    dims[1] = g.nj;
    dims[2] = g.nk;
  }
  if (origin) {
    origin[0] = g.ox;
    origin[1] = g.oy;
    origin[2] = g.oz;
  }
  if (bbx)
    for (int a = 0; a < 3; ++a) {
      bbx[a] = ctx->c.bbx_min[a];
      bbx[3 + a] = ctx->c.bbx_max[a];
    }
  return WCG_OK;
}

long long wcg_field_size(wcg_ctx* ctx, const char* name) {
  if (!ctx || !name) return -1;
  const wcg::Context& c = ctx->c;
  int ncomp = 1;
  if (lookup_field(name, &ncomp) >= -1) return ncomp * c.g.nnode;
  if (!strcmp(name, "active")) return c.g.nb;
  if (!strcmp(name, "dof_index") || !strcmp(name, "valid_x") ||
      !strcmp(name, "valid_y") || !strcmp(name, "valid_z"))
    return c.g.nnode;
  if (!strcmp(name, "array_idx")) return c.np + c.ne;
  if (!strcmp(name, "array_sup")) return 2 * c.g.nb;
  if (!strcmp(name, "stencil_base")) return 15 * (c.np + c.ne);
  if (!strcmp(name, "grid_dims")) return 3;
  return -1;
}

int wcg_download_field(wcg_ctx* ctx, const char* name, double* out, long long n) {
  WCG_CHECK_CTX(ctx);
  if (!name || !out) return fail(WCG_ERR_ARG, "null argument");
  wcg::Context& c = ctx->c;
  int ncomp = 1;
  const int f = lookup_field(name, &ncomp);
  if (f < -1) return fail(WCG_ERR_ARG, std::string("unknown field ") + name);
  if (n < ncomp * c.g.nnode) return fail(WCG_ERR_ARG, "output buffer too small");
  cudaStreamSynchronize(c.stream);
  std::vector<unsigned char> act = host_active(c);
  const double nan = std::numeric_limits<double>::quiet_NaN();
  // a multi-component field (orientation) interleaves its components per node
  for (int q = 0; q < ncomp; ++q) {
    std::vector<double> v = host_field(c, f < 0 ? f : f + q);
    for (long long i = 0; i < c.g.nnode; ++i) out[i * ncomp + q] = act[i >> 6] ? v[i] : nan;
  }
  cudaError_t e = cudaGetLastError();
  return cuda_status(c, e, "download_field");
}

// Node velocities a caller may set between the reference's calls (the
// host-side seam for work not done here, e.g. a solid solve): the liquid face
// velocity G2P reads ("u_*") and the solid-phase face velocity ("vel_*", with
// elasto particles).  Values of nodes in inactive buckets are ignored.
int wcg_upload_field(wcg_ctx* ctx, const char* name, const double* in, long long n) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  if (!name || !in) return fail(WCG_ERR_ARG, "null argument");
  wcg::Context& c = ctx->c;
  int f = -2;
  for (const char* w : {"u_x", "u_y", "u_z", "vel_x", "vel_y", "vel_z"})
    if (!strcmp(name, w)) f = lookup_field(name);
  if (f < 0) return fail(WCG_ERR_ARG, std::string("field is not writable: ") + name);
  const bool ef = f >= kEBase;
  if (ef && c.ne == 0) return fail(WCG_ERR_STATE, "solid-phase fields need elasto particles");
  const long long nn = c.g.nnode;
  if (n < nn) return fail(WCG_ERR_ARG, "input buffer too small");
  cudaStreamSynchronize(c.stream);
  std::vector<double> v = host_field(c, f);
  std::vector<unsigned char> act = host_active(c);
  for (long long i = 0; i < nn; ++i)
    if (act[i >> 6]) v[i] = in[i];
  wcg::DevBuf& buf = ef ? c.efield : c.gfield;
  const size_t off = (size_t)(ef ? f - kEBase : f) * c.gcap;
  cudaError_t e;
  if (c.prm.precision == 0) {
    e = cudaMemcpy(buf.as<double>() + off, v.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  } else {
    std::vector<float> h(v.begin(), v.end());
    e = cudaMemcpy(buf.as<float>() + off, h.data(), nn * sizeof(float), cudaMemcpyHostToDevice);
  }
  return cuda_status(c, e, "upload_field");
}

int wcg_download_ifield(wcg_ctx* ctx, const char* name, long long* out, long long n) {
  WCG_CHECK_CTX(ctx);
  if (!name || !out) return fail(WCG_ERR_ARG, "null argument");
  wcg::Context& c = ctx->c;
  const long long need = wcg_field_size(ctx, name);
  if (need < 0) return fail(WCG_ERR_ARG, std::string("unknown field ") + name);
  if (n < need) return fail(WCG_ERR_ARG, "output buffer too small");
  cudaStreamSynchronize(c.stream);
  const wcg::GridDesc& g = c.g;
  if (!strcmp(name, "grid_dims")) {
    out[0] = g.ni;
    out[1] = g.nj;
    out[2] = g.nk;
    return WCG_OK;
  }
  if (!strcmp(name, "active")) {
    std::vector<unsigned char> a = host_active(c);
    for (long long i = 0; i < g.nb; ++i) out[i] = a[i];
    return WCG_OK;
  }
  if (!strcmp(name, "dof_index")) {
    std::vector<unsigned char> a = host_active(c);
    std::vector<unsigned char> d = host_bytes(c.gdof.p, g.nnode);
    long long k = 0;
    for (long long i = 0; i < g.nnode; ++i) {
      if (!a[i >> 6]) out[i] = -2;
      else out[i] = d[i] ? k++ : -1;
    }
    return WCG_OK;
  }
  if (!strncmp(name, "valid_", 6)) {
    const int comp = name[6] - 'x';
    std::vector<unsigned char> a = host_active(c);
    std::vector<unsigned char> v =
        host_bytes((const unsigned char*)c.gvalid.p + (size_t)comp * c.gcap, g.nnode);
    for (long long i = 0; i < g.nnode; ++i) out[i] = a[i >> 6] ? v[i] : -1;
    return WCG_OK;
  }
  // all particles in the reference's numbering: elasto [0, ne), liquid after
  const long long ne = c.ne, nl = c.np, np = ne + nl;
  std::vector<int> pid(np), pb(np), dl(np);
  std::vector<long long> key(np);
  if (ne) {
    cudaMemcpy(pid.data(), c.epid[c.ecur].p, ne * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(pb.data(), c.ebucket.as<int>() + c.ecur * c.ecap, ne * sizeof(int),
               cudaMemcpyDeviceToHost);
    cudaMemcpy(dl.data(), c.edelta.as<int>() + c.ecur * c.ecap, ne * sizeof(int),
               cudaMemcpyDeviceToHost);
    cudaMemcpy(key.data(), c.ekey.as<long long>() + c.ecur * c.ecap, ne * sizeof(long long),
               cudaMemcpyDeviceToHost);
  }
  if (nl) {
    cudaMemcpy(pid.data() + ne, c.pid[c.cur].p, nl * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(pb.data() + ne, c.pbucket.as<int>() + c.cur * c.pcap, nl * sizeof(int),
               cudaMemcpyDeviceToHost);
    cudaMemcpy(dl.data() + ne, c.pdelta.as<int>() + c.cur * c.pcap, nl * sizeof(int),
               cudaMemcpyDeviceToHost);
    cudaMemcpy(key.data() + ne, c.pkey.as<long long>() + c.cur * c.pcap, nl * sizeof(long long),
               cudaMemcpyDeviceToHost);
    for (long long s = ne; s < np; ++s) pid[s] += (int)ne;
  }
  if (!strcmp(name, "array_idx") || !strcmp(name, "array_sup")) {
    // Sorter::sort keys (bucket << 32 | particle), sorted
    std::vector<unsigned long long> keys(np);
    for (long long s = 0; s < np; ++s)
      keys[s] = ((unsigned long long)(unsigned)pb[s] << 32) | (unsigned)pid[s];
    std::sort(keys.begin(), keys.end());
    if (!strcmp(name, "array_idx")) {
      for (long long s = 0; s < np; ++s) out[s] = (long long)keys[s];
    } else {
      for (long long b = 0; b < 2 * g.nb; ++b) out[b] = 0;
      for (long long s = 0; s < np; ++s) {
        const long long b = (long long)(keys[s] >> 32);
        if (s == 0 || (long long)(keys[s - 1] >> 32) != b) out[2 * b] = s;
        if (s == np - 1 || (long long)(keys[s + 1] >> 32) != b) out[2 * b + 1] = s + 1;
      }
    }
    return WCG_OK;
  }
  if (!strcmp(name, "stencil_base")) {
    for (long long s = 0; s < np; ++s) {
      const long long k = key[s];
      const long long b = k >> 6;
      const int l = (int)(k & 63);
      const long long bk = b / ((long long)g.ni * g.nj);
      const long long rem = b - bk * g.ni * g.nj;
      const long long bj = rem / g.ni;
      const long long bi = rem - bj * g.ni;
      const long long P[3] = {bi * 4 + (l & 3) - 1, bj * 4 + ((l >> 2) & 3) - 1,
                              bk * 4 + (l >> 4) - 1};
      long long d[3];
      for (int a = 0; a < 3; ++a) d[a] = ((dl[s] >> (4 * a)) & 15) - 4;
      long long* o = out + (long long)pid[s] * 15;
      for (int t = 0; t < 5; ++t)
        for (int a = 0; a < 3; ++a) {
          const bool zero = (t == 3) || (t == a);
          o[t * 3 + a] = P[a] + (zero ? d[a] : 0);
        }
    }
    return WCG_OK;
  }
  return fail(WCG_ERR_ARG, std::string("unknown field ") + name);
}

int wcg_export_pressure_system(wcg_ctx* ctx, long long* ndof, long long* nnz,
                               long long* rowstart, long long* col, double* val,
                               double* rhs) {
  WCG_CHECK_CTX(ctx);
  WCG_NEED_GRID(ctx);
  wcg::Context& c = ctx->c;
  cudaStreamSynchronize(c.stream);
  const wcg::GridDesc& g = c.g;
  std::vector<unsigned char> a = host_active(c);
  std::vector<unsigned char> d = host_bytes(c.gdof.p, g.nnode);
  std::vector<double> AD = host_field(c, wcg::G_ADIAG), AX = host_field(c, wcg::G_AX),
                      AY = host_field(c, wcg::G_AY), AZ = host_field(c, wcg::G_AZ),
                      B = host_field(c, wcg::G_B);
  std::vector<long long> num((size_t)g.nnode, -1);
  long long k = 0;
  for (long long i = 0; i < g.nnode; ++i)
    if (a[i >> 6] && d[i]) num[i] = k++;
  auto lin = [&](int I, int J, int K) -> long long {
    if (I < 0 || J < 0 || K < 0 || I >= g.NI || J >= g.NJ || K >= g.NK) return -1;
    const long long q = wcg::node_linear(g, I, J, K);
    return num[q];
  };
  // Structural entries come from the assembly flags (bit1-3: +x/+y/+z
  // coupling, bit4: diagonal); values may be exact zeros.
  long long nz = 0;
  std::vector<std::pair<long long, double>> row;
  for (long long i = 0; i < g.nnode; ++i) {
    if (num[i] < 0) continue;
    int I, J, K;
    {
      const long long b = i >> 6;
      const int l = (int)(i & 63);
      const long long bk = b / ((long long)g.ni * g.nj);
      const long long rem = b - bk * g.ni * g.nj;
      const long long bj = rem / g.ni;
      const long long bi = rem - bj * g.ni;
      I = (int)(bi * 4 + (l & 3));
      J = (int)(bj * 4 + ((l >> 2) & 3));
      K = (int)(bk * 4 + (l >> 4));
    }
    row.clear();
    if (d[i] & 16) row.push_back({num[i], AD[i]});
    const long long nl[6] = {lin(I - 1, J, K), lin(I + 1, J, K), lin(I, J - 1, K),
                             lin(I, J + 1, K), lin(I, J, K - 1), lin(I, J, K + 1)};
    const long long lo[3] = {I > 0 ? wcg::node_linear(g, I - 1, J, K) : -1,
                             J > 0 ? wcg::node_linear(g, I, J - 1, K) : -1,
                             K > 0 ? wcg::node_linear(g, I, J, K - 1) : -1};
    const double* AA[3] = {AX.data(), AY.data(), AZ.data()};
    for (int a = 0; a < 3; ++a) {
      if (nl[2 * a] >= 0 && (d[lo[a]] & (2 << a)))
        row.push_back({nl[2 * a], AA[a][lo[a]]});
      if (nl[2 * a + 1] >= 0 && (d[i] & (2 << a))) row.push_back({nl[2 * a + 1], AA[a][i]});
    }
    std::sort(row.begin(), row.end(),
              [](const std::pair<long long, double>& x, const std::pair<long long, double>& y) {
                return x.first < y.first;
              });
    const long long r = num[i];
    if (rowstart) {
      rowstart[r] = nz;
      for (auto& e : row) {
        col[nz] = e.first;
        val[nz] = e.second;
        ++nz;
      }
      if (rhs) rhs[r] = B[i];
    } else {
      nz += (long long)row.size();
    }
  }
  if (rowstart) rowstart[k] = nz;
  if (ndof) *ndof = k;
  if (nnz) *nnz = nz;
  c.stats.ndof = k;
  return WCG_OK;
}

void* wcg_stream(const wcg_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

long long wcg_launch_count(const wcg_ctx* ctx) { return ctx ? ctx->c.launches : -1; }

int wcg_profile_begin(wcg_ctx* ctx) {
  WCG_CHECK_CTX(ctx);
  wcg::Context& c = ctx->c;
  cudaStreamSynchronize(c.stream);
  for (auto& r : c.prof_recs) {
    c.prof_pool.push_back(r.a);
    c.prof_pool.push_back(r.b);
  }
  c.prof_recs.clear();
  c.prof_on = true;
  return WCG_OK;
}

int wcg_profile_end(wcg_ctx* ctx, double* ms, long long* launches, int ncat) {
  WCG_CHECK_CTX(ctx);
  wcg::Context& c = ctx->c;
  c.prof_on = false;
  WCG_CALL(ctx, cudaStreamSynchronize(c.stream), "profile_end");
  for (int k = 0; k < ncat; ++k) {
    if (ms) ms[k] = 0;
    if (launches) launches[k] = 0;
  }
  for (auto& r : c.prof_recs) {
    float t = 0;
    cudaEventElapsedTime(&t, r.a, r.b);
    if (r.cat < ncat) {
      if (ms) ms[r.cat] += t;
      if (launches) launches[r.cat] += r.nlaunch;
    }
    c.prof_pool.push_back(r.a);
    c.prof_pool.push_back(r.b);
  }
  c.prof_recs.clear();
  return WCG_OK;
}

int wcg_profile_num_phases(void) { return wcg::kNumProfCats; }

const char* wcg_profile_phase_name(int i) {
  static const char* names[] = {"grid_build_sort", "p2g", "grid_ops", "mic_factor",
                                "mic_sweep", "pcg_vector", "refine_fp64", "g2p_advect",
                                "other"};
  return (i >= 0 && i < wcg::kNumProfCats) ? names[i] : "";
}

}  // extern "C"
