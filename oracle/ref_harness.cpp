// Harness around the libWetCloth reference Core (compiled from the reference
// sources by oracle/ref.mk).  TEST INFRASTRUCTURE ONLY: it is the checker that
// pins the C restatement (oracle/wc_oracle.c) and the timed CPU baseline; no
// product code links it.
//
// It builds a TwoDScene programmatically (the XML parser TU needs
// GL headers), replays the fluid hot path in WetClothCore::stepSystem order
// (libWetCloth/Core/WetClothCore.cpp:115-258, minus the particle maintenance,
// elasto and surface-tension calls which are no-ops or out of scope for a
// liquid scene) and snapshots every hot-path field into dense bucket-major
// arrays (bucket index * 64 + local node index, libWetCloth/Core/Sorter.h:63,
// TwoDScene.cpp:3746) that Python reads through ctypes.
//
// Scene set-up follows TwoDScene::sampleLiquidDistanceFields
// (Core/TwoDScene.cpp:5564-5605) for the per-particle attributes and
// TwoDSceneXMLParser::loadLiquidInfo (App/TwoDSceneXMLParser.cpp:1851-1904) for
// the LiquidInfo defaults.  Walls are one DistanceFieldObject of type DFT_BOX,
// usage DFU_SOLID, inside=true (Core/DistanceFields.cpp:478-516).
//
// Pressure: the reference's default solver is the multigrid PCG
// (Core/Pressure.cpp:797).  With mic=1 the harness re-solves the very matrix
// and rhs that solveNodePressure assembled with the reference's own
// robertbridson::PCGSolver<double> (MIC(0), omega 0.97, min ratio 0.25,
// Core/PCGSolver/PCGSolver.h:245-330) and scatters that solution into the
// scene's pressure field, so the rest of the step uses the MIC(0) pressures.
// Standard-library and Eigen headers first, so the access override below only
// reaches the reference's own classes.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <stack>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include "AlgebraicMultigrid.h"
#include "MathDefs.h"
#include <Eigen/Geometry>
#define private public
#define protected public
#include "LinearizedImplicitEuler.h"
#include "PCGSolver/PCGSolver.h"
#include "SimpleGravityForce.h"
#include "TwoDScene.h"
#include "DistanceFields.h"
#include "WetClothCore.h"
#undef private
#undef protected

#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace {

struct Params {
  double dx;
  double gravity[3];
  double liquid_density;
  double flip_coeff;
  double liquid_boundary_friction;
  double box_center[3];
  double box_half[3];
  double box_radius;
  double criterion;
  int maxiters;
  int mic;
};

struct Harness {
  std::shared_ptr<TwoDScene> scene;
  std::shared_ptr<LinearizedImplicitEuler> stepper;
  Params p;
  std::map<std::string, std::vector<double>> f;    // dense double snapshots
  std::map<std::string, std::vector<long long>> ii;  // integer snapshots
  double timers[12];
  int last_iters_amg = 0, last_iters_mic = 0;
  double last_res_amg = 0, last_res_mic = 0;
  unsigned corr_seed = 0, corr_count = 0;
  bool term_on = false;       // terminateParticles first (WetClothCore.cpp:97)
  bool grid_built = false;    // a grid exists for removeEmptyParticles' re-sort
};

// the correction subset of call k of a seeded stream: SplitMix64 (Steele,
// Lea and Flood 2014) of the seed and k, modulo the step -- the stream the
// oracle (wco_correction_selector) and the GPU (wcg_correction_selector) use
uint64_t splitmix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

int seeded_selector(uint64_t seed, uint64_t k, int step) {
  return (int)(splitmix(seed ^ splitmix(k)) % (uint64_t)(step > 0 ? step : 1));
}

double now() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// dense copy of a per-bucket node field; inactive buckets are NaN
void dense(Harness& h, const std::string& name,
           const std::vector<VectorXs>& v, int per_node = 1) {
  const int nb = h.scene->getNumBuckets();
  const int nn = h.scene->getDefaultNumNodes();
  const int count = nn * nn * nn;
  std::vector<double>& out = h.f[name];
  out.assign((size_t)nb * count * per_node,
             std::numeric_limits<double>::quiet_NaN());
  for (int b = 0; b < nb && b < (int)v.size(); ++b) {
    if ((int)v[b].size() != count * per_node) continue;
    for (int i = 0; i < count * per_node; ++i)
      out[(size_t)b * count * per_node + i] = v[b][i];
  }
}

void dense_uc(Harness& h, const std::string& name,
              const std::vector<VectorXuc>& v) {
  const int nb = h.scene->getNumBuckets();
  const int count = 64;
  std::vector<long long>& out = h.ii[name];
  out.assign((size_t)nb * count, -1);
  for (int b = 0; b < nb && b < (int)v.size(); ++b) {
    if ((int)v[b].size() != count) continue;
    for (int i = 0; i < count; ++i) out[(size_t)b * count + i] = v[b][i];
  }
}

void dense_vi(Harness& h, const std::string& name,
              const std::vector<VectorXi>& v) {
  const int nb = h.scene->getNumBuckets();
  const int count = 64;
  std::vector<long long>& out = h.ii[name];
  out.assign((size_t)nb * count, -2);
  for (int b = 0; b < nb && b < (int)v.size(); ++b) {
    if ((int)v[b].size() != count) continue;
    for (int i = 0; i < count; ++i) out[(size_t)b * count + i] = v[b][i];
  }
}

void snap_particles(Harness& h, const std::string& tag) {
  TwoDScene& s = *h.scene;
  const int np = s.getNumParticles();
  std::vector<double>& x = h.f[tag + "x"];
  std::vector<double>& v = h.f[tag + "v"];
  std::vector<double>& c = h.f[tag + "C"];
  std::vector<double>& x4 = h.f[tag + "x4"];
  std::vector<double>& ev = h.f[tag + "ev4"];
  std::vector<double>& eb = h.f[tag + "eB"];
  x.resize((size_t)np * 3);
  v.resize((size_t)np * 3);
  c.resize((size_t)np * 9);
  x4.resize((size_t)np * 4);
  ev.resize((size_t)np * 4);
  eb.resize((size_t)np * 9);
  for (int i = 0; i < np; ++i) {
    for (int r = 0; r < 3; ++r) {
      x[i * 3 + r] = s.m_x(i * 4 + r);
      v[i * 3 + r] = s.m_fluid_v(i * 4 + r);
      for (int q = 0; q < 3; ++q) {
        c[i * 9 + r * 3 + q] = s.m_fB(i * 3 + r, q);
        eb[i * 9 + r * 3 + q] = s.m_B(i * 3 + r, q);
      }
    }
    for (int r = 0; r < 4; ++r) {
      x4[i * 4 + r] = s.m_x(i * 4 + r);
      ev[i * 4 + r] = s.m_v(i * 4 + r);
    }
  }
}

void snap_grid(Harness& h) {
  TwoDScene& s = *h.scene;
  const Sorter& b = s.m_particle_buckets;
  h.f["grid_origin"] = {s.m_grid_mincorner(0), s.m_grid_mincorner(1),
                        s.m_grid_mincorner(2)};
  h.f["bbx"] = {s.m_bbx_min(0), s.m_bbx_min(1), s.m_bbx_min(2),
                s.m_bbx_max(0), s.m_bbx_max(1), s.m_bbx_max(2)};
  h.ii["grid_dims"] = {b.ni, b.nj, b.nk};
  std::vector<long long>& keys = h.ii["array_idx"];
  keys.assign(b.array_idx.begin(), b.array_idx.end());
  std::vector<long long>& sup = h.ii["array_sup"];
  sup.resize(b.array_sup.size() * 2);
  for (size_t i = 0; i < b.array_sup.size(); ++i) {
    sup[i * 2] = b.array_sup[i].first;
    sup[i * 2 + 1] = b.array_sup[i].second;
  }
  std::vector<long long>& act = h.ii["active"];
  act.assign(s.m_bucket_activated.begin(), s.m_bucket_activated.end());
  // first stencil node of each particle per node kind, as global node ijk
  const int np = s.getNumParticles();
  const int nn = s.getDefaultNumNodes();
  const std::vector<Matrix27x2i>* kinds[5] = {
      &s.m_particle_nodes_x, &s.m_particle_nodes_y, &s.m_particle_nodes_z,
      &s.m_particle_nodes_solid_phi, &s.m_particle_nodes_p};
  std::vector<long long>& base = h.ii["stencil_base"];
  base.resize((size_t)np * 15);
  for (int pidx = 0; pidx < np; ++pidx)
    for (int k = 0; k < 5; ++k) {
      const Matrix27x2i& m = (*kinds[k])[pidx];
      Vector3i bh = b.bucket_handle(m(0, 0));
      Vector3i nh = s.getNodeHandle(m(0, 1));
      for (int r = 0; r < 3; ++r)
        base[(size_t)pidx * 15 + k * 3 + r] = (long long)bh(r) * nn + nh(r);
    }
  std::vector<long long>& inside = h.ii["inside"];
  inside.assign(s.m_inside.data(), s.m_inside.data() + s.m_inside.size());
}

void snap_p2g(Harness& h) {
  TwoDScene& s = *h.scene;
  dense(h, "mass_fluid_x", s.m_node_mass_fluid_x);
  dense(h, "mass_fluid_y", s.m_node_mass_fluid_y);
  dense(h, "mass_fluid_z", s.m_node_mass_fluid_z);
  dense(h, "vel_fluid_x", s.m_node_vel_fluid_x);
  dense(h, "vel_fluid_y", s.m_node_vel_fluid_y);
  dense(h, "vel_fluid_z", s.m_node_vel_fluid_z);
  dense(h, "vol_fluid_x", s.m_node_vol_fluid_x);
  dense(h, "vol_fluid_y", s.m_node_vol_fluid_y);
  dense(h, "vol_fluid_z", s.m_node_vol_fluid_z);
  dense(h, "mass_x", s.m_node_mass_x);
  dense(h, "mass_y", s.m_node_mass_y);
  dense(h, "mass_z", s.m_node_mass_z);
  dense(h, "vol_x", s.m_node_vol_x);
  dense(h, "vol_y", s.m_node_vol_y);
  dense(h, "vol_z", s.m_node_vol_z);
  dense(h, "vel_x", s.m_node_vel_x);
  dense(h, "vel_y", s.m_node_vel_y);
  dense(h, "vel_z", s.m_node_vel_z);
  dense(h, "shape_factor_x", s.m_node_shape_factor_x);
  dense(h, "shape_factor_y", s.m_node_shape_factor_y);
  dense(h, "shape_factor_z", s.m_node_shape_factor_z);
  dense(h, "orientation_x", s.m_node_orientation_x, 3);
  dense(h, "orientation_y", s.m_node_orientation_y, 3);
  dense(h, "orientation_z", s.m_node_orientation_z, 3);
  dense(h, "psi_x", s.m_node_psi_x);
  dense(h, "psi_y", s.m_node_psi_y);
  dense(h, "psi_z", s.m_node_psi_z);
  dense(h, "sat_x", s.m_node_sat_x);
  dense(h, "sat_y", s.m_node_sat_y);
  dense(h, "sat_z", s.m_node_sat_z);
  dense(h, "sat_p", s.m_node_sat_p);
  dense(h, "psi_p", s.m_node_psi_p);
  dense(h, "pore_pressure_p", s.m_node_pore_pressure_p);
  dense(h, "liquid_phi", s.m_node_liquid_phi);
  if (s.getLiquidInfo().compute_viscosity) {
    dense(h, "liquid_c_vf", s.m_node_liquid_c_vf);
    dense(h, "liquid_ex_vf", s.m_node_liquid_ex_vf);
    dense(h, "liquid_ey_vf", s.m_node_liquid_ey_vf);
    dense(h, "liquid_ez_vf", s.m_node_liquid_ez_vf);
    if (s.getLiquidInfo().implicit_viscosity) {
      dense(h, "liquid_u_vf", s.m_node_liquid_u_vf);
      dense(h, "liquid_v_vf", s.m_node_liquid_v_vf);
      dense(h, "liquid_w_vf", s.m_node_liquid_w_vf);
    }
  }
  dense(h, "solid_phi", s.m_node_solid_phi);
  dense(h, "solid_weight_x", s.m_node_solid_weight_x);
  dense(h, "solid_weight_y", s.m_node_solid_weight_y);
  dense(h, "solid_weight_z", s.m_node_solid_weight_z);
  dense(h, "solid_vel_x", s.m_node_solid_vel_x);
  dense(h, "solid_vel_y", s.m_node_solid_vel_y);
  dense(h, "solid_vel_z", s.m_node_solid_vel_z);
}

void snap_predict(Harness& h) {
  LinearizedImplicitEuler& e = *h.stepper;
  dense(h, "v_star_x", e.m_node_v_fluid_plus_x);
  dense(h, "v_star_y", e.m_node_v_fluid_plus_y);
  dense(h, "v_star_z", e.m_node_v_fluid_plus_z);
  const LiquidInfo& li = h.scene->getLiquidInfo();
  if (li.compute_viscosity && li.implicit_viscosity) {
    // the last implicit viscosity sub-step's system (Viscosity.cpp:789-1779)
    const robertbridson::SparseMatrix<scalar>& A = e.m_visc_matrix;
    std::vector<long long>& rs = h.ii["V_rowstart"];
    std::vector<long long>& ci = h.ii["V_col"];
    std::vector<double>& va = h.f["V_val"];
    rs.assign(1, 0);
    ci.clear();
    va.clear();
    for (unsigned i = 0; i < A.n; ++i) {
      for (size_t k = 0; k < A.index[i].size(); ++k) {
        ci.push_back(A.index[i][k]);
        va.push_back(A.value[i][k]);
      }
      rs.push_back((long long)ci.size());
    }
    h.f["V_rhs"] = e.m_visc_rhs;
    h.f["V_rhs"].resize(A.n);
    h.f["V_soln"] = e.m_visc_solution;
    h.f["V_soln"].resize(A.n);
  }
  dense(h, "rhs_fluid_x", e.m_node_rhs_fluid_x);
  dense(h, "rhs_fluid_y", e.m_node_rhs_fluid_y);
  dense(h, "rhs_fluid_z", e.m_node_rhs_fluid_z);
  dense(h, "inv_C_x", e.m_node_inv_C_x);
  dense(h, "inv_C_y", e.m_node_inv_C_y);
  dense(h, "inv_C_z", e.m_node_inv_C_z);
  dense(h, "psi_fs_x", e.m_node_psi_fs_x);
  dense(h, "psi_fs_y", e.m_node_psi_fs_y);
  dense(h, "psi_fs_z", e.m_node_psi_fs_z);
}

void snap_system(Harness& h) {
  LinearizedImplicitEuler& e = *h.stepper;
  const robertbridson::SparseMatrix<scalar>& A = e.m_fine_pressure_matrix;
  std::vector<long long>& rs = h.ii["A_rowstart"];
  std::vector<long long>& ci = h.ii["A_col"];
  std::vector<double>& va = h.f["A_val"];
  rs.assign(1, 0);
  ci.clear();
  va.clear();
  for (unsigned i = 0; i < A.n; ++i) {
    for (size_t k = 0; k < A.index[i].size(); ++k) {
      ci.push_back(A.index[i][k]);
      va.push_back(A.value[i][k]);
    }
    rs.push_back((long long)ci.size());
  }
  h.f["b"] = e.m_fine_pressure_rhs;
  h.f["b"].resize(A.n);
  dense_vi(h, "dof_index", e.m_fine_global_indices);
}

// One liquid particle, attribute set of TwoDScene::sampleLiquidDistanceFields
// (Core/TwoDScene.cpp:5564-5605).
void set_liquid_particle(TwoDScene& s, int i, const double* x3, const double* v3,
                         const double* C9, double fmass, double fvol, double radius) {
  s.m_x.segment<4>(i * 4) = Vector4s(x3[0], x3[1], x3[2], 0.0);
  s.m_rest_x.segment<4>(i * 4) = s.m_x.segment<4>(i * 4);
  s.m_v.segment<4>(i * 4).setZero();
  s.m_dv.segment<4>(i * 4).setZero();
  s.m_fluid_v.segment<4>(i * 4) = Vector4s(v3[0], v3[1], v3[2], 0.0);
  s.m_m.segment<4>(i * 4).setZero();
  s.m_fluid_m.segment<3>(i * 4).setConstant(fmass);
  s.m_fluid_m(i * 4 + 3) = fmass * radius * radius * 0.4;
  s.m_fluid_vol(i) = fvol;
  s.m_vol(i) = 0.0;
  s.m_rest_vol(i) = 0.0;
  s.m_shape_factor(i) = 0.0;
  s.m_radius(i * 2 + 0) = s.m_radius(i * 2 + 1) = radius;
  s.m_volume_fraction(i) = 0.0;
  s.m_rest_volume_fraction(i) = 0.0;
  s.m_fixed[i] = 0U;
  s.m_twist[i] = false;
  s.m_particle_rest_length(i) = radius * 2.0;
  s.m_particle_rest_area(i) = M_PI * radius * radius;
  s.m_particle_group[i] = 0;
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) s.m_fB(i * 3 + r, q) = C9 ? C9[r * 3 + q] : 0.0;
  s.m_B.block<3, 3>(i * 3, 0).setZero();
  s.m_is_strand_tip[i] = false;
  s.m_div[i].resize(0);
  s.m_particle_to_surfel[i] = -1;
  s.m_inside[i] = 0U;
  s.m_classifier[i] = PC_o;
  s.m_orientation.segment<3>(i * 3).setZero();
}

}  // namespace

extern "C" {

// params: dx, g[3], rho, flip, friction, box_c[3], box_half[3], box_r,
// criterion, maxiters, mic
void* wcref_create(double dx, const double* g, double rho, double flip,
                   double friction, const double* box_c,
                   const double* box_half, double box_r, double criterion,
                   int maxiters, int mic, int np, const double* x3,
                   const double* v3, const double* C9, const double* fmass,
                   const double* fvol, const double* radius) {
  Harness* h = new Harness();
  memset(h->timers, 0, sizeof(h->timers));
  Params& p = h->p;
  p.dx = dx;
  for (int r = 0; r < 3; ++r) {
    p.gravity[r] = g[r];
    p.box_center[r] = box_c[r];
    p.box_half[r] = box_half[r];
  }
  p.liquid_density = rho;
  p.flip_coeff = flip;
  p.liquid_boundary_friction = friction;
  p.box_radius = box_r;
  p.criterion = criterion;
  p.maxiters = maxiters;
  p.mic = mic;

  h->scene = std::make_shared<TwoDScene>();
  TwoDScene& s = *h->scene;

  // LiquidInfo defaults of App/TwoDSceneXMLParser.cpp:1851-1904, liquid-only.
  LiquidInfo info;
  info.air_density = 1.2041e-3;
  info.liquid_density = rho;
  info.rest_contact_angle = 40.8 / 180.0 * M_PI;
  info.surf_tension_coeff = 72.8;
  info.yazdchi_power = 1.6;
  info.viscosity = 8.9e-3;
  info.air_viscosity = 1.81e-4;
  info.pore_radius = 0.005;
  info.yarn_diameter = 0.01;
  info.rest_volume_fraction = 0.4;
  info.lambda = 2.0;
  info.cohesion_coeff = 0.002;
  info.correction_step = 8;
  info.correction_multiplier = 2.0;
  info.correction_strength = 0.0;
  info.flip_coeff = flip;
  info.elasto_flip_asym_coeff = 1.0;
  info.elasto_flip_coeff = 0.95;
  info.elasto_advect_coeff = 1.0;
  info.particle_cell_multiplier = 0.3535533906;
  info.bending_scheme = 2;
  info.levelset_young_modulus = 6.6e6;
  info.liquid_boundary_friction = friction;
  info.use_surf_tension = false;
  info.surf_tension_smoothing_step = 7;
  info.use_cohesion = false;
  info.soft_cohesion = false;
  info.solid_cohesion = false;
  info.use_drag = true;
  info.use_nonlinear_drag = true;
  info.solve_solid = false;
  info.apply_pressure_solid = false;
  info.use_levelset_force = false;
  info.use_twist = false;
  info.apply_pressure_manifold = false;
  info.apply_pore_pressure_solid = false;
  info.use_bicgstab = false;
  info.use_amgpcg_solid = false;
  info.use_pcr = true;
  info.propagate_solid_velocity = false;
  info.check_divergence = false;
  info.use_varying_fraction = false;
  info.compute_viscosity = false;
  info.implicit_viscosity = true;
  info.drag_by_future_solid = false;
  info.drag_by_air = false;
  info.init_nonuniform_fraction = false;
  info.use_group_precondition = false;
  info.use_lagrangian_mpm = false;
  info.use_cosolve_angular = false;
  info.levelset_thickness = 0.25;
  info.iteration_print_step = 0;
  info.elasto_capture_rate = 1.0;
  s.setLiquidInfo(info);
  s.setBucketInfo(dx * 4.0, 4, 2);  // kernel order is the constant 2

  // walls: solid box, inside (App/TwoDSceneXMLParser.cpp loadDistanceFields)
  VectorXs par(4);
  par << box_half[0], box_half[1], box_half[2], box_r;
  std::vector<DF_SOURCE_DURATION> dur;
  auto box = std::make_shared<DistanceFieldObject>(
      Vector3s(box_c[0], box_c[1], box_c[2]), par, DFT_BOX, DFU_SOLID, true,
      Vector3s(0, 1, 0), 0.0, 0, 0, false, dur);
  s.m_distance_fields.push_back(box);
  s.resizeGroups(1);
  s.initGroupPos();

  // liquid particles (attribute set of sampleLiquidDistanceFields)
  s.resizeParticleSystem(np);
  s.m_fluids.resize(np);
  for (int i = 0; i < np; ++i) {
    set_liquid_particle(s, i, x3 + i * 3, v3 + i * 3, C9 ? C9 + i * 9 : nullptr, fmass[i],
                        fvol[i], radius[i]);
    s.m_fluids[i] = i;
  }
  s.updateRestPos();

  s.insertForce(std::make_shared<SimpleGravityForce>(
      Vector3s(g[0], g[1], g[2])));

  h->stepper = std::make_shared<LinearizedImplicitEuler>(
      1e-6, criterion, 1e-6, 1e-6, maxiters, 1, 1, 1);
  h->stepper->setUseApic(true);
  return h;
}

void wcref_destroy(void* hp) { delete (Harness*)hp; }

// Number of CFL sub-steps WetClothCore::stepSystem would take for dt
// (Core/WetClothCore.cpp:50-62).
int wcref_num_substeps(void* hp, double dt) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  const scalar max_elasto_vel = s.getMaxVelocity();
  const scalar max_fluid_vel = s.getMaxFluidVelocity();
  const scalar dx = s.getCellSize();
  const scalar max_elasto_dt =
      std::min(dx / std::max(1e-63, max_elasto_vel) / 3.0, 1.0 / 30.0);
  const scalar max_fluid_dt =
      std::min(dx / std::max(1e-63, max_fluid_vel) * 3.0, 1.0 / 30.0);
  const scalar max_dt = std::min(max_elasto_dt, max_fluid_dt);
  return std::max(1, (int)ceil(dt / max_dt));
}

// One sub-step of the fluid hot path, in WetClothCore::stepSystem order.
// snapshot != 0 records every intermediate field.
int wcref_substep(void* hp, double sub_dt, int snapshot) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  LinearizedImplicitEuler& e = *h->stepper;
  double t0 = now(), t1;

  // terminateParticles runs every sub-step (WetClothCore.cpp:97); without a
  // terminator only its removeEmptyParticles can change anything, and only
  // when a liquid particle has no fluid volume
  bool any_empty = false;
  for (int i = s.getNumElastoParticles(); i < s.getNumParticles() && !any_empty; ++i)
    any_empty = s.m_fluid_vol(i) < 1e-20;
  if (h->term_on || any_empty) {
    if (!h->grid_built) {
      // the scene parser builds the grid at load (App/TwoDSceneXMLParser.cpp:725-727)
      s.updateParticleBoundingBox();
      s.rebucketizeParticles();
      s.resampleNodes();
    }
    const int before = s.getNumParticles();
    s.terminateParticles();
    h->ii["terminate_removed"] = {(long long)(before - s.getNumParticles())};
  }
  h->grid_built = true;
  s.updateParticleBoundingBox();
  s.rebucketizeParticles();
  s.resampleNodes();
  t1 = now(); h->timers[1] += t1 - t0; t0 = t1;
  if (snapshot) snap_grid(*h);

  s.computeWeights(sub_dt);
  s.updateLiquidPhi(sub_dt);
  s.updateSolidPhi();
  s.updateSolidWeights();
  s.saveParticleVelocity();
  t1 = now(); h->timers[2] += t1 - t0; t0 = t1;

  s.mapParticleNodesAPIC();
  s.saveFluidVelocity();
  s.mapParticleSaturationPsiNodes();
  s.updatePorePressureNodes();
  t1 = now(); h->timers[3] += t1 - t0; t0 = t1;
  if (snapshot) snap_p2g(*h);

  e.stepVelocity(s, sub_dt);
  t1 = now(); h->timers[4] += t1 - t0; t0 = t1;
  if (snapshot) snap_predict(*h);

  e.projectFine(s, sub_dt);
  if (snapshot) {
    snap_system(*h);
    dense(*h, "pressure_amg", s.m_node_pressure);
    // iteration count of the reference's default solve (printed, not kept, by
    // pressure::solveNodePressure): the same AMGPCGSolveSparse call on the
    // same system (Pressure.cpp:402-436, :797)
    const unsigned n = e.m_fine_pressure_matrix.n;
    if (n > 0 && e.m_fine_pressure_rhs.size() >= n) {
      const Sorter& bk = s.getParticleBuckets();
      const int nc = s.getDefaultNumNodes();
      std::vector<Vector3i> dof_ijk(n);
      const int nb = s.getNumBuckets();
      for (int b = 0; b < nb; ++b) {
        const VectorXi& gi = e.m_fine_global_indices[b];
        const Vector3i hnd = bk.bucket_handle(b);
        for (int i = 0; i < (int)gi.size(); ++i)
          if (gi[i] >= 0) {
            const Vector3i lh = s.getNodeHandle(i);
            dof_ijk[gi[i]] = Vector3i(hnd(0) * nc + lh(0), hnd(1) * nc + lh(1), hnd(2) * nc + lh(2));
          }
      }
      std::vector<double> rhs(e.m_fine_pressure_rhs.begin(), e.m_fine_pressure_rhs.begin() + n);
      std::vector<double> result(n, 0.0);
      double res = 0;
      int iters = 0;
      AMGPCGSolveSparse(e.m_fine_pressure_matrix, rhs, result, dof_ijk, h->p.criterion,
                        h->p.maxiters, res, iters, bk.ni * nc, bk.nj * nc, bk.nk * nc);
      h->last_iters_amg = iters;
      h->last_res_amg = res;
    }
  }
  if (h->p.mic) {
    const unsigned n = e.m_fine_pressure_matrix.n;
    if (n > 0 && e.m_fine_pressure_rhs.size() >= n) {
      robertbridson::PCGSolver<double> solver;
      solver.set_solver_parameters(h->p.criterion, h->p.maxiters, 0.97, 0.25);
      std::vector<double> rhs(e.m_fine_pressure_rhs.begin(),
                              e.m_fine_pressure_rhs.begin() + n);
      std::vector<double> result(n, 0.0);
      double res = 0;
      int iters = 0;
      solver.solve(e.m_fine_pressure_matrix, rhs, result, res, iters);
      h->last_iters_mic = iters;
      h->last_res_mic = res;
      const int nb = s.getNumBuckets();
      for (int b = 0; b < nb; ++b) {
        const VectorXi& gi = e.m_fine_global_indices[b];
        for (int i = 0; i < (int)gi.size(); ++i)
          if (gi[i] >= 0) s.m_node_pressure[b][i] = result[gi[i]];
      }
    }
  }
  t1 = now(); h->timers[5] += t1 - t0; t0 = t1;
  if (snapshot) dense(*h, "pressure", s.m_node_pressure);

  e.applyPressureDragFluid(s, sub_dt);
  e.acceptVelocity(s);
  t1 = now(); h->timers[7] += t1 - t0; t0 = t1;
  if (snapshot) {
    dense_uc(*h, "valid_x", s.m_node_liquid_valid_x);
    dense_uc(*h, "valid_y", s.m_node_liquid_valid_y);
    dense_uc(*h, "valid_z", s.m_node_liquid_valid_z);
    dense(*h, "u_proj_x", s.m_node_vel_fluid_x);
    dense(*h, "u_proj_y", s.m_node_vel_fluid_y);
    dense(*h, "u_proj_z", s.m_node_vel_fluid_z);
  }

  s.constrainLiquidVelocity();
  t1 = now(); h->timers[8] += t1 - t0; t0 = t1;
  if (snapshot) {
    dense(*h, "u_final_x", s.m_node_vel_fluid_x);
    dense(*h, "u_final_y", s.m_node_vel_fluid_y);
    dense(*h, "u_final_z", s.m_node_vel_fluid_z);
  }

  {
    // correctLiquidParticles runs in every sub-step (WetClothCore.cpp:242); at
    // correction_strength 0 its spring weights vanish and it only projects
    // its particle subset out of the solid.  The subset is one rand() draw
    // modulo correction_step: rand() is seeded so that the draw equals the
    // selector of the seeded stream the oracle and the GPU use
    const int step = std::max(1, s.getLiquidInfo().correction_step);
    const int want = seeded_selector(h->corr_seed, h->corr_count++, step);
    unsigned seed = 0;
    while (seed < (1u << 24)) {
      srand(seed);
      if (rand() % step == want) break;
      ++seed;
    }
    srand(seed);
    s.correctLiquidParticles(sub_dt);
    h->ii["correction_selector"] = {want};
    if (snapshot) snap_particles(*h, "corr_");
  }

  s.mapNodeParticlesAPIC();
  t1 = now(); h->timers[9] += t1 - t0; t0 = t1;
  if (snapshot) snap_particles(*h, "g2p_");

  e.advectScene(s, sub_dt);
  s.solidProjection(sub_dt);
  t1 = now(); h->timers[10] += t1 - t0; t0 = t1;
  if (snapshot) snap_particles(*h, "adv_");
  return 0;
}

// Full step: CFL sub-stepping as WetClothCore::stepSystem.
int wcref_step(void* hp, double dt, int snapshot) {
  const int n = wcref_num_substeps(hp, dt);
  const double sub_dt = dt / (double)n;
  for (int k = 0; k < n; ++k) wcref_substep(hp, sub_dt, snapshot);
  return n;
}

long long wcref_size(void* hp, const char* name) {
  Harness* h = (Harness*)hp;
  auto it = h->f.find(name);
  if (it != h->f.end()) return (long long)it->second.size();
  auto jt = h->ii.find(name);
  if (jt != h->ii.end()) return (long long)jt->second.size();
  return -1;
}

int wcref_get_f(void* hp, const char* name, double* out) {
  Harness* h = (Harness*)hp;
  auto it = h->f.find(name);
  if (it == h->f.end()) return -1;
  memcpy(out, it->second.data(), it->second.size() * sizeof(double));
  return 0;
}

int wcref_get_i(void* hp, const char* name, long long* out) {
  Harness* h = (Harness*)hp;
  auto it = h->ii.find(name);
  if (it == h->ii.end()) return -1;
  memcpy(out, it->second.data(), it->second.size() * sizeof(long long));
  return 0;
}

void wcref_solver_stats(void* hp, int* iters_mic, double* res_mic) {
  Harness* h = (Harness*)hp;
  *iters_mic = h->last_iters_mic;
  *res_mic = h->last_res_mic;
}

// explicit liquid viscosity: LiquidInfo::compute_viscosity on, implicit off,
// viscosity mu, LinearizedImplicitEuler's viscosity sub-steps (call before
// the first step; mu = 0 turns it off)
void wcref_set_viscosity(void* hp, double mu, int substeps) {
  Harness* h = (Harness*)hp;
  LiquidInfo& li = h->scene->getLiquidInfo();
  li.compute_viscosity = mu > 0.0;
  li.implicit_viscosity = false;
  li.viscosity = mu;
  // the sub-step count is a constructor argument of the stepper
  h->stepper = std::make_shared<LinearizedImplicitEuler>(
      1e-6, h->p.criterion, 1e-6, 1e-6, h->p.maxiters, 1, substeps > 0 ? substeps : 1, 1);
  h->stepper->setUseApic(true);
}

// TwoDScene::updateOptiVolume and mergeLiquidParticles, as
// WetClothCore::stepSystem runs them before a step's grid build (the bucket
// lists are the last step's), with LiquidInfo correction_step = step.
// srand(seed) fixes the merge's rand() draws (the subset selector, then three
// Fisher-Yates colour permutations), which are replayed and recorded
// ("merge_selector", "merge_perm" t, s, r).  Returns the particles removed.
int wcref_merge(void* hp, unsigned seed, int step) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  s.getLiquidInfo().correction_step = step > 0 ? step : 1;
  s.updateOptiVolume();
  srand(seed);
  const int sel = rand() % s.getLiquidInfo().correction_step;
  std::vector<int> pt, ps, pr;
  mathutils::fisherYates(3, pt);
  mathutils::fisherYates(3, ps);
  mathutils::fisherYates(3, pr);
  srand(seed);
  const int before = s.getNumParticles();
  s.mergeLiquidParticles();
  h->ii["merge_selector"] = {sel};
  h->ii["merge_perm"] = {pt[0], pt[1], pt[2], ps[0], ps[1], ps[2], pr[0], pr[1], pr[2]};
  snap_particles(*h, "merge_");
  const int np = s.getNumParticles();
  std::vector<double>& vol = h->f["merge_vol"];
  std::vector<double>& mass = h->f["merge_mass"];
  std::vector<double>& rad = h->f["merge_radius"];
  std::vector<long long>& cls = h->ii["merge_class"];
  vol.assign(np, 0.0);
  mass.assign(np, 0.0);
  rad.assign(np, 0.0);
  cls.assign(np, 0);
  for (int i = 0; i < np; ++i) {
    vol[i] = s.m_fluid_vol(i);
    mass[i] = s.m_fluid_m(i * 4);
    rad[i] = s.m_radius(i * 2);
    cls[i] = (long long)s.m_classifier[i];
  }
  return before - np;
}

// A terminator box (DFT_BOX, DFU_TERMINATOR) in a distance-field group of its
// own (group 1: the group's union operator votes the terminator usage); the
// groups are rebuilt around it (TwoDScene::resizeGroups, initGroupPos), and
// each sub-step then starts with terminateParticles.
void wcref_set_terminator(void* hp, const double* c, const double* half, double radius,
                          int inside) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  VectorXs par(4);
  par << half[0], half[1], half[2], radius;
  std::vector<DF_SOURCE_DURATION> dur;
  auto term = std::make_shared<DistanceFieldObject>(
      Vector3s(c[0], c[1], c[2]), par, DFT_BOX, DFU_TERMINATOR, inside != 0,
      Vector3s(0, 1, 0), 0.0, 1, 0, false, dur);
  s.m_distance_fields.push_back(term);
  for (auto& df : s.m_distance_fields) df->parent.reset();
  s.resizeGroups(2);
  s.initGroupPos();
  // the scene parser builds the grid at load (App/TwoDSceneXMLParser.cpp:725-727),
  // so the first terminateParticles re-sorts valid bucket lists
  s.updateParticleBoundingBox();
  s.rebucketizeParticles();
  s.resampleNodes();
  h->term_on = true;
  h->grid_built = true;
}

// One terminator DistanceFieldObject of any of the four analytic types
// (0 box, 1 sphere, 2 capsule, 3 cylinder; DistanceFields.cpp:477-520), built
// as the scene parser builds it from its rotation axis and angle, in
// distance-field group `group` (>= 1; groups are unions).  rot_out receives
// the rotation quaternion the object holds (w, x, y, z).
void wcref_add_terminator(void* hp, int type, int inside, const double* c, const double* axis,
                          double angle, const double* par4, int group, double* rot_out) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  VectorXs par(4);
  par << par4[0], par4[1], par4[2], par4[3];
  static const DISTANCE_FIELD_TYPE types[4] = {DFT_BOX, DFT_SPHERE, DFT_CAPSULE, DFT_CYLINDER};
  std::vector<DF_SOURCE_DURATION> dur;
  auto term = std::make_shared<DistanceFieldObject>(
      Vector3s(c[0], c[1], c[2]), par, types[type], DFU_TERMINATOR, inside != 0,
      Vector3s(axis[0], axis[1], axis[2]), angle, group, 0, false, dur);
  rot_out[0] = term->rot.w();
  rot_out[1] = term->rot.x();
  rot_out[2] = term->rot.y();
  rot_out[3] = term->rot.z();
  s.m_distance_fields.push_back(term);
  int ngroups = 1;
  for (auto& df : s.m_distance_fields) {
    df->parent.reset();
    ngroups = std::max(ngroups, df->group + 1);
  }
  s.resizeGroups(ngroups);
  s.initGroupPos();
  if (!h->grid_built) {
    s.updateParticleBoundingBox();
    s.rebucketizeParticles();
    s.resampleNodes();
    h->grid_built = true;
  }
  h->term_on = true;
}

// TwoDScene::terminateParticles: liquid particles inside the terminator's
// negative region lose their volume and removeEmptyParticles drops them.
// Returns the particles removed.
int wcref_terminate(void* hp) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  const int before = s.getNumParticles();
  s.terminateParticles();
  snap_particles(*h, "term_");
  return before - s.getNumParticles();
}

// The inputs of the reference's split placement: the sphere-pattern table
// TwoDScene::m_sphere_pattern[n] for n = 2..32 (3n doubles each, concatenated
// into `pattern`) and the Q of the QR decomposition of each Matrix3s::Random()
// that splitLiquidParticles (TwoDScene.cpp:2362-2480, serial build) draws
// after srand(seed), one per splitting parent in fluid-index order, row
// major.  Call before wcref_split with the same seed.  Returns the number of
// splitting parents (rotations written up to `max`).
int wcref_split_inputs(void* hp, unsigned seed, double* pattern, double* rot, int max) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  s.updateOptiVolume();
  int off = 0;
  for (int n = 2; n <= 32; ++n)
    for (int i = 0; i < 3 * n; ++i) pattern[off++] = s.m_sphere_pattern[n](i);
  const scalar rad_fine = mathutils::defaultRadiusMultiplier() * s.getCellSize() *
                          s.getLiquidInfo().particle_cell_multiplier;
  const scalar V_fine = 4.0 / 3.0 * M_PI * rad_fine * rad_fine * rad_fine;
  srand(seed);
  int k = 0;
  const int nf = s.getNumFluidParticles();
  for (int fidx = 0; fidx < nf; ++fidx) {
    const int pidx = s.m_fluids[fidx];
    if (s.m_classifier[pidx] != PC_L) continue;
    const int n_split = std::min((int)ceil(s.m_fluid_vol(pidx) / V_fine), 32);
    if (n_split <= 1) continue;
    Matrix3s M = Matrix3s::Random();
    Matrix3s Q, R;
    mathutils::QRDecompose<scalar, 3>(M, Q, R);
    if (k < max)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) rot[k * 9 + a * 3 + b] = Q(a, b);
    ++k;
  }
  return k;
}

// TwoDScene::updateOptiVolume and splitLiquidParticles, as
// WetClothCore::stepSystem runs them before a step's grid build; the
// children's rotations come from Matrix3s::Random() (rand()), seeded by
// srand(seed).  Returns the particles added.
int wcref_split(void* hp, unsigned seed) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  s.updateOptiVolume();
  srand(seed);
  const int before = s.getNumParticles();
  s.splitLiquidParticles();
  snap_particles(*h, "split_");
  const int np = s.getNumParticles();
  std::vector<double>& vol = h->f["split_vol"];
  std::vector<double>& mass = h->f["split_mass"];
  std::vector<double>& rad = h->f["split_radius"];
  std::vector<long long>& cls = h->ii["split_class"];
  vol.assign(np, 0.0);
  mass.assign(np, 0.0);
  rad.assign(np, 0.0);
  cls.assign(np, 0);
  for (int i = 0; i < np; ++i) {
    vol[i] = s.m_fluid_vol(i);
    mass[i] = s.m_fluid_m(i * 4);
    rad[i] = s.m_radius(i * 2);
    cls[i] = (long long)s.m_classifier[i];
  }
  return np - before;
}

// implicit liquid viscosity: LiquidInfo::compute_viscosity and
// implicit_viscosity on, viscosity mu, the stepper's viscosity sub-steps and
// viscous criterion (call before the first step)
void wcref_set_viscosity_implicit(void* hp, double mu, int substeps, double criterion) {
  Harness* h = (Harness*)hp;
  LiquidInfo& li = h->scene->getLiquidInfo();
  li.compute_viscosity = mu > 0.0;
  li.implicit_viscosity = true;
  li.viscosity = mu;
  h->stepper = std::make_shared<LinearizedImplicitEuler>(
      1e-6, h->p.criterion, 1e-6, criterion, h->p.maxiters, 1, substeps > 0 ? substeps : 1, 1);
  h->stepper->setUseApic(true);
}

// Elasto (cloth/yarn) particles: the scene's particles become [0, ne) elasto
// followed by the current liquid particles (TwoDScene::isFluid :6921,
// getNumElastoParticles :5212-5217).  Per particle: x4/v4 (position, velocity
// and twist), B9 (row-major affine matrix m_B), m4/fm4 (m_m, m_fluid_m),
// m_rest_vol, m_rest_volume_fraction, m_fluid_vol, m_shape_factor,
// m_orientation (3), surfel (m_particle_to_surfel >= 0 when nonzero; only its
// sign is read on the hot path), radius.  Call before the first step.
void wcref_set_elasto(void* hp, int ne, const double* x4, const double* v4, const double* B9,
                      const double* m4, const double* fm4, const double* rest_vol,
                      const double* rest_vf, const double* fluid_vol, const double* shape_factor,
                      const double* orient3, const int* surfel, const double* radius) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  const int nl = (int)s.m_fluids.size();
  std::vector<double> lx(nl * 3), lv(nl * 3), lC(nl * 9), lm(nl), lvol(nl), lr(nl);
  for (int k = 0; k < nl; ++k) {
    const int i = s.m_fluids[k];
    for (int r = 0; r < 3; ++r) {
      lx[k * 3 + r] = s.m_x(i * 4 + r);
      lv[k * 3 + r] = s.m_fluid_v(i * 4 + r);
      for (int q = 0; q < 3; ++q) lC[k * 9 + r * 3 + q] = s.m_fB(i * 3 + r, q);
    }
    lm[k] = s.m_fluid_m(i * 4);
    lvol[k] = s.m_fluid_vol(i);
    lr[k] = s.m_radius(i * 2);
  }
  s.resizeParticleSystem(ne + nl);
  s.m_fluids.resize(nl);
  for (int i = 0; i < ne; ++i) {
    s.m_x.segment<4>(i * 4) = Vector4s(x4[i * 4], x4[i * 4 + 1], x4[i * 4 + 2], x4[i * 4 + 3]);
    s.m_rest_x.segment<4>(i * 4) = s.m_x.segment<4>(i * 4);
    s.m_v.segment<4>(i * 4) = Vector4s(v4[i * 4], v4[i * 4 + 1], v4[i * 4 + 2], v4[i * 4 + 3]);
    s.m_dv.segment<4>(i * 4).setZero();
    s.m_fluid_v.segment<4>(i * 4).setZero();
    s.m_m.segment<4>(i * 4) = Vector4s(m4[i * 4], m4[i * 4 + 1], m4[i * 4 + 2], m4[i * 4 + 3]);
    s.m_fluid_m.segment<4>(i * 4) =
        Vector4s(fm4[i * 4], fm4[i * 4 + 1], fm4[i * 4 + 2], fm4[i * 4 + 3]);
    s.m_vol(i) = rest_vol[i];
    s.m_rest_vol(i) = rest_vol[i];
    s.m_fluid_vol(i) = fluid_vol[i];
    s.m_shape_factor(i) = shape_factor[i];
    s.m_radius(i * 2 + 0) = s.m_radius(i * 2 + 1) = radius[i];
    s.m_volume_fraction(i) = rest_vf[i];
    s.m_rest_volume_fraction(i) = rest_vf[i];
    s.m_fixed[i] = 0U;
    s.m_twist[i] = false;
    s.m_particle_rest_length(i) = radius[i] * 2.0;
    s.m_particle_rest_area(i) = M_PI * radius[i] * radius[i];
    s.m_particle_group[i] = 0;
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) s.m_B(i * 3 + r, q) = B9[i * 9 + r * 3 + q];
    s.m_fB.block<3, 3>(i * 3, 0).setZero();
    s.m_is_strand_tip[i] = false;
    s.m_div[i].resize(0);
    s.m_particle_to_surfel[i] = surfel[i] ? i : -1;
    s.m_inside[i] = 0U;
    s.m_classifier[i] = PC_NONE;
    s.m_orientation.segment<3>(i * 3) =
        Vector3s(orient3[i * 3], orient3[i * 3 + 1], orient3[i * 3 + 2]);
  }
  for (int k = 0; k < nl; ++k) {
    set_liquid_particle(s, ne + k, &lx[k * 3], &lv[k * 3], &lC[k * 9], lm[k], lvol[k], lr[k]);
    s.m_fluids[k] = ne + k;
  }
  s.updateRestPos();
}

// LiquidInfo::elasto_flip_coeff, elasto_flip_asym_coeff, elasto_advect_coeff
void wcref_set_elasto_coeffs(void* hp, double flip, double asym, double advect) {
  LiquidInfo& li = ((Harness*)hp)->scene->getLiquidInfo();
  li.elasto_flip_coeff = flip;
  li.elasto_flip_asym_coeff = asym;
  li.elasto_advect_coeff = advect;
}

// The transfers alone, in WetClothCore::stepSystem order with the solve left
// out: grid, weights, APIC P2G (+ saturation/psi/pore pressure), then G2P
// straight from the P2G node velocities and advection.  Snapshots as in a
// step ("g2p_" / "adv_" particle tags).
int wcref_transfer(void* hp, double dt) {
  Harness* h = (Harness*)hp;
  TwoDScene& s = *h->scene;
  LinearizedImplicitEuler& e = *h->stepper;
  s.updateParticleBoundingBox();
  s.rebucketizeParticles();
  s.resampleNodes();
  snap_grid(*h);
  s.computeWeights(dt);
  s.updateLiquidPhi(dt);
  s.updateSolidPhi();
  s.updateSolidWeights();
  s.saveParticleVelocity();
  s.mapParticleNodesAPIC();
  s.saveFluidVelocity();
  s.mapParticleSaturationPsiNodes();
  s.updatePorePressureNodes();
  snap_p2g(*h);
  s.mapNodeParticlesAPIC();
  snap_particles(*h, "g2p_");
  e.advectScene(s, dt);
  s.solidProjection(dt);
  snap_particles(*h, "adv_");
  return 0;
}

// LiquidInfo correction_strength, correction_step and correction_multiplier
// of TwoDScene::correctLiquidParticles (run in every sub-step between
// constrainLiquidVelocity and G2P, as WetClothCore::stepSystem runs it; at
// strength 0 it only projects its subset out of the solid); the k-th call
// corrects the subset of call k of the seeded stream of `seed`
void wcref_set_correction(void* hp, double strength, int step, double multiplier,
                          unsigned seed) {
  Harness* h = (Harness*)hp;
  LiquidInfo& li = h->scene->getLiquidInfo();
  li.correction_strength = strength;
  li.correction_step = step > 0 ? step : 1;
  li.correction_multiplier = multiplier;
  h->corr_seed = seed;
  h->corr_count = 0;
}

// AMGPCGSolveSparse iterations and residual of the last snapshot step
void wcref_amg_stats(void* hp, int* iters, double* res) {
  Harness* h = (Harness*)hp;
  *iters = h->last_iters_amg;
  *res = h->last_res_amg;
}

// cumulative phase timers (seconds), slots as WetClothCore timing_buffer
void wcref_timers(void* hp, double* out12) {
  memcpy(out12, ((Harness*)hp)->timers, sizeof(double) * 12);
}

int wcref_num_particles(void* hp) {
  return ((Harness*)hp)->scene->getNumParticles();
}

// LiquidInfo::particle_cell_multiplier (V_fine of updateOptiVolume's classes)
void wcref_set_cell_multiplier(void* hp, double m) {
  ((Harness*)hp)->scene->getLiquidInfo().particle_cell_multiplier = m;
}

// The reference's own WetClothCore::stepSystem (WetClothCore.cpp:45-330) on
// the harness's scene, instead of the harness's staged replay; snapshots the
// particle state (adv_x, g2p_v, g2p_C) afterwards.
void wcref_core_step(void* hp, double dt) {
  Harness* h = (Harness*)hp;
  WetClothCore core(h->scene, h->stepper);
  core.stepSystem(dt);
  snap_particles(*h, "adv_");
  snap_particles(*h, "g2p_");
}

// The scene objects of a harness (shared_ptr<TwoDScene>,
// shared_ptr<LinearizedImplicitEuler>), for code that drives them itself: the
// compiled GpuWetClothCore binding test steps them with WetClothCore.
const void* wcref_scene_sp(void* hp) { return &((Harness*)hp)->scene; }
const void* wcref_stepper_sp(void* hp) { return &((Harness*)hp)->stepper; }

// robertbridson::PCGSolver<double>::solve on a matrix given in CSR form: the
// rows become a SparseMatrix (set_element keeps each row's columns sorted),
// set_solver_parameters(tolerance, maxiter, 0.97, 0.25).  Returns the
// solver's bool; x, *res and *iters as it leaves them.
int wcref_pcg_solve_csr(const long long* rowstart, const long long* col, const double* val,
                        int n, const double* rhs, double* x, double tolerance, int maxiter,
                        double* res, int* iters) {
  robertbridson::SparseMatrix<double> A((unsigned)n);
  for (int i = 0; i < n; ++i)
    for (long long p = rowstart[i]; p < rowstart[i + 1]; ++p)
      A.set_element((unsigned)i, (unsigned)col[p], val[p]);
  robertbridson::PCGSolver<double> solver;
  solver.set_solver_parameters(tolerance, maxiter, 0.97, 0.25);
  std::vector<double> b(rhs, rhs + n), out(n, 0.0);
  double r = 0;
  int it = 0;
  const bool ok = solver.solve(A, b, out, r, it);
  for (int i = 0; i < n; ++i) x[i] = out[i];
  *res = r;
  *iters = it;
  return ok ? 1 : 0;
}

}  // extern "C"
