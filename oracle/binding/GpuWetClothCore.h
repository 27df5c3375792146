// GpuWetClothCore: a WetClothCore whose liquid step runs on libwcgpu (one B200).
//
// This is the reference-side binding: a maintainer adds this header to
// libWetCloth/Core/ and links -lwcgpu.  WetClothCore::stepSystem is virtual
// (libWetCloth/Core/WetClothCore.h:38), so a scene loader that constructs a
// GpuWetClothCore instead of a WetClothCore (same constructor arguments plus
// the integrator's pressure criterion, iteration limit and solver) runs the
// liquid step of WetClothCore.cpp:45-330 -- terminateParticles, particle
// maintenance, the grid, both transfers, stepVelocity, projectFine,
// applyPressureDragFluid, constrainLiquidVelocity, correctLiquidParticles,
// advectScene and solidProjection -- as one wcg_step per call, with the
// particle state resident on the GPU between steps.  syncToScene() copies
// positions, velocities and affine matrices back into the TwoDScene when the
// caller needs them (output, rendering, handing back to the CPU core).
//
// Scope: liquid-only scenes (no cloth or yarn particles) whose solids are one
// box distance field holding the fluid (DFT_BOX, DFU_SOLID, inside, not
// rotated or moving) and whose forces on the liquid are SimpleGravityForce
// terms.  Anything else is refused with std::runtime_error at the first step.
//
// The same file is compiled against the reference headers and stepped beside
// the reference's own WetClothCore::stepSystem by the tests
// (oracle/binding/binding_harness.cpp, tests/test_gpu_binding.py).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "DistanceFields.h"
#include "SimpleGravityForce.h"
#include "TwoDScene.h"
#include "WetClothCore.h"
#include "wetcloth_gpu.h"

// Three members have no public accessor in the reference: TwoDScene::m_fB
// (TwoDScene.h:959), TwoDScene::m_forces (:1192) and
// SimpleGravityForce::m_gravity (SimpleGravityForce.h:59).  A maintainer adds
// the one-line accessors getFluidB(), getForces() and getGravity() next to
// them; a translation unit that is compiled with access to the members
// defines WCG_BINDING_MEMBER_ACCESS instead.
namespace wcgbind {
#ifdef WCG_BINDING_MEMBER_ACCESS
inline MatrixXs& fluidB(TwoDScene& s) { return s.m_fB; }
inline const std::vector<std::shared_ptr<Force> >& forces(const TwoDScene& s) {
  return s.m_forces;
}
inline Vector3s gravity(const SimpleGravityForce& f) { return f.m_gravity; }
#else
inline MatrixXs& fluidB(TwoDScene& s) { return s.getFluidB(); }
inline const std::vector<std::shared_ptr<Force> >& forces(const TwoDScene& s) {
  return s.getForces();
}
inline Vector3s gravity(const SimpleGravityForce& f) { return f.getGravity(); }
#endif
}  // namespace wcgbind

// What the scene file gives the integrator (App/TwoDSceneXMLParser.cpp:3240-3280)
// and the choice of pressure solver.
struct GpuStepOptions {
  double criterion = 1e-6;        // pressure criterion: ||r||_inf <= c ||b||_inf
  int maxiters = 100;             // the integrator's iteration limit
  int solver = WCG_SOLVER_MG;     // multigrid-PCG, as solveNodePressure (Pressure.cpp:797)
  int precision = WCG_FP64;       // or WCG_FP32_REFINE
  unsigned long long seed = 0;    // seeded draws of correction / merge / split
};

class GpuWetClothCore : public WetClothCore {
 public:
  GpuWetClothCore(const std::shared_ptr<TwoDScene>& scene,
                  const std::shared_ptr<SceneStepper>& stepper,
                  const GpuStepOptions& opt = GpuStepOptions())
      : WetClothCore(scene, stepper), opt_(opt) {}
  ~GpuWetClothCore() override {
    if (ctx_) wcg_destroy(ctx_);
  }

  void stepSystem(const scalar& dt) override {
    TwoDScene& s = *getScene();
    if (!ctx_) create(s);
    int substeps = 0;
    check(wcg_step(ctx_, dt, &substeps));
    last_substeps_ = substeps;
    dirty_ = true;
  }

  // Copies the GPU state into the TwoDScene (m_x, m_fluid_v, m_fB); with the
  // terminator, split or merge the particle count changes, and the scene's
  // arrays are resized to it first.
  void syncToScene() {
    if (!dirty_) return;
    TwoDScene& s = *getScene();
    const long long n = wcg_num_particles(ctx_);
    std::vector<double> x(3 * n), v(3 * n), C(9 * n), x4(4 * n), r(n);
    check(wcg_download_liquid(ctx_, x.data(), v.data(), C.data()));
    if (n != s.getNumParticles()) {
      s.conservativeResizeParticles((int)n);
      s.getFluidIndices().resize(n);
      for (long long i = 0; i < n; ++i) s.getFluidIndices()[i] = (int)i;
    }
    MatrixXs& fB = wcgbind::fluidB(s);
    for (long long i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a) {
        s.getX()(4 * i + a) = x[3 * i + a];
        s.getFluidV()(4 * i + a) = v[3 * i + a];
        for (int b = 0; b < 3; ++b) fB(3 * i + a, b) = C[9 * i + 3 * a + b];
      }
    }
    dirty_ = false;
  }

  int lastSubsteps() const { return last_substeps_; }
  wcg_ctx* context() const { return ctx_; }

 private:
  void create(TwoDScene& s) {
    if (s.getNumElastoParticles() > 0)
      throw std::runtime_error("GpuWetClothCore: scenes with cloth or yarn particles are not "
                               "bound here (use the wcg_upload_elasto path)");
    const LiquidInfo& li = s.getLiquidInfo();
    wcg_params p;
    wcg_default_params(&p);
    p.dx = s.getCellSize();
    p.liquid_density = li.liquid_density;
    p.flip_coeff = li.flip_coeff;
    p.liquid_boundary_friction = li.liquid_boundary_friction;
    p.criterion = opt_.criterion;
    p.maxiters = opt_.maxiters;
    p.solver = opt_.solver;
    p.precision = opt_.precision;
    p.elasto_flip_coeff = li.elasto_flip_coeff;
    p.elasto_flip_asym_coeff = li.elasto_flip_asym_coeff;
    p.elasto_advect_coeff = li.elasto_advect_coeff;
    p.drag_viscosity = li.viscosity;
    if (li.compute_viscosity) {
      p.viscosity = li.viscosity;
      p.viscosity_implicit = li.implicit_viscosity ? 1 : 0;
    }
    // the particle maintenance of every sub-step (WetClothCore.cpp:97-110,
    // 242): the reference draws its subsets with rand(), this library from
    // seeded streams
    p.correction_strength = li.correction_strength;
    p.correction_step = li.correction_step;
    p.correction_multiplier = li.correction_multiplier;
    p.correction_seed = opt_.seed;
    p.particle_cell_multiplier = li.particle_cell_multiplier;
    p.particle_merge = 1;
    p.merge_seed = opt_.seed ^ 0x6d657267ull;
    p.particle_split = 1;
    p.split_seed = opt_.seed ^ 0x73706c74ull;
    fillGravityAndBox(s, &p);
    check(wcg_create(&p, &ctx_));
    setTerminators(s);
    const long long n = s.getNumFluidParticles();
    std::vector<double> x(3 * n), v(3 * n), C(9 * n), m(n), vol(n), r(n);
    const MatrixXs& fB = wcgbind::fluidB(s);
    for (long long i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a) {
        x[3 * i + a] = s.getX()(4 * i + a);
        v[3 * i + a] = s.getFluidV()(4 * i + a);
        for (int b = 0; b < 3; ++b) C[9 * i + 3 * a + b] = fB(3 * i + a, b);
      }
      m[i] = s.getFluidM()(4 * i);
      vol[i] = s.getFluidVol()(i);
      r[i] = s.getRadius()(2 * i);
    }
    check(wcg_upload_liquid(ctx_, n, x.data(), v.data(), C.data(), m.data(), vol.data(),
                            r.data()));
  }

  // the scene's terminator objects (usage DFU_TERMINATOR, analytic shapes,
  // fixed), which terminateParticles removes the liquid with
  // (TwoDScene.cpp:1756-1771); the groups they sit in are unions
  void setTerminators(const TwoDScene& s) {
    std::vector<wcg_shape> shapes;
    for (const std::shared_ptr<DistanceField>& df : s.getDistanceFields()) {
      if (df->usage != DFU_TERMINATOR) continue;
      const auto obj = std::dynamic_pointer_cast<DistanceFieldObject>(df);
      int type = -1;
      if (obj) {
        switch (obj->type) {
          case DFT_BOX: type = WCG_SHAPE_BOX; break;
          case DFT_SPHERE: type = WCG_SHAPE_SPHERE; break;
          case DFT_CAPSULE: type = WCG_SHAPE_CAPSULE; break;
          case DFT_CYLINDER: type = WCG_SHAPE_CYLINDER; break;
          default: break;
        }
      }
      if (type < 0 || obj->V.squaredNorm() != 0.0 || obj->omega.squaredNorm() != 0.0)
        throw std::runtime_error("GpuWetClothCore: terminators other than fixed boxes, "
                                 "spheres, capsules and cylinders are not bound here");
      wcg_shape sh;
      sh.type = type;
      sh.inside = obj->sign < 0.0 ? 1 : 0;
      for (int a = 0; a < 3; ++a) sh.center[a] = obj->center(a);
      sh.rot[0] = obj->rot.w();
      sh.rot[1] = obj->rot.x();
      sh.rot[2] = obj->rot.y();
      sh.rot[3] = obj->rot.z();
      for (int a = 0; a < 4; ++a) sh.param[a] = a < obj->parameter.size() ? obj->parameter(a) : 0.0;
      shapes.push_back(sh);
    }
    if (shapes.size() > WCG_MAX_TERMINATOR_SHAPES)
      throw std::runtime_error("GpuWetClothCore: more terminators than the library takes");
    if (!shapes.empty())
      check(wcg_set_terminators(ctx_, (int)shapes.size(), shapes.data()));
  }

  // gravity: the sum of the scene's SimpleGravityForce terms (each adds
  // m g to the liquid's node momentum, SimpleGravityForce.cpp:25); walls: the
  // one solid box distance field with the fluid inside
  static void fillGravityAndBox(const TwoDScene& s, wcg_params* p) {
    for (int a = 0; a < 3; ++a) p->gravity[a] = 0.0;
    for (const std::shared_ptr<Force>& f : wcgbind::forces(s)) {
      const auto g = std::dynamic_pointer_cast<SimpleGravityForce>(f);
      if (!g) continue;  // forces on elasto particles only
      const Vector3s gv = wcgbind::gravity(*g);
      for (int a = 0; a < 3; ++a) p->gravity[a] += gv(a);
    }
    int boxes = 0;
    for (const std::shared_ptr<DistanceField>& df : s.getDistanceFields()) {
      if (df->usage != DFU_SOLID) continue;
      const auto obj = std::dynamic_pointer_cast<DistanceFieldObject>(df);
      if (!obj || obj->type != DFT_BOX || obj->sign > 0.0 ||
          obj->rot.coeffs() != Eigen::Quaternion<scalar>::Identity().coeffs() ||
          obj->V.squaredNorm() != 0.0 || obj->omega.squaredNorm() != 0.0)
        throw std::runtime_error("GpuWetClothCore: solids other than one fixed box holding "
                                 "the fluid are not bound here");
      if (++boxes > 1)
        throw std::runtime_error("GpuWetClothCore: more than one solid box");
      for (int a = 0; a < 3; ++a) {
        p->box_center[a] = obj->center(a);
        p->box_half[a] = obj->parameter(a);
      }
      p->box_radius = obj->parameter(3);
      p->walls = 1;
    }
    if (boxes == 0) p->walls = 0;
  }

  static void check(int rc) {
    if (rc != WCG_OK) throw std::runtime_error(std::string("libwcgpu: ") + wcg_last_error());
  }

  GpuStepOptions opt_;
  wcg_ctx* ctx_ = nullptr;
  bool dirty_ = false;
  int last_substeps_ = 0;
};
