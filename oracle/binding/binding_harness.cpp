// Test harness of the compiled reference-side binding (GpuWetClothCore.h).
// TEST INFRASTRUCTURE ONLY.  Built by oracle/ref.mk into
// oracle/_ref/libwcbinding.so, linked against the reference Core of
// oracle/_ref/libwcref.so and against libwcgpu.so.
//
// It takes two reference scenes built from the same inputs by the reference
// harness (oracle/ref_harness.cpp), steps the first with the reference's own
// WetClothCore::stepSystem (libWetCloth/Core/WetClothCore.cpp:45-330) and the
// second with GpuWetClothCore::stepSystem, then returns both scenes' liquid
// state as the reference stores it (m_x, m_fluid_v, m_fB).
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stack>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include "AlgebraicMultigrid.h"
#include "MathDefs.h"
#include <Eigen/Geometry>
#define private public
#define protected public
#include "DistanceFields.h"
#include "LinearizedImplicitEuler.h"
#include "SimpleGravityForce.h"
#include "TwoDScene.h"
#include "WetClothCore.h"
#undef private
#undef protected
#define WCG_BINDING_MEMBER_ACCESS
#include "GpuWetClothCore.h"

extern "C" {
const void* wcref_scene_sp(void* hp);
const void* wcref_stepper_sp(void* hp);
}

namespace {

void store(TwoDScene& s, double* out) {
  const long long n = s.getNumParticles();
  const MatrixXs& fB = wcgbind::fluidB(s);
  for (long long i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      out[3 * i + a] = s.getX()(4 * i + a);
      out[3 * n + 3 * i + a] = s.getFluidV()(4 * i + a);
      for (int b = 0; b < 3; ++b) out[6 * n + 9 * i + 3 * a + b] = fB(3 * i + a, b);
    }
}

}  // namespace

extern "C" {

// `steps` calls of stepSystem(dt) on each scene: href with WetClothCore,
// hgpu with GpuWetClothCore (criterion, maxiters, solver, precision as the
// integrator would pass them).  out_* receive x3 | v3 | C9 (15 n doubles) of
// each scene; n_* the particle counts (the outputs are written only when
// they fit cap particles); substeps_* the sub-steps of the last step.
// Returns 0, or -1 with the exception's message in err.
int wcbind_step_both(void* href, void* hgpu, int steps, double dt, double criterion,
                     int maxiters, int solver, int precision, long long cap, double* out_ref,
                     double* out_gpu, long long* n_ref, long long* n_gpu, int* substeps_gpu,
                     char* err, int errlen) {
  try {
    const auto& sr = *(const std::shared_ptr<TwoDScene>*)wcref_scene_sp(href);
    const auto& er = *(const std::shared_ptr<LinearizedImplicitEuler>*)wcref_stepper_sp(href);
    const auto& sg = *(const std::shared_ptr<TwoDScene>*)wcref_scene_sp(hgpu);
    const auto& eg = *(const std::shared_ptr<LinearizedImplicitEuler>*)wcref_stepper_sp(hgpu);
    WetClothCore ref_core(sr, er);
    GpuStepOptions opt;
    opt.criterion = criterion;
    opt.maxiters = maxiters;
    opt.solver = solver;
    opt.precision = precision;
    GpuWetClothCore gpu_core(sg, eg, opt);
    for (int k = 0; k < steps; ++k) {
      ref_core.stepSystem(dt);
      gpu_core.stepSystem(dt);
    }
    gpu_core.syncToScene();
    *substeps_gpu = gpu_core.lastSubsteps();
    *n_ref = sr->getNumParticles();
    *n_gpu = sg->getNumParticles();
    if (*n_ref <= cap) store(*sr, out_ref);
    if (*n_gpu <= cap) store(*sg, out_gpu);
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(err, (size_t)errlen, "%s", e.what());
    return -1;
  }
}

}  // extern "C"
