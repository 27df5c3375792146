/* libwcgpu: the libWetCloth fluid-step hot path on one NVIDIA B200 (sm_100a).
 *
 * C ABI (plain pointers and sizes).  Every call returns an int status
 * (WCG_OK == 0); the message of the last failure on the calling thread is
 * available from wcg_last_error().
 *
 * The entry points mirror the reference's call sites for the liquid path
 * (libWetCloth/Core/WetClothCore.cpp:115-258): the TwoDScene methods
 * rebucketizeParticles / resampleNodes / computeWeights / updateLiquidPhi /
 * updateSolidPhi / updateSolidWeights / mapParticleNodesAPIC /
 * mapParticleSaturationPsiNodes / constrainLiquidVelocity /
 * mapNodeParticlesAPIC, the SceneStepper virtuals stepVelocity / projectFine /
 * applyPressureDragFluid / acceptVelocity / advectScene, and the whole
 * WetClothCore::stepSystem.  Particle and grid state stays resident on the GPU
 * between calls; upload/download calls move it to and from host (or device)
 * buffers in the reference's layouts.
 */
#ifndef WETCLOTH_GPU_H
#define WETCLOTH_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WCG_OK = 0,
  WCG_ERR_ARG = 1,        /* invalid argument */
  WCG_ERR_CUDA = 2,       /* CUDA runtime error (message has the details) */
  WCG_ERR_NOT_CONVERGED = 3, /* pressure solve hit maxiters or rho was 0/NaN */
  WCG_ERR_DEVICE = 4,     /* a kernel recorded an error (wait limit, index) */
  WCG_ERR_STATE = 5,      /* call out of order (e.g. no grid built yet) */
  WCG_ERR_UNSUPPORTED = 6 /* the call needs a part of the reference not built
                             here (the elasto coupling of the solve) */
};

enum { WCG_FP64 = 0, WCG_FP32_REFINE = 1 };

/* Pressure solver: MIC(0)-PCG (robertbridson::PCGSolver, PCGSolver.h:245-330;
 * the default) or the reference's own default, multigrid-PCG
 * (AMGPCGSolveSparse, AlgebraicMultigrid.h:248-361). */
enum { WCG_SOLVER_MIC0 = 0, WCG_SOLVER_MG = 1 };

/* Scene parameters: the liquid subset of LiquidInfo
 * (libWetCloth/Core/TwoDScene.h:35-91) plus bucket info (numcells fixed at 4,
 * kernel order 2) and one solid box whose inside holds the fluid
 * (DistanceFieldObject DFT_BOX / DFU_SOLID / inside=true). */
typedef struct wcg_params {
  double dx;                       /* cell size = bucket size / 4 */
  double gravity[3];               /* SimpleGravityForce */
  double liquid_density;
  double flip_coeff;               /* LiquidInfo::flip_coeff */
  double liquid_boundary_friction; /* LiquidInfo::liquid_boundary_friction */
  double box_center[3];
  double box_half[3];
  double box_radius;
  int walls;                       /* 1: the box above is present */
  double criterion;                /* pressure criterion: ||r||_inf <= c ||b||_inf */
  int maxiters;                    /* PCG iteration limit.  wcg_default_params sets 1000,
                                      not the reference integrator's 100
                                      (App/TwoDSceneXMLParser.cpp:3265): that limit is sized
                                      for the reference's multigrid-PCG (6-8 iterations),
                                      while MIC(0)-PCG, this library's default solver, takes
                                      up to about 230 iterations at 256^3.  Pass 100 with
                                      WCG_SOLVER_MG for the reference's exact behaviour. */
  int precision;                   /* WCG_FP64 or WCG_FP32_REFINE */
  double refine_inner_tol;         /* FP32 inner-solve relative tolerance (default 1e-5;
                                      0: aim each inner solve at the criterion) */
  int max_refinements;             /* FP64 refinement sweeps (0: 20) */
  int solver;                      /* WCG_SOLVER_MIC0 or WCG_SOLVER_MG */
  double viscosity;                /* LiquidInfo::viscosity; 0: no viscosity */
  int viscosity_substeps;          /* explicit viscosity sub-steps (0: 1) */
  double elasto_flip_coeff;        /* LiquidInfo::elasto_flip_coeff (0.95) */
  double elasto_flip_asym_coeff;   /* LiquidInfo::elasto_flip_asym_coeff (1.0) */
  double elasto_advect_coeff;      /* LiquidInfo::elasto_advect_coeff (1.0) */
  double drag_viscosity;           /* LiquidInfo::viscosity as the liquid-solid drag reads it
                                      while the viscosity term is off (8.9e-3) */
  double correction_strength;      /* LiquidInfo::correction_strength (default here 0; the
                                      reference's scene parser defaults it to 0.2).
                                      correctLiquidParticles runs in every sub-step; at 0
                                      its springs vanish and it only projects its particle
                                      subset out of the solid, as the reference does */
  int correction_step;             /* LiquidInfo::correction_step (8) */
  double correction_multiplier;    /* LiquidInfo::correction_multiplier (2.0) */
  unsigned long long correction_seed; /* seed of the stream that picks each sub-step's
                                         particle subset (rand() in the reference) */
  int viscosity_implicit;          /* LiquidInfo::implicit_viscosity: each viscosity sub-step
                                      solves the implicit system
                                      (stepImplicitViscosityDiagonalPCG,
                                      LinearizedImplicitEuler.cpp:2127) with PCG
                                      preconditioned by its diagonal */
  double viscosity_criterion;      /* LinearizedImplicitEuler::m_viscous_criterion (1e-6):
                                      ||r||_inf <= criterion ||b||_inf */
  int particle_merge;              /* relabelLiquidParticles + mergeLiquidParticles +
                                      removeEmptyParticles before each sub-step
                                      (WetClothCore.cpp:97-110); the subset uses
                                      correction_step, as in the reference */
  unsigned long long merge_seed;   /* seed of the merge's draws (rand() in the reference) */
  double particle_cell_multiplier; /* LiquidInfo::particle_cell_multiplier (0.3535533906):
                                      V_fine = 4/3 pi (dx m / sqrt 3)^3 */
  int particle_split;              /* relabelLiquidParticles + splitLiquidParticles before
                                      each sub-step, ahead of the merge */
  unsigned long long split_seed;   /* seed of the split's rotations */
  int terminator;                  /* 1: one terminator box (a distance field with usage
                                      DFU_TERMINATOR); each sub-step starts with
                                      terminateParticles (TwoDScene.cpp:1756,
                                      WetClothCore.cpp:97) */
  double terminator_center[3];
  double terminator_half[3];
  double terminator_radius;
  int terminator_inside;           /* the box's inside flag: 1 removes the liquid particles
                                      that leave the box, 0 the ones that enter it */
} wcg_params;

typedef struct wcg_ctx wcg_ctx;

typedef struct wcg_stats {
  int substeps;
  int pcg_iters;
  int refinements;
  int converged;
  double residual;   /* final ||b - A p||_inf */
  double rhs_norm;   /* ||b||_inf */
  long long ndof;
  long long nactive_buckets;
  int visc_iters;        /* iterations of the last implicit viscosity solve */
  int visc_converged;    /* every implicit viscosity solve of the last step converged */
  double visc_residual;  /* its final ||b - A u||_inf */
} wcg_stats;

const char* wcg_last_error(void);
void wcg_default_params(wcg_params* p);

/* TwoDScene + LinearizedImplicitEuler + WetClothCore construction. */
int wcg_create(const wcg_params* params, wcg_ctx** out);
int wcg_destroy(wcg_ctx* ctx);

/* Liquid particles (TwoDScene::sampleLiquidDistanceFields attribute set,
 * TwoDScene.cpp:5564-5605): positions x3[3n], fluid velocities v3[3n], affine
 * matrices C9[9n] row-major (m_fB rows; may be NULL = zero), fluid mass,
 * fluid volume and radius per particle.  Host pointers. */
int wcg_upload_liquid(wcg_ctx* ctx, long long n, const double* x3,
                      const double* v3, const double* C9, const double* mass,
                      const double* vol, const double* radius);
/* Same with device pointers (state already resident in HBM). */
int wcg_upload_liquid_device(wcg_ctx* ctx, long long n, const double* x3,
                             const double* v3, const double* C9,
                             const double* mass, const double* vol,
                             const double* radius);
/* Particle state in the original particle order (any pointer may be NULL). */
int wcg_download_liquid(wcg_ctx* ctx, double* x3, double* v3, double* C9);
int wcg_download_liquid_device(wcg_ctx* ctx, double* x3, double* v3,
                               double* C9);
/* wcg_download_liquid without waiting for the copies: the particle state is
 * gathered at once, and its transfer to the host overlaps whatever the caller
 * does next on this context (an upload, the next step).  The host buffers
 * should be pinned (cudaHostAlloc) and must stay untouched until
 * wcg_synchronize returns. */
int wcg_download_liquid_async(wcg_ctx* ctx, double* x3, double* v3, double* C9);
/* The upload of wcg_upload_liquid in two halves, so that the host-to-device
 * copies of the next set overlap the current step: wcg_stage_liquid_async
 * queues the copies into a staging buffer and returns (host buffers pinned
 * and untouched until the set is loaded); wcg_upload_staged loads the staged
 * set into the particle arrays after the work already queued on the context
 * (a step in progress), as wcg_upload_liquid would. */
int wcg_stage_liquid_async(wcg_ctx* ctx, long long n, const double* x3, const double* v3,
                           const double* C9, const double* mass, const double* vol,
                           const double* radius);
int wcg_upload_staged(wcg_ctx* ctx);
/* waits for every operation on the context, asynchronous copies included */
int wcg_synchronize(wcg_ctx* ctx);
long long wcg_num_particles(const wcg_ctx* ctx);

/* Elasto (cloth / yarn) particles, the reference's particles [0, n) ahead of
 * the liquid ones (TwoDScene::isFluid, TwoDScene.cpp:6921;
 * getNumElastoParticles :5212).  Arrays in the reference's layouts: x4/v4 =
 * m_x/m_v (x, y, z, twist; 4n), B9 = m_B rows (9n row-major), m4/fm4 = m_m and
 * m_fluid_m (4n; P2G adds the first three componentwise), m_rest_vol,
 * m_rest_volume_fraction, m_fluid_vol, m_shape_factor (n each), m_orientation
 * (3n), surfel (n; nonzero where m_particle_to_surfel >= 0).  Host pointers.
 * They take part in the grid build, the transfers (mapParticleNodesAPIC
 * :6609-6919, mapParticleSaturationPsiNodes :5952, updatePorePressureNodes
 * :5933, mapNodeParticlesAPIC :6936-7090), the liquid step's coupling to them
 * (constructHDV drag, pore-pressure gradients, the solid volume in the
 * pressure system, applyPressureDragFluid's solid drag) and advection
 * (SceneStepper.cpp:17).  The solid phase itself is not solved
 * (LiquidInfo::solve_solid off): its node velocity is the P2G one, or what
 * wcg_upload_field("vel_*") sets. */
int wcg_upload_elasto(wcg_ctx* ctx, long long n, const double* x4, const double* v4,
                      const double* B9, const double* m4, const double* fm4,
                      const double* rest_vol, const double* rest_vf,
                      const double* fluid_vol, const double* shape_factor,
                      const double* orient3, const int* surfel);
/* Elasto state (m_x, m_v with twists; m_B rows) in the original order. */
int wcg_download_elasto(wcg_ctx* ctx, double* x4, double* v4, double* B9);
long long wcg_num_elasto(const wcg_ctx* ctx);

/* ---- state I/O in the reference's file formats ---- */
/* TwoDSceneSerializer::serializePositionOnly (App/TwoDSceneSerializer.cpp:161):
 * binary, int byte count + m_x (x, y, z, twist = 0 per particle, doubles,
 * original particle order) + int byte count (0: no cloth Gauss points). */
int wcg_save_positions(wcg_ctx* ctx, const char* path);
/* TwoDSceneSerializer::loadPosOnly (App/TwoDSceneSerializer.cpp:172): replaces
 * the particle positions; the file's particle count must match.  Call
 * wcg_rebucketize_and_resample (or wcg_step) afterwards. */
int wcg_load_positions(wcg_ctx* ctx, const char* path);
/* The fluid OBJ of TwoDSceneSerializer (App/TwoDSceneSerializer.cpp:40-47,
 * updateFluid :242): one "v x y z radius" line per particle, 8 digits. */
int wcg_write_fluid_obj(wcg_ctx* ctx, const char* path);

/* ---- the reference call sequence (WetClothCore::stepSystem order) ---- */
/* updateParticleBoundingBox + rebucketizeParticles + resampleNodes
 * (TwoDScene.cpp:1588, :1657, :5069): grid, particle sort, bucket activation */
int wcg_rebucketize_and_resample(wcg_ctx* ctx);
/* computeWeights + updateLiquidPhi + updateSolidPhi + updateSolidWeights +
 * mapParticleNodesAPIC + mapParticleSaturationPsiNodes +
 * updatePorePressureNodes (TwoDScene.cpp:2246, :3286, :7940, :1871, :6609,
 * :5952, :5933) */
int wcg_map_particle_nodes(wcg_ctx* ctx);
/* LinearizedImplicitEuler::stepVelocity (+acceptVelocity of u*),
 * LinearizedImplicitEuler.cpp:224, with the explicit viscosity sub-steps of
 * :272-306 (viscosity::applyNodeViscosityExplicit, Viscosity.cpp:1780) when
 * wcg_params.viscosity > 0 */
int wcg_step_velocity(wcg_ctx* ctx, double dt);
/* LinearizedImplicitEuler::projectFine -> pressure::solveNodePressure
 * (Pressure.cpp:285) with MIC(0)-PCG */
int wcg_project_fine(wcg_ctx* ctx, double dt);
/* applyPressureDragFluid + acceptVelocity (LinearizedImplicitEuler.cpp:2435,
 * :2176) */
int wcg_apply_pressure_drag_fluid(wcg_ctx* ctx, double dt);
/* TwoDScene::constrainLiquidVelocity (TwoDScene.cpp:1827) */
int wcg_constrain_liquid_velocity(wcg_ctx* ctx);
/* TwoDScene::correctLiquidParticles (TwoDScene.cpp:1967-2061) for the liquid
 * particles with index % correction_step == selector (the reference draws the
 * selector with rand(); wcg_substep draws it from wcg_correction_selector).
 * Runs between wcg_constrain_liquid_velocity and wcg_map_node_particles, as
 * WetClothCore::stepSystem does (WetClothCore.cpp:242); G2P then keeps the
 * weights of the positions before the correction.  Coincident pairs (closer
 * than 1e-4 re) are pushed by a SplitMix64 hash of their indices instead of
 * scalarRand.  With correction_strength 0 the subset is only projected out
 * of the solid (the springs vanish), one particle at a time.  selector -1
 * takes the next subset of the context's seeded stream, the one wcg_substep
 * would draw (a stage-by-stage caller reproduces wcg_substep this way). */
int wcg_correct_liquid_particles(wcg_ctx* ctx, double dt, int selector);
/* the subset wcg_substep corrects in its k-th call: SplitMix64 of the seed and
 * k, modulo step */
int wcg_correction_selector(unsigned long long seed, unsigned long long k, int step);
/* sets the call count of the correction stream: the next sub-step (and the
 * sub-step wcg_substep_vjp differentiates) corrects the subset of call k */
int wcg_set_correction_count(wcg_ctx* ctx, unsigned long long k);
/* the call count of the correction stream: the call the next sub-step takes */
unsigned long long wcg_correction_count(const wcg_ctx* ctx);
/* TwoDScene::updateOptiVolume (relabelLiquidParticles TwoDScene.cpp:2484-2505),
 * mergeLiquidParticles (:2510-2666) and removeEmptyParticles (:1713-1745) on
 * the buckets of the last grid build, for the liquid particles with index %
 * correction_step == selector, colours in the order perm9 (three permutations
 * of {0, 1, 2}: z, y, x parities), as the reference draws them with rand().
 * Removed particles leave the arrays with the reference's swap-with-last
 * renumbering; *removed (may be NULL) receives their count. */
int wcg_merge_liquid_particles(wcg_ctx* ctx, int selector, const int* perm9,
                               long long* removed);
/* TwoDScene::updateOptiVolume + splitLiquidParticles (TwoDScene.cpp:2362-2480):
 * every large liquid particle (volume above 2 V_fine) splits into
 * n = min(ceil(V / V_fine), 32) particles of volume V/n, the children
 * appended after all particles in the parents' index order with the parent's
 * velocity and a zero affine matrix.  The children sit on a spherical
 * Fibonacci lattice rotated by a quaternion drawn from SplitMix64 of
 * key ^ parent index (the reference: its compiled sphere-pattern table and
 * Matrix3s::Random()); *added (may be NULL) receives their count. */
int wcg_split_liquid_particles(wcg_ctx* ctx, unsigned long long key, long long* added);
/* The reference's own split placement, for a caller that holds the
 * reference's draws.  wcg_split_parents gives the number of particles the
 * split would split now (the liquid particles above 2 V_fine).
 * wcg_split_liquid_particles_with splits them with the caller's sphere-pattern
 * table -- TwoDScene::m_sphere_pattern[n] for n = 2..32 concatenated, 3n
 * doubles each, WCG_SPLIT_PATTERN_LEN in all -- and one row-major 3x3 rotation
 * per splitting parent in original-index order: the Q of the QR
 * decomposition of the Matrix3s::Random() that splitLiquidParticles draws for
 * that parent (TwoDScene.cpp:2390-2392).  The parent moves to
 * centre + pattern[n][0..2] s, child i (1 <= i < n) sits at
 * centre + Q pattern[n][3i..3i+2] s.  nparents must equal the count
 * wcg_split_parents gives (else WCG_ERR_ARG, nothing changed). */
#define WCG_SPLIT_PATTERN_LEN 1581
int wcg_split_parents(wcg_ctx* ctx, long long* nparents);
int wcg_split_liquid_particles_with(wcg_ctx* ctx, const double* pattern, const double* rot9,
                                    long long nparents, long long* added);
/* TwoDScene::terminateParticles (TwoDScene.cpp:1756-1771): the liquid
 * particles where the terminator box's phi is negative (outside it for
 * terminator_inside = 1) and every liquid particle without volume are
 * removed as removeEmptyParticles does (each hole takes the last survivor);
 * *removed (may be NULL) receives their count.  With params.terminator = 0
 * only particles without volume are removed.  wcg_substep runs it first when
 * params.terminator is set. */
int wcg_terminate_liquid_particles(wcg_ctx* ctx, long long* removed);
/* Terminator shapes: the DistanceFieldObjects of the scene whose usage is
 * DFU_TERMINATOR (DistanceFields.cpp:477-520), any of box, sphere, capsule
 * and cylinder, rotated and inside or not.  A particle is removed where
 *   phi = min(3 bucket size, min over the shapes of their phi)
 * is negative -- TwoDScene::computePhiVel (TwoDScene.cpp:5427-5447) over the
 * distance-field groups, each a union of its members
 * (DistanceFieldOperator, DistanceFields.cpp:835-849).  A shape's phi is
 * DistanceFieldObject::compute_phi (DistanceFields.cpp:601-660): the position
 * is taken into the object's frame by the quaternion sandwich
 * conj(rot) (0, p - c) conj(rot)^-1 (box, capsule, cylinder), then
 *   box      param = half extents x, y, z, corner radius
 *   sphere   param[0] = radius
 *   capsule  param = radius, half length (axis along x)
 *   cylinder param = outer radius, corner radius, half height (axis along y)
 * and negated for an inside object.  rot is the object's rotation
 * (Eigen::AngleAxis of its axis and angle, w x y z).  wcg_set_terminators
 * replaces the terminator of wcg_params (n = 0: none); while any shape is
 * set, wcg_substep runs terminateParticles first. */
enum { WCG_SHAPE_BOX = 0, WCG_SHAPE_SPHERE = 1, WCG_SHAPE_CAPSULE = 2, WCG_SHAPE_CYLINDER = 3 };
#define WCG_MAX_TERMINATOR_SHAPES 16
typedef struct {
  int type;           /* WCG_SHAPE_* */
  int inside;         /* the object's inside flag: phi negated */
  double center[3];
  double rot[4];      /* w, x, y, z */
  double param[4];
} wcg_shape;
int wcg_set_terminators(wcg_ctx* ctx, int n, const wcg_shape* shapes);
/* the key wcg_substep uses for its k-th split */
unsigned long long wcg_split_key(unsigned long long seed, unsigned long long k);
/* the draws wcg_substep uses for its k-th merge: SplitMix64 of the seed and k
 * for the selector, then three Fisher-Yates permutations of {0, 1, 2} */
int wcg_merge_draws(unsigned long long seed, unsigned long long k, int step, int* selector,
                    int* perm9);
/* TwoDScene::mapNodeParticlesAPIC (TwoDScene.cpp:6936) */
int wcg_map_node_particles(wcg_ctx* ctx);
/* SceneStepper::advectScene (SceneStepper.cpp:17) followed by
 * TwoDScene::solidProjection (TwoDScene.cpp:1776-1821) of the liquid
 * particles, as WetClothCore::stepSystem runs them (WetClothCore.cpp:258-262) */
int wcg_advect(wcg_ctx* ctx, double dt);
/* One CFL sub-step of everything above (G2P and advection fused). */
int wcg_substep(wcg_ctx* ctx, double dt);
/* WetClothCore::stepSystem (WetClothCore.cpp:45): CFL sub-stepping + sub-steps */
int wcg_step(wcg_ctx* ctx, double dt, int* substeps_out);
int wcg_num_substeps(wcg_ctx* ctx, double dt, int* n_out);
/* Reverse mode of wcg_substep (no reference counterpart: the reference has
 * no derivatives).  Call with the context holding the particle state before
 * the sub-step; it recomputes the forward grid fields there and leaves the
 * particles unchanged.  In: cotangents of the sub-step's outputs v' (3n),
 * C' (9n, rows as in wcg_download_liquid) and x' (3n).  Out: cotangents of
 * the inputs v (3n) and C (9n), of the liquid viscosity (viscosity_bar, may be
 * NULL; 0 when the viscosity is off) and of the positions x (3n): xbar0 holds
 * xbar3 (the advection's identity part) plus the derivative through the
 * quadratic B-spline weights and the APIC offsets x_node - x of P2G and G2P
 * (TwoDScene::updateParticleWeights TwoDScene.cpp:2084-2174), through the
 * liquid phi behind the ghost-fluid fractions of the pressure matrix, and
 * through the solid projection of the particle correction.  The grid's
 * discrete structure (activation, DOFs, valid faces) and the nearest
 * particle chosen for each node's liquid phi are held at the checkpoint's
 * values.
 * wcg_set_adjoint_positions(ctx, 0) holds x fixed instead (xbar0 = xbar3).
 * Liquid scenes; the solve is the forward's solver on the same (symmetric)
 * matrix (its ghost-fluid fractions' own derivative enters the right-hand
 * side).  With the particle correction on, the sub-step differentiated corrects the subset of the
 * correction stream's next call (wcg_set_correction_count).  Refused
 * (WCG_ERR_UNSUPPORTED) with elasto particles, the implicit viscosity, or the
 * particle split or merge on. */
int wcg_substep_vjp(wcg_ctx* ctx, double dt, const double* vbar3, const double* Cbar9,
                    const double* xbar3, double* vbar0, double* Cbar0, double* xbar0,
                    double* viscosity_bar);
/* 1 (default): wcg_substep_vjp differentiates through the particle positions;
 * 0: positions held fixed (xbar0 = xbar3). */
int wcg_set_adjoint_positions(wcg_ctx* ctx, int differentiate);
/* LiquidInfo::viscosity and the explicit viscosity sub-steps of a context
 * (0: off), as wcg_params sets them at creation. */
int wcg_set_viscosity(wcg_ctx* ctx, double viscosity, int substeps);

/* Failure handling of the MIC(0) wavefront (no reference counterpart; the
 * reference's triangular solves are serial and never wait).  Each poll of a
 * wavefront edge word is bounded by spin_limit polls (default 2^20); a wait
 * that reaches it records a device error, the sweep finishes with zeros in
 * place of the missing values, and the call returns WCG_ERR_DEVICE -- the
 * context stays usable.  stale_patch >= 0 makes that patch of the pencil
 * layout (indices past the last patch mean the last one) wait for a tag that
 * no producer writes, so a test can run the limit out on purpose; -1 turns
 * it off. */
int wcg_set_wait_limit(wcg_ctx* ctx, long long spin_limit, int stale_patch);

int wcg_get_stats(const wcg_ctx* ctx, wcg_stats* out);

/* ---- parity downloads in the reference's dense bucket-major layout ---- */
/* grid: dims[3] buckets, origin[3] (m_grid_mincorner), bbx[6] */
int wcg_grid_info(const wcg_ctx* ctx, int* dims, double* origin, double* bbx);
/* number of values of a named field (-1 if unknown) */
long long wcg_field_size(wcg_ctx* ctx, const char* name);
/* double field by name, nb*64 values (orientation_*: 3 per node,
 * interleaved), NaN in inactive buckets */
int wcg_download_field(wcg_ctx* ctx, const char* name, double* out, long long n);
/* Set a node velocity field between calls: "u_x/y/z" (the liquid face
 * velocity mapNodeParticlesAPIC reads, m_node_vel_fluid_*) or "vel_x/y/z"
 * (the solid-phase m_node_vel_*, with elasto particles) -- the seam where a
 * caller's own solve (e.g. LinearizedImplicitEuler's solid phase) hands its
 * result back.  n >= number of nodes; inactive buckets are ignored. */
int wcg_upload_field(wcg_ctx* ctx, const char* name, const double* in, long long n);
/* integer field by name ("active", "dof_index", "valid_x", "array_idx",
 * "array_sup", "stencil_base", "grid_dims") */
int wcg_download_ifield(wcg_ctx* ctx, const char* name, long long* out, long long n);
/* assembled pressure system in the reference's DOF order and CSR layout of
 * robertbridson::SparseMatrix (sorted columns).  With rowstart == NULL only
 * the sizes are returned. */
int wcg_export_pressure_system(wcg_ctx* ctx, long long* ndof, long long* nnz,
                               long long* rowstart, long long* col,
                               double* val, double* rhs);

/* ---- a sparse solve with the reference's PCGSolver call shape ---- */
/* robertbridson::PCGSolver<double>::solve(matrix, rhs, result, residual_out,
 * iterations_out) after set_solver_parameters(tolerance_factor,
 * max_iterations) (libWetCloth/Core/PCGSolver/PCGSolver.h:249-308): MIC(0)
 * preconditioned CG (modification 0.97, pivot ratio 0.25, as
 * form_preconditioner fixes them) on the symmetric matrix given in CSR form --
 * rowstart[n + 1], col[] strictly ascending inside each row, val[] -- which is
 * the layout of the reference's SparseMatrix / FixedSparseMatrix rows.  x[n]
 * receives the solution from a zero start; the stop rule is the reference's:
 * ||r||_inf <= tolerance_factor * ||rhs||_inf.  Host arrays.  Returns WCG_OK
 * when converged (the reference's true) and WCG_ERR_NOT_CONVERGED at the
 * iteration limit or a zero/NaN rho (its false), with x, *residual_out and
 * *iterations_out filled either way; WCG_ERR_ARG for a malformed matrix. */
int wcg_pcg_solve_csr(const int* rowstart, const int* col, const double* val, int n,
                      const double* rhs, double* x, double tolerance_factor,
                      int max_iterations, double* residual_out, int* iterations_out);

/* ---- many scenes at once (config 4 of the benchmark plan) ---- */
/* A batch steps independent scenes (each created, uploaded and owned by the
 * caller) from a pool of host threads, largest scene first; every scene keeps
 * its own stream, so the kernels of different scenes overlap on the GPU.
 * Each scene's result is what wcg_step on it alone gives.  No reference
 * counterpart: the reference steps one TwoDScene per process. */
typedef struct wcg_batch wcg_batch;
int wcg_batch_create(int n, wcg_ctx* const* scenes, wcg_batch** out);
int wcg_batch_destroy(wcg_batch* b);
/* nsteps wcg_step calls per scene with its own dt[i]; status[i] (may be NULL)
 * receives each scene's last status.  Returns the first hard error, else
 * WCG_ERR_NOT_CONVERGED if any scene's solve did not converge, else WCG_OK. */
int wcg_batch_step(wcg_batch* b, const double* dt, int nsteps, int* status);
int wcg_batch_set_threads(wcg_batch* b, int nthreads);
int wcg_batch_threads(const wcg_batch* b);
/* The shared solve (on: 1, off: 0; default off).  On, the PCG iterations of
 * every scene that reaches its pressure solve during a batch step run in
 * shared launches: one launch per kernel (SpMV, forward and backward MIC(0)
 * sweep) over all waiting scenes of one precision, chunks of 8 iterations,
 * each scene's status read once per chunk, converged scenes released and new
 * ones admitted between chunks.  Each scene's arithmetic, block counts and
 * partial sums are those of its solve alone, so results are unchanged.
 * Needs every scene on one device; the scenes' own sweeps outside the
 * iterations keep their schedules. */
int wcg_batch_set_shared_solve(wcg_batch* b, int on);
/* Scenes whose pressure solve spans more than max_patches pencil patches
 * (16 x 16 lines of the solve's DOF box across its stream axis) iterate
 * alone instead, so the largest scenes do not set the length of every
 * shared chunk (default: no limit; results unchanged either way). */
int wcg_batch_set_shared_solve_limit(wcg_batch* b, int max_patches);
/* kernel launches the batch's shared solves have made (-1: null batch) */
long long wcg_batch_shared_launches(const wcg_batch* b);
/* Times one batch step per candidate thread count (each trial advances every
 * scene by one step), keeps the fastest; ms[k] (may be NULL) gets the times. */
int wcg_batch_autotune(wcg_batch* b, const double* dt, const int* candidates, int ncand,
                       double* ms);

/* Launch schedule of a context's pressure solve (no reference counterpart).
 * Performance only: every schedule gives bit-identical results.
 *   sweep_cluster    CTAs per thread-block cluster along c in the MIC(0)
 *                    sweeps: 0 chosen per solve from the patches along c
 *                    (the default), 1 plain, or 2, 3, 4, 8, 9, 16 (used when
 *                    the box has more than half that many patches along c);
 *   sweep_cluster_a  CTAs along a as well (2-D clusters): 1, 4 (with
 *                    sweep_cluster 1..4) or 8 (with sweep_cluster 1..2);
 *   pcg_batch        PCG iterations launched per convergence check on the
 *                    host (1..64; default 8). */
typedef struct wcg_schedule {
  int sweep_cluster;
  int sweep_cluster_a;
  int pcg_batch;
} wcg_schedule;
int wcg_set_schedule(wcg_ctx* ctx, const wcg_schedule* s);
int wcg_get_schedule(const wcg_ctx* ctx, wcg_schedule* s);
/* Chooses each scene's schedule from timed trials: for each candidate k in
 * turn every scene takes that schedule and the batch is stepped `trials`
 * times (each trial advances every scene by one step, all scenes at once on
 * the thread count set); a scene's time is the device time of its step on
 * its own stream (CUDA events), minimum over the trials.  Each scene keeps
 * its fastest candidate.  ms (may be NULL) gets n x ncand times (scene-major),
 * chosen (may be NULL) the candidate index per scene. */
int wcg_batch_autotune_schedules(wcg_batch* b, const double* dt, const wcg_schedule* cand,
                                 int ncand, int trials, double* ms, int* chosen);

/* ---- instrumentation ---- */
/* the cudaStream_t all of this context's kernels run on */
void* wcg_stream(const wcg_ctx* ctx);
/* number of kernels this context has launched so far */
long long wcg_launch_count(const wcg_ctx* ctx);
/* per-phase CUDA-event timing: begin, run steps, end; end fills ms[ncat] and
 * launches[ncat] with totals per phase (names from wcg_profile_phase_name) */
int wcg_profile_begin(wcg_ctx* ctx);
int wcg_profile_end(wcg_ctx* ctx, double* ms, long long* launches, int ncat);
int wcg_profile_num_phases(void);
const char* wcg_profile_phase_name(int i);

/* ---- allocation-free pressure solve ----
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (an application that owns and pre-reserves all device memory, a strict
 * memory pool or budget, code that must not allocate between frames): solves
 * an already assembled pressure system with the same FP64 MIC(0)-PCG as
 * wcg_project_fine, taking all solver scratch from one static device array
 * of about 17 MB that every GPU loading this library holds until exit.
 * Inputs are dense bucket-major device arrays over ni*nj*nk buckets (64 cells
 * each, index bucket*64 + k*16 + j*4 + i): the DOF mask (nonzero = unknown),
 * the diagonal, the couplings a_x/a_y/a_z between a cell and its +x/+y/+z
 * neighbour, and the rhs; pressure (device, same layout) receives the
 * solution (0 off the DOFs).  Stops when ||r||_inf <= criterion ||rhs||_inf.
 * At most 2048 buckets (131072 cells); larger grids are rejected with
 * WCG_ERR_ARG.  The first call on a device looks up the array's device
 * address (make that first call before any stream capture).  Calls share the
 * array: calls whose GPU work overlaps race and must be serialised. */
int wcg_pressure_solve_noalloc(int ni, int nj, int nk, const unsigned char* dof,
                               const double* a_diag, const double* a_x,
                               const double* a_y, const double* a_z,
                               const double* rhs, double* pressure,
                               double criterion, int maxiters, void* stream,
                               int* iters_out, double* residual_out);

#ifdef __cplusplus
}
#endif

#endif /* WETCLOTH_GPU_H */
