// Device state of one scene and the host-side orchestration of the fluid step.
// Everything here is internal to libwcgpu.so; the public surface is the C-ABI
// in include/wetcloth_gpu.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "wcg_common.cuh"

namespace wcg {

struct Params {
  double dx;
  double gravity[3];
  double liquid_density;
  double flip_coeff;
  double liquid_boundary_friction;
  double box_center[3];
  double box_half[3];
  double box_radius;
  int walls;
  double criterion;
  int maxiters;
  int precision;  // 0: FP64, 1: FP32 transfers + FP32 PCG with FP64 refinement
  double refine_inner_tol;  // relative tolerance of each FP32 inner solve
  int max_refinements;
  int solver;     // 0: MIC(0)-PCG, 1: multigrid-PCG (AMGPCGSolveSparse)
  double viscosity;        // LiquidInfo::viscosity (0: compute_viscosity off)
  int viscosity_substeps;  // viscosity sub-steps per step_velocity
  int viscosity_implicit;  // LiquidInfo::implicit_viscosity
  double viscosity_criterion;  // LinearizedImplicitEuler::m_viscous_criterion
  double elasto_flip;      // LiquidInfo::elasto_flip_coeff
  double elasto_flip_asym; // LiquidInfo::elasto_flip_asym_coeff
  double elasto_advect;    // LiquidInfo::elasto_advect_coeff
  double drag_viscosity;   // LiquidInfo::viscosity as the drag reads it when viscosity == 0
  double correction_strength;    // LiquidInfo::correction_strength (0: no correction)
  int correction_step;           // LiquidInfo::correction_step
  double correction_multiplier;  // LiquidInfo::correction_multiplier
  unsigned long long correction_seed;  // seed of the per-sub-step subset stream
  int particle_merge;            // relabel + mergeLiquidParticles before each sub-step
  int particle_split;            // relabel + splitLiquidParticles before each sub-step
  unsigned long long split_seed; // seed of the split's rotations
  unsigned long long merge_seed; // seed of the merge's draws
  double cell_multiplier;        // LiquidInfo::particle_cell_multiplier (V_fine)
  int terminator;                // a terminator box: terminateParticles first in each sub-step
  double term_center[3], term_half[3], term_radius;
  int term_inside;               // the box's inside flag (sign -1)
};

// A device allocation that grows and never shrinks.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n);
  void release();
  template <typename T>
  T* as() const { return (T*)p; }
};

// Per-step solver and step statistics.
struct Stats {
  int substeps = 0;
  int pcg_iters = 0;          // total inner PCG iterations of the last solve
  int refinements = 0;        // FP64 outer iterations of the last solve
  double residual = 0;        // final ||b - A p||_inf of the last solve
  int visc_iters = 0;         // iterations of the last implicit viscosity solve
  double visc_residual = 0;   // its final ||b - A u||_inf
  int visc_converged = 1;     // every implicit viscosity solve of the step converged
  double rhs_norm = 0;        // ||b||_inf of the last solve
  int converged = 1;
  long long ndof = 0;
  long long nactive = 0;
};

// Names of the particle columns (SoA, sorted order).
enum PCol : int {
  PX = 0, PY, PZ, VX, VY, VZ,
  C00, C01, C02, C10, C11, C12, C20, C21, C22,
  PM, PV, PR,
  kNumPCols
};

// Dense grid field identifiers (nnode values each).
enum GField : int {
  // faces, component-major: field + 0/1/2 for x/y/z
  G_MASS = 0,          // m_node_mass_fluid_{x,y,z}
  G_VEL = 3,           // m_node_vel_fluid_{x,y,z} after P2G
  G_VOL = 6,           // m_node_vol_fluid_{x,y,z}
  G_SAT = 9,           // m_node_sat_{x,y,z}
  G_WEIGHT = 12,       // m_node_solid_weight_{x,y,z}
  G_VSTAR = 15,        // m_node_v_fluid_plus after stepVelocity
  G_RHS = 18,          // m_node_rhs_fluid
  G_INVC = 21,         // m_node_inv_C
  G_PSIFS = 24,        // m_node_psi_fs
  G_U = 27,            // final face velocity (after projection/extrapolation)
  G_UTMP = 30,         // extrapolation double buffer
  // cells
  G_LPHI = 33,         // m_node_liquid_phi
  G_SATP = 34,         // m_node_sat_p
  G_SPHI = 35,         // m_node_solid_phi (corner nodes)
  G_PRESSURE = 36,     // m_node_pressure
  G_ADIAG = 37,        // Poisson matrix diagonal
  G_AX = 38,           // coupling to the +x neighbour
  G_AY = 39,
  G_AZ = 40,
  G_B = 41,            // rhs (divergence)
  G_INVDIAG = 42,      // MIC(0) 1/L_ii
  G_R = 43, G_Z = 44, G_S = 45, G_Q = 46, G_X = 47,
  G_S2 = 48,           // second search-direction buffer (ping-pong)
  G_Y = 49,            // forward-sweep output L^{-1} r
  G_SX = 50,           // MIC(0) scaled couplings S_a = A_a * invdiag
  G_SY = 51,
  G_SZ = 52,
  G_VFC = 53,          // liquid volume fraction at cell centres (viscosity)
  G_VFEX = 54,         // ... at x-, y-, z-edge nodes
  G_VFEY = 55,
  G_VFEZ = 56,
  G_VFU = 57,          // ... at x-, y-, z-faces (implicit viscosity)
  G_VFV = 58,
  G_VFW = 59,
  kNumGFields = 60
};

// Columns of the elasto (cloth / yarn) particle SoA.  Positions come first so
// the bounding-box and particle-pass kernels read them as they read liquid
// particles.  EM* = m(a) + m_fluid(a), ERV/ERF = m_rest_vol and
// m_rest_volume_fraction, EFV = m_fluid_vol, ESF = m_shape_factor, EO* =
// m_orientation, ESURF = 1 for surfels (m_particle_to_surfel >= 0).
enum ECol : int {
  EX = 0, EY, EZ, ETH, EVX, EVY, EVZ, EVT,
  EB00, EB01, EB02, EB10, EB11, EB12, EB20, EB21, EB22,
  EM0, EM1, EM2, ERV, ERF, EFV, ESF, EOX, EOY, EOZ, ESURF,
  kNumECols
};

// Node fields that only elasto particles make nonzero (m_node_mass_*,
// m_node_vel_*, m_node_vol_*, m_node_psi_*, m_node_shape_factor_*,
// m_node_orientation_* (3 per face axis), m_node_psi_p, pore pressure).
enum EField : int {
  E_MASS = 0, E_VEL = 3, E_VOL = 6, E_PSI = 9, E_SF = 12,
  E_ORI = 15,  // E_ORI + 3 * axis + component
  E_PSIP = 24, E_PORE = 25,
  E_Q = 26,    // mshdvm_hdvm: hdV / (m_solid + hdV) of constructHDV, per face axis
  kNumEFields = 29
};

// Geometry of the pencil layout of one pressure solve (wcg_pencil.cuh).
struct PencilGeom {
  int ax_s, ax_a, ax_c;  // physical axis (0 x, 1 y, 2 z) of s, a, c
  int lo[3];             // low corner of the DOF box (grid cells, physical axes)
  int Ls, NA, NC;        // box extent along s, a, c
  int nPA, nPC;          // patches along a, c
  int R;                 // rows per patch (Ls + 2 * (patch edge - 1))
  long long npatch;      // nPA * nPC
  long long len;         // elements per array (npatch * R * lines per patch)
};

// Arrays of the pencil layout (Reals, len each; PL64_* are doubles).
// PL_COEF spans four arrays: the MIC(0) factor interleaved per cell,
// {1/sqrt(d'), S_s, S_a, S_c}.
enum PlField : int {
  PL_AD = 0, PL_AS, PL_AA, PL_AC, PL_B,        // assembled system
  PL_COEF,                                     // MIC(0) factor (4 arrays)
  PL_R = PL_COEF + 4, PL_X, PL_S0, PL_S1, PL_Q, PL_Y, PL_Z,  // PCG vectors
  kNumPlFields
};
enum Pl64Field : int { PL64_X = 0, PL64_R, kNumPl64Fields };

struct SharedSolve;  // a batch's shared PCG iterations (wcg_step.cu)

struct Context {
  Params prm;
  cudaStream_t stream = nullptr;
  // asynchronous downloads: the gather into dstage runs on `stream`, the
  // device-to-host copies on copy_stream, ordered by the two events
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_store = nullptr, ev_d2h = nullptr;
  DevBuf dstage;
  // staged uploads: host-to-device copies into ustage on in_stream, loaded
  // into the particle arrays later on `stream`
  cudaStream_t in_stream = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_loaded = nullptr;
  DevBuf ustage;
  // set by a batch step with the shared solve on: the PCG iterations of the
  // pressure solve join the batch's launches (ordered by the two events)
  SharedSolve* shared_solve = nullptr;
  cudaEvent_t ev_ss_ready = nullptr, ev_ss_done = nullptr;
  long long staged_n = -1;
  bool staged_C = false;
  int device = 0;
  std::string last_error;

  // particles
  long long np = 0;
  long long pcap = 0;
  DevBuf pbuf[2];          // kNumPCols * pcap Reals each (ping-pong)
  int cur = 0;             // which pbuf holds the sorted state
  DevBuf pid[2];           // original particle index, int32
  DevBuf pkey;             // key node (p-stencil centre), int64
  DevBuf pdelta;           // packed stencil offsets, int32
  DevBuf pbucket;          // reference bucket index, int32
  DevBuf perm;             // sorted slot -> source slot, int32
  DevBuf hostorder;        // scratch for downloads in original order

  // elasto particles: same sorted ping-pong scheme as the liquid ones
  long long ne = 0;
  long long ecap = 0;
  DevBuf ebuf[2];          // kNumECols * ecap Reals each
  int ecur = 0;
  DevBuf epid[2];          // original elasto index, int32
  DevBuf ekey, edelta, ebucket;  // as pkey/pdelta/pbucket, 2 * ecap each
  DevBuf eperm;
  DevBuf estage;           // upload/download staging (doubles)
  DevBuf ecell_start;      // int32 per node + 1 (elasto particles per key cell)
  DevBuf efield;           // kNumEFields * gcap Reals (allocated with elasto)
  long long efcap = 0;

  // grid
  GridDesc g{};
  bool have_grid = false;
  double bbx_min[3] = {0, 0, 0}, bbx_max[3] = {0, 0, 0};
  DevBuf active_pre, active;     // uint8 per bucket
  DevBuf cell_start;             // int32 per node + 1
  DevBuf cell_cursor;            // int32 per node
  DevBuf gfield;                 // kNumGFields * gcap Reals
  DevBuf gvalid;                 // 3 * gcap uint8 (+3 tmp)
  DevBuf gdof;                   // uint8 per node
  long long gcap = 0;            // nodes allocated per field
  DevBuf wave_list;              // active 8^3-cell tiles ordered by ti+tj+tk
  DevBuf wave_count;             // per wave index
  DevBuf tile_flag;              // int per tile (epoch of completion)
  DevBuf tile_active;            // uint8 per tile
  DevBuf tile_part;              // per-ticket partial sums / maxima (double)
  int tile_epoch = 0;
  int nti = 0, ntj = 0, ntk = 0; // tiles per axis
  int sweep_variant = 0;         // 0: 8x8x8 block tiles, 1: 8x4x8 warp tiles
  long long n_tiles = 0;         // active tiles
  long long n_tiles_total = 0;   // all tiles of the grid (partials are indexed by tile id)
  long long n_active = 0;
  int drange_h[6] = {0, 0, 0, 1, 1, 1};  // min/max stencil offset per axis
  DevBuf active_list;            // compacted active buckets (int32)
  DevBuf p2g_halo;               // P2G halo tile per bucket (kTileVals Reals)
  int xfer_mode = 0;             // 0: bucket-tile P2G/G2P where they apply, 1: global gathers

  // pressure solve in the pencil layout (default) or on 8^3 tiles
  int pcg_layout = 0;            // 0: pencil layout, 1: bucket-major tiles
  PencilGeom plg{};
  DevBuf pl;                     // kNumPlFields * pl_cap Reals
  DevBuf pl64;                   // kNumPl64Fields * pl_cap doubles
  DevBuf pl_edge;                // tagged edge words
  DevBuf pl_order;               // patches in wave order (int32)
  DevBuf pl_corder;              // cluster columns in wave order (sweep_cluster > 1)
  DevBuf pl_corder2;             // 2-D cluster tiles in wave order (sweep_cluster_a > 1)
  int sweep_cluster = 1;         // CTAs per cluster along c in the MIC(0) sweeps
  int sweep_cluster_a = 1;       // ... and along a (2-D clusters: 4 or 8)
  int pl_cc = 1;                 // the c-extent the current solve uses (<= patches along c)
  int spmv_rows = 1;             // 0: the patch-streamed SpMV instead of the row-parallel one
  int pcg_batch = 8;             // PCG iterations launched per host convergence check
  DevBuf pl_part;                // per-patch partials (double)
  long long pl_cap = 0;
  int pl_tickets = 0;            // sweep tickets handed out in this solve
  long long spin_limit = 1ll << 20;  // polls of a wavefront edge word before giving up
  int adjoint_fixed_x = 0;       // substep_vjp: 1 = positions held fixed (x-bar passes)
  TermSet term{};                // terminator shapes (the params' box, or wcg_set_terminators)
  int stale_patch = -1;          // failure-path test: a patch whose waits cannot succeed
  std::vector<int> pl_order_h;
  // host copies of pl_corder / pl_corder2 and the (nPA, nPC, CC, CA) they
  // were built for: re-uploaded only when that changes
  std::vector<int> pl_corder_h, pl_corder2_h;
  long long pl_corder_key = -1, pl_corder2_key = -1;

  // multigrid-PCG: dense levels (d, ax, ay, az, x, b per cell; masks) and the
  // level-0 PCG vectors
  DevBuf mg, mg_mask, mg_vec;
  struct MgDims { int ni, nj, nk, n; long long off; };
  std::vector<MgDims> mg_dims;     // levels of the last solve

  // particle correction (wcg_correct.cuh): positions before the correction
  // (3 Reals per particle; valid from the correction to the next grid build),
  // the cell lists of correctLiquidParticles' own sort, the subset stream
  DevBuf xw;
  bool xw_valid = false;
  DevBuf corr_start, corr_cursor, corr_list;
  // the reference-exact split: ranks of the splitting parents, the sphere
  // pattern table and the caller's rotations on the device
  DevBuf split_rank, split_pat, split_rot;
  unsigned long long corr_count = 0;
  // particle merge (wcg_merge.cuh): classes, flags, gathered volume and
  // momentum, index maps; the merge's draw counter
  DevBuf mwork;
  unsigned long long merge_count = 0;
  bool buckets_valid = false;    // pbucket holds the bucket of every current particle
  bool maybe_empty = false;      // an upload since the last sub-step may have brought
                                 // liquid particles without fluid volume
  unsigned long long split_count = 0;
  long long merged_removed = 0;  // particles the last merge removed

  // reverse mode of a sub-step (wcg_adjoint.cuh): grid cotangents, particle
  // cotangents (sorted order), the first extrapolation layer's input mask,
  // host staging
  DevBuf adj, adjp, adjmask, adjstage, adjvisc;
  DevBuf adjxc;  // corrected positions of the sub-step (3 Reals per particle)
  DevBuf adjam;  // per cell: the sorted index of the particle that sets its liquid phi

  // implicit viscosity (wcg_visc.cuh): PCG vectors x, r, p, q and the
  // diagonal (3 face fields each), face flags
  DevBuf visc, viscflag;

  // FP64 refinement vectors (precision 1)
  DevBuf rx64, rr64, rb64;       // nnode doubles each

  // reductions / scratch
  DevBuf scratch;                // scan tiles and reduction partials
  DevBuf dscalars;               // device scalars (doubles)
  double* hscalars = nullptr;    // pinned mirror
  // mapped pinned words the small reads of a step land in (read_small)
  unsigned* hmap = nullptr;
  unsigned* hmap_dev = nullptr;
  DevBuf derr;                   // device error word
  DevBuf ticket;                 // wavefront ticket counters

  Stats stats;

  // launch accounting and optional per-phase CUDA-event timing
  long long launches = 0;
  bool prof_on = false;
  struct ProfRec {
    int cat;
    int nlaunch;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof_recs;
  std::vector<cudaEvent_t> prof_pool;

  int real_bytes() const { return prm.precision == 0 ? 8 : 4; }
};

// Timed phases (wcg_profile_*): each groups the kernels of one reference call.
enum ProfCat : int {
  P_GRID = 0,      // bbox, particle pass, activation, sort, gather
  P_P2G = 1,       // P2G gather + liquid phi + solid phi/weights
  P_GRIDOPS = 2,   // predict, assembly, pressure gradient, extrapolation, constraint
  P_MICFACTOR = 3, // MIC(0) factorisation wavefront
  P_MICSWEEP = 4,  // forward/backward triangular-solve wavefronts
  P_PCGVEC = 5,    // SpMV, dots, norms, vector updates
  P_REFINE = 6,    // FP64 residual / refinement kernels
  P_G2P = 7,       // G2P + advection
  P_OTHER = 8,     // CFL reduction, uploads/downloads
  kNumProfCats = 9
};

// RAII scope recording CUDA events around the kernels of one phase.
struct ProfScope {
  Context& c;
  int cat;
  long long l0;
  cudaEvent_t a = nullptr;
  ProfScope(Context& cc, int category);
  ~ProfScope();
};

// ---- orchestration (defined in the .cu files) -------------------------------
cudaError_t ctx_init(Context& c);
void ctx_free(Context& c);
cudaError_t upload_particles(Context& c, long long n, const double* x3,
                             const double* v3, const double* C9,
                             const double* mass, const double* vol,
                             const double* radius, bool device_ptrs);
cudaError_t download_particles(Context& c, double* x3, double* v3, double* C9,
                               bool device_ptrs);
// the same into host buffers without waiting: the copies run on copy_stream
// and overlap later work on `stream` (synchronize() waits for them)
cudaError_t download_particles_async(Context& c, double* x3, double* v3, double* C9);
cudaError_t synchronize(Context& c);
// host-to-device copies of a liquid particle set into the staging buffer on
// in_stream, without waiting (host buffers pinned and untouched until the
// staged set is loaded); load_staged() puts it into the particle arrays on
// `stream`, after whatever was queued there
cudaError_t stage_particles_async(Context& c, long long n, const double* x3, const double* v3,
                                  const double* C9, const double* mass, const double* vol,
                                  const double* radius);
cudaError_t load_staged(Context& c);
// Small device-to-host reads of a step (scalars, counts, the error word;
// bytes a multiple of 4, at most kReadSmallBytes): a kernel on `stream`
// stores them into mapped pinned memory, then the stream is synchronised.
// No copy engine is involved, so a large read-back running on copy_stream
// cannot hold them back.  A context without the mapped words (hmap null:
// one not set up by ctx_init) reads with a plain copy instead.
constexpr size_t kReadSmallBytes = 4096;
cudaError_t read_small(Context& c, const void* d, size_t bytes, void* h);
// The shared solve of a batch of contexts on one device: a coordinator thread
// runs the PCG iterations of every context waiting in its pressure solve as
// one launch per kernel, chunks of 8 iterations, admitting new solves between
// chunks.  Results are those of each solve alone.
SharedSolve* shared_solve_create(int device, std::string* err);
void shared_solve_destroy(SharedSolve* s);
long long shared_solve_launches(const SharedSolve* s);
// solves of more pencil patches than this iterate alone (default: no limit)
void shared_solve_set_limit(SharedSolve* s, int max_patches);
// positions in the reference's m_x layout (x, y, z, 0 per particle) and radii,
// original order, host buffers
cudaError_t download_positions(Context& c, double* x4, double* radius);
cudaError_t upload_positions(Context& c, const double* x4);
// elasto particles in the reference's layouts (x4/v4/m4/fm4 stride 4, B9
// row-major, orient3 stride 3), host buffers
cudaError_t upload_elasto(Context& c, long long n, const double* x4, const double* v4,
                          const double* B9, const double* m4, const double* fm4,
                          const double* rest_vol, const double* rest_vf,
                          const double* fluid_vol, const double* shape_factor,
                          const double* orient3, const int* surfel);
cudaError_t download_elasto(Context& c, double* x4, double* v4, double* B9);
cudaError_t upload_elasto_positions(Context& c, const double* x4);

// reference call sequence
cudaError_t build_grid(Context& c);                 // bbox + rebucketize + resampleNodes
cudaError_t map_particles_to_grid(Context& c);      // weights, liquid phi, solid phi/weights, P2G, sat/psi
cudaError_t step_velocity(Context& c, double dt);
cudaError_t project_fine(Context& c, double dt);
cudaError_t apply_pressure_and_extrapolate(Context& c, double dt);
cudaError_t constrain_liquid_velocity(Context& c);
cudaError_t map_grid_to_particles_and_advect(Context& c, double dt, bool advect);
cudaError_t advect_only(Context& c, double dt);
cudaError_t num_substeps(Context& c, double dt, int* n);
cudaError_t substep(Context& c, double dt);
// TwoDScene::correctLiquidParticles for the liquid particles with original
// index % correction_step == selector
cudaError_t correct_liquid_particles(Context& c, double dt, int selector);
// subset of call k of the seeded correction stream
int correction_selector(unsigned long long seed, unsigned long long k, int step);
// relabelLiquidParticles + mergeLiquidParticles + removeEmptyParticles on the
// buckets of the last grid build, with the given subset and colour order
// (perm: t, s, r permutations of {0, 1, 2}); *removed = particles removed
cudaError_t merge_liquid_particles(Context& c, int selector, const int* perm, long long* removed);
// splitLiquidParticles with the rotations of key (after relabelling);
// *added = particles appended
cudaError_t split_liquid_particles(Context& c, unsigned long long key, long long* added);
// the number of particles the split would split (after the volume update)
cudaError_t split_liquid_parents(Context& c, long long* nparents);
// the split with the caller's pattern table (kSplitPatternLen doubles) and
// nparents row-major rotations (host arrays)
cudaError_t split_liquid_particles_with(Context& c, const double* pattern, const double* rot,
                                        long long nparents, long long* added);
constexpr int kSplitPatternLen = 3 * (32 * 33 / 2 - 1);  // points of n = 2..32
cudaError_t terminate_liquid_particles(Context& c, long long* removed);
unsigned long long split_key(unsigned long long seed, unsigned long long k);
// draws of merge call k of a seeded stream: selector, then three Fisher-Yates
// permutations of {0, 1, 2}
void merge_draws(unsigned long long seed, unsigned long long k, int step, int* selector, int* perm);
// Reverse mode of substep at the current (pre-step) particle state with the
// positions held fixed: cotangents of (v', C', x') in, of (v, C) and of the
// viscosity (mubar, may be null) out (host arrays, original order; x-bar
// passes through unchanged).
// xbar0 null: positions held fixed (x-bar passes through); else the full
// x-cotangent through the transfer weights
cudaError_t substep_vjp(Context& c, double dt, const double* vbar, const double* Cbar,
                        const double* xbar, double* vbar0, double* Cbar0, double* xbar0,
                        double* mubar);
// record the message returned by wcg_last_error() on this thread; returns code
int set_last_error(int code, const std::string& msg);
// FP64 MIC(0)-PCG on a system already placed in the context's fields
// (G_ADIAG, G_AX/AY/AZ, G_B) with caller-provided buffers; writes p to out.
cudaError_t prepared_solve_fp64(Context& c, double* out, int* iters, double* res,
                                int* converged, double* rhs_norm);

}  // namespace wcg

// The C-ABI's opaque scene handle (include/wetcloth_gpu.h).
struct wcg_ctx {
  wcg::Context c;
};
