/*
 * pyro_sim.h — C ABI of the B200 (sm_100a) fire-simulation step.
 *
 * This library replaces pyro's `Sim` (src/sim.rs:42-531) and the WGSL
 * simulation kernels it dispatches (src/shaders/{advect,fluid,combust,mg}.wgsl)
 * with hand-written CUDA kernels behind plain `extern "C"` entry points:
 * no torch types, no C++ types, plain pointers and sizes.  Every entry point
 * returns an int status (PYRO_OK == 0, negative on error) and never exits the
 * process; pyro_last_error() gives a human-readable message for the calling
 * thread's last failure.
 *
 * Layout (identical to the reference, src/shaders/common.wgsl:1-7):
 *   grid nx*ny*nz cells, y up, cell index  x + nx*(y + ny*z)
 *   face arrays u, v, w each padded to (nx+1)(ny+1)(nz+1), index
 *       x + (nx+1)*(y + (ny+1)*z); u at (i, j+1/2, k+1/2) etc.
 *   s0  = (T [K], Y_F, Y_O2, Y_soot)                 float4 per cell
 *   s1  = (Y_smoke, q [W/m^3], S [1/s], 0)           float4 per cell
 *   sol = (material slot, virgin fuel, char, Ts)     float4 per cell
 *   pyr = (m'' volatiles, m'' char, exposed faces, 0) float4 per cell
 *   curl= (wx, wy, wz, |w|)                          float4 per cell
 *   flags uint32 per cell (1 = solid)
 */
#ifndef PYRO_SIM_H
#define PYRO_SIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PYRO_OK 0
#define PYRO_E_INVALID (-1)   /* bad argument (null pointer, size, dims)   */
#define PYRO_E_CUDA (-2)      /* a CUDA runtime call failed                */
#define PYRO_E_NOMEM (-3)     /* device or pinned allocation failed        */
#define PYRO_E_STATE (-4)     /* call not valid in the object's state      */
#define PYRO_E_NOCONV (-5)    /* iterative solve hit its iteration cap     */
#define PYRO_E_TIMEOUT (-6)   /* a bounded device-side wait gave up        */

/* Number of floats in the statistics block: 16 scalars + per-layer HRR
 * (src/sim.rs:12 STATS_N).  Slot meaning (src/shaders/common.wgsl:90-92):
 * 0 HRR W | 1 radiative loss W | 2 pyrolysis kg/s | 3 soot kg | 4 max T K |
 * 5 max |u| m/s | 6 fuel gas kg | 7 solid mass kg | 8 smoke kg |
 * 9 pyrolysing area m^2 | 10 sum r^2 | 11 sum b^2 | 16.. HRR per y layer W */
#define PYRO_STATS_N 1040
#define PYRO_MAX_LAYERS 1024

/* ---- the uniform parameter block -------------------------------------- */
/* Byte-for-byte the reference's `Params` (#[repr(C)], src/scene.rs:424-477,
 * WGSL struct src/shaders/common.wgsl:14-28): 48 scalars + 8 materials of
 * 12 floats = 576 bytes.  Material row: a = (density, L_g, T_p, kind),
 * b = (char yield, emissivity, c_p, k), c = (smoke yield, burn-rate
 * multiplier, 0, 0) (src/shaders/common.wgsl:9-12). */
typedef struct PyroParams {
  uint32_t nx, ny, nz, frame;
  float dx, dt, time, t0;
  float rho0, g, cp, yo2;
  float vort, cs, buoy, smoke_w;
  float wind_x, wind_z, wind_relax, sponge;
  float t_ign, s_o2, dhc, tau_min;
  float soot_form, soot_ox, soot_ox_t, smoke_conv;
  float kap_gas, h_conv, ign_on, ign_temp;
  float ign_x, ign_y, ign_z, ign_r;
  float ign_flux, ign_fuel, char_a, char_e;
  float dh_char, burnout, layer, rad_len;
  float h_mass, vort_t, rad_frac, seed;
  float mats[8][12];
} PyroParams;

/* ---- fields addressable through read/write/device_ptr ------------------- */
enum PyroField {
  PYRO_F_S0 = 0,    /* float4 * N                                         */
  PYRO_F_S1 = 1,    /* float4 * N                                         */
  PYRO_F_SOL = 2,   /* float4 * N, the current solid state (sol[sol_cur]) */
  PYRO_F_PYR = 3,   /* float4 * N                                         */
  PYRO_F_FLAGS = 4, /* uint32 * N                                         */
  PYRO_F_CURL = 5,  /* float4 * N                                         */
  PYRO_F_U = 6,     /* float * Nv, current velocity (vel[cur][0])          */
  PYRO_F_V = 7,     /* float * Nv                                         */
  PYRO_F_W = 8,     /* float * Nv                                         */
  PYRO_F_PHI = 9,   /* float * N, level-0 pressure (warm start)           */
  PYRO_F_B = 10,    /* float * N, level-0 right-hand side                 */
  /* the renderer input pack of the last pyro_sim_render_pack (none before
   * the first call): 4 IEEE binary16 values per cell                     */
  PYRO_F_RVOL = 11,   /* half4 * N: soot ppm, T K, smoke g/m^3, HRR kW/m^3 */
  PYRO_F_RSOL = 12,   /* half4 * N: occupancy, then Ts, char fraction and
                         material slot premultiplied by the occupancy     */
  PYRO_F_RVEL = 13,   /* half4 * N: cell-centred velocity m/s, 0          */
  PYRO_F_BRICKS = 14, /* float * ceil(nx/8)*ceil(ny/8)*ceil(nz/8): the
                         visibility maximum of each 8^3 brick             */
  /* the renderer's fire-light sampling tables of the last
   * pyro_sim_render_emission (none before the first call)                */
  PYRO_F_ECELL = 15,  /* float * N: emission power per cell               */
  PYRO_F_ECDF = 16    /* float * (N + 1): its cumulative distribution,
                         then the total                                   */
};

/* Pressure solver modes for pyro_sim_set_solver / pyro_poisson_solve. */
enum PyroSolver {
  PYRO_SOLVER_VCYCLE = 0,     /* fixed count of V-cycles (the reference)  */
  PYRO_SOLVER_VCYCLE_TOL = 1, /* V-cycles until relative residual <= tol  */
  PYRO_SOLVER_MGPCG = 2,      /* flexible CG, FP32 V-cycle preconditioner */
  PYRO_SOLVER_MGPCG_BF16 = 3, /* flexible CG, BF16-storage V-cycle        */
  PYRO_SOLVER_MGPCG_LEARNED = 4 /* mode 3 after the learned warm start:
                                   phi += alpha net(b - A phi) with alpha
                                   minimising the A-norm error, kept only
                                   when it lowers ||b - A phi|| (needs a
                                   network: pyro_*_set_net)              */
};

typedef struct PyroSolveInfo {
  int32_t mode;        /* PyroSolver used                                 */
  int32_t iterations;  /* V-cycles (modes 0,1) or CG iterations (2,3)     */
  double rel_resid;    /* ||b - A phi|| / ||b|| over fluid cells, FP64     */
  double b_norm;       /* ||b||                                           */
  float ms;            /* device time of the solve, CUDA events            */
  int32_t converged;   /* 1 when rel_resid <= tol                         */
  int32_t learned;     /* learned stage: -1 not run, 0 discarded, 1 kept   */
  float learned_ms;    /* device time of the learned stage                 */
  double rel_resid_start;   /* relative residual of the initial guess      */
  double rel_resid_learned; /* after the learned stage (start if discarded) */
} PyroSolveInfo;

/* The learned pressure stage (pyro_net_* below). */
typedef struct PyroNet PyroNet;

typedef struct PyroSimInfo {
  uint32_t nx, ny, nz, levels;
  uint32_t level_dims[8][3];
  uint64_t cells, faces;
  uint64_t device_bytes; /* bytes of device memory the simulation holds  */
} PyroSimInfo;

/* Thread-local text of the last error (empty string when none). */
const char* pyro_last_error(void);
/* ABI version: bump on any signature or struct change. */
int pyro_abi_version(void);

/* ---- the simulation object (replaces `Sim`) ----------------------------- */
typedef struct PyroSim PyroSim;

/* Sim::new (src/sim.rs:108-232): allocate every field on the current CUDA
 * device, set s0 to ambient (t0, 0, yo2, 0), upload the voxelized solid
 * state `sol_init` (N float4, from Scene::voxelize) into both solid
 * buffers, build the multigrid hierarchy (<= 4 levels, stop when the
 * smallest dimension is < 16, halve with ceil, h doubles;
 * src/sim.rs:142-168) and capture one substep as CUDA graphs.
 * `pressure_cycles` is the V-cycle count per substep (scene default 4). */
int pyro_sim_create(const PyroParams* params, const float* sol_init,
                    uint32_t pressure_cycles, PyroSim** out);

/* Sim::step (src/sim.rs:246-423): one substep.  The host patches dt, time
 * and ign_on exactly as src/sim.rs:247-249 does; the 576-byte parameter
 * block is uploaded on the simulation's stream.  Asynchronous: returns
 * after enqueueing.  When want_stats != 0 the statistics block is cleared
 * first, accumulated by this substep's kernels and copied to pinned host
 * memory at the end (src/sim.rs:255-257,415-417). */
int pyro_sim_step(PyroSim* sim, float dt, float time, float ign_on,
                  int want_stats);

/* Sim::read_stats raw block (src/sim.rs:510-530): waits for the last
 * stats substep and copies min(n, PYRO_STATS_N) floats. */
int pyro_sim_read_stats(PyroSim* sim, float* out, size_t n);
/* The statistics block of the stats substep before the last one: waits
 * only for that substep's copy, so a host loop can enqueue substep k and
 * then read the statistics of substep k - 1 while k runs.  Valid until the
 * next stats substep is enqueued (two copies are kept, used in turn);
 * PYRO_E_INVALID before the second stats substep. */
int pyro_sim_read_stats_prev(PyroSim* sim, float* out, size_t n);

/* Sim::read_scalars generalised (src/sim.rs:494-508): blocking copy of one
 * field in the reference layout; `bytes` must equal the field's size. */
int pyro_sim_read_field(PyroSim* sim, int field, void* host, size_t bytes);
/* Upload a field (checkpoint resume, test set-up). Blocking. */
int pyro_sim_write_field(PyroSim* sim, int field, const void* host,
                         size_t bytes);
/* Borrowed device pointer to a field, valid until the next step or
 * destroy (zero-copy consumers such as a renderer, src/render.rs:255-270). */
int pyro_sim_device_ptr(PyroSim* sim, int field, void** dptr, size_t* bytes);
/* The simulation's CUDA stream (cudaStream_t as void*). */
int pyro_sim_stream(PyroSim* sim, void** stream);
/* One substep like pyro_sim_step, launched kernel by kernel (not as a
 * graph) with CUDA events around each phase; blocks until done and writes
 * the device time in ms of each phase to ms_out[0..min(n, 12)):
 * 0 solid, 1 curl, 2 adv_vel1, 3 adv_vel2, 4 adv_s1, 5 adv_s2, 6 react,
 * 7 forces, 8 divergence, 9 pressure solve, 10 resid+project, 11 total.
 * The state advances exactly as a pyro_sim_step would. */
#define PYRO_PROFILE_PHASES 12
int pyro_sim_profile_step(PyroSim* sim, float dt, float time, float ign_on,
                          int want_stats, float* ms_out, int n);
/* The fixed V-cycle pressure solve of a substep (src/sim.rs:451-491) on the
 * simulation's current right-hand side, launched with a CUDA event after
 * every launch; blocks, leaves every field as it was (the warm start is
 * restored), and writes per launch class the summed device time in ms and
 * the launch count to ms_out / launches_out[0..min(n, 8)):
 * 0 level masks and coarse flags, 1 level-0 colour pass, 2 level-0
 * restriction, 3 prolongation onto level 0, 4 colour pass on a middle
 * level, 5 restriction from a middle level, 6 prolongation onto a middle
 * level, 7 the coarsest-level solve.  No counterpart in the reference. */
#define PYRO_PROFILE_MG_CLASSES 8
int pyro_sim_profile_pressure(PyroSim* sim, float* ms_out, int* launches_out,
                              int n);
/* Wait for all enqueued work. */
int pyro_sim_sync(PyroSim* sim);
int pyro_sim_info(PyroSim* sim, PyroSimInfo* info);
/* Choose the pressure solver used by later steps.  Mode
 * PYRO_SOLVER_VCYCLE with the create-time cycle count is the default and
 * reproduces the reference; the tolerance modes stop at rel. residual
 * `tol` or after `max_iters`. */
int pyro_sim_set_solver(PyroSim* sim, int mode, float tol, int max_iters);
/* Information on the last pressure solve of a tolerance-mode step. */
int pyro_sim_last_solve(PyroSim* sim, PyroSolveInfo* info);
/* Network used by PYRO_SOLVER_MGPCG_LEARNED (NULL detaches; the caller
 * keeps ownership and keeps it alive while attached). */
int pyro_sim_set_net(PyroSim* sim, PyroNet* net);
/* The renderer's per-frame input pack (src/shaders/render.wgsl:3-61, the
 * pack and bricks dispatches of src/render.rs:270-292) from the current
 * fields, into volumes the simulation holds (PYRO_F_RVOL, PYRO_F_RSOL,
 * PYRO_F_RVEL; PYRO_F_BRICKS when with_bricks != 0), read with
 * pyro_sim_read_field or borrowed with pyro_sim_device_ptr.  The
 * reference's rgba16float textures become linear buffers of 4 binary16
 * values per cell (cell index order, round to nearest even).  Asynchronous
 * on the simulation's stream; the first call allocates the volumes
 * (24 bytes per cell) and so must not run inside a stream capture. */
int pyro_sim_render_pack(PyroSim* sim, int with_bricks);
/* The renderer's fire-light sampling tables (src/render.rs:304-333): the
 * ecells kernel (render.wgsl:63-98) on the packed volume, then the emission
 * CDF.  The reference reads the emission back and forms the CDF on the CPU
 * (FP64 running sum, then c / total as f32, and the total last); here it
 * is an FP64 scan on the GPU.  lut_dev: the first 1024 float4 rows of the
 * renderer's colour table (soot emission, src/color.rs:46-70), on the
 * device; chemi: 4 host floats (chemiluminescence strength, soot
 * extinction per ppm at 550 nm, smoke extinction per g/m^3, 0;
 * src/render.rs:169-174).  Needs a pyro_sim_render_pack first.
 * Asynchronous on the simulation's stream; the first call allocates
 * 8 bytes per cell and so must not run inside a stream capture. */
int pyro_sim_render_emission(PyroSim* sim, const float* lut_dev,
                             const float* chemi);
int pyro_sim_destroy(PyroSim* sim);

/* ---- scene voxelizer (Scene::voxelize, src/scene.rs:621-667) ---------- */
enum PyroShapeKind {
  PYRO_SHAPE_BOX = 0, PYRO_SHAPE_CYL = 1, PYRO_SHAPE_SPHERE = 2,
  PYRO_SHAPE_POOL = 3
};
typedef struct PyroShape {
  uint32_t kind;  /* PyroShapeKind                                       */
  uint32_t slot;  /* material slot (index into PyroParams.mats)           */
  float c[3];     /* box / sphere / pool centre; cylinder end a          */
  float e[3];     /* box half sizes; cylinder end b                       */
  float r;        /* cylinder / sphere / pool radius                      */
  float depth;    /* pool depth                                           */
  float sin_yaw, cos_yaw; /* box yaw about +y                            */
} PyroShape;
/* Fill `sol_out` (device pointer, N float4) with (slot, mass, 0, t0):
 * shapes are tested in order and the last one containing the cell centre
 * wins; mass = density * (0.85 + 0.3 * hash(idx ^ seed * 0x9e3779b9)) for
 * combustible slots and 1 for inert ones.  slot_density/slot_kind are 8
 * entries each (host pointers). */
int pyro_voxelize(const PyroShape* shapes, uint32_t n_shapes, uint32_t nx,
                  uint32_t ny, uint32_t nz, float dx, float t0, uint32_t seed,
                  const float* slot_density, const uint32_t* slot_kind,
                  float* sol_out, void* stream);

/* ---- stand-alone pressure Poisson solver ------------------------------- */
/* The multigrid hierarchy of Sim::new plus the solvers, on caller-owned
 * level-0 arrays.  Operator (src/shaders/mg.wgsl:2,25-35):
 * (sum over fluid neighbours phi_n - cnt*phi)/h^2 = b where
 * out-of-domain neighbours count in cnt with phi = 0 (Dirichlet on the
 * sides and the top), y < 0 is skipped (Neumann floor) and solid
 * neighbours are skipped (Neumann at solids).  bc_mode 1 makes the sides
 * Neumann too (Dirichlet on the top face only). */
typedef struct PyroPoisson PyroPoisson;
int pyro_poisson_create(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                        int bc_mode, PyroPoisson** out);
/* Copy the level-0 solid flags (device uint32 * N) and rebuild the coarse
 * flags. */
int pyro_poisson_set_flags(PyroPoisson* ps, const uint32_t* flags);
/* Solve in place: phi (device float * N) is the initial guess and the
 * result; b (device float * N) the right-hand side.  The solve runs on the
 * solver's own stream (pyro_poisson_stream), which does not wait for other
 * streams: b, phi and the flags must be written before the call. */
int pyro_poisson_solve(PyroPoisson* ps, const float* b, float* phi, int mode,
                       float tol, int max_iters, PyroSolveInfo* info);
int pyro_poisson_stream(PyroPoisson* ps, void** stream);
/* Where a CG iteration's time goes: `iters` iterations of mode
 * PYRO_SOLVER_MGPCG or PYRO_SOLVER_MGPCG_BF16 from phi (updated in place as
 * by a solve's iterations; no convergence test, no restart), one launch at
 * a time with a CUDA event after each step instead of the solve's graph.
 * Blocks.  Per class, ms_out / launches_out[0..min(n, 9)) get the summed
 * device time and the number of steps: 0 level masks and weights (only
 * when the flag field changed), 1 level-0 colour pass, 2 restriction from
 * level 0 (residual and gather: two kernels per step), 3 prolongation onto
 * level 0, 4 colour pass on a coarser level, 5 restriction from one, 6
 * prolongation onto one, 7 the coarsest level's direct solve, 8 a CG
 * vector kernel.  Each step carries its event's overhead (a few
 * microseconds).  No counterpart in the reference. */
#define PYRO_PROFILE_CG_CLASSES 9
int pyro_poisson_profile_cg(PyroPoisson* ps, const float* b, float* phi, int mode,
                            int iters, float* ms_out, int* launches_out, int n);
/* Network used by PYRO_SOLVER_MGPCG_LEARNED (NULL detaches). */
int pyro_poisson_set_net(PyroPoisson* ps, PyroNet* net);
/* The learned stage's keep-or-discard rule, on host scalars: given
 * <r,e>, <e,Ae>, <r,Ae>, <Ae,Ae> and <r,r> for the residual r = b - A phi
 * and the network's correction e, alpha = <r,e>/<e,Ae> and the new squared
 * residual <r,r> - 2 alpha <r,Ae> + alpha^2 <Ae,Ae>.  Returns 1 (keep) when
 * alpha is finite and the new residual is finite and below <r,r>, else 0;
 * alpha and rr_new may be NULL. */
int pyro_learned_accept(double re, double eae, double rae, double aeae, double rr,
                        double* alpha, double* rr_new);
int pyro_poisson_destroy(PyroPoisson* ps);

/* ---- individual kernels (parity hooks; device pointers) ----------------- */
/* Each runs one reference kernel once on caller-owned device buffers with
 * the parameter block `params_dev` (device copy of PyroParams).  `stats`
 * (device float * PYRO_STATS_N) may be NULL to skip the statistics.
 * `stream` is a cudaStream_t or NULL for the legacy stream. */
int pyro_k_solid(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                 uint32_t nz, const float* sol_in, float* sol_out, float* pyr,
                 uint32_t* flags, const float* s0, float* stats, void* stream);
int pyro_k_curl(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                uint32_t nz, const float* u, const float* v, const float* w,
                float* curl, float* stats, void* stream);
/* adv_vel1 then adv_vel2; allocates a temporary device buffer for the
 * predictor's limiter bounds and returns after the stream has finished. */
int pyro_k_adv_vel(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                   uint32_t nz, const float* u, const float* v, const float* w,
                   float* hu, float* hv, float* hw, float* ou, float* ov,
                   float* ow, const uint32_t* flags, void* stream);
int pyro_k_adv_scalars(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                       uint32_t nz, const float* u, const float* v,
                       const float* w, const float* s0, const float* s1,
                       float* h0, float* h1, float* o0, float* o1,
                       void* stream);
int pyro_k_react(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                 uint32_t nz, const float* s0in, const float* s1in,
                 float* s0out, float* s1out, const uint32_t* flags,
                 const float* sol, const float* pyr, const float* curl,
                 float* stats, void* stream);
int pyro_k_forces(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                  uint32_t nz, float* u, float* v, float* w, const float* s0,
                  const float* s1, const float* curl, const uint32_t* flags,
                  void* stream);
/* pyro_k_forces without any device allocation (no counterpart in the
 * reference).  For callers that cannot allocate device memory -- code running
 * while another thread captures a CUDA graph, hosts whose pool allocator owns
 * all device memory, loops that cannot afford cudaMalloc's implicit
 * synchronisation -- the per-cell confinement scratch lives in a fixed
 * device array of PYRO_NOALLOC_MAX_CELLS float4 (8 MiB) that the library
 * holds on every GPU that loads it until the process exits.  Grids with more
 * cells are rejected with PYRO_E_INVALID.  The first call on a device, with
 * that device current, looks up the array's device address; make that first
 * call before any stream capture.  All calls share the one array: calls that
 * overlap on the GPU (different streams, other threads) race on it and must
 * be serialised by the caller.  Results equal pyro_k_forces.  The call is
 * stream-ordered: it queues the kernels on `stream` and returns without
 * waiting (pyro_k_forces waits, to free its scratch), so an error raised by
 * a running kernel shows up at the caller's next synchronisation of that
 * stream.  The array's device address is looked up once per device and kept
 * for the process: a cudaDeviceReset after the first call on a device is not
 * supported. */
#define PYRO_NOALLOC_MAX_CELLS (1u << 19)
int pyro_k_forces_noalloc(const PyroParams* params_dev, uint32_t nx,
                          uint32_t ny, uint32_t nz, float* u, float* v,
                          float* w, const float* s0, const float* s1,
                          const float* curl, const uint32_t* flags,
                          void* stream);
int pyro_k_divergence(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                      uint32_t nz, const float* u, const float* v,
                      const float* w, const float* s1, const uint32_t* flags,
                      float* b, void* stream);
int pyro_k_project(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                   uint32_t nz, float* u, float* v, float* w, const float* phi,
                   const uint32_t* flags, void* stream);
/* Multigrid kernels on one level (dims, spacing h), with the reference's
 * per-cell solid flags: mg_smooth (mg.wgsl:5-36), mg_restrict
 * (mg.wgsl:38-83, also writes the coarse flags) and mg_prolong
 * (mg.wgsl:85-120).  They run the kernels the V-cycle launches: the level's
 * neighbour masks are built into a temporary buffer first, and each call
 * waits for its stream before returning. */
int pyro_k_mg_smooth(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                     const float* b, const uint32_t* flags, float* phi,
                     int color, float omega, void* stream);
int pyro_k_mg_restrict(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh,
                       const float* pf, const float* bf, const uint32_t* ff,
                       uint32_t cnx, uint32_t cny, uint32_t cnz, float* bc,
                       float* pc, uint32_t* fc, void* stream);
int pyro_k_mg_prolong(uint32_t fnx, uint32_t fny, uint32_t fnz,
                      const float* pc, const uint32_t* ff, float* pf,
                      uint32_t cnx, uint32_t cny, uint32_t cnz,
                      const uint32_t* fc, void* stream);
/* The same kernels on caller-owned neighbour masks, as the V-cycle runs
 * them, with the storage of phi and b selectable (FP32, or BF16 with FP32
 * arithmetic: the MGPCG preconditioner) and bc_mode as
 * pyro_poisson_create.  The mask byte of a cell (pyro_k_mg_meta): bit k =
 * neighbour k (+x, -x, +y, -y, +z, -z) is inside the level and fluid, bit 6
 * = the cell is solid.  pyro_k_mg_flags_down gives the coarse solid flags
 * (every in-domain child solid, mg.wgsl:73-82).  Asynchronous on `stream`. */
#define PYRO_MG_F32 0
#define PYRO_MG_BF16 1
int pyro_k_mg_meta(uint32_t nx, uint32_t ny, uint32_t nz,
                   const uint32_t* flags, uint8_t* meta, void* stream);
int pyro_k_mg_flags_down(uint32_t fnx, uint32_t fny, uint32_t fnz,
                         const uint32_t* ff, uint32_t cnx, uint32_t cny,
                         uint32_t cnz, uint32_t* fc, void* stream);
int pyro_k_mg_pass(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                   const void* b, const uint8_t* meta, void* phi, int color,
                   float omega, int bc_mode, int storage, void* stream);
int pyro_k_mg_restrict_m(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh,
                         const void* pf, const void* bf, const uint8_t* mf,
                         uint32_t cnx, uint32_t cny, uint32_t cnz, void* bc,
                         void* pc, int bc_mode, int storage, void* stream);
int pyro_k_mg_prolong_m(uint32_t fnx, uint32_t fny, uint32_t fnz,
                        const void* pc, const uint8_t* mf, void* pf,
                        uint32_t cnx, uint32_t cny, uint32_t cnz,
                        const uint8_t* mc, int storage, void* stream);
/* The MGPCG preconditioner's restriction R = P^T / 8, P the fluid-weighted
 * trilinear prolongation of pyro_k_mg_prolong_m: the residual
 * r = b - A phi of each fluid fine cell, divided by its prolongation row's
 * fluid weight sum, gathered into each fluid coarse cell with P's weights
 * and divided by 8 (bc); the coarse guess pc is set to 0.  Waits for the
 * stream (it allocates its temporaries). */
int pyro_k_mg_restrict_sym(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh,
                           const void* pf, const void* bf, const uint8_t* mf,
                           uint32_t cnx, uint32_t cny, uint32_t cnz,
                           const uint8_t* mc, void* bc, void* pc, int bc_mode,
                           int storage, void* stream);
/* The fused first and last level-0 passes of the MGPCG preconditioner's
 * V-cycle.  pass_first:
 * the pass of `color` from phi = 0 with the FP32 right-hand side r, every
 * cell of phi written (cells not updated get 0); with BF16 storage r is
 * also written rounded to BF16 into bq and used rounded.  pass_last: the
 * pass of `color` on BF16 phi and b, its result (every cell) written
 * widened to FP32 into out, phi left as it was.  Each equals the plain
 * pyro_k_mg_pass on the cleared / converted buffers bit for bit. */
int pyro_k_mg_pass_first(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                         const float* r, void* bq, const uint8_t* meta,
                         void* phi, int color, float omega, int bc_mode,
                         int storage, void* stream);
int pyro_k_mg_pass_last(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                        const void* b, const uint8_t* meta, void* phi,
                        float* out, int color, float omega, int bc_mode,
                        void* stream);
int pyro_k_mg_resid(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                    const float* phi, const float* b, const uint32_t* flags,
                    float* stats, void* stream);
/* Renderer input pack on explicit buffers (render.wgsl:3-36): s0, s1, sol
 * float4 * N, flags u32 * N, u, v, w face arrays; vol, sol_out, vel receive
 * 4 binary16 values per cell (8 * N bytes each). */
int pyro_k_render_pack(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                       uint32_t nz, const float* s0, const float* s1,
                       const float* sol, const uint32_t* flags, const float* u,
                       const float* v, const float* w, void* vol, void* sol_out,
                       void* vel, void* stream);
/* Emission power per cell (render.wgsl:63-98) from a packed vol volume;
 * lut (device) and chemi (host) as pyro_sim_render_emission. */
int pyro_k_render_ecells(const PyroParams* params_dev, uint32_t nx,
                         uint32_t ny, uint32_t nz, const void* vol,
                         const float* lut, const float* chemi, float* ecell,
                         void* stream);
/* The emission CDF of n values into cdf (n + 1 floats; src/render.rs:316-333).
 * Allocates its scratch and blocks until done. */
int pyro_k_render_cdf(uint64_t n, const float* ecell, float* cdf, void* stream);
/* Brick maxima (render.wgsl:38-61) from packed vol and sol volumes into
 * bricks, float * ceil(nx/8)*ceil(ny/8)*ceil(nz/8), x fastest. */
int pyro_k_render_bricks(uint32_t nx, uint32_t ny, uint32_t nz,
                         const void* vol, const void* sol_packed, float* bricks,
                         void* stream);

/* The volume path tracer's uniform block (struct RP of
 * src/shaders/trace_lib.wgsl:1-14, filled by src/render.rs:180-210 and per
 * frame / dispatch at src/render.rs:335-337, 410-412): 13 rows of 16 bytes,
 * the same layout. */
typedef struct PyroRenderParams {
  uint32_t res[4];   /* width, height, first sample index, samples now     */
  uint32_t dims[4];  /* nx, ny, nz, frame number                           */
  float cam_pos[4];  /* camera position, tan(half field of view)           */
  float cam_fwd[4];  /* forward unit vector, aspect (width / height)       */
  float cam_right[4];/* right unit vector, aperture radius (m)             */
  float cam_up[4];   /* up unit vector, focus distance (m)                 */
  float a[4];        /* dx (m), march step (cells), shutter (s), sky       */
  float b[4];        /* ground on, ground albedo, bounces, chemi strength  */
  float soot[4];     /* soot extinction per ppm (rgb, 1/m), soot albedo    */
  float c[4];        /* smoke extinction (m^2/g), smoke albedo, HG g, T0   */
  float alb[8];      /* surface albedo per material slot                   */
  float gc[4];       /* ground cache x0, z0, side (m); mode: 1 light cache,
                        0 pure path tracing                                */
} PyroRenderParams;

/* The path tracer's kernels on explicit device buffers.  `rp` is a HOST
 * pointer (copied into the launch).  vol, sol, vel: the packed volumes of
 * pyro_k_render_pack (rp->dims cells, 4 binary16 each); bricks as
 * pyro_k_render_bricks; lut: the colour table, 2048 float4 rows (soot
 * emission, then surface emission; src/color.rs:46-75); ecdf: the emission
 * CDF of pyro_k_render_cdf (cells + 1 floats).  Light-cache volumes are
 * (lz, ly, lx) cells of 4 binary16 values, x fastest; the reference sizes
 * them ceil(n / 2) per axis (src/render.rs:104); the ground cache is
 * gres x gres (256 in the reference, src/render.rs:12). */

/* lightvol (render.wgsl:217-251): per cache cell, `rays` next-event shadow
 * rays (96 in the reference) toward the fire; lvA = mean flux (rgb, 0),
 * lvB = luminance-weighted mean direction (xyz, 0). */
int pyro_k_render_lightvol(const PyroRenderParams* rp, const void* vol,
                           const void* sol, const void* vel,
                           const float* bricks, const float* lut,
                           const float* ecdf, uint32_t lx, uint32_t ly,
                           uint32_t lz, uint32_t rays, void* lvA, void* lvB,
                           void* stream);
/* lightground (render.wgsl:253-269): ground irradiance per texel of the
 * gres x gres cache over the square rp->gc, `rays` shadow rays (128). */
int pyro_k_render_lightground(const PyroRenderParams* rp, const void* vol,
                              const void* sol, const void* vel,
                              const float* bricks, const float* lut,
                              const float* ecdf, uint32_t gres, uint32_t rays,
                              void* gE, void* stream);
/* blur (render.wgsl:271-304): Gaussian of radius `radius` (1..16) along
 * `axis` (0 = x, 1 = y, 2 = z), clamp-to-edge, src -> dst (distinct
 * buffers of nx*ny*nz cells of 4 binary16 values). */
int pyro_k_render_blur(const void* src, void* dst, uint32_t nx, uint32_t ny,
                       uint32_t nz, uint32_t axis, uint32_t radius,
                       void* stream);
/* trace (render.wgsl:132-215): for each pixel of rp->res.xy, adds the sum
 * of samples rp->res.z .. rp->res.z + rp->res.w - 1 to accum (float4 per
 * pixel: rgb, sample count).  Light-cache mode (rp->gc[3] > 0.5) reads the
 * blurred caches lvA, lvB (lx, ly, lz) and gE (gres); pure path tracing
 * (rp->b[2] bounces) ignores them (they may be NULL). */
int pyro_k_render_trace(const PyroRenderParams* rp, const void* vol,
                        const void* sol, const void* vel, const float* bricks,
                        const float* lut, const float* ecdf, const void* lvA,
                        const void* lvB, uint32_t lx, uint32_t ly, uint32_t lz,
                        const void* gE, uint32_t gres, float* accum,
                        void* stream);

/* ---- frame development (src/post.rs:25-160, CPU code in the reference) --- */
/* The tracer's accumulation image `accum` (w*h float4: radiance sums and
 * sample count) to its mean radiance `img` (w*h*3 floats, sums divided by
 * max(count, 1)), and the k-th smallest pixel luminance
 * 0.2126 r + 0.7152 g + 0.0722 b (k counted from 0; the auto exposure uses
 * k = min(floor(0.995 w h), w h - 1), post.rs:31-35) into *kth (host),
 * exactly.  keys: w*h uint32 scratch, sel: PYRO_POST_SEL_WORDS uint32
 * scratch (device).  Blocks until *kth is available. */
#define PYRO_POST_SEL_WORDS 260
int pyro_post_select(const float* accum, uint32_t w, uint32_t h, uint32_t k,
                     float* img, uint32_t* keys, uint32_t* sel, float* kth,
                     void* stream);
/* img * gain, then with glare > 0 the three box-blurred glare scales mixed
 * in (post.rs:90-160, the box filters' running sums in the reference's
 * order), the ACES curve, sRGB, the per-pixel dither and 8-bit
 * quantisation into out (w*h*3 bytes, device).  scratch: 12*w*h floats;
 * lin_out (optional, w*h*3 floats) receives the linear image after the
 * glare mix.  Asynchronous on `stream`.  The gain 2^exposure comes from the
 * host's exposure state (pyro_b200.post.Camera). */
int pyro_post_develop(const float* img, uint32_t w, uint32_t h, float gain,
                      float glare, float* scratch, uint8_t* out,
                      float* lin_out, void* stream);

/* q = A p, the pressure operator of the multigrid levels (mg.wgsl:25-35:
 * (sum of fluid neighbours - count * p) / h^2, Dirichlet faces counted as
 * bc_mode says), evaluated in FP64 and rounded; 0 in solid cells.  The
 * operator of CG solvers built on the level kernels.  Asynchronous on
 * `stream`. */
int pyro_k_mg_apply(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                    const uint32_t* flags, const float* p, float* q,
                    int bc_mode, void* stream);
/* Coarsest-level solve: `iters` red-black SOR sweeps (omega) in one
 * launch (src/sim.rs:473 runs 80 sweeps at omega 1.6 as 160 dispatches). */
int pyro_k_mg_coarse(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                     const float* b, const uint32_t* flags, float* phi,
                     int iters, float omega, void* stream);
/* Coarsest-level solve of the symmetric V-cycle (MGPCG preconditioner):
 * `iters` SOR iterations alternating red-black and black-red (iteration
 * it starts with colour it & 1); bc_mode as pyro_poisson_create.  No
 * counterpart in the reference. */
int pyro_k_mg_coarse_sym(uint32_t nx, uint32_t ny, uint32_t nz, float h,
                         const float* b, const uint32_t* flags, float* phi,
                         int iters, float omega, int bc_mode, void* stream);

/* ---- learned warm start: tcgen05 convolutions --------------------------- */
/* 3x3x3 convolution, padding 1, stride 1, as an implicit GEMM on the
 * tensor cores (BF16 operands, FP32 accumulation in TMEM).  BF16 activations
 * of C channels over V = nb*nz*ny*nx voxels (x fastest) are stored as C/8
 * planes of [V][8 channels] when C is a multiple of 8, else as [V][C]; FP32
 * outputs (y_f32, dx_f32) as [V][C].  Weights BF16 [Cout][27][Cin] with
 * tap = (dz+1)*9 + (dy+1)*3 + (dx+1).  Channels 1..128.  Blocking; returns
 * PYRO_E_TIMEOUT if a bounded tensor-core wait ran out.  No counterpart in
 * the reference (its pressure solve has no learned stage). */
int pyro_conv3_forward(const void* x, int C, int nx, int ny, int nz, int nb,
                       const void* w, int Cout, const float* bias, int relu,
                       void* y, int y_f32, void* stream);
/* dx = conv^T(dy, W), zeroed where `act` (the layer input, may be NULL) is
 * <= 0, i.e. the ReLU derivative of the producing layer. */
int pyro_conv3_backward_data(const void* dy, int Cout, int nx, int ny, int nz,
                             int nb, const void* w, int Cin, const void* act,
                             void* dx, int dx_f32, void* stream);
/* dw[co][tap][ci] += sum over voxels of dy[v][co] * x[v + tap][ci]; dw is
 * FP32 and accumulated into (zero it first). */
int pyro_conv3_backward_weight(const void* x, int Cin, const void* dy, int Cout,
                               int nx, int ny, int nz, int nb, float* dw,
                               void* stream);

/* ---- learned pressure stage (no counterpart in the reference) ----------
 * A 3-level 3D convolutional encoder-decoder (16/32/64 channels, 3x3x3
 * convolutions on the tcgen05 kernels above, BF16 weights and activations,
 * FP32 accumulation) from (b, solid mask) to a pressure estimate
 * phi = net(b / rms(b)) * out_scale * rms(b) * h^2 on fluid cells.  Inputs
 * are nb volumes of nx*ny*nz cells stacked (x fastest), flags as the
 * simulation's (1 = solid); all pointers are device memory.  Parameters are
 * FP32: every layer's weights [Cout][27][Cin] in order, then every layer's
 * biases.  `stream` may be NULL (the network's own stream).  The multigrid
 * solve of src/sim.rs:451-491 remains the fallback (PYRO_SOLVER_MGPCG_LEARNED
 * below). */
int pyro_net_create(uint64_t seed, PyroNet** out);
int pyro_net_destroy(PyroNet* net);
int pyro_net_param_count(const PyroNet* net, uint64_t* count);
int pyro_net_get_params(PyroNet* net, float* host, uint64_t count, float* out_scale);
/* also resets the Adam state */
int pyro_net_set_params(PyroNet* net, const float* host, uint64_t count, float out_scale);
/* phi (device, nb*nx*ny*nz FP32) = the network's estimate; synchronous */
int pyro_net_forward(PyroNet* net, const float* b, const uint32_t* flags, uint32_t nx,
                     uint32_t ny, uint32_t nz, uint32_t nb, float h, float* phi,
                     void* stream);
/* Training loss = w_phi * mean over fluid cells of
 *   (out - phi_t / (out_scale rms(b) h^2))^2
 * + w_res * mean over the fluid cells with all six neighbours inside the
 *   volume of res^2, res = b / rms(b) - out_scale (sum of the fluid
 *   neighbours' out - their count * out), the normalised residual of the
 *   prediction under the solver's operator (solid neighbours excluded).
 * Defaults w_phi = 1, w_res = 0; both >= 0, not both 0. */
int pyro_net_set_loss(PyroNet* net, float w_phi, float w_res);
/* loss and, in grad_host (may be NULL), d loss / d params; synchronous */
int pyro_net_loss_grad(PyroNet* net, const float* b, const uint32_t* flags,
                       const float* phi_t, uint32_t nx, uint32_t ny, uint32_t nz,
                       uint32_t nb, float h, double* loss, float* grad_host, void* stream);
/* loss, gradients and one Adam step (gradient global norm clipped to
 * `clip` when clip > 0); asynchronous on the stream */
int pyro_net_train_step(PyroNet* net, const float* b, const uint32_t* flags,
                        const float* phi_t, uint32_t nx, uint32_t ny, uint32_t nz,
                        uint32_t nb, float h, float lr, float clip, void* stream);
/* waits for the stream and reads the loss of the last step */
int pyro_net_last_loss(PyroNet* net, double* loss, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PYRO_SIM_H */
