/*
 * lbm3d.h — C ABI of liblbm3d.so, the sm_100a implementation of the LBM3D_BB
 * single-domain time step (D3Q19, BGK/TRT, bounce-back solids, face boundaries,
 * momentum-exchange forces).
 *
 * Conventions of every entry point:
 *   - plain pointers and sizes, no framework types; a context (lbm_ctx*) owns the
 *     population storage on one CUDA device;
 *   - the return value is a status (LBM_OK == 0); lbm_last_error() gives the
 *     message of the last failure on that context (lbm_global_error() when no
 *     context exists yet);
 *   - work is enqueued on the stream set by lbm_set_stream() (default: the
 *     legacy default stream) and is asynchronous unless the entry point
 *     returns host data (documented per function);
 *   - lattice directions are 0-based in this header.  The reference numbers them
 *     1..19 (Utilities.jl:949-960); link exports (lbm_get_links) keep the
 *     reference's 1-based numbering so they compare bit-for-bit with its CSR.
 *
 * Each entry point names the reference interface it replaces (file:line inside
 * the LBM3D_BB project).
 */
#ifndef LBM3D_H
#define LBM3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM3D_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------- */
enum {
  LBM_OK = 0,
  LBM_ERR_ARG = 1,         /* invalid argument (null pointer, bad size, bad enum) */
  LBM_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  LBM_ERR_STATE = 3,       /* call not valid in the context's current state */
  LBM_ERR_UNSUPPORTED = 4, /* valid request this build does not implement (e.g. q=27) */
  LBM_ERR_PARSE = 5,       /* params.txt parse/validation failure */
  LBM_ERR_NUMERIC = 6,     /* non-finite populations detected by lbm_check() */
  LBM_ERR_CAPACITY = 7,    /* caller buffer too small (lbm_get_links) */
  LBM_ERR_TIMEOUT = 8      /* a bounded wait inside a kernel gave up; the kernel returned and the
                              context stays usable (lbm_synchronize, lbm_wait_selftest) */
};

/* ---- enums ----------------------------------------------------------------- */
/* Physics mode.
 * LBM_MODE_REFERENCE reproduces the reference step exactly as MainCore.jl:245-379
 *   drives it: solids are collided and streamed as virtual fluid, z is periodic,
 *   inlet (x=1) and y walls are moving-wall bounce-back at U_inf, the outlet
 *   (x=Nx) is anti-bounce-back, the solid is moving-wall simple bounce-back.
 * LBM_MODE_CONFIG is the configurable single-buffer (AA pattern) solver: per-face
 *   boundary kinds, periodic axes, Guo body force, static + one moving body with
 *   fresh-node equilibrium refill, FP32 / FP64 / FP16-deviation storage. */
enum { LBM_MODE_REFERENCE = 0, LBM_MODE_CONFIG = 1 };
enum { LBM_COLL_BGK = 0, LBM_COLL_TRT = 1 };
enum { LBM_STORE_FP32 = 0, LBM_STORE_FP64 = 1, LBM_STORE_FP16DEV = 2 };

/* Face kinds (config mode). Face index: 0 x-lo, 1 x-hi, 2 y-lo, 3 y-hi, 4 z-lo, 5 z-hi.
 * Both faces of an axis must be PERIODIC or neither. */
enum {
  LBM_FACE_PERIODIC = 0,
  LBM_FACE_WALL = 1,     /* half-way bounce-back, wall velocity face_u[f] (0: no-slip) */
  LBM_FACE_EQ_INLET = 2, /* unknown populations set to feq(rho_node, face_u[f]) */
  LBM_FACE_OUTFLOW = 3,  /* zero-gradient: unknown population = same node's post-collision value */
  LBM_FACE_PRESSURE = 4, /* pressure outlet: anti-bounce-back at rho0 with the node's velocity
                            (the outlet rule of velocity_BC!_gpu, OtherBC.jl:153-166, with the
                            density fixed to rho0 instead of the node's) */
  LBM_FACE_HALO = 5      /* z faces only: the plane on this face is a ghost plane of a z-slab
                            decomposition (lbm_halo_pack / lbm_halo_unpack); it is never updated,
                            and its nodes are ordinary fluid or solid neighbours of the slab */
};

/* Body kinds. CYLINDER_Z and NACA_Z are the reference's extruded shapes
 * (Geometry.jl:49-87, evaluated in FP32 exactly as there); SPHERE and ELLIPSOID
 * are 3-D shapes evaluated in FP64. */
enum { LBM_BODY_CYLINDER_Z = 1, LBM_BODY_NACA_Z = 2, LBM_BODY_SPHERE = 3, LBM_BODY_ELLIPSOID = 4 };

/* Layouts for population import/export. */
enum {
  LBM_LAYOUT_SOA = 0,      /* f[d * N + node] */
  LBM_LAYOUT_REFERENCE = 1 /* f[d + q * node]: the reference's column-major f[d, node] */
};
enum { LBM_DTYPE_F32 = 0, LBM_DTYPE_F64 = 1 };
enum { LBM_HOST = 0, LBM_DEVICE = 1 };

/* ---- configuration --------------------------------------------------------- */
/* Node (ix, iy, iz), 0-based, has linear index ix + nx*(iy + ny*iz) — the
 * reference's global order (Partitioning.jl:23-28, 1-based there) — and sits at
 * lattice position (ix + 0.5, iy + 0.5, iz + 0.5) (Utilities.jl:550-551). */
typedef struct {
  int32_t nx, ny, nz;
  int32_t q;          /* must be 19 */
  int32_t mode;       /* LBM_MODE_* */
  int32_t collision;  /* LBM_COLL_* */
  int32_t storage;    /* LBM_STORE_* (reference mode: FP32 or FP64) */
  int32_t face[6];    /* LBM_FACE_* (config mode) */
  int32_t compute_force; /* accumulate momentum-exchange force/torque every step */
  double omega_p;     /* 1/tau (BGK) or 1/tau_plus (TRT) */
  double omega_m;     /* 1/tau_minus (TRT) */
  double rho0;        /* rest density: FP16-deviation offset, refill density */
  double face_u[6][3];/* wall / inlet velocity per face (config mode) */
  double accel[3];    /* uniform body acceleration g: Guo force rho*g (config mode) */
  double u_inf[3];    /* reference mode: U_inf, V_inf, W_inf (Parameters.jl:24-26) */
  double h;           /* reference mode: physical length per cell (Parameters.jl:13) */
  int32_t force_history; /* capacity of the per-step device force ring (>= 1) */
  int32_t solid_bc;   /* LBM_SOLID_* (reference mode; config mode takes LBM_SOLID_SBB) */
} lbm_config;

/* Solid boundary rule of the reference-mode step (solid_BC!, SolidBC.jl:99-153).
 * LBM_SOLID_SBB: moving-wall simple bounce-back, SBB!_gpu (SolidBC.jl:160-210).  The
 *   reference's "IBB" executes this same rule on its bodies: IBB!_gpu evaluates phi at
 *   x_b - c_dir, a fluid node for a convex body, so it always takes its SBB fallback
 *   (SolidBC.jl:290-319), and its interpolating branch needs EPS_Q, defined nowhere.
 * LBM_SOLID_IBB: the interpolated bounce-back IBB!_gpu is written to be (SolidBC.jl:253-338):
 *   linear interpolation (Bouzidi) with q from phi at x_b and at the solid node x_b + c_dir,
 *   the wall point x_b + q c_dir, the fluid-side neighbour x_b - c_dir for q <= 1/2 (z wraps
 *   as in streaming; outside the x/y range the same-node branch), and
 *   q clamped to [1e-4, 1 - 1e-4]; links without a sign change of phi bounce back at the
 *   half-link point x_b + c_dir/2.  Needs the moving body (cylinder or NACA band). */
enum { LBM_SOLID_SBB = 0, LBM_SOLID_IBB = 1 };

/* A rigid body. Reference shapes use centre/theta in physical units (divided by h
 * inside, as MainCore.jl:136-137 does for the node coordinates); config shapes
 * use lattice units. */
typedef struct {
  int32_t kind;        /* LBM_BODY_* */
  int32_t moving;      /* 1: pose-driven through lbm_update_body (at most one body) */
  double center[3];
  double radius;       /* CYLINDER_Z, SPHERE */
  double semi[3];      /* ELLIPSOID semi-axes (body frame) */
  double rot[9];       /* ELLIPSOID orientation, row-major body->world rotation */
  /* NACA_Z (Geometry.jl:14-39): chord, camber m, camber position p, thickness t,
   * trailing-edge squeeze x_int, pivot-to-leading-edge offset along the chord. */
  double chord, naca_m, naca_p, naca_t, x_int, x_le_offset;
} lbm_body;

/* Pose of the moving body.  Flags use the pose at t = (n-1) dt and wall
 * kinematics the pose at t = (n-1/2) dt (Motion.jl:62-63). */
typedef struct {
  double center[3];    /* body reference point */
  double cos_theta, sin_theta; /* planar rotation (reference shapes), host-evaluated */
  double rot[9];       /* full rotation (config ELLIPSOID), row-major body->world */
  double vel[3];       /* translational velocity, lattice units per step */
  double omega[3];     /* angular velocity, radians per step */
} lbm_pose;

/* params.txt, as read by read_params_input (Parameters.jl:87-164) into LBMParams
 * (Parameters.jl:8-82), FP32 derived quantities included. */
typedef struct {
  int32_t Nx, Ny, Nz;
  float h, R, x_c, y_c, theta0; /* theta0 in radians */
  int32_t q;
  float Re, U_inf, V_inf, W_inf, rho_inf, dt;
  int32_t n_max, n_save;
  float nu, omega_p, omega_m, Lambda;
  char bc[16];
  char coll[16];
  int32_t shape;       /* 1: CYL, 2: AIR */
  char naca_code[8];   /* "" when absent */
  float chord;
} lbm_params;

typedef struct lbm_ctx lbm_ctx;

/* ---- library --------------------------------------------------------------- */
int32_t lbm_abi_version(void);
const char* lbm_status_string(int32_t status);
/* Message of the last failure of a call that had no context (create, parse). */
const char* lbm_global_error(void);

/* Replaces read_params_input (Parameters.jl:87-164) and the LBMParams constructor
 * (Parameters.jl:49-81): same line grammar, same 19 positional numbers, same
 * defaults (Coll -> BGK, NACA -> 0012 for AIR) and same assertions, reported as
 * LBM_ERR_PARSE with the assertion text. */
int32_t lbm_read_params(const char* path, lbm_params* out);

/* D3Q19 constants of gen_lattice_sets (Utilities.jl:945-993) with 0-based
 * opposite indices; weights are the FP32-rounded rationals. */
int32_t lbm_lattice(int32_t q, int8_t* cx, int8_t* cy, int8_t* cz, float* w, int8_t* opp);

/* ---- context lifecycle ------------------------------------------------------ */
/* Replaces worker_alloc (Initialization.jl:89-105) and init_bb_buffers!
 * (Initialization.jl:109-130): allocates populations, flags and macro arrays on
 * `device` for cfg->nx*ny*nz nodes.  Blocking. */
int32_t lbm_create(const lbm_config* cfg, int32_t device, lbm_ctx** out);
int32_t lbm_destroy(lbm_ctx* ctx);
const char* lbm_last_error(const lbm_ctx* ctx);
/* Launches go to `stream` (a cudaStream_t, e.g. CUDA.jl's stream().handle). */
int32_t lbm_set_stream(lbm_ctx* ctx, void* stream);
int32_t lbm_synchronize(lbm_ctx* ctx);
/* Bytes of device memory the context holds. */
int64_t lbm_device_bytes(const lbm_ctx* ctx);
/* Thread-block shape of the step kernels (bx along x, by along y; bx*by a
 * multiple of 32, at most 256).  Chosen per lattice size by the autotuner; no
 * reference counterpart (CUDA.jl launches 256 threads, Collision.jl:95-96). */
int32_t lbm_set_launch(lbm_ctx* ctx, int32_t bx, int32_t by);
int32_t lbm_get_launch(const lbm_ctx* ctx, int32_t* bx, int32_t* by);

/* ---- geometry --------------------------------------------------------------- */
/* Replaces init_solid_mask_state (Geometry.jl:26-39) + the body part of
 * LBMParams.  A static body is rasterised once; the moving body is rasterised by
 * lbm_update_body at every step.  Bodies are added before the first step. */
int32_t lbm_add_body(lbm_ctx* ctx, const lbm_body* body);
/* Bulk static spheres: xyzr[4*i..4*i+3] = centre x, y, z, radius (lattice units,
 * periodic images on periodic axes).  Config mode only. */
int32_t lbm_add_spheres(lbm_ctx* ctx, int32_t count, const double* xyzr);
/* Replaces motion! (Motion.jl:41-122): solid flags at pose_n
 * (generate_mask_s_local!, Geometry.jl:92-117), boundary flags
 * (generate_mask_bb_local!, Geometry.jl:153-173) and the wall kinematics of
 * pose_half used by the bounce-back (SolidBC.jl:195-203).  The link CSR of
 * compile_bb_data! (Geometry.jl:268-311) is not materialised on the hot path —
 * links are resolved from the flags inside the step kernel — and is produced on
 * demand by lbm_get_links. */
int32_t lbm_update_body(lbm_ctx* ctx, const lbm_pose* pose_n, const lbm_pose* pose_half);

/* ---- initial state ----------------------------------------------------------- */
/* Replaces initialize_f (Initialization.jl:57-80) followed by compute_macros!
 * (MainCore.jl:221): populations set to feq(rho, u) per node.  Null arrays mean
 * uniform rho0 / zero velocity; arrays are host, length nx*ny*nz, FP64.  The
 * reference's random velocity perturbation is passed in through u/v/w. */
int32_t lbm_init_equilibrium(lbm_ctx* ctx, const double* rho, const double* u, const double* v,
                             const double* w);
/* Sets the populations S_n (pre-collision state) from a caller array in `layout`.
 * Restart/checkpoint load; pairs with lbm_get_populations. */
int32_t lbm_set_populations(lbm_ctx* ctx, const void* f, int32_t dtype, int32_t layout, int32_t where);

/* ---- time stepping ------------------------------------------------------------ */
/* One call = `nsteps` reference time steps (MainCore.jl:245-379 bodies) with the
 * current flags/kinematics.  Replaces, fused into one kernel per step:
 *   collision! (Collision.jl:14-45, BGK :212-242, TRT :112-174),
 *   streaming! (Streaming.jl:116-137), periodic_BC! (OtherBC.jl:87-107),
 *   solid_BC! SBB (SolidBC.jl:129-248), velocity_BC! (OtherBC.jl:174-219),
 *   the per-node part of compute_aero! (MEA.jl:76-116) and compute_macros!
 *   (ComputeMacro.jl:11-48, reference mode keeps rho/u/v/w current every step). */
int32_t lbm_step(lbm_ctx* ctx, int32_t nsteps);
/* Completed steps since initialisation. */
int64_t lbm_step_count(const lbm_ctx* ctx);
/* Kernels launched by lbm_step on this context so far (step kernels and the
 * moving-body flag kernels); no reference counterpart. */
int64_t lbm_launch_count(const lbm_ctx* ctx);

/* ---- outputs ------------------------------------------------------------------ */
/* Replaces compute_aero!'s reduction (MEA.jl:30-54): momentum-exchange force
 * (out[0..2]) and torque about the moving body's half-step centre (out[3..5]) of
 * step `step` (1-based, within the last force_history steps), FP64, lattice units.
 * Blocking (device->host copy of 48 bytes). */
int32_t lbm_get_force(lbm_ctx* ctx, int64_t step, double out[6]);
/* Forces of steps first..first+count-1 into out[6*count] (blocking). */
int32_t lbm_get_force_history(lbm_ctx* ctx, int64_t first, int32_t count, double* out);
/* Replaces compute_macros! (ComputeMacro.jl:53-83): rho, u, v, w of the current
 * state into caller arrays (dtype, host or device).  Config mode writes 0 at solid
 * nodes. */
int32_t lbm_get_macros(lbm_ctx* ctx, void* rho, void* u, void* v, void* w, int32_t dtype,
                       int32_t where);
/* Current pre-collision populations S_n (the reference's f_old after step n) in
 * `layout` (blocking when where == LBM_HOST).  Config mode writes 0 at solid nodes. */
int32_t lbm_get_populations(lbm_ctx* ctx, void* f, int32_t dtype, int32_t layout, int32_t where);
/* mask_s_local / mask_bb_local (Geometry.jl:92-173) as bytes 0/1, host arrays of
 * nx*ny*nz.  Blocking. */
int32_t lbm_get_flags(lbm_ctx* ctx, uint8_t* mask_s, uint8_t* mask_bb);
/* The link CSR of compile_bb_data! (Geometry.jl:268-311), bit-exact: bb_ptr[N+1]
 * (bb_ptr[0] = 1), bb_lidxs[nnz] (1-based node), bb_dirs[nnz] (1-based direction),
 * ordered by node then direction.  Host arrays; `cap` = capacity of the link
 * arrays; *nnz is always written.  LBM_ERR_CAPACITY when cap < nnz.  Blocking. */
int32_t lbm_get_links(lbm_ctx* ctx, int32_t* bb_ptr, int32_t* bb_lidxs, int8_t* bb_dirs,
                      int64_t cap, int64_t* nnz);
/* Link CSR export that allocates nothing; no counterpart in the reference.
 * Writes the same CSR as lbm_get_links, bit for bit, into caller-provided DEVICE
 * arrays: d_bb_ptr[N+1], d_bb_lidxs[cap], d_bb_dirs[cap].  For callers that cannot
 * call cudaMalloc: a host runtime that owns the device memory pool and must account
 * for every byte (CUDA.jl's allocator when MainCore.jl drives this library), and loops
 * that must not pay the device-wide synchronisation that cudaMalloc/cudaFree imply
 * (the reference rebuilds its link list every step, Motion.jl:82-93).
 * Its only scratch is a file-scope device array of 131,073 int64 (1 MiB), one entry
 * per 1024 nodes: every GPU that loads the library holds it until the process exits,
 * and lattices above 134,217,728 nodes (512^3) are rejected with LBM_ERR_CAPACITY.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.  All calls
 * share the array and it keeps the last call's contents (each call overwrites every
 * entry it reads); calls that overlap on the GPU — other streams or host threads —
 * race on it.  *nnz is always written; LBM_ERR_CAPACITY when cap < nnz (link entries
 * beyond cap are not written).  The three arrays must be device (or managed) memory of
 * the context's device (LBM_ERR_ARG otherwise) and are written on the context's stream
 * (lbm_set_stream): a caller that fills or reads them on another stream orders those
 * accesses against it.  Blocking: waits for nnz on the context's stream. */
int32_t lbm_get_links_noalloc(lbm_ctx* ctx, int32_t* d_bb_ptr, int32_t* d_bb_lidxs, int8_t* d_bb_dirs,
                              int64_t cap, int64_t* nnz);
/* Self-test of the bounded device waits; no counterpart in the reference (its kernels
 * never wait on the device).  Launches one block on the context's stream that waits on
 * an mbarrier nothing arrives on, through the same bounded wait the TMA-staged step
 * kernel uses, with a limit of `polls` polls (1 .. 2^22) instead of 2^22.  The wait
 * gives up, the block sets the context's error word and returns with nothing in
 * flight; the call then reports LBM_ERR_TIMEOUT, as lbm_synchronize does after a step
 * kernel whose wait gave up, and clears the word.  Blocking. */
int32_t lbm_wait_selftest(lbm_ctx* ctx, int32_t polls);
/* FP64 sum of all populations over fluid nodes (reference mode: all nodes).
 * Blocking. */
int32_t lbm_mass(lbm_ctx* ctx, double* out);
/* Scans the populations for NaN/Inf; LBM_ERR_NUMERIC when any is found.  Blocking. */
int32_t lbm_check(lbm_ctx* ctx);

/* ---- batched sweeps ------------------------------------------------------------- */
/* Many independent config-mode domains of uneven sizes stepped together: every step
 * is ONE persistent launch over a per-domain work table (runs of 128 cells of one
 * domain per work item), followed by a one-thread kernel that advances a device step
 * counter, so a sequence of steps can be captured once in a CUDA graph and replayed.
 * No reference counterpart: the reference runs one domain per process (MainCore.jl).
 *
 * Members: initialised contexts on one device and one stream, all with the same
 * storage and collision, static bodies only (no moving body).  They keep their own
 * populations, flags and force rings; lbm_get_force / lbm_get_macros /
 * lbm_get_populations on a member read the batched result.  A member may still be
 * stepped alone with lbm_step between batch calls (the table follows it); the batch
 * must be destroyed before any of its members.  Calls are ordered on the members'
 * stream. */
typedef struct lbm_batch lbm_batch;
int32_t lbm_batch_create(lbm_ctx* const* ctxs, int32_t count, lbm_batch** out);
int32_t lbm_batch_destroy(lbm_batch* b);
const char* lbm_batch_last_error(const lbm_batch* b);
/* `nsteps` batched steps, enqueued as 3 launches per step (the even-phase and the
 * odd-phase kernel, each skipping the domains of the other phase, and the counter). */
int32_t lbm_batch_step(lbm_batch* b, int32_t nsteps);
/* Records `nsteps` batched steps into a CUDA graph (replacing an earlier one); runs
 * nothing.  The capture uses a private stream. */
int32_t lbm_batch_capture(lbm_batch* b, int32_t nsteps);
/* Launches the captured graph `times` times on the members' stream. */
int32_t lbm_batch_replay(lbm_batch* b, int32_t times);
/* Kernels the batch has launched, graph nodes included. */
int64_t lbm_batch_launch_count(const lbm_batch* b);
/* Waits for the members' stream; LBM_ERR_CUDA with the CUDA error otherwise. */
int32_t lbm_batch_synchronize(lbm_batch* b);

/* ---- z-slab decomposition (replaces the halo exchange of Exchange.jl) ----
 * A domain split along z into slabs, one context per slab (per GPU), each holding its
 * owned planes plus one ghost plane on every LBM_FACE_HALO face (z = 0 and/or
 * z = nz - 1 of the slab).  Static bodies only (bodies placed in slab coordinates, the
 * ghost planes included).  After EVERY step, on each halo face, the caller moves one
 * message from this slab to the neighbouring slab and one back:
 *     lbm_halo_pack(mine, side, buf)  ->  transport  ->  lbm_halo_unpack(neighbour, 1 - side, buf)
 * The message of a face is 5 populations (the directions crossing it) times nx*ny
 * elements of the storage type: lbm_halo_bytes().  After an even-phase step the
 * boundary plane's post-collision values fill the neighbour's ghost plane; after an
 * odd-phase step the values streamed into the ghost plane go to the neighbour's
 * boundary plane (where the ghost node is fluid; a bounce-back value the neighbour
 * wrote itself is kept).  The phase follows from the context's step count, so both
 * calls must come after the same step on both sides.  Enqueued on the context's stream.
 * Replaces begin_halo_exchange! / gather_halo! (Exchange.jl:11-66, 112-129) and
 * finish_halo_exchange! / scatter_halo! (Exchange.jl:69-107, 131-145); the
 * transport between the calls (MPI Isend/Irecv there) is the caller's. */
int64_t lbm_halo_bytes(const lbm_ctx* ctx);
/* side: 0 = z-lo face, 1 = z-hi face (must be LBM_FACE_HALO).  d_buf: device memory of
 * lbm_halo_bytes() bytes. */
int32_t lbm_halo_pack(lbm_ctx* ctx, int32_t side, void* d_buf);
int32_t lbm_halo_unpack(lbm_ctx* ctx, int32_t side, const void* d_buf);

#ifdef __cplusplus
}
#endif
#endif /* LBM3D_H */
