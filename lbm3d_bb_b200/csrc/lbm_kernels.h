// lbm_kernels.h — kernel parameter blocks and host launchers of liblbm3d.
#pragma once

#include "lbm_internal.cuh"

namespace lbm {

// TMA-staged persistent variant of the config-mode step.
struct TmaCfg {
  int enabled;
  int tw;          // tile width (cells along x), = block size
  int halo;        // elements in a 16-byte halo chunk
  int ntx;         // tiles per row
  long long ntiles;
  int stages;      // pipeline depth
  int stage_bytes; // shared memory per stage (19 direction buffers)
  int buf_elems;   // elements per direction buffer (tw + halo)
  const uint8_t* tile_slow;  // per tile: bit 0 even / bit 1 odd phase needs the direct path
  int* err;                  // set to 1 when a pipeline wait gives up
};

// Config-mode (AA) step.
struct AAParams {
  Grid g;
  int face_kind[6];
  double face_u[6][3];
  double omega_p, omega_m, rho0;
  double gacc[3];
  Kinematics kin;
  int compute_force;
  double* force;      // 6 doubles of this step
  double* zero_next;  // force record of the next step, cleared by this launch (may be null)
  // interior fast path: element offsets, relative to the node, of the 19 reads and
  // the 19 writes of this phase (even: own slots; odd: neighbour slots)
  long long off_rd[19];
  long long off_wr[19];
  long long offb_rd[19];  // the same in bytes (pair kernel: one 64-bit add per access)
  long long offb_wr[19];
  TmaCfg tma;
  // per-node link words of NEAR nodes (see near_kernel): static no-slip links stay
  // on the fast path, everything else takes the general path
  const unsigned long long* links;
  int pair;  // all axes periodic, nx % 128 == 0: two cells per thread (aa_pair_kernel)
  int quad;  // with pair, FP16-deviation: 1 four cells per thread (aa_quad_even/odd_kernel), 2 eight in the even phase (aa_octo_even_kernel)
  int xshuffle;  // with pair, FP32 odd phase: x-shifted directions as shuffled words (aa_pair_odd_kernel)
};

// Batched step over many independent config-mode domains (one launch per step).
constexpr int BATCH_ITEM = 128;  // cells per work item = threads per block
// polls after which a bounded mbarrier wait in a step kernel gives up (each try_wait
// blocks for a hardware-defined interval: seconds in all)
constexpr int MBAR_WAIT_POLLS = 1 << 22;
constexpr int BATCH_LAUNCHES_PER_STEP = 3;  // even-phase and odd-phase kernels, counter advance

struct BatchDom {
  AAParams p[2];         // parameter blocks of the even [0] and odd [1] phase
  void* A;               // populations
  const uint8_t* flags;
  double* ring;          // force records (ring_slots x FORCE_RECORD doubles)
  int ring_slots;
  int phase0;            // phase of batch step 0 (0 even, 1 odd)
  long long base_step;   // steps the domain had completed before batch step 0
  long long item_begin;  // first work item of the domain
  long long item_end;    // one past its last work item
};

struct BatchParams {
  const BatchDom* doms;
  const int* item_dom;       // domain of every work item
  long long items;           // work items in total
  const long long* counter;  // batch steps completed (advanced on the device)
};

// The moving body as the interpolated bounce-back sees it (Motion.jl:104-119): planar
// shape at the half-step pose, lattice units, FP32.
struct IbbGeom {
  int shape;       // LBM_BODY_CYLINDER_Z or LBM_BODY_NACA_Z
  float xc, yc;    // half-step centre (x_c_lat, y_c_lat)
  float ct, st;    // cos / sin of the half-step angle (c_theta_half, s_theta_half)
  float R, chord, x_le, m, p, t, x_int;  // R_lat, chord_lat, x_le_offset_lat, NACA m p t, x_int
};

// Reference-mode step (two population buffers, virtual-fluid solids).
struct RefParams {
  Grid g;
  float omega_p, omega_m;
  float U, V, W;  // U_inf, V_inf, W_inf
  float h;
  Kinematics kin;  // lattice-unit half-step kinematics (Motion.jl:96-100), FP32-valued
  uint8_t solid_bit;
  int compute_force;
  double* force;
  double* zero_next;
  int solid_bc;  // LBM_SOLID_SBB or LBM_SOLID_IBB
  IbbGeom ibb;
};

// Read-back of the state of the last completed step.
struct ReadParams {
  Grid g;
  double rho0;
  int swapped;        // AA: state in swapped layout (after an even phase)
  uint8_t solid_bit;  // flag bit holding the solids of the last completed step
  double gacc[3];
};

struct ExportOut {
  void* f;  // populations (nullable)
  int f_dtype, f_layout;
  void* rho;  // macros (nullable)
  void* u;
  void* v;
  void* w;
  int m_dtype;
};

struct InitParams {
  Grid g;
  double rho0;
  double uni[3];
  const double* rho;  // device arrays (nullable)
  const double* u;
  const double* v;
  const double* w;
  const void* f_in;  // device populations to import (nullable)
  int f_dtype, f_layout;
};

template <class T>
__device__ __forceinline__ void put(void* base, long long k, int dtype, T v) {
  if (dtype == LBM_DTYPE_F64)
    ((double*)base)[k] = (double)v;
  else
    ((float*)base)[k] = (float)v;
}

__device__ __forceinline__ double import_value(const InitParams& p, const Grid& g, long long i, int d) {
  const long long k = p.f_layout == LBM_LAYOUT_SOA ? (long long)d * g.N + i : (long long)d + (long long)g.q * i;
  return p.f_dtype == LBM_DTYPE_F64 ? ((const double*)p.f_in)[k] : (double)((const float*)p.f_in)[k];
}

// Writes one node's populations and/or moments (config-mode moments: u = j/rho + g/2).
template <class C>
__device__ __forceinline__ void export_node(const ExportOut& o, const Grid& g, long long i, const C* f,
                                            bool solid, const double* gacc) {
  if (o.f) {
#pragma unroll
    for (int d = 0; d < 19; d++) {
      const long long k = o.f_layout == LBM_LAYOUT_SOA ? (long long)d * g.N + i : (long long)d + 19LL * i;
      put<C>(o.f, k, o.f_dtype, f[d]);
    }
  }
  if (o.rho || o.u || o.v || o.w) {
    C r = f[0], jx = C(0), jy = C(0), jz = C(0);
#pragma unroll
    for (int d = 1; d < 19; d++) r += f[d];
#pragma unroll
    for (int d = 0; d < 19; d++) {
      jx += f[d] * C(cx(d));
      jy += f[d] * C(cy(d));
      jz += f[d] * C(cz(d));
    }
    C ux = C(0), uy = C(0), uz = C(0);
    if (!solid) {
      ux = jx / r + C(0.5) * C(gacc[0]);
      uy = jy / r + C(0.5) * C(gacc[1]);
      uz = jz / r + C(0.5) * C(gacc[2]);
    } else {
      r = C(0);
    }
    if (o.rho) put<C>(o.rho, i, o.m_dtype, r);
    if (o.u) put<C>(o.u, i, o.m_dtype, ux);
    if (o.v) put<C>(o.v, i, o.m_dtype, uy);
    if (o.w) put<C>(o.w, i, o.m_dtype, uz);
  }
}

// A step's force record: FORCE_SLOTS cache lines of 8 doubles (F, T, pad); each
// block adds into line (block index mod FORCE_SLOTS) so that same-address FP64
// atomics spread over many L2 lines.  The host sums the lines.
constexpr int FORCE_SLOTS = 32;
constexpr int FORCE_RECORD = FORCE_SLOTS * 8;  // doubles per step

__device__ __forceinline__ int block_stripe() {
  const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  return (int)(b % FORCE_SLOTS) * 8;
}

// Clears the next step's force record (block 0 only; read by the next launch).
__device__ __forceinline__ void clear_record(double* rec) {
  if (rec == nullptr || (blockIdx.x | blockIdx.y | blockIdx.z) != 0) return;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  for (int t = tid; t < FORCE_RECORD; t += blockDim.x * blockDim.y) rec[t] = 0.0;
}

// Block reduction of the six force/torque components; one FP64 atomic each.
__device__ __forceinline__ void block_force_reduce(double* acc, bool has, double* out) {
  __shared__ double red[32][6];
  const int nthreads = blockDim.x * blockDim.y;
  if (!__syncthreads_or(has)) return;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (tid == 0) {
    const int nw = (nthreads + 31) >> 5;
    for (int k = 0; k < 6; k++) {
      double s = 0.0;
      for (int w = 0; w < nw; w++) s += red[w][k];
      atomicAdd(out + k, s);
    }
  }
}

// ---- launchers (kernels_aa.cu; kernels in aa_impl.cuh) ----
// faces: some axis is not periodic (selects the kernel that keeps face nodes on the
// fast path; the other kernel sends them to the general path).
cudaError_t aa_launch_step(int storage, const AAParams& p, void* A, const uint8_t* flags, bool odd,
                           bool trt, int force, bool faces, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t aa_launch_batch(int storage, const BatchParams& bp, bool trt, bool force, bool faces, int blocks,
                            cudaStream_t s);
cudaError_t aa_batch_blocks_per_sm(int storage, bool trt, bool force, bool faces, int* per_sm);
cudaError_t aa_launch_batch_advance(long long* counter, cudaStream_t s);
// z-slab halo message of one face (side 0 z-lo, 1 z-hi); elem = bytes per population
cudaError_t aa_launch_halo(const Grid& g, int elem, int side, bool after_even, bool pack, void* A,
                           const uint8_t* flags, void* buf, cudaStream_t s);
cudaError_t aa_launch_export(int storage, const ReadParams& p, const void* A, const uint8_t* flags,
                             const ExportOut& out, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t aa_launch_reduce(int storage, const ReadParams& p, const void* A, const uint8_t* flags,
                             double* out, dim3 grid, dim3 block, cudaStream_t s);
// Self-test of the bounded wait: one block waits on an mbarrier that nothing arrives on,
// gives up after `polls` polls and sets *err, exactly as a step kernel does.
cudaError_t aa_launch_wait_probe(int polls, int* err, cudaStream_t s);
cudaError_t aa_launch_tile_flags(const Grid& g, int tw, long long ntiles, const uint8_t* flags, uint8_t* tiles,
                                 cudaStream_t s);
cudaError_t aa_launch_init(int storage, const InitParams& p, void* A, const uint8_t* flags, dim3 grid,
                           dim3 block, cudaStream_t s);

// ---- launchers (kernels_ref.cu) ----
// Fp/Rp: post-collision populations and macros of the previous state; Fn/Rn: outputs.
cudaError_t ref_launch_step(bool fp64, bool trt, const RefParams& p, const void* Fp, const void* Rp,
                            void* Fn, void* Rn, const uint8_t* flags, dim3 grid, dim3 block,
                            cudaStream_t s);
// S_n export (pull of Fp with Rp), or direct export of a stored S (direct != 0).
cudaError_t ref_launch_export(bool fp64, const RefParams& p, const void* Fp, const void* Rp, int direct,
                              const uint8_t* flags, const ExportOut& out, double* mass, dim3 grid,
                              dim3 block, cudaStream_t s);
// From S (pre-collision, SoA in the context's precision) compute R = moments(S)
// and F = collide(S, R) (the state the next step pulls from).
cudaError_t ref_launch_prepare(bool fp64, bool trt, const RefParams& p, const void* Sdirect, void* F,
                               void* R, dim3 grid, dim3 block, cudaStream_t s);
// S = feq_ref(rho, u) or imported populations, in the context's precision.
cudaError_t ref_launch_init(bool fp64, const InitParams& p, void* S, dim3 grid, dim3 block, cudaStream_t s);
// Copies the stored macros R (4 planes) into caller arrays.
cudaError_t ref_launch_macros(bool fp64, const Grid& g, const void* R, const ExportOut& out, dim3 grid,
                              dim3 block, cudaStream_t s);

// ---- geometry (geometry.cu) ----
struct FlagParams {
  Grid g;
  int mode;       // LBM_MODE_*
  Box box;        // region (unwrapped coordinates; wrapped on periodic axes)
  BodyDev body;   // moving body
  BodyDev body_prev;  // same body at the pose of the last completed step
  int has_moving;
};
cudaError_t geo_launch_static(const Grid& g, const BodyDev& b, const Box& box, uint8_t* flags,
                              cudaStream_t s);
cudaError_t geo_launch_spheres(const Grid& g, const double* xyzr, int count, uint8_t* flags,
                               cudaStream_t s);
cudaError_t geo_launch_moving(const FlagParams& p, uint8_t* flags, cudaStream_t s);
cudaError_t geo_launch_near(const Grid& g, int mode, const Box& box, uint8_t* flags, unsigned long long* links,
                            cudaStream_t s);
cudaError_t geo_launch_sync_prev(const Grid& g, uint8_t* flags, cudaStream_t s);
// Link export: counts per node (cur solid bits), exclusive scan, CSR fill.
cudaError_t geo_links(const Grid& g, int mode, const uint8_t* flags, uint8_t solid_bit, int32_t* d_count,
                      long long* d_scan, long long* d_blocksums, int32_t* d_ptr, int32_t* d_lidx,
                      int8_t* d_dirs, long long cap, long long* h_nnz, cudaStream_t s);
// Link CSR into caller device arrays with no allocation (file-scope scratch); sets
// *too_large when the lattice exceeds geo_links_noalloc_max_nodes() and does nothing.
cudaError_t geo_links_noalloc(const Grid& g, int mode, const uint8_t* flags, uint8_t sbit, int32_t* d_ptr,
                              int32_t* d_lidx, int8_t* d_dirs, long long cap, long long* h_nnz, int* too_large,
                              cudaStream_t s);
long long geo_links_noalloc_max_nodes();
cudaError_t geo_masks(const Grid& g, int mode, const uint8_t* flags, uint8_t solid_bit, uint8_t* ms,
                      uint8_t* mb, cudaStream_t s);

}  // namespace lbm
