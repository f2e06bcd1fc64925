// geometry.cu — solid/boundary flags and the link CSR.
//
// Replaces generate_mask_s_local! (Geometry.jl:49-117), generate_mask_bb_local!
// (Geometry.jl:122-173) and compile_bb_data! with its count / scan / fill kernels
// (Geometry.jl:181-311).  On the hot path only the per-node flag byte is kept
// current (for the moving body, inside a bounding box of its old and new poses);
// the CSR is produced on demand for export, in the reference's order (node-major,
// direction-minor, 1-based).
//
// Compiled with --fmad=false: every predicate rounds as written, exactly like the
// CPU restatement built with -ffp-contract=off, so flags and links are bit-exact.
#include <mutex>

#include "lbm_internal.cuh"
#include "lbm_kernels.h"
#include "shapes.cuh"

namespace lbm {

// ---- predicates -----------------------------------------------------------------------
__device__ __forceinline__ double min_image(double d, int n, int periodic) {
  if (!periodic) return d;
  const double hn = 0.5 * n;
  if (d > hn) d -= n;
  else if (d < -hn) d += n;
  return d;
}

__device__ bool inside_body(const BodyDev& b, const Grid& g, int x, int y, int z) {
  switch (b.kind) {
    case LBM_BODY_CYLINDER_Z: {
      // generate_mask_s_local!_gpu, cylinder branch (Geometry.jl:66-73), FP32
      const float h = (float)b.h;
      const float xl = ((float)(x + 1) - 0.5f) * h;
      const float yl = ((float)(y + 1) - 0.5f) * h;
      const float dx = xl - (float)b.center[0];
      const float dy = yl - (float)b.center[1];
      const float R = (float)b.radius;
      const float R2 = R * R;
      return (dx * dx + dy * dy) <= (R2 + 1e-6f * R2);
    }
    case LBM_BODY_NACA_Z: {
      // airfoil branch (Geometry.jl:75-82), FP32
      const float h = (float)b.h;
      const float xl = ((float)(x + 1) - 0.5f) * h;
      const float yl = ((float)(y + 1) - 0.5f) * h;
      const float dx = xl - (float)b.center[0];
      const float dy = yl - (float)b.center[1];
      const float ct = (float)b.cos_t, st = (float)b.sin_t;
      const float xB = ct * dx + st * dy;
      const float yB = -st * dx + ct * dy;
      const float chord = (float)b.chord;
      const float xle = xB + (float)b.x_le_offset;
      if (!(0.0f <= xle && xle <= chord)) return false;
      float yL, yU;
      naca_upper_lower(xle, chord, (float)b.naca_m, (float)b.naca_p, (float)b.naca_t, (float)b.x_int, &yL,
                       &yU);
      const float tol = 1e-6f * chord;
      return (yL - tol <= yB) && (yB <= yU + tol);
    }
    case LBM_BODY_SPHERE: {
      const double dx = min_image((x + 0.5) - b.center[0], g.nx, g.per[0]);
      const double dy = min_image((y + 0.5) - b.center[1], g.ny, g.per[1]);
      const double dz = min_image((z + 0.5) - b.center[2], g.nz, g.per[2]);
      return (dx * dx + dy * dy) + dz * dz <= b.radius * b.radius;
    }
    case LBM_BODY_ELLIPSOID: {
      const double dx = min_image((x + 0.5) - b.center[0], g.nx, g.per[0]);
      const double dy = min_image((y + 0.5) - b.center[1], g.ny, g.per[1]);
      const double dz = min_image((z + 0.5) - b.center[2], g.nz, g.per[2]);
      const double* r = b.rot;
      const double b0 = (r[0] * dx + r[3] * dy) + r[6] * dz;
      const double b1 = (r[1] * dx + r[4] * dy) + r[7] * dz;
      const double b2 = (r[2] * dx + r[5] * dy) + r[8] * dz;
      const double q0 = b0 / b.semi[0], q1 = b1 / b.semi[1], q2 = b2 / b.semi[2];
      return (q0 * q0 + q1 * q1) + q2 * q2 <= 1.0;
    }
  }
  return false;
}

__device__ __forceinline__ int wrapc(int v, int n) { return ((v % n) + n) % n; }

__device__ __forceinline__ void set_bits(uint8_t* flags, long long i, uint8_t bits) {
  unsigned int* word = (unsigned int*)((uintptr_t)(flags + i) & ~(uintptr_t)3);
  const unsigned int shift = (unsigned int)(((uintptr_t)(flags + i) & 3u) * 8u);
  atomicOr(word, (unsigned int)bits << shift);
}

// ---- rasterisation ---------------------------------------------------------------------------
__global__ void static_raster_kernel(const Grid g, const BodyDev b, const Box box, uint8_t* flags) {
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ex = box.hi[0] - box.lo[0] + 1;
  if (bx >= ex) return;
  const int x = wrapc(box.lo[0] + bx, g.nx);
  const int y = wrapc(box.lo[1] + (int)blockIdx.y, g.ny);
  const int z = wrapc(box.lo[2] + (int)blockIdx.z, g.nz);
  if (inside_body(b, g, x, y, z))
    set_bits(flags, node_index(g, x, y, z), (uint8_t)(F_STATIC | F_SOLID | F_SOLID_PREV));
}

// One block per sphere over its bounding box (periodic images on periodic axes).
__global__ void spheres_kernel(const Grid g, const double* __restrict__ xyzr, int count, uint8_t* flags) {
  const int s = blockIdx.x;
  if (s >= count) return;
  const double c[3] = {xyzr[4 * s], xyzr[4 * s + 1], xyzr[4 * s + 2]};
  const double r = xyzr[4 * s + 3];
  const int n3[3] = {g.nx, g.ny, g.nz};
  int lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = (int)floor(c[a] - r - 1.0);
    hi[a] = (int)ceil(c[a] + r + 1.0);
    if (!g.per[a]) {
      lo[a] = max(lo[a], 0);
      hi[a] = min(hi[a], n3[a] - 1);
    } else if (hi[a] - lo[a] + 1 >= n3[a]) {
      lo[a] = 0;
      hi[a] = n3[a] - 1;
    }
  }
  const long long ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
  if (ex <= 0 || ey <= 0 || ez <= 0) return;
  BodyDev b{};
  b.kind = LBM_BODY_SPHERE;
  b.center[0] = c[0];
  b.center[1] = c[1];
  b.center[2] = c[2];
  b.radius = r;
  for (long long t = threadIdx.x; t < ex * ey * ez; t += blockDim.x) {
    const int xx = (int)(t % ex), yy = (int)((t / ex) % ey), zz = (int)(t / (ex * ey));
    const int x = wrapc(lo[0] + xx, g.nx), y = wrapc(lo[1] + yy, g.ny), z = wrapc(lo[2] + zz, g.nz);
    if (inside_body(b, g, x, y, z))
      set_bits(flags, node_index(g, x, y, z), (uint8_t)(F_STATIC | F_SOLID | F_SOLID_PREV));
  }
}

// Moving body inside `box`: SOLID/MOVING from the latest pose, SOLID_PREV/MOVING_PREV
// from the pose of the last completed step; NEAR is recomputed afterwards.
__global__ void moving_kernel(const __grid_constant__ FlagParams p, uint8_t* flags) {
  const Grid& g = p.g;
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ex = p.box.hi[0] - p.box.lo[0] + 1;
  if (bx >= ex) return;
  const int x = wrapc(p.box.lo[0] + bx, g.nx);
  const int y = wrapc(p.box.lo[1] + (int)blockIdx.y, g.ny);
  const int z = wrapc(p.box.lo[2] + (int)blockIdx.z, g.nz);
  const long long i = node_index(g, x, y, z);
  const uint8_t st = flags[i] & F_STATIC;
  uint8_t v = st ? (uint8_t)(F_STATIC | F_SOLID | F_SOLID_PREV) : (uint8_t)0;
  if (p.has_moving) {
    if (inside_body(p.body, g, x, y, z)) v |= F_MOVING | F_SOLID;
    if (inside_body(p.body_prev, g, x, y, z)) v |= F_MOVING_PREV | F_SOLID_PREV;
  }
  flags[i] = v;
}

// NEAR: the node is fluid in either flag set and (it was uncovered, or a
// neighbour is solid in either set).  Reference mode ignores the periodic wrap,
// as nbr_lli does (Utilities.jl:559-569).  Config mode also stores, per node, the
// link word used by the step kernel: bit d (0..17) = the source x - c_d of incoming
// direction d is solid now, bit 18+d = it was solid at the last step, bit 36+d =
// it belongs to the moving body now (sources outside a non-periodic face: no bit).
__global__ void near_kernel(const Grid g, int mode, const Box box, uint8_t* flags,
                            unsigned long long* links) {
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ex = box.hi[0] - box.lo[0] + 1;
  if (bx >= ex) return;
  const int x = wrapc(box.lo[0] + bx, g.nx);
  const int y = wrapc(box.lo[1] + (int)blockIdx.y, g.ny);
  const int z = wrapc(box.lo[2] + (int)blockIdx.z, g.nz);
  const long long i = node_index(g, x, y, z);
  const uint8_t fl = flags[i];
  const bool sc = fl & F_SOLID, sp = fl & F_SOLID_PREV;
  const bool wrap = (mode == LBM_MODE_CONFIG);
  bool near = sp && !sc;
  unsigned long long lw = 0;
#pragma unroll
  for (int d = 0; d < 18; d++) {
    int nx_ = x - cx(d), ny_ = y - cy(d), nz_ = z - cz(d);
    if (nx_ < 0 || nx_ >= g.nx) {
      if (!(wrap && g.per[0])) continue;
      nx_ = wrapc(nx_, g.nx);
    }
    if (ny_ < 0 || ny_ >= g.ny) {
      if (!(wrap && g.per[1])) continue;
      ny_ = wrapc(ny_, g.ny);
    }
    if (nz_ < 0 || nz_ >= g.nz) {
      if (!(wrap && g.per[2])) continue;
      nz_ = wrapc(nz_, g.nz);
    }
    const uint8_t fn = flags[node_index(g, nx_, ny_, nz_)];
    if (fn & (F_SOLID | F_SOLID_PREV)) near = true;
    if (fn & F_SOLID) lw |= 1ull << d;
    if (fn & F_SOLID_PREV) lw |= 1ull << (18 + d);
    if (fn & F_MOVING) lw |= 1ull << (36 + d);
  }
  if (g.q == 27) {  // D3Q27 (reference mode, no wrap): the corner neighbours count for mask_bb
    for (int d = 18; d < 26; d++) {
      const int nx_ = x - cx27(d), ny_ = y - cy27(d), nz_ = z - cz27(d);
      if (nx_ < 0 || nx_ >= g.nx || ny_ < 0 || ny_ >= g.ny || nz_ < 0 || nz_ >= g.nz) continue;
      if (flags[node_index(g, nx_, ny_, nz_)] & (F_SOLID | F_SOLID_PREV)) near = true;
    }
  }
  near = near && (!sc || !sp);
  flags[i] = near ? (uint8_t)(fl | F_NEAR) : (uint8_t)(fl & ~F_NEAR);
  if (links) links[i] = lw;
}

// ---- link CSR ----------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t link_mask(const Grid& g, int mode, const uint8_t* flags, uint8_t sbit,
                                              int x, int y, int z) {
  const long long i = node_index(g, x, y, z);
  if (flags[i] & sbit) return 0;
  const bool wrap = (mode == LBM_MODE_CONFIG);
  uint32_t m = 0;
#pragma unroll
  for (int d = 0; d < 18; d++) {
    int nx_ = x + cx(d), ny_ = y + cy(d), nz_ = z + cz(d);
    if (nx_ < 0 || nx_ >= g.nx) {
      if (!(wrap && g.per[0])) continue;
      nx_ = wrapc(nx_, g.nx);
    }
    if (ny_ < 0 || ny_ >= g.ny) {
      if (!(wrap && g.per[1])) continue;
      ny_ = wrapc(ny_, g.ny);
    }
    if (nz_ < 0 || nz_ >= g.nz) {
      if (!(wrap && g.per[2])) continue;
      nz_ = wrapc(nz_, g.nz);
    }
    if (flags[node_index(g, nx_, ny_, nz_)] & sbit) m |= 1u << d;
  }
  if (g.q == 27) {  // D3Q27 (reference mode, no wrap): links to the corner neighbours, bits 18..25
    for (int d = 18; d < 26; d++) {
      const int nx_ = x + cx27(d), ny_ = y + cy27(d), nz_ = z + cz27(d);
      if (nx_ < 0 || nx_ >= g.nx || ny_ < 0 || ny_ >= g.ny || nz_ < 0 || nz_ >= g.nz) continue;
      if (flags[node_index(g, nx_, ny_, nz_)] & sbit) m |= 1u << d;
    }
  }
  return m;
}

constexpr int SCAN_B = 1024;

__global__ void count_kernel(const Grid g, int mode, const uint8_t* __restrict__ flags, uint8_t sbit,
                             int32_t* __restrict__ count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int x = (int)(i % g.nx);
  const int y = (int)((i / g.nx) % g.ny);
  const int z = (int)(i / ((long long)g.nx * g.ny));
  count[i] = __popc(link_mask(g, mode, flags, sbit, x, y, z));
}

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* total) {
  __shared__ long long warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    long long ws = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += t;
    }
    if (lane < nw) warp_sums[lane] = ws;  // inclusive warp prefix
  }
  __syncthreads();
  const long long before = warp == 0 ? 0 : warp_sums[warp - 1];
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  const long long excl = before + inc - v;
  __syncthreads();
  return excl;
}

__global__ void block_sum_kernel(const Grid g, const int32_t* __restrict__ count, long long* __restrict__ bs) {
  const long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
  long long v = i < g.N ? count[i] : 0;
  long long total;
  block_exclusive_scan(v, &total);
  if (threadIdx.x == 0) bs[blockIdx.x] = total;
}

// single block: exclusive scan of the block sums in place; bs[nb] = grand total
__global__ void scan_blocksums_kernel(long long* bs, long long nb) {
  long long carry = 0;
  for (long long base = 0; base < nb; base += SCAN_B) {
    const long long k = base + threadIdx.x;
    const long long v = k < nb ? bs[k] : 0;
    long long total;
    const long long ex = block_exclusive_scan(v, &total);
    if (k < nb) bs[k] = carry + ex;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) bs[nb] = carry;
}

__global__ void ptr_kernel(const Grid g, const int32_t* __restrict__ count, const long long* __restrict__ bs,
                           long long* __restrict__ scan, int32_t* __restrict__ ptr, long long nb) {
  const long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
  const long long v = i < g.N ? count[i] : 0;
  const long long ex = block_exclusive_scan(v, nullptr) + bs[blockIdx.x];
  if (i < g.N) {
    scan[i] = ex;
    ptr[i] = (int32_t)(1 + ex);  // bb_ptr[a] = 1 + inclusive_scan[a-1] (Geometry.jl:214-227)
  }
  if (i == 0) ptr[g.N] = (int32_t)(1 + bs[nb]);
}

__global__ void fill_kernel(const Grid g, int mode, const uint8_t* __restrict__ flags, uint8_t sbit,
                            const long long* __restrict__ scan, int32_t* __restrict__ lidx,
                            int8_t* __restrict__ dirs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int x = (int)(i % g.nx);
  const int y = (int)((i / g.nx) % g.ny);
  const int z = (int)(i / ((long long)g.nx * g.ny));
  const uint32_t m = link_mask(g, mode, flags, sbit, x, y, z);
  if (!m) return;
  long long k = scan[i];
  for (int d = 0; d < 26; d++) {  // bits 18..25: D3Q27 corners
    if ((m >> d) & 1u) {
      lidx[k] = (int32_t)(i + 1);
      dirs[k] = (int8_t)(d + 1);
      k++;
    }
  }
}

__global__ void masks_kernel(const Grid g, int mode, const uint8_t* __restrict__ flags, uint8_t sbit,
                             uint8_t* __restrict__ ms, uint8_t* __restrict__ mb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int x = (int)(i % g.nx);
  const int y = (int)((i / g.nx) % g.ny);
  const int z = (int)(i / ((long long)g.nx * g.ny));
  if (ms) ms[i] = (flags[i] & sbit) ? 1 : 0;
  if (mb) mb[i] = link_mask(g, mode, flags, sbit, x, y, z) ? 1 : 0;
}

__global__ void sync_prev_kernel(const Grid g, uint8_t* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const uint8_t fl = flags[i];
  uint8_t v = fl & (uint8_t)~(F_SOLID_PREV | F_MOVING_PREV);
  if (fl & F_SOLID) v |= F_SOLID_PREV;
  if (fl & F_MOVING) v |= F_MOVING_PREV;
  flags[i] = v;
}

// ---- launchers --------------------------------------------------------------------------------------
static dim3 box_grid(const Box& b, int bx) {
  const int ex = b.hi[0] - b.lo[0] + 1, ey = b.hi[1] - b.lo[1] + 1, ez = b.hi[2] - b.lo[2] + 1;
  return dim3((unsigned)((ex + bx - 1) / bx), (unsigned)ey, (unsigned)ez);
}

cudaError_t geo_launch_static(const Grid& g, const BodyDev& b, const Box& box, uint8_t* flags, cudaStream_t s) {
  static_raster_kernel<<<box_grid(box, 128), 128, 0, s>>>(g, b, box, flags);
  return cudaGetLastError();
}

cudaError_t geo_launch_spheres(const Grid& g, const double* xyzr, int count, uint8_t* flags, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  spheres_kernel<<<count, 256, 0, s>>>(g, xyzr, count, flags);
  return cudaGetLastError();
}

cudaError_t geo_launch_moving(const FlagParams& p, uint8_t* flags, cudaStream_t s) {
  moving_kernel<<<box_grid(p.box, 128), 128, 0, s>>>(p, flags);
  return cudaGetLastError();
}

cudaError_t geo_launch_near(const Grid& g, int mode, const Box& box, uint8_t* flags, unsigned long long* links,
                            cudaStream_t s) {
  near_kernel<<<box_grid(box, 128), 128, 0, s>>>(g, mode, box, flags, links);
  return cudaGetLastError();
}

cudaError_t geo_launch_sync_prev(const Grid& g, uint8_t* flags, cudaStream_t s) {
  sync_prev_kernel<<<(unsigned)((g.N + 255) / 256), 256, 0, s>>>(g, flags);
  return cudaGetLastError();
}

cudaError_t geo_links(const Grid& g, int mode, const uint8_t* flags, uint8_t sbit, int32_t* d_count,
                      long long* d_scan, long long* d_bs, int32_t* d_ptr, int32_t* d_lidx, int8_t* d_dirs,
                      long long cap, long long* h_nnz, cudaStream_t s) {
  const long long nb = (g.N + SCAN_B - 1) / SCAN_B;
  count_kernel<<<(unsigned)((g.N + 255) / 256), 256, 0, s>>>(g, mode, flags, sbit, d_count);
  block_sum_kernel<<<(unsigned)nb, SCAN_B, 0, s>>>(g, d_count, d_bs);
  scan_blocksums_kernel<<<1, SCAN_B, 0, s>>>(d_bs, nb);
  ptr_kernel<<<(unsigned)nb, SCAN_B, 0, s>>>(g, d_count, d_bs, d_scan, d_ptr, nb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(h_nnz, d_bs + nb, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if (*h_nnz > cap || d_lidx == nullptr) return cudaSuccess;  // caller reports capacity
  fill_kernel<<<(unsigned)((g.N + 255) / 256), 256, 0, s>>>(g, mode, flags, sbit, d_scan, d_lidx, d_dirs);
  return cudaGetLastError();
}

cudaError_t geo_masks(const Grid& g, int mode, const uint8_t* flags, uint8_t sbit, uint8_t* ms, uint8_t* mb,
                      cudaStream_t s) {
  masks_kernel<<<(unsigned)((g.N + 255) / 256), 256, 0, s>>>(g, mode, flags, sbit, ms, mb);
  return cudaGetLastError();
}

// ---- link CSR without allocation -----------------------------------------------------
// Same CSR as geo_links, for callers that cannot allocate device memory.  The only
// scratch is one int64 per 1024-node block (the block's link count, then its
// exclusive offset), kept in this file-scope array; per-node offsets are recomputed
// from the flags in the fill pass instead of being stored.  The array lives on every
// device that loads the library until the process exits, holds the last call's
// contents between calls, and is shared by all calls: calls that overlap on the GPU
// race on it.
constexpr long long NOALLOC_MAX_BLOCKS = 131072;  // 131072 * 1024 = 134,217,728 nodes (512^3)
static __device__ __align__(256) long long g_noalloc_block_sums[NOALLOC_MAX_BLOCKS + 1];

__global__ void na_count_kernel(const Grid g, int mode, const uint8_t* __restrict__ flags, uint8_t sbit,
                                long long* __restrict__ bs) {
  const long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
  long long v = 0;
  if (i < g.N) {
    const int x = (int)(i % g.nx);
    const int y = (int)((i / g.nx) % g.ny);
    const int z = (int)(i / ((long long)g.nx * g.ny));
    v = __popc(link_mask(g, mode, flags, sbit, x, y, z));
  }
  long long total;
  block_exclusive_scan(v, &total);
  if (threadIdx.x == 0) bs[blockIdx.x] = total;  // every block of this call overwrites its entry
}

__global__ void na_fill_kernel(const Grid g, int mode, const uint8_t* __restrict__ flags, uint8_t sbit,
                               const long long* __restrict__ bs, long long nb, int32_t* __restrict__ ptr,
                               int32_t* __restrict__ lidx, int8_t* __restrict__ dirs, long long cap) {
  const long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
  uint32_t m = 0;
  if (i < g.N) {
    const int x = (int)(i % g.nx);
    const int y = (int)((i / g.nx) % g.ny);
    const int z = (int)(i / ((long long)g.nx * g.ny));
    m = link_mask(g, mode, flags, sbit, x, y, z);
  }
  const long long ex = block_exclusive_scan((long long)__popc(m), nullptr) + bs[blockIdx.x];
  if (i < g.N) {
    ptr[i] = (int32_t)(1 + ex);
    long long k = ex;
    for (int d = 0; d < 26; d++) {  // bits 18..25: D3Q27 corners
      if ((m >> d) & 1u) {
        if (k < cap) {  // never write past the caller's capacity
          lidx[k] = (int32_t)(i + 1);
          dirs[k] = (int8_t)(d + 1);
        }
        k++;
      }
    }
  }
  if (i == 0) ptr[g.N] = (int32_t)(1 + bs[nb]);
}

namespace {
// Device address of g_noalloc_block_sums per device.  Host code must not use the
// array's name as a device pointer: it is a host-side stand-in.
constexpr int NOALLOC_MAX_DEVICES = 64;
long long* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
std::mutex g_noalloc_mutex;
}  // namespace

cudaError_t geo_links_noalloc(const Grid& g, int mode, const uint8_t* flags, uint8_t sbit, int32_t* d_ptr,
                              int32_t* d_lidx, int8_t* d_dirs, long long cap, long long* h_nnz, int* too_large,
                              cudaStream_t s) {
  const long long nb = (g.N + SCAN_B - 1) / SCAN_B;
  *too_large = nb > NOALLOC_MAX_BLOCKS ? 1 : 0;
  if (*too_large) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  long long* bs = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {  // once per device, with that device current
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_block_sums);
      if (e != cudaSuccess) return e;
      g_noalloc_ptr[dev] = (long long*)ptr;
    }
    bs = g_noalloc_ptr[dev];
  }
  na_count_kernel<<<(unsigned)nb, SCAN_B, 0, s>>>(g, mode, flags, sbit, bs);
  scan_blocksums_kernel<<<1, SCAN_B, 0, s>>>(bs, nb);
  na_fill_kernel<<<(unsigned)nb, SCAN_B, 0, s>>>(g, mode, flags, sbit, bs, nb, d_ptr, d_lidx, d_dirs,
                                                 d_lidx && d_dirs ? cap : 0);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(h_nnz, bs + nb, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

long long geo_links_noalloc_max_nodes() { return NOALLOC_MAX_BLOCKS * SCAN_B; }

}  // namespace lbm
