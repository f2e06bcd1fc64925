// kernels_aa.cu — storage dispatch of the configurable AA step (the kernels are
// instantiated per storage in kernels_aa_fp32.cu / kernels_aa_fp64.cu /
// kernels_aa_fp16.cu from aa_impl.cuh), the TMA tile bits and the batch counter.
#include "lbm_internal.cuh"
#include "lbm_kernels.h"

namespace lbm {

#define LBM_AA_DECLARE_OPS(NAME)                                                                                  \
  cudaError_t aa_step_##NAME(const AAParams& p, void* A, const uint8_t* flags, bool odd, bool trt, int force,     \
                             bool faces, dim3 grid, dim3 block, cudaStream_t s);                                  \
  cudaError_t aa_batch_##NAME(const BatchParams& bp, bool trt, bool force, bool faces, int blocks, int* per_sm,  \
                              cudaStream_t s);                                                                    \
  cudaError_t aa_export_##NAME(const ReadParams& p, const void* A, const uint8_t* flags, const ExportOut& out,    \
                               dim3 grid, dim3 block, cudaStream_t s);                                            \
  cudaError_t aa_reduce_##NAME(const ReadParams& p, const void* A, const uint8_t* flags, double* out, dim3 grid,  \
                               dim3 block, cudaStream_t s);                                                       \
  cudaError_t aa_init_##NAME(const InitParams& p, void* A, const uint8_t* flags, dim3 grid, dim3 block,           \
                             cudaStream_t s);
LBM_AA_DECLARE_OPS(fp32)
LBM_AA_DECLARE_OPS(fp64)
LBM_AA_DECLARE_OPS(fp16)
#undef LBM_AA_DECLARE_OPS

cudaError_t aa_launch_step(int storage, const AAParams& p, void* A, const uint8_t* flags, bool odd, bool trt,
                           int force, bool faces, dim3 grid, dim3 block, cudaStream_t s) {
  switch (storage) {
    case LBM_STORE_FP32: return aa_step_fp32(p, A, flags, odd, trt, force, faces, grid, block, s);
    case LBM_STORE_FP64: return aa_step_fp64(p, A, flags, odd, trt, force, faces, grid, block, s);
    case LBM_STORE_FP16DEV: return aa_step_fp16(p, A, flags, odd, trt, force, faces, grid, block, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aa_launch_batch(int storage, const BatchParams& bp, bool trt, bool force, bool faces, int blocks,
                            cudaStream_t s) {
  switch (storage) {
    case LBM_STORE_FP32: return aa_batch_fp32(bp, trt, force, faces, blocks, nullptr, s);
    case LBM_STORE_FP64: return aa_batch_fp64(bp, trt, force, faces, blocks, nullptr, s);
    case LBM_STORE_FP16DEV: return aa_batch_fp16(bp, trt, force, faces, blocks, nullptr, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aa_batch_blocks_per_sm(int storage, bool trt, bool force, bool faces, int* per_sm) {
  BatchParams none{};
  switch (storage) {
    case LBM_STORE_FP32: return aa_batch_fp32(none, trt, force, faces, 0, per_sm, nullptr);
    case LBM_STORE_FP64: return aa_batch_fp64(none, trt, force, faces, 0, per_sm, nullptr);
    case LBM_STORE_FP16DEV: return aa_batch_fp16(none, trt, force, faces, 0, per_sm, nullptr);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aa_launch_export(int storage, const ReadParams& p, const void* A, const uint8_t* flags,
                             const ExportOut& out, dim3 grid, dim3 block, cudaStream_t s) {
  switch (storage) {
    case LBM_STORE_FP32: return aa_export_fp32(p, A, flags, out, grid, block, s);
    case LBM_STORE_FP64: return aa_export_fp64(p, A, flags, out, grid, block, s);
    case LBM_STORE_FP16DEV: return aa_export_fp16(p, A, flags, out, grid, block, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aa_launch_reduce(int storage, const ReadParams& p, const void* A, const uint8_t* flags, double* out,
                             dim3 grid, dim3 block, cudaStream_t s) {
  switch (storage) {
    case LBM_STORE_FP32: return aa_reduce_fp32(p, A, flags, out, grid, block, s);
    case LBM_STORE_FP64: return aa_reduce_fp64(p, A, flags, out, grid, block, s);
    case LBM_STORE_FP16DEV: return aa_reduce_fp16(p, A, flags, out, grid, block, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aa_launch_init(int storage, const InitParams& p, void* A, const uint8_t* flags, dim3 grid, dim3 block,
                           cudaStream_t s) {
  switch (storage) {
    case LBM_STORE_FP32: return aa_init_fp32(p, A, flags, grid, block, s);
    case LBM_STORE_FP64: return aa_init_fp64(p, A, flags, grid, block, s);
    case LBM_STORE_FP16DEV: return aa_init_fp16(p, A, flags, grid, block, s);
  }
  return cudaErrorInvalidValue;
}

// Per-tile boundary bits: 1 = the even phase needs the direct path, 2 = the odd
// phase does (boundary node in the tile, or a y/z-periodic wrap row).
__global__ void tile_flags_kernel(const Grid g, int tw, long long ntiles, const uint8_t* __restrict__ flags,
                                  uint8_t* __restrict__ tiles) {
  const long long tile = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tile >= ntiles) return;
  const long long ntx = g.nx / tw;
  const long long row = tile / ntx;
  const int x0 = (int)(tile - row * ntx) * tw;
  const int y = (int)(row % g.ny), z = (int)(row / g.ny);
  bool face = (!g.per[1] && (y == 0 || y == g.ny - 1)) || (!g.per[2] && (z == 0 || z == g.nz - 1)) ||
              (!g.per[0] && (x0 == 0 || x0 + tw == g.nx));
  bool bnd = face;
  const uint8_t* f = flags + row * g.nx + x0;
  for (int k = 0; k < tw && !bnd; k++) bnd = (f[k] & (F_SOLID | F_SOLID_PREV | F_NEAR)) != 0;
  const bool wrap_row = y == 0 || y == g.ny - 1 || z == 0 || z == g.nz - 1;
  tiles[tile] = (uint8_t)((bnd ? 1 : 0) | ((bnd || wrap_row) ? 2 : 0));
}

cudaError_t aa_launch_tile_flags(const Grid& g, int tw, long long ntiles, const uint8_t* flags, uint8_t* tiles,
                                 cudaStream_t s) {
  tile_flags_kernel<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(g, tw, ntiles, flags, tiles);
  return cudaGetLastError();
}

// One thread advances the batch step counter (read by the next batched step).
__global__ void batch_advance_kernel(long long* counter) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *counter += 1;
}

cudaError_t aa_launch_batch_advance(long long* counter, cudaStream_t s) {
  batch_advance_kernel<<<1, 32, 0, s>>>(counter);
  return cudaGetLastError();
}

// ---- z-slab halo messages ------------------------------------------------------------
// One thread per (crossing direction k, x, y) of a face.  `inward` = c_z of the
// directions entering the slab through this face (+1 at z-lo, -1 at z-hi).
//   after an even-phase step (swapped layout):
//     pack   the boundary plane's slots with c_z = inward (post-collision values that the
//            neighbour's first plane pulls across the face in the odd phase);
//     unpack into the ghost plane's slots with c_z = -inward (the neighbour's values that
//            this slab's boundary plane pulls);
//   after an odd-phase step:
//     pack   the ghost plane's slots with c_z = -inward (what the boundary plane pushed
//            across the face: they belong to the neighbour's boundary plane);
//     unpack into the boundary plane's slots with c_z = inward, only where the source node
//            x - c_d (a ghost node) is fluid: otherwise the node wrote that slot itself
//            (bounce-back) or, outside a non-periodic face, its face rule did.
// The crossing directions are taken in ascending order on both sides of a face, so a
// message packed by one slab unpacks unchanged in its neighbour.
template <class T>
__global__ void halo_kernel(const Grid g, const int side, const int after_even, const int pack, T* __restrict__ A,
                            const uint8_t* __restrict__ flags, T* __restrict__ buf) {
  const long long nxy = (long long)g.nx * g.ny;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 5 * nxy) return;
  const int k = (int)(t / nxy);
  const long long r = t - (long long)k * nxy;
  const int y = (int)(r / g.nx), x = (int)(r - (long long)y * g.nx);
  const int inward = side == 0 ? 1 : -1;
  const int zg = side == 0 ? 0 : g.nz - 1;  // ghost plane
  const int zb = zg + inward;                // boundary plane
  // slot set and plane of this call
  const bool boundary_side = after_even ? pack : !pack;
  const int sgn = boundary_side ? inward : -inward;
  const int z = boundary_side ? zb : zg;
  int d = -1;
  for (int e = 0, n = 0; e < 19; e++)
    if (cz(e) == sgn && n++ == k) d = e;
  T* slot = A + (long long)d * g.plane + node_index(g, x, y, z);
  if (pack) {
    buf[t] = *slot;
    return;
  }
  if (!after_even) {
    int sx = x - cx(d), sy = y - cy(d);
    if (sx < 0 || sx >= g.nx) {
      if (!g.per[0]) return;
      sx = (sx + g.nx) % g.nx;
    }
    if (sy < 0 || sy >= g.ny) {
      if (!g.per[1]) return;
      sy = (sy + g.ny) % g.ny;
    }
    if (flags[node_index(g, sx, sy, zg)] & F_SOLID) return;
  }
  *slot = buf[t];
}

cudaError_t aa_launch_halo(const Grid& g, int elem, int side, bool after_even, bool pack, void* A,
                           const uint8_t* flags, void* buf, cudaStream_t s) {
  const long long n = 5LL * g.nx * g.ny;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  const int ae = after_even ? 1 : 0, pk = pack ? 1 : 0;
  if (elem == 2)
    halo_kernel<uint16_t><<<blocks, 256, 0, s>>>(g, side, ae, pk, (uint16_t*)A, flags, (uint16_t*)buf);
  else if (elem == 4)
    halo_kernel<uint32_t><<<blocks, 256, 0, s>>>(g, side, ae, pk, (uint32_t*)A, flags, (uint32_t*)buf);
  else
    halo_kernel<uint64_t><<<blocks, 256, 0, s>>>(g, side, ae, pk, (uint64_t*)A, flags, (uint64_t*)buf);
  return cudaGetLastError();
}

}  // namespace lbm
