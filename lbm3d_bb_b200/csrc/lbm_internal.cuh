// lbm_internal.cuh — shared definitions of the liblbm3d kernels.
//
// D3Q19 lattice in the reference's direction order (Utilities.jl:949-960),
// 0-based; opposite pairs are (2k, 2k+1) and the rest direction is 18.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lbm3d.h"

namespace lbm {

constexpr int Q = 19;

__host__ __device__ __forceinline__ constexpr int cx(int d) {
  constexpr int t[19] = {1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0};
  return t[d];
}
__host__ __device__ __forceinline__ constexpr int cy(int d) {
  constexpr int t[19] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0};
  return t[d];
}
__host__ __device__ __forceinline__ constexpr int cz(int d) {
  constexpr int t[19] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 0};
  return t[d];
}
__host__ __device__ __forceinline__ constexpr int opp(int d) { return d == 18 ? 18 : (d ^ 1); }

// Weights as FP32/FP64-rounded rationals (Float32.(W), Utilities.jl:954-958).
template <class T>
__host__ __device__ __forceinline__ T wgt(int d) {
  return d < 6 ? T(1) / T(18) : (d < 18 ? T(1) / T(36) : T(1) / T(3));
}

// D3Q27 of gen_lattice_sets (Utilities.jl:962-976), 0-based: directions 0..17 are the
// D3Q19 ones, 18..25 the corners, 26 the rest; opposite pairs (2k, 2k+1); weights 2/27,
// 1/54, 1/216, 8/27.  The reference-mode step runs on either lattice.
__host__ __device__ __forceinline__ constexpr int cx27(int d) {
  constexpr int t[27] = {1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 0};
  return t[d];
}
__host__ __device__ __forceinline__ constexpr int cy27(int d) {
  constexpr int t[27] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 0};
  return t[d];
}
__host__ __device__ __forceinline__ constexpr int cz27(int d) {
  constexpr int t[27] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, 0};
  return t[d];
}
template <class T>
__host__ __device__ __forceinline__ T wgt27(int d) {
  return d < 6 ? T(2) / T(27) : (d < 18 ? T(1) / T(54) : (d < 26 ? T(1) / T(216) : T(8) / T(27)));
}

// ---- node flag byte ----------------------------------------------------------------
// SOLID / MOVING describe the flags of the latest body update; SOLID_PREV /
// MOVING_PREV those of the last completed step.  NEAR marks a node whose step
// needs the neighbour flags: config mode — a fluid node with a solid neighbour in
// either flag set, or an uncovered (fresh) node; reference mode — mask_bb
// (Geometry.jl:122-148).
enum : uint8_t {
  F_SOLID = 1u << 0,
  F_SOLID_PREV = 1u << 1,
  F_NEAR = 1u << 2,
  F_STATIC = 1u << 3,
  F_MOVING = 1u << 4,
  F_MOVING_PREV = 1u << 5,
};

// Body description in device-friendly form.
struct BodyDev {
  int kind;
  double center[3];
  double cos_t, sin_t;
  double rot[9];
  double radius;
  double semi[3];
  double chord, naca_m, naca_p, naca_t, x_int, x_le_offset;
  double h;  // reference shapes: physical length per cell
};

// Half-step rigid-body kinematics of the moving body (lattice units).
struct Kinematics {
  double center[3];
  double vel[3];
  double omega[3];
  double cos_t, sin_t;  // planar angle of the pose (reference shapes: phi of the interpolated bounce-back)
};

// Domain geometry shared by the step kernels.
struct Grid {
  int nx, ny, nz;
  int per[3];
  long long N;      // nodes
  long long plane;  // elements between direction planes
  int q;            // lattice: 19, or 27 (reference mode)
};

struct Box {
  int lo[3], hi[3];  // inclusive; may wrap on periodic axes (hi < lo not used: split by host)
};

inline __host__ __device__ long long node_index(const Grid& g, int x, int y, int z) {
  return (long long)x + (long long)g.nx * ((long long)y + (long long)g.ny * z);
}

}  // namespace lbm
