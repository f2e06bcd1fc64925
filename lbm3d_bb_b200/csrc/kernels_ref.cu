// kernels_ref.cu — the reference step (MainCore.jl:245-379), fused into one kernel.
//
// The reference keeps two population arrays and runs, per step,
//   collision! -> streaming! -> periodic_BC! -> solid_BC! -> velocity_BC!
//   -> compute_aero! -> compute_macros!
// with every node (solids included) collided and streamed.  Here the state
// between steps is F = f*_{n-1} (post-collision) plus R = (rho, u, v, w) of
// S_{n-1}; one kernel per step pulls S_n from F with the reference's wrap rules,
// applies the solid bounce-back and the face conditions in registers, reduces the
// momentum exchange, writes R_n (compute_macros!) and F_n = collide(S_n, R_n)
// into the other buffer pair.
//
// This file is compiled with --fmad=false and keeps the reference's operation
// order, so FP32 results round exactly as the reference kernels written in
// plain Float32 arithmetic (no fused multiply-add) do.
#include "lbm_internal.cuh"
#include "lbm_kernels.h"
#include "shapes.cuh"

namespace lbm {

// D3Q19: the lattice of lbm_internal.cuh.
namespace ref19 {
#include "ref_impl.cuh"
}  // namespace ref19

// D3Q27 (Utilities.jl:962-976): the D3Q19 directions first, then the eight corners, rest
// last; opposite pairs (2k, 2k+1); weights 2/27, 1/54, 1/216, 8/27.
namespace ref27 {
constexpr int Q = 27;
__host__ __device__ __forceinline__ constexpr int cx(int d) { return cx27(d); }
__host__ __device__ __forceinline__ constexpr int cy(int d) { return cy27(d); }
__host__ __device__ __forceinline__ constexpr int cz(int d) { return cz27(d); }
__host__ __device__ __forceinline__ constexpr int opp(int d) { return d == 26 ? 26 : (d ^ 1); }
template <class T>
__host__ __device__ __forceinline__ T wgt(int d) {
  return wgt27<T>(d);
}
#include "ref_impl.cuh"
}  // namespace ref27

// ---- launchers (the lattice follows the grid: g.q = 19 or 27) ------------------------
template <class T, bool TRT, int QN>
static void step_one(const RefParams& p, const void* Fp, const void* Rp, void* Fn, void* Rn, const uint8_t* flags,
                     dim3 grid, dim3 block, cudaStream_t s) {
  if constexpr (QN == 27)
    ref27::ref_step_kernel<T, TRT><<<grid, block, 0, s>>>(p, (const T*)Fp, (const T*)Rp, (T*)Fn, (T*)Rn, flags);
  else
    ref19::ref_step_kernel<T, TRT><<<grid, block, 0, s>>>(p, (const T*)Fp, (const T*)Rp, (T*)Fn, (T*)Rn, flags);
}

cudaError_t ref_launch_step(bool fp64, bool trt, const RefParams& p, const void* Fp, const void* Rp,
                            void* Fn, void* Rn, const uint8_t* flags, dim3 grid, dim3 block,
                            cudaStream_t s) {
  const bool q27 = p.g.q == 27;
  if (fp64) {
    if (trt)
      q27 ? step_one<double, true, 27>(p, Fp, Rp, Fn, Rn, flags, grid, block, s)
          : step_one<double, true, 19>(p, Fp, Rp, Fn, Rn, flags, grid, block, s);
    else
      q27 ? step_one<double, false, 27>(p, Fp, Rp, Fn, Rn, flags, grid, block, s)
          : step_one<double, false, 19>(p, Fp, Rp, Fn, Rn, flags, grid, block, s);
  } else {
    if (trt)
      q27 ? step_one<float, true, 27>(p, Fp, Rp, Fn, Rn, flags, grid, block, s)
          : step_one<float, true, 19>(p, Fp, Rp, Fn, Rn, flags, grid, block, s);
    else
      q27 ? step_one<float, false, 27>(p, Fp, Rp, Fn, Rn, flags, grid, block, s)
          : step_one<float, false, 19>(p, Fp, Rp, Fn, Rn, flags, grid, block, s);
  }
  return cudaGetLastError();
}

template <class T>
static void export_one(const RefParams& p, const void* Fp, const void* Rp, int direct, const uint8_t* flags,
                       const ExportOut& out, double* mass, dim3 grid, dim3 block, cudaStream_t s) {
  if (p.g.q == 27)
    ref27::ref_export_kernel<T><<<grid, block, 0, s>>>(p, (const T*)Fp, (const T*)Rp, direct, flags, out, mass);
  else
    ref19::ref_export_kernel<T><<<grid, block, 0, s>>>(p, (const T*)Fp, (const T*)Rp, direct, flags, out, mass);
}

cudaError_t ref_launch_export(bool fp64, const RefParams& p, const void* Fp, const void* Rp, int direct,
                              const uint8_t* flags, const ExportOut& out, double* mass, dim3 grid,
                              dim3 block, cudaStream_t s) {
  if (fp64)
    export_one<double>(p, Fp, Rp, direct, flags, out, mass, grid, block, s);
  else
    export_one<float>(p, Fp, Rp, direct, flags, out, mass, grid, block, s);
  return cudaGetLastError();
}

template <class T, bool TRT>
static void prepare_one(const RefParams& p, const void* S0, void* F, void* R, dim3 grid, dim3 block,
                        cudaStream_t s) {
  if (p.g.q == 27)
    ref27::ref_prepare_kernel<T, TRT><<<grid, block, 0, s>>>(p, (const T*)S0, (T*)F, (T*)R);
  else
    ref19::ref_prepare_kernel<T, TRT><<<grid, block, 0, s>>>(p, (const T*)S0, (T*)F, (T*)R);
}

cudaError_t ref_launch_prepare(bool fp64, bool trt, const RefParams& p, const void* S0, void* F, void* R,
                               dim3 grid, dim3 block, cudaStream_t s) {
  if (fp64) {
    if (trt)
      prepare_one<double, true>(p, S0, F, R, grid, block, s);
    else
      prepare_one<double, false>(p, S0, F, R, grid, block, s);
  } else {
    if (trt)
      prepare_one<float, true>(p, S0, F, R, grid, block, s);
    else
      prepare_one<float, false>(p, S0, F, R, grid, block, s);
  }
  return cudaGetLastError();
}

cudaError_t ref_launch_init(bool fp64, const InitParams& p, void* S, dim3 grid, dim3 block, cudaStream_t s) {
  const bool q27 = p.g.q == 27;
  if (fp64) {
    if (q27)
      ref27::ref_init_kernel<double><<<grid, block, 0, s>>>(p, (double*)S);
    else
      ref19::ref_init_kernel<double><<<grid, block, 0, s>>>(p, (double*)S);
  } else {
    if (q27)
      ref27::ref_init_kernel<float><<<grid, block, 0, s>>>(p, (float*)S);
    else
      ref19::ref_init_kernel<float><<<grid, block, 0, s>>>(p, (float*)S);
  }
  return cudaGetLastError();
}

cudaError_t ref_launch_macros(bool fp64, const Grid& g, const void* R, const ExportOut& out, dim3 grid,
                              dim3 block, cudaStream_t s) {
  if (fp64)
    ref19::ref_macros_kernel<double><<<grid, block, 0, s>>>(g, (const double*)R, out);
  else
    ref19::ref_macros_kernel<float><<<grid, block, 0, s>>>(g, (const float*)R, out);
  return cudaGetLastError();
}

}  // namespace lbm
