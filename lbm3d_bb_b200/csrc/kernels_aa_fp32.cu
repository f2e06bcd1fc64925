// kernels_aa_fp32.cu — the configurable AA step kernels for StF32 storage.
#include "aa_impl.cuh"

namespace lbm {
LBM_AA_DEFINE_OPS(StF32, fp32)

cudaError_t aa_launch_wait_probe(int polls, int* err, cudaStream_t s) {
  wait_probe_kernel<<<1, 32, 0, s>>>(polls, err);
  return cudaGetLastError();
}
}  // namespace lbm
