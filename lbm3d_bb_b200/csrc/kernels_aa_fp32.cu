// kernels_aa_fp32.cu — the configurable AA step kernels for StF32 storage.
#include "aa_impl.cuh"

namespace lbm {
LBM_AA_DEFINE_OPS(StF32, fp32)
}  // namespace lbm
