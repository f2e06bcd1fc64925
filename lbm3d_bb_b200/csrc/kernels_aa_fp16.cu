// kernels_aa_fp16.cu — the configurable AA step kernels for StF16 storage.
#include "aa_impl.cuh"

namespace lbm {
LBM_AA_DEFINE_OPS(StF16, fp16)
}  // namespace lbm
