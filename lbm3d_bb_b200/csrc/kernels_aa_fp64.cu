// kernels_aa_fp64.cu — the configurable AA step kernels for StF64 storage.
#include "aa_impl.cuh"

namespace lbm {
LBM_AA_DEFINE_OPS(StF64, fp64)
}  // namespace lbm
