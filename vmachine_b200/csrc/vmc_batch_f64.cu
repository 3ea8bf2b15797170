// double instantiation of the multi-system kernels (its own unit, with its own
// constant-memory system table and Hermite coefficients).
#include "vmc_batch_kernels.cuh"

namespace vmc {

BatchOps batch_ops_f64() { return make_batch_ops<double>(); }

}  // namespace vmc
