// double instantiations of the walker kernels (compiled as their own unit so the two
// precisions build in parallel).  Each unit carries its own Hermite coefficient
// table in constant memory.
#include "vmc_kernels.cuh"

namespace vmc {

bool select_kernels_f64(int dim, int K, int flags, KernelSet &out)
{
    return select_kernels<double>(dim, K, flags, out);
}

cudaError_t upload_hermite_f64(const HermiteCoef &h)
{
    return cudaMemcpyToSymbol(c_herm, &h, sizeof(h));
}

}  // namespace vmc
