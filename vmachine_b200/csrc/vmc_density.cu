// Electron densities (Sampler::computeOneBodyDensity, computeOneBodyDensity2,
// computeTwoBodyDensity and their printers, src/sampler.cpp:518-581,639-692).
//
// The reference counts, at every sampled step of its last iteration, each
// particle's radial bin, its cell of a square grid in the first two coordinates,
// and the radial bins of every pair; the counts of all ranks are summed.  Here the
// sweep adds the same counts for every walker to 64-bit histograms in device memory
// (lanes over particles, atomics; the two-body counts take N(N-1)/2 atomics per
// walker-step), and the host reads them once.  Files are written as the reference's
// Eigen integer vectors and matrices: one common right-aligned width, one space
// between values, one row per line.
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "vmc_engine.hpp"

using namespace vmc;

namespace {

int dn_fail(int code, const std::string &m) { return set_last_error(code, m.c_str()); }

#define DNCUDA(expr)                                                                         \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) return dn_fail(VMC_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

}  // namespace

namespace vmc {

// Turn the density histograms of the next vmc_sample calls on (bins > 0) or off.
int density_begin(vmc_engine *e, int bins, double max_radius, bool radial, bool spatial, bool pair)
{
    const size_t b = (size_t)bins, b2 = b * b;
    if (radial) DNCUDA(cudaMalloc(&e->d_dens_radial, b * sizeof(unsigned long long)));
    if (spatial) DNCUDA(cudaMalloc(&e->d_dens_grid, b2 * sizeof(unsigned long long)));
    if (pair) DNCUDA(cudaMalloc(&e->d_dens_pair, b2 * sizeof(unsigned long long)));
    if (radial) DNCUDA(cudaMemsetAsync(e->d_dens_radial, 0, b * sizeof(unsigned long long), e->stream));
    if (spatial) DNCUDA(cudaMemsetAsync(e->d_dens_grid, 0, b2 * sizeof(unsigned long long), e->stream));
    if (pair) DNCUDA(cudaMemsetAsync(e->d_dens_pair, 0, b2 * sizeof(unsigned long long), e->stream));
    e->dens_bins = bins;
    e->dens_max = max_radius;
    e->dens_step = max_radius / bins;  // m_radialStep (sampler.cpp:43)
    return VMC_OK;
}

// Copy the histograms out (null: skip) and release them.
int density_end(vmc_engine *e, uint64_t *radial, uint64_t *spatial, uint64_t *pair)
{
    const size_t b = (size_t)e->dens_bins, b2 = b * b;
    int rc = VMC_OK;
    auto get = [&](unsigned long long *d, uint64_t *h, size_t n) {
        if (d && h && rc == VMC_OK) {
            const cudaError_t ce = cudaMemcpyAsync(h, d, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream);
            if (ce != cudaSuccess) rc = dn_fail(VMC_E_CUDA, std::string("density copy: ") + cudaGetErrorString(ce));
        }
    };
    get(e->d_dens_radial, radial, b);
    get(e->d_dens_grid, spatial, b2);
    get(e->d_dens_pair, pair, b2);
    cudaStreamSynchronize(e->stream);
    cudaFree(e->d_dens_radial);
    cudaFree(e->d_dens_grid);
    cudaFree(e->d_dens_pair);
    e->d_dens_radial = e->d_dens_grid = e->d_dens_pair = nullptr;
    e->dens_bins = 0;
    return rc;
}

std::string format_counts(const uint64_t *v, int rows, int cols)
{
    size_t width = 0;
    for (size_t i = 0; i < (size_t)rows * cols; ++i) width = std::max(width, std::to_string(v[i]).size());
    std::ostringstream os;
    for (int r = 0; r < rows; ++r) {
        if (r) os << '\n';
        for (int c = 0; c < cols; ++c) {
            if (c) os << ' ';
            const std::string t = std::to_string(v[(size_t)r * cols + c]);
            os << std::string(width - t.size(), ' ') << t;
        }
    }
    os << '\n';
    return os.str();
}

int write_counts(const std::string &path, const uint64_t *v, int rows, int cols)
{
    std::ofstream out(path);
    if (!out) return dn_fail(VMC_E_ARG, "cannot write '" + path + "'");
    out << format_counts(v, rows, cols);
    return out ? VMC_OK : dn_fail(VMC_E_ARG, "cannot write '" + path + "'");
}

}  // namespace vmc

extern "C" {

int vmc_densities(vmc_engine *e, int steps, int burn_in, int bins, double max_radius, uint64_t *radial,
                  uint64_t *spatial, uint64_t *two_body)
{
    if (!e) return dn_fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) return dn_fail(VMC_E_STATE, "vmc_init_walkers first");
    if (bins < 2 || bins > 1 << 14 || !(max_radius > 0.0)) return dn_fail(VMC_E_ARG, "bad density grid");
    if (!radial && !spatial && !two_body) return dn_fail(VMC_E_ARG, "no density requested");
    if (spatial && e->dim < 2) return dn_fail(VMC_E_ARG, "the spatial density needs two dimensions");
    DNCUDA(cudaSetDevice(e->device));
    int rc = density_begin(e, bins, max_radius, radial, spatial, two_body);
    if (!rc) {
        vmc_sums s{};
        rc = vmc_sample(e, 0, steps, burn_in, &s, nullptr, nullptr);
    }
    const int rc2 = density_end(e, radial, spatial, two_body);
    return rc ? rc : rc2;
}

}  // extern "C"
