// Allocation-free local energies: vmc_local_energies_noalloc (include/vmc_b200.h).
//
// Some callers cannot allocate device memory at the moment they need an energy:
// a serving process whose memory is held by another framework's caching pool
// (an extra cudaMalloc would fail or fragment it), a loop that must not stall
// other streams (cudaFree synchronises the whole device), or code that runs
// while a CUDA stream is being captured into a graph, where allocation calls are
// not permitted.  This entry point therefore creates no engine and allocates
// nothing: every intermediate (walker records, pair sums, masks, status words,
// gradients) lives in one file-scope device array of fixed size, and the caller
// passes its own device buffers for the positions and the energies.
//
// The array is shared by every call in the process on a device.  Two calls
// whose work overlaps on the GPU (different streams, or different host threads,
// without ordering between them) race on it and corrupt each other's results:
// callers serialise their calls, e.g. by issuing them on one stream.
//
// The work per call is four launches on the caller's stream: stage (positions
// into zeroed records, cleared pair sums / status words, masks set), the
// engine's FP64 rebuild of every derived array (Gauss-Jordan inversion of the
// Slater blocks, Pade pair sums), the engine's FP64 evaluation, and a flag pass
// that marks walkers with a singular Slater block.  The values equal those of
// vmc_init_walkers + vmc_eval on an FP64 engine at the same positions.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "vmc_b200.h"
#include "vmc_config.hpp"
#include "vmc_kernels.cuh"

namespace vmc {
bool select_kernels_f64(int dim, int K, int flags, KernelSet &out);
cudaError_t upload_hermite_f64(const HermiteCoef &h);
int set_last_error(int code, const char *msg);  // vmc_engine.cu: message for vmc_last_error
unsigned long long current_context_id();        // vmc_engine.cu: 0 when it cannot be told
}  // namespace vmc

using namespace vmc;

// The scratch array.  Its size is VMC_NOALLOC_SCRATCH_BYTES (32 MiB); the
// device memory is reserved when this file's module is loaded on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[VMC_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
unsigned long long g_setup_ctx[kMaxDevices] = {0};  // the context the set-up was made in

int err(int code, const std::string &msg) { return set_last_error(code, msg.c_str()); }

int cuda_err(const char *what, cudaError_t e)
{
    return err(VMC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Once per device and context, with that device current: address of the scratch
// array and the Hermite recurrence coefficients of the FP64 kernels (synchronous
// copies, which is why the first call on a device must not come during stream
// capture).  A new context on the device (after cudaDeviceReset, the module loaded
// again) gets the set-up again: the array's address and the constant tables are the
// context's.
int setup_device(int device, unsigned char **scratch)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_context_id();
    if (g_scratch_ptr[device] && ctx != 0 && g_setup_ctx[device] == ctx) {
        *scratch = g_scratch_ptr[device];
        return VMC_OK;
    }
    void *ptr = nullptr;
    cudaError_t ce = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (ce != cudaSuccess) return cuda_err("cudaGetSymbolAddress(scratch)", ce);
    // the recurrence coefficients the kernels read (the values vmc_create uploads)
    HermiteCoef h;
    for (int m = 0; m < HMAX; ++m) {
        h.A[m] = std::sqrt(2.0 / (m + 1));
        h.B[m] = std::sqrt((double)m / (m + 1));
        h.C[m] = std::sqrt(2.0 * m);
        h.E[m] = 2.0 * std::sqrt((double)m * (m - 1 > 0 ? m - 1 : 0));
        h.Af[m] = (float)h.A[m];
        h.Bf[m] = (float)h.B[m];
        h.Cf[m] = (float)h.C[m];
        h.Ef[m] = (float)h.E[m];
    }
    ce = upload_hermite_f64(h);
    if (ce != cudaSuccess) return cuda_err("Hermite coefficient upload", ce);
    g_scratch_ptr[device] = static_cast<unsigned char *>(ptr);
    g_setup_ctx[device] = ctx;
    *scratch = g_scratch_ptr[device];
    return VMC_OK;
}

// The validated system: the same acceptance rules as vmc_create.
struct System {
    Config c;
    int flags = 0, K = 0, D = 0, n_orb = 0, E = 0, Pmax = 0, EP = 0, nacc = 0;
};

int describe(const char *text, System &s)
{
    const std::string msg = parse_config(text, s.c);
    if (!msg.empty()) return err(VMC_E_CONFIG, msg);
    const Config &c = s.c;
    auto reject = [](const std::string &m) { return err(VMC_E_UNSUPPORTED, m); };
    if (c.hamiltonian.empty()) return reject("no hamiltonian given (the reference requires one)");
    if (c.hamiltonian != "harmonicOscillator" && c.hamiltonian != "atomicNucleus")
        return reject("hamiltonian '" + c.hamiltonian + "' is not on the engine's path");
    if (c.dim != 2 && c.dim != 3) return reject("numDimensions must be 2 or 3");
    if (c.elements.empty()) return reject("no wave function elements");
    if ((int)c.elements.size() > MAX_ELEM) return reject("too many elements");
    if (c.N < 2 || c.N > MAX_N) return reject("numParticles must be in [2, 64]");
    int n_gauss = 0, n_pade = 0, n_slater = 0;
    for (int el : c.elements) {
        switch (el) {
        case E_GAUSSIAN: s.flags |= F_GAUSS; ++n_gauss; break;
        case E_PADE: s.flags |= F_PADE; ++n_pade; break;
        case E_HYDROGENLIKE: s.flags |= F_HYDROGENLIKE; break;
        case E_SLATER: {
            if (c.basis != "hermite") return reject("Slater determinant needs basis: hermite on this engine");
            // closed shells: 2 * C(K-1+dim, dim) == N
            s.K = -1;
            for (int k = 1; k <= 9; ++k) {
                long n = 1;
                for (int i = 1; i <= c.dim; ++i) n = n * (k - 1 + i) / i;
                if (2 * n == c.N) { s.K = k; break; }
                if (2 * n > c.N) break;
            }
            if (s.K < 0) return reject("open shell: numParticles is not a closed shell");
            if ((c.dim == 2 && s.K > 7) || (c.dim == 3 && s.K > 4)) return reject("too many shells");
            s.flags |= F_SLATER;
            ++n_slater;
            break;
        }
        default: return reject("wave function element not implemented on the engine");
        }
    }
    if (n_gauss > 1 || n_pade > 1 || n_slater > 1) return reject("repeated element");
    if (c.coulomb) s.flags |= F_COULOMB;
    if (c.hamiltonian == "atomicNucleus") s.flags |= F_ATOM;
    if (c.compat) s.flags |= Q_PADE_RATIO | Q_PADE_DGAMMA | Q_IS_GREEN | Q_PADE_STALE;
    if (c.sampling != "bruteForce") s.flags |= F_IS;
    s.D = c.N * c.dim;
    s.n_orb = s.K > 0 ? c.N / 2 : 0;
    s.E = (int)c.elements.size();
    for (int el : c.elements) s.Pmax = std::max(s.Pmax, element_parameters(c, el));
    s.EP = s.E * s.Pmax;
    s.nacc = 9 + 2 * s.EP;
    if (s.nacc > 32) return reject("more than 11 parameters per walker is not supported");
    return VMC_OK;
}

// Offsets of the per-call regions inside the scratch array, each 256-byte aligned.
struct Carve {
    size_t rec, scal, mask, status, grad, lap, pgrad, total;
};

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

Carve carve(const System &s, const Layout &L, size_t W)
{
    Carve k{};
    size_t o = 0;
    k.rec = o;    o += align256(W * L.rec * sizeof(double));
    k.scal = o;   o += align256(W * NSCAL * sizeof(double));
    k.mask = o;   o += align256(W * s.c.N * sizeof(unsigned long long));
    k.status = o; o += align256(W * sizeof(unsigned));
    k.grad = o;   o += align256(W * s.E * s.D * sizeof(double));
    k.lap = o;    o += align256(W * s.E * sizeof(double));
    k.pgrad = o;  o += align256(W * s.E * s.Pmax * sizeof(double));
    k.total = o;
    return k;
}

// Stage the walkers: each record is zero except its positions; pair sums and
// status words start at zero, and every Pade pair is marked current (as
// vmc_init_walkers leaves them).  These are the parts of the shared array that
// must not carry values over from an earlier call.
__global__ void noalloc_stage_kernel(Layout L, int W, int N, const double *__restrict__ pos,
                                     double *__restrict__ rec, double *__restrict__ scal,
                                     unsigned long long *__restrict__ mask,
                                     unsigned *__restrict__ status)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n_rec = (size_t)W * L.rec;
    for (size_t i = t0; i < n_rec; i += stride) {
        const size_t w = i / L.rec;
        const int c = (int)(i - w * L.rec) - L.off_x;
        rec[i] = (c >= 0 && c < L.D) ? pos[w * L.D + c] : 0.0;
    }
    for (size_t i = t0; i < (size_t)W * NSCAL; i += stride) scal[i] = 0.0;
    for (size_t i = t0; i < (size_t)W * N; i += stride) mask[i] = ~0ull;
    for (size_t i = t0; i < (size_t)W; i += stride) status[i] = 0u;
}

// Walkers whose Slater block was singular at these positions get NaN energies.
__global__ void noalloc_flag_kernel(int W, const unsigned *__restrict__ status,
                                    double *__restrict__ energies)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < W && (status[w] & ST_SINGULAR)) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        energies[3 * (size_t)w] = energies[3 * (size_t)w + 1] = energies[3 * (size_t)w + 2] = nan;
    }
}

int check_device_pointer(const void *p, int device, const char *name)
{
    cudaPointerAttributes at{};
    const cudaError_t ce = cudaPointerGetAttributes(&at, p);
    if (ce != cudaSuccess) return cuda_err(name, ce);
    if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != device)
        return err(VMC_E_ARG, std::string(name) + " is not device memory of the current device");
    if (reinterpret_cast<uintptr_t>(p) % alignof(double))
        return err(VMC_E_ARG, std::string(name) + " is not 8-byte aligned");
    return VMC_OK;
}

}  // namespace

extern "C" int vmc_local_energies_noalloc(const char *input_in_text, const double *theta,
                                          int n_elements, int p_max, const double *positions,
                                          int n_walkers, double *energies, void *stream)
{
    if (!input_in_text || !theta) return err(VMC_E_ARG, "null argument");
    if (n_walkers < 0) return err(VMC_E_ARG, "n_walkers must be >= 0");
    System s;
    int rc = describe(input_in_text, s);
    if (rc) return rc;
    if (n_elements != s.E || p_max != s.Pmax) return err(VMC_E_ARG, "parameter shape mismatch");
    const Layout L = make_layout(s.c.N, s.c.dim, s.n_orb, (int)sizeof(double));
    const size_t W = (size_t)n_walkers;
    const Carve k = carve(s, L, W);
    if (k.total > VMC_NOALLOC_SCRATCH_BYTES) {
        size_t fit = 0;  // largest walker count whose regions fit
        for (size_t step = (size_t)1 << 20; step; step >>= 1)
            if (carve(s, L, fit + step).total <= VMC_NOALLOC_SCRATCH_BYTES) fit += step;
        return err(VMC_E_ARG, "n_walkers=" + std::to_string(n_walkers) + " needs " +
                                  std::to_string(k.total) + " bytes of scratch; the fixed array holds " +
                                  std::to_string((size_t)VMC_NOALLOC_SCRATCH_BYTES) +
                                  " bytes, at most " + std::to_string(fit) +
                                  " walkers of this system");
    }
    if (n_walkers == 0) return VMC_OK;
    if (!positions || !energies) return err(VMC_E_ARG, "null argument");
    KernelSet ks;
    if (!select_kernels_f64(s.c.dim, s.K, s.flags, ks)) return err(VMC_E_UNSUPPORTED, "no kernel for this shape");
    int device = 0;
    cudaError_t ce = cudaGetDevice(&device);
    if (ce != cudaSuccess) return cuda_err("cudaGetDevice", ce);
    if (device < 0 || device >= kMaxDevices) return err(VMC_E_ARG, "device index out of range");
    if ((rc = check_device_pointer(positions, device, "positions"))) return rc;
    if ((rc = check_device_pointer(energies, device, "energies"))) return rc;
    unsigned char *scratch = nullptr;
    if ((rc = setup_device(device, &scratch))) return rc;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);

    Params P{};
    P.L = L;
    P.W = n_walkers;
    P.N = s.c.N;
    P.n_elem = s.E;
    P.ep = s.EP;
    P.nacc = s.nacc;
    for (int i = 0; i < s.E; ++i) P.elem_kind[i] = s.c.elements[i];
    P.flags = s.flags;
    P.sampling = s.c.sampling == "bruteForce" ? SAMPLER_BF : SAMPLER_IS;
    P.omega = s.c.omega;
    P.Z = s.c.Z;
    P.step = s.c.step_length;
    P.idx_alpha = P.idx_gamma = P.idx_alpha_h = -1;
    for (int i = 0; i < s.E && s.Pmax > 0; ++i) {  // no parameters: nothing to read
        const double t0 = theta[(size_t)i * s.Pmax];
        switch (s.c.elements[i]) {
        case E_GAUSSIAN: P.alpha = t0; P.idx_alpha = i * s.Pmax; break;
        case E_PADE: P.gamma = t0; P.idx_gamma = i * s.Pmax; break;
        case E_HYDROGENLIKE: P.alpha_h = t0; P.idx_alpha_h = i * s.Pmax; break;
        default: break;
        }
    }
    P.gamma_prev = P.gamma;
    // Pade spin coefficients (padejastrow.cpp:140-170)
    P.beta_same = s.c.dim == 2 ? 1.0 / 3 : 1.0 / 4;
    P.beta_anti = s.c.dim == 2 ? 1.0 : 1.0 / 2;
    P.state = scratch + k.rec;
    P.scal = reinterpret_cast<double *>(scratch + k.scal);
    P.mask = reinterpret_cast<unsigned long long *>(scratch + k.mask);
    P.status = reinterpret_cast<unsigned *>(scratch + k.status);
    P.counter = nullptr;  // neither the rebuild nor the evaluation draws random numbers
    P.acc = nullptr;      // nor accumulates samples

    const int stage_grid = (int)std::min<size_t>((W * L.rec + 255) / 256, 4096);
    noalloc_stage_kernel<<<stage_grid, 256, 0, st>>>(L, n_walkers, s.c.N, positions,
                                                     static_cast<double *>(P.state), P.scal, P.mask,
                                                     P.status);
    if ((ce = cudaGetLastError()) != cudaSuccess) return cuda_err("stage launch", ce);

    RebuildArgs ra{};
    ra.P = P;
    ra.mode = RB_INIT;
    ra.drift = nullptr;
    ra.wpb = 4;
    ra.smem_per_warp = rebuild_smem_per_warp(s.c.N, s.c.dim, s.n_orb);
    const size_t rb_smem = (size_t)ra.wpb * ra.smem_per_warp;  // <= 4 x 6.9 KB (28 orbitals): below the 48 KB default
    void *rb_args[1] = {&ra};
    ce = cudaLaunchKernel(ks.rebuild, dim3((n_walkers + ra.wpb - 1) / ra.wpb), dim3(32 * ra.wpb), rb_args,
                          rb_smem, st);
    if (ce != cudaSuccess) return cuda_err("rebuild launch", ce);

    EvalArgs ea{};
    ea.P = P;
    ea.p_max = s.Pmax;
    ea.grad = reinterpret_cast<double *>(scratch + k.grad);
    ea.lap = reinterpret_cast<double *>(scratch + k.lap);
    ea.pgrad = reinterpret_cast<double *>(scratch + k.pgrad);
    ea.energies = energies;
    void *ev_args[1] = {&ea};
    ce = cudaLaunchKernel(ks.eval, dim3((n_walkers + 3) / 4), dim3(128), ev_args, 0, st);
    if (ce != cudaSuccess) return cuda_err("eval launch", ce);

    noalloc_flag_kernel<<<(n_walkers + 255) / 256, 256, 0, st>>>(n_walkers, P.status, energies);
    if ((ce = cudaGetLastError()) != cudaSuccess) return cuda_err("flag launch", ce);
    return VMC_OK;
}
