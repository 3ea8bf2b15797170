// Host side of the walker engine: the C ABI declared in include/vmc_b200.h.
//
// Owns the device buffers and one CUDA stream per engine, selects the kernel
// instantiation for (precision, dimension, Hermite shells), and runs the
// reference's iteration semantics: burn-in, gradient window, averages, optimiser
// step, parameter broadcast (src/system.cpp:81-139, src/sampler.cpp:52-226).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "vmc_engine.hpp"

using namespace vmc;

namespace vmc {
// The same with packed FP32 pairs (FFMA2): 2 FMAs per instruction.
__global__ void fma2_peak_kernel(float *out, int iters, float m)
{
    float2 v[FMA_CHAINS];
    const float2 mm = make_float2(m, m);
#pragma unroll
    for (int i = 0; i < FMA_CHAINS; ++i) v[i] = make_float2(threadIdx.x + i, threadIdx.x - i);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < FMA_CHAINS; ++i) v[i] = __ffma2_rn(v[i], mm, mm);
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < FMA_CHAINS; ++i) s += v[i].x + v[i].y;
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace vmc

namespace vmc {
// Deterministic compensated reduction of the per-walker accumulators:
// one block, thread group per accumulator, fixed summation order.
__global__ void reduce_acc_kernel(const double *acc, int W, int nacc, double *out)
{
    const int a = blockIdx.x;  // accumulator index
    double s = 0.0, c = 0.0;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        kadd(s, c, acc[((size_t)w * nacc + a) * 2]);
        kadd(s, c, acc[((size_t)w * nacc + a) * 2 + 1]);
    }
    __shared__ double ss[256], cc[256];
    ss[threadIdx.x] = s;
    cc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, C = 0.0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            kadd(S, C, ss[t]);
            kadd(S, C, cc[t]);
        }
        out[a] = S + C;
    }
}

// Per-walker mean energy (accumulator 0: sum plus its compensation) gathered into one
// contiguous array, so that the host reads W doubles in one copy instead of W strided
// 16-byte rows.
__global__ void walker_means_kernel(const double *acc, int W, int nacc, double inv_n, double *out)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < W) out[w] = (acc[(size_t)w * nacc * 2] + acc[(size_t)w * nacc * 2 + 1]) * inv_n;
}
}  // namespace vmc

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

}  // namespace

// Error channel for entry points defined in other files (vmc_noalloc.cu).
int vmc::set_last_error(int code, const char *msg) { return fail(code, msg); }

namespace {

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess)                                                           \
            return fail(VMC_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

}  // namespace

namespace vmc {
bool select_kernels_f32(int dim, int K, int flags, KernelSet &out);
bool select_kernels_f64(int dim, int K, int flags, KernelSet &out);
cudaError_t upload_hermite_f32(const HermiteCoef &h);
cudaError_t upload_hermite_f64(const HermiteCoef &h);
}  // namespace vmc

namespace {

bool select_set(int precision, int dim, int K, int flags, KernelSet &out)
{
    return precision == VMC_PRECISION_MIXED ? select_kernels_f32(dim, K, flags, out)
                                            : select_kernels_f64(dim, K, flags, out);
}

}  // namespace

// Unique identifier of the calling thread's current CUDA context (cuCtxGetId through
// the runtime's driver entry points, so the library needs no link to the driver
// library), or 0 when it cannot be told.
unsigned long long vmc::current_context_id()
{
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
    return 0;
}

namespace {

uint4 host_philox(uint4 c, uint2 k)
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k.x, (uint32_t)p1,
                       (uint32_t)(p0 >> 32) ^ c.w ^ k.y, (uint32_t)p0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Constant-memory tables belong to the context the modules were loaded in: the
// upload is redone whenever the device's current context is not the one uploaded to
// (a context created after cudaDeviceReset starts with empty tables).
int hermite_init_device(int device)
{
    static std::mutex mu;
    static unsigned long long done[64] = {0};
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_context_id();
    if (device < 64 && ctx != 0 && done[device] == ctx) return VMC_OK;
    const HermiteCoef h = hermite_coefficients();
    CUDA_TRY(upload_hermite_f32(h));
    CUDA_TRY(upload_hermite_f64(h));
    CUDA_TRY(upload_hermite_gen(h));
    if (device < 64) done[device] = ctx;
    return VMC_OK;
}

}  // namespace

namespace {

void free_engine(vmc_engine *e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    cudaFree(e->d_state);
    cudaFree(e->d_scal);
    cudaFree(e->d_acc);
    cudaFree(e->d_out);
    cudaFree(e->d_drift);
    cudaFree(e->d_wmean);
    cudaFree(e->d_mask);
    cudaFree(e->d_counter);
    cudaFree(e->d_status);
    cudaFree(e->d_replay);
    cudaFree(e->d_theta);
    cudaFree(e->d_act);
    cudaFree(e->d_mlpw);
    cudaFree(e->d_snap_x);
    cudaFree(e->d_snap_e);
    cudaFree(e->d_mlp_out);
    cudaFree(e->d_pos);
    cudaFree(e->d_mlp_cache);
    cudaFree(e->d_dens_radial);
    cudaFree(e->d_dens_grid);
    cudaFree(e->d_dens_pair);
    for (cudaEvent_t ev : e->sweep_events) cudaEventDestroy(ev);
    if (e->sw0) cudaEventDestroy(e->sw0);
    if (e->sw1) cudaEventDestroy(e->sw1);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int closed_shells_2d(int N, int dim)
{
    // number of Hermite shells K with 2 * C(K-1+dim, dim) == N, or -1
    for (int K = 1; K <= 9; ++K) {
        long c = 1;
        for (int i = 1; i <= dim; ++i) c = c * (K - 1 + i) / i;
        if (2 * c == N) return K;
        if (2 * c > N) return -1;
    }
    return -1;
}

Params make_params(const vmc_engine *e)
{
    Params P{};
    P.L = e->L;
    P.W = e->W;
    P.N = e->N;
    P.n_elem = e->E;
    P.ep = e->EP;
    P.nacc = e->nacc_dev;
    P.walker_offset = e->cfg.walker_offset;
    P.drift_limit = e->cfg.drift_limit;
    for (int i = 0; i < e->E && i < MAX_ELEM; ++i) P.elem_kind[i] = e->cfg.elements[i];
    P.flags = e->flags;
    P.sampling = e->sampling;
    P.omega = e->cfg.omega;
    P.Z = e->cfg.Z;
    P.step = e->cfg.step_length;
    P.alpha = 0.0;
    P.gamma = 0.0;
    P.alpha_h = 0.0;
    P.idx_alpha = P.idx_gamma = P.idx_alpha_h = -1;
    for (int i = 0; i < e->E && e->Pmax > 0; ++i) {  // no parameters: nothing to read
        const double t0 = e->theta[(size_t)i * e->Pmax];
        switch (e->cfg.elements[i]) {
        case E_GAUSSIAN: P.alpha = t0; P.idx_alpha = i * e->Pmax; break;
        case E_PADE: P.gamma = t0; P.idx_gamma = i * e->Pmax; break;
        case E_HYDROGENLIKE: P.alpha_h = t0; P.idx_alpha_h = i * e->Pmax; break;
        default: break;
        }
    }
    P.gamma_prev = e->gamma_prev;
    P.mlpw = e->d_mlpw;
    P.mlp_cache = e->d_mlp_cache;
    P.mlp_cache_stride = e->N * e->N * 3 + e->N * 3;
    if (e->flags == FX_MLP_DOT) {  // compact accumulators: the Gaussian's alpha only
        P.ep = (int)e->act.size();
        P.idx_alpha = 0;
        P.idx_gamma = -1;
    }
    // Pade spin coefficients (padejastrow.cpp:140-170)
    P.beta_same = e->dim == 2 ? 1.0 / 3 : e->dim == 3 ? 1.0 / 4 : 1.0 / 5;
    P.beta_anti = e->dim == 2 ? 1.0 : e->dim == 3 ? 1.0 / 2 : 1.0 / 3;
    P.state = e->d_state;
    P.scal = e->d_scal;
    P.mask = e->d_mask;
    P.counter = e->d_counter;
    P.acc = e->d_acc;
    P.status = e->d_status;
    return P;
}

int launch(const void *fn, int grid, int block, size_t smem, cudaStream_t st, void *args)
{
    void *argv[1] = {args};
    CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(block), argv, smem, st));
    return VMC_OK;
}

int sweep_smem_per_warp(const vmc_engine *e)
{
    const int staged = e->L.rec;  // the whole record (InvInRegisters is off for every shape)
    return round_up(staged * (int)e->elem_bytes + e->N * 8 + NSCAL * 8, 16);
}

int run_rebuild(vmc_engine *e, int mode, double *drift)
{
    if (e->general) {
        // the FP32 sweep's refresh re-inverts in FP64; otherwise the FP64 inverse is
        // carried and only the evaluation is redone
        const int gm = mode == RB_INIT ? GEN_INIT : (e->gen.f32 && mode == RB_REFRESH) ? GEN_REFRESH : GEN_STATE;
        CUDA_TRY(gen_launch_state(make_params(e), e->gen, gm, nullptr, nullptr, nullptr, nullptr, e->stream));
        return VMC_OK;
    }
    RebuildArgs a{};
    a.P = make_params(e);
    a.mode = mode;
    a.drift = drift;
    a.wpb = 4;
    a.smem_per_warp = rebuild_smem_per_warp(e->N, e->dim, e->n_orb);
    const size_t smem = (size_t)a.wpb * a.smem_per_warp;
    CUDA_TRY(cudaFuncSetAttribute(e->ks.rebuild, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (e->W + a.wpb - 1) / a.wpb;
    int rc = launch(e->ks.rebuild, grid, 32 * a.wpb, smem, e->stream, &a);
    if (!rc && e->ks.rebuild_mlp) rc = launch(e->ks.rebuild_mlp, (e->W + 3) / 4, 128, 0, e->stream, &a);
    return rc;
}

void fill_owner_constants(const vmc_engine *e, SweepArgs &a)
{
    const Params &P = a.P;
    a.oc[OC_WA] = P.omega * P.alpha;
    a.oc[OC_HDT] = 0.5 * P.step;
    a.oc[OC_SDT] = std::sqrt(P.step);
    a.oc[OC_GAM] = P.gamma;
    a.oc[OC_GAMP] = P.gamma_prev;
    a.oc[OC_M2GAM] = -2.0 * P.gamma;
    a.oc[OC_BSAME] = P.beta_same;
    a.oc[OC_BANTI] = P.beta_anti;
    a.oc[OC_W2H] = 0.5 * P.omega * P.omega;
    a.oc[OC_MHOM] = -0.5 * P.omega;
    a.oc[OC_DGK] = (e->flags & Q_PADE_DGAMMA) ? -0.5 : -1.0;
    a.oc[OC_LAPC] = P.omega * P.alpha * e->D;
    for (int i = 0; i < OC_N; ++i) a.ocf[i] = (float)a.oc[i];
}

int run_sweep(vmc_engine *e, SweepArgs &a)
{
    a.P = make_params(e);
    if (e->general) {
        CUDA_TRY(gen_launch_sweep(a, e->gen, e->stream));
        return VMC_OK;
    }
    const bool plain = !a.probe_k && !a.replay && !a.rec_en && !a.rec_acc && !a.dens_bins;
    if (plain && e->owner) {
        fill_owner_constants(e, a);
        a.wpb = OWNER_WPB;
        a.smem_per_warp = e->ks.owner_smem;
        const size_t smem = (size_t)OWNER_WPB * a.smem_per_warp;
        CUDA_TRY(cudaFuncSetAttribute(e->ks.sweep_owner, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        return launch(e->ks.sweep_owner, (e->W + OWNER_WPB - 1) / OWNER_WPB, 32 * OWNER_WPB, smem, e->stream, &a);
    }
    const void *fn = plain ? e->ks.sweep_plain : e->ks.sweep;
    const int g = plain ? e->ks.seg : 1;  // walkers per warp
    a.wpb = e->wpb;
    a.smem_per_warp = g * sweep_smem_per_warp(e);
    // the MLP dot adds the CTA's weight block and tensor-core tiles in front
    const size_t smem = (size_t)a.wpb * a.smem_per_warp + (e->flags == FX_MLP_DOT ? MLP_FAST_BYTES + TC_SMEM : 0);
    CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (e->W + a.wpb * g - 1) / (a.wpb * g);
    return launch(fn, grid, 32 * a.wpb, smem, e->stream, &a);
}

int choose_wpb(vmc_engine *e)
{
    if (e->general) {
        e->wpb = 4;  // the general kernels' fixed warps per CTA
        return VMC_OK;
    }
    if (e->flags == FX_MLP_DOT) {
        e->wpb = 4;  // the CTA's four walkers fill one 128-row tensor-core tile
        return VMC_OK;
    }
    if (e->cfg.walkers_per_block > 0) {
        e->wpb = e->cfg.walkers_per_block;
        return VMC_OK;
    }
    const int per_warp = e->ks.seg * sweep_smem_per_warp(e);
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, e->ks.sweep_plain));
    int best = 1, best_warps = -1;
    for (int wpb : {8, 4, 2, 1}) {
        if (32 * wpb > fa.maxThreadsPerBlock) continue;
        const size_t smem = (size_t)wpb * per_warp;
        if (smem > 227 * 1024) continue;
        CUDA_TRY(cudaFuncSetAttribute(e->ks.sweep_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int blocks = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, e->ks.sweep_plain, 32 * wpb, smem));
        if (blocks * wpb > best_warps) {
            best_warps = blocks * wpb;
            best = wpb;
        }
    }
    e->wpb = best;
    return VMC_OK;
}

// Automatize::setupInitialWeights (automatize.cpp:55-105) with the configured
// initialWeights method.  Random methods draw from host Philox (stream tag 2).
int initial_weights(vmc_engine *e)
{
    const Config &c = e->cfg;
    e->theta.assign((size_t)e->E * e->Pmax, 0.0);
    std::string method = c.initial_weights;
    double factor = c.weights_factor;
    bool xavier = false;
    if (method == "automatize" && e->mlp_e >= 0) {
        // Slater / Gaussian next to the MLP Jastrow: the "VMC" rule (constant 1); the
        // MLP row is set below
        method = "constant";
        factor = 1.0;
    } else if (method == "automatize") {
        const std::string &t = c.trial_label;
        if (t == "VMC" || t == "BVMC") { method = "constant"; factor = 1.0; }
        else if (t == "RBM" || t == "RBMSJ" || t == "RBMPJ") { xavier = true; }
        else if (t == "PRBM") { method = "constant"; factor = 0.0; }
        else if (t == "SSJ") { method = "randomuniform"; factor = 0.2; }
        else { method = "randomuniform"; factor = 0.01; }
    }
    const unsigned long long s = e->seed;
    auto uniform = [&](uint32_t i) {
        const uint4 v = host_philox(make_uint4(i, 0u, 0u, 2u), make_uint2((uint32_t)s, (uint32_t)(s >> 32)));
        return v.x * 2.3283064365386963e-10;
    };
    if (xavier) {  // xavier.cpp:10-23
        const double lim = 1.0 / std::sqrt((double)e->D);
        for (size_t i = 0; i < e->theta.size(); ++i) e->theta[i] = -lim + 2 * lim * uniform((uint32_t)i);
        if (e->E > 3)
            for (int j = 0; j < e->Pmax; ++j) e->theta[3 * e->Pmax + j] = 0.2 * uniform((uint32_t)(e->theta.size() + j));
    } else if (method == "constant") {  // constant.cpp:11-26
        std::fill(e->theta.begin(), e->theta.end(), factor);
    } else if (method == "randomuniform") {  // randomuniform.cpp (weights)
        for (size_t i = 0; i < e->theta.size(); ++i) e->theta[i] = factor * uniform((uint32_t)i);
    } else if (method == "fromfile") {  // fromfile.cpp:30-79
        std::vector<double> th;
        const std::string why = read_weights_file(c.weights_file, e->E, e->Pmax, th);
        if (!why.empty()) return fail(VMC_E_CONFIG, why);
        e->theta = th;
    }
    if (e->mlp_e >= 0 && method != "fromfile") {
        // MLP Jastrow: Xavier-uniform hidden layers, zero biases and output layers, so
        // the factor starts as its cusp term alone (host Philox, stream tag 3)
        double *t = e->theta.data() + (size_t)e->mlp_e * e->Pmax;
        std::fill(t, t + e->Pmax, 0.0);
        auto u3 = [&](uint32_t i) {
            const uint4 v = host_philox(make_uint4(i, 0u, 0u, 3u), make_uint2((uint32_t)s, (uint32_t)(s >> 32)));
            return v.x * 2.3283064365386963e-10;
        };
        auto fill = [&](int off, int n, int fan_in, int fan_out) {
            const double lim = std::sqrt(6.0 / (fan_in + fan_out));
            for (int i = 0; i < n; ++i) t[off + i] = -lim + 2 * lim * u3((uint32_t)(off + i));
        };
        fill(MW_W1, MLP_H * 2, 2, MLP_H);
        fill(MW_W2, MLP_H * MLP_H, MLP_H, MLP_H);
        fill(MW_V1, MLP_G, 1, MLP_G);
        fill(MW_V2, MLP_G * MLP_G, MLP_G, MLP_G);
    }
    return VMC_OK;
}

int upload_theta(vmc_engine *e)
{
    if (!e->general && e->mlp_e < 0) return VMC_OK;  // the quantum-dot kernels take their scalars by value
    if (e->general)
        CUDA_TRY(cudaMemcpyAsync(e->d_theta, e->theta.data(), e->theta.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, e->stream));
    if (e->mlp_e >= 0) {
        // the networks run with their weights rounded to bfloat16 (nearest even); the
        // device block also holds W2 and V2 transposed (MW_W2T, MW_V2T)
        std::vector<float> w(MLP_SMEM_FLOATS, 0.0f);
        for (int i = 0; i < MLP_PARAMS; ++i) {
            const float f = (float)e->theta[(size_t)e->mlp_e * e->Pmax + i];
            uint32_t b;
            std::memcpy(&b, &f, 4);
            b = ((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16) << 16;
            std::memcpy(&w[i], &b, 4);
        }
        for (int k = 0; k < MLP_H; ++k)
            for (int m = 0; m < MLP_H; ++m) w[MW_W2T + k * MLP_H + m] = w[MW_W2 + m * MLP_H + k];
        for (int k = 0; k < MLP_G; ++k)
            for (int m = 0; m < MLP_G; ++m) w[MW_V2T + k * MLP_G + m] = w[MW_V2 + m * MLP_G + k];
        CUDA_TRY(cudaMemcpyAsync(e->d_mlpw, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));  // w is a local buffer
    }
    return VMC_OK;
}

int refresh_all(vmc_engine *e)
{
    if (!e->have_walkers) return VMC_OK;
    return run_rebuild(e, RB_REFRESH, nullptr);
}

}  // namespace

// ======================================================================= C ABI

extern "C" {

int vmc_abi_version(void) { return VMC_ABI_VERSION; }

const char *vmc_last_error(void) { return g_last_error.c_str(); }

int vmc_create(const char *text, const vmc_options *opt, vmc_engine **out)
{
    if (!text || !out) return fail(VMC_E_ARG, "null argument");
    *out = nullptr;
    vmc_engine *e = new vmc_engine();
    std::string msg = parse_config(text, e->cfg);
    if (!msg.empty()) {
        delete e;
        return fail(VMC_E_CONFIG, msg);
    }
    Config &c = e->cfg;
    if (opt) {
        e->device = opt->device;
        if (opt->precision >= 0) c.precision = opt->precision;
        if (opt->num_walkers > 0) c.walkers = opt->num_walkers;
        if (opt->walkers_per_block > 0) c.walkers_per_block = opt->walkers_per_block;
        if (opt->refresh_interval >= 0) c.refresh_interval = opt->refresh_interval;
        if (opt->compat >= 0) c.compat = opt->compat;
    }
    auto reject = [&](const std::string &m) {
        delete e;
        return fail(VMC_E_UNSUPPORTED, m);
    };
    if (c.hamiltonian.empty()) return reject("no hamiltonian given (the reference requires one)");
    if (c.hamiltonian != "harmonicOscillator" && c.hamiltonian != "atomicNucleus")
        return reject("hamiltonian '" + c.hamiltonian + "' is not on the engine's path");
    if (c.dim != 2 && c.dim != 3) return reject("numDimensions must be 2 or 3");
    if (c.elements.empty()) return reject("no wave function elements");
    if ((int)c.elements.size() > MAX_ELEM) return reject("too many elements");
    if (c.N < 2 || c.N > MAX_N) return reject("numParticles must be in [2, 64]");
    int flags = 0;
    int K = 0;
    // SimpleJastrow, the RBM elements and hydrogen orbitals run on the general path
    bool general = false;
    for (int el : c.elements)
        general |= el == E_SIMPLEJASTROW || el == E_RBMGAUSSIAN || el == E_RBMPRODUCT || el == E_MLP ||
                   (el == E_SLATER && c.basis == "hydrogenOrbital");
    // the learned MLP Jastrow on the FP32 dot sweep: mixed precision, 2D closed-shell
    // Slater(Hermite) x Gaussian x MLP, Coulomb, importance sampling, corrected mode,
    // N <= 30 (one partner per lane); the general FP64 path takes the rest
    bool mlp_dot = false;
    if (c.precision == VMC_PRECISION_MIXED && c.mlp_tc && c.dim == 2 && c.basis == "hermite" && c.coulomb && !c.compat &&
        c.sampling != "bruteForce" && c.elements.size() == 3 && c.hamiltonian == "harmonicOscillator") {
        const auto has = [&](int el) { return std::count(c.elements.begin(), c.elements.end(), el) == 1; };
        const int k = closed_shells_2d(c.N, 2);
        if (has(E_SLATER) && has(E_GAUSSIAN) && has(E_MLP) && k >= 1 && k <= 5) {
            mlp_dot = true;
            general = false;
        }
    }
    for (int el : c.elements) {
        switch (el) {
        case E_GAUSSIAN: flags |= F_GAUSS; break;
        case E_PADE: flags |= F_PADE; break;
        case E_HYDROGENLIKE: flags |= F_HYDROGENLIKE; break;
        case E_SIMPLEJASTROW: flags |= F_SIMPLEJ; break;
        case E_RBMGAUSSIAN: flags |= F_RBMG; break;
        case E_RBMPRODUCT: flags |= F_RBMP; break;
        case E_MLP: flags |= F_MLP; break;
        case E_SLATER:
            if (c.basis != "hermite" && c.basis != "hydrogenOrbital")
                return reject("Slater determinant needs basis: hermite or hydrogenOrbital");
            if (!general) {
                K = closed_shells_2d(c.N, c.dim);
                if (K < 0) return reject("open shell: numParticles is not a closed shell");
                if ((c.dim == 2 && K > 7) || (c.dim == 3 && K > 4)) return reject("too many shells");
            }
            flags |= F_SLATER;
            break;
        default: return reject("wave function element not implemented on the engine");
        }
    }
    for (int el : {E_PADE, E_GAUSSIAN, E_SLATER, E_SIMPLEJASTROW, E_RBMGAUSSIAN, E_RBMPRODUCT, E_MLP})
        if (std::count(c.elements.begin(), c.elements.end(), (int)el) > 1) return reject("repeated element");
    if (c.coulomb) flags |= F_COULOMB;
    if (c.hamiltonian == "atomicNucleus") flags |= F_ATOM;
    if (c.compat) flags |= Q_PADE_RATIO | Q_PADE_DGAMMA | Q_IS_GREEN | Q_PADE_STALE;
    // the drift limiter changes the proposal and needs the Fokker-Planck Green's ratio:
    // importance sampling in the corrected mode only
    if (c.drift_limit > 0.0 && (c.compat || c.sampling == "bruteForce"))
        return reject("driftLimit needs importanceSampling with compat: corrected");
    // quirk bits of the general-path elements only where those elements are present,
    // so a quantum dot keeps its compiled-in flag set
    if (c.compat && (flags & F_SIMPLEJ)) flags |= Q_SJ_RATIO;
    if (c.compat && c.sorting && (flags & F_RBMP)) flags |= Q_RBM_SORT;
    if (c.sampling != "bruteForce") flags |= F_IS;
    e->general = general;
    e->flags = flags;
    e->K = K;
    e->compat = c.compat;
    e->sampling = c.sampling == "bruteForce" ? SAMPLER_BF : SAMPLER_IS;
    e->precision = c.precision;
    e->W = c.walkers;
    if (e->W < 1) return reject("numWalkers must be >= 1");
    e->N = c.N;
    e->dim = c.dim;
    e->D = c.N * c.dim;
    e->n_orb = K > 0 ? c.N / 2 : 0;
    e->E = (int)c.elements.size();
    e->Pmax = 0;
    for (int el : c.elements) e->Pmax = std::max(e->Pmax, element_parameters(c, el));
    e->EP = e->E * e->Pmax;
    e->nacc = 9 + 2 * e->EP;
    if (!general && !mlp_dot && e->nacc > 32) return reject("more than 11 parameters per walker is not supported");
    e->nacc_dev = e->nacc;
    if (mlp_dot) {  // per walker: the Gaussian's alpha; the network's gradient comes from snapshots
        for (int i = 0; i < e->E; ++i) {
            if (c.elements[i] == E_MLP) e->mlp_e = i;
            if (c.elements[i] == E_GAUSSIAN) e->act.push_back(i * e->Pmax);
        }
        e->nacc_dev = 9 + 2 * (int)e->act.size();
        e->gen.mlp_tc = c.mlp_tc ? 1 : 0;
    }
    if (general) {
        const std::string why = gen_configure(c, e->E, e->Pmax, e->gen);
        if (!why.empty()) return reject(why);
        // mixed precision on the general path: the compiled atom form (3D hydrogen-orbital
        // Slater determinants with SimpleJastrow / Pade), FP32 sweeps between FP64
        // re-inversions
        if (e->precision == VMC_PRECISION_MIXED) {
            if (e->gen.variant != GV_ATOM)
                return reject("mixed precision covers the dots, hydrogen-like systems and the atoms' "
                              "hydrogen-orbital Slater x SimpleJastrow / Pade form; this system runs with "
                              "precision: fp64");
            e->gen.f32 = 1;
        }
        e->n_orb = e->gen.n;
        e->nacc_dev = 0;  // set below from the active parameters
        for (int i = 0; i < e->E; ++i)
            if (c.elements[i] == E_MLP) e->mlp_e = i;
        // every parameter but the MLP row's, less SimpleJastrow's beta_ij with i >= j,
        // whose gradient is identically zero (the reference's distance matrix holds only
        // i < j, simplejastrow.cpp:106-111): their sums stay exact zeros on the host
        for (int i = 0; i < e->E; ++i)
            if (i != e->mlp_e)
                for (int q = 0; q < element_parameters(c, c.elements[i]); ++q) {
                    if (c.elements[i] == E_SIMPLEJASTROW && q % c.N >= q / c.N) continue;
                    e->act.push_back(i * e->Pmax + q);
                }
        e->nacc_dev = 9 + 2 * (int)e->act.size();
    }
    // userinput.cpp:60-81 with walkers in place of ranks: numSteps is the total
    // over walkers; each walker burns in its own share times the fraction.
    e->steps_per_walker = (int)(c.num_steps / e->W);
    if (e->steps_per_walker < 1) return reject("numSteps smaller than numWalkers");
    e->burn_in = (int)(e->steps_per_walker * c.eq_fraction);
    e->batches = c.optimization == "adam" ? 10 : 1;  // adam.h:15, gradientdescent.h:13
    // the general path keeps its record in FP64 (its FP32 sweep stages it in FP32)
    e->elem_bytes = e->precision == VMC_PRECISION_MIXED && !general ? 4 : 8;
    e->L = make_layout(e->N, e->dim, e->n_orb, (int)e->elem_bytes);
    if (general) {  // positions first in the general record (vmc_general.hpp)
        e->L.off_x = 0;
        e->L.rec = e->gen.rec;
        if (!select_set(VMC_PRECISION_FP64, e->dim, 0, 0, e->ks)) return reject("no kernel for this shape");
    } else if (!select_set(e->precision, e->dim, K, e->flags, e->ks)) {
        return reject("no kernel for this shape");
    }
    // walkers per warp of the compiled-in dots: the kernel set's default, or at most
    // the configured count; the accumulators (one lane each, two with 8-lane segments)
    // must fit 16 slots
    if (e->ks.sweep_plain2) {
        const void *four = e->ks.seg == 4 ? e->ks.sweep_plain : nullptr;
        int want = c.walkers_per_warp > 0 ? c.walkers_per_warp : e->ks.seg;
        if (e->nacc_dev > 16) want = 1;
        if (want >= 4 && four) {
            e->ks.sweep_plain = four;
            e->ks.seg = 4;
        } else if (want >= 2) {
            e->ks.sweep_plain = e->ks.sweep_plain2;
            e->ks.seg = 2;
        } else {
            e->ks.sweep_plain = e->ks.sweep_plain1;
            e->ks.seg = 1;
        }
    }
    // the owner form of the production dot sweep: by default where one walker per warp
    // remains (N = 42 and 56), on request for N = 20 and 30
    if (c.sweep_form == 2 && !e->ks.sweep_owner) return reject("sweepForm: owner covers the 2D dots of N = 20 to 56");
    e->owner = e->ks.sweep_owner && (c.sweep_form == 2 || (c.sweep_form == 0 && e->ks.seg == 1));
    if (e->owner) e->ks.seg = 1;
    // auto: start at 4 D steps (at least 512) and let the drift test tune it
    e->refresh_interval = c.refresh_interval >= 0 ? c.refresh_interval
                          : (e->precision == VMC_PRECISION_MIXED ? std::max(4 * e->D, 512) : 0);
    // the general path's refresh measures no drift: its cadence stays as configured
    e->refresh_auto = c.refresh_interval < 0 && e->precision == VMC_PRECISION_MIXED && !general;
    e->seed = c.have_seed ? (unsigned long long)c.seed : 0x5eedULL;

    int rc;
    if ((rc = [&]() -> int {
            CUDA_TRY(cudaSetDevice(e->device));
            CUDA_TRY(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device));
            int hrc = hermite_init_device(e->device);
            if (hrc) return hrc;
            CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreate(&e->ev0));
            CUDA_TRY(cudaEventCreate(&e->ev1));
            const size_t W = e->W;
            CUDA_TRY(cudaMalloc(&e->d_state, W * e->L.rec * e->elem_bytes));
            CUDA_TRY(cudaMalloc(&e->d_scal, W * NSCAL * sizeof(double)));
            CUDA_TRY(cudaMalloc(&e->d_acc, W * e->nacc_dev * 2 * sizeof(double)));
            CUDA_TRY(cudaMalloc(&e->d_out, std::max(64, e->nacc_dev) * sizeof(double)));
            CUDA_TRY(cudaMalloc(&e->d_drift, W * sizeof(double)));
            CUDA_TRY(cudaMalloc(&e->d_wmean, W * sizeof(double)));
            CUDA_TRY(cudaMalloc(&e->d_mask, W * e->N * sizeof(unsigned long long)));
            CUDA_TRY(cudaMalloc(&e->d_counter, W * sizeof(unsigned long long)));
            CUDA_TRY(cudaMalloc(&e->d_status, W * sizeof(unsigned)));
            CUDA_TRY(cudaMalloc(&e->d_pos, W * e->D * sizeof(double)));
            if (e->general) {
                CUDA_TRY(cudaMalloc(&e->d_theta, std::max<size_t>(1, (size_t)e->EP) * sizeof(double)));
                e->gen.theta = e->d_theta;
                CUDA_TRY(cudaMalloc(&e->d_act, std::max<size_t>(1, e->act.size()) * sizeof(int)));
                if (!e->act.empty())
                    CUDA_TRY(cudaMemcpy(e->d_act, e->act.data(), e->act.size() * sizeof(int), cudaMemcpyHostToDevice));
                e->gen.act = e->d_act;
                e->gen.n_act = (int)e->act.size();
            }
            if (mlp_dot) {
                const size_t stride = (size_t)e->N * e->N * 3 + e->N * 3;
                CUDA_TRY(cudaMalloc(&e->d_mlp_cache, W * stride * sizeof(float)));
                CUDA_TRY(cudaMemsetAsync(e->d_mlp_cache, 0, W * stride * sizeof(float), e->stream));
            }
            if (e->mlp_e >= 0) {
                CUDA_TRY(cudaMalloc(&e->d_mlpw, MLP_SMEM_FLOATS * sizeof(float)));
                CUDA_TRY(cudaMalloc(&e->d_mlp_out, 2 * MLP_PARAMS * sizeof(double)));
                e->gen.mlp = e->d_mlpw;
            }
            CUDA_TRY(cudaMemsetAsync(e->d_state, 0, W * e->L.rec * e->elem_bytes, e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_scal, 0, W * NSCAL * sizeof(double), e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_acc, 0, W * e->nacc_dev * 2 * sizeof(double), e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_drift, 0, W * sizeof(double), e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_mask, 0xff, W * e->N * sizeof(unsigned long long), e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_counter, 0, W * sizeof(unsigned long long), e->stream));
            CUDA_TRY(cudaMemsetAsync(e->d_status, 0, W * sizeof(unsigned), e->stream));
            return choose_wpb(e);
        }())) {
        free_engine(e);
        return rc;
    }
    if ((rc = initial_weights(e)) || (rc = upload_theta(e))) {
        free_engine(e);
        return rc;
    }
    const size_t P = e->theta.size();
    // adam.cpp:35-36 and gradientdescent.cpp/sgd.cpp start their moments at ones;
    // compat: corrected starts ADAM from zero
    const double m0 = (e->compat || c.optimization != "adam") ? 1.0 : 0.0;
    e->opt_m.assign(P, m0);
    e->opt_v.assign(P, m0);
    e->gamma_prev = make_params(e).gamma;
    *out = e;
    return VMC_OK;
}

void vmc_destroy(vmc_engine *e) { free_engine(e); }

int vmc_get_info(const vmc_engine *e, vmc_info *o)
{
    if (!e || !o) return fail(VMC_E_ARG, "null argument");
    std::memset(o, 0, sizeof(*o));
    o->n_particles = e->N;
    o->n_dimensions = e->dim;
    o->n_coords = e->D;
    o->n_elements = e->E;
    o->p_max = e->Pmax;
    o->n_walkers = e->W;
    o->precision = e->precision;
    o->sampling = e->sampling;
    o->steps_per_walker = e->steps_per_walker;
    o->burn_in = e->burn_in;
    o->batches = e->batches;
    o->n_iterations = e->cfg.iterations;
    o->compat = e->compat;
    o->n_accumulators = e->nacc_dev;
    o->walkers_per_block = e->wpb;
    o->refresh_interval = e->refresh_interval;
    for (int i = 0; i < e->E && i < 8; ++i) o->element_kind[i] = e->cfg.elements[i];
    o->kernel_variant = e->general ? VMC_KERNEL_GENERAL
                        : (e->flags == FX_DOT_COMPAT || e->flags == FX_DOT_CORRECTED || e->flags == FX_MLP_DOT) && e->K > 0
                            ? VMC_KERNEL_DOT : VMC_KERNEL_RUNTIME_FLAGS;
    o->walkers_per_warp = e->general ? (e->gen.variant == GV_ATOM ? e->gen.seg : 1) : e->ks.seg;
    o->sweep_form = e->owner ? VMC_SWEEP_OWNER : VMC_SWEEP_STAGED;
    if (e->owner) o->walkers_per_block = OWNER_WPB;
    return VMC_OK;
}

int vmc_set_parameters(vmc_engine *e, const double *theta, int n_elements, int p_max)
{
    if (!e || !theta) return fail(VMC_E_ARG, "null argument");
    if (n_elements != e->E || p_max != e->Pmax) return fail(VMC_E_ARG, "parameter shape mismatch");
    return set_parameters(e, theta, true);
}

int vmc_get_parameters(const vmc_engine *e, double *theta, int n_elements, int p_max)
{
    if (!e || !theta) return fail(VMC_E_ARG, "null argument");
    if (n_elements != e->E || p_max != e->Pmax) return fail(VMC_E_ARG, "parameter shape mismatch");
    std::copy(e->theta.begin(), e->theta.end(), theta);
    return VMC_OK;
}

int vmc_init_walkers(vmc_engine *e, const double *pos, uint64_t seed)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    e->seed = seed;
    const size_t W = e->W;
    if (pos) {
        // positions only over the host link; the records are cleared and filled on the device
        const size_t n = W * e->D;
        CUDA_TRY(cudaMemsetAsync(e->d_state, 0, W * e->L.rec * e->elem_bytes, e->stream));
        CUDA_TRY(cudaMemcpyAsync(e->d_pos, pos, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        Layout L = e->L;
        int Wi = e->W;
        const double *dp = e->d_pos;
        void *st = e->d_state;
        void *args[] = {&L, &Wi, &dp, &st};
        CUDA_TRY(cudaLaunchKernel(e->ks.scatter, dim3((unsigned)((n + 255) / 256)), dim3(256), args, 0, e->stream));
    } else {
        const bool normal = e->cfg.initial_state == "randomNormal";
        const double sd = 1.0 / e->cfg.omega;  // randomnormal.cpp:19
        const int n = e->W * e->D;
        Layout L = e->L;
        int Wi = e->W;
        void *st = e->d_state;
        unsigned long long sd_seed = seed;
        int nrm = normal ? 1 : 0;
        double sdv = sd;
        int off = e->cfg.walker_offset;
        void *args[] = {&L, &Wi, &st, &sd_seed, &nrm, &sdv, &off};
        CUDA_TRY(cudaLaunchKernel(e->ks.initpos, dim3((n + 255) / 256), dim3(256), args, 0, e->stream));
    }
    CUDA_TRY(cudaMemsetAsync(e->d_counter, 0, W * sizeof(unsigned long long), e->stream));
    CUDA_TRY(cudaMemsetAsync(e->d_status, 0, W * sizeof(unsigned), e->stream));
    CUDA_TRY(cudaMemsetAsync(e->d_mask, 0xff, W * e->N * sizeof(unsigned long long), e->stream));
    e->gamma_prev = make_params(e).gamma;
    int rc = run_rebuild(e, RB_INIT, nullptr);
    if (rc) return rc;
    std::vector<unsigned> st(W);
    CUDA_TRY(cudaMemcpyAsync(st.data(), e->d_status, W * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (unsigned s : st)
        if (s & ST_SINGULAR) return fail(VMC_E_SINGULAR, "singular Slater block at initialisation");
    e->have_walkers = true;
    return VMC_OK;
}

int vmc_get_positions(const vmc_engine *e, double *pos)
{
    if (!e || !pos) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    // gathered on the device: only the positions cross the host link
    const size_t n = (size_t)e->W * e->D;
    Layout L = e->L;
    int Wi = e->W;
    const void *st = e->d_state;
    double *dp = e->d_pos;
    void *args[] = {&L, &Wi, &st, &dp};
    CUDA_TRY(cudaLaunchKernel(e->ks.gather, dim3((unsigned)((n + 255) / 256)), dim3(256), args, 0, e->stream));
    CUDA_TRY(cudaMemcpyAsync(pos, e->d_pos, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return VMC_OK;
}

int vmc_sample(vmc_engine *e, int iteration, int steps, int burn_in, vmc_sums *out,
               double *grad_sum, double *egrad_sum)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) return fail(VMC_E_STATE, "vmc_init_walkers first");
    if (steps < 1 || burn_in < 0 || burn_in >= steps) return fail(VMC_E_ARG, "bad step counts");
    CUDA_TRY(cudaSetDevice(e->device));
    const size_t W = e->W;
    CUDA_TRY(cudaMemsetAsync(e->d_acc, 0, W * e->nacc_dev * 2 * sizeof(double), e->stream));
    const int bs = (steps - burn_in) / e->batches;
    const int m = iteration % e->batches;
    std::vector<double> drift;
    CUDA_TRY(cudaMemsetAsync(e->d_drift, 0, W * sizeof(double), e->stream));
    CUDA_TRY(cudaEventRecord(e->ev0, e->stream));
    const int chunk = e->refresh_interval > 0 ? e->refresh_interval : e->sweep_chunk;
    const int n_launch = (steps + chunk - 1) / chunk;
    while ((int)e->sweep_events.size() < 2 * n_launch) {
        cudaEvent_t ev;
        CUDA_TRY(cudaEventCreate(&ev));
        e->sweep_events.push_back(ev);
    }
    // MLP Jastrow parameter gradient: snapshots every D steps of the gradient window
    // (steps win_lo < s < win_hi, sampled ones s >= burn_in); slot = (s - win_lo) / D - first
    const int win_lo = bs * m, win_hi = bs * (m + 1);
    int snap_interval = 0, snap_first = 0, n_slots = 0, n_win = 0;
    if (e->mlp_e >= 0) {
        snap_interval = e->D;
        const int lo = std::max(win_lo + 1, burn_in), hi = std::min(win_hi - 1, steps - 1);
        n_win = std::max(0, hi - lo + 1);
        snap_first = std::max(1, (lo - win_lo + snap_interval - 1) / snap_interval);
        const int last = hi >= win_lo ? (hi - win_lo) / snap_interval : 0;
        n_slots = std::max(0, last - snap_first + 1);
        const size_t need = W * (size_t)n_slots;
        if (need > e->snap_cap) {
            cudaFree(e->d_snap_x);
            cudaFree(e->d_snap_e);
            e->d_snap_x = nullptr;
            e->d_snap_e = nullptr;
            e->snap_cap = 0;
            CUDA_TRY(cudaMalloc(&e->d_snap_x, need * e->D * sizeof(float)));
            CUDA_TRY(cudaMalloc(&e->d_snap_e, need * sizeof(double)));
            e->snap_cap = need;
        }
    }
    int n_refresh = 0, li = 0;
    for (int off = 0; off < steps; off += chunk, ++li) {
        SweepArgs a{};
        a.steps = std::min(chunk, steps - off);
        a.step_offset = off;
        a.burn_in = burn_in;
        a.win_lo = win_lo;
        a.win_hi = win_hi;
        a.seed = e->seed;
        if (n_slots > 0) {
            a.snap_x = e->d_snap_x;
            a.snap_e = e->d_snap_e;
            a.snap_stride = n_slots;
            a.snap_interval = snap_interval;
            a.snap_first = snap_first;
        }
        if (e->d_rec) {
            a.rec_en = e->d_rec;
            a.rec_stride = e->rec_stride;
        }
        if (e->dens_bins > 0) {
            a.dens_radial = e->d_dens_radial;
            a.dens_grid = e->d_dens_grid;
            a.dens_pair = e->d_dens_pair;
            a.dens_bins = e->dens_bins;
            a.dens_step = e->dens_step;
            a.dens_max = e->dens_max;
        }
        if (e->d_replay) {
            if (e->replay_pos + steps > e->replay_len) return fail(VMC_E_ARG, "replay stream exhausted");
            a.replay = e->d_replay;
            a.replay_stride = e->replay_len;
            a.replay_offset = e->replay_pos;
        }
        CUDA_TRY(cudaEventRecord(e->sweep_events[2 * li], e->stream));
        int rc = run_sweep(e, a);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(e->sweep_events[2 * li + 1], e->stream));
        if (e->refresh_interval > 0) {
            rc = run_rebuild(e, RB_REFRESH, e->d_drift);
            if (rc) return rc;
            ++n_refresh;
        }
    }
    if (n_slots > 0) {
        CUDA_TRY(cudaMemsetAsync(e->d_mlp_out, 0, 2 * MLP_PARAMS * sizeof(double), e->stream));
        CUDA_TRY(mlp_launch_grad(e->gen, e->N, e->dim, e->d_snap_x, e->d_snap_e, (long long)W * n_slots,
                                 e->d_mlp_out, e->stream, e->d_status));
    }
    CUDA_TRY(cudaEventRecord(e->ev1, e->stream));
    if (e->d_replay) e->replay_pos += steps;
    reduce_acc_kernel<<<e->nacc_dev, 256, 0, e->stream>>>(e->d_acc, e->W, e->nacc_dev, e->d_out);
    CUDA_TRY(cudaGetLastError());
    std::vector<double> dev_sums(e->nacc_dev);
    CUDA_TRY(cudaMemcpyAsync(dev_sums.data(), e->d_out, e->nacc_dev * sizeof(double), cudaMemcpyDeviceToHost,
                             e->stream));
    std::vector<double> mlp_sums(n_slots > 0 ? 2 * MLP_PARAMS : 0);
    if (n_slots > 0)
        CUDA_TRY(cudaMemcpyAsync(mlp_sums.data(), e->d_mlp_out, mlp_sums.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, e->stream));
    std::vector<unsigned> st(W);
    CUDA_TRY(cudaMemcpyAsync(st.data(), e->d_status, W * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    if (n_refresh) {
        drift.resize(W);
        CUDA_TRY(cudaMemcpyAsync(drift.data(), e->d_drift, W * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    double sweep_ms = 0.0;
    for (int i = 0; i < n_launch; ++i) {
        float t = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&t, e->sweep_events[2 * i], e->sweep_events[2 * i + 1]));
        sweep_ms += t;
    }
    unsigned status = 0;
    for (unsigned v : st) status |= v;
    const SamplePass pass{steps, burn_in, bs, n_launch, n_refresh, dev_sums.data(), status,
                          n_refresh ? &drift : nullptr, (double)ms, sweep_ms, -1.0};
    vmc_sums s{};
    std::vector<double> sums;
    const int frc = finish_sample(e, pass, &s, sums);
    if (frc) return frc;
    if (out) *out = s;
    if (n_slots > 0) {
        // the MLP row: snapshot sums scaled to the window's sample count (one snapshot
        // stands for n_win / n_slots sampled steps of its walker)
        const double scale = (double)n_win / n_slots;
        const size_t o = 9 + (size_t)e->mlp_e * e->Pmax;
        for (int i = 0; i < MLP_PARAMS; ++i) {
            sums[o + i] = scale * mlp_sums[i];
            sums[o + e->EP + i] = scale * mlp_sums[MLP_PARAMS + i];
        }
    }
    if (grad_sum) std::copy(sums.begin() + 9, sums.begin() + 9 + e->EP, grad_sum);
    if (egrad_sum) std::copy(sums.begin() + 9 + e->EP, sums.begin() + 9 + 2 * e->EP, egrad_sum);
    return VMC_OK;
}

int vmc_get_walker_energies(const vmc_engine *e, double *mean_energy)
{
    if (!e || !mean_energy) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    const double n = std::max(1.0, e->last_samples_per_walker);
    walker_means_kernel<<<(e->W + 255) / 256, 256, 0, e->stream>>>(e->d_acc, e->W, e->nacc_dev, 1.0 / n,
                                                                   e->d_wmean);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(mean_energy, e->d_wmean, (size_t)e->W * sizeof(double), cudaMemcpyDeviceToHost,
                             e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return VMC_OK;
}

int vmc_apply_sums(vmc_engine *e, const vmc_sums *total, const double *grad_sum,
                   const double *egrad_sum, vmc_averages *out)
{
    return apply_sums(e, total, grad_sum, egrad_sum, out, true);
}

int vmc_run_iteration(vmc_engine *e, int iteration, vmc_averages *out)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    const int steps = e->steps_per_walker + e->burn_in;
    std::vector<double> g(e->EP), ge(e->EP);
    vmc_sums s{};
    const int rc = vmc_sample(e, iteration, steps, e->burn_in, &s, g.data(), ge.data());
    if (rc) return rc;
    return vmc_apply_sums(e, &s, g.data(), ge.data(), out);
}

int vmc_run_simulation(vmc_engine *e, vmc_averages *history, int n_history)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) {
        int rc = vmc_init_walkers(e, nullptr, e->seed);
        if (rc) return rc;
    }
    // System::runSimulation (system.cpp:81-139): the last iteration is number
    // normal + rangeOfAdaptiveSteps; with adaptive steps the iterations from `normal`
    // on sample 2^additionalSteps times the steps and the last 2^additionalStepsLastIter
    // times (system.cpp:214-224); the convergence check moves `normal` to the next
    // iteration once the energy of numberOfEnergies iterations ago is within
    // `tolerance` of the latest (system.cpp:197-207).  The reference's loop has no exit
    // at the last iteration (system.cpp:93): after it the remaining iterations up to
    // numIterations run with 2^additionalSteps times the steps; compat: corrected ends
    // the run there.  The convergence window starts at zeros, as setConvergenceTools
    // sizes it (userinput.cpp:194-200).
    const Config &c = e->cfg;
    int normal = c.iterations - c.range_adaptive - 1;
    bool check = c.check_convergence;
    std::vector<double> window(std::max(1, c.n_energies), 0.0);
    std::ofstream ef[4];
    if (c.print_energy) {  // sampler.cpp:443-452, 491-498
        const char *names[4] = {"energy.dat", "kinetic.dat", "external.dat", "interaction.dat"};
        for (int q = 0; q < 4; ++q) {
            ef[q].open(c.path + names[q]);
            if (!ef[q]) return fail(VMC_E_ARG, "cannot write '" + c.path + names[q] + "'");
        }
    }
    e->have_final = false;
    const bool dens = c.ob_density || (c.ob_density2 && e->dim >= 2) || c.tb_density;
    int it = 0;
    for (; it < c.iterations; ++it) {
        const bool last = it == normal + c.range_adaptive;
        long long mult = 1;
        if (c.adaptive_steps) mult = last ? (1LL << c.add_steps_last) : it >= normal ? (1LL << c.add_steps) : 1;
        const long long sampled = (long long)e->steps_per_walker * mult;
        if (sampled + e->burn_in > (1LL << 30)) return fail(VMC_E_ARG, "adaptive steps: too many steps per walker");
        const int steps = (int)sampled + e->burn_in;
        // the last iteration keeps every walker's energies for blocking (doResampling)
        // when they fit in FINAL_RECORD_BYTES of device memory, and counts densities
        double *rec = nullptr;
        if (last && c.do_resampling && (double)e->W * steps * 24.0 <= FINAL_RECORD_BYTES) {
            CUDA_TRY(cudaMalloc(&rec, (size_t)e->W * steps * 3 * sizeof(double)));
            e->d_rec = rec;
            e->rec_stride = steps;
        }
        int rc = (last && dens) ? density_begin(e, c.n_bins, c.max_radius, c.ob_density,
                                                c.ob_density2 && e->dim >= 2, c.tb_density)
                                : VMC_OK;
        std::vector<double> g(e->EP), ge(e->EP);
        vmc_sums s{};
        vmc_averages a{};
        if (!rc) rc = vmc_sample(e, it, steps, e->burn_in, &s, g.data(), ge.data());
        e->d_rec = nullptr;
        e->rec_stride = 0;
        if (!rc) rc = apply_sums(e, &s, g.data(), ge.data(), &a, true);
        if (history && it < n_history) history[it] = a;
        if (!rc && last && rec) {
            rc = block_record(e, rec, steps, e->burn_in, &e->final_blocking);
            e->have_final = rc == VMC_OK;
            // the instant energies the reference blocks (sampler.cpp:624-632, appended over
            // ranks by appendInstantFiles, sampler.cpp:407-425): the walkers' sampled E_L,
            // walker after walker, one per line, into <path>0_0.dat (its instant number
            // is 0 here), when at most INSTANT_FILE_LINES
            const double lines = (double)e->W * (steps - e->burn_in);
            if (!rc && lines <= INSTANT_FILE_LINES) {
                std::vector<double> h((size_t)e->W * steps * 3);
                CUDA_TRY(cudaMemcpyAsync(h.data(), rec, h.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
                CUDA_TRY(cudaStreamSynchronize(e->stream));
                std::ofstream f(c.path + "0_0.dat");
                if (!f) rc = fail(VMC_E_ARG, "cannot write '" + c.path + "0_0.dat'");
                for (int w = 0; w < e->W && !rc; ++w)
                    for (int t = e->burn_in; t < steps; ++t) {
                        const double *q = h.data() + ((size_t)w * steps + t) * 3;
                        f << (q[0] + q[1]) + q[2] << '\n';
                    }
            }
        }
        if (rec) {
            cudaStreamSynchronize(e->stream);
            cudaFree(rec);
        }
        if (last && dens) {
            const size_t b = (size_t)c.n_bins;
            std::vector<uint64_t> r1(c.ob_density ? b : 0), r2(c.ob_density2 && e->dim >= 2 ? b * b : 0),
                r3(c.tb_density ? b * b : 0);
            const int drc = density_end(e, r1.empty() ? nullptr : r1.data(), r2.empty() ? nullptr : r2.data(),
                                        r3.empty() ? nullptr : r3.data());
            if (!rc) rc = drc;
            // sampler.cpp:522-581: onebody.dat (a column), onebody2.dat, twobody.dat
            if (!rc && !r1.empty()) rc = write_counts(c.path + "onebody.dat", r1.data(), c.n_bins, 1);
            if (!rc && !r2.empty()) rc = write_counts(c.path + "onebody2.dat", r2.data(), c.n_bins, c.n_bins);
            if (!rc && !r3.empty()) rc = write_counts(c.path + "twobody.dat", r3.data(), c.n_bins, c.n_bins);
        }
        if (rc) return rc;
        // checkpointing (system.cpp:116-118, sampler.cpp:507-515)
        if (c.print_params && c.checkpoint_freq > 0 && it % c.checkpoint_freq == 0)
            if ((rc = write_weights_file(e, c.path + "weights_" + std::to_string(it) + ".dat", 6))) return rc;
        if (c.print_energy) {
            ef[0] << a.energy << std::endl;
            ef[1] << a.kinetic << std::endl;
            ef[2] << a.external << std::endl;
            ef[3] << a.interaction << std::endl;
        }
        if (last && !e->compat) {
            ++it;
            break;
        }
        if (check) {
            std::rotate(window.begin(), window.begin() + 1, window.end());
            window.back() = a.energy;
            if (std::fabs(window.front() - window.back()) < c.tolerance) {
                normal = it + 1;
                check = false;
            }
        }
    }
    return it;
}

int vmc_last_blocking(const vmc_engine *e, vmc_blocking_result *out)
{
    if (!e || !out) return fail(VMC_E_ARG, "null argument");
    if (!e->have_final) return fail(VMC_E_STATE, "no blocked final iteration (doResampling: true in vmc_run_simulation)");
    *out = e->final_blocking;
    return VMC_OK;
}

int vmc_eval(vmc_engine *e, double *grad, double *lap, double *pgrad, double *energies)
{
    if (!e || !grad || !lap || !pgrad || !energies) return fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) return fail(VMC_E_STATE, "vmc_init_walkers first");
    CUDA_TRY(cudaSetDevice(e->device));
    const size_t W = e->W;
    double *d = nullptr;
    const size_t ng = W * e->E * e->D, nl = W * e->E, np = W * e->E * e->Pmax, ne = W * 3;
    CUDA_TRY(cudaMalloc(&d, (ng + nl + np + ne) * sizeof(double)));
    EvalArgs a{};
    a.P = make_params(e);
    a.p_max = e->Pmax;
    a.grad = d;
    a.lap = d + ng;
    a.pgrad = d + ng + nl;
    a.energies = d + ng + nl + np;
    int rc = VMC_OK;
    if (e->flags == FX_MLP_DOT) {
        cudaFree(d);
        return fail(VMC_E_UNSUPPORTED, "vmc_eval: the MLP Jastrow dot in mixed precision samples only; "
                                       "evaluate with precision: fp64");
    }
    if (e->general) {
        const cudaError_t ge = gen_launch_state(a.P, e->gen, GEN_STATE, a.grad, a.lap, a.pgrad, a.energies, e->stream);
        if (ge != cudaSuccess) rc = fail(VMC_E_CUDA, cudaGetErrorString(ge));
    } else {
        rc = launch(e->ks.eval, (e->W + 3) / 4, 128, 0, e->stream, &a);
    }
    if (rc) { cudaFree(d); return rc; }
    std::vector<double> h(ng + nl + np + ne);
    cudaError_t ce = cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    cudaFree(d);
    if (ce != cudaSuccess) return fail(VMC_E_CUDA, cudaGetErrorString(ce));
    std::copy(h.begin(), h.begin() + ng, grad);
    std::copy(h.begin() + ng, h.begin() + ng + nl, lap);
    std::copy(h.begin() + ng + nl, h.begin() + ng + nl + np, pgrad);
    std::copy(h.begin() + ng + nl + np, h.end(), energies);
    if (e->mlp_e >= 0) {
        // MLP row: the production backward kernel, one walker's positions at a time
        std::vector<double> pos(W * e->D);
        int prc = vmc_get_positions(e, pos.data());
        if (prc) return prc;
        std::vector<float> xf(pos.begin(), pos.end());
        float *dx = nullptr;
        double *dout = nullptr;
        CUDA_TRY(cudaMalloc(&dx, xf.size() * sizeof(float)));
        CUDA_TRY(cudaMalloc(&dout, W * 2 * MLP_PARAMS * sizeof(double)));
        cudaError_t ge = cudaMemcpyAsync(dx, xf.data(), xf.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream);
        if (ge == cudaSuccess) ge = cudaMemsetAsync(dout, 0, W * 2 * MLP_PARAMS * sizeof(double), e->stream);
        for (size_t w = 0; w < W && ge == cudaSuccess; ++w)
            ge = mlp_launch_grad(e->gen, e->N, e->dim, dx + w * e->D, nullptr, 1, dout + w * 2 * MLP_PARAMS, e->stream,
                                 e->d_status + w);
        std::vector<double> g(W * 2 * MLP_PARAMS);
        if (ge == cudaSuccess)
            ge = cudaMemcpyAsync(g.data(), dout, g.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
        if (ge == cudaSuccess) ge = cudaStreamSynchronize(e->stream);
        cudaFree(dx);
        cudaFree(dout);
        if (ge != cudaSuccess) return fail(VMC_E_CUDA, cudaGetErrorString(ge));
        for (size_t w = 0; w < W; ++w)
            std::copy(g.begin() + w * 2 * MLP_PARAMS, g.begin() + w * 2 * MLP_PARAMS + MLP_PARAMS,
                      pgrad + (w * e->E + e->mlp_e) * e->Pmax);
    }
    return VMC_OK;
}

int vmc_probe_move(vmc_engine *e, const int *k, const double *xnew, double *ratios)
{
    if (!e || !k || !xnew || !ratios) return fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) return fail(VMC_E_STATE, "vmc_init_walkers first");
    CUDA_TRY(cudaSetDevice(e->device));
    const size_t W = e->W;
    for (size_t w = 0; w < W; ++w)
        if (k[w] < 0 || k[w] >= e->D) return fail(VMC_E_ARG, "coordinate out of range");
    int *dk = nullptr;
    double *dx = nullptr, *dr = nullptr;
    CUDA_TRY(cudaMalloc(&dk, W * sizeof(int)));
    CUDA_TRY(cudaMalloc(&dx, W * sizeof(double)));
    CUDA_TRY(cudaMalloc(&dr, W * e->E * sizeof(double)));
    CUDA_TRY(cudaMemcpyAsync(dk, k, W * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(dx, xnew, W * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    SweepArgs a{};
    a.steps = 1;
    a.step_offset = 0;
    a.burn_in = 1 << 30;
    a.win_lo = a.win_hi = 0;
    a.seed = e->seed;
    a.probe_k = dk;
    a.probe_x = dx;
    a.probe_ratio = dr;
    int rc = run_sweep(e, a);
    cudaError_t ce = cudaSuccess;
    if (!rc) {
        ce = cudaMemcpyAsync(ratios, dr, W * e->E * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    }
    cudaFree(dk);
    cudaFree(dx);
    cudaFree(dr);
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(VMC_E_CUDA, cudaGetErrorString(ce));
    return VMC_OK;
}

int vmc_set_replay(vmc_engine *e, const double *stream, int length)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    cudaFree(e->d_replay);
    e->d_replay = nullptr;
    e->replay_len = e->replay_pos = 0;
    if (!stream) return VMC_OK;
    if (length < 1) return fail(VMC_E_ARG, "bad replay length");
    const size_t bytes = (size_t)e->W * length * 3 * sizeof(double);
    CUDA_TRY(cudaMalloc(&e->d_replay, bytes));
    CUDA_TRY(cudaMemcpyAsync(e->d_replay, stream, bytes, cudaMemcpyHostToDevice, e->stream));
    e->replay_len = length;
    return VMC_OK;
}

int vmc_set_refresh_interval(vmc_engine *e, int steps)
{
    if (!e || steps < 1) return fail(VMC_E_ARG, "bad argument");
    if (e->precision != VMC_PRECISION_MIXED) return fail(VMC_E_STATE, "the FP64 engine has no refresh cadence");
    e->refresh_interval = steps;
    return VMC_OK;
}

int vmc_replay(vmc_engine *e, const double *stream, int steps, uint8_t *accepted, double *energies)
{
    if (!e || steps < 1) return fail(VMC_E_ARG, "bad argument");
    if (!e->have_walkers) return fail(VMC_E_STATE, "vmc_init_walkers first");
    CUDA_TRY(cudaSetDevice(e->device));
    const size_t W = e->W;
    double *ds = nullptr, *den = nullptr;
    unsigned char *dacc = nullptr;
    if (stream) {
        CUDA_TRY(cudaMalloc(&ds, W * steps * 3 * sizeof(double)));
        CUDA_TRY(cudaMemcpyAsync(ds, stream, W * steps * 3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    }
    CUDA_TRY(cudaMalloc(&dacc, W * steps));
    CUDA_TRY(cudaMalloc(&den, W * steps * 3 * sizeof(double)));
    SweepArgs a{};
    a.steps = steps;
    a.step_offset = 0;
    a.burn_in = 1 << 30;
    a.seed = e->seed;
    a.replay = ds;  // null: the engine's Philox streams
    a.replay_stride = steps;
    a.rec_acc = dacc;
    a.rec_en = den;
    a.rec_stride = steps;
    int rc = run_sweep(e, a);
    cudaError_t ce = cudaSuccess;
    if (!rc) {
        if (accepted) ce = cudaMemcpyAsync(accepted, dacc, W * steps, cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess && energies)
            ce = cudaMemcpyAsync(energies, den, W * steps * 3 * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    }
    cudaFree(ds);
    cudaFree(dacc);
    cudaFree(den);
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(VMC_E_CUDA, cudaGetErrorString(ce));
    return VMC_OK;
}

int vmc_get_status(const vmc_engine *e, uint32_t *status)
{
    if (!e || !status) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    CUDA_TRY(cudaMemcpyAsync(status, e->d_status, e->W * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return VMC_OK;
}

int vmc_stopwatch(vmc_engine *e, int mode, double *ms)
{
    if (!e) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(e->device));
    if (!e->sw0) {
        CUDA_TRY(cudaEventCreate(&e->sw0));
        CUDA_TRY(cudaEventCreate(&e->sw1));
    }
    if (mode == 0) {
        CUDA_TRY(cudaEventRecord(e->sw0, e->stream));
        return VMC_OK;
    }
    CUDA_TRY(cudaEventRecord(e->sw1, e->stream));
    CUDA_TRY(cudaEventSynchronize(e->sw1));
    float t = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&t, e->sw0, e->sw1));
    if (ms) *ms = t;
    return VMC_OK;
}

int vmc_measure_fma_peak(int device, int precision, double *tflops)
{
    if (!tflops) return fail(VMC_E_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    // about 2 ms per launch, best of the launches after the first; FP32 takes the
    // better of scalar FFMA and packed FFMA2 chains
    const int threads = 256, blocks = sms * 8, iters = precision == VMC_PRECISION_MIXED ? 32768 : 8192;
    float *out = nullptr;
    CUDA_TRY(cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)));
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    double best = 0.0;
    const int variants = precision == VMC_PRECISION_MIXED ? 2 : 1;
    for (int var = 0; var < variants; ++var)
        for (int rep = 0; rep < 4; ++rep) {
            CUDA_TRY(cudaEventRecord(a));
            if (precision != VMC_PRECISION_MIXED)
                fma_peak_kernel<double><<<blocks, threads>>>(reinterpret_cast<double *>(out), iters, 1.0 + 1e-15);
            else if (var == 0)
                fma_peak_kernel<float><<<blocks, threads>>>(reinterpret_cast<float *>(out), iters, 1.0f + 1e-7f);
            else
                fma2_peak_kernel<<<blocks, threads>>>(reinterpret_cast<float *>(out), iters / 2, 1.0f + 1e-7f);
            CUDA_TRY(cudaEventRecord(b));
            CUDA_TRY(cudaEventSynchronize(b));
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
            const double flops = 2.0 * FMA_CHAINS * (double)iters * blocks * threads;
            if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    *tflops = best;
    return VMC_OK;
}

}  // extern "C"

namespace vmc {

HermiteCoef hermite_coefficients()
{
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
    return h;
}

Params engine_params(const vmc_engine *e) { return make_params(e); }
void owner_constants(const vmc_engine *e, SweepArgs &a) { fill_owner_constants(e, a); }
int upload_parameters(vmc_engine *e) { return upload_theta(e); }
int engine_sweep_smem_per_warp(const vmc_engine *e) { return sweep_smem_per_warp(e); }
int engine_rebuild_smem_per_warp(const vmc_engine *e) { return rebuild_smem_per_warp(e->N, e->dim, e->n_orb); }
int engine_refresh(vmc_engine *e, double *drift) { return run_rebuild(e, RB_REFRESH, drift); }

int set_parameters(vmc_engine *e, const double *theta, bool refresh)
{
    const double old_gamma = make_params(e).gamma;
    e->theta.assign(theta, theta + (size_t)e->E * e->Pmax);
    CUDA_TRY(cudaSetDevice(e->device));
    if (e->have_walkers && (e->flags & Q_PADE_STALE)) {
        // Pade pairs keep the gamma they were computed with until one of their
        // particles moves (padejastrow.cpp:65-68 only stores gamma)
        e->gamma_prev = old_gamma;
        CUDA_TRY(cudaMemsetAsync(e->d_mask, 0, (size_t)e->W * e->N * sizeof(unsigned long long), e->stream));
    } else {
        e->gamma_prev = make_params(e).gamma;
    }
    int rc = upload_theta(e);
    return rc ? rc : refresh ? refresh_all(e) : VMC_OK;
}

int apply_sums(vmc_engine *e, const vmc_sums *total, const double *grad_sum, const double *egrad_sum,
               vmc_averages *out, bool refresh)
{
    if (!e || !total || !grad_sum || !egrad_sum) return fail(VMC_E_ARG, "null argument");
    const vmc_sums &s = *total;
    if (!(s.n_samples > 0) || !(s.n_window > 0)) return fail(VMC_E_ARG, "empty totals");
    // Sampler::computeAverages (sampler.cpp:194-226)
    const double M = s.n_samples;
    vmc_averages a{};
    a.energy = s.energy / M;
    a.kinetic = s.kinetic / M;
    a.external = s.external / M;
    a.interaction = s.interaction / M;
    const double var = (s.energy2 / M - a.energy * a.energy) / M;
    a.std_error = var > 0 ? std::sqrt(var) : 0.0;
    a.acceptance = s.accepts / M;
    a.walker_std_error = e->last_walker_std_error;
    if (std::isnan(a.kinetic)) {
        if (out) *out = a;
        return fail(VMC_E_NAN, "Energy exploded, please decrease the learning rate");
    }
    // a NaN local energy from the potential alone (the kinetic average finite) would
    // otherwise reach the parameters through the gradient: no optimiser step either
    if (std::isnan(a.energy)) {
        if (out) *out = a;
        return fail(VMC_E_NAN, "NaN local energy; the parameters are left unchanged");
    }
    // Optimization::getEnergyGradient (optimization.cpp:10-16)
    const size_t P = e->theta.size();
    std::vector<double> grad(P), delta(P);
    for (size_t i = 0; i < P; ++i) {
        const double dg = grad_sum[i] / s.n_window, dge = egrad_sum[i] / s.n_window;
        grad[i] = 2.0 * (dge - a.energy * dg);
    }
    e->opt_step += 1;
    const double eta = e->cfg.eta;
    if (e->cfg.optimization == "adam") {  // adam.cpp:22-37
        // compat: reference beta1 = 0.89 with moments started at ones (adam.cpp:35-36,
        // adam.h:72); corrected: the standard method (beta1 = 0.9, moments from zero)
        const double b1 = e->compat ? 0.89 : 0.9, b2 = 0.999, eps = 1e-8;
        for (size_t i = 0; i < P; ++i) {
            e->opt_m[i] = b1 * e->opt_m[i] + (1 - b1) * grad[i];
            e->opt_v[i] = b2 * e->opt_v[i] + (1 - b2) * grad[i] * grad[i];
            const double mh = e->opt_m[i] / (1 - std::pow(b1, e->opt_step));
            const double vh = e->opt_v[i] / (1 - std::pow(b2, e->opt_step));
            delta[i] = eta * mh / (std::sqrt(vh) + eps);
        }
    } else {  // gradientdescent.cpp:24-29, sgd.cpp:23-28
        const double mono = 1.0 / std::pow((double)e->opt_step, e->cfg.opt_power);
        for (size_t i = 0; i < P; ++i) {
            e->opt_v[i] = e->cfg.opt_gamma * e->opt_v[i] + eta * grad[i] * mono;
            delta[i] = e->opt_v[i];
        }
    }
    std::vector<double> th(e->theta);
    for (size_t i = 0; i < P; ++i) th[i] -= delta[i];  // system.cpp:114
    const int rc = set_parameters(e, th.data(), refresh);
    if (rc) return rc;
    if (out) *out = a;
    return VMC_OK;
}


int finish_sample(vmc_engine *e, const SamplePass &p, vmc_sums *out, std::vector<double> &sums)
{
    // a walker whose tensor-core wait gave up stopped sampling part-way: its sums are
    // incomplete and its record may be too, so neither the pass nor the walkers are used
    // until they are set up again (the status words are cumulative)
    if (p.status & ST_TC_TIMEOUT)
        return fail(VMC_E_TIMEOUT, "a tensor-core completion wait gave up; re-initialise the walkers");
    const double *dev_sums = p.dev_sums;
    sums.assign(e->nacc, 0.0);
    if (e->general || e->flags == FX_MLP_DOT) {  // active parameters back to their (element, parameter) slots
        std::copy(dev_sums, dev_sums + 9, sums.begin());
        const size_t na = e->act.size();
        for (size_t c = 0; c < na; ++c) {
            sums[9 + e->act[c]] = dev_sums[9 + c];
            sums[9 + e->EP + e->act[c]] = dev_sums[9 + na + c];
        }
    } else {
        std::copy(dev_sums, dev_sums + e->nacc, sums.begin());
    }
    double max_drift = 0.0, q99_drift = 0.0;
    if (p.drift && !p.drift->empty()) {
        std::vector<double> &drift = *p.drift;
        for (double d : drift) max_drift = std::max(max_drift, d);
        const size_t i99 = (size_t)(0.99 * (drift.size() - 1));
        std::nth_element(drift.begin(), drift.begin() + i99, drift.end());
        q99_drift = drift[i99];
    }
    if (e->refresh_auto && p.n_refresh) {
        // FP64 re-inversion cadence against the drift of the FP32 Sherman-Morrison
        // inverse: the 99th percentile over walkers (the maximum is set by the few
        // walkers sitting near a node of the determinant) halves the interval past
        // the tolerance and doubles it below 1/2.5 of it (drift grows about in
        // proportion to the interval, so a doubling stays under the tolerance), up to
        // 64 D steps or REFRESH_CAP_MIN (small blocks drift little: one refresh per
        // sweep of a few thousand steps)
        if (q99_drift > e->drift_tol) e->refresh_interval = std::max(e->D, e->refresh_interval / 2);
        else if (q99_drift < e->drift_tol / 2.5)
            e->refresh_interval = std::min(std::max(64 * e->D, REFRESH_CAP_MIN), e->refresh_interval * 2);
    }
    const double W = e->W;
    vmc_sums s{};
    s.energy = sums[0];
    s.energy2 = sums[1];
    s.kinetic = sums[2];
    s.kinetic2 = sums[3];
    s.external = sums[4];
    s.external2 = sums[5];
    s.interaction = sums[6];
    s.interaction2 = sums[7];
    s.accepts = sums[8];
    s.n_samples = W * (p.steps - p.burn_in);
    s.n_window = W * p.bs;
    s.seconds = p.ms * 1e-3;
    s.sweep_seconds = p.sweep_ms * 1e-3;
    s.sweep_launches = p.n_launch;
    s.max_drift = max_drift;
    s.q99_drift = q99_drift;
    s.status = p.status;
    e->last = s;
    e->last_samples_per_walker = p.steps - p.burn_in;
    e->last_walker_std_error = 0.0;
    if (p.walker_std_error >= 0.0) {
        e->last_walker_std_error = p.walker_std_error;
    } else if (e->W > 1) {  // independent chains: spread of the per-walker means
        std::vector<double> we(e->W);
        const int rc = vmc_get_walker_energies(e, we.data());
        if (rc) return rc;
        double mu = 0.0, v2 = 0.0;
        for (double x : we) mu += x;
        mu /= e->W;
        for (double x : we) v2 += (x - mu) * (x - mu);
        e->last_walker_std_error = std::sqrt(v2 / (e->W - 1) / e->W);
    }
    if (out) *out = s;
    return VMC_OK;
}

}  // namespace vmc
