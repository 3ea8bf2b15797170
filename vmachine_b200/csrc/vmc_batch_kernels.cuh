// Multi-system kernels: many quantum dots and atoms (different N, omega, Z), each
// with its own walker pool and parameters, swept by one persistent kernel.
//
// Work queue.  The host lists work items (system s, first walker w0), each of
// `per_item` consecutive walkers, ordered by decreasing cost (walker-steps x the
// system's work per step), so the longest items start first and the short ones fill
// the tail.  A persistent grid (CTAs = occupancy x SMs) runs until the list is
// empty: each warp takes the next item with one atomicAdd on the round's counter and
// sweeps its walkers with the system's own code path (the 2D closed-shell dot sweep
// compiled for the system's Hermite shell count, or the general FP64 path).  Warps
// never wait on each other: no block-wide barrier, no spin.
//
// Per-system arguments live in constant memory (c_sys, c_gen), written from pinned
// host memory at the start of every iteration, so a captured CUDA graph of the
// iteration replays with the current parameters.  The warp's index into them is
// uniform, so the loads are broadcasts.
//
// Rounds.  A system sweeps `a.steps` steps per round (its FP64 refresh interval in
// mixed precision), `total_steps` per iteration; round r covers steps
// [r a.steps, min((r + 1) a.steps, total_steps)).  The rebuild kernel refreshes the
// systems that swept in round r; with round = -1 it re-derives the walkers of the
// systems whose parameters changed since their last sweep.
#pragma once
#include "vmc_general_dev.cuh"

namespace vmc {

constexpr int BATCH_MAX_SYS = 64;
constexpr int BATCH_MAX_GEN = 16;
constexpr int BATCH_GENERAL = 0;  // BatchSys::kind of a general-path system (else the Hermite shells K)
constexpr int BATCH_EXTRA = 4;    // per-system outputs after the accumulators (see batch_reduce_kernel)

struct BatchSys {
    SweepArgs a;        // P, burn-in, gradient window, seed; a.steps = steps per round
    int total_steps;    // steps of the iteration
    int kind;           // Hermite shells K of a 2D closed-shell dot, or BATCH_GENERAL
    int gen;            // index into c_gen (general path)
    int refresh;        // FP64 rebuild after each round
    int theta_refresh;  // parameters changed: re-derive the walkers before round 0
    int samples;        // sampled steps per walker (total_steps - burn-in)
    int seg;            // walkers per warp in the sweep: the engine's for N <= 30, else 1
    int owner;          // N = 42, 56: the owner-form sweep (a.oc / a.ocf hold its constants)
    double *drift;      // W: inverse drift of the refreshes
};

struct BatchLaunch {
    const int2 *items;  // (system, first walker)
    int n_items, per_item;
    int *queue;         // this launch's counter (zeroed before the launch)
    int round;          // sweep round, or -1 (rebuild: parameter refresh)
    int smem_per_warp;
};

static __constant__ BatchSys c_sys[BATCH_MAX_SYS];
static __constant__ GenParams c_gen[BATCH_MAX_GEN];

__device__ __forceinline__ bool batch_next(const BatchLaunch &b, int lane, int2 &item)
{
    int it = 0;
    if (lane == 0) it = atomicAdd(b.queue, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= b.n_items) return false;
    item = b.items[it];
    return true;
}

// The general-path walkers of an item, out of line: its FP64 code is register-hungry
// and would otherwise raise the pressure in the dot paths of the same kernel.
// The warp's slice (`slice` doubles): GEN_SCR scratch doubles, then the staged record
// and, when they fit too, the accumulators (the slice is sized by the batch's largest
// dot record, so a large general-path walker stages less or nothing).
// N = 42, 56: the owner-form sweep, with the drift limiter's instance where it is on
template <typename T, int K, int FX>
__device__ __forceinline__ void batch_owner_walkers(const BatchSys &sy, int steps, int off, unsigned char *ws, int w0,
                                                    int w_end)
{
    if constexpr ((FX & Q_IS_GREEN) == 0) {
        if (sy.a.P.drift_limit > 0.0) {
            owner_sweep_walkers<T, K, FX, true>(sy.a, steps, off, ws, w0, w_end, 1);
            return;
        }
    }
    owner_sweep_walkers<T, K, FX>(sy.a, steps, off, ws, w0, w_end, 1);
}

// The atoms' FP32 sweep (g.f32): the same slice, with FP32 scratch and staged records
// (the FP64 Slater inverse and the accumulators after each record).  Returns false when
// the staged records do not fit the slice; the caller then runs the FP64 sweep on the
// FP64 records.
static __device__ __noinline__ bool batch_gen_walkers_f32(const SweepArgs &a, int steps, int off, const GenParams &g,
                                                          int w0, int w_end, double *scr, int slice)
{
    TcMlp tc{};
    const int full = gen_stage_bytes(g, a.P.nacc, 4);
    float *scr32 = reinterpret_cast<float *>(scr);
    unsigned char *base = reinterpret_cast<unsigned char *>(scr + GEN_SCR);
    const long long room = (long long)(slice - GEN_SCR) * 8;
    if (g.variant != GV_ATOM || full == 0) return false;
    if (g.seg == 4) {
        if (4LL * full > room) return false;
        const int seg = (threadIdx.x & 31) >> 3;
        float *st4 = reinterpret_cast<float *>(base + seg * full);
        for (int wb = w0; wb < w_end; wb += 4) {
            const int w = wb + seg;
            if (w < w_end)
                gen_sweep_walker<false, GV_ATOM, 8, float>(a, steps, off, g, w, true, scr32 + seg * (GEN_SCR / 4),
                                                           nullptr, tc, nullptr, st4, true);
        }
        return true;
    }
    if (full > room) return false;
    for (int w = w0; w < w_end; ++w)
        gen_sweep_walker<false, GV_ATOM, 32, float>(a, steps, off, g, w, true, scr32, nullptr, tc, nullptr,
                                                    reinterpret_cast<float *>(base), true);
    return true;
}

static __device__ __noinline__ void batch_gen_walkers(const SweepArgs &a, int steps, int off, const GenParams &g, int w0,
                                               int w_end, double *scr, int slice)
{
    TcMlp tc{};  // the general systems of a batch have no MLP factor
    if (g.f32 && batch_gen_walkers_f32(a, steps, off, g, w0, w_end, scr, slice)) return;
    const int full = gen_stage_doubles(g, a.P.nacc);
    const bool rec_fits = !g.mlp && GEN_SCR + g.rec <= slice, acc_fits = full && GEN_SCR + full <= slice;
    double *stage = rec_fits ? scr + GEN_SCR : nullptr;
    if (g.variant == GV_ATOM && g.seg == 4) {
        // four walkers per warp: 8-lane segments, each with a quarter of the scratch and,
        // when they fit after it, its own staged record and accumulators
        const int seg = (threadIdx.x & 31) >> 3;
        const bool fits4 = !g.mlp && GEN_SCR + 4 * full <= slice && full > 0;
        double *st4 = fits4 ? scr + GEN_SCR + seg * full : nullptr;
        for (int wb = w0; wb < w_end; wb += 4) {
            const int w = wb + seg;
            if (w < w_end)
                gen_sweep_walker<false, GV_ATOM, 8>(a, steps, off, g, w, true, scr + seg * (GEN_SCR / 4), nullptr, tc,
                                                    nullptr, st4, fits4);
        }
        return;
    }
    for (int w = w0; w < w_end; ++w) {
        if (g.variant == GV_ATOM)
            gen_sweep_walker<false, GV_ATOM>(a, steps, off, g, w, true, scr, nullptr, tc, nullptr, stage, acc_fits);
        else
            gen_sweep_walker<false>(a, steps, off, g, w, true, scr, nullptr, tc, nullptr, stage, acc_fits);
    }
}

// CTAs per SM the batch sweep is compiled for, its register budget (3: 80 registers
// at 256 threads; 2, 128 registers, ran the 64-system workload 5 % slower)
#ifndef BATCH_MIN_BLOCKS
#define BATCH_MIN_BLOCKS 3
#endif
template <typename T, int FX>
__global__ void __launch_bounds__(sizeof(T) == 4 ? 256 : 128, BATCH_MIN_BLOCKS) batch_sweep_kernel(const BatchLaunch b)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ws = smem_raw + (size_t)wib * b.smem_per_warp;
    int2 item;
    while (batch_next(b, lane, item)) {
        const BatchSys &sy = c_sys[item.x];
        const int off = b.round * sy.a.steps;
        if (off >= sy.total_steps) continue;
        const int steps = min(sy.a.steps, sy.total_steps - off);
        const int w_end = min(item.y + b.per_item * sy.seg, sy.a.P.W);
        const int seg_stride = (b.smem_per_warp / max(1, sy.seg)) & ~15;  // 16-byte aligned walker slices
        switch (sy.kind) {
        case 1:
            if (sy.seg == 4) sweep_walkers<T, 2, 1, FX, true, 4>(sy.a, steps, off, ws, item.y, w_end, 4, nullptr, seg_stride);
            else if (sy.seg == 2) sweep_walkers<T, 2, 1, FX, true, 2>(sy.a, steps, off, ws, item.y, w_end, 2, nullptr, seg_stride);
            else sweep_walkers<T, 2, 1, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 2:
            if (sy.seg == 4) sweep_walkers<T, 2, 2, FX, true, 4>(sy.a, steps, off, ws, item.y, w_end, 4, nullptr, seg_stride);
            else if (sy.seg == 2) sweep_walkers<T, 2, 2, FX, true, 2>(sy.a, steps, off, ws, item.y, w_end, 2, nullptr, seg_stride);
            else sweep_walkers<T, 2, 2, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 3:
            if (sy.seg == 2) sweep_walkers<T, 2, 3, FX, true, 2>(sy.a, steps, off, ws, item.y, w_end, 2, nullptr, seg_stride);
            else sweep_walkers<T, 2, 3, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 4:
            if (sy.seg == 2) sweep_walkers<T, 2, 4, FX, true, 2>(sy.a, steps, off, ws, item.y, w_end, 2, nullptr, seg_stride);
            else sweep_walkers<T, 2, 4, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 5:
            if (sy.seg == 2) sweep_walkers<T, 2, 5, FX, true, 2>(sy.a, steps, off, ws, item.y, w_end, 2, nullptr, seg_stride);
            else sweep_walkers<T, 2, 5, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 6:
            if (sy.owner) batch_owner_walkers<T, 6, FX>(sy, steps, off, ws, item.y, w_end);
            else sweep_walkers<T, 2, 6, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        case 7:
            if (sy.owner) batch_owner_walkers<T, 7, FX>(sy, steps, off, ws, item.y, w_end);
            else sweep_walkers<T, 2, 7, FX, true>(sy.a, steps, off, ws, item.y, w_end, 1);
            break;
        default:
            batch_gen_walkers(sy.a, steps, off, c_gen[sy.gen], item.y, w_end, reinterpret_cast<double *>(ws),
                              b.smem_per_warp / (int)sizeof(double));
            break;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128, 3) batch_rebuild_kernel(const BatchLaunch b)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *ws = smem_raw + (size_t)wib * b.smem_per_warp;
    int2 item;
    while (batch_next(b, lane, item)) {
        const BatchSys &sy = c_sys[item.x];
        if (sy.kind == BATCH_GENERAL) continue;
        double *drift = nullptr;
        if (b.round < 0) {
            if (!sy.theta_refresh) continue;
        } else {
            if (!sy.refresh || b.round * sy.a.steps >= sy.total_steps) continue;
            drift = sy.drift;
        }
        const int w_end = min(item.y + b.per_item * sy.seg, sy.a.P.W);
        switch (sy.kind) {
        case 1: rebuild_walkers<T, 2, 1>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 2: rebuild_walkers<T, 2, 2>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 3: rebuild_walkers<T, 2, 3>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 4: rebuild_walkers<T, 2, 4>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 5: rebuild_walkers<T, 2, 5>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 6: rebuild_walkers<T, 2, 6>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        case 7: rebuild_walkers<T, 2, 7>(sy.a.P, RB_REFRESH, drift, ws, item.y, w_end, 1); break;
        default: break;
        }
    }
}

// Zero every system's accumulators and drift (blockIdx.y = system).  (T only keeps
// the two precisions' units apart: each reads its own c_sys.)
template <typename T>
__global__ void batch_clear_kernel()
{
    const BatchSys &sy = c_sys[blockIdx.y];
    const size_t W = sy.a.P.W, n = W * sy.a.P.nacc * 2;
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
    for (size_t i = t0; i < n; i += st) sy.a.P.acc[i] = 0.0;
    for (size_t i = t0; i < W; i += st) sy.drift[i] = 0.0;
}

// Per system (blockIdx.y) and accumulator (blockIdx.x < nacc): the same compensated
// reduction over walkers, in the same order, as the single-system engine's, so a
// system gives the same totals alone or in a batch.  Block gridDim.x - 1 writes the
// extras at out[s * stride + stride - BATCH_EXTRA ..]: OR of the walkers' status
// words, the mean of the walkers' mean energies and the sum of squared deviations
// from it; and copies the walkers' drift to drift_all[drift_off[s] ..].
template <typename T>
__global__ void __launch_bounds__(256) batch_reduce_kernel(double *out, int stride, double *drift_all,
                                                           const long long *drift_off)
{
    const int s = blockIdx.y, a = blockIdx.x;
    const BatchSys &sy = c_sys[s];
    const int W = sy.a.P.W, nacc = sy.a.P.nacc;
    const double *acc = sy.a.P.acc;
    __shared__ double ss[256], cc[256];
    __shared__ unsigned so[256];
    if (a < nacc) {
        double S = 0.0, C = 0.0;
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            kadd(S, C, acc[((size_t)w * nacc + a) * 2]);
            kadd(S, C, acc[((size_t)w * nacc + a) * 2 + 1]);
        }
        ss[threadIdx.x] = S;
        cc[threadIdx.x] = C;
        __syncthreads();
        if (threadIdx.x == 0) {
            double S2 = 0.0, C2 = 0.0;
            for (int t = 0; t < (int)blockDim.x; ++t) {
                kadd(S2, C2, ss[t]);
                kadd(S2, C2, cc[t]);
            }
            out[(size_t)s * stride + a] = S2 + C2;
        }
        return;
    }
    if (a != (int)gridDim.x - 1) return;
    double *o = out + (size_t)s * stride + stride - BATCH_EXTRA;
    const double n = sy.samples > 1 ? (double)sy.samples : 1.0;
    unsigned st = 0u;
    double S = 0.0, C = 0.0;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        st |= sy.a.P.status[w];
        const double m = (acc[(size_t)w * nacc * 2] + acc[(size_t)w * nacc * 2 + 1]) / n;
        kadd(S, C, m);
        if (sy.refresh) drift_all[drift_off[s] + w] = sy.drift[w];
    }
    ss[threadIdx.x] = S + C;
    so[threadIdx.x] = st;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S2 = 0.0, C2 = 0.0;
        unsigned st2 = 0u;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            kadd(S2, C2, ss[t]);
            st2 |= so[t];
        }
        ss[0] = (S2 + C2) / W;
        o[0] = (double)st2;
        o[1] = ss[0];
    }
    __syncthreads();
    const double mu = ss[0];
    double V = 0.0, VC = 0.0;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        const double d = (acc[(size_t)w * nacc * 2] + acc[(size_t)w * nacc * 2 + 1]) / n - mu;
        kadd(V, VC, d * d);
    }
    __syncthreads();
    cc[threadIdx.x] = V + VC;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S2 = 0.0, C2 = 0.0;
        for (int t = 0; t < (int)blockDim.x; ++t) kadd(S2, C2, cc[t]);
        o[2] = S2 + C2;
    }
}

// Kernel handles and constant-memory upload of one precision's translation unit.
struct BatchOps {
    const void *sweep_compat, *sweep_corrected, *rebuild, *clear, *reduce;
    cudaError_t (*upload)(const BatchSys *sys, int n_sys, const GenParams *gen, int n_gen, cudaStream_t st);
    cudaError_t (*upload_hermite)(const HermiteCoef &h);
};

template <typename T>
cudaError_t batch_upload(const BatchSys *sys, int n_sys, const GenParams *gen, int n_gen, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyToSymbolAsync(c_sys, sys, sizeof(BatchSys) * n_sys, 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n_gen > 0)
        e = cudaMemcpyToSymbolAsync(c_gen, gen, sizeof(GenParams) * n_gen, 0, cudaMemcpyHostToDevice, st);
    return e;
}

template <typename T>
cudaError_t batch_upload_hermite(const HermiteCoef &h)
{
    return cudaMemcpyToSymbol(c_herm, &h, sizeof(h));
}

template <typename T>
BatchOps make_batch_ops()
{
    BatchOps o;
    o.sweep_compat = reinterpret_cast<const void *>(&batch_sweep_kernel<T, FX_DOT_COMPAT>);
    o.sweep_corrected = reinterpret_cast<const void *>(&batch_sweep_kernel<T, FX_DOT_CORRECTED>);
    o.rebuild = reinterpret_cast<const void *>(&batch_rebuild_kernel<T>);
    o.clear = reinterpret_cast<const void *>(&batch_clear_kernel<T>);
    o.reduce = reinterpret_cast<const void *>(&batch_reduce_kernel<T>);
    o.upload = &batch_upload<T>;
    o.upload_hermite = &batch_upload_hermite<T>;
    return o;
}

}  // namespace vmc
