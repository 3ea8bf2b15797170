// Blocking analysis of local-energy series (Sampler::doResampling,
// src/sampler.cpp:319-405, with the Blocker of include/block/blocker.cpp:10-71: the
// automatic blocking method of M. Jonsson, Phys. Rev. E 98, 043304 (2018)).
//
// The reference writes every rank's instant energies (E_L, T, V_ext, V_int per
// sampled step) to files, appends them and blocks each concatenated series.  Here
// the walkers' series stay in HBM (the sweep records (T, V_ext, V_int) per walker and
// step) and are blocked on the device:
//   block_levels_kernel  one CTA per walker: the blocking transform x <- (x_2i +
//     x_2i+1) / 2 level by level on the walker's first 2^d sampled steps, for the
//     four series at once, with the per-level sums the test needs (centred on the
//     global mean); the walker's own blocking estimate of the variance of its mean;
//     its fully blocked value;
//   block_reduce_kernel  per (series, level): the sums over walkers, with the lag-1
//     products across walker boundaries of the concatenated series.
// The host completes the levels above a walker (the W fully blocked values) and
// applies the test.  A walker-major concatenation of the series is the reference's
// appended file with walkers in place of ranks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "vmc_engine.hpp"

using namespace vmc;

namespace {

constexpr int BL_MAX = 40;      // levels (series of up to 2^40 samples)
constexpr int BL_PARTS = 4;     // E_L, T, V_ext, V_int
constexpr int BL_STATS = 5;     // sum X, sum X^2, sum X_i X_i+1, first X, last X  (X = x - global mean)
constexpr int BL_THREADS = 256;

__constant__ double c_chi2[BL_MAX];  // 95% quantiles of chi-square, 1..BL_MAX degrees of freedom

// Regularised lower incomplete gamma P(a, x): power series below a + 1, Lentz's
// continued fraction for Q = 1 - P above (Numerical Recipes, 3rd ed., 6.2).
double gamma_p(double a, double x)
{
    if (x <= 0.0) return 0.0;
    const double lg = std::lgamma(a);
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int n = 0; n < 1000; ++n) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (std::fabs(del) < std::fabs(sum) * 1e-16) break;
        }
        return sum * std::exp(-x + a * std::log(x) - lg);
    }
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 1000; ++i) {
        const double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-16) break;
    }
    return 1.0 - std::exp(-x + a * std::log(x) - lg) * h;
}

// q with P(chi^2_k <= q) = p, by bisection on P(k / 2, q / 2).
double chi2_quantile(int k, double p)
{
    double lo = 0.0, hi = k + 20.0 * std::sqrt(2.0 * k) + 20.0;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (gamma_p(0.5 * k, 0.5 * mid) < p) lo = mid;
        else hi = mid;
    }
    return 0.5 * (lo + hi);
}

const std::vector<double> &chi2_table()
{
    static const std::vector<double> t = [] {
        std::vector<double> v(BL_MAX);
        for (int k = 0; k < BL_MAX; ++k) v[k] = chi2_quantile(k + 1, 0.95);
        return v;
    }();
    return t;
}

// The test of blocker.cpp:42-71 on per-level statistics: levels k = 0..d-1 with
// m_k = 2^(d-k) values, gamma_k = lag-1 autocovariance, s_k = variance (both / m_k).
// M_j = (gamma_j / s_j)^2 2^(d-j); the chosen level K is d - (k + 1) for the largest
// k with sum_{j >= d-1-k} M_j below the 95% quantile of chi^2 with k + 1 degrees of
// freedom.  Returns s_K / 2^(d-K) (the variance of the mean) and n_K = 2^(d-K).  A
// level with zero variance contributes M = 0 (a constant series has error 0).
__host__ __device__ inline double jonsson(const double *gam, const double *s, int d, const double *q,
                                          double &nK)
{
    double M[BL_MAX];
    for (int j = 0; j < d; ++j) {
        const double r = s[j] > 0.0 ? gam[j] / s[j] : 0.0;
        M[j] = r * r * ldexp(1.0, d - j);
    }
    // scan from the top as the reference does (first k from d-1 down that passes)
    int k;
    for (k = d - 1; k >= 0; --k) {
        double c = 0.0;
        for (int j = d - 1 - k; j < d; ++j) c += M[j];
        if (c < q[k]) break;
    }
    const int K = d - (k + 1);
    nK = ldexp(1.0, d - K);
    return s[K] / nK;
}

struct LevelArgs {
    const double *rec;   // W x stride x 3: (T, V_ext, V_int) per step
    int stride, first;   // steps per walker in rec, first sampled step
    int d;               // levels: 2^d samples per walker
    const double *mu;    // BL_PARTS global means
    double *scratch;     // W x BL_PARTS x 2^d
    double *stats;       // W x BL_PARTS x d x BL_STATS
    double *wout;        // W x BL_PARTS x 3: fully blocked value, walker mean, blocked variance of it
};

__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < BL_THREADS / 32; ++i) t += red[i];
    return t;
}

__global__ void __launch_bounds__(BL_THREADS) block_levels_kernel(const LevelArgs a)
{
    __shared__ double st[BL_PARTS][BL_MAX][BL_STATS];
    const int w = blockIdx.x, d = a.d;
    const long long n = 1LL << d;
    double *scr = a.scratch + (size_t)w * BL_PARTS * n;
    const double *rw = a.rec + ((size_t)w * a.stride + a.first) * 3;
    __shared__ double vred[BL_THREADS / 32][3 * BL_PARTS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < d; ++k) {
        const long long m = n >> k;
        // level k values: level 0 from the record, level k >= 1 at scratch[n - 2m .. n - m)
        const long long in_off = n - 2 * m, out_off = n - m;
        double S[BL_PARTS] = {0, 0, 0, 0}, Q[BL_PARTS] = {0, 0, 0, 0}, C[BL_PARTS] = {0, 0, 0, 0};
        auto value = [&](long long i, int p) -> double {
            if (k == 0) {
                const double *t = rw + i * 3;
                return p == 0 ? (t[0] + t[1]) + t[2] : t[p - 1];
            }
            return scr[(size_t)p * n + in_off + i];
        };
        // thread t takes the pairs (2i, 2i + 1), i = t, t + BL_THREADS, ...: their sums,
        // the lag-1 products inside the pair and to the next pair's first value, and the
        // pair mean (the next level)
        for (long long i2 = 2 * threadIdx.x; i2 < m; i2 += 2 * BL_THREADS) {
            for (int p = 0; p < BL_PARTS; ++p) {
                const double x0 = value(i2, p), x1 = value(i2 + 1, p);
                const double X0 = x0 - a.mu[p], X1 = x1 - a.mu[p];
                S[p] += X0 + X1;
                Q[p] += X0 * X0 + X1 * X1;
                C[p] += X0 * X1;
                if (i2 + 2 < m) C[p] += X1 * (value(i2 + 2, p) - a.mu[p]);
                scr[(size_t)p * n + out_off + i2 / 2] = 0.5 * (x0 + x1);
            }
        }
        // one block reduction for the twelve sums: shuffles, then one shared round
        double v[3 * BL_PARTS];
        for (int p = 0; p < BL_PARTS; ++p) {
            v[3 * p] = S[p];
            v[3 * p + 1] = Q[p];
            v[3 * p + 2] = C[p];
        }
#pragma unroll
        for (int q = 0; q < 3 * BL_PARTS; ++q)
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 3 * BL_PARTS; ++q) vred[wid][q] = v[q];
        __syncthreads();  // also: the next level reads what this one wrote
        if (threadIdx.x < 3 * BL_PARTS) {
            double t = 0.0;
            for (int q = 0; q < BL_THREADS / 32; ++q) t += vred[q][threadIdx.x];
            st[threadIdx.x / 3][k][threadIdx.x % 3] = t;
        } else if (threadIdx.x < 4 * BL_PARTS) {
            const int p = threadIdx.x - 3 * BL_PARTS;
            st[p][k][3] = value(0, p) - a.mu[p];
            st[p][k][4] = value(m - 1, p) - a.mu[p];
        }
        __syncthreads();  // vred reused by the next level
    }
    if (threadIdx.x == 0) {
        for (int p = 0; p < BL_PARTS; ++p) {
            double *o = a.stats + ((size_t)w * BL_PARTS + p) * d * BL_STATS;
            for (int k = 0; k < d; ++k)
                for (int q = 0; q < BL_STATS; ++q) o[k * BL_STATS + q] = st[p][k][q];
            // this walker's own series, centred on its own mean
            const double delta = st[p][0][0] / (double)n;
            double gam[BL_MAX], s[BL_MAX];
            for (int k = 0; k < d; ++k) {
                const double m = (double)(n >> k), Sk = st[p][k][0];
                const double Qw = st[p][k][1] - 2.0 * delta * Sk + m * delta * delta;
                const double Cw = st[p][k][2] - delta * (2.0 * Sk - st[p][k][3] - st[p][k][4]) +
                                  (m - 1.0) * delta * delta;
                gam[k] = Cw / m;
                s[k] = Qw / m;
            }
            double nK = 0.0;
            const double var = jonsson(gam, s, d, c_chi2, nK);
            double *wo = a.wout + ((size_t)w * BL_PARTS + p) * 3;
            wo[0] = scr[(size_t)p * n + n - 2];  // the level-d value (the pair mean of level d - 1)
            wo[1] = a.mu[p] + delta;
            wo[2] = var;
        }
    }
}

// Per (series p = blockIdx.x, level k = blockIdx.y): sums over walkers of the level
// statistics and of the lag-1 products across walker boundaries; level 0 also sums
// the walkers' means and blocked variances.  out[(p * d + k) * 4 + {0..3}] =
// {sum X, sum X^2, sum X_i X_i+1 (concatenated), 0}; wsum[p * 2 + {0, 1}].
__global__ void __launch_bounds__(BL_THREADS) block_reduce_kernel(const double *stats, const double *wout, int W,
                                                                  int d, double *out, double *wsum)
{
    __shared__ double red[BL_THREADS / 32];
    const int p = blockIdx.x, k = blockIdx.y;
    double S = 0.0, Q = 0.0, C = 0.0, M = 0.0, V = 0.0;
    for (int w = threadIdx.x; w < W; w += BL_THREADS) {
        const double *o = stats + (((size_t)w * BL_PARTS + p) * d + k) * BL_STATS;
        S += o[0];
        Q += o[1];
        C += o[2];
        if (w + 1 < W) C += o[4] * stats[(((size_t)(w + 1) * BL_PARTS + p) * d + k) * BL_STATS + 3];
        if (k == 0) {
            M += wout[((size_t)w * BL_PARTS + p) * 3 + 1];
            V += wout[((size_t)w * BL_PARTS + p) * 3 + 2];
        }
    }
    S = block_sum(S, red);
    Q = block_sum(Q, red);
    C = block_sum(C, red);
    M = block_sum(M, red);
    V = block_sum(V, red);
    if (threadIdx.x == 0) {
        double *r = out + ((size_t)p * d + k) * 4;
        r[0] = S;
        r[1] = Q;
        r[2] = C;
        r[3] = 0.0;
        if (k == 0) {
            wsum[p * 2] = M;
            wsum[p * 2 + 1] = V;
        }
    }
}

// Sum of each walker's first 2^d sampled values of the four series (one CTA per
// walker): the global means the levels are centred on.
__global__ void __launch_bounds__(BL_THREADS) block_sum_kernel(const double *rec, int stride, int first, int d,
                                                               double *wsum)
{
    __shared__ double red[BL_THREADS / 32];
    const int w = blockIdx.x;
    const long long n = 1LL << d;
    const double *rw = rec + ((size_t)w * stride + first) * 3;
    double s[BL_PARTS] = {0, 0, 0, 0};
    for (long long i = threadIdx.x; i < n; i += BL_THREADS) {
        const double *t = rw + i * 3;
        s[0] += (t[0] + t[1]) + t[2];
        s[1] += t[0];
        s[2] += t[1];
        s[3] += t[2];
    }
    for (int p = 0; p < BL_PARTS; ++p) {
        const double v = block_sum(s[p], red);
        if (threadIdx.x == 0) wsum[(size_t)w * BL_PARTS + p] = v;
    }
}

void fill_block(vmc_block &b, double mean, double var, double nK)
{
    b.mean = mean;
    b.mse_mean = var;
    b.std_error = std::sqrt(var);
    b.mse_std_error = nK > 0 ? (2.0 * nK - 1.0) * var * var / (nK * nK) : 0.0;
    b.n_k = (long long)nK;
}

void fail_block(vmc_block &b)
{
    b.mean = b.std_error = b.mse_mean = b.mse_std_error = -1.0;
    b.n_k = 0;
}

int bl_fail(int code, const std::string &m) { return set_last_error(code, m.c_str()); }

#define BLCUDA(expr)                                                                         \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) return bl_fail(VMC_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

}  // namespace

namespace vmc {

int block_record(vmc_engine *e, const double *rec, int steps, int burn_in, vmc_blocking_result *out)
{
    if (steps - burn_in < 2) return bl_fail(VMC_E_ARG, "fewer than two sampled steps");
    std::memset(out, 0, sizeof(*out));
    int d = 0;
    while ((2LL << d) <= (long long)(steps - burn_in)) ++d;
    if (d > BL_MAX) return bl_fail(VMC_E_ARG, "too many steps");
    const long long n = 1LL << d;
    const size_t W = e->W;
    BLCUDA(cudaSetDevice(e->device));
    BLCUDA(cudaMemcpyToSymbolAsync(c_chi2, chi2_table().data(), sizeof(double) * BL_MAX, 0,
                                   cudaMemcpyHostToDevice, e->stream));
    double *scratch = nullptr, *stats = nullptr, *wout = nullptr, *wsum = nullptr, *red = nullptr,
           *mu = nullptr;
    auto release = [&]() {
        cudaFree(scratch);
        cudaFree(stats);
        cudaFree(wout);
        cudaFree(wsum);
        cudaFree(red);
        cudaFree(mu);
    };
    int rc = [&]() -> int {
        BLCUDA(cudaMalloc(&scratch, W * BL_PARTS * (size_t)n * sizeof(double)));
        BLCUDA(cudaMalloc(&stats, W * BL_PARTS * (size_t)d * BL_STATS * sizeof(double)));
        BLCUDA(cudaMalloc(&wout, W * BL_PARTS * 3 * sizeof(double)));
        BLCUDA(cudaMalloc(&wsum, W * BL_PARTS * sizeof(double)));
        BLCUDA(cudaMalloc(&red, (BL_PARTS * (size_t)d * 4 + BL_PARTS * 2) * sizeof(double)));
        BLCUDA(cudaMalloc(&mu, BL_PARTS * sizeof(double)));
        // ---- global means, then the levels
        block_sum_kernel<<<(unsigned)W, BL_THREADS, 0, e->stream>>>(rec, steps, burn_in, d, wsum);
        BLCUDA(cudaGetLastError());
        std::vector<double> ws(W * BL_PARTS);
        BLCUDA(cudaMemcpyAsync(ws.data(), wsum, ws.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        BLCUDA(cudaStreamSynchronize(e->stream));
        double m[BL_PARTS] = {0, 0, 0, 0};
        for (size_t w = 0; w < W; ++w)
            for (int p = 0; p < BL_PARTS; ++p) m[p] += ws[w * BL_PARTS + p];
        for (int p = 0; p < BL_PARTS; ++p) m[p] /= (double)W * (double)n;
        BLCUDA(cudaMemcpyAsync(mu, m, sizeof(m), cudaMemcpyHostToDevice, e->stream));
        LevelArgs la{rec, steps, burn_in, d, mu, scratch, stats, wout};
        block_levels_kernel<<<(unsigned)W, BL_THREADS, 0, e->stream>>>(la);
        BLCUDA(cudaGetLastError());
        double *lev = red, *wred = red + BL_PARTS * (size_t)d * 4;
        block_reduce_kernel<<<dim3(BL_PARTS, d), BL_THREADS, 0, e->stream>>>(stats, wout, (int)W, d, lev, wred);
        BLCUDA(cudaGetLastError());
        std::vector<double> hl(BL_PARTS * (size_t)d * 4 + BL_PARTS * 2), hw(W * BL_PARTS * 3);
        BLCUDA(cudaMemcpyAsync(hl.data(), red, hl.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        BLCUDA(cudaMemcpyAsync(hw.data(), wout, hw.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        BLCUDA(cudaStreamSynchronize(e->stream));
        // ---- results
        out->samples_per_walker = n;
        const bool pow2 = (W & (W - 1)) == 0;
        int dw = 0;
        while ((1ULL << dw) < W) ++dw;
        vmc_block *parts[BL_PARTS] = {&out->energy, &out->kinetic, &out->external, &out->interaction};
        for (int p = 0; p < BL_PARTS; ++p) {
            const double *wr = hl.data() + BL_PARTS * (size_t)d * 4;
            if (p == 0) {
                // independent chains: mean of the walkers' means, variance sum / W^2
                const double vsum = wr[1];
                fill_block(out->energy_walkers, wr[0] / (double)W, vsum / ((double)W * W), 0.0);
                out->energy_walkers.n_k = 0;
            }
            if (!pow2) {
                fail_block(*parts[p]);
                continue;
            }
            // the concatenated series: levels inside a walker from the device sums,
            // then the W fully blocked values (blocks spanning walkers)
            const int D = d + dw;
            if (D > BL_MAX) {
                fail_block(*parts[p]);
                continue;
            }
            double gam[BL_MAX], s[BL_MAX];
            const double total = (double)W * (double)n;
            for (int k = 0; k < d; ++k) {
                const double *r = hl.data() + ((size_t)p * d + k) * 4;
                const double mk = total / std::ldexp(1.0, k);
                gam[k] = r[2] / mk;
                s[k] = r[1] / mk;
            }
            std::vector<double> v(W);
            for (size_t w = 0; w < W; ++w) v[w] = hw[(w * BL_PARTS + p) * 3];
            size_t mm = W;
            for (int k = d; k < D; ++k) {
                double g = 0.0, q = 0.0;
                for (size_t i = 0; i + 1 < mm; ++i) g += (v[i] - m[p]) * (v[i + 1] - m[p]);
                for (size_t i = 0; i < mm; ++i) q += (v[i] - m[p]) * (v[i] - m[p]);
                gam[k] = g / mm;
                s[k] = q / mm;
                for (size_t i = 0; i < mm / 2; ++i) v[i] = 0.5 * (v[2 * i] + v[2 * i + 1]);
                mm /= 2;
            }
            double nK = 0.0;
            const double var = jonsson(gam, s, D, chi2_table().data(), nK);
            fill_block(*parts[p], m[p], var, nK);
        }
        return VMC_OK;
    }();
    cudaStreamSynchronize(e->stream);
    release();
    return rc;
}

}  // namespace vmc

extern "C" {

int vmc_block_series(const double *x, long long n, vmc_block *out)
{
    if (!out || (n > 0 && !x)) return bl_fail(VMC_E_ARG, "null argument");
    if (n < 2 || (n & (n - 1))) {  // blocker.cpp:20-25
        fail_block(*out);
        return VMC_OK;
    }
    int d = 0;
    while ((1LL << d) < n) ++d;
    if (d > BL_MAX) return bl_fail(VMC_E_ARG, "series longer than 2^40");
    double mean = 0.0;
    for (long long i = 0; i < n; ++i) mean += x[i];
    mean /= (double)n;
    std::vector<double> v(x, x + n);
    double gam[BL_MAX], s[BL_MAX];
    long long m = n;
    for (int k = 0; k < d; ++k) {
        double g = 0.0, q = 0.0;
        for (long long i = 0; i + 1 < m; ++i) g += (v[i] - mean) * (v[i + 1] - mean);
        for (long long i = 0; i < m; ++i) q += (v[i] - mean) * (v[i] - mean);
        gam[k] = g / m;
        s[k] = q / m;
        for (long long i = 0; i < m / 2; ++i) v[i] = 0.5 * (v[2 * i] + v[2 * i + 1]);
        m /= 2;
    }
    double nK = 0.0;
    const double var = jonsson(gam, s, d, chi2_table().data(), nK);
    fill_block(*out, mean, var, nK);
    return VMC_OK;
}

int vmc_blocking(vmc_engine *e, int steps, int burn_in, vmc_blocking_result *out)
{
    if (!e || !out) return bl_fail(VMC_E_ARG, "null argument");
    if (!e->have_walkers) return bl_fail(VMC_E_STATE, "vmc_init_walkers first");
    if (steps < 2 || burn_in < 0 || burn_in >= steps - 1) return bl_fail(VMC_E_ARG, "bad step counts");
    BLCUDA(cudaSetDevice(e->device));
    double *rec = nullptr;
    BLCUDA(cudaMalloc(&rec, (size_t)e->W * steps * 3 * sizeof(double)));
    e->d_rec = rec;
    e->rec_stride = steps;
    vmc_sums s{};
    int rc = vmc_sample(e, 0, steps, burn_in, &s, nullptr, nullptr);
    e->d_rec = nullptr;
    e->rec_stride = 0;
    if (!rc) rc = block_record(e, rec, steps, burn_in, out);
    cudaStreamSynchronize(e->stream);
    cudaFree(rec);
    return rc;
}

}  // extern "C"
