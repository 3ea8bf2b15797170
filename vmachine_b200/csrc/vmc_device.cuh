// Device building blocks of the walker engine (sm_100a).
//
// One warp owns one walker.  Everything here is warp-synchronous: a value that is
// the same in all 32 lanes ("uniform") is computed redundantly by every lane, which
// costs one warp instruction, and lane-parallel work is spread over lanes by
// particle or by orbital.  Reductions are xor-butterflies so that every lane ends
// with the total.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vmc {

constexpr unsigned FULL = 0xffffffffu;

// ------------------------------------------------------------------ flags
enum : int {
    F_GAUSS = 1 << 0,        // Gaussian element, exp(-omega alpha sum x^2 / 2)
    F_SLATER = 1 << 1,       // Slater determinant (Hermite basis)
    F_PADE = 1 << 2,         // Pade-Jastrow
    F_COULOMB = 1 << 3,      // Coulomb interaction
    F_ATOM = 1 << 4,         // atomic nucleus potential (else harmonic oscillator)
    Q_PADE_RATIO = 1 << 5,   // Pade ratio over partners j > moved particle only
    Q_PADE_DGAMMA = 1 << 6,  // dlnPsi/dgamma halved
    Q_IS_GREEN = 1 << 7,     // importance-sampling Green's ratio with the cached force
    Q_PADE_STALE = 1 << 8,   // Pade pairs keep the previous gamma until their particle moves
    F_HYDROGENLIKE = 1 << 9, // exp(-alpha Z sum r_i)
    F_IS = 1 << 10,          // importance sampling (else brute force)
    // general path only
    F_SIMPLEJ = 1 << 11,     // SimpleJastrow
    F_RBMG = 1 << 12,        // RBMGaussian
    F_RBMP = 1 << 13,        // RBMProduct
    Q_SJ_RATIO = 1 << 14,    // SimpleJastrow ratio over partners j > moved particle only
    Q_RBM_SORT = 1 << 15,    // RBMProduct hidden units see the sorted coordinates
    F_MLP = 1 << 16,         // learned MLP Jastrow
};

// Flag sets with a compiled-in sweep: the 2D quantum dot, Slater x Gaussian x Pade
// with Coulomb and importance sampling, with and without the reference quirks.
constexpr int FX_DOT_COMPAT = F_GAUSS | F_SLATER | F_PADE | F_COULOMB | F_IS | Q_PADE_RATIO |
                              Q_PADE_DGAMMA | Q_IS_GREEN | Q_PADE_STALE;
constexpr int FX_DOT_CORRECTED = F_GAUSS | F_SLATER | F_PADE | F_COULOMB | F_IS;
// the same dot with the learned MLP Jastrow in place of the Pade factor (corrected
// mode): the sweep runs the CTA's walkers in lockstep for the tensor-core layer
constexpr int FX_MLP_DOT = F_GAUSS | F_SLATER | F_MLP | F_COULOMB | F_IS;

enum : int { SAMPLER_IS = 0, SAMPLER_BF = 1 };

// walker status bits
enum : int {
    ST_NAN_ENERGY = 1,
    ST_BAD_RATIO = 2,
    ST_SINGULAR = 4,
    ST_TC_TIMEOUT = 8,  // a tensor-core completion wait gave up (its results are not used)
};

// ------------------------------------------------------------------ RNG
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

constexpr double TWO_M32 = 2.3283064365386963e-10;

// ------------------------------------------------------------------ reductions
template <typename R>
__device__ __forceinline__ R warp_sum(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Neumaier-compensated accumulation (Neumaier 1974): s + c carries the sum.
__device__ __forceinline__ void kadd(double &s, double &c, double v)
{
    const double t = s + v;
    c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
    s = t;
}

// ------------------------------------------------------------------ math
// FP32 PTX approximate instructions with subnormals flushed, one MUFU each (the
// non-flushing forms add a rescaling of subnormal operands around it): for the FP32
// sweeps' distances, denominators and exponents, which stay far from that range.
// exp(x) = 2^(x log2 e).
__device__ __forceinline__ float approx_rsqrt(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float approx_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float approx_exp(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x * 1.4426950408889634f));
    return r;
}

// Coefficients of the normalised Hermite functions h_m = H_m / sqrt(2^m m!):
//   h_{m+1} = A_m x h_m - B_m h_{m-1},  A_m = sqrt(2/(m+1)), B_m = sqrt(m/(m+1))
//   h'_m = C_m h_{m-1},  C_m = sqrt(2m);   h''_m = E_m h_{m-2},  E_m = 2 sqrt(m(m-1))
// Filled once per device from the host (same double expressions as the CPU oracle).
// One copy per translation unit (internal linkage); each precision's kernel unit
// uploads its own copy.
constexpr int HMAX = 24;
struct HermiteCoef {
    double A[HMAX], B[HMAX], C[HMAX], E[HMAX];
    float Af[HMAX], Bf[HMAX], Cf[HMAX], Ef[HMAX];
};
static __constant__ HermiteCoef c_herm;

template <typename R> __device__ __forceinline__ R hA(int m);
template <> __device__ __forceinline__ double hA<double>(int m) { return c_herm.A[m]; }
template <> __device__ __forceinline__ float hA<float>(int m) { return c_herm.Af[m]; }
template <typename R> __device__ __forceinline__ R hB(int m);
template <> __device__ __forceinline__ double hB<double>(int m) { return c_herm.B[m]; }
template <> __device__ __forceinline__ float hB<float>(int m) { return c_herm.Bf[m]; }
template <typename R> __device__ __forceinline__ R hC(int m);
template <> __device__ __forceinline__ double hC<double>(int m) { return c_herm.C[m]; }
template <> __device__ __forceinline__ float hC<float>(int m) { return c_herm.Cf[m]; }
template <typename R> __device__ __forceinline__ R hE(int m);
template <> __device__ __forceinline__ double hE<double>(int m) { return c_herm.E[m]; }
template <> __device__ __forceinline__ float hE<float>(int m) { return c_herm.Ef[m]; }

// h_0..h_{M-1} at x (registers; M is a compile-time count so indices stay static)
template <int M, typename R>
__device__ __forceinline__ void hermite_values(R x, R (&h)[M])
{
    h[0] = R(1);
    if (M > 1) h[1] = hA<R>(0) * x;
#pragma unroll
    for (int m = 1; m + 1 < M; ++m) h[m + 1] = hA<R>(m) * x * h[m] - hB<R>(m) * h[m - 1];
}

template <int M, typename R>
__device__ __forceinline__ void hermite_derivs(const R (&h)[M], R (&h1)[M], R (&h2)[M])
{
#pragma unroll
    for (int m = 0; m < M; ++m) {
        h1[m] = m >= 1 ? hC<R>(m) * h[m - 1] : R(0);
        h2[m] = m >= 2 ? hE<R>(m) * h[m - 2] : R(0);
    }
}

// ------------------------------------------------------------------ orbitals
// Closed-shell Hermite orbitals in the reference's order (basis.cpp:81-116):
// 2D shell s: (s-j, j), j = 0..s;  3D shell s: (s-j-l, j, l).
template <int DIM, int K> struct Shells;
template <int K> struct Shells<2, K> { static constexpr int n = K * (K + 1) / 2; };
template <int K> struct Shells<3, K> { static constexpr int n = K * (K + 1) * (K + 2) / 6; };

// Calls f(o, mx, my, mz) for every orbital o, fully unrolled.
template <int DIM, int K, typename F>
__device__ __forceinline__ void for_each_orbital(F &&f)
{
    int o = 0;
#pragma unroll
    for (int s = 0; s < K; ++s) {
        if (DIM == 2) {
#pragma unroll
            for (int j = 0; j <= s; ++j) { f(o, s - j, j, 0); ++o; }
        } else {
#pragma unroll
            for (int j = 0; j <= s; ++j)
#pragma unroll
                for (int l = 0; l <= s - j; ++l) { f(o, s - j - l, j, l); ++o; }
        }
    }
}

}  // namespace vmc
