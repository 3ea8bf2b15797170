// The learned MLP Jastrow's network on the device: weight layout, FP32 evaluation
// with analytic radial derivatives (CUDA cores), and the pair network's second layer
// on the tensor cores (tcgen05).  Used by the FP32 dot sweep, its FP64 rebuild and
// the general FP64 path.
#pragma once
#include <cuda_bf16.h>

#include "vmc_config.hpp"
#include "vmc_device.cuh"

namespace vmc {

// MLP Jastrow weight offsets (floats) in the packed parameter row
enum : int {
    MW_W1 = 0, MW_B1 = 128, MW_W2 = 192, MW_B2 = 4288, MW_W3 = 4352, MW_B3 = 4416,
    MW_V1 = 4417, MW_C1 = 4449, MW_V2 = 4481, MW_C2 = 5505, MW_V3 = 5537, MW_C3 = 5569,
};
static_assert(MW_C3 + 1 == MLP_PARAMS, "MLP layout");

// ------------------------------------------------------------ MLP Jastrow
// J = sum_{i<j} u(r_ij, s_ij) + sum_i chi(r_i) with
//   u(r, s) = a_s r / (1 + r) + w3 . tanh(W2 tanh(W1 [r, s] + b1) + b2) + b3   (2 -> 64 -> 64 -> 1)
//   chi(r)  = v3 . tanh(V2 tanh(V1 r + c1) + c2) + c3                        (1 -> 32 -> 32 -> 1)
// evaluated in FP32 with the weights rounded to bfloat16; a_s is the Pade cusp
// coefficient (s = 1 same spin).  Radial derivatives by forward-mode
// differentiation: h' = (1 - h^2) z', h'' = (1 - h^2)(z'' - 2 h z'^2).
// Shared-memory weight block of a CTA: the packed row, W2 transposed ([k][m]) and
// V2 transposed, so that lanes over output units read consecutive words.
constexpr int MLP_SMEM_FLOATS = MLP_PARAMS + 2 + MLP_H * MLP_H + MLP_G * MLP_G;  // 10692
constexpr int MW_W2T = MLP_PARAMS + 2, MW_V2T = MW_W2T + MLP_H * MLP_H;
constexpr int MLP_SMEM_DOUBLES = (MLP_SMEM_FLOATS + 3) / 4 * 2;  // 16-byte multiple

__device__ __forceinline__ float mlp_tanh(float x)
{
    x = fminf(fmaxf(x, -9.0f), 9.0f);  // tanh(9) = 1 in FP32
    return 1.0f - 2.0f * approx_rcp(approx_exp(2.0f * x) + 1.0f);
}

// Cooperative copy of the weights into shared memory (all threads of the CTA);
// without w2t the W2-transposed region is left free (the tensor-core sweep uses it
// as an operand tile).
static __device__ void mlp_stage(const float *__restrict__ src, float *w, bool w2t = true)
{
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) w[i] = src[i];
    for (int i = threadIdx.x; w2t && i < MLP_H * MLP_H; i += blockDim.x) {
        const int k = i / MLP_H, m = i - k * MLP_H;
        w[MW_W2T + i] = src[MW_W2 + m * MLP_H + k];
    }
    for (int i = threadIdx.x; i < MLP_G * MLP_G; i += blockDim.x) {
        const int k = i / MLP_G, m = i - k * MLP_G;
        w[MW_V2T + i] = src[MW_V2 + m * MLP_G + k];
    }
}

__device__ __forceinline__ float mlp_cusp(int dim, bool same)
{
    return same ? (dim == 2 ? 1.0f / 3 : 0.25f) : (dim == 2 ? 1.0f : 0.5f);
}

// u, du/dr, d2u/dr2 of the pair network for one pair (one lane).
static __device__ void mlp_pair(const float *w, float r, float s, float a, float &u, float &du, float &ddu)
{
    float uo = w[MW_B3], duo = 0.0f, dduo = 0.0f;
    for (int half = 0; half < 2; ++half) {
        float z[32], dz[32], ddz[32];
#pragma unroll
        for (int m = 0; m < 32; ++m) {
            z[m] = w[MW_B2 + half * 32 + m];
            dz[m] = 0.0f;
            ddz[m] = 0.0f;
        }
        for (int k = 0; k < MLP_H; ++k) {
            const float w1r = w[MW_W1 + 2 * k], w1s = w[MW_W1 + 2 * k + 1];
            const float h = mlp_tanh(fmaf(w1r, r, fmaf(w1s, s, w[MW_B1 + k])));
            const float d = (1.0f - h * h) * w1r, dd = -2.0f * h * d * w1r;
            const float4 *col = reinterpret_cast<const float4 *>(w + MW_W2T + k * MLP_H + half * 32);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 v = col[q];
                const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    z[4 * q + e] = fmaf(vv[e], h, z[4 * q + e]);
                    dz[4 * q + e] = fmaf(vv[e], d, dz[4 * q + e]);
                    ddz[4 * q + e] = fmaf(vv[e], dd, ddz[4 * q + e]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < 32; ++m) {
            const float h2 = mlp_tanh(z[m]), g2 = 1.0f - h2 * h2, w3 = w[MW_W3 + half * 32 + m];
            uo = fmaf(w3, h2, uo);
            duo = fmaf(w3, g2 * dz[m], duo);
            dduo = fmaf(w3, g2 * (ddz[m] - 2.0f * h2 * dz[m] * dz[m]), dduo);
        }
    }
    const float q = 1.0f / (1.0f + r);
    u = uo + a * r * q;
    du = duo + a * q * q;
    ddu = dduo - 2.0f * a * q * q * q;
}

// chi, dchi/dr, d2chi/dr2 of the one-body network at r: warp-cooperative, lane m
// is hidden unit m of the second layer; every lane returns the totals.
// v2t: V2 transposed ([k][m]; the CTA's weight block keeps it at MW_V2T).
static __device__ void mlp_body(const float *w, const float *v2t, float r, int lane, float &c, float &dc, float &ddc)
{
    float z = w[MW_C2 + lane], dz = 0.0f, ddz = 0.0f;
    for (int k = 0; k < MLP_G; ++k) {
        const float v1 = w[MW_V1 + k];
        const float h = mlp_tanh(fmaf(v1, r, w[MW_C1 + k]));
        const float d = (1.0f - h * h) * v1, dd = -2.0f * h * d * v1, vv = v2t[k * MLP_G + lane];
        z = fmaf(vv, h, z);
        dz = fmaf(vv, d, dz);
        ddz = fmaf(vv, dd, ddz);
    }
    const float h2 = mlp_tanh(z), g2 = 1.0f - h2 * h2, v3 = w[MW_V3 + lane];
    c = warp_sum(v3 * h2) + w[MW_C3];
    dc = warp_sum(v3 * g2 * dz);
    ddc = warp_sum(v3 * g2 * (ddz - 2.0f * h2 * dz * dz));
}

// pair index q < N(N-1)/2 -> (i, j), i < j, row-major over i
__device__ __forceinline__ void pair_of(int q, int N, int &i, int &j)
{
    i = 0;
    while (q >= N - 1 - i) {
        q -= N - 1 - i;
        ++i;
    }
    j = i + 1 + q;
}

// ------------------------------------------------------------ MLP second layer on tcgen05
// During a sweep the CTA's four walkers move in lockstep; the partners of the four
// proposals fill one 128-row tile (warp w: rows 32 w .. 32 w + 31, lane = partner).
// First layer and its radial derivatives (CUDA cores) go to three A tiles in
// bfloat16 (the values as a high and a low bfloat16 part, about 16 significant
// bits); z2 = W2 h1 and its two radial derivatives are M = 128, N = 64, K = 64
// products on the 5th-generation tensor cores (kind::f16, BF16 in, FP32 accumulate
// in tensor memory), issued by one thread; each lane then reads its row back
// (tcgen05.ld) and finishes the third layer.
// Shared-memory operands are K-major without swizzle: 8-row x 16-byte core
// matrices, offset(row, k) = (row % 8) 16 + (row / 8) 1024 + (k / 8) 128 + (k % 8) 2,
// so the two K chunks of a K = 16 step are 128 bytes apart (leading byte offset)
// and 8-row groups 1024 bytes apart (stride byte offset).  Tensor memory holds D
// for order o (value, d/dr, d2/dr2) in columns [64 o, 64 o + 64); lane = tile row.
constexpr int TC_COLS = 256;  // TMEM columns per CTA (192 used); two CTAs per SM fit 512
constexpr int TC_A_BYTES = 128 * MLP_H * 2, TC_B_BYTES = MLP_H * MLP_H * 2;
constexpr int TC_SMEM = 3 * TC_A_BYTES + TC_B_BYTES + 1024;  // with alignment slack
constexpr long TC_WAIT_LIMIT = 1L << 24;                     // bounded completion wait
// kind::f16 instruction word: D F32 (bits 4-5), A and B BF16 (7-9, 10-12), both
// K-major, N / 8 (17-22), M / 16 (24-28)
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

struct TcMlp {
    unsigned char *a[4];  // A tiles: value (high bfloat16 part), d/dr, d2/dr2, value (low part)
    uint32_t a_s[4], b_s; // their shared-window addresses, and B's
    uint32_t bar;         // completion mbarrier
    uint32_t tmem;        // TMEM base address (lane 0, first allocated column)
    uint32_t phase;
};

__device__ __forceinline__ uint32_t tc_off(int row, int k)
{
    return (row & 7) * 16 + (row >> 3) * 1024 + (k >> 3) * 128 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start address, LBO 128 B, SBO 1024 B, version 1,
// base offset 0, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                   "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                   "=r"(v[14]), "=r"(v[15])
                 : "r"(addr));
}

// Tiles after the weights, B = W2 ([out n][in k]; the weights are bfloat16 values
// already), the mbarrier, and the TMEM allocation (warp 0).  The caller synchronises
// the CTA and then calls tc_ready.
// lo: where the value's low-part A tile goes (16 KB, 16-byte aligned; null: the W2^T
// slot of the weight block, which the tensor-core path does not otherwise use).
static __device__ void tc_setup(TcMlp &t, unsigned char *base, float *w, const float *__restrict__ src,
                                unsigned long long *bar, uint32_t *slot, int wib, float *lo = nullptr)
{
    unsigned char *p = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(base) + 1023) & ~uintptr_t(1023));
    for (int o = 0; o < 3; ++o) {
        t.a[o] = p + o * TC_A_BYTES;
        t.a_s[o] = (uint32_t)__cvta_generic_to_shared(t.a[o]);
    }
    t.a[3] = reinterpret_cast<unsigned char *>(lo ? lo : w + MW_W2T);  // 16 KB, 16-byte aligned
    t.a_s[3] = (uint32_t)__cvta_generic_to_shared(t.a[3]);
    unsigned char *bt = p + 3 * TC_A_BYTES;
    t.b_s = (uint32_t)__cvta_generic_to_shared(bt);
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) {
        const int n = i >> 6, k = i & 63;
        *reinterpret_cast<__nv_bfloat16 *>(bt + tc_off(n, k)) = __float2bfloat16_rn(src[MW_W2 + n * MLP_H + k]);
    }
    t.bar = (uint32_t)__cvta_generic_to_shared(bar);
    t.phase = 0;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(t.bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (wib == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(slot)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_ready(TcMlp &t, const uint32_t *slot)
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    t.tmem = *slot;
}

// One step of the pair network's second layer for the whole CTA (every thread
// calls it).  valid: this lane's row is a partner of its walker's proposal at
// distance r, same-spin s, cusp coefficient a.  Writes u, du/dr, d2u/dr2 of the
// row to pre[lane], pre[32 + lane], pre[64 + lane]; returns ST_TC_TIMEOUT when the
// completion wait gave up.
static __device__ unsigned tc_pair_layer(TcMlp &t, const float *w, bool valid, float r, float s, float a, int lane,
                                  int wib, float *pre)
{
    const int row = wib * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < 8; ++c) {  // 8 inputs of the second layer per 16-byte store
        uint32_t hv[4], lv[4], dv[4], ddv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float h[2], d[2], dd[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k = 8 * c + 2 * e + q;
                const float w1r = w[MW_W1 + 2 * k], w1s = w[MW_W1 + 2 * k + 1];
                const float hh = valid ? mlp_tanh(fmaf(w1r, r, fmaf(w1s, s, w[MW_B1 + k]))) : 0.0f;
                h[q] = hh;
                d[q] = valid ? (1.0f - hh * hh) * w1r : 0.0f;
                dd[q] = -2.0f * hh * d[q] * w1r;
            }
            // value: high and low bfloat16 parts (about 16 significant bits together)
            hv[e] = pack_bf16(h[0], h[1]);
            const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162 *>(&hv[e]);
            lv[e] = pack_bf16(h[0] - __bfloat162float(hi.x), h[1] - __bfloat162float(hi.y));
            dv[e] = pack_bf16(d[0], d[1]);
            ddv[e] = pack_bf16(dd[0], dd[1]);
        }
        const uint32_t off = tc_off(row, 8 * c);
        *reinterpret_cast<uint4 *>(t.a[0] + off) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<uint4 *>(t.a[1] + off) = make_uint4(dv[0], dv[1], dv[2], dv[3]);
        *reinterpret_cast<uint4 *>(t.a[2] + off) = make_uint4(ddv[0], ddv[1], ddv[2], ddv[3]);
        *reinterpret_cast<uint4 *>(t.a[3] + off) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    }
    // generic-proxy tile writes visible to the tensor cores; earlier TMEM reads done
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
#pragma unroll
        for (int o = 0; o < 4; ++o)  // value high, d/dr, d2/dr2, then value low into the value columns
#pragma unroll
            for (int st = 0; st < 4; ++st) {
                const uint64_t ad = tc_desc(t.a_s[o] + st * 256), bd = tc_desc(t.b_s + st * 256);
                const uint32_t dcol = t.tmem + 64 * (o == 3 ? 0 : o);
                const uint32_t accumulate = (st > 0 || o == 3) ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                 dcol),
                             "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
                             : "memory");
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(t.bar)
                     : "memory");
    }
    uint32_t done = 0;
    for (long it = 0; it < TC_WAIT_LIMIT && !done; ++it)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(t.bar), "r"(t.phase)
                     : "memory");
    t.phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // third layer, two output units at a time in packed FP32 (FADD2 / FMUL2 / FFMA2):
    // with ng = h^2 - 1 = -(1 - h^2) the sums collect -du and -d2u
    float2 u2 = make_float2(0.0f, 0.0f), ndu2 = u2, nddu2 = u2;
    const uint32_t lb = t.tmem + ((uint32_t)(wib * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
        uint32_t z[16], dz[16], ddz[16];
        tmem_ld16(lb + 16 * c, z);
        tmem_ld16(lb + 64 + 16 * c, dz);
        tmem_ld16(lb + 128 + 16 * c, ddz);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 16; e += 4) {
            const int m = 16 * c + e;
            const float4 b4 = *reinterpret_cast<const float4 *>(w + MW_B2 + m);
            const float4 w4 = *reinterpret_cast<const float4 *>(w + MW_W3 + m);
#pragma unroll
            for (int hp = 0; hp < 2; ++hp) {
                const int q = e + 2 * hp;
                const float2 bb = hp ? make_float2(b4.z, b4.w) : make_float2(b4.x, b4.y);
                const float2 ww = hp ? make_float2(w4.z, w4.w) : make_float2(w4.x, w4.y);
                const float2 zz = __fadd2_rn(make_float2(__uint_as_float(z[q]), __uint_as_float(z[q + 1])), bb);
                const float2 d1 = make_float2(__uint_as_float(dz[q]), __uint_as_float(dz[q + 1]));
                const float2 d2 = make_float2(__uint_as_float(ddz[q]), __uint_as_float(ddz[q + 1]));
                const float2 h2 = make_float2(mlp_tanh(zz.x), mlp_tanh(zz.y));
                const float2 ng = __ffma2_rn(h2, h2, make_float2(-1.0f, -1.0f));
                u2 = __ffma2_rn(ww, h2, u2);
                ndu2 = __ffma2_rn(ww, __fmul2_rn(ng, d1), ndu2);
                const float2 inner = __ffma2_rn(__fmul2_rn(h2, __fmul2_rn(d1, d1)), make_float2(-2.0f, -2.0f), d2);
                nddu2 = __ffma2_rn(ww, __fmul2_rn(ng, inner), nddu2);
            }
        }
    }
    const float u = w[MW_B3] + (u2.x + u2.y), du = -(ndu2.x + ndu2.y), ddu = -(nddu2.x + nddu2.y);
    const float q = 1.0f / (1.0f + r);
    pre[lane] = u + a * r * q;
    pre[32 + lane] = du + a * q * q;
    pre[64 + lane] = ddu - 2.0f * a * q * q * q;
    __syncwarp();
    return done ? 0u : (unsigned)ST_TC_TIMEOUT;
}

static __device__ void tc_teardown(TcMlp &t, int wib)
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (wib == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t.tmem), "r"(TC_COLS) : "memory");
}

}  // namespace vmc
