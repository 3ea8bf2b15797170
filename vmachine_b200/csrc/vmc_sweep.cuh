// Metropolis sweep kernel: one warp per walker (or, for the dots up to N = 30, two or
// four walkers per warp in 16- or 8-lane segments), WPB warps per CTA.
//
// Per step (System::runMetropolisCycles body, src/system.cpp:149-163):
//   1. draw (k, displacement, uniform) from the walker's Philox stream (or a replay
//      stream); propose x_k' (brute force: bruteforce.cpp:34; importance sampling
//      with the drift 2 grad ln Psi: importancesampling.cpp:49-60);
//   2. |Psi'|^2/|Psi|^2 per element without touching the state:
//      Slater  R = phi(r_p') . inv[:, p]   (lane j reads row j of the transposed inverse)
//      Pade    sum over partners of beta (h' - h)   (lanes over partners)
//   3. accept: Sherman-Morrison rank-1 update of the moved particle's spin block,
//      refresh of that block's d ln det / d^2 det / det vectors, Pade gradient
//      vector and running pair sums (Laplacian, beta h^2, Coulomb);
//   4. sample E_L = T + V_ext + V_int and dlnPsi/dtheta every step after burn-in
//      into per-lane Neumaier-compensated FP64 accumulators (sampler.cpp:52-90).
// Nothing is snapshotted: a rejected move leaves the state untouched.
//
// Orbital sums are factorised over Hermite degrees: phi_o(r) = prod_c h_{m_c(o)}(x_c),
// so phi(r) . v = sum_{m0} h_{m0}(x) sum_{m1} h_{m1}(y) v_o and the derivative
// vectors contract per-degree partial sums with h' and h''.
//
// Template FX: 0 = element flags read at run time (any supported system); a
// non-zero flag set compiles the flags in (the quantum-dot paths).
//
// Shared memory per walker: the walker record (see Layout), the Pade pair mask
// (N x u64) and the FP64 running scalars (NSCAL doubles).
#pragma once
#include <type_traits>

namespace vmc {

template <typename T> struct Fast;
// FP32: the PTX approximate instructions (vmc_device.cuh)
template <> struct Fast<float> {
    static __device__ __forceinline__ float rsqrt(float x) { return approx_rsqrt(x); }
    static __device__ __forceinline__ float rcp(float x) { return approx_rcp(x); }
    static __device__ __forceinline__ float exp(float x) { return approx_exp(x); }
};
template <> struct Fast<double> {
    static __device__ __forceinline__ double rsqrt(double x) { return ::rsqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
};

// Two values of T in one register pair: FP32 pairs issue one packed sm_100
// instruction (FFMA2 / FMUL2 / FADD2) for both, FP64 pairs stay two instructions.
template <typename T> using Two = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
__device__ __forceinline__ float2 two(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 two(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c)
{
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 mul2(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// phi(r) . v, where v(o) returns the column entry of orbital o (shared memory or a
// lane's registers).
template <typename T, int DIM, int K, typename V>
__device__ __forceinline__ T orbital_dot(const T (&hv)[DIM][K], V &&v)
{
    T part[K];
#pragma unroll
    for (int m = 0; m < K; ++m) part[m] = T(0);
    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
        T f = hv[1][m1];
        if (DIM == 3) f *= hv[DIM - 1][m2];
        part[m0] += f * v(o);
    });
    T s = T(0);
#pragma unroll
    for (int m = 0; m < K; ++m) s += hv[0][m] * part[m];
    return s;
}

// phi(r) . v and d_A phi(r) . v together, the orbital sum factorised along axis A:
// part[m] = sum over orbitals with m_A = m of prod_{c != A} h_{m_c}(x_c) v_o, then
// phi . v = sum_m h_m(x_A) part[m] and d_A phi . v = sum_m h'_m(x_A) part[m].
template <typename T, int DIM, int K, int A, typename V>
__device__ __forceinline__ T orbital_dot_axis(const T (&hv)[DIM][K], V &&v, T &grad)
{
    T part[K];
#pragma unroll
    for (int m = 0; m < K; ++m) part[m] = T(0);
    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
        const int mc[3] = {m0, m1, m2};
        T f = T(1);
#pragma unroll
        for (int c = 0; c < DIM; ++c)
            if (c != A) f = (c == (A == 0 ? 1 : 0)) ? hv[c][mc[c]] : f * hv[c][mc[c]];
        part[mc[A]] += f * v(o);
    });
    T s = T(0), g = T(0);
#pragma unroll
    for (int m = 0; m < K; ++m) s += hv[A][m] * part[m];
#pragma unroll
    for (int m = 1; m < K; ++m) g += hC<T>(m) * hv[A][m - 1] * part[m];
    grad = g;
    return s;
}

// orbital_dot_axis with the axis chosen at run time (a warp-uniform branch).
template <typename T, int DIM, int K, typename V>
__device__ __forceinline__ T orbital_dot_grad(const T (&hv)[DIM][K], V &&v, int axis, T &grad)
{
    if (axis == 0) return orbital_dot_axis<T, DIM, K, 0>(hv, v, grad);
    if (DIM == 2 || axis == 1) return orbital_dot_axis<T, DIM, K, (DIM > 1 ? 1 : 0)>(hv, v, grad);
    return orbital_dot_axis<T, DIM, K, DIM - 1>(hv, v, grad);
}

// Per-degree partial sums of the derivative vectors: orbital o = (m0, m1, m2) with
// inverse entry v adds, for each dimension c, prod_{c' != c} h_{m_c'} * v to
// part[c][m_c].
template <typename T, int DIM, int K>
__device__ __forceinline__ void accumulate_orbital(const T (&hv)[DIM][K], T (&part)[DIM][K], T v,
                                                   int m0, int m1, int m2)
{
    if (DIM == 2) {
        part[0][m0] += hv[1][m1] * v;
        part[1][m1] += hv[0][m0] * v;
    } else {
        part[0][m0] += (hv[1][m1] * hv[DIM - 1][m2]) * v;
        part[1][m1] += (hv[0][m0] * hv[DIM - 1][m2]) * v;
        part[DIM - 1][m2] += (hv[0][m0] * hv[1][m1]) * v;
    }
}

// d_c phi . v = sum_m h'_m(x_c) part[c][m],  d_c^2 phi . v = sum_m h''_m(x_c) part[c][m]
template <typename T, int DIM, int K>
__device__ __forceinline__ void contract_orbitals(const T (&hv)[DIM][K], const T (&part)[DIM][K],
                                                  T (&gd)[DIM], T (&sd)[DIM])
{
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        T g = T(0), s2 = T(0);
#pragma unroll
        for (int m = 1; m < K; ++m) g += hC<T>(m) * hv[c][m - 1] * part[c][m];
#pragma unroll
        for (int m = 2; m < K; ++m) s2 += hE<T>(m) * hv[c][m - 2] * part[c][m];
        gd[c] = g;
        sd[c] = s2;
    }
}

// d_c phi(r) . v and d_c^2 phi(r) . v for every dimension c.
template <typename T, int DIM, int K, typename V>
__device__ __forceinline__ void orbital_derivs(const T (&hv)[DIM][K], V &&vf, T (&gd)[DIM],
                                               T (&sd)[DIM])
{
    T part[DIM][K];
#pragma unroll
    for (int c = 0; c < DIM; ++c)
#pragma unroll
        for (int m = 0; m < K; ++m) part[c][m] = T(0);
    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
        accumulate_orbital<T, DIM, K>(hv, part, vf(o), m0, m1, m2);
    });
    contract_orbitals<T, DIM, K>(hv, part, gd, sd);
}

// 16-byte shared-memory vector of 4 floats or 2 doubles
template <typename T>
__device__ __forceinline__ void vload(const T *p, T *out)
{
    if constexpr (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
    } else {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        out[0] = v.x; out[1] = v.y;
    }
}

template <typename T>
__device__ __forceinline__ void vstore(T *p, const T *in)
{
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(in[0], in[1], in[2], in[3]);
    } else {
        *reinterpret_cast<double2 *>(p) = make_double2(in[0], in[1]);
    }
}

// Coordinates of particle j (2D: one 8- or 16-byte load, no bank conflicts).
template <typename T, int DIM>
__device__ __forceinline__ void load_coords(const T *x, int j, T (&out)[DIM])
{
    if constexpr (DIM == 2) {
        using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
        const V v = reinterpret_cast<const V *>(x)[j];
        out[0] = v.x;
        out[1] = v.y;
    } else {
#pragma unroll
        for (int c = 0; c < DIM; ++c) out[c] = x[j * DIM + c];
    }
}

template <typename T, int DIM>
__device__ __forceinline__ void store_coords(T *x, int j, const T (&in)[DIM])
{
    if constexpr (DIM == 2) {
        using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
        V v;
        v.x = in[0];
        v.y = in[1];
        reinterpret_cast<V *>(x)[j] = v;
    } else {
#pragma unroll
        for (int c = 0; c < DIM; ++c) x[j * DIM + c] = in[c];
    }
}

// Reduce-scatter of 8 per-lane values over a segment of SEG lanes (the warp, or
// half of it when a warp carries two walkers): an xor butterfly that halves the
// value set at each stage returns, in segment lane L, the segment total of value
// L / (SEG / 8).  9 shuffles instead of 40 for eight all-reduces over a warp.
template <typename R, int SEG = 32>
__device__ __forceinline__ R warp_reduce_scatter8(const R (&v)[8], int lane)
{
    const bool h4 = lane & (SEG / 2);
    R w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const R mine = h4 ? v[4 + i] : v[i];
        const R other = h4 ? v[i] : v[4 + i];
        w[i] = mine + __shfl_xor_sync(FULL, other, SEG / 2);
    }
    const bool h3 = lane & (SEG / 4);
    R u[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const R mine = h3 ? w[2 + i] : w[i];
        const R other = h3 ? w[i] : w[2 + i];
        u[i] = mine + __shfl_xor_sync(FULL, other, SEG / 4);
    }
    const bool h2 = lane & (SEG / 8);
    R t = (h2 ? u[1] : u[0]) + __shfl_xor_sync(FULL, h2 ? u[0] : u[1], SEG / 8);
#pragma unroll
    for (int o = SEG / 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
    return t;
}

// Sum over a segment of SEG lanes (every lane of the segment gets the total).
template <int SEG, typename R>
__device__ __forceinline__ R seg_sum(R v)
{
#pragma unroll
    for (int o = SEG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// A register-resident inverse (each lane keeping its two rows in registers) was
// measured with ptxas at N = 56: the two 28-entry rows plus the step's working set
// need more than 200 registers per thread and spill, so rows stay in shared memory.

// The sweep of walkers w_first, w_first + w_stride, ... < w_end by the calling warp
// (steps step_offset .. step_offset + steps - 1 of the iteration), whose slice of
// shared memory starts at warp_smem.  The single-system kernel below
// strides over its whole population; the multi-system kernel hands each warp the
// walkers of one work item.
//
// G walkers per warp: G = 2 (4) splits the warp into 16-lane (8-lane) segments,
// segment s sweeping walker w + s of each group (its record at warp_smem +
// s * seg_stride), for the dots up to N = 30 (G = 2: at most 15 orbitals per block,
// one row per lane, partners in two passes above 16; G = 4: N <= 6, with two
// accumulator slots per lane for the 15 accumulators), which would leave much of a
// 32-lane warp idle.  The walkers step in
// lockstep; every shuffle stays inside a segment, and a segment whose walker does not
// exist (a population that is not a multiple of G) replays the group's first walker
// on its own shared memory and writes nothing back.
template <typename T, int DIM, int K, int FX, bool PL, int G = 1>
__device__ __forceinline__ void sweep_walkers(const SweepArgs &a, int steps, int step_offset,
                                              unsigned char *warp_smem, int w_first, int w_end, int w_stride,
                                              MlpCtx *mctx = nullptr, int seg_stride = 0)
{
    static_assert(G == 1 || (PL && FX != 0 && FX != FX_MLP_DOT && K > 0 && (G == 2 || (G == 4 && K <= 2))),
                  "several walkers per warp: production dot sweeps (G = 4: at most 3 orbitals per block)");
    constexpr int SEG = 32 / G;        // lanes per walker
    constexpr int VL = SEG / 8;        // lanes per reduce-scatter value
    constexpr int NSLOT = G == 4 ? 2 : 1;  // accumulator slots per lane (slot lane + SEG i)
    // the MLP Jastrow dot: the CTA's warps step in lockstep (one tensor-core layer per step)
    constexpr bool MLPJ = FX == FX_MLP_DOT;
    // PL: the production form (Philox numbers, no probe, no recording), with the
    // branches of the test and replay modes compiled out
    const int *const probe_k = PL ? nullptr : a.probe_k;
    const double *const replay = PL ? nullptr : a.replay;
    double *const rec_en = PL ? nullptr : a.rec_en;
    unsigned char *const rec_acc = PL ? nullptr : a.rec_acc;
    using F = Fast<T>;
    constexpr int NO = K > 0 ? Shells<DIM, K>::n : 0;
    constexpr int NK = 2 * NO;                  // particles when the Slater fixes N
    constexpr int DK = NK * DIM;                // coordinates when the Slater fixes N
    constexpr int VE = 16 / (int)sizeof(T);                     // entries per 16-byte vector
    constexpr int IS = K > 0 ? inv_row_stride(NO, sizeof(T)) : 0; // inverse row stride
    constexpr int NQ = (NO + VE - 1) / VE;                        // vectors per inverse row
    constexpr int RP = K > 0 ? (NO + 32 / G - 1) / (32 / G) : 1;  // inverse rows per lane
    const Params &P = a.P;
    const Layout L = P.L;
    const int lane = threadIdx.x & (SEG - 1);   // lane within the walker's segment
    const int seg = (threadIdx.x & 31) / SEG;
    const unsigned segmask = G == 1 ? FULL : (((1u << SEG) - 1u) << (SEG * seg));
    T *sm = reinterpret_cast<T *>(warp_smem + (size_t)seg * seg_stride);
    const int N = K > 0 ? NK : P.N;
    const int D = K > 0 ? DK : L.D;
    unsigned long long *smask = reinterpret_cast<unsigned long long *>(sm + L.rec);
    double *ssc = reinterpret_cast<double *>(smask + N);
    T *x = sm + L.off_x, *fc = sm + L.off_fc, *dd = sm + L.off_dd, *sdd = sm + L.off_sdd;
    T *gj = sm + L.off_gj, *inv = sm + L.off_inv;
    const int flags = FX ? FX : P.flags;
    const bool is = flags & F_IS;
    const int jas = flags & (F_PADE | F_MLP);  // a pair Jastrow with gradient vector gj and Laplacian sum
    const int wib_l = threadIdx.x >> 5;
    bool tc_fail = false;

    // accumulator slots of this lane (lane + SEG i): 0..7 energy moments, 8 accepts,
    // then the parameter gradients (kind 1 alpha, 2 gamma, 3 hydrogen-like alpha)
    // and the same times E_L.
    int pkind[NSLOT];
    bool times_e[NSLOT];
#pragma unroll
    for (int i = 0; i < NSLOT; ++i) {
        const int slot = lane + SEG * i;
        pkind[i] = 0;
        times_e[i] = false;
        if (slot >= 9 && slot < P.nacc) {
            int j = slot - 9;
            times_e[i] = j >= P.ep;
            if (times_e[i]) j -= P.ep;
            pkind[i] = j == P.idx_alpha ? 1 : j == P.idx_gamma ? 2 : j == P.idx_alpha_h ? 3 : 0;
        }
    }

    for (int w0 = w_first; MLPJ ? (w0 - wib_l < w_end) : (w0 < w_end); w0 += w_stride) {
        const bool wact = G == 1 || w0 + seg < w_end;  // this segment has a walker to write back
        const int w = G == 1 ? w0 : (wact ? w0 + seg : w0);
        if constexpr (MLPJ) {
            if (w >= w_end || tc_fail) {  // no walker for this warp: join the CTA's tensor-core steps
                for (int s = 0; s < steps && !tc_fail; ++s) {
                    const unsigned st = tc_pair_layer(*mctx->tc, mctx->w, false, 0.0f, 0.0f, 0.0f, lane, wib_l, mctx->pre);
                    tc_fail = __syncthreads_or(st != 0u);
                }
                continue;
            }
        }
        T *g_rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
        {
            const int nv = L.rec * (int)sizeof(T) / 16;
            const uint4 *s4 = reinterpret_cast<const uint4 *>(g_rec);
            uint4 *d4 = reinterpret_cast<uint4 *>(sm);
            for (int i = lane; i < nv; i += SEG) d4[i] = s4[i];
        }
        for (int j = lane; j < N; j += SEG) smask[j] = P.mask[(size_t)w * N + j];
        if (lane < NSCAL) ssc[lane] = P.scal[(size_t)w * NSCAL + lane];
        double acc_s[NSLOT], acc_c[NSLOT];
#pragma unroll
        for (int i = 0; i < NSLOT; ++i) {
            const int slot = lane + SEG * i;
            acc_s[i] = acc_c[i] = 0.0;
            if (slot < P.nacc) {
                acc_s[i] = P.acc[((size_t)w * P.nacc + slot) * 2];
                acc_c[i] = P.acc[((size_t)w * P.nacc + slot) * 2 + 1];
            }
        }
        unsigned long long ctr = P.counter[w];
        unsigned status = 0;
        int rng_k = 0;        // this lane's step of the current SEG-step random block
        T rng_z = T(0);
        unsigned rng_u = 0u;
        __syncwarp(segmask);

        const bool use_philox = !probe_k && !replay;
        float *mcache = MLPJ ? P.mlp_cache + (size_t)w * P.mlp_cache_stride : nullptr;
        for (int s0 = 0; s0 < steps && !(MLPJ && tc_fail); s0 += SEG) {
          if (use_philox) {
            // Lane-parallel Philox: lane i draws the numbers of step counter ctr + i
            // (the same per-step stream as a serial draw); each step of this block
            // takes its triple from lane (step - s0) by shuffle.
            const unsigned long long c = ctr + (unsigned long long)lane;
            const uint4 v = philox(make_uint4((uint32_t)c, (uint32_t)(c >> 32), (uint32_t)(w + P.walker_offset), 0u),
                                   make_uint2((uint32_t)a.seed, (uint32_t)(a.seed >> 32)));
            rng_k = (int)__umulhi(v.x, (unsigned)D);
            if (is) {
                if (sizeof(T) == 8) {
                    const double u1 = ((double)v.y + 1.0) * TWO_M32, u2 = v.z * TWO_M32;
                    rng_z = T(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
                } else {
                    const float u1 = ((float)v.y + 1.0f) * 2.3283064e-10f;
                    const float u2 = (float)v.z * 2.3283064e-10f;
                    rng_z = T(sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2));
                }
            } else {
                rng_z = T(v.y * TWO_M32);
            }
            rng_u = v.w;
          }
          const int s_end = min(s0 + SEG, steps);
          for (int s = s0; s < s_end && !(MLPJ && tc_fail); ++s) {
            const int it_step = step_offset + s;
            const T wa = T(P.omega * P.alpha);
            // ---- 1. random numbers and the proposal
            int k;
            T r1;
            double r2;
            if (probe_k) {
                k = probe_k[w];
                r1 = T(0);
                r2 = 0.0;
            } else if (replay) {
                const double *q = replay + ((size_t)w * a.replay_stride + a.replay_offset + it_step) * 3;
                k = (int)floor(q[0] * D);
                r1 = T(q[1]);
                r2 = q[2];
            } else {
                const int slot = (s - s0) & (SEG - 1);  // s - s0 < SEG (the mask frees a register)
                ++ctr;
                k = __shfl_sync(FULL, rng_k, slot, SEG);
                r1 = __shfl_sync(FULL, rng_z, slot, SEG);
                r2 = __shfl_sync(FULL, rng_u, slot, SEG) * TWO_M32;
            }
            const int p = k / DIM, adim = k - p * DIM;
            const T xo = x[k];
            T Gk = T(0);
            if (flags & F_GAUSS) Gk += -wa * xo;
            if (K > 0) Gk += dd[k];
            if (jas) Gk += gj[k];
            T rpo = T(0);
            if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                T r2s = T(0);
#pragma unroll
                for (int c = 0; c < DIM; ++c) r2s += x[p * DIM + c] * x[p * DIM + c];
                rpo = r2s * F::rsqrt(r2s);
                if (flags & F_HYDROGENLIKE) Gk += -T(P.alpha_h * P.Z) * xo / rpo;
            }
            T dx, Fn = T(0);
            if (probe_k) {
                dx = T(a.probe_x[w]) - xo;
            } else if (is) {
                // the drift limiter is a corrected-mode option (no cost in the reference form)
                Fn = T(2) * ((flags & Q_IS_GREEN) ? Gk : limited_drift<T>(Gk, P));
                dx = T(0.5 * P.step) * Fn + r1 * T(sqrt(P.step));
            } else {
                dx = T(10) * (r1 - T(0.5)) * T(P.step);
            }
            const T xn = probe_k ? T(a.probe_x[w]) : xo + dx;
            T xpn[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) xpn[c] = (c == adim) ? xn : x[p * DIM + c];

            // ---- 2a. Slater: S_j = phi(r_p') . inv[:, j] for lane j, R = S_pl
            // the corrected Green's ratio needs d ln Psi / d x_k at the proposed point:
            // its Slater part d_adim phi(r_p') . inv[:, p] / R comes out of the same
            // row contraction as R (lane pl)
            const bool green_grad = is && !(flags & Q_IS_GREEN) && !probe_k;
            // rows per lane: lane holds rows lane + SEG rp (more than one only when a
            // segment is narrower than a Slater block)
            T Sj[RP], R = T(1), Gs = T(0);
            int b = 0, pl = 0;
#pragma unroll
            for (int rp = 0; rp < RP; ++rp) Sj[rp] = T(0);
            if constexpr (K > 0) {
                b = p / NO;
                pl = p - b * NO;
                T hv[DIM][K];
#pragma unroll
                for (int c = 0; c < DIM; ++c) hermite_values<K>(xpn[c], hv[c]);
                T Gj[RP], Sp = T(0), Gp = T(0);
#pragma unroll
                for (int rp = 0; rp < RP; ++rp) {
                    const int r = lane + SEG * rp;
                    Gj[rp] = T(0);
                    if (r < NO) {
                        // row r (column r of A^{-1}), 16-byte vector loads
                        T rv[NQ * VE];
                        const T *row = inv + (b * NO + r) * IS;
#pragma unroll
                        for (int q = 0; q < NQ; ++q) vload<T>(row + q * VE, rv + q * VE);
                        if (green_grad)
                            Sj[rp] = orbital_dot_grad<T, DIM, K>(hv, [&](int o) { return rv[o]; }, adim, Gj[rp]);
                        else
                            Sj[rp] = orbital_dot<T, DIM, K>(hv, [&](int o) { return rv[o]; });
                    }
                    if (rp == pl / SEG) {
                        Sp = Sj[rp];
                        Gp = Gj[rp];
                    }
                }
                R = __shfl_sync(FULL, Sp, pl & (SEG - 1), SEG);
                if (green_grad) Gs = __shfl_sync(FULL, Gp, pl & (SEG - 1), SEG);
            }

            // ---- 2b. pair terms of the moved particle (Pade, Coulomb)
            constexpr int NJ = K > 0 ? (NK + SEG - 1) / SEG : 2;
            T sum_ratio = T(0), d_lap = T(0), d_bh2 = T(0), d_vint = T(0), pair_total = T(0);
            T gp_new[DIM], gdel[NJ][DIM];
            // Pade pairs keep the previous gamma until one of their particles moves
            // (reference quirk, the pair masks); without the quirk the masks are unused
            const bool stale = flags & Q_PADE_STALE;
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                gp_new[c] = T(0);
#pragma unroll
                for (int jj = 0; jj < NJ; ++jj) gdel[jj][c] = T(0);
            }
            float mlp_un = 0.0f, mlp_dun = 0.0f, mlp_ddun = 0.0f, mlp_cn = 0.0f, mlp_dcn = 0.0f, mlp_ddcn = 0.0f;
            if constexpr (MLPJ) {
                // pair values of the moved particle's partners (lane j; N <= 32): new ones
                // from the network (second layer on the tensor cores, the CTA in lockstep),
                // old ones from the walker's cache
                const int j = lane;
                const bool pv = j < N && j != p;
                float dvo[DIM], dvn[DIM], r2o = 0.0f, r2n = 0.0f;
#pragma unroll
                for (int c = 0; c < DIM; ++c) {
                    const float xj = pv ? (float)x[j * DIM + c] : 0.0f;
                    const float xp = (float)((c == adim) ? xo : xpn[c]);
                    dvo[c] = xp - xj;
                    dvn[c] = (float)xpn[c] - xj;
                    r2o = fmaf(dvo[c], dvo[c], r2o);
                    r2n = fmaf(dvn[c], dvn[c], r2n);
                }
                const float iro = pv ? approx_rsqrt(r2o) : 0.0f, irn = pv ? approx_rsqrt(r2n) : 0.0f;
                const bool same = same_spin(p, j, N);
                const unsigned tst = tc_pair_layer(*mctx->tc, mctx->w, pv, r2n * irn, same ? 1.0f : 0.0f,
                                                   mlp_cusp(DIM, same), lane, wib_l, mctx->pre);
                tc_fail = __syncthreads_or(tst != 0u);
                if (tc_fail) break;
                if (pv) {
                    mlp_un = mctx->pre[lane];
                    mlp_dun = mctx->pre[32 + lane];
                    mlp_ddun = mctx->pre[64 + lane];
                    const float *co = mcache + (size_t)(p * N + j) * 3;
                    const float uo = co[0], duo = co[1], dduo = co[2];
                    sum_ratio = T(mlp_un - uo);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) {
                        gp_new[c] = T(mlp_dun * dvn[c] * irn);
                        gdel[0][c] = T(duo * dvo[c] * iro - mlp_dun * dvn[c] * irn);
                    }
                    d_lap = T(2.0f * ((mlp_ddun + (DIM - 1) * mlp_dun * irn) - (dduo + (DIM - 1) * duo * iro)));
                    d_vint = T(irn - iro);
                }
                // one-body term of the moved particle (lanes over the 32 hidden units)
                float rp2n = 0.0f, rp2o = 0.0f;
#pragma unroll
                for (int c = 0; c < DIM; ++c) {
                    const float xp = (float)((c == adim) ? xo : xpn[c]);
                    rp2n = fmaf((float)xpn[c], (float)xpn[c], rp2n);
                    rp2o = fmaf(xp, xp, rp2o);
                }
                const float rpn1 = sqrtf(rp2n), rpo1 = sqrtf(rp2o);
                mlp_body(mctx->w, mctx->w + MW_W2T, rpn1, lane, mlp_cn, mlp_dcn, mlp_ddcn);
                if (lane == 0) {
                    const float *oc = mcache + (size_t)N * N * 3 + p * 3;
                    sum_ratio += T(mlp_cn - oc[0]);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) gp_new[c] += T(mlp_dcn * (float)xpn[c] / rpn1);
                    d_lap += T((mlp_ddcn + (DIM - 1) * mlp_dcn / rpn1) - (oc[2] + (DIM - 1) * oc[1] / rpo1));
                }
                T vals[8] = {sum_ratio, d_lap, T(0), d_vint, T(0), T(0), T(0), T(0)};
#pragma unroll
                for (int c = 0; c < DIM; ++c) vals[4 + c] = gp_new[c];
                pair_total = warp_reduce_scatter8<T, SEG>(vals, lane);
                sum_ratio = __shfl_sync(FULL, pair_total, 0, SEG);
            } else if (flags & (F_PADE | F_COULOMB)) {
                const unsigned long long mp = stale ? smask[p] : ~0ull;
                const T gam = T(P.gamma), gamp = T(P.gamma_prev);
                // old and new position of the moved particle side by side: every pair
                // quantity below is a (before, after) pair computed by packed instructions
                Two<T> xon[DIM];
#pragma unroll
                for (int c = 0; c < DIM; ++c) xon[c] = two((c == adim) ? xo : xpn[c], xpn[c]);
                const Two<T> lap_c = two(T(DIM - 1), T(DIM - 1)), m2gam = two(T(-2) * gam, T(-2) * gam);
#pragma unroll
                for (int jj = 0; jj < NJ; ++jj) {
                    const int j = lane + SEG * jj;
                    if (j < N && j != p) {
                        T xjv[DIM];
                        load_coords<T, DIM>(x, j, xjv);
                        Two<T> dv[DIM], r2 = two(T(0), T(0));
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            dv[c] = add2(xon[c], two(-xjv[c], -xjv[c]));
                            r2 = fma2(dv[c], dv[c], r2);
                        }
                        const Two<T> ir = two(F::rsqrt(r2.x), F::rsqrt(r2.y));
                        if (flags & F_PADE) {
                            const Two<T> r = mul2(r2, ir);
                            const T beta = same_spin(p, j, N) ? T(P.beta_same) : T(P.beta_anti);
                            const T gpair = (stale && !((mp >> j) & 1ull)) ? gamp : gam;
                            const Two<T> den = fma2(two(gpair, gam), r, two(T(1), T(1)));
                            const Two<T> f1 = two(F::rcp(den.x), F::rcp(den.y));
                            const Two<T> h = mul2(r, f1);                              // r / (1 + g r)
                            const Two<T> fi = mul2(mul2(f1, f1), mul2(two(beta, beta), ir));  // beta f1^2 / r
                            if (!(flags & Q_PADE_RATIO) || j > p) sum_ratio += beta * (h.y - h.x);
#pragma unroll
                            for (int c = 0; c < DIM; ++c) {
                                const Two<T> t = mul2(fi, dv[c]);
                                gp_new[c] += t.y;
                                gdel[jj][c] = t.x - t.y;  // particle j sees -(x_p - x_j)
                            }
                            // 2 f (DIM - (1 + 2 gamma h)) / r, new minus old
                            const Two<T> lq = mul2(fi, fma2(m2gam, h, lap_c));
                            d_lap += T(2) * (lq.y - lq.x);
                            const Two<T> hh = mul2(h, h);
                            d_bh2 += beta * (hh.y - hh.x);
                        }
                        if (flags & F_COULOMB) d_vint += ir.y - ir.x;
                    }
                }
                // one reduce-scatter for all pair sums: lane L ends with the total of
                // value L >> 2 (0 ratio exponent, 1 Laplacian, 2 beta h^2, 3 Coulomb,
                // 4.. the moved particle's new Pade gradient)
                T vals[8] = {sum_ratio, d_lap, d_bh2, d_vint, T(0), T(0), T(0), T(0)};
#pragma unroll
                for (int c = 0; c < DIM; ++c) vals[4 + c] = gp_new[c];
                pair_total = warp_reduce_scatter8<T, SEG>(vals, lane);
                sum_ratio = __shfl_sync(FULL, pair_total, 0, SEG);
            }

            // ---- 2c. element ratios, multiplied in configuration order
            T rpn = T(0);
            if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                T r2s = T(0);
#pragma unroll
                for (int c = 0; c < DIM; ++c) r2s += xpn[c] * xpn[c];
                rpn = r2s * F::rsqrt(r2s);
            }
            const T rat_g = (flags & F_GAUSS) ? F::exp(wa * (xo * xo - xn * xn)) : T(1);
            const T rat_p = jas ? F::exp(T(2) * sum_ratio) : T(1);
            const T rat_h = (flags & F_HYDROGENLIKE) ? F::exp(T(2 * P.alpha_h * P.Z) * (rpo - rpn)) : T(1);
            double prob = 1.0;
            if (FX && !probe_k) {
                // compiled-in dot: Slater x Gaussian x Pade (order only affects rounding)
                prob = (double)(R * R) * (double)rat_g * (double)rat_p;
            } else {
                for (int e = 0; e < P.n_elem; ++e) {
                    const int kind = P.elem_kind[e];
                    const T r = kind == 0 ? rat_g : kind == 1 ? R * R : (kind == 2 || kind == 7) ? rat_p
                                : kind == 6 ? rat_h : T(1);
                    prob *= (double)r;
                    if (probe_k && lane == 0) a.probe_ratio[(size_t)w * P.n_elem + e] = (double)r;
                }
            }

            // ---- 2d. accept / reject
            bool accept = true;
            if (!probe_k) {
                double wgt = prob;
                if (is) {
                    if (flags & Q_IS_GREEN) {
                        // importancesampling.cpp:43-47: exp(0.5 (F_old(k) - F_new(k)) dx) + 1
                        const T ex = F::exp(T(0.5) * (fc[k] - Fn) * dx);
                        wgt = ((double)ex + 1.0) * prob;
                    } else {
                        T gy = T(0);
                        if (flags & F_GAUSS) gy += -wa * xn;
                        if (jas) gy += __shfl_sync(FULL, pair_total, VL * (4 + adim), SEG);
                        if (flags & F_HYDROGENLIKE) gy += -T(P.alpha_h * P.Z) * xn / rpn;
                        if constexpr (K > 0) gy += Gs / R;
                        const double fy = 2.0 * (double)limited_drift<T>(gy, P), fo2 = (double)Fn;
                        wgt = prob * exp(0.5 * (fo2 + fy) * (0.25 * P.step * (fo2 - fy) - (double)dx));
                    }
                }
                // the reference rejects when weight < u (bruteforce.cpp:44,
                // importancesampling.cpp:72); a NaN weight (an FP32 overflow of a proposal
                // thrown far out by the drift near a node) is flagged and rejected here
                // instead of accepted
                if (wgt != wgt) status |= ST_BAD_RATIO;
                accept = wgt >= r2;
            }

            if (accept) {
                // ---- 3. state update
                __syncwarp(segmask);
                if (lane == 0) {
                    x[k] = xn;
                    if (is) fc[k] = Fn;
                    ssc[SC_SUMX2] += (double)xn * (double)xn - (double)xo * (double)xo;
                    if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                        ssc[SC_INVR] += 1.0 / (double)rpn - 1.0 / (double)rpo;
                        ssc[SC_SUMR] += (double)rpn - (double)rpo;
                    }
                }
                // owners of the reduced pair sums apply them: value v (lanes VL v ..)
                // 1, 2 -> SC_LAPJ, SC_BH2 (= v); 3 -> SC_VINT (= v); 4 + c -> gj of p
                if ((flags & (F_PADE | F_MLP | F_COULOMB)) && (lane % VL) == 0 && lane >= VL && lane < VL * (4 + DIM)) {
                    const int v = lane / VL;
                    if (v < 4) {
                        if ((v == 3) ? (flags & F_COULOMB) : jas) ssc[v] += (double)pair_total;
                    } else if (jas) {
                        gj[p * DIM + v - 4] = pair_total;
                    }
                }
                if constexpr (MLPJ) {  // the moved particle's pair and one-body values into the cache
                    if (lane < N && lane != p) {
                        float *c1 = mcache + (size_t)(p * N + lane) * 3, *c2 = mcache + (size_t)(lane * N + p) * 3;
                        c1[0] = c2[0] = mlp_un;
                        c1[1] = c2[1] = mlp_dun;
                        c1[2] = c2[2] = mlp_ddun;
                    }
                    if (lane == 0) {
                        float *oc = mcache + (size_t)N * N * 3 + p * 3;
                        oc[0] = mlp_cn;
                        oc[1] = mlp_dcn;
                        oc[2] = mlp_ddcn;
                    }
                }
                if constexpr (K > 0) {
                    // Sherman-Morrison (slaterdeterminant.cpp:165-175) on the rows of
                    // block b, fused with the refresh of the block's derivative vectors
                    // (slaterdeterminant.cpp:155-163): lane j updates row j and feeds
                    // the new entries straight into particle j's d ln det sums.
                    const T rinv = F::rcp(R);  // an accepted move has |R| well above underflow
                    // row j -= (S_j / R) row p for j != p; row p *= 1 / R, written as
                    // row p += (1 / R - 1) row p (exact when 1 / R lies in [0.5, 2]):
                    // one fused multiply-add per entry on every lane
                    __syncwarp(segmask);  // x[k] written by lane 0
                    const T *row_p = inv + (b * NO + pl) * IS;
                    // with several rows per lane the pass holding row p goes last, so
                    // every other row reads row p before it changes
#pragma unroll 1
                    for (int i = 0; i < RP; ++i) {
                        const int rp = RP == 1 ? 0 : (pl / SEG + 1 + i) % RP;
                        const int r = lane + SEG * rp;
                        T s_r = Sj[0];
#pragma unroll
                        for (int q = 1; q < RP; ++q)
                            if (q == rp) s_r = Sj[q];
                        const T tl = (r == pl) ? rinv - T(1) : -(s_r * rinv);
                        const int lr = r < NO ? r : pl;   // rows >= NO shadow row pl, store nothing
                        T *row_j = inv + (b * NO + lr) * IS;
                        T hv[DIM][K];
                        {
                            T xq[DIM];
                            load_coords<T, DIM>(x, b * NO + lr, xq);
#pragma unroll
                            for (int c = 0; c < DIM; ++c) hermite_values<K>(xq[c], hv[c]);
                        }
                        T part[DIM][K];
#pragma unroll
                        for (int c = 0; c < DIM; ++c)
#pragma unroll
                            for (int m = 0; m < K; ++m) part[c][m] = T(0);
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            T cv[VE], vv[VE];
                            vload<T>(row_p + q * VE, cv);   // old row of the moved particle
                            vload<T>(row_j + q * VE, vv);
                            __syncwarp(segmask);            // row p read by all before it changes
#pragma unroll
                            for (int e = 0; e < VE; e += 2) {
                                const Two<T> nv = fma2(two(cv[e], cv[e + 1]), two(tl, tl), two(vv[e], vv[e + 1]));
                                vv[e] = nv.x;
                                vv[e + 1] = nv.y;
                            }
                            if (r < NO) vstore<T>(row_j + q * VE, vv);
                            for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                                if (o / VE == q) accumulate_orbital<T, DIM, K>(hv, part, vv[o % VE], m0, m1, m2);
                            });
                        }
                        if (r < NO) {
                            T gd[DIM], sd[DIM];
                            contract_orbitals<T, DIM, K>(hv, part, gd, sd);
                            store_coords<T, DIM>(dd, b * NO + r, gd);
                            store_coords<T, DIM>(sdd, b * NO + r, sd);
                        }
                    }
                }
                if (jas) {
#pragma unroll
                    for (int jj = 0; jj < NJ; ++jj) {
                        const int j = lane + SEG * jj;
                        if (j < N && j != p) {
                            T gv[DIM];
                            load_coords<T, DIM>(gj, j, gv);
#pragma unroll
                            for (int c = 0; c < DIM; ++c) gv[c] += gdel[jj][c];
                            store_coords<T, DIM>(gj, j, gv);
                            if (stale) smask[j] |= (1ull << p);
                        }
                    }
                    if (stale && lane == (p & (SEG - 1))) smask[p] = ~0ull;
                }
                __syncwarp(segmask);
            }

            // ---- 4. local energy and parameter gradients (Sampler::sample)
            if (it_step >= a.burn_in || rec_en) {
                // per coordinate: (sum_e grad_e)^2 + Slater's d2/det - (d ln det)^2; the
                // Slater-fixed shapes read VW consecutive coordinates per lane
                constexpr int VW = sizeof(T) == 4 ? 4 : 2;
                constexpr bool VEC = K > 0 && DK % VW == 0;
                constexpr int NV = VEC ? DK / VW : 1;
                T ks = T(0);
                auto coord_term = [&](int c, T xc, T g_s, T s_s, T g_j) {
                    T Gc = T(0), lc = T(0);
                    if (flags & F_GAUSS) Gc += -wa * xc;
                    if (K > 0) {
                        Gc += g_s;
                        lc += s_s - g_s * g_s;
                    }
                    if (jas) Gc += g_j;
                    if (flags & F_HYDROGENLIKE) {
                        const int q = c / DIM;
                        T r2s = T(0);
#pragma unroll
                        for (int e2 = 0; e2 < DIM; ++e2) r2s += x[q * DIM + e2] * x[q * DIM + e2];
                        Gc += -T(P.alpha_h * P.Z) * xc * F::rsqrt(r2s);
                    }
                    ks += Gc * Gc + lc;
                };
                if constexpr (VEC) {
                    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
#pragma unroll
                    for (int i = 0; i < (NV + SEG - 1) / SEG; ++i) {
                        const int vi = lane + SEG * i;
                        if (vi < NV) {
                            const V vx = reinterpret_cast<const V *>(x)[vi];
                            const V vd = reinterpret_cast<const V *>(dd)[vi];
                            const V vs = reinterpret_cast<const V *>(sdd)[vi];
                            const V vj = reinterpret_cast<const V *>(gj)[vi];
                            const T *ax = reinterpret_cast<const T *>(&vx), *ad = reinterpret_cast<const T *>(&vd);
                            const T *as = reinterpret_cast<const T *>(&vs), *aj = reinterpret_cast<const T *>(&vj);
                            if (!(flags & F_HYDROGENLIKE)) {
                                // G^2 + s - g^2 = (G - g)(G + g) + s with G - g the
                                // Gaussian + Pade part: coordinates two at a time
                                Two<T> k2 = two(T(0), T(0));
#pragma unroll
                                for (int e = 0; e < VW; e += 2) {
                                    Two<T> A = two(T(0), T(0));
                                    if (flags & F_GAUSS) A = mul2(two(-wa, -wa), two(ax[e], ax[e + 1]));
                                    if (jas) A = add2(A, two(aj[e], aj[e + 1]));
                                    const Two<T> B = fma2(two(T(2), T(2)), two(ad[e], ad[e + 1]), A);
                                    k2 = fma2(A, B, add2(k2, two(as[e], as[e + 1])));
                                }
                                ks += k2.x + k2.y;
                            } else {
#pragma unroll
                                for (int e = 0; e < VW; ++e) coord_term(vi * VW + e, ax[e], ad[e], as[e], aj[e]);
                            }
                        }
                    }
                } else {
                    constexpr int NC = K > 0 ? (DK + SEG - 1) / SEG : 6;
#pragma unroll
                    for (int i = 0; i < NC; ++i) {
                        const int c = lane + SEG * i;
                        if (c < D)
                            coord_term(c, x[c], K > 0 ? dd[c] : T(0), K > 0 ? sdd[c] : T(0),
                                       jas ? gj[c] : T(0));
                    }
                }
                ks = seg_sum<SEG>(ks);
                double lap = (double)ks;
                if (jas) lap += ssc[SC_LAPJ];
                if (flags & F_GAUSS) lap -= P.omega * P.alpha * D;
                if (flags & F_HYDROGENLIKE) lap -= 2.0 * P.alpha_h * P.Z * ssc[SC_INVR];
                const double ekin = -0.5 * lap;
                const double vext = (flags & F_ATOM) ? -P.Z * ssc[SC_INVR]
                                                     : 0.5 * P.omega * P.omega * ssc[SC_SUMX2];
                const double vint = (flags & F_COULOMB) ? ssc[SC_VINT] : 0.0;
                const double el = ekin + vext + vint;
                if (el != el) status |= ST_NAN_ENERGY;
                if (rec_en && lane == 0) {
                    double *o = rec_en + ((size_t)w * a.rec_stride + it_step) * 3;
                    o[0] = ekin;
                    o[1] = vext;
                    o[2] = vint;
                }
                if (it_step >= a.burn_in) {
                    // branch-free slot selection; slots past the accumulators add zero
                    const bool win = it_step > a.win_lo && it_step < a.win_hi;
#pragma unroll
                    for (int i = 0; i < NSLOT; ++i) {
                        const int slot = lane + SEG * i;
                        const int g2 = (slot >> 1) & 3;
                        const double base = g2 == 0 ? el : g2 == 1 ? ekin : g2 == 2 ? vext : vint;
                        const double qe = (slot & 1) ? base * base : base;
                        const double g = pkind[i] == 1 ? -0.5 * P.omega * ssc[SC_SUMX2]
                                       : pkind[i] == 2 ? ((flags & Q_PADE_DGAMMA) ? -0.5 : -1.0) * ssc[SC_BH2]
                                       : pkind[i] == 3 ? -P.Z * ssc[SC_SUMR] : 0.0;
                        const double qp = win ? (times_e[i] ? g * el : g) : 0.0;
                        const double q = slot < 8 ? qe : slot == 8 ? (accept ? 1.0 : 0.0) : qp;
                        kadd(acc_s[i], acc_c[i], q);
                    }
                    if (!PL && a.dens_bins > 0) density_sample<T>(a, x, N, DIM, lane);
                    if constexpr (MLPJ) {
                        // the MLP row's parameter gradient: positions and E_L every
                        // snap_interval steps of the window, for the backward kernel
                        if (win && a.snap_x && (it_step - a.win_lo) % a.snap_interval == 0) {
                            const int slot = (it_step - a.win_lo) / a.snap_interval - a.snap_first;
                            if (slot >= 0 && slot < a.snap_stride) {
                                const size_t base = (size_t)w * a.snap_stride + slot;
                                for (int t = lane; t < D; t += 32) a.snap_x[base * D + t] = (float)x[t];
                                if (lane == 0) a.snap_e[base] = el;
                            }
                        }
                    }
                }
            }
            if (rec_acc && lane == 0) rec_acc[(size_t)w * a.rec_stride + it_step] = accept ? 1 : 0;
          }
        }

        // ---- write the walker back
        __syncwarp(segmask);
        if (MLPJ && tc_fail) status |= ST_TC_TIMEOUT;
#pragma unroll
        for (int o = SEG / 2; o > 0; o >>= 1) status |= __shfl_xor_sync(FULL, status, o);
        if (wact) {
            const int nv = L.rec * (int)sizeof(T) / 16;
            const uint4 *s4 = reinterpret_cast<const uint4 *>(sm);
            uint4 *d4 = reinterpret_cast<uint4 *>(g_rec);
            for (int i = lane; i < nv; i += SEG) d4[i] = s4[i];
            for (int j = lane; j < N; j += SEG) P.mask[(size_t)w * N + j] = smask[j];
            if (lane < NSCAL) P.scal[(size_t)w * NSCAL + lane] = ssc[lane];
            if (lane == 0) P.counter[w] = ctr;
#pragma unroll
            for (int i = 0; i < NSLOT; ++i) {
                const int slot = lane + SEG * i;
                if (slot < P.nacc) {
                    P.acc[((size_t)w * P.nacc + slot) * 2] = acc_s[i];
                    P.acc[((size_t)w * P.nacc + slot) * 2 + 1] = acc_c[i];
                }
            }
            if (lane == 0 && status) P.status[w] |= status;
        }
        __syncwarp(segmask);
    }
}

// G walkers per warp (see sweep_walkers): a.smem_per_warp holds G walker slices.
template <typename T, int DIM, int K, int FX, bool PL, int G = 1>
__global__ void __launch_bounds__(FX == FX_MLP_DOT ? 128 : sizeof(T) == 4 ? 256 : 128, FX == FX_MLP_DOT ? 2 : 3)
    sweep_kernel(const SweepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5;
    if constexpr (FX == FX_MLP_DOT) {
        // shared memory: the MLP weight block | the tensor-core tiles | the warps' walkers
        __shared__ __align__(8) unsigned long long tc_bar;
        __shared__ uint32_t tc_slot;
        __shared__ float tc_pre[4][96];
        float *mw = reinterpret_cast<float *>(smem_raw);
        for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) mw[i] = a.P.mlpw[i];
        for (int i = threadIdx.x; i < MLP_G * MLP_G; i += blockDim.x) mw[MW_W2T + i] = a.P.mlpw[MW_V2T + i];
        TcMlp tc{};
        tc_setup(tc, smem_raw + MLP_FAST_BYTES, mw, a.P.mlpw, &tc_bar, &tc_slot, wib, mw + MW_W2);
        __syncthreads();
        tc_ready(tc, &tc_slot);
        MlpCtx ctx{mw, &tc, tc_pre[wib & 3]};
        sweep_walkers<T, DIM, K, FX, PL>(a, a.steps, a.step_offset,
                                         smem_raw + MLP_FAST_BYTES + TC_SMEM + (size_t)wib * a.smem_per_warp,
                                         blockIdx.x * a.wpb + wib, a.P.W, gridDim.x * a.wpb, &ctx);
        tc_teardown(tc, wib);
    } else {
        sweep_walkers<T, DIM, K, FX, PL, G>(a, a.steps, a.step_offset, smem_raw + (size_t)wib * a.smem_per_warp,
                                            (blockIdx.x * a.wpb + wib) * G, a.P.W, gridDim.x * a.wpb * G, nullptr,
                                            a.smem_per_warp / G);
    }
}

}  // namespace vmc
