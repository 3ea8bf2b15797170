// Production Metropolis sweep of the 2D closed-shell quantum dots with one walker per
// warp (N = 42 and 56; N = 20 and 30 on request: Slater(Hermite) x Gaussian x
// Pade-Jastrow, Coulomb, importance sampling), in the "owner" form: every lane owns two
// particles of its walker.
//
// Lane l < n (n = N / 2 orbitals per spin block) owns particle l (spin up, row l of the
// first inverse block) and particle n + l (spin down, row l of the second block).  For
// those two particles it keeps, in registers, one pair (particle l, particle n + l) per
// coordinate of: the positions, d ln det / dx and the Pade gradient.  The pair terms of a move (the moved particle against both of a lane's
// particles), the Jastrow gradient update and the kinetic energy are therefore packed
// two-wide instructions on register operands.  Shared memory holds what the whole warp
// reads at one index: the inverse blocks and, per coordinate, the position, the drift
// gradient d ln Psi / dx and the importance-sampling force cache of the proposal.
//
// Per step (System::runMetropolisCycles body, src/system.cpp:149-163; the quantities
// are those of the staged sweep in vmc_sweep.cuh, whose comments cite the reference for
// every term):
//   1. k, the normal and the accept uniform from the walker's Philox stream (drawn 32
//      steps at a time, lane-parallel); the drifted proposal of coordinate k;
//   2. the Slater ratio R = sigma_p phi(r_p') . row p (lane l: its row of the moved
//      particle's block), the Pade / Coulomb pair terms of both own particles against the
//      moved one, one reduce-scatter of the pair sums (which also carries the previous
//      step's per-lane kinetic terms, so the kinetic energy costs no reduction of its own);
//   3. accept: Sherman-Morrison through the row scales (below), the block's gradient
//      vectors d ln det / dx recomputed from the updated rows, the Pade gradient, the
//      running sums;
//   4. E_L and dlnPsi/dtheta of every step after burn-in (one step late: the kinetic sum of
//      step s is the total carried by the reduce-scatter of step s + 1).
//
// Staged inverse rows.  Orbitals are reordered in shared memory so that the transposed
// pair (a, b), (b, a) sits in adjacent slots (the diagonal orbitals (a, a) last), and the
// entries are written for the basis hh_m(u) = He_m(u) / m!, u = sqrt(2) x (probabilists'
// Hermite polynomials), whose derivatives are hh'_m = hh_{m-1}: the engine's normalised
// functions are h_m(x) = H_m(x) / sqrt(2^m m!) = sqrt(m!) hh_m(sqrt(2) x), so a staged
// entry is the record's entry times sqrt(m0! m1!), a column scaling of the Slater matrix
// under which ratios and derivative vectors are unchanged.  Each row also carries a scale
// sigma (true row = sigma x staged row): an accepted move divides the moved particle's
// row by R through its sigma alone, so the rank-1 pass updates every other row from a
// row that nobody writes (no warp barrier between the reads and the writes).
//
// Laplacian of the determinants.  The kinetic energy needs only the sum over particles of
// (d^2 det / dx^2) / det, and for Hermite orbitals that sum follows from the gradients:
// with u = sqrt(2) x, hh_m'' = u hh_m' - m hh_m (He_m'' - u He_m' + m He_m = 0), so
//   (d^2 det / dx_j^2) / det = 2 x_j d ln det / dx_j - 2 sum_i m0_i phi_i(r_j) Binv_ij
// and summed over the particles of a block (sum_j phi_i(r_j) Binv_ij = 1) the second
// terms give 2 sum_i (m0_i + m1_i), twice the sum of the occupied shells.  Each lane adds
// 2 x.d ln det / dx minus its share of that constant, 4 (K - 1) / 3 per particle; the
// per-particle second derivatives are written to the walker record once, at the end.
//
// Sums.  The running pair sums (Pade Laplacian, sum beta h^2, Coulomb) and sum x^2 are
// FP64 per walker.  In the FP32 form the per-step changes go to FP32 partial sums that
// are added to the FP64 values every 32 steps.  Its samples are taken 32 steps at a
// time: every step leaves in shared memory its kinetic sum, the partial sums' values and
// its accept / window / after-burn-in bits (three stores by single lanes), and every 32
// steps lane i evaluates step i's energies and gradients, shifted by the walker's values
// at the start of the launch, the warp sums the twelve moments, and each lane folds the
// one of its accumulator slot into its FP64 Neumaier accumulator.  The FP64 form adds to
// the FP64 sums and accumulators every step, as the staged sweep does.
#pragma once

namespace vmc {

// Orbital order of the staged inverse rows: slot 2q holds orbital (b, a) and slot 2q + 1
// orbital (a, b) of the q-th transposed pair (a < b, a + b < K, by b then a); the
// diagonal orbitals (d, d), 2d < K, follow.  (m0, m1) are the degrees along (x, y), so a
// slot pair times (hh_b(x), hh_b(y)) gives the two orbitals' partial sums over the
// larger index without exchanging the halves of a packed register pair.  Per slot: the Hermite degrees along x (m0)
// and y (m1), the orbital's index in the record (the reference's order: shell s = m0 + m1,
// then m1) and the staging scale sqrt(m0! m1!).
struct PairTable {
    int m0[32], m1[32], orb[32];
    double scale[32];
    int np;  // transposed pairs (slots 0 .. 2 np - 1)
};

__host__ __device__ constexpr double owner_factorial(int m) { return m <= 1 ? 1.0 : m * owner_factorial(m - 1); }
// square root by Newton's iteration (compile-time staging scales)
__host__ __device__ constexpr double owner_sqrt(double v)
{
    double r = v > 1.0 ? v : 1.0;
    for (int i = 0; i < 64; ++i) r = 0.5 * (r + v / r);
    return r;
}

template <int K> __host__ __device__ constexpr PairTable make_pair_table()
{
    PairTable t{};
    int i = 0;
    for (int b = 1; b < K; ++b)
        for (int a = 0; a < b && a + b < K; ++a) {
            t.m0[i] = b;
            t.m1[i] = a;
            t.m0[i + 1] = a;
            t.m1[i + 1] = b;
            i += 2;
        }
    t.np = i / 2;
    for (int d = 0; 2 * d < K; ++d) {
        t.m0[i] = d;
        t.m1[i] = d;
        ++i;
    }
    for (int j = 0; j < i; ++j) {
        const int s = t.m0[j] + t.m1[j];
        t.orb[j] = s * (s + 1) / 2 + t.m1[j];
        t.scale[j] = owner_sqrt(owner_factorial(t.m0[j]) * owner_factorial(t.m1[j]));
    }
    return t;
}

template <typename T> __device__ __forceinline__ T fmaT(T a, T b, T c);
template <> __device__ __forceinline__ float fmaT<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <> __device__ __forceinline__ double fmaT<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

// hh_0..hh_{K-1} at u: hh_{m+1} = (u hh_m - hh_{m-1}) / (m + 1)
template <int K, typename T>
__device__ __forceinline__ void hermite_pe(T u, T (&h)[K])
{
    h[0] = T(1);
    if (K > 1) h[1] = u;
#pragma unroll
    for (int m = 1; m + 1 < K; ++m) h[m + 1] = (u * h[m] - h[m - 1]) * T(1.0 / (m + 1));
}

// hh_0..hh_{K-1} at both coordinates of U: H[m] = (hh_m(U.x), hh_m(U.y))
template <int K, typename T>
__device__ __forceinline__ void hermite_pe2(Two<T> U, Two<T> (&H)[K])
{
    H[0] = two(T(1), T(1));
    if (K > 1) H[1] = U;
#pragma unroll
    for (int m = 1; m + 1 < K; ++m) {
        const T c = T(1.0 / (m + 1));
        H[m + 1] = mul2(fma2(U, H[m], two(-H[m - 1].x, -H[m - 1].y)), two(c, c));
    }
}

template <typename T> __device__ __forceinline__ T oconst(const SweepArgs &a, int i);
template <> __device__ __forceinline__ float oconst<float>(const SweepArgs &a, int i) { return a.ocf[i]; }
template <> __device__ __forceinline__ double oconst<double>(const SweepArgs &a, int i) { return a.oc[i]; }

#ifndef OWNER_PACK_DOT
#define OWNER_PACK_DOT 1
#endif
#ifndef OWNER_PACK_ACC
#define OWNER_PACK_ACC 1
#endif
#ifndef OWNER_SHM64
#define OWNER_SHM64 1
#endif

// One walker (warp) per CTA, and the register budget of 20 resident warps per SM for
// the FP32 form (5 per scheduler: 102 registers, 94 used without spills) and 12 for the
// FP64 form.  The register file is split between the four schedulers, so occupancy
// moves in steps of four warps; against 4-warp CTAs at 16 warps (128 registers), 20
// one-warp CTAs ran the N = 56 sweep 11 % faster (1.62 against 1.46 x 10^9 walker-moves/s;
// 4-warp CTAs at 96 or 80 registers spilled and ran at 1.47 and 1.13).  Shared memory:
// 20 x (8.6 KB + the 1 KB every CTA reserves) for the FP32 form at N = 56.
#ifndef OWNER_WALKERS_PER_CTA
#define OWNER_WALKERS_PER_CTA 1
#endif
constexpr int OWNER_WPB = OWNER_WALKERS_PER_CTA;  // walkers (warps) per CTA
// CTAs per SM each form is compiled for (register budget: 65536 / (32 OWNER_WPB x this))
#ifndef OWNER_MIN_CTAS_F32
#define OWNER_MIN_CTAS_F32 20
#endif
#ifndef OWNER_MIN_CTAS_F64
#define OWNER_MIN_CTAS_F64 12
#endif

// FP64 values of the FP32 form that only the 32-step folds touch, kept in shared memory:
// the lanes' accumulators (sums, compensations), the walker's running sums and energies
// at the start of the launch
constexpr int OWNER_FOLD_DOUBLES = 72;
enum : int { OF_ACCS = 0, OF_ACCC = 32, OF_LAPJ = 64, OF_BH2, OF_VINT, OF_SUMX2, OF_T0, OF_V0, OF_I0, OF_E0 };

// Per step of a 32-step block, FP32 form: the partial sums (lap, sum x^2, V_int,
// sum beta h^2) after the step, its kinetic sum and its bits
constexpr int OWNER_STEP_BYTES = 16 + 4 + 4;
enum : unsigned { SB_ACCEPT = 1u, SB_WINDOW = 2u, SB_SAMPLED = 4u };

// Shared bytes per warp: the inverse blocks, then per coordinate the positions, drift
// gradients and force cache, then the Pade pair masks, the fold values and (FP32) the
// 32-step sample buffer.
__host__ __device__ constexpr int owner_smem_per_warp(int K, int elem_bytes)
{
    const int n = K * (K + 1) / 2, D = 4 * n;
    return (2 * n * inv_row_stride(n, elem_bytes) + 3 * D) * elem_bytes + 2 * n * 8 + OWNER_FOLD_DOUBLES * 8 +
           (elem_bytes == 4 ? 32 * OWNER_STEP_BYTES : 0);
}

// Steps step_offset .. step_offset + steps - 1 of walkers w0, w0 + w_stride, ... < w_end
// by the calling warp, whose owner_smem_per_warp bytes of shared memory start at ws.
// The sweep kernel below runs it over a launch's walkers; the multi-system batch kernel
// over a work item's.
// LIMIT: the corrected mode's drift limiter (P.drift_limit > 0) compiled in; the callers
// pick the instance per launch, so the default sweep carries none of it.
template <typename T, int K, int FX, bool LIMIT = false>
__device__ __forceinline__ void owner_sweep_walkers(const SweepArgs &a, int steps, int step_offset, unsigned char *ws,
                                                    int w0, int w_end, int w_stride)
{
    constexpr PairTable PO = make_pair_table<K>();
    using T2 = Two<T>;
    using Fs = Fast<T>;
    constexpr int n = K * (K + 1) / 2, N = 2 * n, D = 2 * N;
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr int IS = inv_row_stride(n, (int)sizeof(T));
    constexpr int NQ = (n + VE - 1) / VE;
    constexpr bool F32 = sizeof(T) == 4;
    constexpr bool GREEN_Q = (FX & Q_IS_GREEN) != 0;
    constexpr bool STALE = (FX & Q_PADE_STALE) != 0;
    constexpr bool RATIO_Q = (FX & Q_PADE_RATIO) != 0;
    static_assert(n <= 32 && (FX & F_IS) && (FX & F_PADE) && (FX & F_COULOMB) && (FX & F_GAUSS) &&
                      (FX & F_SLATER) && !(FX & (F_ATOM | F_HYDROGENLIKE | F_MLP)),
                  "the owner sweep covers the 2D closed-shell dots with Pade and Coulomb");

    const Params &P = a.P;
    const Layout L = P.L;
    const int l = threadIdx.x & 31;
    const bool own = l < n;
    const int lc = own ? l : n - 1;  // lanes without particles shadow the last row and store nothing
    T *inv = reinterpret_cast<T *>(ws);
    T *xs = inv + 2 * n * IS, *gs = xs + D, *fcs = gs + D;
    unsigned long long *msk = reinterpret_cast<unsigned long long *>(fcs + D);
    double *fd = reinterpret_cast<double *>(msk + N);  // fold values (OF_*)
    // FP32 form: the block's per-step records
    float4 *sbd = reinterpret_cast<float4 *>(fd + OWNER_FOLD_DOUBLES);
    float *sbk = reinterpret_cast<float *>(sbd + 32);
    unsigned *sbf = reinterpret_cast<unsigned *>(sbk + 32);

    constexpr bool SHM = F32 && OWNER_SHM64;
    const T wa = oconst<T>(a, OC_WA), hdt = oconst<T>(a, OC_HDT), sdt = oconst<T>(a, OC_SDT);
    const T gam = oconst<T>(a, OC_GAM), gamp = oconst<T>(a, OC_GAMP);
    const T bsame = oconst<T>(a, OC_BSAME), banti = oconst<T>(a, OC_BANTI);
    const T2 gam2 = two(gam, gam), m2gam = two(oconst<T>(a, OC_M2GAM), oconst<T>(a, OC_M2GAM));
    const T2 one2 = two(T(1), T(1)), mwa2 = two(-wa, -wa);
    const T sq2 = T(1.4142135623730951);
    const double dgk = a.oc[OC_DGK], lapc = a.oc[OC_LAPC], w2h = a.oc[OC_W2H];
    // accumulator slot of this lane: 0..7 energy moments, 8 accepts, then the parameter
    // gradients (1 alpha, 2 gamma) and the same times E_L
    int pk = 0;
    bool te = false;
    if (l >= 9 && l < P.nacc) {
        int j = l - 9;
        te = j >= P.ep;
        if (te) j -= P.ep;
        pk = j == P.idx_alpha ? 1 : j == P.idx_gamma ? 2 : 0;
    }
    const int eg = (l >> 1) & 3;  // energy slots: 0 E, 1 T, 2 V_ext, 3 V_int

    for (int w = w0; w < w_end; w += w_stride) {
        T *rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
        // ---- stage the walker: inverse rows reordered and rescaled, own particles' arrays
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const T *src = rec + L.off_inv + (size_t)(h * n + lc) * L.inv_stride;
            T *dst = inv + (h * n + lc) * IS;
            T v[IS];
#pragma unroll
            for (int i = 0; i < IS; ++i) v[i] = i < n ? src[PO.orb[i < n ? i : 0]] * T(PO.scale[i < n ? i : 0]) : T(0);
            if (own)
#pragma unroll
                for (int q = 0; q < IS / VE; ++q) vstore<T>(dst + q * VE, v + q * VE);
        }
        T2 X[2], DD[2], GJ[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int ka = 2 * lc + c, kb = 2 * (n + lc) + c;
            const T z = T(0);
            X[c] = own ? two(rec[L.off_x + ka], rec[L.off_x + kb]) : two(z, z);
            DD[c] = own ? two(rec[L.off_dd + ka], rec[L.off_dd + kb]) : two(z, z);
            GJ[c] = own ? two(rec[L.off_gj + ka], rec[L.off_gj + kb]) : two(z, z);
        }
        for (int i = l; i < D; i += 32) {
            xs[i] = rec[L.off_x + i];
            fcs[i] = rec[L.off_fc + i];
        }
        // Pade pairs keep the previous gamma until one of their particles moves (the
        // reference quirk); once every particle of the walker has moved, all pairs are
        // current and the masks are left alone
        bool allcur = true, mdirty = false;
        if constexpr (STALE) {
            if (P.gamma != P.gamma_prev) {
                const unsigned long long *gm = P.mask + (size_t)w * N;
                for (int j = l; j < N; j += 32) msk[j] = gm[j];
                const unsigned long long mm = own ? (gm[l] & gm[n + l]) : ~0ull;
                allcur = __all_sync(FULL, mm == ~0ull);
                mdirty = !allcur;
            }
        }
        const double *sc = P.scal + (size_t)w * NSCAL;
        double sumx2 = sc[SC_SUMX2], lapj = sc[SC_LAPJ], bh2 = sc[SC_BH2], vint = sc[SC_VINT];
        T2 SIG = two(T(1), T(1));

        // drift gradient G = -omega alpha x + d ln det + Pade gradient of the own particles
        // into shared memory, and this lane's kinetic terms: G^2 - dd^2 + the determinants'
        // Laplacian as 2 x dd - 4 (K - 1) / 3 per particle (the Hermite identity above)
        const T shell_share = T(4.0 * (K - 1) / 3.0);
        const T2 kc2 = own ? two(-shell_share, -shell_share) : two(T(0), T(0));
        const T2 two2 = two(T(2), T(2));
        auto publish = [&]() -> T {
            T2 k2 = kc2;
            T2 G[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                G[c] = fma2(mwa2, X[c], add2(DD[c], GJ[c]));
                k2 = fma2(G[c], G[c], k2);
                k2 = fma2(DD[c], fma2(two2, X[c], two(-DD[c].x, -DD[c].y)), k2);
            }
            if (own) {
                reinterpret_cast<T2 *>(gs)[l] = two(G[0].x, G[1].x);
                reinterpret_cast<T2 *>(gs)[n + l] = two(G[0].y, G[1].y);
            }
            return k2.x + k2.y;
        };
        T kp = publish();  // this lane's kinetic terms after the last update
        const T ks0 = seg_sum<32>(kp);
        __syncwarp();

        double acc_s = 0.0, acc_c = 0.0;
        if (l < P.nacc) {
            acc_s = P.acc[((size_t)w * P.nacc + l) * 2];
            acc_c = P.acc[((size_t)w * P.nacc + l) * 2 + 1];
        }
        // FP32 form: the walker's energies at the start of the launch (the shifts of the
        // per-step samples) and the FP32 parts of the running sums since the last fold
        const double T0 = -0.5 * ((double)ks0 + lapj - lapc), V0 = w2h * sumx2, I0 = vint, E0 = T0 + V0 + I0;
        const double myref = l < 8 ? (eg == 0 ? E0 : eg == 1 ? T0 : eg == 2 ? V0 : I0) : E0;
        T cT = T(0), cV = T(0), cI = T(0), gA = T(0), gG = T(0);  // FP32 shifted bases at the fold
        T dlap = T(0), dbh2 = T(0), dvint = T(0), dsx2 = T(0);    // FP32 changes since the fold
        if constexpr (SHM) {
            if (l == 0) {
                fd[OF_LAPJ] = lapj;
                fd[OF_BH2] = bh2;
                fd[OF_VINT] = vint;
                fd[OF_SUMX2] = sumx2;
                fd[OF_T0] = T0;
                fd[OF_V0] = V0;
                fd[OF_I0] = I0;
                fd[OF_E0] = E0;
            }
            fd[OF_ACCS + l] = acc_s;
            fd[OF_ACCC + l] = acc_c;
            __syncwarp();
        }
        auto fp32_bases = [&]() {
            if constexpr (SHM) {
                cT = T(-0.5 * fd[OF_LAPJ] + 0.5 * lapc - fd[OF_T0]);
                cV = T(w2h * fd[OF_SUMX2] - fd[OF_V0]);
                cI = T(fd[OF_VINT] - fd[OF_I0]);
                gA = T(a.oc[OC_MHOM] * fd[OF_SUMX2]);
                gG = T(dgk * fd[OF_BH2]);
            } else {
                cT = T(-0.5 * lapj + 0.5 * lapc - T0);
                cV = T(w2h * sumx2 - V0);
                cI = T(vint - I0);
                gA = T(a.oc[OC_MHOM] * sumx2);
                gG = T(dgk * bh2);
            }
        };
        unsigned status = 0;
        // the samples of a block's nb steps (FP32 form): lane i evaluates step i from its
        // record, the warp sums (T, V_ext), (V_int, accepts), their squares (T, V_ext),
        // (V_int, E), the windowed parameter gradients (alpha, gamma) and the same times
        // E, and each lane adds its accumulator slot's value
        auto fold = [&](int nb) {
            if constexpr (F32) {
                __syncwarp();
                const unsigned fl = l < nb ? sbf[l] : 0u;
                T2 u_tv = two(T(0), T(0)), u_ia = u_tv, u_tv2 = u_tv, u_ie2 = u_tv, u_g = u_tv, u_eg = u_tv;
                if (fl & SB_SAMPLED) {
                    const float4 d = sbd[l];
                    const T Ts = fmaT(T(-0.5), sbk[l] + d.x, cT);
                    const T Vs = fmaT(oconst<T>(a, OC_W2H), d.y, cV);
                    const T Is = cI + d.z;
                    const T Es = Ts + Vs + Is;
                    const T wf = (fl & SB_WINDOW) ? T(1) : T(0);
                    u_tv = two(Ts, Vs);
                    u_ia = two(Is, (fl & SB_ACCEPT) ? T(1) : T(0));
                    u_tv2 = mul2(u_tv, u_tv);
                    u_ie2 = mul2(two(Is, Es), two(Is, Es));
                    u_g = mul2(two(fmaT(oconst<T>(a, OC_MHOM), d.y, gA), fmaT(oconst<T>(a, OC_DGK), d.w, gG)), two(wf, wf));
                    u_eg = mul2(two(Es, Es), u_g);
                }
                const int ns = __popc(__ballot_sync(FULL, (fl & SB_SAMPLED) != 0u));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    u_tv = add2(u_tv, two(__shfl_xor_sync(FULL, u_tv.x, o), __shfl_xor_sync(FULL, u_tv.y, o)));
                    u_ia = add2(u_ia, two(__shfl_xor_sync(FULL, u_ia.x, o), __shfl_xor_sync(FULL, u_ia.y, o)));
                    u_tv2 = add2(u_tv2, two(__shfl_xor_sync(FULL, u_tv2.x, o), __shfl_xor_sync(FULL, u_tv2.y, o)));
                    u_ie2 = add2(u_ie2, two(__shfl_xor_sync(FULL, u_ie2.x, o), __shfl_xor_sync(FULL, u_ie2.y, o)));
                    u_g = add2(u_g, two(__shfl_xor_sync(FULL, u_g.x, o), __shfl_xor_sync(FULL, u_g.y, o)));
                    u_eg = add2(u_eg, two(__shfl_xor_sync(FULL, u_eg.x, o), __shfl_xor_sync(FULL, u_eg.y, o)));
                }
                // a NaN energy reaches the sum of E^2
                if (u_ie2.y != u_ie2.y) status |= ST_NAN_ENERGY;
                // this lane's slot
                const T lin = eg == 0 ? u_tv.x + u_tv.y + u_ia.x : eg == 1 ? u_tv.x : eg == 2 ? u_tv.y : u_ia.x;
                const T sq = eg == 0 ? u_ie2.y : eg == 1 ? u_tv2.x : eg == 2 ? u_tv2.y : u_ie2.x;
                const T gsum = pk == 1 ? u_g.x : pk == 2 ? u_g.y : T(0);
                const T eg_ = pk == 1 ? u_eg.x : pk == 2 ? u_eg.y : T(0);
                const T part = lin;
                const T accf = l < 8 ? ((l & 1) ? sq : lin) : l == 8 ? u_ia.y : te ? eg_ : gsum;
                const double ref = SHM ? fd[l < 8 ? (eg == 0 ? OF_E0 : OF_T0 + eg - 1) : OF_E0] : myref;
                double v = (double)accf;
                if (l < 8) v += (l & 1) ? ns * ref * ref + 2.0 * ref * (double)part : ns * ref;
                else if (te) v += ref * (double)gsum;
                // the FP32 running-sum changes into the FP64 sums
                if constexpr (SHM) {
                    double s_ = fd[OF_ACCS + l], c_ = fd[OF_ACCC + l];
                    kadd(s_, c_, v);
                    fd[OF_ACCS + l] = s_;
                    fd[OF_ACCC + l] = c_;
                    const double nl = fd[OF_LAPJ] + (double)dlap, nb = fd[OF_BH2] + (double)dbh2;
                    const double nv = fd[OF_VINT] + (double)dvint, nx = fd[OF_SUMX2] + (double)dsx2;
                    __syncwarp();
                    if (l == 0) {
                        fd[OF_LAPJ] = nl;
                        fd[OF_BH2] = nb;
                        fd[OF_VINT] = nv;
                        fd[OF_SUMX2] = nx;
                    }
                    __syncwarp();
                } else {
                    kadd(acc_s, acc_c, v);
                    lapj += (double)dlap;
                    bh2 += (double)dbh2;
                    vint += (double)dvint;
                    sumx2 += (double)dsx2;
                }
                dlap = dbh2 = dvint = dsx2 = T(0);
                fp32_bases();
            }
        };
        if constexpr (F32) fp32_bases();

        unsigned long long ctr = P.counter[w];
        // the step whose sample is pending (taken with the next step's reduce-scatter)
        bool pend = false, pend_acc = false, pend_win = false;

        // FP64 form: E_L and dlnPsi/dtheta of the pending step from its kinetic sum ks
        auto sample = [&](T ks) {
            if constexpr (!F32) {
                const double lap = (double)ks + lapj - lapc;
                const double ekin = -0.5 * lap, vext = w2h * sumx2, el = ekin + vext + vint;
                if (el != el) status |= ST_NAN_ENERGY;
                const double base = eg == 0 ? el : eg == 1 ? ekin : eg == 2 ? vext : vint;
                const double qe = (l & 1) ? base * base : base;
                const double g = pk == 1 ? a.oc[OC_MHOM] * sumx2 : pk == 2 ? dgk * bh2 : 0.0;
                const double qp = pend_win ? (te ? g * el : g) : 0.0;
                kadd(acc_s, acc_c, l < 8 ? qe : l == 8 ? (pend_acc ? 1.0 : 0.0) : qp);
            }
        };

        for (int s0 = 0; s0 < steps; s0 += 32) {
            // lane i draws the numbers of step ctr + i; step s0 + i reads them by shuffle
            int rng_k;
            T rng_z;
            unsigned rng_u;
            {
                const unsigned long long c = ctr + (unsigned long long)l;
                const uint4 v = philox(make_uint4((uint32_t)c, (uint32_t)(c >> 32), (uint32_t)(w + P.walker_offset), 0u),
                                       make_uint2((uint32_t)a.seed, (uint32_t)(a.seed >> 32)));
                rng_k = (int)__umulhi(v.x, (unsigned)D);
                if constexpr (F32) {
                    const float u1 = ((float)v.y + 1.0f) * 2.3283064e-10f;
                    const float u2 = (float)v.z * 2.3283064e-10f;
                    rng_z = sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2);
                } else {
                    const double u1 = ((double)v.y + 1.0) * TWO_M32, u2 = v.z * TWO_M32;
                    rng_z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
                }
                rng_u = v.w;
            }
            if constexpr (STALE) {
                if (!allcur) {
                    const unsigned long long mm = own ? (msk[l] & msk[n + l]) : ~0ull;
                    allcur = __all_sync(FULL, mm == ~0ull);
                }
            }
            const int s_end = min(s0 + 32, steps);
            for (int s = s0; s < s_end; ++s) {
                const int it_step = step_offset + s;
                const int slot = (s - s0) & 31;
                ++ctr;
                const int k = __shfl_sync(FULL, rng_k, slot);
                const T zr = __shfl_sync(FULL, rng_z, slot);
                const unsigned ur = __shfl_sync(FULL, rng_u, slot);
                // ---- 1. proposal of coordinate k (particle p, axis adim; owner lane pl of block b)
                const int p = k >> 1, adim = k & 1;
                const int b = p >= n ? 1 : 0;
                const int pl = p - b * n;
                const T2 xp = reinterpret_cast<const T2 *>(xs)[p];
                const T xo = adim ? xp.y : xp.x;
                // the drift limiter is a corrected-mode option: compiled out of the reference form
                T Fn;
                if constexpr (!LIMIT) Fn = T(2) * gs[k];
                else Fn = T(2) * limited_drift<T>(gs[k], P);
                const T dx = hdt * Fn + zr * sdt;
                const T xn = xo + dx;
                const T qx = adim ? xp.x : xn, qy = adim ? xn : xp.y;  // proposed position of p

                // ---- 2a. Slater: s_l = phi(r_p') . staged row l of block b (lane l), R = sigma_p s_pl
                T sl, gl_ = T(0);
                if constexpr (GREEN_Q && OWNER_PACK_DOT) {
                    // packed: for the pair (a < b) in slots (b, a), (a, b),
                    //   Qd[a] += (hh_b(x), hh_b(y)) * (v(b,a), v(a,b)),
                    // a diagonal (d, d) adds hh_d(x) v to Qd[d].x, and
                    //   s = sum_a hh_a(y) Qd[a].x + hh_a(x) Qd[a].y
                    constexpr int QN = (K + 1) / 2;  // smaller indices of the pairs and diagonals
                    T2 H[K];
                    hermite_pe2<K, T>(two(sq2 * qx, sq2 * qy), H);
                    const T *row = inv + (b * n + lc) * IS;
                    T2 Qd[QN];
#pragma unroll
                    for (int m = 0; m < QN; ++m) Qd[m] = two(T(0), T(0));
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        T v[VE];
                        vload<T>(row + q * VE, v);
#pragma unroll
                        for (int e = 0; e < VE; e += 2) {
                            const int i = q * VE + e;
                            if (i < 2 * PO.np) {
                                const int qa = PO.m1[i], qb = PO.m0[i];
                                Qd[qa] = fma2(H[qb], two(v[e], v[e + 1]), Qd[qa]);
                            } else {
#pragma unroll
                                for (int t = 0; t < 2; ++t)
                                    if (i + t < n) {
                                        const int d = PO.m0[i + t];
                                        Qd[d].x = fmaT(H[d].x, v[e + t], Qd[d].x);
                                    }
                            }
                        }
                    }
                    T s = T(0);
#pragma unroll
                    for (int m = 0; m < QN; ++m) s = fmaT(H[m].x, Qd[m].y, fmaT(H[m].y, Qd[m].x, s));
                    sl = s;
                } else {
                T hu[K], hv[K];
                hermite_pe<K>(sq2 * qx, hu);
                hermite_pe<K>(sq2 * qy, hv);
                    const T *row = inv + (b * n + lc) * IS;
                    T part[K];
#pragma unroll
                    for (int m = 0; m < K; ++m) part[m] = T(0);
                    if (GREEN_Q || adim == 0) {
                        // factorised along x: part[m0] = sum_m1 hh_m1(v) row
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            T v[VE];
                            vload<T>(row + q * VE, v);
#pragma unroll
                            for (int e = 0; e < VE; ++e) {
                                const int i = q * VE + e;
                                if (i < n) part[PO.m0[i]] = fmaT(hv[PO.m1[i]], v[e], part[PO.m0[i]]);
                            }
                        }
                        T s2 = T(0), g2 = T(0);
#pragma unroll
                        for (int m = 0; m < K; ++m) s2 = fmaT(hu[m], part[m], s2);
                        if (!GREEN_Q)
#pragma unroll
                            for (int m = 1; m < K; ++m) g2 = fmaT(hu[m - 1], part[m], g2);
                        sl = s2;
                        gl_ = g2;
                    } else {
                        // factorised along y (corrected mode, a move along y)
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            T v[VE];
                            vload<T>(row + q * VE, v);
#pragma unroll
                            for (int e = 0; e < VE; ++e) {
                                const int i = q * VE + e;
                                if (i < n) part[PO.m1[i]] = fmaT(hu[PO.m0[i]], v[e], part[PO.m1[i]]);
                            }
                        }
                        T s2 = T(0), g2 = T(0);
#pragma unroll
                        for (int m = 0; m < K; ++m) s2 = fmaT(hv[m], part[m], s2);
#pragma unroll
                        for (int m = 1; m < K; ++m) g2 = fmaT(hv[m - 1], part[m], g2);
                        sl = s2;
                        gl_ = g2;
                    }
                }
                const T sig_l = b ? SIG.y : SIG.x;  // this lane's row scale in block b
                const T R = __shfl_sync(FULL, sig_l * sl, pl);

                // ---- 2b. pair terms: the moved particle against both own particles (packed)
                T2 gdx, gdy;  // Pade gradient change of the own particles
                T vals[8];
                {
                    const T2 pxo = two(-xp.x, -xp.x), pyo = two(-xp.y, -xp.y);
                    const T2 pxn = two(-qx, -qx), pyn = two(-qy, -qy);
                    const T2 dxo = add2(X[0], pxo), dyo = add2(X[1], pyo);  // partner minus moved
                    const T2 dxn = add2(X[0], pxn), dyn = add2(X[1], pyn);
                    const T2 r2o = fma2(dyo, dyo, mul2(dxo, dxo)), r2n = fma2(dyn, dyn, mul2(dxn, dxn));
                    // partners: particle l (block 0) and n + l (block 1), not the moved one
                    const bool va = own && !(b == 0 && l == pl), vb = own && !(b == 1 && l == pl);
                    const T2 iro = two(va ? Fs::rsqrt(r2o.x) : T(0), vb ? Fs::rsqrt(r2o.y) : T(0));
                    const T2 irn = two(va ? Fs::rsqrt(r2n.x) : T(0), vb ? Fs::rsqrt(r2n.y) : T(0));
                    const T2 ro = mul2(r2o, iro), rn = mul2(r2n, irn);
                    // spin coefficients: particle l has spin up, n + l spin down
                    const T2 B = b ? two(banti, bsame) : two(bsame, banti);
                    T2 gpo = gam2;
                    if constexpr (STALE) {
                        if (!allcur) {
                            const unsigned long long mp = msk[p];
                            gpo = two(((mp >> l) & 1ull) ? gam : gamp, ((mp >> (n + l)) & 1ull) ? gam : gamp);
                        }
                    }
                    const T2 deno = fma2(gpo, ro, one2), denn = fma2(gam2, rn, one2);
                    const T2 f1o = two(Fs::rcp(deno.x), Fs::rcp(deno.y)), f1n = two(Fs::rcp(denn.x), Fs::rcp(denn.y));
                    const T2 ho = mul2(ro, f1o), hn = mul2(rn, f1n);
                    const T2 fio = mul2(mul2(f1o, f1o), mul2(B, iro));  // beta f1^2 / r
                    const T2 fin = mul2(mul2(f1n, f1n), mul2(B, irn));
                    T2 dh = add2(hn, two(-ho.x, -ho.y));
                    if constexpr (RATIO_Q) dh = two(l > p ? dh.x : T(0), n + l > p ? dh.y : T(0));
                    const T2 sr = mul2(B, dh);
                    // d J / d x_j = beta f1^2 (x_j - x_p) / r for the partner j, the negative
                    // for the moved particle: the partners' change is new minus old
                    const T2 tnx = mul2(fin, dxn), tny = mul2(fin, dyn);
                    gdx = fma2(fio, two(-dxo.x, -dxo.y), tnx);
                    gdy = fma2(fio, two(-dyo.x, -dyo.y), tny);
                    // 2 f (DIM - (1 + 2 gamma h)) / r, new minus old (DIM = 2)
                    const T2 lqo = mul2(fio, fma2(m2gam, ho, one2)), lqn = mul2(fin, fma2(m2gam, hn, one2));
                    const T2 dl = add2(lqn, two(-lqo.x, -lqo.y));
                    const T2 hh = fma2(hn, hn, mul2(two(-ho.x, -ho.y), ho));
                    const T2 db = mul2(B, hh);
                    const T2 dv = add2(irn, two(-iro.x, -iro.y));
                    vals[0] = sr.x + sr.y;
                    vals[1] = T(2) * (dl.x + dl.y);
                    vals[2] = db.x + db.y;
                    vals[3] = dv.x + dv.y;
                    vals[4] = -(tnx.x + tnx.y);
                    vals[5] = -(tny.x + tny.y);
                    vals[6] = kp;  // the previous step's kinetic terms
                    vals[7] = T(0);
                }
                // one reduce-scatter: lane L ends with the total of value L / 4
                const T tot = warp_reduce_scatter8<T, 32>(vals, l);
                const T sum_ratio = __shfl_sync(FULL, tot, 0);
                if constexpr (F32) {
                    if (pend && l == 24) sbk[slot - 1] = tot;  // the previous step's kinetic sum
                } else {
                    if (pend) sample(__shfl_sync(FULL, tot, 24));  // E_L of the previous step
                }
                pend = false;

                // ---- 2c/2d. ratio, Green's ratio, accept
                // the Gaussian and Pade factors of the ratio: FP32 takes them as one
                // exponential of the summed exponents; FP64 keeps the reference's two
                // factors (and so its rounding)
                T rat_g, rat_p;
                if constexpr (F32) {
                    rat_g = Fs::exp(fmaf(wa, (xo - xn) * (xo + xn), 2.0f * sum_ratio));
                    rat_p = 1.0f;
                } else {
                    rat_g = Fs::exp(wa * (xo * xo - xn * xn));
                    rat_p = Fs::exp(T(2) * sum_ratio);
                }
                bool accept;
                if constexpr (GREEN_Q) {
                    // importancesampling.cpp:43-47: exp(0.5 (F_old(k) - F_new(k)) dx) + 1
                    const T ex = Fs::exp(T(0.5) * (fcs[k] - Fn) * dx);
                    if constexpr (F32) {
                        const float wgt = (ex + 1.0f) * (R * R * rat_g);
                        if (wgt != wgt) status |= ST_BAD_RATIO;
                        accept = wgt >= __uint2float_rn(ur) * 2.3283064365386963e-10f;
                    } else {
                        const double wgt = ((double)ex + 1.0) * ((double)(R * R) * (double)rat_g * (double)rat_p);
                        if (wgt != wgt) status |= ST_BAD_RATIO;
                        accept = wgt >= ur * TWO_M32;
                    }
                } else {
                    // Fokker-Planck Green's ratio with the drift at the proposed point
                    const T gsl = __shfl_sync(FULL, sig_l * gl_, pl) * sq2;
                    const T gy = -wa * xn + __shfl_sync(FULL, tot, 16 + 4 * adim) + gsl / R;
                    const double prob = (double)(R * R) * (double)rat_g * (double)rat_p;
                    const double fy = 2.0 * (double)(LIMIT ? limited_drift<T>(gy, P) : gy), fo2 = (double)Fn;
                    const double wgt = prob * exp(0.5 * (fo2 + fy) * (0.25 * P.step * (fo2 - fy) - (double)dx));
                    if (wgt != wgt) status |= ST_BAD_RATIO;
                    accept = wgt >= ur * TWO_M32;
                }

                if (accept) {
                    // ---- 3. state update
                    // the moved particle's block as a compile-time constant: its rows, row
                    // scale and register halves are fixed offsets and halves, not selections
                    auto update = [&](auto block) {
                        constexpr int b = decltype(block)::value;
                        const bool mine = l == pl;
                        if (adim == 0) {
                            if (mine) X[0] = b ? two(X[0].x, xn) : two(xn, X[0].y);
                        } else {
                            if (mine) X[1] = b ? two(X[1].x, xn) : two(xn, X[1].y);
                        }
                        if (l == 0) {
                            xs[k] = xn;
                            fcs[k] = Fn;
                        }
                        // running sums (the pair totals sit in lanes 4, 8, 12; the new
                        // gradient of the moved particle in lanes 16, 20)
                        const T tl = __shfl_sync(FULL, tot, 4), tb = __shfl_sync(FULL, tot, 8);
                        const T tv = __shfl_sync(FULL, tot, 12);
                        const T tgx = __shfl_sync(FULL, tot, 16), tgy = __shfl_sync(FULL, tot, 20);
                        if constexpr (F32) {
                            dlap += tl;
                            dbh2 += tb;
                            dvint += tv;
                            dsx2 += (xn - xo) * (xn + xo);
                        } else {
                            sumx2 += (double)xn * (double)xn - (double)xo * (double)xo;
                            lapj += (double)tl;
                            bh2 += (double)tb;
                            vint += (double)tv;
                        }
                        // Pade gradients: partners by their change, the moved particle anew
                        GJ[0] = add2(GJ[0], gdx);
                        GJ[1] = add2(GJ[1], gdy);
                        if (mine) {
                            GJ[0] = b ? two(GJ[0].x, tgx) : two(tgx, GJ[0].y);
                            GJ[1] = b ? two(GJ[1].x, tgy) : two(tgy, GJ[1].y);
                        }
                        if constexpr (STALE) {
                            if (!allcur) {
                                if (own && l != p) msk[l] |= 1ull << p;
                                if (own && n + l != p) msk[n + l] |= 1ull << p;
                                if (mine) msk[p] = ~0ull;
                            }
                        }
                        // Sherman-Morrison on block b (slaterdeterminant.cpp:165-175) through the
                        // row scales: row l += t_l row p with t_l = -s_l sigma_p / R (staged
                        // rows), sigma_p /= R; then the block's gradient vectors
                        // (slaterdeterminant.cpp:155-163) from the updated rows
                        const T sig_p = __shfl_sync(FULL, sig_l, pl);
                        const T rinv = Fs::rcp(R);
                        const T tcoef = (own && !mine) ? -(sl * sig_p * rinv) : T(0);
                        const T sig_new = mine ? sig_l * rinv : sig_l;
                        if (b) SIG.y = sig_new;
                        else SIG.x = sig_new;
                        const T ux = sq2 * (b ? X[0].y : X[0].x), uy = sq2 * (b ? X[1].y : X[1].x);
                        T *rowj = inv + (b * n + lc) * IS;
                        const T *rowp = inv + (b * n + pl) * IS;
                        const bool store = own && !mine;
                        T gx, gy2;
                        if constexpr (OWNER_PACK_ACC) {
                            // packed, with Hj[m] = (hh_m(x), hh_m(y)) of the lane's particle, its
                            // swaps Hs[a] = (hh_a(y), hh_a(x)), P0[m0] = sum_m1 hh_m1(y) v(m0, m1)
                            // and P1[m1] = sum_m0 hh_m0(x) v(m0, m1): for the pair (a < b) with
                            // S = (v(b,a), v(a,b)),
                            //   Q[a] = (P1[a], P0[a]) += Hj[b] * S,  Rb[b] = (P0[b], P1[b]) += Hs[a] * S,
                            // and a diagonal (d, d) adds Hj[d] * (v, v) to Q[d]
                            constexpr int QN = (K + 1) / 2;
                            T2 Hj[K];
                            hermite_pe2<K, T>(two(ux, uy), Hj);
                            T2 Hs[QN];
    #pragma unroll
                            for (int m = 0; m < QN; ++m) Hs[m] = two(Hj[m].y, Hj[m].x);
                            T2 Q[QN], Rb[K];
    #pragma unroll
                            for (int m = 0; m < QN; ++m) Q[m] = two(T(0), T(0));
    #pragma unroll
                            for (int m = 0; m < K; ++m) Rb[m] = two(T(0), T(0));
    #pragma unroll
                            for (int q = 0; q < NQ; ++q) {
                                T cv[VE], vv[VE];
                                vload<T>(rowp + q * VE, cv);
                                vload<T>(rowj + q * VE, vv);
    #pragma unroll
                                for (int e = 0; e < VE; e += 2) {
                                    const T2 nv = fma2(two(cv[e], cv[e + 1]), two(tcoef, tcoef), two(vv[e], vv[e + 1]));
                                    vv[e] = nv.x;
                                    vv[e + 1] = nv.y;
                                }
                                if (store) vstore<T>(rowj + q * VE, vv);
    #pragma unroll
                                for (int e = 0; e < VE; e += 2) {
                                    const int i = q * VE + e;
                                    if (i < 2 * PO.np) {
                                        const int qa = PO.m1[i], qb = PO.m0[i];
                                        const T2 S = two(vv[e], vv[e + 1]);
                                        Q[qa] = fma2(Hj[qb], S, Q[qa]);
                                        Rb[qb] = fma2(Hs[qa], S, Rb[qb]);
                                    } else {
    #pragma unroll
                                        for (int t = 0; t < 2; ++t)
                                            if (i + t < n) {
                                                const int d = PO.m0[i + t];
                                                Q[d] = fma2(Hj[d], two(vv[e + t], vv[e + t]), Q[d]);
                                            }
                                    }
                                }
                            }
                            // d/dx = sum_m hh_{m-1}(x) P0[m], d/dy = sum_m hh_{m-1}(y) P1[m]
                            T2 GR = two(T(0), T(0)), GQ = GR;
    #pragma unroll
                            for (int m = 1; m < K; ++m) GR = fma2(Hj[m - 1], Rb[m], GR);
    #pragma unroll
                            for (int m = 1; m < QN; ++m) GQ = fma2(Hs[m - 1], Q[m], GQ);
                            gx = GR.x + GQ.y;
                            gy2 = GR.y + GQ.x;
                        } else {
                            T au[K], av[K];
                            hermite_pe<K>(ux, au);
                            hermite_pe<K>(uy, av);
                            T P0[K], P1[K];  // P0[m0] = sum_m1 hh_m1(y) v, P1[m1] = sum_m0 hh_m0(x) v
    #pragma unroll
                            for (int m = 0; m < K; ++m) P0[m] = P1[m] = T(0);
    #pragma unroll
                            for (int q = 0; q < NQ; ++q) {
                                T cv[VE], vv[VE];
                                vload<T>(rowp + q * VE, cv);
                                vload<T>(rowj + q * VE, vv);
    #pragma unroll
                                for (int e = 0; e < VE; e += 2) {
                                    const T2 nv = fma2(two(cv[e], cv[e + 1]), two(tcoef, tcoef), two(vv[e], vv[e + 1]));
                                    vv[e] = nv.x;
                                    vv[e + 1] = nv.y;
                                }
                                if (store) vstore<T>(rowj + q * VE, vv);
    #pragma unroll
                                for (int e = 0; e < VE; ++e) {
                                    const int i = q * VE + e;
                                    if (i < n) {
                                        P0[PO.m0[i]] = fmaT(av[PO.m1[i]], vv[e], P0[PO.m0[i]]);
                                        P1[PO.m1[i]] = fmaT(au[PO.m0[i]], vv[e], P1[PO.m1[i]]);
                                    }
                                }
                            }
                            gx = gy2 = T(0);
    #pragma unroll
                            for (int m = 1; m < K; ++m) {
                                gx = fmaT(au[m - 1], P0[m], gx);
                                gy2 = fmaT(av[m - 1], P1[m], gy2);
                            }
                        }
                        {
                            // lanes without particles keep zeros
                            const T g1 = own ? sig_new * sq2 : T(0);
                            if (b) {
                                DD[0].y = g1 * gx;
                                DD[1].y = g1 * gy2;
                            } else {
                                DD[0].x = g1 * gx;
                                DD[1].x = g1 * gy2;
                            }
                        }
                    };
                    if (b)
                        update(std::integral_constant<int, 1>{});
                    else
                        update(std::integral_constant<int, 0>{});
                    kp = publish();
                    __syncwarp();
                }
                // ---- 4. this step's sample, taken with the next step's reduce-scatter
                const bool sampled = it_step >= a.burn_in, win = it_step > a.win_lo && it_step < a.win_hi;
                if (sampled) {
                    pend = true;
                    pend_acc = accept;
                    pend_win = win;
                }
                if constexpr (F32) {
                    if (l == 0) {
                        sbd[slot] = make_float4(dlap, dsx2, dvint, dbh2);
                        sbf[slot] = (sampled ? SB_SAMPLED : 0u) | (accept ? SB_ACCEPT : 0u) | (win ? SB_WINDOW : 0u);
                    }
                }
            }
            if constexpr (F32) {
                if (pend) {  // the block's last step: its kinetic sum by a reduction of its own
                    const T ks = seg_sum<32>(kp);
                    if (l == 0) sbk[s_end - 1 - s0] = ks;
                    pend = false;
                }
                fold(s_end - s0);
            }
        }
        if (pend) sample(seg_sum<32>(kp));

        // ---- write the walker back
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (own) {
                T *dst = rec + L.off_inv + (size_t)(h * n + l) * L.inv_stride;
                const T *src = inv + (h * n + l) * IS;
                const T sg = h ? SIG.y : SIG.x;
                T v[IS];
#pragma unroll
                for (int q = 0; q < IS / VE; ++q) vload<T>(src + q * VE, v + q * VE);
#pragma unroll
                for (int i = 0; i < n; ++i) dst[PO.orb[i]] = v[i] * (sg * T(1.0 / PO.scale[i]));
            }
        }
        if (own) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int ka = 2 * l + c, kb = 2 * (n + l) + c;
                rec[L.off_x + ka] = X[c].x;
                rec[L.off_x + kb] = X[c].y;
                rec[L.off_dd + ka] = DD[c].x;
                rec[L.off_dd + kb] = DD[c].y;
                rec[L.off_gj + ka] = GJ[c].x;
                rec[L.off_gj + kb] = GJ[c].y;
            }
            // (d^2 det / dx^2) / det of both own particles from their final rows:
            // 2 sigma sum_m hh_{m-2}(x) P0[m] and 2 sigma sum_m hh_{m-2}(y) P1[m]
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                T au[K], av[K];
                hermite_pe<K>(sq2 * (h ? X[0].y : X[0].x), au);
                hermite_pe<K>(sq2 * (h ? X[1].y : X[1].x), av);
                const T *src = inv + (h * n + l) * IS;
                T P0[K], P1[K];
#pragma unroll
                for (int m = 0; m < K; ++m) P0[m] = P1[m] = T(0);
#pragma unroll
                for (int i = 0; i < n; ++i) {
                    const T v = src[i];
                    P0[PO.m0[i]] = fmaT(av[PO.m1[i]], v, P0[PO.m0[i]]);
                    P1[PO.m1[i]] = fmaT(au[PO.m0[i]], v, P1[PO.m1[i]]);
                }
                T sx = T(0), sy = T(0);
#pragma unroll
                for (int m = 2; m < K; ++m) {
                    sx = fmaT(au[m - 2], P0[m], sx);
                    sy = fmaT(av[m - 2], P1[m], sy);
                }
                const T g2 = T(2) * (h ? SIG.y : SIG.x);
                rec[L.off_sdd + 2 * (h * n + l)] = g2 * sx;
                rec[L.off_sdd + 2 * (h * n + l) + 1] = g2 * sy;
            }
        }
        for (int i = l; i < D; i += 32) rec[L.off_fc + i] = fcs[i];
        if (mdirty)
            for (int j = l; j < N; j += 32) P.mask[(size_t)w * N + j] = msk[j];
        if constexpr (SHM) {
            sumx2 = fd[OF_SUMX2];
            lapj = fd[OF_LAPJ];
            bh2 = fd[OF_BH2];
            vint = fd[OF_VINT];
            acc_s = fd[OF_ACCS + l];
            acc_c = fd[OF_ACCC + l];
        }
        if (l == 0) {
            double *so = P.scal + (size_t)w * NSCAL;
            so[SC_SUMX2] = sumx2;
            so[SC_LAPJ] = lapj;
            so[SC_BH2] = bh2;
            so[SC_VINT] = vint;
            P.counter[w] = ctr;
        }
        if (l < P.nacc) {
            P.acc[((size_t)w * P.nacc + l) * 2] = acc_s;
            P.acc[((size_t)w * P.nacc + l) * 2 + 1] = acc_c;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) status |= __shfl_xor_sync(FULL, status, o);
        if (l == 0 && status) P.status[w] |= status;
        __syncwarp();
    }
}

template <typename T, int K, int FX>
__global__ void __launch_bounds__(OWNER_WPB * 32, sizeof(T) == 4 ? OWNER_MIN_CTAS_F32 : OWNER_MIN_CTAS_F64) owner_sweep_kernel(const SweepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5;
    unsigned char *ws = smem_raw + (size_t)wib * a.smem_per_warp;
    const int w0 = blockIdx.x * OWNER_WPB + wib, stride = gridDim.x * OWNER_WPB;
    if constexpr ((FX & Q_IS_GREEN) == 0) {  // the limiter is a corrected-mode option
        if (a.P.drift_limit > 0.0) {
            owner_sweep_walkers<T, K, FX, true>(a, a.steps, a.step_offset, ws, w0, a.P.W, stride);
            return;
        }
    }
    owner_sweep_walkers<T, K, FX>(a, a.steps, a.step_offset, ws, w0, a.P.W, stride);
}

}  // namespace vmc
