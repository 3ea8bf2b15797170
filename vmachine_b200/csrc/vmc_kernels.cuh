// Walker kernels: Metropolis sweep with E_L / dlnPsi sampling, FP64 rebuild
// (initialisation, periodic refresh, drift measurement) and per-element evaluation.
//
// Mapping: one warp per walker, WPB walkers per CTA, persistent grid-stride loop
// over walkers.  A walker's state record lives in HBM between launches and in the
// warp's slice of shared memory during a sweep:
//
//   x[D]      positions, particle-major (k = p*DIM + dim) as System::m_positions
//   fc[D]     importance-sampling force cache (ImportanceSampling::m_quantumForceNew)
//   dd[D]     d ln det / dx_k  (SlaterDeterminant::m_determinantDerivative)
//   sdd[D]    (d^2 det / dx_k^2) / det (m_determinantSecondDerivative)
//   gj[D]     d J / dx_k of the Pade factor, J = sum_{i<j} beta r/(1 + gamma r)
//   inv[2][n][S]  inverse Slater blocks stored by particle: row i of block b holds
//                 A_b^{-1}(o, i) for the orbitals o (the reference's
//                 m_slaterMatrixInverse, n x N, column b*n + i), row stride S
//
// plus FP64 per-walker scalars (running sums, see SC_*), a 64-bit per-particle mask
// of Pade pairs computed with the current gamma, and the Philox step counter.
#pragma once
#include "vmc_device.cuh"
#include "vmc_mlp.cuh"

namespace vmc {

// FP64 per-walker scalars
enum : int {
    SC_SUMX2 = 0,  // sum_k x_k^2
    SC_LAPJ = 1,   // Pade Laplacian, sum over pairs
    SC_BH2 = 2,    // sum over pairs beta h^2 (dlnPsi/dgamma = -BH2, or -BH2/2 in compat)
    SC_VINT = 3,   // sum_{i<j} 1/r_ij
    SC_INVR = 4,   // sum_i 1/r_i (atomic potential, hydrogen-like Laplacian)
    SC_LOGDET = 5, // ln|det up| + ln|det down|, updated by ln|R| per accepted move
    SC_SUMR = 6,   // sum_i r_i
    NSCAL = 8,
};

struct Layout {
    int N, D, n;  // particles, coordinates, orbitals per spin block (0: no Slater)
    int off_x, off_fc, off_dd, off_sdd, off_gj, off_inv, rec;  // in elements of T
    int inv_stride;  // row stride S of the inverse blocks
};

__host__ __device__ inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Row stride of an inverse block: a multiple of the 16-byte vector width VE (4
// floats or 2 doubles) with an odd number of vectors, so that the 8 lanes of one
// 128-bit shared-memory phase start on distinct 4-bank groups (no conflicts).
__host__ __device__ constexpr int inv_row_stride(int n, int elem_bytes)
{
    const int ve = 16 / elem_bytes;
    int s = (n + ve - 1) / ve * ve;
    if (s > 0 && ((s / ve) & 1) == 0) s += ve;
    return s;
}

__host__ __device__ inline Layout make_layout(int N, int dim, int n, int elem_bytes)
{
    const int a = 16 / elem_bytes;  // keep every array 16-byte aligned
    Layout L;
    L.N = N;
    L.D = N * dim;
    L.n = n;
    const int Dp = round_up(L.D, a);
    L.off_x = 0;
    L.off_fc = L.off_x + Dp;
    L.off_dd = L.off_fc + Dp;
    L.off_sdd = L.off_dd + Dp;
    L.off_gj = L.off_sdd + Dp;
    L.off_inv = L.off_gj + Dp;
    L.inv_stride = inv_row_stride(n, elem_bytes);
    L.rec = round_up(L.off_inv + 2 * n * L.inv_stride, a);
    return L;
}

// Shared memory per warp of the rebuild kernel: the pivot row, M (odd row stride)
// and the pivot rows of the Slater phase, or the positions of the pair phase.
__host__ __device__ inline int rebuild_smem_per_warp(int N, int dim, int n)
{
    const int slater = n > 0 ? ((n + 1) & ~1) * 8 + n * (n | 1) * 8 + n * 4 : 0;
    return round_up(slater > N * dim * 8 ? slater : N * dim * 8, 16);
}

constexpr int MAX_ELEM = 8;
constexpr int MAX_N = 64;

struct Params {
    Layout L;
    int W, N, n_elem, ep, nacc;
    // index of this engine's first walker in a population sharded over engines: walker
    // w's random streams are keyed by w + walker_offset, so shards reproduce one engine
    int walker_offset;
    int elem_kind[MAX_ELEM];  // element kinds in configuration order
    int flags, sampling;
    double omega, alpha, gamma, gamma_prev, alpha_h, Z;
    double step;               // stepLength (brute force) or dt (importance sampling)
    double drift_limit;        // importance sampling, corrected mode: the limiter's a (0: off)
    int idx_alpha, idx_gamma, idx_alpha_h;  // parameter slots (e*p_max + j) or -1
    double beta_same, beta_anti;            // Pade spin coefficients
    // device buffers
    void *state;               // W x L.rec elements of T
    double *scal;              // W x NSCAL
    unsigned long long *mask;  // W x N
    unsigned long long *counter;  // W Philox step counters
    double *acc;               // W x nacc x 2 (sum, compensation)
    unsigned *status;          // W
    // MLP Jastrow on the dot sweep: the weights (bfloat16-rounded floats in the CTA
    // block layout, MLP_SMEM_FLOATS) and per walker the pair and one-body caches,
    // (u, u', u'') of every ordered pair [i][j] then (chi, chi', chi'') of every
    // particle, mlp_cache_stride floats
    const float *mlpw;
    float *mlp_cache;
    int mlp_cache_stride;
};

// The corrected mode's drift limiter (Umrigar, Nightingale and Runge, J. Chem. Phys. 99,
// 2865 (1993)): v = d ln Psi / dx_k becomes v (-1 + sqrt(1 + 2 a dt v^2)) / (a dt v^2),
// written as 2 v / (1 + sqrt(1 + 2 a dt v^2)), in the proposal and in the Green's ratio
// alike, so the chain stays exact; a = P.drift_limit, 0 leaves v alone.  It bounds the
// step a walker next to a node of the determinant takes, where v grows like 1 / distance.
template <typename T>
__device__ __forceinline__ T limited_drift(T v, const Params &P)
{
    if (!(P.drift_limit > 0.0)) return v;
    const T c = T(2.0 * P.drift_limit * P.step);
    return T(2) * v / (T(1) + sqrt(T(1) + c * v * v));
}


// Per-launch constants of the owner sweep, computed by the host in FP64 and passed in
// both precisions, so the kernel reads them as constant operands
enum : int {
    OC_WA = 0,    // omega alpha
    OC_HDT,       // dt / 2
    OC_SDT,       // sqrt(dt)
    OC_GAM,       // Pade gamma
    OC_GAMP,      // the previous gamma (stale pairs)
    OC_M2GAM,     // -2 gamma
    OC_BSAME,     // Pade beta, equal spins
    OC_BANTI,     // Pade beta, opposite spins
    OC_W2H,       // omega^2 / 2
    OC_MHOM,      // -omega / 2
    OC_DGK,       // dlnPsi/dgamma per sum beta h^2 (-1, or -1/2 under the reference quirk)
    OC_LAPC,      // omega alpha D, the Gaussian's -Laplacian
    OC_N = 16
};

struct SweepArgs {
    Params P;
    double oc[OC_N];  // owner sweep constants (OC_*)
    float ocf[OC_N];  // the same in FP32
    int steps, step_offset, burn_in, win_lo, win_hi;
    unsigned long long seed;
    const double *replay;  // W x replay_stride x 3 or null
    int replay_stride, replay_offset;  // entry of step s: replay_offset + step_offset + s
    unsigned char *rec_acc;  // W x rec_stride or null
    double *rec_en;          // W x rec_stride x 3 or null
    int rec_stride;
    const int *probe_k;      // W or null: forced move of coordinate probe_k[w] ...
    const double *probe_x;   // ... to probe_x[w], accepted; ratios to probe_ratio
    double *probe_ratio;     // W x n_elem
    int wpb, smem_per_warp;
    // MLP Jastrow parameter-gradient snapshots (general path): positions and local
    // energy every snap_interval steps inside the gradient window, snap_stride per walker
    float *snap_x;
    double *snap_e;
    int snap_stride, snap_interval, snap_first;  // slot = (step - win_lo) / interval - first
    // electron densities over the sampled steps (0 bins: off): radial one-body counts
    // (bins), the spatial one-body grid and the radial two-body counts (bins x bins,
    // row-major), each optional
    unsigned long long *dens_radial, *dens_grid, *dens_pair;
    int dens_bins;
    double dens_step, dens_max;  // maxRadius / bins, maxRadius
};

// Electron densities at a walker's current positions (Sampler::computeOneBodyDensity,
// computeOneBodyDensity2, computeTwoBodyDensity: sampler.cpp:639-692), added to 64-bit
// device histograms: radial bin floor(r / step) for r < maxRadius; spatial cell
// (trunc(y / 2 step) + bins/2, trunc(x / 2 step) + bins/2) inside the grid; two-body
// cell (floor(r_i / step) + 1, floor(r_j / step) + 1) for i < j, both below bins.
// Lanes over particles (two per lane above 32); called by the whole warp.
__device__ __forceinline__ int density_bin(double q)
{
    return (q == q && q < 2.0e9 && q > -2.0e9) ? (int)q : 2000000000;  // truncation toward zero
}

template <typename T>
__device__ void density_sample(const SweepArgs &a, const T *x, int N, int dim, int lane)
{
    const int bins = a.dens_bins, half = bins / 2;
    const double step = a.dens_step;
    int pb0 = bins, pb1 = bins;  // two-body bins of particles lane and lane + 32
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        if (i >= N) continue;
        double r2 = 0.0;
        for (int c = 0; c < dim; ++c) {
            const double v = (double)x[i * dim + c];
            r2 += v * v;
        }
        const double r = sqrt(r2);
        if (a.dens_radial && r < a.dens_max) {
            const int b = density_bin(r / step);
            if (b < bins) atomicAdd(&a.dens_radial[b], 1ull);
        }
        if (a.dens_grid) {
            const int ix = density_bin((double)x[i * dim] / (2.0 * step));
            const int iy = density_bin((double)x[i * dim + 1] / (2.0 * step));
            if (abs(ix) < half && abs(iy) < half)
                atomicAdd(&a.dens_grid[(size_t)(iy + half) * bins + ix + half], 1ull);
        }
        const int pb = density_bin(r / step);
        (h ? pb1 : pb0) = pb < bins ? pb + 1 : bins;
    }
    if (a.dens_pair) {
        for (int j = 1; j < N; ++j) {
            const int bj = __shfl_sync(0xffffffffu, j < 32 ? pb0 : pb1, j & 31);
            if (bj >= bins) continue;  // uniform over the warp
            if (lane < j && pb0 < bins) atomicAdd(&a.dens_pair[(size_t)pb0 * bins + bj], 1ull);
            if (lane + 32 < j && pb1 < bins) atomicAdd(&a.dens_pair[(size_t)pb1 * bins + bj], 1ull);
        }
    }
}

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ bool same_spin(int i, int j, int N)
{
    const int h = N >> 1;
    return (i < h) == (j < h);
}

}  // namespace vmc

namespace vmc {

// The tensor-core context of the MLP dot sweep: the CTA's weight block, its
// tcgen05 state, and this warp's slot for the layer's per-partner outputs.
struct MlpCtx {
    float *w;
    TcMlp *tc;
    float *pre;
};
// shared-memory weight block of the MLP dot sweep: the packed row (its FP32 W2 slot
// holds the value's low-part A tile) and V2 transposed in the W2^T slot
constexpr int MLP_FAST_FLOATS = MLP_PARAMS + 2 + MLP_G * MLP_G;
constexpr int MLP_FAST_BYTES = MLP_FAST_FLOATS * 4;
static_assert(MLP_FAST_BYTES % 16 == 0 && (MW_W2 * 4) % 16 == 0, "MLP block alignment");

}  // namespace vmc

#include "vmc_sweep.cuh"
#include "vmc_owner_sweep.cuh"

namespace vmc {

// ------------------------------------------------------------------ FP64 rebuild

enum : int { RB_INIT = 0, RB_REFRESH = 1 };

struct RebuildArgs {
    Params P;
    int mode;
    double *drift;  // W: max |inv_old - inv_new| / max |inv_new| (refresh), or null
    int wpb, smem_per_warp;
};

// Rebuild every derived array of a walker from its positions in FP64:
// Slater blocks (Gauss-Jordan with partial pivoting), their derivative vectors,
// the Pade gradient vector and pair sums, Coulomb, radial sums and, at
// initialisation, the importance-sampling force cache.
// Per warp (walkers w_first, w_first + w_stride, ... < w_end; shared slice at
// warp_smem), called by the single-system kernel and the multi-system kernel.
template <typename T, int DIM, int K>
__device__ __forceinline__ void rebuild_walkers(const Params &P, int mode, double *drift, unsigned char *warp_smem,
                                                int w_first, int w_end, int w_stride)
{
    constexpr int NO = K > 0 ? Shells<DIM, K>::n : 0;
    const Layout L = P.L;
    const int lane = threadIdx.x & 31;
    double *A = reinterpret_cast<double *>(warp_smem);
    const int N = P.N, D = L.D, flags = P.flags;
    const double wa = P.omega * P.alpha, az = P.alpha_h * P.Z;

    for (int w = w_first; w < w_end; w += w_stride) {
        T *rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
        const T *x = rec + L.off_x;
        T *fc = rec + L.off_fc, *dd = rec + L.off_dd, *sdd = rec + L.off_sdd, *gj = rec + L.off_gj;
        T *inv = rec + L.off_inv;
        unsigned long long *mask = P.mask + (size_t)w * N;
        if (mode == RB_INIT)
            for (int j = lane; j < N; j += 32) mask[j] = ~0ull;
        __syncwarp();
        unsigned status = 0;
        double sumx2 = 0.0;
        for (int c = lane; c < D; c += 32) sumx2 += (double)x[c] * (double)x[c];
        sumx2 = warp_sum(sumx2);
        double logdet = 0.0, drift_num = 0.0, drift_den = 0.0;

        if constexpr (K > 0) {
            // Per block, lane r < NO holds row r of the Slater block, a[o] = phi_o(r_r),
            // in registers.  Gauss-Jordan with implicit partial pivoting: column c
            // takes the unused row with the largest |a_rc| (a 32-bit magnitude key
            // reduced by redux.sync; the lowest lane wins ties), the pivot row goes
            // through shared memory, and every row is updated in place.  Rows are never
            // interchanged, so the result M satisfies M[p_c][o] = A^{-1}[c][p_o], with
            // p_c the pivot row of column c.
            constexpr int MS = NO | 1;  // odd row stride of M: conflict-free 8-byte access
            double *buf = A;                                       // pivot row, NO (+1) doubles
            double *Msm = A + ((NO + 1) & ~1);                      // NO x MS
            int *prow_of = reinterpret_cast<int *>(Msm + NO * MS);  // p_c, NO ints
            constexpr int VE = 16 / (int)sizeof(T);
            constexpr int S = inv_row_stride(NO, (int)sizeof(T));
            const bool mine = lane < NO;
            for (int b = 0; b < 2; ++b) {
                double av[NO];
                const int q = b * NO + (mine ? lane : 0);
                {
                    double hv[DIM][K];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) hermite_values<K>((double)x[q * DIM + c], hv[c]);
                    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                        double phi = hv[0][m0] * hv[1][m1];
                        if (DIM == 3) phi *= hv[DIM - 1][m2];
                        av[o] = mine ? phi : 0.0;
                    });
                }
                bool used = !mine;
                int col_mine = 0;
                double pivprod = 1.0;  // |product of pivots| as mantissa x 2^pivexp
                int pivexp = 0;
#pragma unroll
                for (int c = 0; c < NO; ++c) {
                    const unsigned key =
                        used ? 0u : ((__float_as_uint((float)fabs(av[c])) >> 1) | 0x80000000u);
                    const unsigned kmax = __reduce_max_sync(FULL, key);
                    const int p = __ffs(__ballot_sync(FULL, key == kmax)) - 1;  // an unused row < NO
                    if (lane == p) {
                        used = true;
                        col_mine = c;
                        prow_of[c] = p;
#pragma unroll
                        for (int o = 0; o < NO; ++o) buf[o] = (o == c) ? 1.0 : av[o];
                    }
                    const double piv = __shfl_sync(FULL, av[c], p);
                    if (!(fabs(piv) > 0.0)) status |= ST_SINGULAR;
                    pivprod *= fabs(piv);
                    if (c % 6 == 5 || c == NO - 1) {
                        // renormalise: move the binary exponent into pivexp (normal numbers;
                        // a zero product already carries ST_SINGULAR)
                        const long long bits = __double_as_longlong(pivprod);
                        const int e = (int)((bits >> 52) & 0x7ff);
                        if (e != 0 && e != 0x7ff) {
                            pivexp += e - 1023;
                            pivprod = __longlong_as_double((bits & ~(0x7ffll << 52)) | (1023ll << 52));
                        }
                    }
                    const double ip = 1.0 / piv;
                    __syncwarp();
                    // rows r != p: a_r -= (a_rc / piv) * a_p, with a_rc <- -a_rc / piv;
                    // row p: a_p <- a_p / piv, with a_pc <- 1 / piv
                    const double f = (lane == p) ? 1.0 - ip : av[c] * ip;
                    av[c] = 0.0;
#pragma unroll
                    for (int o = 0; o + 1 < NO; o += 2) {
                        const double2 bv = *reinterpret_cast<const double2 *>(buf + o);
                        av[o] = fma(-f, bv.x, av[o]);
                        av[o + 1] = fma(-f, bv.y, av[o + 1]);
                    }
                    if (NO & 1) av[NO - 1] = fma(-f, buf[NO - 1], av[NO - 1]);
                    if (lane == p) av[c] = ip;
                    __syncwarp();
                }
                logdet += log(pivprod) + pivexp * 0.6931471805599453;  // ln 2
                if (mine)
#pragma unroll
                    for (int o = 0; o < NO; ++o) Msm[lane * MS + o] = av[o];
                __syncwarp();
                if (mine) {
                    // row i of the stored inverse holds A^{-1}(c, i) = M[p_c][col(i)], c = 0..NO-1
                    const double *mcol = Msm + col_mine;
                    T *row = inv + (size_t)q * L.inv_stride;
#pragma unroll
                    for (int v = 0; v < S / VE; ++v) {
                        T ov[VE], nv[VE];
                        if (mode == RB_REFRESH) vload<T>(row + v * VE, ov);
#pragma unroll
                        for (int e2 = 0; e2 < VE; ++e2) {
                            const int o = v * VE + e2;
                            const double val = o < NO ? mcol[prow_of[o < NO ? o : 0] * MS] : 0.0;
                            if (mode == RB_REFRESH && o < NO) {
                                drift_num = fmax(drift_num, fabs((double)ov[e2] - val));
                                drift_den = fmax(drift_den, fabs(val));
                            }
                            nv[e2] = T(val);
                        }
                        vstore<T>(row + v * VE, nv);
                    }
                    // derivative vectors of particle q with the FP64 inverse row
                    double hv[DIM][K];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) hermite_values<K>((double)x[q * DIM + c], hv[c]);
                    double gd[DIM], sd[DIM];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) { gd[c] = 0.0; sd[c] = 0.0; }
                    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                        const int mm[3] = {m0, m1, m2};
                        const double iv = mcol[prow_of[o] * MS];
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            double t = iv;
#pragma unroll
                            for (int e2 = 0; e2 < DIM; ++e2)
                                if (e2 != c) t *= hv[e2][mm[e2]];
                            const int m = mm[c];
                            const double d1 = m >= 1 ? hC<double>(m) * hv[c][m >= 1 ? m - 1 : 0] : 0.0;
                            const double d2 = m >= 2 ? hE<double>(m) * hv[c][m >= 2 ? m - 2 : 0] : 0.0;
                            gd[c] += d1 * t;
                            sd[c] += d2 * t;
                        }
                    });
#pragma unroll
                    for (int c = 0; c < DIM; ++c) {
                        dd[q * DIM + c] = T(gd[c]);
                        sdd[q * DIM + c] = T(sd[c]);
                    }
                }
                __syncwarp();
            }
        }

        // positions in shared memory for the pair loop (the Slater scratch is free again)
        double *xs = A;
        for (int c = lane; c < D; c += 32) xs[c] = (double)x[c];
        __syncwarp();

        // pair sums: lanes over particles i; pairs j > i counted once
        double lapj = 0.0, bh2 = 0.0, vint = 0.0, invr = 0.0, sumr = 0.0;
        for (int i = lane; i < N; i += 32) {
            double xi[DIM], r2s = 0.0;
#pragma unroll
            for (int c = 0; c < DIM; ++c) { xi[c] = xs[i * DIM + c]; r2s += xi[c] * xi[c]; }
            const double ri = sqrt(r2s);
            invr += 1.0 / ri;
            sumr += ri;
            double g[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) g[c] = 0.0;
            const unsigned long long mi = mask[i];
            for (int j = 0; j < N; ++j) {
                if (j == i) continue;
                double dxv[DIM], r2 = 0.0;
#pragma unroll
                for (int c = 0; c < DIM; ++c) { dxv[c] = xi[c] - xs[j * DIM + c]; r2 += dxv[c] * dxv[c]; }
                const double ir = rsqrt(r2), r = r2 * ir;
                if (flags & F_PADE) {
                    const double beta = same_spin(i, j, N) ? P.beta_same : P.beta_anti;
                    const double gp = ((flags & Q_PADE_STALE) && !((mi >> j) & 1ull)) ? P.gamma_prev : P.gamma;
                    const double f1 = 1.0 / (1.0 + gp * r), f = beta * f1 * f1, h = r * f1;
#pragma unroll
                    for (int c = 0; c < DIM; ++c) g[c] += f * dxv[c] * ir;
                    if (j > i) {
                        lapj += 2.0 * f * ((double)DIM - (1.0 + 2.0 * P.gamma * h)) * ir;
                        bh2 += beta * h * h;
                    }
                }
                if ((flags & F_COULOMB) && j > i) vint += ir;
            }
            if (flags & F_PADE)
#pragma unroll
                for (int c = 0; c < DIM; ++c) gj[i * DIM + c] = T(g[c]);
        }
        lapj = warp_sum(lapj);
        bh2 = warp_sum(bh2);
        vint = warp_sum(vint);
        invr = warp_sum(invr);
        sumr = warp_sum(sumr);
        __syncwarp();
        if (mode == RB_INIT && P.sampling == SAMPLER_IS) {
            // ImportanceSampling::initialize: F = 2 * sum_e grad_e
            for (int c = lane; c < D; c += 32) {
                double G = 0.0;
                if (flags & F_GAUSS) G += -wa * (double)x[c];
                if (K > 0) G += (double)dd[c];
                if (flags & F_PADE) G += (double)gj[c];
                if (flags & F_HYDROGENLIKE) {
                    const int q = c / DIM;
                    double r2s = 0.0;
#pragma unroll
                    for (int e2 = 0; e2 < DIM; ++e2) r2s += (double)x[q * DIM + e2] * (double)x[q * DIM + e2];
                    G += -az * (double)x[c] / sqrt(r2s);
                }
                fc[c] = T(2.0 * G);
            }
        }
        // max over lanes
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            drift_num = fmax(drift_num, __shfl_xor_sync(FULL, drift_num, o));
            drift_den = fmax(drift_den, __shfl_xor_sync(FULL, drift_den, o));
        }
        status = __reduce_or_sync(FULL, status);
        if (lane == 0) {
            double *sc = P.scal + (size_t)w * NSCAL;
            sc[SC_SUMX2] = sumx2;
            sc[SC_LAPJ] = lapj;
            sc[SC_BH2] = bh2;
            sc[SC_VINT] = vint;
            sc[SC_INVR] = invr;
            sc[SC_LOGDET] = logdet;
            sc[SC_SUMR] = sumr;
            if (drift) drift[w] = fmax(drift[w], drift_den > 0.0 ? drift_num / drift_den : 0.0);
            if (status) P.status[w] |= status;
        }
        __syncwarp();
    }
}

// The MLP Jastrow part of a rebuild, after rebuild_kernel (which leaves the Jastrow
// gradient vector and Laplacian sum at zero for these systems): every ordered pair's
// (u, u', u'') and every particle's (chi, chi', chi'') from the FP32 network into the
// walker's cache, the gradient vector gj, the Laplacian sum, and at initialisation
// the Jastrow part of the importance-sampling force.  One warp per walker.
template <typename T, int DIM>
__global__ void __launch_bounds__(128) rebuild_mlp_kernel(const RebuildArgs a)
{
    const Params &P = a.P;
    const Layout L = P.L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int w = blockIdx.x * 4 + wib;
    if (w >= P.W) return;
    const int N = P.N;
    const float *wt = P.mlpw;
    T *rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
    const T *x = rec + L.off_x;
    T *gj = rec + L.off_gj, *fc = rec + L.off_fc;
    float *cache = P.mlp_cache + (size_t)w * P.mlp_cache_stride, *oc = cache + (size_t)N * N * 3;
    for (int i = 0; i < N; ++i) {
        double r2 = 0.0;
#pragma unroll
        for (int c = 0; c < DIM; ++c) r2 += (double)x[i * DIM + c] * (double)x[i * DIM + c];
        float c0, c1, c2;
        mlp_body(wt, wt + MW_V2T, (float)sqrt(r2), lane, c0, c1, c2);
        if (lane == 0) {
            oc[i * 3] = c0;
            oc[i * 3 + 1] = c1;
            oc[i * 3 + 2] = c2;
        }
    }
    __syncwarp();
    double lap = 0.0;
    for (int i = lane; i < N; i += 32) {
        double g[DIM], ri2 = 0.0;
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            g[c] = 0.0;
            ri2 += (double)x[i * DIM + c] * (double)x[i * DIM + c];
        }
        for (int j = 0; j < N; ++j) {
            if (j == i) continue;
            double dxv[DIM], r2 = 0.0;
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                dxv[c] = (double)x[i * DIM + c] - (double)x[j * DIM + c];
                r2 += dxv[c] * dxv[c];
            }
            const double r = sqrt(r2);
            const bool same = same_spin(i, j, N);
            float u, du, ddu;
            mlp_pair(wt, (float)r, same ? 1.0f : 0.0f, mlp_cusp(DIM, same), u, du, ddu);
            float *c3 = cache + (size_t)(i * N + j) * 3;
            c3[0] = u;
            c3[1] = du;
            c3[2] = ddu;
#pragma unroll
            for (int c = 0; c < DIM; ++c) g[c] += du * dxv[c] / r;
            lap += ddu + (DIM - 1) * du / r;  // grad_i^2 u(r_ij); every ordered pair once
        }
        const double ri = sqrt(ri2), dc = oc[i * 3 + 1];
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            const double gc = g[c] + dc * (double)x[i * DIM + c] / ri;
            gj[i * DIM + c] = T(gc);
            if (a.mode == RB_INIT && P.sampling == SAMPLER_IS) fc[i * DIM + c] += T(2.0 * gc);
        }
        lap += oc[i * 3 + 2] + (DIM - 1) * dc / ri;
    }
    lap = warp_sum(lap);
    if (lane == 0) P.scal[(size_t)w * NSCAL + SC_LAPJ] = lap;
}

template <typename T, int DIM, int K>
__global__ void __launch_bounds__(128, 3) rebuild_kernel(const RebuildArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5;
    rebuild_walkers<T, DIM, K>(a.P, a.mode, a.drift, smem_raw + (size_t)wib * a.smem_per_warp,
                               blockIdx.x * a.wpb + wib, a.P.W, gridDim.x * a.wpb);
}

// ------------------------------------------------------------------ evaluation

struct EvalArgs {
    Params P;
    int p_max;
    double *grad, *lap, *pgrad, *energies;  // W x E x D, W x E, W x E x p_max, W x 3
};

// Per-element gradient/Laplacian/parameter gradient and energy parts of every
// walker from its carried state (after a rebuild or a probe move).
template <typename T, int DIM, int K>
__global__ void eval_kernel(const EvalArgs a)
{
    const Params &P = a.P;
    const Layout L = P.L;
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= P.W) return;
    const T *rec = reinterpret_cast<const T *>(P.state) + (size_t)w * L.rec;
    const T *x = rec + L.off_x, *dd = rec + L.off_dd, *sdd = rec + L.off_sdd, *gj = rec + L.off_gj;
    const double *sc = P.scal + (size_t)w * NSCAL;
    const int D = L.D, E = P.n_elem, flags = P.flags;
    const double wa = P.omega * P.alpha, az = P.alpha_h * P.Z;
    double gsum2 = 0.0, slap = 0.0;
    for (int c = lane; c < D; c += 32) {
        double G = 0.0;
        const int q = c / DIM;
        double rq = 0.0;
        for (int e2 = 0; e2 < DIM; ++e2) rq += (double)x[q * DIM + e2] * (double)x[q * DIM + e2];
        rq = sqrt(rq);
        for (int e = 0; e < E; ++e) {
            double g = 0.0;
            switch (P.elem_kind[e]) {
            case 0: g = -wa * (double)x[c]; break;
            case 1: g = (double)dd[c]; break;
            case 2: g = (double)gj[c]; break;
            case 6: g = -az * (double)x[c] / rq; break;
            default: break;
            }
            a.grad[((size_t)w * E + e) * D + c] = g;
            G += g;
        }
        gsum2 += G * G;
        if (K > 0) slap += (double)sdd[c] - (double)dd[c] * (double)dd[c];
    }
    gsum2 = warp_sum(gsum2);
    slap = warp_sum(slap);
    if (lane == 0) {
        double lapsum = 0.0;
        for (int e = 0; e < E; ++e) {
            double l = 0.0;
            double *pg = a.pgrad + ((size_t)w * E + e) * a.p_max;
            for (int j = 0; j < a.p_max; ++j) pg[j] = 0.0;
            switch (P.elem_kind[e]) {
            case 0: l = -wa * D; pg[0] = -0.5 * P.omega * sc[SC_SUMX2]; break;
            case 1: l = slap; break;
            case 2: l = sc[SC_LAPJ]; pg[0] = ((flags & Q_PADE_DGAMMA) ? -0.5 : -1.0) * sc[SC_BH2]; break;
            case 6: l = -2.0 * az * sc[SC_INVR]; pg[0] = -P.Z * sc[SC_SUMR]; break;
            default: break;
            }
            a.lap[(size_t)w * E + e] = l;
            lapsum += l;
        }
        double *en = a.energies + (size_t)w * 3;
        en[0] = -0.5 * (lapsum + gsum2);
        en[1] = (flags & F_ATOM) ? -P.Z * sc[SC_INVR] : 0.5 * P.omega * P.omega * sc[SC_SUMX2];
        en[2] = (flags & F_COULOMB) ? sc[SC_VINT] : 0.0;
    }
}

// ------------------------------------------------------------------ initial state

// Per-walker Philox stream tag 1: RandomNormal N(0, sd) (randomnormal.cpp:19 uses
// sd = 1/omega) or RandomUniform U[0, 1) (randomuniform.cpp:18).
template <typename T>
__global__ void initial_positions_kernel(Layout L, int W, void *state, unsigned long long seed,
                                         int normal, double sd, int walker_offset)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * L.D) return;
    const int w = i / L.D, c = i - w * L.D;
    const uint4 v = philox(make_uint4((uint32_t)c, 0u, (uint32_t)(w + walker_offset), 1u),
                           make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    double val;
    if (normal) {
        const double u1 = ((double)v.x + 1.0) * TWO_M32, u2 = v.y * TWO_M32;
        val = sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    } else {
        val = v.x * TWO_M32;
    }
    reinterpret_cast<T *>(state)[(size_t)w * L.rec + L.off_x + c] = T(val);
}

// Caller positions (W x D doubles, device) into the walker records, and back:
// only the positions cross the host link, the rest of the record stays on the device.
template <typename T>
__global__ void scatter_positions_kernel(Layout L, int W, const double *__restrict__ pos, void *state)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)W * L.D) return;
    const size_t w = i / L.D, c = i - w * L.D;
    reinterpret_cast<T *>(state)[w * L.rec + L.off_x + c] = T(pos[i]);
}

template <typename T>
__global__ void gather_positions_kernel(Layout L, int W, const void *state, double *__restrict__ pos)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)W * L.D) return;
    const size_t w = i / L.D, c = i - w * L.D;
    pos[i] = (double)reinterpret_cast<const T *>(state)[w * L.rec + L.off_x + c];
}

// FMA throughput calibration: FMA_CHAINS independent register chains per thread.
constexpr int FMA_CHAINS = 8;
template <typename R>
__global__ void fma_peak_kernel(R *out, int iters, R m)
{
    R v[FMA_CHAINS];
#pragma unroll
    for (int i = 0; i < FMA_CHAINS; ++i) v[i] = R(threadIdx.x + i);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < FMA_CHAINS; ++i) v[i] = v[i] * m + m;
    R s = R(0);
#pragma unroll
    for (int i = 0; i < FMA_CHAINS; ++i) s += v[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// ------------------------------------------------------------------ dispatch

struct KernelSet {
    const void *sweep = nullptr, *rebuild = nullptr, *eval = nullptr, *initpos = nullptr;
    const void *sweep_plain = nullptr;  // production sweep: no probe, replay or recording
    const void *scatter = nullptr, *gather = nullptr;  // positions in and out of the records
    const void *rebuild_mlp = nullptr;                  // MLP Jastrow dot: completes each rebuild
    int seg = 1;                                        // walkers per warp of sweep_plain
    const void *sweep_plain1 = nullptr;                 // production sweep, one walker per warp
    const void *sweep_plain2 = nullptr;                 // two walkers per warp (dots of N <= 12), or null
    const void *sweep_owner = nullptr;                  // production dot sweep, owner form, or null
    int owner_smem = 0;                                 // its shared bytes per warp
};

template <typename T, int DIM, int K, int FX>
KernelSet make_set()
{
    KernelSet s;
    s.sweep = reinterpret_cast<const void *>(&sweep_kernel<T, DIM, K, FX, false>);
    if constexpr (FX != 0 && FX != FX_MLP_DOT && DIM == 2 && K >= 1) {
        // compiled-in dots: four (N <= 6), two (N <= 30) or one walker per warp by
        // default (two on request for N = 42 and 56: rows in two passes, measured at
        // 1.05x and 0.89x, the 5-9 KB records of two walkers halving the warps per SM)
        s.sweep_plain2 = reinterpret_cast<const void *>(&sweep_kernel<T, DIM, K, FX, true, 2>);
        s.sweep_plain1 = reinterpret_cast<const void *>(&sweep_kernel<T, DIM, K, FX, true>);
        if constexpr (K >= 4) {
            // the owner form: the default for one walker per warp (N = 42, 56), on request
            // for N = 20 and 30
            s.sweep_owner = reinterpret_cast<const void *>(&owner_sweep_kernel<T, K, FX>);
            s.owner_smem = owner_smem_per_warp(K, (int)sizeof(T));
        }
        if constexpr (K <= 2) {
            s.sweep_plain = reinterpret_cast<const void *>(&sweep_kernel<T, DIM, K, FX, true, 4>);
            s.seg = 4;
        } else if constexpr (K <= 5) {
            s.sweep_plain = s.sweep_plain2;
            s.seg = 2;
        } else {
            s.sweep_plain = s.sweep_plain1;
            s.seg = 1;
        }
    } else if constexpr (FX != 0) {
        s.sweep_plain = s.sweep_plain1 = reinterpret_cast<const void *>(&sweep_kernel<T, DIM, K, FX, true>);
    } else {
        s.sweep_plain = s.sweep_plain1 = s.sweep;
    }
    s.rebuild = reinterpret_cast<const void *>(&rebuild_kernel<T, DIM, K>);
    s.eval = reinterpret_cast<const void *>(&eval_kernel<T, DIM, K>);
    s.initpos = reinterpret_cast<const void *>(&initial_positions_kernel<T>);
    s.scatter = reinterpret_cast<const void *>(&scatter_positions_kernel<T>);
    s.gather = reinterpret_cast<const void *>(&gather_positions_kernel<T>);
    return s;
}

template <typename T, int K>
bool select_2d(int flags, KernelSet &out)
{
    if constexpr (sizeof(T) == 4 && K >= 1 && K <= 5) {
        if (flags == FX_MLP_DOT) {
            out = make_set<T, 2, K, FX_MLP_DOT>();
            out.rebuild_mlp = reinterpret_cast<const void *>(&rebuild_mlp_kernel<T, 2>);
            return true;
        }
    }
    if (K > 0 && flags == FX_DOT_COMPAT) { out = make_set<T, 2, K, (K > 0 ? FX_DOT_COMPAT : 0)>(); return true; }
    if (K > 0 && flags == FX_DOT_CORRECTED) { out = make_set<T, 2, K, (K > 0 ? FX_DOT_CORRECTED : 0)>(); return true; }
    out = make_set<T, 2, K, 0>();
    return true;
}

// Kernel set for (dimension, Hermite shells, flags) in precision T.
template <typename T>
bool select_kernels(int dim, int K, int flags, KernelSet &out)
{
    if (dim == 2) {
        switch (K) {
        case 0: return select_2d<T, 0>(flags, out);
        case 1: return select_2d<T, 1>(flags, out);
        case 2: return select_2d<T, 2>(flags, out);
        case 3: return select_2d<T, 3>(flags, out);
        case 4: return select_2d<T, 4>(flags, out);
        case 5: return select_2d<T, 5>(flags, out);
        case 6: return select_2d<T, 6>(flags, out);
        case 7: return select_2d<T, 7>(flags, out);
        default: return false;
        }
    }
    if (dim == 3) {
        switch (K) {
        case 0: out = make_set<T, 3, 0, 0>(); return true;
        case 1: out = make_set<T, 3, 1, 0>(); return true;
        case 2: out = make_set<T, 3, 2, 0>(); return true;
        case 3: out = make_set<T, 3, 3, 0>(); return true;
        case 4: out = make_set<T, 3, 4, 0>(); return true;
        default: return false;
        }
    }
    return false;
}

}  // namespace vmc
