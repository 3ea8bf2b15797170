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
//   inv[2][n][n]  inverse Slater blocks, inv[b][o][i] = A_b^{-1}(o, i) for orbital o,
//                 particle i of spin block b (m_slaterMatrixInverse, n x N)
//
// plus FP64 per-walker scalars (running sums, see SC_*), a 64-bit per-particle mask
// of Pade pairs computed with the current gamma, and the Philox step counter.
#pragma once
#include "vmc_device.cuh"

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
};

__host__ __device__ inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

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
    L.rec = round_up(L.off_inv + 2 * n * n, a);
    return L;
}

constexpr int MAX_ELEM = 8;
constexpr int MAX_N = 64;

struct Params {
    Layout L;
    int W, N, n_elem, ep, nacc;
    int elem_kind[MAX_ELEM];  // element kinds in configuration order
    int flags, sampling;
    double omega, alpha, gamma, gamma_prev, alpha_h, Z;
    double step;               // stepLength (brute force) or dt (importance sampling)
    int idx_alpha, idx_gamma, idx_alpha_h;  // parameter slots (e*p_max + j) or -1
    double beta_same, beta_anti;            // Pade spin coefficients
    // device buffers
    void *state;               // W x L.rec elements of T
    double *scal;              // W x NSCAL
    unsigned long long *mask;  // W x N
    unsigned long long *counter;  // W Philox step counters
    double *acc;               // W x nacc x 2 (sum, compensation)
    unsigned *status;          // W
};

struct SweepArgs {
    Params P;
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
};

// ------------------------------------------------------------------ helpers

template <typename T>
__device__ __forceinline__ void copy_in(T *dst, const T *src, int n_elems, int lane)
{
    const int nv = n_elems * (int)sizeof(T) / 16;
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    for (int i = lane; i < nv; i += 32) d[i] = s[i];
}

__device__ __forceinline__ bool same_spin(int i, int j, int N)
{
    const int h = N >> 1;
    return (i < h) == (j < h);
}

// ------------------------------------------------------------------ sweep kernel

template <typename T, int DIM, int K>
__global__ void __launch_bounds__(256) sweep_kernel(const SweepArgs a)
{
    constexpr int NO = K > 0 ? Shells<DIM, K>::n : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Params &P = a.P;
    const Layout L = P.L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T *sm = reinterpret_cast<T *>(smem_raw + (size_t)wib * a.smem_per_warp);
    unsigned long long *smask = reinterpret_cast<unsigned long long *>(sm + L.rec);
    T *x = sm + L.off_x, *fc = sm + L.off_fc, *dd = sm + L.off_dd, *sdd = sm + L.off_sdd;
    T *gj = sm + L.off_gj, *inv = sm + L.off_inv;
    const int N = P.N, D = L.D, flags = P.flags;
    const bool is = P.sampling == SAMPLER_IS;
    const T wa = T(P.omega * P.alpha);
    const T gam = T(P.gamma), gamp = T(P.gamma_prev);
    const T az = T(P.alpha_h * P.Z);
    const double half_dt = 0.5 * P.step, sq_dt = sqrt(P.step);
    const uint2 key = make_uint2((uint32_t)a.seed, (uint32_t)(a.seed >> 32));

    for (int w = blockIdx.x * a.wpb + wib; w < P.W; w += gridDim.x * a.wpb) {
        T *g_rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
        copy_in(sm, g_rec, L.rec, lane);
        for (int j = lane; j < N; j += 32) smask[j] = P.mask[(size_t)w * N + j];
        double sc[NSCAL];
#pragma unroll
        for (int i = 0; i < NSCAL; ++i) sc[i] = P.scal[(size_t)w * NSCAL + i];
        double acc_s = 0.0, acc_c = 0.0;
        if (lane < P.nacc) {
            acc_s = P.acc[((size_t)w * P.nacc + lane) * 2];
            acc_c = P.acc[((size_t)w * P.nacc + lane) * 2 + 1];
        }
        unsigned long long ctr = P.counter[w];
        unsigned status = 0;
        __syncwarp();

        for (int s = 0; s < a.steps; ++s) {
            const int it_step = a.step_offset + s;
            // ---- random numbers: coordinate, displacement, acceptance
            int k;
            double r1, r2;
            if (a.probe_k) {
                k = a.probe_k[w];
                r1 = 0.0;
                r2 = 0.0;
            } else if (a.replay) {
                const double *q = a.replay + ((size_t)w * a.replay_stride + a.replay_offset + it_step) * 3;
                k = (int)floor(q[0] * D);
                r1 = q[1];
                r2 = q[2];
            } else {
                const uint4 v = philox(
                    make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), (uint32_t)w, 0u), key);
                ++ctr;
                k = (int)__umulhi(v.x, (unsigned)D);
                if (is) {
                    if (sizeof(T) == 8) {
                        const double u1 = ((double)v.y + 1.0) * TWO_M32, u2 = v.z * TWO_M32;
                        r1 = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
                    } else {
                        const float u1 = ((float)v.y + 1.0f) * 2.3283064e-10f;
                        const float u2 = (float)v.z * 2.3283064e-10f;
                        r1 = (double)(sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2));
                    }
                } else {
                    r1 = v.y * TWO_M32;
                }
                r2 = v.w * TWO_M32;
            }
            const int p = k / DIM, adim = k - p * DIM;
            const T xo = x[k];
            T xpo[DIM], xpn[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) xpo[c] = x[p * DIM + c];

            // ---- gradient of ln Psi along k at the current point (QuantumForce)
            T rpo = T(0);
            if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                T r2s = T(0);
#pragma unroll
                for (int c = 0; c < DIM; ++c) r2s += xpo[c] * xpo[c];
                rpo = vsqrt(r2s);
            }
            T Gk = T(0);
            if (flags & F_GAUSS) Gk += -wa * xo;
            if (K > 0) Gk += dd[k];
            if (flags & F_PADE) Gk += gj[k];
            if (flags & F_HYDROGENLIKE) Gk += -az * xo / rpo;

            T dx, Fn = T(0), Fo = T(0);
            if (a.probe_k) {
                dx = T(a.probe_x[w]) - xo;
            } else if (is) {
                Fn = T(2) * Gk;
                Fo = (flags & Q_IS_GREEN) ? fc[k] : Fn;
                dx = T(half_dt) * Fn + T(r1) * T(sq_dt);
            } else {
                dx = T(10) * (T(r1) - T(0.5)) * T(P.step);
            }
            const T xn = a.probe_k ? T(a.probe_x[w]) : xo + dx;
#pragma unroll
            for (int c = 0; c < DIM; ++c) xpn[c] = (c == adim) ? xn : xpo[c];

            // ---- Slater: S_j = phi(r_p') . inv[:, j]; R = S_pl
            T Sj = T(0), R = T(1);
            int b = 0, pl = 0;
            if constexpr (K > 0) {
                b = p / NO;
                pl = p - b * NO;
                T hv[DIM][K];
#pragma unroll
                for (int c = 0; c < DIM; ++c) hermite_values<K>(xpn[c], hv[c]);
                const T *invb = inv + b * NO * NO;
                if (lane < NO) {
                    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                        T phi = hv[0][m0] * hv[1][m1];
                        if (DIM == 3) phi *= hv[DIM - 1][m2];
                        Sj += phi * invb[o * NO + lane];
                    });
                }
                R = __shfl_sync(FULL, Sj, pl);
            }

            // ---- pair terms of the moved particle (Pade, Coulomb)
            T sum_ratio = T(0), d_lap = T(0), d_bh2 = T(0), d_vint = T(0);
            T gp_new[DIM], gdel[2][DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) { gp_new[c] = T(0); gdel[0][c] = T(0); gdel[1][c] = T(0); }
            if (flags & (F_PADE | F_COULOMB)) {
                const unsigned long long mp = smask[p];
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int j = lane + 32 * jj;
                    if (j < N && j != p) {
                        T dxo[DIM], dxn[DIM], r2o = T(0), r2n = T(0);
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            const T xj = x[j * DIM + c];
                            dxo[c] = xpo[c] - xj;
                            dxn[c] = xpn[c] - xj;
                            r2o += dxo[c] * dxo[c];
                            r2n += dxn[c] * dxn[c];
                        }
                        const T ro = vsqrt(r2o), rn = vsqrt(r2n);
                        const T iro = T(1) / ro, irn = T(1) / rn;
                        if (flags & F_PADE) {
                            const T beta = same_spin(p, j, N) ? T(P.beta_same) : T(P.beta_anti);
                            const T gpair = ((flags & Q_PADE_STALE) && !((mp >> j) & 1ull)) ? gamp : gam;
                            const T fo1 = T(1) / (T(1) + gpair * ro), fo = beta * fo1 * fo1, ho = ro * fo1;
                            const T fn1 = T(1) / (T(1) + gam * rn), fn = beta * fn1 * fn1, hn = rn * fn1;
                            if (!(flags & Q_PADE_RATIO) || j > p) sum_ratio += beta * (hn - ho);
#pragma unroll
                            for (int c = 0; c < DIM; ++c) {
                                const T tn = fn * dxn[c] * irn, to = fo * dxo[c] * iro;
                                gp_new[c] += tn;
                                gdel[jj][c] = to - tn;  // particle j sees -(x_p - x_j)
                            }
                            d_lap += T(2) * fn * (T(DIM) - (T(1) + T(2) * gam * hn)) * irn -
                                     T(2) * fo * (T(DIM) - (T(1) + T(2) * gam * ho)) * iro;
                            d_bh2 += beta * (hn * hn - ho * ho);
                        }
                        if (flags & F_COULOMB) d_vint += irn - iro;
                    }
                }
                if (flags & F_PADE) {
                    sum_ratio = warp_sum(sum_ratio);
                    d_lap = warp_sum(d_lap);
                    d_bh2 = warp_sum(d_bh2);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) gp_new[c] = warp_sum(gp_new[c]);
                }
                if (flags & F_COULOMB) d_vint = warp_sum(d_vint);
            }

            // ---- element ratios, multiplied in configuration order
            T rpn = T(0);
            if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                T r2s = T(0);
#pragma unroll
                for (int c = 0; c < DIM; ++c) r2s += xpn[c] * xpn[c];
                rpn = vsqrt(r2s);
            }
            double prob = 1.0;
            double ratios[MAX_ELEM];
            for (int e = 0; e < P.n_elem; ++e) {
                double r = 1.0;
                switch (P.elem_kind[e]) {
                case 0: r = (double)vexp(wa * (xo * xo - xn * xn)); break;
                case 1: r = (double)(R * R); break;
                case 2: r = (double)vexp(T(2) * sum_ratio); break;
                case 6: r = (double)vexp(T(2) * az * (rpo - rpn)); break;
                default: break;
                }
                ratios[e] = r;
                prob *= r;
            }

            bool accept;
            if (a.probe_k) {
                accept = true;
                if (lane == 0)
                    for (int e = 0; e < P.n_elem; ++e) a.probe_ratio[(size_t)w * P.n_elem + e] = ratios[e];
            } else {
                double wgt = prob;
                if (is) {
                    if (flags & Q_IS_GREEN) {
                        wgt = (exp(0.5 * (double)(Fo - Fn) * (double)dx) + 1.0) * prob;
                    } else {
                        // Fokker-Planck Green's function ratio; needs F_k at the new point
                        T gy = T(0);
                        if (flags & F_GAUSS) gy += -wa * xn;
                        if (flags & F_PADE) gy += gp_new[adim];
                        if (flags & F_HYDROGENLIKE) gy += -az * xn / rpn;
                        if constexpr (K > 0) {
                            T hv[DIM][K], h1[DIM][K], h2u[DIM][K];
#pragma unroll
                            for (int c = 0; c < DIM; ++c) {
                                hermite_values<K>(xpn[c], hv[c]);
                                hermite_derivs<K>(hv[c], h1[c], h2u[c]);
                            }
                            T dphi = T(0);
                            const T *invb = inv + b * NO * NO;
                            if (lane < NO) {
                                for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                                    if (o == lane) {
                                        const int mm[3] = {m0, m1, m2};
                                        T v = T(1);
#pragma unroll
                                        for (int c = 0; c < DIM; ++c) v *= (c == adim) ? h1[c][mm[c]] : hv[c][mm[c]];
                                        dphi = v * invb[o * NO + pl];
                                    }
                                });
                            }
                            gy += warp_sum(dphi) / R;
                        }
                        const double fy = 2.0 * (double)gy, fo2 = (double)Fn;
                        wgt = prob * exp(0.5 * (fo2 + fy) * (0.25 * P.step * (fo2 - fy) - (double)dx));
                    }
                }
                if (wgt != wgt) status |= ST_BAD_RATIO;
                accept = !(wgt < r2);
            }

            if (accept) {
                // ---- positions and running scalars
                __syncwarp();
                if (lane == 0) {
                    x[k] = xn;
                    if (is) fc[k] = Fn;
                }
                sc[SC_SUMX2] += (double)xn * (double)xn - (double)xo * (double)xo;
                if (flags & (F_HYDROGENLIKE | F_ATOM)) {
                    sc[SC_INVR] += 1.0 / (double)rpn - 1.0 / (double)rpo;
                    sc[SC_SUMR] += (double)rpn - (double)rpo;
                }
                // ---- Sherman-Morrison update of block b (slaterdeterminant.cpp:165-175)
                if constexpr (K > 0) {
                    T *invb = inv + b * NO * NO;
                    const T rinv = T(1) / R;
                    const T coef = Sj * rinv;
                    const T colp = lane < NO ? invb[lane * NO + pl] : T(0);
                    __syncwarp();
#pragma unroll
                    for (int o = 0; o < NO; ++o) {
                        const T c = __shfl_sync(FULL, colp, o);
                        if (lane < NO) {
                            const T v = invb[o * NO + lane];
                            invb[o * NO + lane] = (lane == pl) ? c * rinv : v - coef * c;
                        }
                    }
                    sc[SC_LOGDET] += log(fabs((double)R));
                    __syncwarp();
                    // ---- derivative refresh of the block (slaterdeterminant.cpp:155-163)
                    if (lane < NO) {
                        const int q = b * NO + lane;
                        T hv[DIM][K], h1[DIM][K], h2u[DIM][K];
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            hermite_values<K>(x[q * DIM + c], hv[c]);
                            hermite_derivs<K>(hv[c], h1[c], h2u[c]);
                        }
                        T gd[DIM], sd[DIM];
#pragma unroll
                        for (int c = 0; c < DIM; ++c) { gd[c] = T(0); sd[c] = T(0); }
                        for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                            const T iv = invb[o * NO + lane];
                            if (DIM == 2) {
                                const T t0 = hv[1][m1] * iv, t1 = hv[0][m0] * iv;
                                gd[0] += h1[0][m0] * t0;
                                sd[0] += h2u[0][m0] * t0;
                                gd[1] += h1[1][m1] * t1;
                                sd[1] += h2u[1][m1] * t1;
                            } else {
                                const T t0 = hv[1][m1] * hv[DIM - 1][m2] * iv;
                                const T t1 = hv[0][m0] * hv[DIM - 1][m2] * iv;
                                const T t2 = hv[0][m0] * hv[1][m1] * iv;
                                gd[0] += h1[0][m0] * t0;
                                sd[0] += h2u[0][m0] * t0;
                                gd[1] += h1[1][m1] * t1;
                                sd[1] += h2u[1][m1] * t1;
                                gd[DIM - 1] += h1[DIM - 1][m2] * t2;
                                sd[DIM - 1] += h2u[DIM - 1][m2] * t2;
                            }
                        });
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            dd[q * DIM + c] = gd[c];
                            sdd[q * DIM + c] = sd[c];
                        }
                    }
                }
                // ---- Pade gradient vector, running sums and pair masks
                if (flags & F_PADE) {
#pragma unroll
                    for (int jj = 0; jj < 2; ++jj) {
                        const int j = lane + 32 * jj;
                        if (j < N && j != p) {
#pragma unroll
                            for (int c = 0; c < DIM; ++c) gj[j * DIM + c] += gdel[jj][c];
                            smask[j] |= (1ull << p);
                        }
                    }
                    if (lane == (p & 31)) {
#pragma unroll
                        for (int c = 0; c < DIM; ++c) gj[p * DIM + c] = gp_new[c];
                        smask[p] = ~0ull;
                    }
                    sc[SC_LAPJ] += (double)d_lap;
                    sc[SC_BH2] += (double)d_bh2;
                }
                if (flags & F_COULOMB) sc[SC_VINT] += (double)d_vint;
                __syncwarp();
            }

            // ---- local energy and parameter gradients (Sampler::sample)
            if (it_step >= a.burn_in || a.rec_en) {
                T ks = T(0);
                for (int c = lane; c < D; c += 32) {
                    const T xc = x[c];
                    T G = T(0), lc = T(0);
                    if (flags & F_GAUSS) G += -wa * xc;
                    if (K > 0) {
                        const T g = dd[c];
                        G += g;
                        lc += sdd[c] - g * g;
                    }
                    if (flags & F_PADE) G += gj[c];
                    if (flags & F_HYDROGENLIKE) {
                        const int q = c / DIM;
                        T r2s = T(0);
#pragma unroll
                        for (int e2 = 0; e2 < DIM; ++e2) r2s += x[q * DIM + e2] * x[q * DIM + e2];
                        G += -az * xc / vsqrt(r2s);
                    }
                    ks += G * G + lc;
                }
                const double lap = (double)warp_sum(ks) + sc[SC_LAPJ] * ((flags & F_PADE) ? 1.0 : 0.0) +
                                   ((flags & F_GAUSS) ? -(double)wa * D : 0.0) +
                                   ((flags & F_HYDROGENLIKE) ? -2.0 * (double)az * sc[SC_INVR] : 0.0);
                const double ekin = -0.5 * lap;
                const double vext = (flags & F_ATOM) ? -P.Z * sc[SC_INVR]
                                                     : 0.5 * P.omega * P.omega * sc[SC_SUMX2];
                const double vint = (flags & F_COULOMB) ? sc[SC_VINT] : 0.0;
                const double el = ekin + vext + vint;
                if (el != el) status |= ST_NAN_ENERGY;
                if (a.rec_en && lane == 0) {
                    double *o = a.rec_en + ((size_t)w * a.rec_stride + it_step) * 3;
                    o[0] = ekin;
                    o[1] = vext;
                    o[2] = vint;
                }
                if (it_step >= a.burn_in) {
                    const bool win = it_step > a.win_lo && it_step < a.win_hi;
                    double q = 0.0;
                    const int i = lane;
                    if (i < 9) {
                        q = i == 0 ? el : i == 1 ? el * el : i == 2 ? ekin : i == 3 ? ekin * ekin
                          : i == 4 ? vext : i == 5 ? vext * vext : i == 6 ? vint : i == 7 ? vint * vint
                          : (accept ? 1.0 : 0.0);
                    } else if (win && i < 9 + 2 * P.ep) {
                        const int j = (i - 9) % P.ep;
                        double g = 0.0;
                        if (j == P.idx_alpha) g = -0.5 * P.omega * sc[SC_SUMX2];
                        else if (j == P.idx_gamma) g = ((flags & Q_PADE_DGAMMA) ? -0.5 : -1.0) * sc[SC_BH2];
                        else if (j == P.idx_alpha_h) g = -P.Z * sc[SC_SUMR];
                        q = (i - 9 < P.ep) ? g : g * el;
                    }
                    if (lane < P.nacc) kadd(acc_s, acc_c, q);
                }
            }
            if (a.rec_acc && lane == 0) a.rec_acc[(size_t)w * a.rec_stride + it_step] = accept ? 1 : 0;
        }

        // ---- write the walker back
        __syncwarp();
        {
            const int nv = L.rec * (int)sizeof(T) / 16;
            const uint4 *s4 = reinterpret_cast<const uint4 *>(sm);
            uint4 *d4 = reinterpret_cast<uint4 *>(g_rec);
            for (int i = lane; i < nv; i += 32) d4[i] = s4[i];
        }
        for (int j = lane; j < N; j += 32) P.mask[(size_t)w * N + j] = smask[j];
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NSCAL; ++i) P.scal[(size_t)w * NSCAL + i] = sc[i];
            P.counter[w] = ctr;
        }
        if (lane < P.nacc) {
            P.acc[((size_t)w * P.nacc + lane) * 2] = acc_s;
            P.acc[((size_t)w * P.nacc + lane) * 2 + 1] = acc_c;
        }
        status = __reduce_or_sync(FULL, status);
        if (lane == 0 && status) P.status[w] |= status;
        __syncwarp();
    }
}

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
template <typename T, int DIM, int K>
__global__ void __launch_bounds__(128) rebuild_kernel(const RebuildArgs a)
{
    constexpr int NO = K > 0 ? Shells<DIM, K>::n : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Params &P = a.P;
    const Layout L = P.L;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *A = reinterpret_cast<double *>(smem_raw + (size_t)wib * a.smem_per_warp);
    double *B = A + NO * NO;
    const int N = P.N, D = L.D, flags = P.flags;
    const double wa = P.omega * P.alpha, az = P.alpha_h * P.Z;

    for (int w = blockIdx.x * a.wpb + wib; w < P.W; w += gridDim.x * a.wpb) {
        T *rec = reinterpret_cast<T *>(P.state) + (size_t)w * L.rec;
        const T *x = rec + L.off_x;
        T *fc = rec + L.off_fc, *dd = rec + L.off_dd, *sdd = rec + L.off_sdd, *gj = rec + L.off_gj;
        T *inv = rec + L.off_inv;
        unsigned long long *mask = P.mask + (size_t)w * N;
        if (a.mode == RB_INIT)
            for (int j = lane; j < N; j += 32) mask[j] = ~0ull;
        __syncwarp();
        unsigned status = 0;
        double sumx2 = 0.0;
        for (int c = lane; c < D; c += 32) sumx2 += (double)x[c] * (double)x[c];
        sumx2 = warp_sum(sumx2);
        double logdet = 0.0, drift_num = 0.0, drift_den = 0.0;

        if constexpr (K > 0) {
            for (int b = 0; b < 2; ++b) {
                // A[i][o] = phi_o(r_i), i in block b
                if (lane < NO) {
                    const int q = b * NO + lane;
                    double hv[DIM][K];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) hermite_values<K>((double)x[q * DIM + c], hv[c]);
                    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                        double phi = hv[0][m0] * hv[1][m1];
                        if (DIM == 3) phi *= hv[DIM - 1][m2];
                        A[lane * NO + o] = phi;
                    });
                    for (int o = 0; o < NO; ++o) B[lane * NO + o] = (o == lane) ? 1.0 : 0.0;
                }
                __syncwarp();
                for (int c = 0; c < NO; ++c) {
                    double v = (lane >= c && lane < NO) ? fabs(A[lane * NO + c]) : -1.0;
                    int idx = lane;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const double v2 = __shfl_xor_sync(FULL, v, o);
                        const int i2 = __shfl_xor_sync(FULL, idx, o);
                        if (v2 > v || (v2 == v && i2 < idx)) { v = v2; idx = i2; }
                    }
                    const int pr = idx;
                    if (!(v > 0.0)) status |= ST_SINGULAR;
                    __syncwarp();
                    if (pr != c && lane < NO) {
                        double t = A[c * NO + lane]; A[c * NO + lane] = A[pr * NO + lane]; A[pr * NO + lane] = t;
                        t = B[c * NO + lane]; B[c * NO + lane] = B[pr * NO + lane]; B[pr * NO + lane] = t;
                    }
                    __syncwarp();
                    const double piv = A[c * NO + c];
                    logdet += log(fabs(piv));
                    const double ip = 1.0 / piv;
                    __syncwarp();
                    if (lane < NO) { A[c * NO + lane] *= ip; B[c * NO + lane] *= ip; }
                    __syncwarp();
                    for (int r = 0; r < NO; ++r) {
                        if (r == c) continue;
                        const double f = A[r * NO + c];
                        __syncwarp();
                        if (lane < NO && f != 0.0) {
                            A[r * NO + lane] -= f * A[c * NO + lane];
                            B[r * NO + lane] -= f * B[c * NO + lane];
                        }
                        __syncwarp();
                    }
                }
                // B[o][i] = A^{-1}(o, i): store, measure drift of the carried inverse
                T *invb = inv + b * NO * NO;
                if (lane < NO) {
                    for (int o = 0; o < NO; ++o) {
                        const double nv = B[o * NO + lane];
                        if (a.mode == RB_REFRESH) {
                            drift_num = fmax(drift_num, fabs((double)invb[o * NO + lane] - nv));
                            drift_den = fmax(drift_den, fabs(nv));
                        }
                        invb[o * NO + lane] = T(nv);
                    }
                    // derivative vectors with the FP64 inverse
                    const int q = b * NO + lane;
                    double hv[DIM][K], h1[DIM][K], h2u[DIM][K];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) {
                        hermite_values<K>((double)x[q * DIM + c], hv[c]);
                        hermite_derivs<K>(hv[c], h1[c], h2u[c]);
                    }
                    double gd[DIM], sd[DIM];
#pragma unroll
                    for (int c = 0; c < DIM; ++c) { gd[c] = 0.0; sd[c] = 0.0; }
                    for_each_orbital<DIM, K>([&](int o, int m0, int m1, int m2) {
                        const int mm[3] = {m0, m1, m2};
                        const double iv = B[o * NO + lane];
#pragma unroll
                        for (int c = 0; c < DIM; ++c) {
                            double t = iv;
#pragma unroll
                            for (int e2 = 0; e2 < DIM; ++e2)
                                if (e2 != c) t *= hv[e2][mm[e2]];
                            gd[c] += h1[c][mm[c]] * t;
                            sd[c] += h2u[c][mm[c]] * t;
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

        // pair sums: lanes over particles i; pairs j > i counted once
        double lapj = 0.0, bh2 = 0.0, vint = 0.0, invr = 0.0, sumr = 0.0;
        for (int i = lane; i < N; i += 32) {
            double xi[DIM], r2s = 0.0;
#pragma unroll
            for (int c = 0; c < DIM; ++c) { xi[c] = (double)x[i * DIM + c]; r2s += xi[c] * xi[c]; }
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
                for (int c = 0; c < DIM; ++c) { dxv[c] = xi[c] - (double)x[j * DIM + c]; r2 += dxv[c] * dxv[c]; }
                const double r = sqrt(r2), ir = 1.0 / r;
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
        if (a.mode == RB_INIT && P.sampling == SAMPLER_IS) {
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
            if (a.drift) a.drift[w] = fmax(a.drift[w], drift_den > 0.0 ? drift_num / drift_den : 0.0);
            if (status) P.status[w] |= status;
        }
        __syncwarp();
    }
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
                                         int normal, double sd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * L.D) return;
    const int w = i / L.D, c = i - w * L.D;
    const uint4 v = philox(make_uint4((uint32_t)c, 0u, (uint32_t)w, 1u),
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

}  // namespace vmc
