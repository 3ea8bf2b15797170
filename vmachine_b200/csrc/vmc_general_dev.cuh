// General walker path: every wave-function element of the reference on one FP64
// warp-per-walker kernel family, for the systems the quantum-dot sweep does not
// take: SimpleJastrow (simplejastrow.cpp), RBMGaussian (rbmgaussian.cpp),
// RBMProduct (rbmproduct.cpp), and Slater determinants of hydrogen orbitals
// (hydrogenorbital.cpp) or Hermite functions next to those elements.
//
// One warp owns one walker; its record lives in HBM (small systems: it stays in
// L1/L2) and holds the positions, the importance-sampling force cache, the total
// gradient of ln|Psi| at the current positions, the local-energy parts and the
// parameter gradients at the current positions, and the transposed inverse of
// each Slater block.  A proposal computes each element's |Psi'|^2/|Psi|^2 without
// touching the record; an accepted move applies the Sherman-Morrison update to
// the moved particle's block and re-evaluates the walker (gradients, Laplacians,
// energies, parameter gradients) from its new positions, so rejected steps sample
// the stored values.  Every parameter gradient is accumulated (nothing caps the
// parameter count): lanes stride over the accumulators in HBM.
//
// Elements, Hamiltonians, samplers and the reference's quirks follow the CPU
// restatement in oracle/vmc_oracle.c function for function (eval_impl,
// ratio_impl, vmo_run).
//
// The device functions are templated on the walker's real type R: double is the FP64
// path; float is the compiled atom form's mixed-precision sweep, whose record is staged
// in FP32 while the Slater inverse, its contractions and the accumulators stay FP64.
//
// This header holds the path's device functions; vmc_general.cu has its kernels and
// launchers, and the multi-system kernel (vmc_batch.cu) calls gen_sweep_walker.
#pragma once
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <string>

#include <cuda_bf16.h>

#include "vmc_general.hpp"

namespace vmc {

namespace {


constexpr int GEN_WPB = 4;     // warps per CTA
constexpr int GEN_SCR = 256;   // shared reals (R) per warp (a warp of G walkers: GEN_SCR / G each)
// shared scratch of a walker: orbital values at the proposal | moved row | RBM visible
// (sorted) | RBM hidden p_j = 1/(1+e^v) | RBM hidden e^v/(1+e^v); the pair elements'
// per-pair terms reuse it from offset 0 during an evaluation (the compiled atom form
// with four walkers per warp has 64 doubles: the proposal's orbitals and moved row)
constexpr int SCR_PHI = 0, SCR_ROW = 32, SCR_XS = 64, SCR_PN = 128, SCR_NN = 192;

// R: the walker's real type (double; float in the atoms' mixed-precision sweep)
template <typename R>
__device__ __forceinline__ R gen_dist(const R *x, int dim, int i, int j)
{
    R s = R(0);
    for (int c = 0; c < dim; ++c) {
        const R t = x[i * dim + c] - x[j * dim + c];
        s += t * t;
    }
    return sqrt(s);
}

template <typename R>
__device__ __forceinline__ R gen_radius(const R *x, int dim, int i)
{
    R s = R(0);
    for (int c = 0; c < dim; ++c) s += x[i * dim + c] * x[i * dim + c];
    return sqrt(s);
}

// h_m(x), h_m'(x), h_m''(x) of the normalised Hermite functions by the recurrence
// h_{j+1} = A_j x h_j - B_j h_{j-1}; h_m' = C_m h_{m-1}, h_m'' = E_m h_{m-2}.
__device__ __forceinline__ void herm3(int m, double x, double &h, double &h1, double &h2)
{
    double hm2 = 0.0, hm1 = 0.0, hc = 1.0;
    for (int j = 0; j < m; ++j) {
        const double nx = hA<double>(j) * x * hc - hB<double>(j) * hm1;
        hm2 = hm1;
        hm1 = hc;
        hc = nx;
    }
    h = hc;
    h1 = m >= 1 ? hC<double>(m) * hm1 : 0.0;
    h2 = m >= 2 ? hE<double>(m) * hm2 : 0.0;
}

// Value, d/dx_c and d^2/dx_c^2 (c = 0..dim-1) of orbital o at point r.
// Hermite: prod_c h_{m_c}(x_c) (basis.cpp:81-116, argument unscaled, hermite.h:8).
// Hydrogen (3D, hydrogenorbital.cpp:108-394 with alpha = 1, k = Z): a polynomial
// angular factor A (1 or one coordinate) times a radial factor
// R(r) = f(r) exp(-k r / n); derivatives by the chain rule:
//   d_i phi   = (d_i A) R + A R' x_i / r
//   d_i^2 phi = 2 (d_i A) R' x_i / r + A (R'' x_i^2 / r^2 + R' (1/r - x_i^2 / r^3))
template <int GV, typename R = double>
__device__ __forceinline__ void gen_orbital_t(const GenParams &g, int dim_rt, double Z, int o, const R *r,
                                              R &v, R *d1, R *d2)
{
    const int dim = gv_dim(GV, dim_rt);
    if constexpr (GV == GV_ANY) {
        if (g.basis == BASIS_HERMITE) {
            double h[3], h1[3], h2[3];
            for (int c = 0; c < dim; ++c) herm3(g.orb[o][c], r[c], h[c], h1[c], h2[c]);
            v = 1.0;
            for (int c = 0; c < dim; ++c) v *= h[c];
            for (int c = 0; c < dim; ++c) {
                double rest = 1.0;
                for (int c2 = 0; c2 < dim; ++c2)
                    if (c2 != c) rest *= h[c2];
                d1[c] = h1[c] * rest;
                d2[c] = h2[c] * rest;
            }
            return;
        }
    }
    using T = R;
    const int nq = g.orb[o][0], l = g.orb[o][1], m = (int)g.orb[o][2] - 1;
    const T k = T(Z);
    const T rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    T f = T(1), fp = T(0), fpp = T(0);
    if (nq == 2 && l == 0) { f = T(2) - k * rr; fp = -k; }
    if (nq == 3 && l == 0) { f = T(2) * k * k * rr * rr - T(18) * k * rr + T(27); fp = T(4) * k * k * rr - T(18) * k; fpp = T(4) * k * k; }
    if (nq == 3 && l == 1) { f = k * rr - T(6); fp = k; }
    const T a = k * (nq == 1 ? T(1) : nq == 2 ? T(0.5) : T(1.0 / 3.0)), ex = exp(-a * rr), irr = T(1) / rr;
    const T Rr = f * ex, R1 = (fp - a * f) * ex, R2 = (fpp - T(2) * a * fp + a * a * f) * ex;
    const int ca = l == 1 ? (m == 1 ? 0 : m == -1 ? 1 : 2) : -1;  // m = 1: x, -1: y, 0: z
    const T A = ca >= 0 ? r[ca] : T(1);
    v = A * Rr;
    for (int c = 0; c < 3; ++c) {
        const T xc = r[c], u = xc * irr, dA = (c == ca) ? T(1) : T(0);
        d1[c] = dA * Rr + A * R1 * u;
        d2[c] = T(2) * dA * R1 * u + A * (R2 * u * u + R1 * (T(1) - u * u) * irr);
        if (nq == 3 && g.horb3) {
            // compat: the reference's n = 3 "second derivatives" (hydrogenorbital.cpp:351-364),
            // which are not d^2/dx_c^2
            const T kr = k * rr, pre = k * ex / (T(81) * rr * rr * rr);
            d2[c] = l == 0 ? pre * (rr * rr * (T(2) * kr * (T(5) - T(3) * kr) - T(27)) +
                                    xc * xc * (kr * (T(2) * kr * (kr - T(18)) + T(9)) + T(27)))
                           : pre * A * (kr - T(18)) * (kr - T(6)) / rr;
        }
    }
}

__device__ void gen_orbital(const GenParams &g, int dim, double Z, int o, const double *r, double &v,
                            double *d1, double *d2)
{
    gen_orbital_t<GV_ANY, double>(g, dim, Z, o, r, v, d1, d2);
}

// orbital o at r in variant GV: the generic variant calls the out-of-line function,
// the compiled-in variants inline their own
template <int GV, typename R = double>
__device__ __forceinline__ void gen_orb(const GenParams &g, int dim, double Z, int o, const R *r, R &v, R *d1,
                                        R *d2)
{
    if constexpr (GV == GV_ANY)
        gen_orbital(g, dim, Z, o, r, v, d1, d2);
    else
        gen_orbital_t<GV, R>(g, dim, Z, o, r, v, d1, d2);
}

// RBMProduct visible vector: the coordinates, sorted ascending under the
// reference's in-place sort (wavefunction.cpp:40-55; stable, as the oracle's
// insertion sort), with coordinate k replaced by xk_new when k >= 0.
template <typename R>
__device__ void rbm_visible(const R *x, int D, int k, R xk_new, bool sort, R *xs, int lane)
{
    for (int i = lane; i < D; i += 32) {
        const R xi = i == k ? xk_new : x[i];
        int rank = i;
        if (sort) {
            rank = 0;
            for (int j = 0; j < D; ++j) {
                const R xj = j == k ? xk_new : x[j];
                rank += (xj < xi) || (xj == xi && j < i);
            }
        }
        xs[rank] = xi;
    }
    __syncwarp();
}

// hidden activations: v_j = b_j + sum_i W_ij xs_i / sigma^2 (rbmproduct.cpp:191-197),
// p_j = 1 / (e^v + 1), n_j = e^v p_j into the scratch
template <typename R>
__device__ void rbm_hidden(const double *th, int D, int H, R s2, const R *xs, R *pn,
                           R *nn, int lane)
{
    for (int j = lane; j < H; j += 32) {
        R acc = R(0.0);
        for (int i = 0; i < D; ++i) acc += th[H + i + D * j] * xs[i];
        const R v = th[j] + acc / s2, e = exp(v);
        pn[j] = R(1.0) / (e + R(1.0));
        nn[j] = e * pn[j];
    }
    __syncwarp();
}

// Pade-Jastrow gamma of pair (i, j): the previous gamma while the pair is stale
__device__ __forceinline__ double pade_gamma(const Params &P, const unsigned long long *mask, int i, int j,
                                             double gam)
{
    return ((P.flags & Q_PADE_STALE) && !((mask[i] >> j) & 1ull)) ? P.gamma_prev : gam;
}

__device__ __forceinline__ double pade_beta_of(const Params &P, int i, int j)
{
    return same_spin(i, j, P.N) ? P.beta_same : P.beta_anti;
}

// Lanes of the calling thread's segment when a warp carries 32 / SEG walkers of the
// general path (SEG = 32: the whole warp), and sums over them.
template <int SEG>
__device__ __forceinline__ unsigned gen_segmask()
{
    return SEG == 32 ? FULL : (((1u << SEG) - 1u) << ((threadIdx.x & 31) & ~(SEG - 1)));
}

template <int SEG, typename V>
__device__ __forceinline__ V seg_reduce(unsigned mask, V v)
{
#pragma unroll
    for (int o = SEG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// Per-particle sums of pair vectors: tp holds t(i, j) for each pair i < j (pair
// index as pair_of), particle i takes +t(i, j) for j > i and -t(j, i) for j < i, j
// ascending; lanes over particles add the sums to G (and the per-element output).
template <int SEG = 32, typename R = double>
__device__ __forceinline__ void gen_pair_gather(const R *tp, int N, int dim, R *G, double *oge, int lane)
{
    const unsigned segmask = gen_segmask<SEG>();
    __syncwarp(segmask);
    for (int i = lane; i < N; i += SEG) {
        R gi[3] = {R(0), R(0), R(0)};
        for (int j = 0; j < N; ++j) {
            if (j == i) continue;
            const int lo = min(i, j), hi = max(i, j);
            const R *t = tp + (lo * (2 * N - lo - 1) / 2 + hi - lo - 1) * dim;
            for (int c = 0; c < dim; ++c) gi[c] += i < j ? t[c] : -t[c];
        }
        for (int c = 0; c < dim; ++c) {
            G[i * dim + c] += gi[c];
            if (oge) oge[i * dim + c] = gi[c];
        }
    }
    __syncwarp(segmask);  // the scratch is free again for the next element
}

// Evaluate the walker at its positions (eval_impl): per-element gradient,
// Laplacian and parameter gradient, the local-energy parts.  Writes the total
// gradient, energies and parameter gradients into the record and, when given,
// the per-element outputs of one walker (grad E x D, lap E, pgrad E x p_max,
// energies 3).
// moved: the particle whose position changed since the last evaluation (its cached
// orbital derivatives are refreshed), or -1 to refresh every particle's.
template <int GV = GV_ANY, int SEG = 32, typename R = double>
__device__ void gen_evaluate(const Params &P, const GenParams &g, int dim_rt, R *rec,
                             const unsigned long long *mask, R *scr, int lane, double *o_grad,
                             double *o_lap, double *o_pg, double *o_en, const float *mw = nullptr,
                             bool full = true, int moved = -1, const double *inv64 = nullptr)
{
    const int N = P.N, D = g.D, E = P.n_elem, PM = g.p_max, dim = gv_dim(GV, dim_rt);
    const unsigned segmask = gen_segmask<SEG>();
    constexpr int SCR = GEN_SCR * SEG / 32;  // this walker's scratch doubles
    const R *x = rec;
    // the Slater inverse is FP64 in both real types (FP32 walkers keep it apart: its
    // contraction with the orbital Laplacians cancels to a small fraction of its terms)
    const double *inv = inv64;
    if constexpr (std::is_same<R, double>::value)
        if (!inv) inv = rec + g.off_inv;
    R *G = rec + g.off_g, *pg = rec + g.off_pg;
    for (int k = lane; k < D; k += SEG) G[k] = R(0.0);
    // only the accumulated parameters are ever written (padding and the MLP row stay
    // zero from the record's initialisation): clear those
    for (int c = lane; c < g.n_act; c += SEG) pg[g.act[c]] = R(0.0);
    __syncwarp(segmask);
    R lap_total = R(0.0);
    for (int e = 0; e < E; ++e) {
        const double *th = g.theta + (size_t)e * PM;
        R *pge = pg + (size_t)e * PM;
        R lap_l = R(0.0), lap_u = R(0.0);  // lane partial, uniform part
        double *oge = o_grad ? o_grad + (size_t)e * D : nullptr;
        switch (P.elem_kind[e]) {
        case 0: {  // Gaussian (gaussian.cpp:62-78)
            if (!gv_has(GV, 0)) break;
            const R wa = P.omega * th[0];
            R x2 = R(0.0);
            for (int k = lane; k < D; k += SEG) {
                const R gk = -wa * x[k];
                G[k] += gk;
                if (oge) oge[k] = gk;
                x2 += x[k] * x[k];
            }
            x2 = seg_reduce<SEG>(segmask, x2);
            lap_u = -wa * D;
            if (lane == 0) pge[0] = -R(0.5) * P.omega * x2;
            break;
        }
        case 1: {  // Slater determinant (slaterdeterminant.cpp:155-191)
            if (!gv_has(GV, 1)) break;
            const int n = g.n, nd = 2 * dim;
            R *dphi = rec + g.off_dphi;
            // orbital derivatives of the particles that moved (lanes over (particle,
            // orbital)); the other particles' are unchanged in the cache
            const int q0 = moved < 0 ? 0 : moved, nq = moved < 0 ? N : 1;
            for (int t = lane; t < nq * n; t += SEG) {
                const int q = q0 + t / n, o = t - (t / n) * n;
                R v, d1[3], d2[3];
                gen_orb<GV>(g, dim, P.Z, o, x + q * dim, v, d1, d2);
                R *cq = dphi + (size_t)(q * n + o) * nd;
                for (int c = 0; c < dim; ++c) {
                    cq[c] = d1[c];
                    cq[dim + c] = d2[c];
                }
            }
            __syncwarp(segmask);
            for (int q = lane; q < N; q += SEG) {
                const int b = q / n, il = q - b * n;
                const double *row = inv + (size_t)(b * n + il) * n;
                double dd[3] = {0.0, 0.0, 0.0}, sdd[3] = {0.0, 0.0, 0.0};
                for (int o = 0; o < n; ++o) {
                    const R *cq = dphi + (size_t)(q * n + o) * nd;
                    for (int c = 0; c < dim; ++c) {
                        dd[c] += (double)cq[c] * row[o];
                        sdd[c] += (double)cq[dim + c] * row[o];
                    }
                }
                for (int c = 0; c < dim; ++c) {
                    G[q * dim + c] += (R)dd[c];
                    if (oge) oge[q * dim + c] = dd[c];
                    lap_l += (R)(sdd[c] - dd[c] * dd[c]);
                }
            }
            break;
        }
        case 2: {  // Pade-Jastrow (padejastrow.cpp:75-116)
            if (!gv_has(GV, 2)) break;
            const R gam = th[0];
            R dg = R(0.0);
            const int npair = N * (N - 1) / 2;
            if (npair * dim <= SCR) {
                // lanes over the pairs i < j (as SimpleJastrow below)
                R *tp = scr;
                for (int q = lane; q < npair; q += SEG) {
                    int i, j;
                    pair_of(q, N, i, j);
                    R d[3], r2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        d[c] = x[i * dim + c] - x[j * dim + c];
                        r2 += d[c] * d[c];
                    }
                    const R r = sqrt(r2), ir = R(1.0) / r, beta = pade_beta_of(P, i, j);
                    const R gp = pade_gamma(P, mask, i, j, gam);
                    const R f1 = R(1.0) / (R(1.0) + gp * r), f = beta * f1 * f1, h = r * f1;
                    R c2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        const R cc = d[c] * ir;
                        tp[q * dim + c] = f * cc;
                        c2 += R(2.0) * f * (R(1.0) - (R(1.0) + R(2.0) * gam * h) * cc * cc) * ir;
                    }
                    lap_l += c2;
                    dg += beta * h * h;
                }
                gen_pair_gather<SEG>(tp, N, dim, G, oge, lane);
                dg = seg_reduce<SEG>(segmask, dg);
                if (lane == 0) pge[0] = (P.flags & Q_PADE_DGAMMA) ? -R(0.5) * dg : -dg;
                break;
            }
            for (int i = lane; i < N; i += SEG) {
                R gi[3] = {R(0.0), R(0.0), R(0.0)};
                for (int j = 0; j < N; ++j) {
                    if (j == i) continue;
                    const int lo = min(i, j), hi = max(i, j);
                    const R r = gen_dist(x, dim, i, j), beta = pade_beta_of(P, i, j);
                    const R gp = pade_gamma(P, mask, lo, hi, gam);
                    const R f1 = R(1.0) / (R(1.0) + gp * r), f = beta * f1 * f1, h = r * f1;
                    R c2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        const R cc = (x[i * dim + c] - x[j * dim + c]) / r;
                        gi[c] += f * cc;
                        c2 += R(2.0) * f * (R(1.0) - (R(1.0) + R(2.0) * gam * h) * cc * cc) / r;
                    }
                    if (j > i) {
                        lap_l += c2;
                        dg += beta * h * h;
                    }
                }
                for (int c = 0; c < dim; ++c) {
                    G[i * dim + c] += gi[c];
                    if (oge) oge[i * dim + c] = gi[c];
                }
            }
            dg = seg_reduce<SEG>(segmask, dg);
            if (lane == 0) pge[0] = (P.flags & Q_PADE_DGAMMA) ? -R(0.5) * dg : -dg;
            break;
        }
        case 3: {  // SimpleJastrow (simplejastrow.cpp:67-111)
            if (!gv_has(GV, 3)) break;
            const int npair = N * (N - 1) / 2;
            if (npair * dim <= SCR) {
                // lanes over the pairs i < j: beta (x_i - x_j) / r into the scratch,
                // the pair's Laplacian term and dJ/dbeta_ij = r; then lanes over the
                // particles sum their pairs' terms (j ascending, as the reference)
                R *tp = scr;
                for (int q = lane; q < npair; q += SEG) {
                    int i, j;
                    pair_of(q, N, i, j);
                    R d[3], r2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        d[c] = x[i * dim + c] - x[j * dim + c];
                        r2 += d[c] * d[c];
                    }
                    const R r = sqrt(r2), ir = R(1.0) / r, beta = th[i + N * j];
                    R c2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        const R cc = d[c] * ir;
                        tp[q * dim + c] = beta * cc;
                        c2 += R(2.0) * beta * (R(1.0) - cc * cc) * ir;
                    }
                    lap_l += c2;
                    pge[i + N * j] = r;
                }
                gen_pair_gather<SEG>(tp, N, dim, G, oge, lane);
                break;
            }
            for (int i = lane; i < N; i += SEG) {
                R gi[3] = {R(0.0), R(0.0), R(0.0)};
                for (int j = 0; j < N; ++j) {
                    if (j == i) continue;
                    const int lo = min(i, j), hi = max(i, j);
                    const R r = gen_dist(x, dim, i, j), beta = th[lo + N * hi];
                    R c2 = R(0.0);
                    for (int c = 0; c < dim; ++c) {
                        const R cc = (x[i * dim + c] - x[j * dim + c]) / r;
                        gi[c] += beta * cc;
                        c2 += R(2.0) * beta * (R(1.0) - cc * cc) / r;
                    }
                    if (j > i) {
                        lap_l += c2;
                        pge[i + N * j] = r;
                    }
                }
                for (int c = 0; c < dim; ++c) {
                    G[i * dim + c] += gi[c];
                    if (oge) oge[i * dim + c] = gi[c];
                }
            }
            break;
        }
        case 4: {  // RBMGaussian (rbmgaussian.cpp:67-87)
            if (!gv_has(GV, 4)) break;
            const R s2 = g.sigma * g.sigma;
            for (int k = lane; k < D; k += SEG) {
                const R t = (x[k] - th[k]) / s2;
                G[k] += -t;
                if (oge) oge[k] = -t;
                pge[k] = t;
            }
            lap_u = -D / s2;
            break;
        }
        case 5: {  // RBMProduct (rbmproduct.cpp:167-189)
            if (!gv_has(GV, 5)) break;
            const int H = g.hidden;
            const R s2 = R(100.0) * g.sigma * g.sigma, s4 = s2 * s2;
            R *xs = scr + SCR_XS, *pn = scr + SCR_PN, *nn = scr + SCR_NN;
            rbm_visible(x, D, -1, R(0), P.flags & Q_RBM_SORT, xs, lane);
            rbm_hidden(th, D, H, s2, xs, pn, nn, lane);
            for (int k = lane; k < D; k += SEG) {
                R acc = R(0.0), acc2 = R(0.0);
                for (int j = 0; j < H; ++j) {
                    const R w = th[H + k + D * j];
                    acc += w * nn[j];
                    acc2 += w * w * pn[j] * nn[j];
                }
                G[k] += acc / s2;
                if (oge) oge[k] = acc / s2;
                lap_l += acc2 / s4;
            }
            for (int t = lane; t < H * (D + 1); t += SEG) {
                if (t < H) pge[t] = nn[t];
                else {
                    const int j = (t - H) / D, i = (t - H) - j * D;
                    pge[H + i + D * j] = xs[i] * nn[j];
                }
            }
            break;
        }
        case 7: {  // MLP Jastrow: caches of (u, u', u'') per pair and (chi, chi', chi'') per particle
            if (!gv_has(GV, 7)) break;
            R *uc = rec + g.off_uc, *oc = rec + g.off_oc;
            if (full) {  // from scratch (initialisation, parameter update, evaluation)
                const int npair = N * (N - 1) / 2;
                for (int q = lane; q < npair; q += SEG) {
                    int i, j;
                    pair_of(q, N, i, j);
                    const bool same = same_spin(i, j, N);
                    float u, du, ddu;
                    mlp_pair(mw, (float)gen_dist(x, dim, i, j), same ? 1.0f : 0.0f, mlp_cusp(dim, same), u, du, ddu);
                    R *c3 = uc + (size_t)(i * N + j) * 3;
                    c3[0] = u;
                    c3[1] = du;
                    c3[2] = ddu;
                }
                for (int i = 0; i < N; ++i) {
                    float c, dc, ddc;
                    mlp_body(mw, mw + MW_V2T, (float)gen_radius(x, dim, i), lane, c, dc, ddc);
                    if (lane == 0) {
                        oc[i * 3] = c;
                        oc[i * 3 + 1] = dc;
                        oc[i * 3 + 2] = ddc;
                    }
                }
                __syncwarp(segmask);
            }
            // from the caches in FP32 (the network values are FP32 already)
            for (int i = lane; i < N; i += SEG) {
                float gi[3] = {0.0f, 0.0f, 0.0f}, li = 0.0f, xi[3];
                for (int c = 0; c < dim; ++c) xi[c] = (float)x[i * dim + c];
                for (int j = 0; j < N; ++j) {
                    if (j == i) continue;
                    const int lo = min(i, j), hi = max(i, j);
                    const R *c3 = uc + (size_t)(lo * N + hi) * 3;
                    float dv[3], r2 = 0.0f;
                    for (int c = 0; c < dim; ++c) {
                        dv[c] = xi[c] - (float)x[j * dim + c];
                        r2 += dv[c] * dv[c];
                    }
                    const float ir = approx_rsqrt(r2), du = (float)c3[1];
                    for (int c = 0; c < dim; ++c) gi[c] += du * dv[c] * ir;
                    if (j > i) li += 2.0f * ((float)c3[2] + (dim - 1) * du * ir);
                }
                float r2i = 0.0f;
                for (int c = 0; c < dim; ++c) r2i += xi[c] * xi[c];
                const float iri = approx_rsqrt(r2i), dc = (float)oc[i * 3 + 1];
                for (int c = 0; c < dim; ++c) gi[c] += dc * xi[c] * iri;
                lap_l += (R)li + oc[i * 3 + 2] + (dim - 1) * dc * iri;
                for (int c = 0; c < dim; ++c) {
                    G[i * dim + c] += gi[c];
                    if (oge) oge[i * dim + c] = gi[c];
                }
            }
            break;  // parameter gradients: mlp_grad_kernel, from snapshots
        }
        case 6: {  // HydrogenLike (hydrogenlike.cpp:268-286)
            if (!gv_has(GV, 6)) break;
            const R az = th[0] * P.Z;
            R rs = R(0.0);
            for (int i = lane; i < N; i += SEG) {
                const R r = gen_radius(x, dim, i);
                rs += r;
                for (int c = 0; c < dim; ++c) {
                    const R gk = -az * x[i * dim + c] / r;
                    G[i * dim + c] += gk;
                    if (oge) oge[i * dim + c] = gk;
                }
                lap_l -= R(2.0) / r;
            }
            rs = seg_reduce<SEG>(segmask, rs);
            lap_l *= az;
            if (lane == 0) pge[0] = -P.Z * rs;
            break;
        }
        default: break;
        }
        __syncwarp(segmask);
        const R lap_e = seg_reduce<SEG>(segmask, lap_l) + lap_u;
        lap_total += lap_e;
        if (o_lap && lane == 0) o_lap[e] = lap_e;
    }
    // System::getKineticEnergy (elementoperation.cpp:95-109) and the potentials
    R g2 = R(0.0), vx = R(0.0), vi = R(0.0);
    for (int k = lane; k < D; k += SEG) g2 += G[k] * G[k];
    if (P.flags & F_ATOM) {
        for (int i = lane; i < N; i += SEG) vx += R(1.0) / gen_radius(x, dim, i);
    } else {
        for (int k = lane; k < D; k += SEG) vx += x[k] * x[k];
    }
    if (P.flags & F_COULOMB) {  // lanes over the pairs i < j
        const int npair = N * (N - 1) / 2;
        for (int q = lane; q < npair; q += SEG) {
            int i, j;
            pair_of(q, N, i, j);
            R r2 = R(0.0);
            for (int c = 0; c < dim; ++c) {
                const R t = x[i * dim + c] - x[j * dim + c];
                r2 += t * t;
            }
            vi += rsqrt(r2);
        }
    }
    g2 = seg_reduce<SEG>(segmask, g2);
    vx = seg_reduce<SEG>(segmask, vx);
    vi = seg_reduce<SEG>(segmask, vi);
    const R ekin = -R(0.5) * (lap_total + g2);
    const R vext = (P.flags & F_ATOM) ? -P.Z * vx : R(0.5) * P.omega * P.omega * vx;
    R *en = rec + g.off_en;
    if (lane == 0) {
        en[0] = ekin;
        en[1] = vext;
        en[2] = vi;
    }
    if (o_pg)
        for (int j = lane; j < g.EP; j += SEG) o_pg[j] = pg[j];
    if (o_en && lane == 0) {
        o_en[0] = ekin;
        o_en[1] = vext;
        o_en[2] = vi;
    }
    __syncwarp(segmask);
}

// Element ratios |Psi(y)|^2 / |Psi(x)|^2 for coordinate k moved to xn (ratio_impl)
// and, when grad_y is given, d ln Psi / d y_k at the proposal (the corrected
// Fokker-Planck Green's ratio).  Orbital values at the proposal go to the scratch
// (the Sherman-Morrison update reuses them).  Returns the product in element order.
template <int GV = GV_ANY, int SEG = 32, typename R = double>
__device__ R gen_ratios(const Params &P, const GenParams &g, int dim_rt, const R *rec,
                             const unsigned long long *mask, R *scr, int lane, int k, R xn,
                             double *ratios, R *grad_y, double &R_out, const float *mw = nullptr,
                             const float *pre = nullptr, const double *inv64 = nullptr)
{
    const int N = P.N, D = g.D, E = P.n_elem, PM = g.p_max, dim = gv_dim(GV, dim_rt);
    const unsigned segmask = gen_segmask<SEG>();
    const R *x = rec;
    const int p = k / dim, adim = k - p * dim;
    R yp[3];
    for (int c = 0; c < dim; ++c) yp[c] = c == adim ? xn : x[p * dim + c];
    const R xo = x[k];
    R prob = R(1.0), gy = R(0.0);
    R_out = 1.0;
    for (int e = 0; e < E; ++e) {
        const double *th = g.theta + (size_t)e * PM;
        R r = R(1.0);
        switch (P.elem_kind[e]) {
        case 0:  // gaussian.cpp:23-28
            if (!gv_has(GV, 0)) break;
            r = exp(P.omega * th[0] * (xo * xo - xn * xn));
            gy += -P.omega * th[0] * xn;
            break;
        case 1: {  // slaterdeterminant.cpp:150-153, 177-180
            if (!gv_has(GV, 1)) break;
            const int n = g.n, b = p / n, pl = p - b * n;
            // the inverse in FP64 (gen_evaluate)
            const double *inv = inv64;
            if constexpr (std::is_same<R, double>::value)
                if (!inv) inv = rec + g.off_inv;
            double s = 0.0, sg = 0.0;
            for (int o = lane; o < n; o += SEG) {
                R v, d1[3], d2[3];
                gen_orb<GV>(g, dim, P.Z, o, yp, v, d1, d2);
                scr[SCR_PHI + o] = v;
                const double iv = inv[(size_t)(b * n + pl) * n + o];
                s += (double)v * iv;
                sg += (double)d1[adim] * iv;
            }
            const double Rs = seg_reduce<SEG>(segmask, s);
            R_out = Rs;
            r = (R)(Rs * Rs);
            if (grad_y) gy += (R)(seg_reduce<SEG>(segmask, sg) / Rs);
            __syncwarp(segmask);
            break;
        }
        case 2: {  // padejastrow.cpp:211-218
            if (!gv_has(GV, 2)) break;
            const R gam = th[0];
            const int j0 = (P.flags & Q_PADE_RATIO) ? p + 1 : 0;
            R acc = R(0.0), gyl = R(0.0);
            for (int j = lane; j < N; j += SEG) {
                if (j == p) continue;
                const int lo = min(p, j), hi = max(p, j);
                R rn2 = R(0.0);
                for (int c = 0; c < dim; ++c) {
                    const R t = yp[c] - x[j * dim + c];
                    rn2 += t * t;
                }
                const R ro = gen_dist(x, dim, p, j), rn = sqrt(rn2), beta = pade_beta_of(P, p, j);
                const R gp = pade_gamma(P, mask, lo, hi, gam);
                if (j >= j0) acc += beta * (rn / (R(1.0) + gam * rn) - ro / (R(1.0) + gp * ro));
                const R f1 = R(1.0) / (R(1.0) + gam * rn);
                gyl += beta * f1 * f1 * (yp[adim] - x[j * dim + adim]) / rn;
            }
            acc = seg_reduce<SEG>(segmask, acc);
            r = exp(R(2.0) * acc);
            if (grad_y) gy += seg_reduce<SEG>(segmask, gyl);
            break;
        }
        case 3: {  // simplejastrow.cpp:145-156
            if (!gv_has(GV, 3)) break;
            const int j0 = (P.flags & Q_SJ_RATIO) ? p + 1 : 0;
            R acc = R(0.0), gyl = R(0.0);
            for (int j = lane; j < N; j += SEG) {
                if (j == p) continue;
                const int lo = min(p, j), hi = max(p, j);
                R rn2 = R(0.0);
                for (int c = 0; c < dim; ++c) {
                    const R t = yp[c] - x[j * dim + c];
                    rn2 += t * t;
                }
                const R rn = sqrt(rn2), beta = th[lo + N * hi];
                if (j >= j0) acc += beta * (rn - gen_dist(x, dim, p, j));
                gyl += beta * (yp[adim] - x[j * dim + adim]) / rn;
            }
            acc = seg_reduce<SEG>(segmask, acc);
            r = exp(R(2.0) * acc);
            if (grad_y) gy += seg_reduce<SEG>(segmask, gyl);
            break;
        }
        case 4: {  // rbmgaussian.cpp:34-46
            if (!gv_has(GV, 4)) break;
            const R s2 = g.sigma * g.sigma, a = xo - th[k], bn = xn - th[k];
            r = exp((a * a - bn * bn) / (R(2.0) * s2));
            gy += -bn / s2;
            break;
        }
        case 5: {  // rbmproduct.cpp:199-203
            if (!gv_has(GV, 5)) break;
            const int H = g.hidden;
            const R s2 = R(100.0) * g.sigma * g.sigma;
            R *xs = scr + SCR_XS, *pn = scr + SCR_PN, *nn = scr + SCR_NN;
            const bool sort = P.flags & Q_RBM_SORT;
            rbm_visible(x, D, -1, R(0), sort, xs, lane);
            rbm_hidden(th, D, H, s2, xs, pn, nn, lane);
            R po[2] = {R(1.0), R(1.0)};
            for (int t = 0; t < 2; ++t) {
                const int j = lane + 32 * t;
                if (j < H) po[t] = pn[j];
            }
            __syncwarp(segmask);
            rbm_visible(x, D, k, xn, sort, xs, lane);
            rbm_hidden(th, D, H, s2, xs, pn, nn, lane);
            R prod = R(1.0), gyl = R(0.0);
            for (int t = 0; t < 2; ++t) {
                const int j = lane + 32 * t;
                if (j < H) {
                    prod *= po[t] / pn[j];
                    gyl += th[H + k + D * j] * nn[j];
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) prod *= __shfl_xor_sync(FULL, prod, o);
            r = prod * prod;
            if (grad_y) gy += seg_reduce<SEG>(segmask, gyl) / s2;
            __syncwarp(segmask);
            break;
        }
        case 7: {  // MLP Jastrow: exp(2 (J(y) - J(x))); the new pair and one-body values
            if (!gv_has(GV, 7)) break;
                   // go to the scratch for an accepted move
            const R *uc = rec + g.off_uc, *oc = rec + g.off_oc;
            R acc = R(0.0), gyl = R(0.0);
            for (int j = lane; j < N; j += SEG) {
                if (j == p) continue;
                R rn2 = R(0.0);
                for (int c = 0; c < dim; ++c) {
                    const R t = yp[c] - x[j * dim + c];
                    rn2 += t * t;
                }
                const R rn = sqrt(rn2);
                const bool same = same_spin(p, j, N);
                float u, du, ddu;
                if (pre) {  // from the tensor-core pass of this step (lane j = partner j)
                    u = pre[j];
                    du = pre[32 + j];
                    ddu = pre[64 + j];
                } else {
                    mlp_pair(mw, (float)rn, same ? 1.0f : 0.0f, mlp_cusp(dim, same), u, du, ddu);
                }
                scr[SCR_XS + j] = u;
                scr[SCR_XS + 32 + j] = du;
                scr[SCR_PN + j] = ddu;
                acc += (R)u - uc[(size_t)(min(p, j) * N + max(p, j)) * 3];
                gyl += du * (float)(yp[adim] - x[j * dim + adim]) * (float)(R(1.0) / rn);
            }
            R rp2 = R(0.0);
            for (int c = 0; c < dim; ++c) rp2 += yp[c] * yp[c];
            const R rp = sqrt(rp2);
            float cn, dcn, ddcn;
            mlp_body(mw, mw + MW_V2T, (float)rp, lane, cn, dcn, ddcn);
            if (lane == 0) {
                scr[SCR_PN + 32] = cn;
                scr[SCR_PN + 33] = dcn;
                scr[SCR_PN + 34] = ddcn;
            }
            const R dj = seg_reduce<SEG>(segmask, acc) + ((R)cn - oc[p * 3]);
            r = exp(R(2.0) * dj);
            if (grad_y) gy += seg_reduce<SEG>(segmask, gyl) + dcn * yp[adim] / rp;
            __syncwarp(segmask);
            break;
        }
        case 6: {  // hydrogenlike.cpp:231-242
            if (!gv_has(GV, 6)) break;
            R rn2 = R(0.0);
            for (int c = 0; c < dim; ++c) rn2 += yp[c] * yp[c];
            const R rn = sqrt(rn2);
            r = exp(R(2.0) * P.Z * th[0] * (gen_radius(x, dim, p) - rn));
            gy += -th[0] * P.Z * xn / rn;
            break;
        }
        default: break;
        }
        if (ratios) ratios[e] = r;
        prob *= r;  // elementoperation.cpp:80-87
    }
    if (grad_y) *grad_y = gy;
    return prob;
}

// Transposed inverse of both Slater blocks by Gauss-Jordan elimination with
// partial pivoting on [A | I] in shared memory (n <= 32); row i of block b holds
// A^{-1}(o, i) over orbitals o.  Returns the warp's singular flag.
__device__ unsigned gen_invert(const Params &P, const GenParams &g, int dim, double *rec, double *M,
                               int lane)
{
    const int n = g.n, w2 = 2 * n;
    unsigned status = 0;
    for (int b = 0; b < 2; ++b) {
        for (int i = 0; i < n; ++i)
            for (int c = lane; c < w2; c += 32) M[i * w2 + c] = c >= n ? (c - n == i ? 1.0 : 0.0) : 0.0;
        __syncwarp();
        if (lane < n)
            for (int i = 0; i < n; ++i) {
                double v, d1[3], d2[3];
                gen_orbital(g, dim, P.Z, lane, rec + (b * n + i) * dim, v, d1, d2);
                M[i * w2 + lane] = v;  // A[i][o] = phi_o(r_i)
            }
        __syncwarp();
        for (int c = 0; c < n; ++c) {
            double v = (lane >= c && lane < n) ? fabs(M[lane * w2 + c]) : -1.0;
            int idx = lane;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double v2 = __shfl_xor_sync(FULL, v, o);
                const int i2 = __shfl_xor_sync(FULL, idx, o);
                if (v2 > v || (v2 == v && i2 < idx)) { v = v2; idx = i2; }
            }
            if (!(v > 0.0)) status |= ST_SINGULAR;
            const int pr = idx < n ? idx : c;
            if (pr != c)
                for (int col = lane; col < w2; col += 32) {
                    const double t = M[c * w2 + col];
                    M[c * w2 + col] = M[pr * w2 + col];
                    M[pr * w2 + col] = t;
                }
            __syncwarp();
            const double ip = 1.0 / M[c * w2 + c];
            __syncwarp();
            for (int col = lane; col < w2; col += 32) M[c * w2 + col] *= ip;
            __syncwarp();
            for (int r = 0; r < n; ++r) {
                if (r == c) continue;
                const double f = M[r * w2 + c];
                __syncwarp();
                for (int col = lane; col < w2; col += 32) M[r * w2 + col] -= f * M[c * w2 + col];
                __syncwarp();
            }
        }
        // A^{-1}(o, i) = M[o][n + i]
        for (int i = 0; i < n; ++i)
            for (int o = lane; o < n; o += 32) rec[g.off_inv + (size_t)(b * n + i) * n + o] = M[o * w2 + n + i];
        __syncwarp();
    }
    return status;
}

// Shared doubles a warp needs to stage a walker of the general path (record and
// accumulators), or 0 when the walker is not staged (MLP systems, whose record holds
// the per-pair caches and the full parameter-gradient row, and records above 16 KB).
constexpr int GEN_STAGE_MAX = 2048;
__host__ __device__ inline int gen_stage_doubles(const GenParams &g, int nacc)
{
    const int n = g.rec + 2 * nacc;
    return (g.mlp || n > GEN_STAGE_MAX) ? 0 : n;
}
// The same in bytes for a record staged in real type R: the record, then the FP64
// accumulators from the next 8-byte boundary (for R = double, gen_stage_doubles x 8);
// FP32 records add the FP64 Slater inverse (2 n n) and its moved row (n)
__host__ __device__ inline int gen_stage_rec_bytes(const GenParams &g, int rbytes) { return (g.rec * rbytes + 7) & ~7; }
__host__ __device__ inline int gen_stage_bytes(const GenParams &g, int nacc, int rbytes)
{
    if (!gen_stage_doubles(g, nacc)) return 0;
    return gen_stage_rec_bytes(g, rbytes) + 16 * nacc + (rbytes == 8 ? 0 : 8 * (2 * g.n * g.n + g.n));
}

// Steps step_offset .. step_offset + steps - 1 of walker w by the calling warp.  scr: the warp's
// GEN_SCR shared doubles; mw: the CTA's staged MLP weights or null; with TC the
// CTA's four warps run in lockstep (inactive ones join the tensor-core steps).
// stage: shared memory for the walker's record (g.rec doubles) and, with stage_acc,
// its accumulators after it (gen_stage_doubles in all), or null to work on them in
// global memory; staged, every step's reads and writes stay on chip and the record
// goes back once at the end.
// R = float (the atoms' mixed precision): the FP64 record is staged in FP32, every step
// runs in FP32 (the accumulators stay FP64), and the record goes back converted.
template <bool TC, int GV = GV_ANY, int SEG = 32, typename R = double>
__device__ __forceinline__ void gen_sweep_walker(const SweepArgs &a, int steps, int step_offset, const GenParams &g,
                                                 int w, bool active, R *scr, float *mw, TcMlp &tc, float *pre_w,
                                                 R *stage = nullptr, bool stage_acc = true)
{
    static_assert(SEG == 32 || (!TC && GV != GV_ANY), "several walkers per warp: compiled forms only");
    static_assert(std::is_same<R, double>::value || (!TC && GV == GV_ATOM), "FP32 walkers: the compiled atom form");
    const Params &P = a.P;
    const int lane = threadIdx.x & (SEG - 1), wib = threadIdx.x >> 5;
    const unsigned segmask = gen_segmask<SEG>();

    const int N = P.N, D = g.D, dim = gv_dim(GV, D / N);
    const int ws = active ? w : 0;  // record pointers of a warp without a walker are never used
    double *const grec = reinterpret_cast<double *>(P.state) + (size_t)ws * g.rec;
    double *const gacc = P.acc + (size_t)ws * P.nacc * 2;
    constexpr bool F64 = std::is_same<R, double>::value;
    R *rec = stage;
    if constexpr (F64) rec = grec;
    double *acc = gacc;
    // the Slater inverse and the moved row of an update, in FP64 (apart from an FP32 record)
    double *inv64 = nullptr, *row64 = nullptr;
    const bool staged = stage && active, acc_staged = staged && stage_acc;
    if (staged) {
        double *sacc = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(stage) +
                                                  gen_stage_rec_bytes(g, (int)sizeof(R)));
        for (int i = lane; i < g.rec; i += SEG) stage[i] = (R)grec[i];
        if (acc_staged)
            for (int i = lane; i < 2 * P.nacc; i += SEG) sacc[i] = gacc[i];
        if constexpr (!F64) {
            inv64 = sacc + 2 * P.nacc;
            row64 = inv64 + 2 * g.n * g.n;
            for (int i = lane; i < 2 * g.n * g.n; i += SEG) inv64[i] = grec[g.off_inv + i];
        }
        __syncwarp(segmask);
        rec = stage;
        if (acc_staged) acc = sacc;
    }
    if constexpr (F64) {
        inv64 = rec + g.off_inv;
        row64 = scr + SCR_ROW;
    }
    R *x = rec, *fc = rec + g.off_fc;
    unsigned long long *mask = P.mask + (size_t)ws * N;
    unsigned long long ctr = active ? P.counter[ws] : 0ull;
    unsigned status = 0;
    const bool is = P.sampling == SAMPLER_IS;
    const double dt = P.step, sqdt = sqrt(P.step);

    for (int s = 0; s < steps; ++s) {
        const int it_step = step_offset + s;
        int k = 0;
        double r1 = 0.0, r2 = 0.0;
        R xo = R(0), dx = R(0), fn = R(0), xn = R(0);
        if (active) {
            // ---- random numbers (vmo_step_randoms) or the caller's
            k = 0;
            r1 = r2 = 0.0;
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
                const uint4 v = philox(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32),
                                                  (uint32_t)(w + a.P.walker_offset), 0u),
                                       make_uint2((uint32_t)a.seed, (uint32_t)(a.seed >> 32)));
                ++ctr;
                k = (int)__umulhi(v.x, (unsigned)D);
                if (is) {
                    const double u1 = ((double)v.y + 1.0) * TWO_M32, u2 = v.z * TWO_M32;
                    r1 = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
                } else {
                    r1 = v.y * TWO_M32;
                }
                r2 = v.w * TWO_M32;
            }
            // ---- proposal (importancesampling.cpp:49-60, bruteforce.cpp:34)
            xo = x[k];
            fn = 0.0;
            if (a.probe_k) {
                dx = a.probe_x[w] - xo;
            } else if (is) {
                fn = R(2) * limited_drift<R>(rec[g.off_g + k], P);
                dx = 0.5 * dt * fn + r1 * sqdt;
            } else {
                dx = 10.0 * (r1 - 0.5) * P.step;
            }
            xn = a.probe_k ? a.probe_x[w] : xo + dx;
        }
        if (TC) {
            // second layer of the pair network for the proposal's partners of all the
            // CTA's walkers: one 128-row tile, tensor cores (value, d/dr, d2/dr2)
            const int p = k / dim;
            double yp[3] = {0.0, 0.0, 0.0};
            for (int c = 0; c < dim; ++c) yp[c] = (active && c == k - p * dim) ? xn : (active ? x[p * dim + c] : 0.0);
            float r = 0.0f, sv = 0.0f;
            bool valid = active && lane < N && lane != p;
            if (valid) {
                double r2s = 0.0;
                for (int c = 0; c < dim; ++c) {
                    const double t = yp[c] - x[lane * dim + c];
                    r2s += t * t;
                }
                r = (float)sqrt(r2s);
                sv = same_spin(p, lane, N) ? 1.0f : 0.0f;
            }
            status |= tc_pair_layer(tc, mw, valid, r, sv, mlp_cusp(dim, sv > 0.5f), lane, wib, pre_w);
        }
        if (active) {
            const bool corrected = is && !(P.flags & Q_IS_GREEN) && !a.probe_k;
            R gy = R(0);
            double Rdet = 1.0;
            double *ratios = (a.probe_k && lane == 0) ? a.probe_ratio + (size_t)w * P.n_elem : nullptr;
            const double prob = gen_ratios<GV, SEG, R>(P, g, dim, rec, mask, scr, lane, k, xn, ratios,
                                                       corrected ? &gy : nullptr, Rdet, mw, TC ? pre_w : nullptr,
                                                       inv64);
            bool accept = true;
            if (!a.probe_k) {
                double wgt = prob;
                if (is) {
                    if (P.flags & Q_IS_GREEN) {
                        wgt = (exp(0.5 * (fc[k] - fn) * dx) + 1.0) * prob;  // importancesampling.cpp:43-47
                    } else {
                        const double fy = 2.0 * (double)limited_drift<R>(gy, P), fnd = fn;
                        wgt = prob * exp(0.5 * (fnd + fy) * (0.25 * dt * (fnd - fy) - (double)dx));
                    }
                }
                // the reference rejects when weight < u (importancesampling.cpp:72,
                // bruteforce.cpp:44); a NaN weight is flagged and rejected
                if (wgt != wgt) status |= ST_BAD_RATIO;
                accept = wgt >= r2;
            }
            if (accept) {
                const int p = k / dim;
                if (P.flags & F_SLATER) {
                    // Sherman-Morrison on the moved particle's block (slaterdeterminant.cpp:165-175)
                    const int n = g.n, b = p / n, pl = p - b * n;
                    double *rows = inv64 + (size_t)b * n * n;
                    for (int o = lane; o < n; o += SEG) row64[o] = rows[(size_t)pl * n + o];
                    __syncwarp(segmask);
                    for (int r = lane; r < n; r += SEG) {
                        double *row = rows + (size_t)r * n;
                        double S = 0.0;
                        for (int o = 0; o < n; ++o) S += (double)scr[SCR_PHI + o] * row[o];
                        const double c = S / Rdet;
                        for (int o = 0; o < n; ++o) row[o] = r == pl ? row64[o] / Rdet : row[o] - c * row64[o];
                    }
                    __syncwarp(segmask);
                }
                if (lane == 0) {
                    x[k] = xn;
                    if (is) fc[k] = fn;
                }
                if (P.flags & F_MLP) {  // the moved particle's pair and one-body values from the proposal
                    R *uc = rec + g.off_uc;
                    for (int j = lane; j < N; j += SEG)
                        if (j != p) {
                            R *c3 = uc + (size_t)(min(p, j) * N + max(p, j)) * 3;
                            c3[0] = scr[SCR_XS + j];
                            c3[1] = scr[SCR_XS + 32 + j];
                            c3[2] = scr[SCR_PN + j];
                        }
                    if (lane == 0)
                        for (int t = 0; t < 3; ++t) rec[g.off_oc + p * 3 + t] = scr[SCR_PN + 32 + t];
                }
                if (P.flags & Q_PADE_STALE) {  // the moved particle's pairs take the current gamma
                    for (int j = lane; j < N; j += SEG)
                        if (j != p) mask[j] |= 1ull << p;
                    if (lane == 0) mask[p] = ~0ull;
                }
                __syncwarp(segmask);
                gen_evaluate<GV, SEG, R>(P, g, dim, rec, mask, scr, lane, nullptr, nullptr, nullptr, nullptr, mw, false, p,
                                         inv64);
            }
            if (a.rec_acc && lane == 0) a.rec_acc[(size_t)w * a.rec_stride + it_step] = accept ? 1 : 0;
            const R *en = rec + g.off_en;
            if (a.rec_en && lane == 0) {
                double *o = a.rec_en + ((size_t)w * a.rec_stride + it_step) * 3;
                o[0] = en[0];
                o[1] = en[1];
                o[2] = en[2];
            }
            if (SEG == 32 && it_step >= a.burn_in && a.dens_bins > 0) density_sample<R>(a, x, N, dim, lane);
            if (it_step >= a.burn_in) {  // Sampler::sample (sampler.cpp:52-90)
                const double el = (double)en[0] + (double)en[1] + (double)en[2];
                if (el != el) status |= ST_NAN_ENERGY;
                const bool win = it_step > a.win_lo && it_step < a.win_hi;
                if (win && a.snap_x && (it_step - a.win_lo) % a.snap_interval == 0) {
                    // MLP Jastrow parameter gradient: positions and E_L for mlp_grad_kernel
                    const int slot = (it_step - a.win_lo) / a.snap_interval - a.snap_first;
                    if (slot >= 0 && slot < a.snap_stride) {
                        const size_t base = (size_t)w * a.snap_stride + slot;
                        for (int t = lane; t < D; t += SEG) a.snap_x[base * D + t] = (float)x[t];
                        if (lane == 0) a.snap_e[base] = el;
                    }
                }
                const int top = win ? 9 + 2 * g.n_act : 9;  // == P.nacc inside the window
                const R *pg = rec + g.off_pg;
                for (int t = lane; t < top; t += SEG) {
                    double q;
                    if (t < 8) {
                        const double base = t < 2 ? el : en[(t >> 1) - 1];
                        q = (t & 1) ? base * base : base;
                    } else if (t == 8) {
                        q = accept ? 1.0 : 0.0;
                    } else {
                        const int c = t - 9;
                        q = c < g.n_act ? pg[g.act[c]] : el * pg[g.act[c - g.n_act]];
                    }
                    double s1 = acc[2 * t], c1 = acc[2 * t + 1];
                    kadd(s1, c1, q);
                    acc[2 * t] = s1;
                    acc[2 * t + 1] = c1;
                }
            }
            __syncwarp(segmask);
        }
    }
    if (staged) {
        __syncwarp(segmask);
        for (int i = lane; i < g.rec; i += SEG) grec[i] = rec[i];
        if constexpr (!F64)
            for (int i = lane; i < 2 * g.n * g.n; i += SEG) grec[g.off_inv + i] = inv64[i];
        if (acc_staged)
            for (int i = lane; i < 2 * P.nacc; i += SEG) gacc[i] = acc[i];
    }
    if (active && lane == 0) {
        P.counter[w] = ctr;
        if (status) P.status[w] |= status;
    }
}

}  // namespace

}  // namespace vmc
