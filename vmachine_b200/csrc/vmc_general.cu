// General walker path: kernels and launchers (device functions in vmc_general_dev.cuh).
#include "vmc_general_dev.cuh"

namespace vmc {

namespace {

__global__ void __launch_bounds__(32 * GEN_WPB) gen_state_kernel(const Params P, const GenParams g, int mode,
                                                                double *o_grad, double *o_lap, double *o_pg,
                                                                double *o_en)
{
    extern __shared__ __align__(16) double gsm[];
    __shared__ double scratch[GEN_WPB][GEN_SCR];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int w = blockIdx.x * GEN_WPB + wib;
    // dynamic shared memory: MLP weights (when present), then the inversion matrices
    float *mw = g.mlp ? reinterpret_cast<float *>(gsm) : nullptr;
    double *inv_area = gsm + (g.mlp ? MLP_SMEM_DOUBLES : 0);
    if (mw) {
        mlp_stage(g.mlp, mw);
        __syncthreads();
    }
    if (w >= P.W) return;
    const int dim = g.D / P.N;
    double *rec = reinterpret_cast<double *>(P.state) + (size_t)w * g.rec;
    unsigned long long *mask = P.mask + (size_t)w * P.N;
    unsigned status = 0;
    if (mode == GEN_INIT) {
        for (int j = lane; j < P.N; j += 32) mask[j] = ~0ull;
        if (P.flags & F_SLATER) status = gen_invert(P, g, dim, rec, inv_area + (size_t)wib * g.n * 2 * g.n, lane);
        __syncwarp();
    }
    const size_t E = P.n_elem;
    gen_evaluate(P, g, dim, rec, mask, scratch[wib], lane, o_grad ? o_grad + (size_t)w * E * g.D : nullptr,
                 o_lap ? o_lap + (size_t)w * E : nullptr, o_pg ? o_pg + (size_t)w * g.EP : nullptr,
                 o_en ? o_en + (size_t)w * 3 : nullptr, mw, true);
    if (mode == GEN_INIT && P.sampling == SAMPLER_IS)  // ImportanceSampling::initialize: F = 2 grad
        for (int k = lane; k < g.D; k += 32) rec[g.off_fc + k] = 2.0 * rec[g.off_g + k];
    status = __reduce_or_sync(FULL, status);
    if (lane == 0 && status) P.status[w] |= status;
}

template <bool TC>
__global__ void __launch_bounds__(32 * GEN_WPB) gen_sweep_kernel(const SweepArgs a, const GenParams g)
{
    extern __shared__ __align__(16) double gsm[];
    __shared__ double scratch[GEN_WPB][GEN_SCR];
    __shared__ float pre[GEN_WPB][3 * 32];  // TC: u, du/dr, d2u/dr2 of each partner of the proposal
    __shared__ __align__(8) unsigned long long tc_bar;
    __shared__ uint32_t tc_slot;
    const Params &P = a.P;
    const int wib = threadIdx.x >> 5;
    const int w = blockIdx.x * GEN_WPB + wib;
    float *mw = g.mlp ? reinterpret_cast<float *>(gsm) : nullptr;
    if (mw) mlp_stage(g.mlp, mw, !TC);
    TcMlp tc{};
    if (TC) tc_setup(tc, reinterpret_cast<unsigned char *>(gsm) + MLP_SMEM_DOUBLES * sizeof(double), mw, g.mlp,
                     &tc_bar, &tc_slot, wib);
    __syncthreads();
    if (TC) tc_ready(tc, &tc_slot);
    const bool active = w < P.W;
    if (!TC && !active) return;
    const int nst = gen_stage_doubles(g, P.nacc);  // 0 with the MLP (gsm holds its weights)
    gen_sweep_walker<TC>(a, a.steps, a.step_offset, g, w, active, scratch[wib], mw, tc, pre[wib],
                         nst ? gsm + (size_t)wib * nst : nullptr);
    if (TC) tc_teardown(tc, wib);
}

// dJ/dtheta of the MLP Jastrow for a set of position snapshots (backpropagation,
// summed over pairs and particles), accumulated plain and weighted by each
// snapshot's local energy.  One CTA of 256 threads per snapshot at a time; the
// pair rows of a snapshot go through in tiles of 64:
//   A: r, s and h1 = tanh(W1 [r, s] + b1) per row (warps over rows, lanes over units)
//   B: z2 = W2 h1 + b2, h2 = tanh z2, delta2 = w3 (1 - h2^2)
//   C: dJ/dW2 += delta2 (x) h1 over the rows (thread t: unit m = t / 4, 16 inputs)
//   D: delta1 = (W2^T delta2)(1 - h1^2); dJ/dW1, dJ/db1
// The one-body network (N rows) goes through one warp per particle with shared-
// memory accumulation.  FP64 accumulators per thread, atomically added at the end.
constexpr int MG_TILE = 64;
constexpr int MG_BODY = MLP_G * MLP_G + 4 * MLP_G;  // one-body sums of a snapshot: V2, V1, c1, c2, v3
constexpr int MG_SMEM_FLOATS = MLP_SMEM_FLOATS + 2 * MG_TILE * MLP_H + 2 * MG_TILE + 96 + MG_BODY;

__global__ void __launch_bounds__(256) mlp_grad_kernel(const GenParams g, int N, int dim,
                                                       const float *__restrict__ snap_x,
                                                       const double *__restrict__ snap_e,
                                                       long long n_snap, double *out)
{
    extern __shared__ __align__(16) float msm[];
    float *w = msm;
    float *h1s = w + MLP_SMEM_FLOATS;           // [MG_TILE][64]
    float *d2s = h1s + MG_TILE * MLP_H;         // [MG_TILE][64]
    float *rr = d2s + MG_TILE * MLP_H;          // [MG_TILE]
    float *ss = rr + MG_TILE;                   // [MG_TILE]
    float *xs = ss + MG_TILE;                   // positions, D <= 96
    float *bv2 = xs + 96;                       // one-body sums: V2 [32][32], V1, c1, c2, v3 [32] each
    float *bu = bv2 + MLP_G * MLP_G;
    mlp_stage(g.mlp, w);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int D = N * dim, npair = N * (N - 1) / 2;
    const int cm = t >> 2, ck = (t & 3) * 16;  // phase C ownership
    double aW2[16], eW2[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) aW2[i] = eW2[i] = 0.0;
    // lane-owned units k in {lane, lane + 32} (phases A, B, D), accumulated per warp
    double aU[2][5], eU[2][5];  // [unit][b1, W1r, W1s, b2, w3]
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 5; ++q) aU[u][q] = eU[u][q] = 0.0;
    double aV[4], eV[4], aB[4], eB[4];  // one-body: V2 entries 4t..4t+3; t < 32: V1/c1/c2/v3 of unit t
#pragma unroll
    for (int q = 0; q < 4; ++q) aV[q] = eV[q] = aB[q] = eB[q] = 0.0;
    double n_rows = 0.0, e_rows = 0.0, n_body = 0.0, e_body = 0.0;
    for (int i = t; i < MG_BODY; i += blockDim.x) bv2[i] = 0.0f;
    __syncthreads();

    for (long long sn = blockIdx.x; sn < n_snap; sn += gridDim.x) {
        const double E = snap_e ? snap_e[sn] : 0.0;
        for (int i = t; i < D; i += blockDim.x) xs[i] = snap_x[sn * D + i];
        __syncthreads();
        float sW2[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) sW2[i] = 0.0f;
        float sU[2][5];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int q = 0; q < 5; ++q) sU[u][q] = 0.0f;
        for (int base = 0; base < npair; base += MG_TILE) {
            const int nrow = min(MG_TILE, npair - base);
            // A
            for (int row = warp; row < nrow; row += 8) {
                int i, j;
                pair_of(base + row, N, i, j);
                float r2 = 0.0f;
                for (int c = 0; c < dim; ++c) {
                    const float d = xs[i * dim + c] - xs[j * dim + c];
                    r2 += d * d;
                }
                const float r = sqrtf(r2), sv = same_spin(i, j, N) ? 1.0f : 0.0f;
                if (lane == 0) {
                    rr[row] = r;
                    ss[row] = sv;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int k = lane + 32 * u;
                    h1s[row * MLP_H + k] = mlp_tanh(fmaf(w[MW_W1 + 2 * k], r, fmaf(w[MW_W1 + 2 * k + 1], sv, w[MW_B1 + k])));
                }
            }
            __syncthreads();
            // B
            for (int row = warp; row < nrow; row += 8) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int m = lane + 32 * u;
                    float z = w[MW_B2 + m];
                    for (int k = 0; k < MLP_H; ++k) z = fmaf(w[MW_W2T + k * MLP_H + m], h1s[row * MLP_H + k], z);
                    const float h2 = mlp_tanh(z), d2 = w[MW_W3 + m] * (1.0f - h2 * h2);
                    d2s[row * MLP_H + m] = d2;
                    sU[u][3] += d2;
                    sU[u][4] += h2;
                }
            }
            __syncthreads();
            // C
            for (int row = 0; row < nrow; ++row) {
                const float dm = d2s[row * MLP_H + cm];
                const float4 *hv = reinterpret_cast<const float4 *>(h1s + row * MLP_H + ck);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 v = hv[q];
                    sW2[4 * q] = fmaf(dm, v.x, sW2[4 * q]);
                    sW2[4 * q + 1] = fmaf(dm, v.y, sW2[4 * q + 1]);
                    sW2[4 * q + 2] = fmaf(dm, v.z, sW2[4 * q + 2]);
                    sW2[4 * q + 3] = fmaf(dm, v.w, sW2[4 * q + 3]);
                }
            }
            // D
            for (int row = warp; row < nrow; row += 8) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int k = lane + 32 * u;
                    float acc = 0.0f;
                    for (int m = 0; m < MLP_H; ++m) acc = fmaf(d2s[row * MLP_H + m], w[MW_W2 + m * MLP_H + k], acc);
                    const float hk = h1s[row * MLP_H + k], d1 = acc * (1.0f - hk * hk);
                    sU[u][0] += d1;
                    sU[u][1] += d1 * rr[row];
                    sU[u][2] += d1 * ss[row];
                }
            }
            __syncthreads();
        }
        // one-body network: warp per particle, lane = hidden unit
        for (int i = warp; i < N; i += 8) {
            float r2 = 0.0f;
            for (int c = 0; c < dim; ++c) r2 += xs[i * dim + c] * xs[i * dim + c];
            const float r = sqrtf(r2);
            const float h = mlp_tanh(fmaf(w[MW_V1 + lane], r, w[MW_C1 + lane]));
            float z = w[MW_C2 + lane];
            for (int k = 0; k < MLP_G; ++k) z = fmaf(w[MW_V2T + k * MLP_G + lane], __shfl_sync(FULL, h, k), z);
            const float h2 = mlp_tanh(z), e2 = w[MW_V3 + lane] * (1.0f - h2 * h2);
            // dJ/dV2[m][k] = e2_m h_k (lane m), dJ/dc2 = e2, dJ/dv3 = h2
            for (int k = 0; k < MLP_G; ++k) atomicAdd(&bv2[lane * MLP_G + k], e2 * __shfl_sync(FULL, h, k));
            float acc = 0.0f;  // backpropagated to the first layer: lane k
            for (int m = 0; m < MLP_G; ++m) acc = fmaf(__shfl_sync(FULL, e2, m), w[MW_V2 + m * MLP_G + lane], acc);
            const float e1 = acc * (1.0f - h * h);
            atomicAdd(&bu[lane], e1 * r);               // V1
            atomicAdd(&bu[MLP_G + lane], e1);           // c1
            atomicAdd(&bu[2 * MLP_G + lane], e2);       // c2
            atomicAdd(&bu[3 * MLP_G + lane], h2);       // v3
        }
        __syncthreads();
        // fold the snapshot into the FP64 accumulators
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            aW2[i] += sW2[i];
            eW2[i] += E * sW2[i];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                aU[u][q] += sU[u][q];
                eU[u][q] += E * sU[u][q];
            }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float v = bv2[4 * t + q];
            aV[q] += v;
            eV[q] += E * v;
        }
        if (t < MLP_G) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float b = bu[q * MLP_G + t];
                aB[q] += b;
                eB[q] += E * b;
            }
        }
        n_rows += npair;
        e_rows += E * npair;
        n_body += N;
        e_body += E * N;
        __syncthreads();
        for (int i = t; i < MG_BODY; i += blockDim.x) bv2[i] = 0.0f;
        __syncthreads();
    }
    const int P = MLP_PARAMS;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        atomicAdd(&out[MW_W2 + cm * MLP_H + ck + i], aW2[i]);
        atomicAdd(&out[P + MW_W2 + cm * MLP_H + ck + i], eW2[i]);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int k = lane + 32 * u;
        const int idx[5] = {MW_B1 + k, MW_W1 + 2 * k, MW_W1 + 2 * k + 1, MW_B2 + k, MW_W3 + k};
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            atomicAdd(&out[idx[q]], aU[u][q]);
            atomicAdd(&out[P + idx[q]], eU[u][q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int e = 4 * t + q;  // V2 entry (m, k) = (e / 32, e % 32)
        atomicAdd(&out[MW_V2 + e], aV[q]);
        atomicAdd(&out[P + MW_V2 + e], eV[q]);
    }
    if (t < MLP_G) {
        const int idx[4] = {MW_V1 + t, MW_C1 + t, MW_C2 + t, MW_V3 + t};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            atomicAdd(&out[idx[q]], aB[q]);
            atomicAdd(&out[P + idx[q]], eB[q]);
        }
    }
    if (t == 0) {
        atomicAdd(&out[MW_B3], n_rows);
        atomicAdd(&out[P + MW_B3], e_rows);
        atomicAdd(&out[MW_C3], n_body);
        atomicAdd(&out[P + MW_C3], e_body);
    }
}

}  // namespace

cudaError_t upload_hermite_gen(const HermiteCoef &h) { return cudaMemcpyToSymbol(c_herm, &h, sizeof(h)); }

std::string gen_configure(const Config &c, int E, int p_max, GenParams &g)
{
    g = GenParams{};
    const int N = c.N, dim = c.dim, D = N * dim;
    g.D = D;
    g.p_max = p_max;
    g.EP = E * p_max;
    g.hidden = c.hidden;
    g.sigma = c.sigma;
    g.basis = c.basis == "hydrogenOrbital" ? BASIS_HYDROGEN : BASIS_HERMITE;
    g.horb3 = c.compat ? 1 : 0;
    g.mlp_tc = c.mlp_tc ? 1 : 0;
    const bool slater = std::count(c.elements.begin(), c.elements.end(), (int)E_SLATER) > 0;
    g.n = slater ? N / 2 : 0;
    if (slater) {
        if (N % 2) return "Slater determinant needs an even particle count";
        if (g.n > 32) return "more than 32 orbitals per spin block";
        if (g.basis == BASIS_HERMITE) {
            int o = 0;
            for (int s = 0; o < g.n; ++s) {  // shells in the reference's order (basis.cpp:81-116)
                if (dim == 2) {
                    for (int j = 0; j <= s && o < g.n; ++j, ++o) {
                        g.orb[o][0] = (unsigned char)(s - j);
                        g.orb[o][1] = (unsigned char)j;
                        g.orb[o][2] = 0;
                    }
                } else {
                    for (int j = 0; j <= s && o < g.n; ++j)
                        for (int l = 0; l <= s - j && o < g.n; ++l, ++o) {
                            g.orb[o][0] = (unsigned char)(s - j - l);
                            g.orb[o][1] = (unsigned char)j;
                            g.orb[o][2] = (unsigned char)l;
                        }
                }
                if (s > 12) return "too many Hermite shells";
            }
            // closed shells only (basis.cpp:62-79)
            int count = 0, s = 0;
            while (count < g.n) {
                count += dim == 2 ? s + 1 : (s + 1) * (s + 2) / 2;
                ++s;
            }
            if (count != g.n) return "open shell: numParticles is not a closed shell";
        } else {
            if (dim != 3) return "hydrogen orbitals are three-dimensional (hydrogenorbital.cpp:17)";
            // closed-shell atoms He, Be, Ne, Mg, Ar (hydrogenorbital.cpp:28-58) with
            // orbitals (n, l, m) in the reference's order (generateLOS), l <= 1
            if (N != 2 && N != 4 && N != 10 && N != 12 && N != 18)
                return "hydrogen orbitals: numParticles must be 2, 4, 10, 12 or 18 on this engine";
            int o = 0;
            for (int nq = 1; nq <= 3 && o < g.n; ++nq)
                for (int l = 0; l < nq && o < g.n; ++l)
                    for (int m = -l; m <= l && o < g.n; ++m, ++o) {
                        g.orb[o][0] = (unsigned char)nq;
                        g.orb[o][1] = (unsigned char)l;
                        g.orb[o][2] = (unsigned char)(m + 1);
                    }
        }
    }
    const bool rbmp = std::count(c.elements.begin(), c.elements.end(), (int)E_RBMPRODUCT) > 0;
    if (rbmp && (D > GEN_SCR / 4 || c.hidden > 64)) return "RBMProduct: at most 64 coordinates and 64 hidden units";
    // record layout (doubles): x | fc | grad | energies (4) | pgrad (E p_max) | inverse (2 n n)
    g.off_fc = D;
    g.off_g = 2 * D;
    g.off_en = 3 * D;
    g.off_pg = 3 * D + 4;
    g.off_inv = round_up(g.off_pg + g.EP, 2);
    const bool mlp = std::count(c.elements.begin(), c.elements.end(), (int)E_MLP) > 0;
    if (mlp && (N > 32 || dim * N > 96)) return "MLP Jastrow: at most 32 particles on this engine";
    g.off_uc = g.off_inv + 2 * g.n * g.n;                 // MLP caches: N x N x 3, N x 3
    g.off_oc = g.off_uc + (mlp ? N * N * 3 : 0);
    g.rec = round_up(g.off_oc + (mlp ? N * 3 : 0), 2);
    return "";
}

int gen_smem_per_warp(const GenParams &g) { return g.n * 2 * g.n * 8; }

cudaError_t gen_launch_state(const Params &P, const GenParams &g, int mode, double *o_grad, double *o_lap,
                             double *o_pg, double *o_en, cudaStream_t st)
{
    const size_t smem = (g.mlp ? MLP_SMEM_DOUBLES * sizeof(double) : 0) +
                        (mode == GEN_INIT ? (size_t)GEN_WPB * gen_smem_per_warp(g) : 0);
    cudaError_t e = cudaFuncSetAttribute(gen_state_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    gen_state_kernel<<<(P.W + GEN_WPB - 1) / GEN_WPB, 32 * GEN_WPB, smem, st>>>(P, g, mode, o_grad, o_lap, o_pg,
                                                                                o_en);
    return cudaGetLastError();
}

cudaError_t gen_launch_sweep(const SweepArgs &a, const GenParams &g, cudaStream_t st)
{
    const bool tc = g.mlp && g.mlp_tc;
    const size_t smem = (g.mlp ? MLP_SMEM_DOUBLES * sizeof(double) : 0) + (tc ? TC_SMEM : 0) +
                        (size_t)GEN_WPB * gen_stage_doubles(g, a.P.nacc) * sizeof(double);
    const void *fn = tc ? (const void *)gen_sweep_kernel<true> : (const void *)gen_sweep_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (tc)
        gen_sweep_kernel<true><<<(a.P.W + GEN_WPB - 1) / GEN_WPB, 32 * GEN_WPB, smem, st>>>(a, g);
    else
        gen_sweep_kernel<false><<<(a.P.W + GEN_WPB - 1) / GEN_WPB, 32 * GEN_WPB, smem, st>>>(a, g);
    return cudaGetLastError();
}

}  // namespace vmc

namespace vmc {

cudaError_t mlp_launch_grad(const GenParams &g, int N, int dim, const float *snap_x, const double *snap_e,
                            long long n_snap, double *out, cudaStream_t st)
{
    if (n_snap <= 0) return cudaSuccess;
    const size_t smem = (size_t)MG_SMEM_FLOATS * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long grid = std::min<long long>(n_snap, (long long)sms);
    mlp_grad_kernel<<<(unsigned)grid, 256, smem, st>>>(g, N, dim, snap_x, snap_e, n_snap, out);
    return cudaGetLastError();
}

}  // namespace vmc
