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
    if (mode == GEN_INIT)
        for (int j = lane; j < P.N; j += 32) mask[j] = ~0ull;
    if (mode != GEN_STATE) {
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

// G walkers per warp (compiled forms only): each takes a 32 / G-lane segment, a
// GEN_SCR / G slice of the warp's scratch and its own staging area.
template <bool TC, int GV, int G = 1, typename R = double>
__global__ void __launch_bounds__(32 * GEN_WPB) gen_sweep_kernel(const SweepArgs a, const GenParams g)
{
    extern __shared__ __align__(16) double gsm[];
    __shared__ R scratch[GEN_WPB][GEN_SCR];
    __shared__ float pre[GEN_WPB][3 * 32];  // TC: u, du/dr, d2u/dr2 of each partner of the proposal
    __shared__ __align__(8) unsigned long long tc_bar;
    __shared__ uint32_t tc_slot;
    const Params &P = a.P;
    const int wib = threadIdx.x >> 5, seg = (threadIdx.x & 31) / (32 / G);
    const int w = (blockIdx.x * GEN_WPB + wib) * G + seg;
    float *mw = g.mlp ? reinterpret_cast<float *>(gsm) : nullptr;
    if (mw) mlp_stage(g.mlp, mw, !TC);
    TcMlp tc{};
    if (TC) tc_setup(tc, reinterpret_cast<unsigned char *>(gsm) + MLP_SMEM_DOUBLES * sizeof(double), mw, g.mlp,
                     &tc_bar, &tc_slot, wib);
    __syncthreads();
    if (TC) tc_ready(tc, &tc_slot);
    const bool active = w < P.W;
    if (!TC && !active) return;
    const int nst = gen_stage_bytes(g, P.nacc, (int)sizeof(R));  // 0 with the MLP (gsm holds its weights)
    R *stage = nst ? reinterpret_cast<R *>(reinterpret_cast<unsigned char *>(gsm) + (size_t)(wib * G + seg) * nst)
                   : nullptr;
    gen_sweep_walker<TC, GV, 32 / G, R>(a, a.steps, a.step_offset, g, w, active, scratch[wib] + seg * (GEN_SCR / G),
                                        mw, tc, pre[wib], stage);
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

// The same gradient sums with the pair network's GEMM-shaped work on the tensor
// cores.  The pair rows of all snapshots (n_snap x N(N-1)/2) go through in tiles of
// 128 rows, one row per thread of a 4-warp CTA (TMEM lane = row):
//   G1  z2 = h1 W2^T                  M 128, N 64,  K 64   A = h1 (rows r, k inputs)
//   G2  e1 = delta2 W2                M 128, N 64,  K 64   A = delta2 (rows r, j outputs)
//   G3  [dW2 | db2] += [delta2^T; (E delta2)^T] [h1 | 1]      M 128 (j, then j E-weighted),
//                                     N 80, K 128 (the tile's rows), accumulated in TMEM
//   G4  [delta1 sums | h2 sums] += [delta1^T; h2^T] [1, E, r, s, E r, E s]
//                                     M 128, N 16, K 128, accumulated in TMEM
// with delta2 = w3 (1 - h2^2), h2 = tanh(z2 + b2), delta1 = e1 (1 - h1^2): G4 gives
// db1, dW1 (r and s columns) and dw3 with their E-weighted forms.  Operands are
// bfloat16, every non-weight operand as a high and a low part (the products of the
// parts, 2 or 3 MMAs per K step, keep about 16 significant bits); W2 is bfloat16
// already.  FP32 accumulation in TMEM, added to the FP64 output once per CTA.  The
// one-body network (N rows per snapshot) runs on the CUDA cores as in
// mlp_grad_kernel.  Every completion wait is bounded (TC_WAIT_LIMIT polls); on
// expiry the CTA stops, sets *fail and still releases its tensor memory.
constexpr int BT_ROWS = 128;
constexpr int BT_A1 = 0;                   // h1 [r][k] K64: hi 16 KB, lo 16 KB
constexpr int BT_A2 = 32768;               // delta2 [r][j] K64: hi, lo; later A4 hi [128][128]
constexpr int BT_A3 = 65536;               // [delta2^T; E delta2^T] [128][K128]: hi 32 KB, lo 32 KB; A4 lo in the first half
constexpr int BT_B3 = 131072;              // [h1^T; 1; 0] [80][K128]: hi 20 KB, lo 20 KB
constexpr int BT_B4 = BT_B3 + 40960;       // [1, E, r, s, E r, E s, 0] [16][K128]: hi 4 KB, lo 4 KB
constexpr int BT_W2 = BT_B4 + 8192;        // W2 [j][m] K64
constexpr int BT_W2T = BT_W2 + 8192;       // W2^T [m][j] K64
constexpr int BT_TILES = BT_W2T + 8192;    // 196 608 bytes of operand tiles
constexpr int BT_SMEM = BT_TILES + 1024;  // + alignment slack
constexpr int BT_COLS = 256;               // TMEM: G1 [0,64), G2 [64,128), G3 [128,208), G4 [208,224)
__host__ __device__ constexpr uint32_t bt_idesc(int n) { return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24); }

__device__ __forceinline__ uint32_t bt_off128(int row, int k)
{
    return (row & 7) * 16 + (row >> 3) * 2048 + (k >> 3) * 128 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t bt_desc(uint32_t saddr, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void bt_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
                 "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
                 : "memory");
}

__device__ __forceinline__ void bt_put(unsigned char *t, uint32_t off_hi, uint32_t lo_bytes, float v)
{
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    *reinterpret_cast<__nv_bfloat16 *>(t + off_hi) = h;
    *reinterpret_cast<__nv_bfloat16 *>(t + off_hi + lo_bytes) = __float2bfloat16_rn(v - __bfloat162float(h));
}

// The CTA's MMAs are visible and this thread's earlier TMEM reads are done; thread
// 0 issues, the commit arrives on bar.  Returns false when the wait gave up.
__device__ bool bt_commit_wait(uint32_t bar, uint32_t &phase)
{
    if (threadIdx.x == 0)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
    uint32_t done = 0;
    for (long it = 0; it < TC_WAIT_LIMIT && !done; ++it)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(phase)
                     : "memory");
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return done != 0;
}

// tile writes by every thread visible to the tensor cores, then thread 0 may issue
__device__ __forceinline__ void bt_publish()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__global__ void __launch_bounds__(BT_ROWS) mlp_grad_tc_kernel(const GenParams g, int N, int dim,
                                                              const float *__restrict__ snap_x,
                                                              const double *__restrict__ snap_e, long long n_snap,
                                                              double *out, unsigned *fail)
{
    extern __shared__ __align__(16) unsigned char btsm[];
    __shared__ __align__(8) unsigned long long bar_mem;
    __shared__ uint32_t tslot;
    __shared__ int stop;
    unsigned char *T = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(btsm) + 1023) & ~uintptr_t(1023));
    const float *w = g.mlp;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int D = N * dim, npair = N * (N - 1) / 2;
    const long long rows = n_snap * npair, tiles = (rows + BT_ROWS - 1) / BT_ROWS;
    const uint32_t ts = (uint32_t)__cvta_generic_to_shared(T);
    // constant tiles: W2 and W2^T, the ones row of B3, zero rows of B3 and B4
    for (int i = t; i < MLP_H * MLP_H; i += BT_ROWS) {
        const int a = i >> 6, b = i & 63;  // W2[a][b]: output a, input b
        const __nv_bfloat16 v = __float2bfloat16_rn(w[MW_W2 + i]);
        *reinterpret_cast<__nv_bfloat16 *>(T + BT_W2 + tc_off(a, b)) = v;
        *reinterpret_cast<__nv_bfloat16 *>(T + BT_W2T + tc_off(b, a)) = v;
    }
    for (int i = t; i < 16 * BT_ROWS; i += BT_ROWS) {
        const int n = i / BT_ROWS, k = i % BT_ROWS;
        if (n >= 1) {  // B3 rows 65..79 stay zero (row 64 = ones, written per tile)
            *reinterpret_cast<__nv_bfloat16 *>(T + BT_B3 + bt_off128(64 + n, k)) = __float2bfloat16_rn(0.0f);
            *reinterpret_cast<__nv_bfloat16 *>(T + BT_B3 + 20480 + bt_off128(64 + n, k)) = __float2bfloat16_rn(0.0f);
        }
        if (n >= 6) {
            *reinterpret_cast<__nv_bfloat16 *>(T + BT_B4 + bt_off128(n, k)) = __float2bfloat16_rn(0.0f);
            *reinterpret_cast<__nv_bfloat16 *>(T + BT_B4 + 4096 + bt_off128(n, k)) = __float2bfloat16_rn(0.0f);
        }
    }
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&bar_mem);
    uint32_t phase = 0;
    if (t == 0) {
        stop = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&tslot)),
                     "r"(BT_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tslot;
    const uint32_t lb = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes
    bool first = true;
    double n_rows = 0.0, e_rows = 0.0;

    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        // ---- this thread's row: pair (i, j) of snapshot sn
        const long long R = tile * BT_ROWS + t;
        const bool valid = R < rows;
        float r = 0.0f, sv = 0.0f, E = 0.0f;
        if (valid) {
            const long long sn = R / npair;
            int i, j;
            pair_of((int)(R - sn * npair), N, i, j);
            float r2 = 0.0f;
            for (int c = 0; c < dim; ++c) {
                const float d = snap_x[sn * D + i * dim + c] - snap_x[sn * D + j * dim + c];
                r2 += d * d;
            }
            r = sqrtf(r2);
            sv = same_spin(i, j, N) ? 1.0f : 0.0f;
            E = snap_e ? (float)snap_e[sn] : 0.0f;
            n_rows += 1.0;
            e_rows += snap_e ? snap_e[sn] : 0.0;
        }
        // ---- h1 into A1 (rows) and B3 (columns); the ones row; B4's weights
        for (int c = 0; c < 8; ++c) {
            uint32_t hv[4], lv[4];
            for (int e = 0; e < 4; ++e) {
                float h[2];
                for (int q = 0; q < 2; ++q) {
                    const int k = 8 * c + 2 * e + q;
                    h[q] = valid ? mlp_tanh(fmaf(w[MW_W1 + 2 * k], r, fmaf(w[MW_W1 + 2 * k + 1], sv, w[MW_B1 + k])))
                                 : 0.0f;
                    bt_put(T + BT_B3, bt_off128(k, t), 20480, h[q]);
                }
                hv[e] = pack_bf16(h[0], h[1]);
                const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162 *>(&hv[e]);
                lv[e] = pack_bf16(h[0] - __bfloat162float(hi.x), h[1] - __bfloat162float(hi.y));
            }
            *reinterpret_cast<uint4 *>(T + BT_A1 + tc_off(t, 8 * c)) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
            *reinterpret_cast<uint4 *>(T + BT_A1 + 16384 + tc_off(t, 8 * c)) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
        }
        bt_put(T + BT_B3, bt_off128(64, t), 20480, valid ? 1.0f : 0.0f);
        const float wv[6] = {valid ? 1.0f : 0.0f, E, r, sv, E * r, E * sv};
        for (int n = 0; n < 6; ++n) bt_put(T + BT_B4, bt_off128(n, t), 4096, wv[n]);
        // ---- G1: z2 = h1 W2^T
        bt_publish();
        if (t == 0)
            for (int st = 0; st < 4; ++st) {
                const uint64_t b = bt_desc(ts + BT_W2 + st * 256, 1024);
                bt_mma(tmem, bt_desc(ts + BT_A1 + st * 256, 1024), b, bt_idesc(64), st > 0);
                bt_mma(tmem, bt_desc(ts + BT_A1 + 16384 + st * 256, 1024), b, bt_idesc(64), 1);
            }
        if (!bt_commit_wait(bar, phase)) stop = 1;
        __syncthreads();
        if (stop) break;
        // ---- delta2 into A2 (rows) and A3 (columns, plain and E-weighted)
        for (int c = 0; c < 4; ++c) {
            uint32_t z[16];
            tmem_ld16(lb + 16 * c, z);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int e = 0; e < 16; e += 8) {
                uint32_t dh[4], dl[4];
                for (int q = 0; q < 8; q += 2) {
                    float dd[2];
                    for (int u = 0; u < 2; ++u) {
                        const int m = 16 * c + e + q + u;
                        const float h2 = mlp_tanh(__uint_as_float(z[e + q + u]) + w[MW_B2 + m]);
                        dd[u] = valid ? w[MW_W3 + m] * (1.0f - h2 * h2) : 0.0f;
                        bt_put(T + BT_A3, bt_off128(m, t), 32768, dd[u]);
                        bt_put(T + BT_A3, bt_off128(64 + m, t), 32768, E * dd[u]);
                    }
                    dh[q / 2] = pack_bf16(dd[0], dd[1]);
                    const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162 *>(&dh[q / 2]);
                    dl[q / 2] = pack_bf16(dd[0] - __bfloat162float(hi.x), dd[1] - __bfloat162float(hi.y));
                }
                const uint32_t off = tc_off(t, 16 * c + e);
                *reinterpret_cast<uint4 *>(T + BT_A2 + off) = make_uint4(dh[0], dh[1], dh[2], dh[3]);
                *reinterpret_cast<uint4 *>(T + BT_A2 + 16384 + off) = make_uint4(dl[0], dl[1], dl[2], dl[3]);
            }
        }
        // ---- G2: e1 = delta2 W2;  G3: [dW2 | db2] += A3 B3
        bt_publish();
        if (t == 0) {
            for (int st = 0; st < 4; ++st) {
                const uint64_t b = bt_desc(ts + BT_W2T + st * 256, 1024);
                bt_mma(tmem + 64, bt_desc(ts + BT_A2 + st * 256, 1024), b, bt_idesc(64), st > 0);
                bt_mma(tmem + 64, bt_desc(ts + BT_A2 + 16384 + st * 256, 1024), b, bt_idesc(64), 1);
            }
            for (int st = 0; st < 8; ++st) {
                const uint64_t ah = bt_desc(ts + BT_A3 + st * 256, 2048), al = bt_desc(ts + BT_A3 + 32768 + st * 256, 2048);
                const uint64_t bh = bt_desc(ts + BT_B3 + st * 256, 2048), bl = bt_desc(ts + BT_B3 + 20480 + st * 256, 2048);
                bt_mma(tmem + 128, ah, bh, bt_idesc(80), (first && st == 0) ? 0u : 1u);
                bt_mma(tmem + 128, ah, bl, bt_idesc(80), 1);
                bt_mma(tmem + 128, al, bh, bt_idesc(80), 1);
            }
        }
        if (!bt_commit_wait(bar, phase)) stop = 1;
        __syncthreads();
        if (stop) break;
        // ---- delta1 (from e1 and h1) and h2 (from z2) into A4 = [delta1^T; h2^T]:
        // hi in the A2 region, lo in the first half of the A3 region (both free now)
        for (int c = 0; c < 4; ++c) {
            uint32_t ez[16], z[16];
            tmem_ld16(lb + 64 + 16 * c, ez);
            tmem_ld16(lb + 16 * c, z);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int e = 0; e < 16; ++e) {
                const int k = 16 * c + e;
                const uint32_t o = tc_off(t, k);
                const float hk = __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(T + BT_A1 + o)) +
                                 __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(T + BT_A1 + 16384 + o));
                const float d1 = valid ? __uint_as_float(ez[e]) * (1.0f - hk * hk) : 0.0f;
                const float h2 = valid ? mlp_tanh(__uint_as_float(z[e]) + w[MW_B2 + k]) : 0.0f;
                const uint32_t o1 = bt_off128(k, t), o2 = bt_off128(64 + k, t);
                const __nv_bfloat16 a = __float2bfloat16_rn(d1), b = __float2bfloat16_rn(h2);
                *reinterpret_cast<__nv_bfloat16 *>(T + BT_A2 + o1) = a;
                *reinterpret_cast<__nv_bfloat16 *>(T + BT_A3 + o1) = __float2bfloat16_rn(d1 - __bfloat162float(a));
                *reinterpret_cast<__nv_bfloat16 *>(T + BT_A2 + o2) = b;
                *reinterpret_cast<__nv_bfloat16 *>(T + BT_A3 + o2) = __float2bfloat16_rn(h2 - __bfloat162float(b));
            }
        }
        // ---- G4: [delta1 | h2] sums += A4 B4
        bt_publish();
        if (t == 0)
            for (int st = 0; st < 8; ++st) {
                const uint64_t ah = bt_desc(ts + BT_A2 + st * 256, 2048), al = bt_desc(ts + BT_A3 + st * 256, 2048);
                const uint64_t bh = bt_desc(ts + BT_B4 + st * 256, 2048), bl = bt_desc(ts + BT_B4 + 4096 + st * 256, 2048);
                bt_mma(tmem + 208, ah, bh, bt_idesc(16), (first && st == 0) ? 0u : 1u);
                bt_mma(tmem + 208, ah, bl, bt_idesc(16), 1);
                bt_mma(tmem + 208, al, bh, bt_idesc(16), 1);
            }
        if (!bt_commit_wait(bar, phase)) stop = 1;
        __syncthreads();
        if (stop) break;
        first = false;
    }
    // ---- the TMEM sums to the FP64 output: row t of G3 and G4
    const int P = MLP_PARAMS;
    if (!stop && !first) {
        const int j = t & 63;
        double *o = out + (t < 64 ? 0 : P);  // rows 64..127: E-weighted
        for (int c = 0; c < 5; ++c) {
            uint32_t v[16];
            tmem_ld16(lb + 128 + 16 * c, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int e = 0; e < 16; ++e) {
                const int m = 16 * c + e;
                const double x = (double)__uint_as_float(v[e]);
                if (m < 64) atomicAdd(&o[MW_W2 + j * MLP_H + m], x);
                else if (m == 64) atomicAdd(&o[MW_B2 + j], x);
            }
        }
        uint32_t v[16];
        tmem_ld16(lb + 208, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (t < 64) {  // delta1 rows: 1, E, r, s, E r, E s
            const int k = t;
            atomicAdd(&out[MW_B1 + k], (double)__uint_as_float(v[0]));
            atomicAdd(&out[P + MW_B1 + k], (double)__uint_as_float(v[1]));
            atomicAdd(&out[MW_W1 + 2 * k], (double)__uint_as_float(v[2]));
            atomicAdd(&out[MW_W1 + 2 * k + 1], (double)__uint_as_float(v[3]));
            atomicAdd(&out[P + MW_W1 + 2 * k], (double)__uint_as_float(v[4]));
            atomicAdd(&out[P + MW_W1 + 2 * k + 1], (double)__uint_as_float(v[5]));
        } else {  // h2 rows: 1, E
            atomicAdd(&out[MW_W3 + (t - 64)], (double)__uint_as_float(v[0]));
            atomicAdd(&out[P + MW_W3 + (t - 64)], (double)__uint_as_float(v[1]));
        }
    }
    if (stop && t == 0) atomicOr(fail, (unsigned)ST_TC_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BT_COLS) : "memory");
    // b3: one per pair row
    if (!stop) {
        atomicAdd(&out[MW_B3], n_rows);
        atomicAdd(&out[P + MW_B3], e_rows);
    }
    // ---- the one-body network of each snapshot, warp per particle (CUDA cores)
    for (long long sn = blockIdx.x; sn < n_snap && !stop; sn += gridDim.x) {
        const double Es = snap_e ? snap_e[sn] : 0.0;
        for (int i = warp; i < N; i += BT_ROWS / 32) {
            float r2 = 0.0f;
            for (int c = 0; c < dim; ++c) r2 += snap_x[sn * D + i * dim + c] * snap_x[sn * D + i * dim + c];
            const float r = sqrtf(r2);
            const float h = mlp_tanh(fmaf(w[MW_V1 + lane], r, w[MW_C1 + lane]));
            float z = w[MW_C2 + lane];
            for (int k = 0; k < MLP_G; ++k) z = fmaf(w[MW_V2 + lane * MLP_G + k], __shfl_sync(FULL, h, k), z);
            const float h2 = mlp_tanh(z), e2 = w[MW_V3 + lane] * (1.0f - h2 * h2);
            float acc = 0.0f;
            for (int m = 0; m < MLP_G; ++m) acc = fmaf(__shfl_sync(FULL, e2, m), w[MW_V2 + m * MLP_G + lane], acc);
            const float e1 = acc * (1.0f - h * h);
            for (int k = 0; k < MLP_G; ++k) {
                const float v = e2 * __shfl_sync(FULL, h, k);
                atomicAdd(&out[MW_V2 + lane * MLP_G + k], (double)v);
                atomicAdd(&out[P + MW_V2 + lane * MLP_G + k], Es * v);
            }
            const int idx[4] = {MW_V1 + lane, MW_C1 + lane, MW_C2 + lane, MW_V3 + lane};
            const float vals[4] = {e1 * r, e1, e2, h2};
            for (int q = 0; q < 4; ++q) {
                atomicAdd(&out[idx[q]], (double)vals[q]);
                atomicAdd(&out[P + idx[q]], Es * vals[q]);
            }
        }
        if (t == 0) {
            atomicAdd(&out[MW_C3], (double)N);
            atomicAdd(&out[P + MW_C3], Es * N);
        }
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
    // record layout (doubles): x | fc | grad | energies (4) | pgrad (E p_max) | inverse (2 n n) |
    // orbital derivatives at every particle (N n 2 dim) | MLP caches
    g.off_fc = D;
    g.off_g = 2 * D;
    g.off_en = 3 * D;
    g.off_pg = 3 * D + 4;
    g.off_inv = round_up(g.off_pg + g.EP, 2);
    const bool mlp = std::count(c.elements.begin(), c.elements.end(), (int)E_MLP) > 0;
    if (mlp && (N > 32 || dim * N > 96)) return "MLP Jastrow: at most 32 particles on this engine";
    g.off_dphi = g.off_inv + 2 * g.n * g.n;               // orbital derivatives: N x n x 2 dim
    g.off_uc = g.off_dphi + N * g.n * 2 * dim;             // MLP caches: N x N x 3, N x 3
    g.off_oc = g.off_uc + (mlp ? N * N * 3 : 0);
    g.rec = round_up(g.off_oc + (mlp ? N * 3 : 0), 2);
    bool atom_set = slater && dim == 3 && g.basis == BASIS_HYDROGEN;
    for (int e : c.elements) atom_set = atom_set && (e == (int)E_SLATER || e == (int)E_PADE || e == (int)E_SIMPLEJASTROW);
    g.variant = atom_set ? GV_ATOM : GV_ANY;
    // at most 2 orbitals per block, 6 pairs and 12 coordinates: an 8-lane segment and a
    // 64-double scratch slice hold a walker
    g.seg = atom_set && N <= 4 ? 4 : 1;
    return "";
}

int gen_smem_per_warp(const GenParams &g) { return g.n * 2 * g.n * 8; }

cudaError_t gen_launch_state(const Params &P, const GenParams &g, int mode, double *o_grad, double *o_lap,
                             double *o_pg, double *o_en, cudaStream_t st)
{
    const size_t smem = (g.mlp ? MLP_SMEM_DOUBLES * sizeof(double) : 0) +
                        (mode != GEN_STATE ? (size_t)GEN_WPB * gen_smem_per_warp(g) : 0);
    // not while the stream is being captured (the batch's refresh of its FP32 atoms, a
    // few KB, within the default limit): the attribute is set outside any capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return e;
    if (cap == cudaStreamCaptureStatusNone) {
        e = cudaFuncSetAttribute(gen_state_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    gen_state_kernel<<<(P.W + GEN_WPB - 1) / GEN_WPB, 32 * GEN_WPB, smem, st>>>(P, g, mode, o_grad, o_lap, o_pg,
                                                                                o_en);
    return cudaGetLastError();
}

cudaError_t gen_launch_sweep(const SweepArgs &a, const GenParams &g, cudaStream_t st)
{
    const bool tc = g.mlp && g.mlp_tc;
    const bool atom = !tc && g.variant == GV_ATOM;
    // four walkers per warp for the small atoms (not while sampling densities, whose
    // histogram code takes a whole warp per walker)
    const int G = atom && g.seg == 4 && a.dens_bins == 0 ? 4 : 1;
    // the FP32 sweep: the compiled atom form with its record staged (every atom's is)
    const bool f32 = g.f32 && atom && gen_stage_doubles(g, a.P.nacc) > 0;
    if (g.f32 && !f32) return cudaErrorInvalidConfiguration;
    const size_t smem = (g.mlp ? MLP_SMEM_DOUBLES * sizeof(double) : 0) + (tc ? TC_SMEM : 0) +
                        (size_t)GEN_WPB * G * gen_stage_bytes(g, a.P.nacc, f32 ? 4 : 8);
    const void *fn = tc            ? (const void *)gen_sweep_kernel<true, GV_ANY>
                     : f32 && G == 4 ? (const void *)gen_sweep_kernel<false, GV_ATOM, 4, float>
                     : f32           ? (const void *)gen_sweep_kernel<false, GV_ATOM, 1, float>
                     : G == 4        ? (const void *)gen_sweep_kernel<false, GV_ATOM, 4>
                     : atom          ? (const void *)gen_sweep_kernel<false, GV_ATOM>
                                     : (const void *)gen_sweep_kernel<false, GV_ANY>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (a.P.W + GEN_WPB * G - 1) / (GEN_WPB * G);
    if (f32 && G == 4)
        gen_sweep_kernel<false, GV_ATOM, 4, float><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    else if (f32)
        gen_sweep_kernel<false, GV_ATOM, 1, float><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    else if (tc)
        gen_sweep_kernel<true, GV_ANY><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    else if (G == 4)
        gen_sweep_kernel<false, GV_ATOM, 4><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    else if (atom)
        gen_sweep_kernel<false, GV_ATOM><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    else
        gen_sweep_kernel<false, GV_ANY><<<grid, 32 * GEN_WPB, smem, st>>>(a, g);
    return cudaGetLastError();
}

}  // namespace vmc

namespace vmc {

cudaError_t mlp_launch_grad(const GenParams &g, int N, int dim, const float *snap_x, const double *snap_e,
                            long long n_snap, double *out, cudaStream_t st, unsigned *fail)
{
    if (n_snap <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (g.mlp_tc && fail) {  // pair network on the tensor cores
        cudaError_t e = cudaFuncSetAttribute(mlp_grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, BT_SMEM);
        if (e != cudaSuccess) return e;
        const long long rows = n_snap * (N * (N - 1) / 2), tiles = (rows + BT_ROWS - 1) / BT_ROWS;
        const long long grid = std::min<long long>(std::max(1LL, tiles), (long long)sms);
        mlp_grad_tc_kernel<<<(unsigned)grid, BT_ROWS, BT_SMEM, st>>>(g, N, dim, snap_x, snap_e, n_snap, out, fail);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)MG_SMEM_FLOATS * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long grid = std::min<long long>(n_snap, (long long)sms);
    mlp_grad_kernel<<<(unsigned)grid, 256, smem, st>>>(g, N, dim, snap_x, snap_e, n_snap, out);
    return cudaGetLastError();
}

}  // namespace vmc
