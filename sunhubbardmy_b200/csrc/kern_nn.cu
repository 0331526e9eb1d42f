// Learned effective action for global block proposals (tensor-core kernels).
//
//   h1 = tanh(W1 * s + b1)        3x3x3 periodic conv over (t, y, x), 1 -> 32 channels
//   h2 = tanh(W2 * h1 + b2)       3x3x3 periodic conv, 32 -> 32
//   S  = sum_v w3 . h2(v) + b3 V  1x1x1 conv to one channel, summed over space-time
//
// s = +-1 is the HS field (value 1 -> -1, 2 -> +1).  The 32 -> 32 layer runs on
// the tensor cores as an implicit GEMM (M = sites, N = 32, K = 27 taps x 32
// channels) with mma.sync m16n8k16 BF16 x BF16 -> FP32: BF16 weights and
// activations, FP32 accumulation.  Its data gradient is the same GEMM with
// mirrored taps and transposed weights; its weight gradient is a per-tap GEMM
// over sites.  Layer 1 and the reductions run on the FP32 pipes.
//
// Sites are processed in bricks of 4 x 4 x 8 (t, y, x) with a one-site halo
// for layer 2 (two for layer 1), gathered with periodic wrap-around.
#include <cuda_bf16.h>
#include "chain_access.cuh"
#include "kernels.h"
#include "nn.h"

typedef __nv_bfloat16 bf16;

#define NN_C 32
#define NN_K 864              // 27 taps x 32 channels
#define NN_WLD 872            // padded bf16 row of the weight tiles (436 words = 20 mod 32: conflict-free ldmatrix)
#define BT 4
#define BY 4
#define BX 8
#define BQ (BT * BY * BX)     // 128 core sites, 16 per warp
#define HT (BT + 2)
#define HY (BY + 2)
#define HX (BX + 2)
#define HQ (HT * HY * HX)     // 360 halo sites
#define SIT (BT + 4)
#define SIY (BY + 4)
#define SIX (BX + 4)
#define SIQ (SIT * SIY * SIX) // 768 input sites
#define HLD 40                // bf16 per halo row (20 words: conflict-free ldmatrix)

DQ_DEV int pmod(int a, int n) { a %= n; return a < 0 ? a + n : a; }

DQ_DEV void ldsm_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
DQ_DEV void ldsm_x4_t(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
DQ_DEV void mma_bf16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// brick geometry of the output range
struct Brick { int t0, y0, x0; };
DQ_DEV Brick brick_of(const NNIn& in, int id) {
    const int nbx = (in.L + BX - 1) / BX, nby = (in.L + BY - 1) / BY;
    Brick b;
    b.x0 = (id % nbx) * BX;
    b.y0 = ((id / nbx) % nby) * BY;
    b.t0 = (id / (nbx * nby)) * BT;    // relative to t_lo
    return b;
}
DQ_DEV bool core_valid(const NNIn& in, const Brick& br, int q) {
    const int qt = q / (BY * BX), qy = (q / BX) % BY, qx = q % BX;
    return br.t0 + qt < in.nT && br.y0 + qy < in.L && br.x0 + qx < in.L;
}
DQ_DEV int core_site(const NNIn& in, const Brick& br, int q) {   // global site index v = (t L + y) L + x
    const int qt = q / (BY * BX), qy = (q / BX) % BY, qx = q % BX;
    const int t = pmod(in.t_lo + br.t0 + qt, in.Lt);
    return (t * in.L + (br.y0 + qy)) * in.L + (br.x0 + qx);
}
// halo row of core site q shifted by tap (dt, dy, dx in 0..2)
DQ_DEV int halo_row(int q, int tap) {
    const int qt = q / (BY * BX), qy = (q / BX) % BY, qx = q % BX;
    const int dt = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
    return ((qt + dt) * HY + (qy + dy)) * HX + (qx + dx);
}

// the HS field as +-1 at (t, y, x) of field b (periodic coordinates)
DQ_DEV float field_at(const NNIn& in, int b, int t, int y, int x) {
    t = pmod(t, in.Lt); y = pmod(y, in.L); x = pmod(x, in.L);
    const int v = (t * in.L + y) * in.L + x;
    if (in.mode == 0) return (float)in.f8[(size_t)b * in.V + v];
    const ChainDev& c = in.chains[b >> 1];
    float s = (float)(2 * c.conf[(size_t)t * c.N + y * in.L + x] - 3);
    if (b & 1) {   // odd fields: the chain's proposed block flipped
        const int* bd = c.blk + c.N;   // [N+4..N+6] = block origin (t, y, x), extents NN_BLK_*
        const int dt = pmod(t - bd[4], in.Lt), dy = pmod(y - bd[5], in.L), dx = pmod(x - bd[6], in.L);
        if (dt < NN_BLK_T && dy < NN_BLK_Y && dx < NN_BLK_X) s = -s;
    }
    return s;
}

// ---------------------------------------------------------------------------
// layer-2 implicit GEMM of one warp: acc[4][4] (n-tiles of 8 channels) for the
// warp's 16 core sites; A rows from the halo H (stride HLD), B from Wt
// ([32 n][NN_WLD], k = tap*32 + channel)
// ---------------------------------------------------------------------------
DQ_DEV void conv_mma(const bf16* H, const bf16* Wt, int warp, int lane, float acc[4][4]) {
    const int r = (lane & 7) + ((lane >> 3) & 1) * 8;
    const int koffA = (lane >> 4) * 8;
    const int q = warp * 16 + r;
    const int m = lane >> 3;
    const int nB = (m >> 1) * 8 + (lane & 7), koffB = (m & 1) * 8;
#pragma unroll 1
    for (int tap = 0; tap < 27; ++tap) {
        const bf16* arow = H + halo_row(q, tap) * HLD + koffA;
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            uint32_t a0, a1, a2, a3, b0, b1, b2, b3, b4, b5, b6, b7;
            ldsm_x4(a0, a1, a2, a3, arow + ch * 16);
            const int kb = tap * 32 + ch * 16 + koffB;
            ldsm_x4(b0, b1, b2, b3, Wt + nB * NN_WLD + kb);
            ldsm_x4(b4, b5, b6, b7, Wt + (nB + 16) * NN_WLD + kb);
            mma_bf16(acc[0], a0, a1, a2, a3, b0, b1);
            mma_bf16(acc[1], a0, a1, a2, a3, b2, b3);
            mma_bf16(acc[2], a0, a1, a2, a3, b4, b5);
            mma_bf16(acc[3], a0, a1, a2, a3, b6, b7);
        }
    }
}

struct NNSmem {
    float W1[27 * NN_C], b1[NN_C], b2[NN_C], w3[NN_C];
    float Sin[SIQ];
    float red[32];
};

static size_t nn_fwd_smem() {
    return (size_t)NN_C * NN_WLD * sizeof(bf16) + (size_t)HQ * HLD * sizeof(bf16) + sizeof(NNSmem) + 64;
}

DQ_DEV void load_wt(bf16* dst, const bf16* src) {
    const uint4* s4 = (const uint4*)src;
    uint4* d4 = (uint4*)dst;
    for (int e = threadIdx.x; e < NN_C * NN_WLD / 8; e += blockDim.x) d4[e] = s4[e];
}

// Forward: S[b] += sum over the output range of field b.  train: store h1 and
// h2 (bf16, [b][v][32]) of the core sites for the backward kernels.
template <bool TRAIN>
__global__ void __launch_bounds__(256) k_nn_fwd(NNW w, NNIn in, double* S, bf16* h1g, bf16* h2g) {
    extern __shared__ __align__(16) unsigned char smraw[];
    bf16* Wt = (bf16*)smraw;
    bf16* H = Wt + NN_C * NN_WLD;
    NNSmem* sm = (NNSmem*)(H + HQ * HLD);
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.y;
    const Brick br = brick_of(in, blockIdx.x);
    load_wt(Wt, w.W2T);
    for (int e = tid; e < 27 * NN_C; e += nth) sm->W1[e] = w.W1[e];
    if (tid < NN_C) { sm->b1[tid] = w.b1[tid]; sm->b2[tid] = w.b2[tid]; sm->w3[tid] = w.w3[tid]; }
    for (int e = tid; e < SIQ; e += nth) {
        const int it = e / (SIY * SIX), iy = (e / SIX) % SIY, ix = e % SIX;
        sm->Sin[e] = field_at(in, b, in.t_lo + br.t0 - 2 + it, br.y0 - 2 + iy, br.x0 - 2 + ix);
    }
    __syncthreads();
    // layer 1 on the halo
    for (int e = tid; e < HQ * NN_C; e += nth) {
        const int hs = e / NN_C, ch = e % NN_C;
        const int ht = hs / (HY * HX), hy = (hs / HX) % HY, hx = hs % HX;
        float pre = sm->b1[ch];
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) {
            const int dt = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
            pre = fmaf(sm->W1[tap * NN_C + ch], sm->Sin[((ht + dt) * SIY + (hy + dy)) * SIX + (hx + dx)], pre);
        }
        H[hs * HLD + ch] = __float2bfloat16(tanhf(pre));
    }
    __syncthreads();
    float acc[4][4] = {};
    conv_mma(H, Wt, warp, lane, acc);
    // epilogue: rows g and g + 8 of the warp's 16 sites, channels 8j + 2t, +1
    const int g = lane >> 2, t4 = lane & 3;
    float e0 = 0.f, e1 = 0.f;
    const int q0 = warp * 16 + g, q1 = q0 + 8;
    const bool v0 = core_valid(in, br, q0), v1 = core_valid(in, br, q1);
    const int s0 = v0 ? core_site(in, br, q0) : 0, s1 = v1 ? core_site(in, br, q1) : 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int co = 8 * j + 2 * t4 + cc;
            const float h20 = tanhf(acc[j][cc] + sm->b2[co]);
            const float h21 = tanhf(acc[j][2 + cc] + sm->b2[co]);
            e0 = fmaf(sm->w3[co], h20, e0);
            e1 = fmaf(sm->w3[co], h21, e1);
            if (TRAIN) {
                if (v0) h2g[((size_t)b * in.V + s0) * NN_C + co] = __float2bfloat16(h20);
                if (v1) h2g[((size_t)b * in.V + s1) * NN_C + co] = __float2bfloat16(h21);
            }
        }
    if (TRAIN) {
        // h1 of the core sites (the halo row of tap 13 = no shift)
        for (int e = tid; e < BQ * NN_C; e += nth) {
            const int q = e / NN_C, ch = e % NN_C;
            if (core_valid(in, br, q))
                h1g[((size_t)b * in.V + core_site(in, br, q)) * NN_C + ch] = H[halo_row(q, 13) * HLD + ch];
        }
    }
    float tot = (v0 ? e0 : 0.f) + (v1 ? e1 : 0.f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) sm->red[warp] = tot;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        int nv = 0;
        for (int k = 0; k < nth / 32; ++k) s += sm->red[k];
        for (int q = 0; q < BQ; ++q) nv += core_valid(in, br, q);
        s += (double)w.b3 * nv;
        atomicAdd(&S[b], s);
    }
}

// ---------------------------------------------------------------------------
// backward, data part: dpre2 = r_b w3 (1 - h2^2); dh1 = conv^T(W2, dpre2);
// dpre1 = dh1 (1 - h1^2); accumulates dW1, db1, db2, dw3, db3 and writes dpre2
// (bf16, [b][v][32]) for the weight-gradient kernel.
// ---------------------------------------------------------------------------
struct NNBSmem {
    float W1g[27 * NN_C], b1g[NN_C], b2g[NN_C], w3g[NN_C], w3[NN_C];
    float Sin[SIQ];
    float dp1[BQ * NN_C];
};

static size_t nn_bwd_smem() {
    return (size_t)NN_C * NN_WLD * sizeof(bf16) + (size_t)HQ * HLD * sizeof(bf16) + sizeof(NNBSmem) + 64;
}

__global__ void __launch_bounds__(256) k_nn_bwd_data(NNW w, NNIn in, const double* r, const bf16* h1g, const bf16* h2g,
                                                     bf16* dp2g, float* grad) {
    extern __shared__ __align__(16) unsigned char smraw[];
    bf16* Wt = (bf16*)smraw;
    bf16* D = Wt + NN_C * NN_WLD;          // dpre2 on the halo
    NNBSmem* sm = (NNBSmem*)(D + HQ * HLD);
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.y;
    const Brick br = brick_of(in, blockIdx.x);
    const float rb = (float)r[b];
    load_wt(Wt, w.W2R);
    for (int e = tid; e < 27 * NN_C; e += nth) sm->W1g[e] = 0.f;
    if (tid < NN_C) { sm->b1g[tid] = 0.f; sm->b2g[tid] = 0.f; sm->w3g[tid] = 0.f; sm->w3[tid] = w.w3[tid]; }
    for (int e = tid; e < SIQ; e += nth) {
        const int it = e / (SIY * SIX), iy = (e / SIX) % SIY, ix = e % SIX;
        sm->Sin[e] = field_at(in, b, in.t_lo + br.t0 - 2 + it, br.y0 - 2 + iy, br.x0 - 2 + ix);
    }
    __syncthreads();
    // dpre2 on the halo (periodic gather of h2)
    for (int e = tid; e < HQ * NN_C; e += nth) {
        const int hs = e / NN_C, ch = e % NN_C;
        const int ht = hs / (HY * HX), hy = (hs / HX) % HY, hx = hs % HX;
        const int t = pmod(in.t_lo + br.t0 - 1 + ht, in.Lt), y = pmod(br.y0 - 1 + hy, in.L), x = pmod(br.x0 - 1 + hx, in.L);
        const float h2 = __bfloat162float(h2g[((size_t)b * in.V + (t * in.L + y) * in.L + x) * NN_C + ch]);
        D[hs * HLD + ch] = __float2bfloat16(rb * sm->w3[ch] * (1.f - h2 * h2));
    }
    __syncthreads();
    // core-site sums: db2 = sum dpre2, dw3 = r_b sum h2
    for (int e = tid; e < BQ * NN_C; e += nth) {
        const int q = e / NN_C, ch = e % NN_C;
        if (!core_valid(in, br, q)) continue;
        const size_t gi = ((size_t)b * in.V + core_site(in, br, q)) * NN_C + ch;
        const bf16 d = D[halo_row(q, 13) * HLD + ch];
        dp2g[gi] = d;
        atomicAdd(&sm->b2g[ch], __bfloat162float(d));
        atomicAdd(&sm->w3g[ch], rb * __bfloat162float(h2g[gi]));
    }
    float acc[4][4] = {};
    conv_mma(D, Wt, warp, lane, acc);   // W2R holds mirrored taps: the transposed convolution
    const int g = lane >> 2, t4 = lane & 3;
    const int q0 = warp * 16 + g, q1 = q0 + 8;
    const bool v0 = core_valid(in, br, q0), v1 = core_valid(in, br, q1);
    const int s0 = v0 ? core_site(in, br, q0) : 0, s1 = v1 ? core_site(in, br, q1) : 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int ch = 8 * j + 2 * t4 + cc;
            float d0 = 0.f, d1 = 0.f;
            if (v0) { float h1 = __bfloat162float(h1g[((size_t)b * in.V + s0) * NN_C + ch]); d0 = acc[j][cc] * (1.f - h1 * h1); }
            if (v1) { float h1 = __bfloat162float(h1g[((size_t)b * in.V + s1) * NN_C + ch]); d1 = acc[j][2 + cc] * (1.f - h1 * h1); }
            sm->dp1[q0 * NN_C + ch] = d0;
            sm->dp1[q1 * NN_C + ch] = d1;
        }
    __syncthreads();
    // dW1[tap][c] = sum_q s(q + tap) dpre1(q)[c]; db1 = sum dpre1
    for (int e = tid; e < 28 * NN_C; e += nth) {
        const int tap = e / NN_C, ch = e % NN_C;
        float a = 0.f;
        for (int q = 0; q < BQ; ++q) {
            const float d = sm->dp1[q * NN_C + ch];
            if (tap == 27) { a += d; continue; }
            const int qt = q / (BY * BX), qy = (q / BX) % BY, qx = q % BX;
            const int dt = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
            a = fmaf(sm->Sin[((qt + 1 + dt) * SIY + (qy + 1 + dy)) * SIX + (qx + 1 + dx)], d, a);
        }
        if (tap < 27) sm->W1g[tap * NN_C + ch] = a;
        else sm->b1g[ch] = a;
    }
    __syncthreads();
    // gradient layout: W1 [27][32], b1 [32], W2 [27][32][32], b2 [32], w3 [32], b3
    for (int e = tid; e < 27 * NN_C; e += nth) atomicAdd(&grad[e], sm->W1g[e]);
    if (tid < NN_C) {
        atomicAdd(&grad[NN_GB1 + tid], sm->b1g[tid]);
        atomicAdd(&grad[NN_GB2 + tid], sm->b2g[tid]);
        atomicAdd(&grad[NN_GW3 + tid], sm->w3g[tid]);
    }
    if (tid == 0) {
        int nv = 0;
        for (int q = 0; q < BQ; ++q) nv += core_valid(in, br, q);
        atomicAdd(&grad[NN_GB3], rb * (float)nv);
    }
}

// ---------------------------------------------------------------------------
// backward, weight part: dW2[tap][ci][co] = sum_v h1(v + tap)[ci] dpre2(v)[co],
// per brick as 27 GEMMs (M = ci, N = co, K = 128 sites); a persistent CTA
// accumulates its bricks in shared memory and adds them to grad once.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_nn_wgrad(NNIn in, int nbricks, int B, const bf16* h1g, const bf16* dp2g,
                                                  float* grad) {
    extern __shared__ __align__(16) unsigned char smraw[];
    float* acc_s = (float*)smraw;                       // 27 x 32 x 32
    bf16* H = (bf16*)(acc_s + 27 * NN_C * NN_C);        // h1 halo, HQ x HLD
    bf16* D = H + HQ * HLD;                             // dpre2 core, BQ x HLD
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < 27 * NN_C * NN_C; e += nth) acc_s[e] = 0.f;
    for (int job = blockIdx.x; job < nbricks * B; job += gridDim.x) {
        const int b = job / nbricks;
        const Brick br = brick_of(in, job % nbricks);
        __syncthreads();
        for (int e = tid; e < HQ * NN_C; e += nth) {
            const int hs = e / NN_C, ch = e % NN_C;
            const int ht = hs / (HY * HX), hy = (hs / HX) % HY, hx = hs % HX;
            const int t = pmod(in.t_lo + br.t0 - 1 + ht, in.Lt), y = pmod(br.y0 - 1 + hy, in.L), x = pmod(br.x0 - 1 + hx, in.L);
            H[hs * HLD + ch] = h1g[((size_t)b * in.V + (t * in.L + y) * in.L + x) * NN_C + ch];
        }
        for (int e = tid; e < BQ * NN_C; e += nth) {
            const int q = e / NN_C, ch = e % NN_C;
            D[q * HLD + ch] = core_valid(in, br, q) ? dp2g[((size_t)b * in.V + core_site(in, br, q)) * NN_C + ch]
                                                    : __float2bfloat16(0.f);
        }
        __syncthreads();
        const int mm = lane >> 3;
        for (int tap = warp; tap < 27; tap += nth / 32) {
            float c[2][4][4] = {};
#pragma unroll 1
            for (int kb = 0; kb < BQ; kb += 16) {
                uint32_t a[2][4], bq[2][4];
                // A[m = ci][k = site]: stored rows = sites (k), columns = ci -> transposed loads
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    const int site = kb + (mm >> 1) * 8 + (lane & 7);
                    const bf16* p = H + halo_row(site, tap) * HLD + mt * 16 + (mm & 1) * 8;
                    ldsm_x4_t(a[mt][0], a[mt][1], a[mt][2], a[mt][3], p);
                }
                // B[k = site][n = co]: stored rows = sites, columns = co -> transposed loads
#pragma unroll
                for (int np = 0; np < 2; ++np) {
                    const int site = kb + (mm & 1) * 8 + (lane & 7);
                    const bf16* p = D + site * HLD + np * 16 + (mm >> 1) * 8;
                    ldsm_x4_t(bq[np][0], bq[np][1], bq[np][2], bq[np][3], p);
                }
#pragma unroll
                for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                    for (int np = 0; np < 2; ++np) {
                        mma_bf16(c[mt][2 * np], a[mt][0], a[mt][1], a[mt][2], a[mt][3], bq[np][0], bq[np][1]);
                        mma_bf16(c[mt][2 * np + 1], a[mt][0], a[mt][1], a[mt][2], a[mt][3], bq[np][2], bq[np][3]);
                    }
            }
            const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int ci0 = mt * 16 + g, co = 8 * j + 2 * t4;
                    float* dst = acc_s + (tap * NN_C) * NN_C;
                    dst[ci0 * NN_C + co] += c[mt][j][0];
                    dst[ci0 * NN_C + co + 1] += c[mt][j][1];
                    dst[(ci0 + 8) * NN_C + co] += c[mt][j][2];
                    dst[(ci0 + 8) * NN_C + co + 1] += c[mt][j][3];
                }
        }
    }
    __syncthreads();
    for (int e = tid; e < 27 * NN_C * NN_C; e += nth) atomicAdd(&grad[NN_GW2 + e], acc_s[e]);
}

// Adam on the FP32 master weights, then the BF16 tiles of W2 for both GEMMs.
__global__ void k_nn_adam(float* theta, const float* grad, float* m1, float* m2, int n, float lr, float b1c, float b2c) {
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        const float a = beta1 * m1[i] + (1.f - beta1) * gi;
        const float v = beta2 * m2[i] + (1.f - beta2) * gi * gi;
        m1[i] = a; m2[i] = v;
        theta[i] -= lr * (a / b1c) / (sqrtf(v / b2c) + eps);
    }
}

__global__ void k_nn_pack(const float* theta, bf16* W2T, bf16* W2R) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NN_C * NN_WLD; e += gridDim.x * blockDim.x) {
        const int n = e / NN_WLD, k = e % NN_WLD;
        float vt = 0.f, vr = 0.f;
        if (k < NN_K) {
            const int tap = k / NN_C, j = k % NN_C;
            vt = theta[NN_GW2 + (tap * NN_C + j) * NN_C + n];              // W2[tap][ci = j][co = n]
            vr = theta[NN_GW2 + ((26 - tap) * NN_C + n) * NN_C + j];       // W2[mirror tap][ci = n][co = j]
        }
        W2T[e] = __float2bfloat16(vt);
        W2R[e] = __float2bfloat16(vr);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int g_nn_attr = 0;
static void nn_attrs() {
    if (g_nn_attr) return;
    cudaFuncSetAttribute(k_nn_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nn_fwd_smem());
    cudaFuncSetAttribute(k_nn_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nn_fwd_smem());
    cudaFuncSetAttribute(k_nn_bwd_data, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nn_bwd_smem());
    size_t wg = (size_t)27 * NN_C * NN_C * sizeof(float) + (size_t)(HQ + BQ) * HLD * sizeof(bf16) + 64;
    cudaFuncSetAttribute(k_nn_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wg);
    g_nn_attr = 1;
}

int nn_nbricks(const NNIn& in) {
    return ((in.nT + BT - 1) / BT) * ((in.L + BY - 1) / BY) * ((in.L + BX - 1) / BX);
}

void launch_nn_forward(const NNW& w, const NNIn& in, int B, double* S, bf16* h1g, bf16* h2g, cudaStream_t st) {
    nn_attrs();
    dim3 grid(nn_nbricks(in), B);
    if (h1g) k_nn_fwd<true><<<grid, 256, nn_fwd_smem(), st>>>(w, in, S, h1g, h2g);
    else k_nn_fwd<false><<<grid, 256, nn_fwd_smem(), st>>>(w, in, S, nullptr, nullptr);
}

void launch_nn_backward(const NNW& w, const NNIn& in, int B, const double* r, const bf16* h1g, const bf16* h2g,
                        bf16* dp2g, float* grad, int nsm, cudaStream_t st) {
    nn_attrs();
    dim3 grid(nn_nbricks(in), B);
    k_nn_bwd_data<<<grid, 256, nn_bwd_smem(), st>>>(w, in, r, h1g, h2g, dp2g, grad);
    size_t wg = (size_t)27 * NN_C * NN_C * sizeof(float) + (size_t)(HQ + BQ) * HLD * sizeof(bf16) + 64;
    int nb = nn_nbricks(in);
    int g = std::min(nb * B, nsm);
    k_nn_wgrad<<<g, 256, wg, st>>>(in, nb, B, h1g, dp2g, grad);
}

void launch_nn_adam(float* theta, const float* grad, float* m1, float* m2, int n, float lr, float b1c, float b2c,
                    bf16* W2T, bf16* W2R, cudaStream_t st) {
    k_nn_adam<<<(n + 255) / 256, 256, 0, st>>>(theta, grad, m1, m2, n, lr, b1c, b2c);
    k_nn_pack<<<(NN_C * NN_WLD + 255) / 256, 256, 0, st>>>(theta, W2T, W2R);
}

void launch_nn_pack(const float* theta, bf16* W2T, bf16* W2R, cudaStream_t st) {
    k_nn_pack<<<(NN_C * NN_WLD + 255) / 256, 256, 0, st>>>(theta, W2T, W2R);
}
