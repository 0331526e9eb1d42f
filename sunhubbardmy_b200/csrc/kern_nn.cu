// Learned effective action for global block proposals (tensor-core kernels).
//
//   h1 = tanh(W1 * s + b1)        3x3x3 periodic conv over (t, y, x), 1 -> 32 channels
//   h2 = tanh(W2 * h1 + b2)       3x3x3 periodic conv, 32 -> 32
//   S  = sum_v w3 . h2(v) + b3 V  1x1x1 conv to one channel, summed over space-time
//
// s = +-1 is the HS field (value 1 -> -1, 2 -> +1).  The 32 -> 32 layer runs on
// the fifth-generation tensor cores as an implicit GEMM per brick of 128 sites
// (M = 128 sites, N = 32 channels, K = 27 taps x 32 channels): one thread issues
// tcgen05.mma kind::f16 (BF16 x BF16 -> FP32) with the accumulator in tensor
// memory, the tap's im2col tile and the weights staged in shared memory in the
// canonical K-major layout, and the result read back with tcgen05.ld.  Its data
// gradient is the same GEMM with mirrored taps and transposed weights.  The
// weight gradient (a per-tap 32 x 32 product over sites) stays on mma.sync
// m16n8k16, and layer 1 and the reductions run on the FP32 pipes.
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
// tcgen05 (UMMA) implicit GEMM of the 32 -> 32 layer
// ---------------------------------------------------------------------------
DQ_DEV uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// canonical K-major, no-swizzle operand layout: element (row, k) of a tile with
// G groups of 8 rows sits in the 8 x 8 core matrix (k / 8, row / 8), 128 bytes
// each, core matrices k-group major: ((k / 8) G + row / 8) 64 + (row % 8) 8 + k % 8
__host__ __device__ inline int umma_canon(int row, int k, int G) {
    return ((k >> 3) * G + (row >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}
// shared-memory matrix descriptor: start address, leading (k-group) and stride
// (row-group) byte offsets, version 1, no swizzle
DQ_DEV uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 32, M = 128
constexpr uint32_t NN_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
#define NN_TAP_B 1024            // canonical weights of one tap: 32 x 32 bf16
#define NN_TILE_A 4096           // canonical im2col tile of one tap: 128 x 32 bf16
#define NN_SPIN (1 << 24)        // bound of every mbarrier wait

__device__ int g_nn_timeout;     // set when a tensor-core wait ran out (checked by the host)

DQ_DEV bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < NN_SPIN; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// Weights of the layer in canonical per-tap tiles: Bc[tap][umma_canon(n, k, 4)]
// = Wt[n][tap 32 + k] (Wt: [32 n][NN_WLD] with k = tap*32 + channel), 16-byte copies.
DQ_DEV void load_wt_canon(bf16* Bc, const bf16* Wt) {
    for (int e = threadIdx.x; e < 27 * NN_C * 4; e += blockDim.x) {
        const int n = e % NN_C, kg = (e / NN_C) & 3, tap = e / (NN_C * 4);
        *(uint4*)(Bc + tap * NN_TAP_B + umma_canon(n, kg * 8, 4)) = *(const uint4*)(Wt + (size_t)n * NN_WLD + tap * NN_C + kg * 8);
    }
}

// D[q][n] = sum_tap sum_c X(halo_row(q, tap))[c] B[n][tap 32 + c] for the 128 core
// sites q of the brick, accumulated in tensor memory (128 lanes x 32 columns).
// X: the halo (stride HLD bf16), Bc: canonical weights, At: two canonical
// im2col tiles, bars: three mbarriers, tslot: the tensor-memory address.
// Tap t's tile is gathered while the MMAs of tap t - 1 run; a tile is
// overwritten only after the MMAs that read it completed.  On return warps
// 0..3 hold the accumulator row 32 w + lane in acc[32] (other warps: zeros);
// the caller frees the tensor memory with umma_free after its last use.
// Returns false (and sets g_nn_timeout) when a wait ran out.
DQ_DEV bool conv_umma(const bf16* X, const bf16* Bc, bf16* At, uint64_t* bars, uint32_t* tslot, float acc[32]) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_addr(tslot)), "r"(32));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        for (int k = 0; k < 3; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(&bars[k])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;
    bool ok = true;
    for (int tap = 0; tap < 27; ++tap) {
        const int buf = tap & 1;
        bf16* A = At + buf * NN_TILE_A;
        if (tap >= 2) ok = mbar_wait(&bars[buf], ((tap - 2) >> 1) & 1) && ok;   // MMAs of tap - 2 done
        for (int e = tid; e < 128 * 4; e += blockDim.x) {
            // consecutive threads take consecutive rows of one k group: 16-byte
            // steps inside the core matrices, conflict-free stores
            const int m = e & 127, kg = e >> 7;
            *(uint4*)(A + umma_canon(m, kg * 8, 16)) = *(const uint4*)(X + halo_row(m, tap) * HLD + kg * 8);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint64_t da = umma_desc(smem_addr(A + c * 2 * 16 * 64), 16 * 128, 128);
                const uint64_t db = umma_desc(smem_addr(Bc + tap * NN_TAP_B + c * 2 * 4 * 64), 4 * 128, 128);
                const uint32_t en = (tap | c) ? 1u : 0u, z = 0u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                             :: "r"(tmem), "l"(da), "l"(db), "r"(NN_IDESC), "r"(en), "r"(z), "r"(z), "r"(z), "r"(z));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_addr(&bars[buf])));
        }
    }
    if (tid == 0)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(smem_addr(&bars[2])));
    ok = mbar_wait(&bars[2], 0) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
    for (int c = 0; c < 32; ++c) acc[c] = 0.f;
    if (warp < 4 && ok) {
        uint32_t r[32];
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                     "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                       "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                       "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                       "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                     : "r"(ta));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::);
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = __uint_as_float(r[c]);
    }
    if (!ok && lane == 0) atomicExch(&g_nn_timeout, 1);
    return ok;
}

// Releases the tensor memory of conv_umma (every thread of the CTA calls it).
DQ_DEV void umma_free(const uint32_t* tslot) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(*tslot), "r"(32));
}

struct NNSmem {
    float W1[27 * NN_C], b1[NN_C], b2[NN_C], w3[NN_C];
    __align__(16) float Sin[SIQ];     // rows of SIX = 12 floats, read as float4
    float red[32];
};

static_assert((27 * NN_TAP_B + HQ * HLD + 2 * NN_TILE_A) * sizeof(bf16) % 16 == 0 && SIX % 4 == 0,
              "NNSmem and its Sin rows start on 16-byte boundaries");

// canonical weights, halo, two im2col tiles, NNSmem, three mbarriers and the
// tensor-memory address
static size_t nn_fwd_smem() {
    return (size_t)(27 * NN_TAP_B + HQ * HLD + 2 * NN_TILE_A) * sizeof(bf16) + sizeof(NNSmem) + 64;
}


// Forward: S[b] += sum over the output range of field b.  train: store h1 and
// h2 (bf16, [b][v][32]) of the core sites for the backward kernels.
template <bool TRAIN>
__global__ void __launch_bounds__(256) k_nn_fwd(NNW w, NNIn in, double* S, bf16* h1g, bf16* h2g) {
    extern __shared__ __align__(16) unsigned char smraw[];
    bf16* Bc = (bf16*)smraw;
    bf16* H = Bc + 27 * NN_TAP_B;
    bf16* At = H + HQ * HLD;
    NNSmem* sm = (NNSmem*)(At + 2 * NN_TILE_A);
    uint64_t* bars = (uint64_t*)(sm + 1);
    uint32_t* tslot = (uint32_t*)(bars + 3);
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.y;
    const Brick br = brick_of(in, blockIdx.x);
    load_wt_canon(Bc, w.W2T);
    for (int e = tid; e < 27 * NN_C; e += nth) sm->W1[e] = w.W1[e];
    if (tid < NN_C) { sm->b1[tid] = w.b1[tid]; sm->b2[tid] = w.b2[tid]; sm->w3[tid] = w.w3[tid]; }
    for (int e = tid; e < SIQ; e += nth) {
        const int it = e / (SIY * SIX), iy = (e / SIX) % SIY, ix = e % SIX;
        sm->Sin[e] = field_at(in, b, in.t_lo + br.t0 - 2 + it, br.y0 - 2 + iy, br.x0 - 2 + ix);
    }
    __syncthreads();
    // layer 1 on the halo: lane = channel (its 27 weights in registers), one
    // warp per halo row of HX sites, the input rows read as float4 broadcasts
    // and reused across the three x taps (taps accumulated in order 0..26)
    {
        float w1r[27];
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) w1r[tap] = sm->W1[tap * NN_C + lane];
        const float bias = sm->b1[lane];
        for (int row = warp; row < HT * HY; row += nth >> 5) {
            const int ht = row / HY, hy = row % HY;
            float pre[HX];
#pragma unroll
            for (int hx = 0; hx < HX; ++hx) pre[hx] = bias;
#pragma unroll
            for (int tdy = 0; tdy < 9; ++tdy) {
                const float4* src = (const float4*)(sm->Sin + ((ht + tdy / 3) * SIY + (hy + tdy % 3)) * SIX);
                float sv[SIX];
#pragma unroll
                for (int k = 0; k < SIX / 4; ++k) *(float4*)&sv[4 * k] = src[k];
#pragma unroll
                for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                    for (int hx = 0; hx < HX; ++hx) pre[hx] = fmaf(w1r[tdy * 3 + dx], sv[hx + dx], pre[hx]);
            }
#pragma unroll
            for (int hx = 0; hx < HX; ++hx) H[(row * HX + hx) * HLD + lane] = __float2bfloat16(tanhf(pre[hx]));
        }
    }
    __syncthreads();
    float acc[32];
    conv_umma(H, Bc, At, bars, tslot, acc);
    // epilogue: warps 0..3 hold the row of core site q = 32 warp + lane
    float e0 = 0.f;
    const int q0 = 32 * warp + lane;
    const bool v0 = warp < 4 && core_valid(in, br, q0);
    if (v0) {
        const int s0 = core_site(in, br, q0);
        bf16 hv[NN_C];
#pragma unroll
        for (int co = 0; co < NN_C; ++co) {
            const float h2 = tanhf(acc[co] + sm->b2[co]);
            e0 = fmaf(sm->w3[co], h2, e0);
            hv[co] = __float2bfloat16(h2);
        }
        if (TRAIN) {
            uint4* dst = (uint4*)(h2g + ((size_t)b * in.V + s0) * NN_C);
#pragma unroll
            for (int k = 0; k < NN_C / 8; ++k) dst[k] = *(const uint4*)(hv + 8 * k);
        }
    }
    umma_free(tslot);
    if (TRAIN) {
        // h1 of the core sites (the halo row of tap 13 = no shift)
        for (int e = tid; e < BQ * NN_C; e += nth) {
            const int q = e / NN_C, ch = e % NN_C;
            if (core_valid(in, br, q))
                h1g[((size_t)b * in.V + core_site(in, br, q)) * NN_C + ch] = H[halo_row(q, 13) * HLD + ch];
        }
    }
    float tot = v0 ? e0 : 0.f;
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
#define NN_DP1 (NN_C + 1)     // padded dp1 row: a warp's per-site column writes hit 32 banks
struct NNBSmem {
    float W1g[27 * NN_C], b1g[NN_C], b2g[NN_C], w3g[NN_C], w3[NN_C];
    __align__(16) float Sin[SIQ];     // rows of SIX = 12 floats, read as float4
    float dp1[BQ * NN_DP1];           // dpre1 of the core sites, row q at q NN_DP1
};

// canonical weights, the dpre2 halo, NNBSmem (whose dp1 holds the two im2col
// tiles during the convolution), three mbarriers and the tensor-memory address
static size_t nn_bwd_smem() {
    return (size_t)(27 * NN_TAP_B + HQ * HLD) * sizeof(bf16) + sizeof(NNBSmem) + 64;
}
static_assert(sizeof(float) * BQ * NN_DP1 >= sizeof(bf16) * 2 * NN_TILE_A, "im2col tiles overlay dp1");
static_assert((27 * NN_TAP_B + HQ * HLD) * sizeof(bf16) % 16 == 0, "NNBSmem starts on a 16-byte boundary");

__global__ void __launch_bounds__(256) k_nn_bwd_data(NNW w, NNIn in, const double* r, const bf16* h1g, const bf16* h2g,
                                                     bf16* dp2g, float* grad) {
    extern __shared__ __align__(16) unsigned char smraw[];
    bf16* Bc = (bf16*)smraw;
    bf16* D = Bc + 27 * NN_TAP_B;          // dpre2 on the halo
    NNBSmem* sm = (NNBSmem*)(D + HQ * HLD);
    bf16* At = (bf16*)sm->dp1;             // im2col tiles, before dp1 is written
    uint64_t* bars = (uint64_t*)(sm + 1);
    uint32_t* tslot = (uint32_t*)(bars + 3);
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.y;
    const Brick br = brick_of(in, blockIdx.x);
    const float rb = (float)r[b];
    load_wt_canon(Bc, w.W2R);
    for (int e = tid; e < 27 * NN_C; e += nth) sm->W1g[e] = 0.f;
    if (tid < NN_C) { sm->b1g[tid] = 0.f; sm->b2g[tid] = 0.f; sm->w3g[tid] = 0.f; sm->w3[tid] = w.w3[tid]; }
    for (int e = tid; e < SIQ; e += nth) {
        const int it = e / (SIY * SIX), iy = (e / SIX) % SIY, ix = e % SIX;
        sm->Sin[e] = field_at(in, b, in.t_lo + br.t0 - 2 + it, br.y0 - 2 + iy, br.x0 - 2 + ix);
    }
    __syncthreads();
    // dpre2 on the halo (periodic gather of h2, 16 bytes = 8 channels a thread)
    for (int e = tid; e < HQ * 4; e += nth) {
        const int hs = e >> 2, piece = e & 3;
        const int ht = hs / (HY * HX), hy = (hs / HX) % HY, hx = hs % HX;
        const int t = pmod(in.t_lo + br.t0 - 1 + ht, in.Lt), y = pmod(br.y0 - 1 + hy, in.L), x = pmod(br.x0 - 1 + hx, in.L);
        const uint4 u = ((const uint4*)(h2g + ((size_t)b * in.V + (t * in.L + y) * in.L + x) * NN_C))[piece];
        const bf16* hv = (const bf16*)&u;
        uint4 o;
        bf16* ov = (bf16*)&o;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float h2 = __bfloat162float(hv[j]);
            ov[j] = __float2bfloat16(rb * sm->w3[piece * 8 + j] * (1.f - h2 * h2));
        }
        *(uint4*)(D + hs * HLD + piece * 8) = o;
    }
    __syncthreads();
    // core-site sums: db2 = sum dpre2, dw3 = r_b sum h2 (a thread keeps one
    // 8-channel piece; the eight lanes of a piece are summed by shuffles)
    {
        float b2p[8], w3p[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) b2p[j] = w3p[j] = 0.f;
        const int piece = tid & 3;
        for (int e = tid; e < BQ * 4; e += nth) {
            const int q = e >> 2;
            if (!core_valid(in, br, q)) continue;
            const size_t gi = ((size_t)b * in.V + core_site(in, br, q)) * NN_C + piece * 8;
            const uint4 d = *(const uint4*)(D + halo_row(q, 13) * HLD + piece * 8);
            *(uint4*)(dp2g + gi) = d;
            const uint4 u = *(const uint4*)(h2g + gi);
            const bf16* dv = (const bf16*)&d;
            const bf16* hv = (const bf16*)&u;
#pragma unroll
            for (int j = 0; j < 8; ++j) { b2p[j] += __bfloat162float(dv[j]); w3p[j] += rb * __bfloat162float(hv[j]); }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                b2p[j] += __shfl_xor_sync(0xffffffffu, b2p[j], o);
                w3p[j] += __shfl_xor_sync(0xffffffffu, w3p[j], o);
            }
        if (lane < 4) {
#pragma unroll
            for (int j = 0; j < 8; ++j) { atomicAdd(&sm->b2g[lane * 8 + j], b2p[j]); atomicAdd(&sm->w3g[lane * 8 + j], w3p[j]); }
        }
    }
    float acc[32];
    conv_umma(D, Bc, At, bars, tslot, acc);   // W2R holds mirrored taps: the transposed convolution
    // warps 0..3 hold the row of core site q = 32 warp + lane (the MMAs that
    // read the im2col tiles have completed, so dp1 may be written)
    if (warp < 4) {
        const int q0 = 32 * warp + lane;
        const bool v0 = core_valid(in, br, q0);
        uint4 h1r[NN_C / 8];      // the site's h1 row, 64 bytes
#pragma unroll
        for (int k = 0; k < NN_C / 8; ++k) h1r[k] = make_uint4(0u, 0u, 0u, 0u);
        if (v0) {
            const uint4* src = (const uint4*)(h1g + ((size_t)b * in.V + core_site(in, br, q0)) * NN_C);
#pragma unroll
            for (int k = 0; k < NN_C / 8; ++k) h1r[k] = src[k];
        }
        const bf16* h1 = (const bf16*)h1r;
#pragma unroll
        for (int ch = 0; ch < NN_C; ++ch) {
            const float hv = __bfloat162float(h1[ch]);
            sm->dp1[q0 * NN_DP1 + ch] = v0 ? acc[ch] * (1.f - hv * hv) : 0.f;
        }
    }
    umma_free(tslot);
    __syncthreads();
    // dW1[tap][c] = sum_q s(q + tap) dpre1(q)[c]; db1 = sum dpre1.  Lane =
    // channel, one warp per row of BX core sites; the field rows are read as
    // float4 broadcasts and the warps' partial sums added in shared memory.
    {
        float a[28];
#pragma unroll
        for (int k = 0; k < 28; ++k) a[k] = 0.f;
        for (int row = warp; row < BT * BY; row += nth >> 5) {
            const int qt = row / BY, qy = row % BY;
            float d[BX];
#pragma unroll
            for (int qx = 0; qx < BX; ++qx) { d[qx] = sm->dp1[(row * BX + qx) * NN_DP1 + lane]; a[27] += d[qx]; }
#pragma unroll
            for (int tdy = 0; tdy < 9; ++tdy) {
                const float4* src = (const float4*)(sm->Sin + ((qt + 1 + tdy / 3) * SIY + (qy + 1 + tdy % 3)) * SIX);
                float sv[SIX];
#pragma unroll
                for (int k = 0; k < SIX / 4; ++k) *(float4*)&sv[4 * k] = src[k];
#pragma unroll
                for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                    for (int qx = 0; qx < BX; ++qx) a[tdy * 3 + dx] = fmaf(sv[qx + 1 + dx], d[qx], a[tdy * 3 + dx]);
            }
        }
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) atomicAdd(&sm->W1g[tap * NN_C + lane], a[tap]);
        atomicAdd(&sm->b1g[lane], a[27]);
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
// backward, weight part: dW2[tap][ci][co] = sum over fields b and core sites q
// of h1(q + tap)[ci] dpre2(q)[co], per brick a 32 x 32 GEMM with K = 128 sites
// for each tap.  Grid (CTAs, 3): blockIdx.y = dt, the nine warps take the nine
// taps (dt, dy, dx).  A CTA walks bricks x fields holding its warps' 32 x 32
// tiles in registers and adds them to grad once; each job's gather (the h1
// halo slices dt .. dt + BT - 1 and the dpre2 core) is loaded into registers
// while the previous job's MMAs run.
// ---------------------------------------------------------------------------
#define WG_THREADS 288
#define WG_H (BT * HY * HX)                                  // halo sites of one dt range: 144
#define WG_PIECES ((WG_H + BQ) * NN_C / 8)                    // 16-byte pieces per job: 1088
#define WG_PER ((WG_PIECES + WG_THREADS - 1) / WG_THREADS)   // 4

__global__ void __launch_bounds__(WG_THREADS, 2) k_nn_wgrad(NNIn in, int nbricks, int B, const bf16* h1g,
                                                        const bf16* dp2g, float* grad) {
    extern __shared__ __align__(16) unsigned char smraw[];
    bf16* H = (bf16*)smraw;                             // h1 halo, HQ x HLD (slices dt .. dt + BT - 1 filled)
    bf16* D = H + HQ * HLD;                             // dpre2 core, BQ x HLD
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int dt = blockIdx.y, tap = 9 * dt + warp;
    const int njobs = nbricks * B;
    uint4 pre[WG_PER];
    auto fetch = [&](int job) {
        const int b = job / nbricks;
        const Brick br = brick_of(in, job % nbricks);
#pragma unroll
        for (int k = 0; k < WG_PER; ++k) {
            const int e = tid + k * WG_THREADS, r = e >> 2, piece = e & 3;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r < WG_H) {
                const int hs = dt * HY * HX + r;
                const int ht = hs / (HY * HX), hy = (hs / HX) % HY, hx = hs % HX;
                const int t = pmod(in.t_lo + br.t0 - 1 + ht, in.Lt), y = pmod(br.y0 - 1 + hy, in.L),
                          x = pmod(br.x0 - 1 + hx, in.L);
                v = ((const uint4*)(h1g + ((size_t)b * in.V + (t * in.L + y) * in.L + x) * NN_C))[piece];
            } else if (r < WG_H + BQ && core_valid(in, br, r - WG_H)) {
                v = ((const uint4*)(dp2g + ((size_t)b * in.V + core_site(in, br, r - WG_H)) * NN_C))[piece];
            }
            pre[k] = v;
        }
    };
    float c[2][4][4] = {};
    int job = blockIdx.x;
    if (job < njobs) fetch(job);
    for (; job < njobs; job += gridDim.x) {
        __syncthreads();                                // the previous job's MMAs are done with H and D
#pragma unroll
        for (int k = 0; k < WG_PER; ++k) {
            const int e = tid + k * WG_THREADS, r = e >> 2, piece = e & 3;
            if (r < WG_H + BQ) {
                bf16* dst = r < WG_H ? H + (dt * HY * HX + r) * HLD : D + (r - WG_H) * HLD;
                *(uint4*)(dst + piece * 8) = pre[k];
            }
        }
        __syncthreads();
        if (job + (int)gridDim.x < njobs) fetch(job + gridDim.x);
        const int mm = lane >> 3;
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
    }
    const int g = lane >> 2, t4 = lane & 3;
    float* dst = grad + NN_GW2 + tap * NN_C * NN_C;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int ci0 = mt * 16 + g, co = 8 * j + 2 * t4;
            atomicAdd((float2*)(dst + ci0 * NN_C + co), make_float2(c[mt][j][0], c[mt][j][1]));
            atomicAdd((float2*)(dst + (ci0 + 8) * NN_C + co), make_float2(c[mt][j][2], c[mt][j][3]));
        }
}
static size_t nn_wgrad_smem() { return (size_t)(HQ + BQ) * HLD * sizeof(bf16); }
static_assert(NN_GW2 % 2 == 0, "float2 atomics on the W2 gradient");

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
    cudaFuncSetAttribute(k_nn_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nn_wgrad_smem());
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
    // about two CTAs per SM over the three tap groups; each CTA adds its
    // 9 x 32 x 32 tile to grad once
    int nb = nn_nbricks(in);
    int gx = std::max(1, std::min(nb * B, (2 * nsm + 2) / 3));
    k_nn_wgrad<<<dim3(gx, 3), WG_THREADS, nn_wgrad_smem(), st>>>(in, nb, B, h1g, dp2g, grad);
}

void launch_nn_adam(float* theta, const float* grad, float* m1, float* m2, int n, float lr, float b1c, float b2c,
                    bf16* W2T, bf16* W2R, cudaStream_t st) {
    k_nn_adam<<<(n + 255) / 256, 256, 0, st>>>(theta, grad, m1, m2, n, lr, b1c, b2c);
    k_nn_pack<<<(NN_C * NN_WLD + 255) / 256, 256, 0, st>>>(theta, W2T, W2R);
}

void launch_nn_pack(const float* theta, bf16* W2T, bf16* W2R, cudaStream_t st) {
    k_nn_pack<<<(NN_C * NN_WLD + 255) / 256, 256, 0, st>>>(theta, W2T, W2R);
}

// 1 when a tensor-core wait of the network kernels ran out since the last call (then cleared)
int nn_timed_out() {
    int v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, g_nn_timeout, sizeof(int));
    if (v) cudaMemcpyToSymbol(g_nn_timeout, &z, sizeof(int));
    return v;
}
