// CTA-level complex FP64 GEMM on the FP64 tensor pipe (DMMA, mma.sync m8n8k4).
//
//   C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C
//
// Operand tiles are staged global -> shared with 16-byte cp.async (one complex
// element per copy, zero-filled outside the matrix) in a ring of Cfg::NS
// stages with one CTA barrier per stage.
// A complex product is four real DMMAs on split real/imaginary fragments:
//   Cr += Ar Br - Ai Bi,  Ci += Ar Bi + Ai Br.
// The CTA walks output tiles tile0, tile0+tstep, ..., so a single CTA can do a
// whole matrix (one CTA per Markov chain) or several CTAs can share one.
#pragma once
#include "common.cuh"

enum { OP_N = 0, OP_T = 1, OP_C = 2 };

struct ZGemmArgs {
    int M, N, K;
    cplx alpha, beta;
    const cplx* A; int lda; int opA;
    const cplx* B; int ldb; int opB;
    cplx* C; int ldc;
    // optional row gathers: row m of op(A) = A row arow[m] (opA = OP_N), row n of
    // op(B)^T = B row brow[n] (opB = OP_T / OP_C); nullptr = contiguous rows
    const int* arow = nullptr;
    const int* brow = nullptr;
    // op(A) upper triangular (opA = OP_N): A(m, k) = 0 for k < m, so a tile of
    // rows m0.. starts its k loop at m0
    int triA = 0;
};

// no `volatile`: the compiler may interleave independent DMMAs
DQ_DEV void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

DQ_DEV void cp_async16(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(s), "l"(gmem), "r"(n));
}
DQ_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
DQ_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

template <int BM_, int BN_, int BK_, int WM_, int WN_, int NS_ = 2>
struct ZGemmCfg {
    static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_;
    static constexpr int NS = NS_;                         // staging buffers (pipeline depth)
    static constexpr int NT = WM * WN * 32;
    static constexpr int WTM = BM / WM, WTN = BN / WN;
    static constexpr int FM = WTM / 8, FN = WTN / 8;
    // pitch = 2 (mod 8) in 16-byte elements: a quarter warp's fragment load
    // (k rows lane & 3, columns lane >> 2) touches 8 distinct 16-byte bank
    // groups.  (An odd pitch makes the staging stores of transposed operands
    // conflict-free instead, but doubles the wavefronts of every fragment load,
    // which run 2-4 times per stored element.)
    static constexpr int LDA = BM + 2, LDB = BN + 2;
    static constexpr int SA = BK * LDA, SB = BK * LDB;
    static constexpr int SMEM_ELEMS = NS * (SA + SB);      // double2 elements
    static_assert(BK % 4 == 0 && WTM % 8 == 0 && WTN % 8 == 0, "tile shape");
    static_assert(NS >= 2, "at least two staging buffers");
};

template <class Cfg>
DQ_DEV void zgemm_load_stage(const ZGemmArgs& g, int m0, int n0, int k0, cplx* As, cplx* Bs, int tid, int nthr) {
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
    // A tile -> As[k][m]
    if (g.opA == OP_N) {
        for (int e = tid; e < BM * BK; e += nthr) {
            int m = e % BM, k = e / BM;
            int gm = m0 + m, gk = k0 + k;
            bool v = gm < g.M && gk < g.K;
            const cplx* src = v ? g.A + MIDX(g.arow ? g.arow[gm] : gm, gk, g.lda) : g.A;
            cp_async16(&As[k * Cfg::LDA + m], src, v);
        }
    } else {
        for (int e = tid; e < BM * BK; e += nthr) {
            int k = e % BK, m = e / BK;
            int gm = m0 + m, gk = k0 + k;
            bool v = gm < g.M && gk < g.K;
            const cplx* src = v ? g.A + MIDX(gk, gm, g.lda) : g.A;
            cp_async16(&As[k * Cfg::LDA + m], src, v);
        }
    }
    // B tile -> Bs[k][n]
    if (g.opB == OP_N) {
        for (int e = tid; e < BN * BK; e += nthr) {
            int k = e % BK, n = e / BK;
            int gn = n0 + n, gk = k0 + k;
            bool v = gn < g.N && gk < g.K;
            const cplx* src = v ? g.B + MIDX(gk, gn, g.ldb) : g.B;
            cp_async16(&Bs[k * Cfg::LDB + n], src, v);
        }
    } else {
        for (int e = tid; e < BN * BK; e += nthr) {
            int n = e % BN, k = e / BN;
            int gn = n0 + n, gk = k0 + k;
            bool v = gn < g.N && gk < g.K;
            const cplx* src = v ? g.B + MIDX(g.brow ? g.brow[gn] : gn, gk, g.ldb) : g.B;
            cp_async16(&Bs[k * Cfg::LDB + n], src, v);
        }
    }
}

// Compute all tiles assigned to this CTA.  Must be called by all threads of
// the CTA (threadIdx.x < Cfg::NT do the math; extra threads only help load).
// smem must hold Cfg::SMEM_ELEMS double2.
template <class Cfg>
__device__ void zgemm_cta(const ZGemmArgs& g, int tile0, int tstep, cplx* smem) {
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, FM = Cfg::FM, FN = Cfg::FN;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const bool mathw = warp < Cfg::WM * Cfg::WN;
    const int wm0 = (warp % Cfg::WM) * Cfg::WTM, wn0 = (warp / Cfg::WM) * Cfg::WTN;
    const int tm = (g.M + BM - 1) / BM, tn = (g.N + BN - 1) / BN;
    const int ntiles = tm * tn;
    const bool conjA = (g.opA == OP_C), conjB = (g.opB == OP_C);
    const bool beta0 = (g.beta.x == 0.0 && g.beta.y == 0.0);
    constexpr int NS = Cfg::NS, SST = Cfg::SA + Cfg::SB;

    for (int t = tile0; t < ntiles; t += tstep) {
        const int m0 = (t % tm) * BM, n0 = (t / tm) * BN;
        double accr[FM][FN][2], acci[FM][FN][2];
#pragma unroll
        for (int a = 0; a < FM; ++a)
#pragma unroll
            for (int b = 0; b < FN; ++b) { accr[a][b][0] = accr[a][b][1] = acci[a][b][0] = acci[a][b][1] = 0.0; }

        const int kbeg = g.triA ? (m0 / BK) * BK : 0;
        const int nk = (g.K - kbeg + BK - 1) / BK;
        // NS-stage ring: stages 0 .. NS-2 in flight before the first product;
        // one commit group per stage (empty past the end), so that waiting
        // until NS-2 groups remain means stage kt has landed
#pragma unroll
        for (int st = 0; st < NS - 1; ++st) {
            if (st < nk) zgemm_load_stage<Cfg>(g, m0, n0, kbeg + st * BK, smem + st * SST, smem + st * SST + Cfg::SA, tid, nthr);
            cp_async_commit();
        }
        for (int kt = 0; kt < nk; ++kt) {
            cp_async_wait<NS - 2>();
            // stage kt is visible to every thread, and every warp is done with
            // stage kt - 1, whose buffer the next load reuses
            __syncthreads();
            {
                const int st = kt + NS - 1;
                if (st < nk) {
                    cplx* b = smem + (st % NS) * SST;
                    zgemm_load_stage<Cfg>(g, m0, n0, kbeg + st * BK, b, b + Cfg::SA, tid, nthr);
                }
                cp_async_commit();
            }
            const cplx* As = smem + (kt % NS) * SST;
            const cplx* Bs = As + Cfg::SA;
            if (mathw) {
#pragma unroll
                for (int kk = 0; kk < BK; kk += 4) {
                    const int kr = kk + (lane & 3);
                    double ar[FM], ai[FM], ain[FM], br[FN], bi[FN];
#pragma unroll
                    for (int a = 0; a < FM; ++a) {
                        cplx v = As[kr * Cfg::LDA + wm0 + a * 8 + (lane >> 2)];
                        ar[a] = v.x; ai[a] = conjA ? -v.y : v.y; ain[a] = -ai[a];
                    }
#pragma unroll
                    for (int b = 0; b < FN; ++b) {
                        cplx v = Bs[kr * Cfg::LDB + wn0 + b * 8 + (lane >> 2)];
                        br[b] = v.x; bi[b] = conjB ? -v.y : v.y;
                    }
                    // four independent sweeps over the fragments, so that two
                    // DMMAs into one accumulator are 2*FM*FN instructions apart
#pragma unroll
                    for (int a = 0; a < FM; ++a)
#pragma unroll
                        for (int b = 0; b < FN; ++b) dmma(accr[a][b][0], accr[a][b][1], ar[a], br[b]);
#pragma unroll
                    for (int a = 0; a < FM; ++a)
#pragma unroll
                        for (int b = 0; b < FN; ++b) dmma(acci[a][b][0], acci[a][b][1], ar[a], bi[b]);
#pragma unroll
                    for (int a = 0; a < FM; ++a)
#pragma unroll
                        for (int b = 0; b < FN; ++b) dmma(accr[a][b][0], accr[a][b][1], ain[a], bi[b]);
#pragma unroll
                    for (int a = 0; a < FM; ++a)
#pragma unroll
                        for (int b = 0; b < FN; ++b) dmma(acci[a][b][0], acci[a][b][1], ai[a], br[b]);
                }
            }
        }
        // the next tile's first stages overwrite the buffers of the last ones
        __syncthreads();
        // epilogue straight from the accumulators: C(m, n) = alpha acc + beta C;
        // the 8 lanes of a (lane & 3) group store 8 consecutive rows of a column
        if (mathw) {
#pragma unroll
            for (int a = 0; a < FM; ++a)
#pragma unroll
                for (int b = 0; b < FN; ++b)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int gm = m0 + wm0 + a * 8 + (lane >> 2), gn = n0 + wn0 + b * 8 + (lane & 3) * 2 + h;
                        if (gm < g.M && gn < g.N) {
                            cplx* cp = g.C + MIDX(gm, gn, g.ldc);
                            cplx r = cmul(g.alpha, cmk(accr[a][b][h], acci[a][b][h]));
                            if (!beta0) r = cfma(g.beta, *cp, r);
                            *cp = r;
                        }
                    }
        }
    }
    __syncthreads();     // C is complete for every thread of the CTA
}

// Default tile configurations (256 threads).
typedef ZGemmCfg<64, 64, 16, 2, 4> GemmBig;     // square-ish products
typedef ZGemmCfg<32, 64, 16, 2, 4> GemmMid;     // panels with M <= 32
typedef ZGemmCfg<16, 128, 16, 1, 8> GemmWide;   // M = 16 rows (reflector blocks)
// small shapes whose sides are multiples of 16 or 48 (the projective update's
// window GEMMs: window rows 32, ne = 144 at the benchmark size)
typedef ZGemmCfg<48, 48, 16, 3, 2> Gemm48x48;
typedef ZGemmCfg<32, 48, 16, 2, 2> Gemm32x48;
typedef ZGemmCfg<48, 32, 16, 3, 2> Gemm48x32;
typedef ZGemmCfg<32, 32, 16, 2, 2> Gemm32x32;

// tile shape with the least padded area for an M x N product (ties: larger tiles)
enum { ZT_64x64 = 0, ZT_48x48, ZT_32x48, ZT_48x32, ZT_32x32, ZT_COUNT };
__host__ __device__ inline int zt_bm(int c) { const int v[ZT_COUNT] = {64, 48, 32, 48, 32}; return v[c]; }
__host__ __device__ inline int zt_bn(int c) { const int v[ZT_COUNT] = {64, 48, 48, 32, 32}; return v[c]; }
__host__ __device__ inline int zt_tiles(int c, int M, int N) {
    return ((M + zt_bm(c) - 1) / zt_bm(c)) * ((N + zt_bn(c) - 1) / zt_bn(c));
}
__host__ __device__ inline int zt_pick(int M, int N) {
    int best = 0;
    long long ba = (long long)zt_tiles(0, M, N) * 64 * 64;
    for (int c = 1; c < ZT_COUNT; ++c) {
        long long a = (long long)zt_tiles(c, M, N) * zt_bm(c) * zt_bn(c);
        if (a < ba) { ba = a; best = c; }
    }
    return best;
}
constexpr int ZT_SMEM_ELEMS = GemmBig::SMEM_ELEMS;   // the largest of the shapes above

// tile t (0 <= t < zt_tiles) of C = alpha op(A) op(B) + beta C in shape class cls
DQ_DEV void zgemm_tile(const ZGemmArgs& g, int cls, int t, cplx* smem) {
    const int big = 1 << 30;
    switch (cls) {
    case ZT_48x48: zgemm_cta<Gemm48x48>(g, t, big, smem); break;
    case ZT_32x48: zgemm_cta<Gemm32x48>(g, t, big, smem); break;
    case ZT_48x32: zgemm_cta<Gemm48x32>(g, t, big, smem); break;
    case ZT_32x32: zgemm_cta<Gemm32x32>(g, t, big, smem); break;
    default: zgemm_cta<GemmBig>(g, t, big, smem); break;
    }
}
// every tile, by the whole CTA, in the best-fitting shape
DQ_DEV void zgemm_fit(const ZGemmArgs& g, cplx* smem) {
    const int cls = zt_pick(g.M, g.N), nt = zt_tiles(cls, g.M, g.N);
    for (int t = 0; t < nt; ++t) zgemm_tile(g, cls, t, smem);
}
