// The delayed updates' flush, G += A B^T over the first K columns of the
// N x nb factors A and B, by one CTA on the FP64 tensor pipe (DMMA).
#pragma once
#include "zgemm.cuh"

typedef GemmBig UpdGemm;

// G += A B^T over the first K columns of the N x nb factors (alpha = beta = 1),
// every output tile by this CTA: the accumulators start from the G tile (read
// while the first A and B stages are in flight) and are stored straight back,
// so the epilogue needs no shared-memory pass and no second read of G.
DQ_DEV void flush_addto(double2* G, const double2* A, const double2* B, int N, int K, cplx* smem) {
    typedef UpdGemm Cfg;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, FM = Cfg::FM, FN = Cfg::FN;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const bool mathw = warp < Cfg::WM * Cfg::WN;
    const int wm0 = (warp % Cfg::WM) * Cfg::WTM, wn0 = (warp / Cfg::WM) * Cfg::WTN;
    const int tm = (N + BM - 1) / BM, ntiles = tm * tm;
    ZGemmArgs g;
    g.M = N; g.N = N; g.K = K; g.alpha = cmk(1, 0); g.beta = cmk(1, 0);
    g.A = A; g.lda = N; g.opA = OP_N; g.B = B; g.ldb = N; g.opB = OP_T; g.C = G; g.ldc = N;
    cplx* As0 = smem;
    cplx* Bs0 = smem + Cfg::SA;
    cplx* As1 = smem + Cfg::SA + Cfg::SB;
    cplx* Bs1 = smem + 2 * Cfg::SA + Cfg::SB;
    const int nk = (K + BK - 1) / BK;
    for (int t = 0; t < ntiles; ++t) {
        const int m0 = (t % tm) * BM, n0 = (t / tm) * BN;
        zgemm_load_stage<Cfg>(g, m0, n0, 0, As0, Bs0, tid, nthr);
        cp_async_commit();
        double accr[FM][FN][2], acci[FM][FN][2];
#pragma unroll
        for (int a = 0; a < FM; ++a)
#pragma unroll
            for (int b = 0; b < FN; ++b) {
                const int m = m0 + wm0 + a * 8 + (lane >> 2), n = n0 + wn0 + b * 8 + (lane & 3) * 2;
                double2 c0 = cmk(0, 0), c1 = cmk(0, 0);
                if (mathw && m < N && n < N) c0 = G[MIDX(m, n, N)];
                if (mathw && m < N && n + 1 < N) c1 = G[MIDX(m, n + 1, N)];
                accr[a][b][0] = c0.x; acci[a][b][0] = c0.y;
                accr[a][b][1] = c1.x; acci[a][b][1] = c1.y;
            }
        for (int kt = 0; kt < nk; ++kt) {
            cplx* As = (kt & 1) ? As1 : As0;
            cplx* Bs = (kt & 1) ? Bs1 : Bs0;
            if (kt + 1 < nk) {
                zgemm_load_stage<Cfg>(g, m0, n0, (kt + 1) * BK, (kt & 1) ? As0 : As1, (kt & 1) ? Bs0 : Bs1, tid, nthr);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (mathw) {
#pragma unroll
                for (int kk = 0; kk < BK; kk += 4) {
                    const int kr = kk + (lane & 3);
                    double ar[FM], ai[FM], ain[FM], br[FN], bi[FN];
#pragma unroll
                    for (int a = 0; a < FM; ++a) {
                        cplx v = As[kr * Cfg::LDA + wm0 + a * 8 + (lane >> 2)];
                        ar[a] = v.x; ai[a] = v.y; ain[a] = -v.y;
                    }
#pragma unroll
                    for (int b = 0; b < FN; ++b) {
                        cplx v = Bs[kr * Cfg::LDB + wn0 + b * 8 + (lane >> 2)];
                        br[b] = v.x; bi[b] = v.y;
                    }
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
            __syncthreads();
        }
        if (mathw) {
#pragma unroll
            for (int a = 0; a < FM; ++a)
#pragma unroll
                for (int b = 0; b < FN; ++b) {
                    const int m = m0 + wm0 + a * 8 + (lane >> 2), n = n0 + wn0 + b * 8 + (lane & 3) * 2;
                    if (m < N && n < N) G[MIDX(m, n, N)] = cmk(accr[a][b][0], acci[a][b][0]);
                    if (m < N && n + 1 < N) G[MIDX(m, n + 1, N)] = cmk(accr[a][b][1], acci[a][b][1]);
                }
        }
    }
    __syncthreads();
}
