// Local Hubbard-Stratonovich updates of one time slice, one CTA per chain.
//
// Reference: src/dqmc_config_u/dqmc_update_delay.f90:1-137 (delayed update),
// dqmc_update.f90 (fast update) and dqmc_update_submatrix.f90 (submatrix
// update).  All three visit the sites in order with two SFMT draws per site
// and accept with |Re(R phase)/Re(phase)| > r; they differ only in how the
// accepted rank-1 changes are folded into G.  This kernel runs all of them as
// one scheme: the accept walk of a window of consecutive sites needs only the
// window's block of G plus the window's own new columns (the submatrix
// update's observation), all in shared memory and walked by one warp; the
// rank-1 changes are carried as delayed columns (A, B), G' = G + A B^T, and
// flushed after nublock accepted sites as one DMMA tensor-core GEMM (the
// delayed update's blocking).  The accept/reject sequence equals the
// reference's in exact arithmetic.
#include "chain_access.cuh"
#include "kernels.h"
#include "flush.cuh"

#define UPD_NT 256                 // threads per CTA

DQ_DEV double u32_to_stream(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

// Window of UPD_L consecutive sites, walked by warp 0 (lane p owns site
// w0 + p).  Its state overlays the GEMM staging buffer, which is only used by
// the flush after the window has been closed.
#define UPD_L 32
#define UPD_LP (UPD_L + 1)       // odd pitch: rows and columns of gW are both conflict-free
#define UPD_CH 4                 // window columns extended to all rows per pass
struct UpdWin {
    double2 gW[UPD_L * UPD_LP];  // G'(w0 + p, w0 + q) at gW[q * UPD_LP + p], G' = G + A B^T
    double2 aW[UPD_L][UPD_L];    // [m][p]: window row p of the window's m-th new column of A
    double2 bW[UPD_L][UPD_L];    // the same for B
    double2 sg[UPD_L];           // scale of the m-th accepted flip (delta / ratio)
    int pm[UPD_L];               // window position of the m-th accepted site
    int r, wend;                 // accepted sites; sites the walk consumed
};
static_assert(sizeof(UpdWin) % 16 == 0, "window state alignment");
// dynamic shared memory of the update kernel: the window state plus the staged
// rows (2 UPD_CH nb <= 2 UPD_CH 64 values), or the flush staging, whichever is larger
constexpr size_t UPD_WIN_BYTES = sizeof(UpdWin) + 2 * UPD_CH * 64 * sizeof(double2);
constexpr size_t UPD_SMEM_BYTES = UPD_WIN_BYTES > UpdGemm::SMEM_ELEMS * sizeof(double2)
                                      ? UPD_WIN_BYTES : UpdGemm::SMEM_ELEMS * sizeof(double2);

// One CTA per chain; the slice's sites are visited in windows of UPD_L:
//   1. the window block of the current G' = G + A B^T (A, B: the k delayed
//      columns since the last flush) is formed in shared memory;
//   2. warp 0 walks the window: lane p tests site w0 + p against its running
//      diagonal, the first passing lane (a ballot) is accepted, every lane
//      updates the phase identically and appends its row of the new window
//      columns (a = s (G'(:,f) + Aw Bw(f,:)^T), b = G'(f,:)^T + Bw Aw(f,:)^T - e_f
//      restricted to the window) -- no block barrier per accepted site;
//   3. the whole CTA extends A and B by the window's columns on all N rows;
//   4. after nublock delayed columns (and at the end of the slice) the
//      factors are flushed, G += A B^T, on the FP64 tensor pipe.
// A window also ends at the accepted site that fills the nublock columns.
//
// forced = 1: the global block move's forced flips of slice nt (sites with
// blk[i] != 0 go to the next field value, no random test, chains whose block
// did not pass the first stage do nothing); the log of the product of the
// flips' ratios is accumulated in stats[ST_BLK_LR_*].
__global__ void __launch_bounds__(UPD_NT, 2) k_update_delay(const ChainDev* __restrict__ chains, int nt, int visit, int forced,
                                                            int dir) {
    extern __shared__ double2 dsm[];
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, nb = md.nublock, lc = md.lcomp, nflr = md.nflr;
    if (forced && c.blk[N] == 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nth = blockDim.x;
    cplx* gsm = dsm;                                   // GEMM staging
    UpdWin* W = (UpdWin*)dsm;                          // window state (same memory)
    int32_t* cf = c.conf + (size_t)(nt - 1) * N;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_u[dir];
    double2* G = c.G;
    double2* A = c.A;
    double2* B = c.B;

    // walk state, kept by warp 0
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, lr_re = 0.0, lr_im = 0.0;
    if (forced && tid == 0) { lr_re = c.stats[ST_BLK_LR_RE]; lr_im = c.stats[ST_BLK_LR_IM]; }

    int k = 0, s = 0;
    while (s < N) {
        const int w0 = s, L = min(UPD_L, N - w0);
        // 1. window block of G': thread (p, g) forms rows p of the columns
        //    q = g + 8 u, so each A(w0 + p, m) is loaded once for four products
        {
            const int p = tid % UPD_L, g = tid / UPD_L;     // 8 column groups
            double2 v[UPD_L / 8];
#pragma unroll
            for (int u = 0; u < UPD_L / 8; ++u) {
                const int q = g + 8 * u;
                v[u] = (p < L && q < L) ? G[MIDX(w0 + p, w0 + q, N)] : cmk(0, 0);
            }
            if (p < L) {
#pragma unroll 4
                for (int m = 0; m < k; ++m) {
                    const double2 a = A[MIDX(w0 + p, m, N)];
#pragma unroll
                    for (int u = 0; u < UPD_L / 8; ++u) {
                        const int q = g + 8 * u;
                        if (q < L) v[u] = cfma(a, B[MIDX(w0 + q, m, N)], v[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < UPD_L / 8; ++u) {
                    const int q = g + 8 * u;
                    if (q < L) W->gW[q * UPD_LP + p] = v[u];
                }
            }
        }
        __syncthreads();
        // 2. walk (dqmc_update_delay.f90:52-60 per site)
        if (warp == 0) {
            const int p = lane, j = w0 + p;
            bool cand = false;
            double2 dl = cmk(0, 0), phr = cmk(0, 0), dW = cmk(0, 0);
            double gam = 0.0, thr = 0.0;
            int nvv = 0;
            if (p < L) {
                const int is = cf[j];
                const int iflip = forced ? 1 : (int)ceil(u32_to_stream(rw[2 * j]) * (lc - 1));
                const int kk = (is - 1) * (lc - 1) + (iflip - 1);
                dl = md.delta[kk];
                gam = md.gam_ratio[kk];
                phr = md.phase_ratio[kk];
                thr = forced ? 0.0 : u32_to_stream(rw[2 * j + 1]);
                nvv = (is + iflip - 1) % lc + 1;
                cand = !forced || c.blk[j] != 0;
                dW = W->gW[p * UPD_LP + p];
            }
            int r = 0, pc = 0, wend = L, nties = 0;
            while (pc < L) {
                bool pass = false, tie = false;
                double2 rt = cmk(0, 0), sscl = cmk(0, 0);
                if (cand && p >= pc) {
                    const double2 ratio1 = cadd(cmul(csub(cmk(1, 0), dW), dl), cmk(1, 0));
                    double2 rr = ratio1;
                    for (int f = 1; f < nflr; ++f) rr = cmul(rr, ratio1);
                    rr = cscale(rr, gam);
                    rt = cmul(rr, phr);
                    const double ra = fabs(cmul(rt, ph).x / ph.x);
                    pass = forced ? true : ra > thr;
                    tie = !forced && fabs(ra - thr) < DQ_NEAR_TIE;
                    if (pass) sscl = cdiv(dl, ratio1);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                // this iteration decides the lanes up to the first passing one
                // (all remaining lanes when none passes); later lanes are
                // tested again with the updated diagonal
                nties += tie && (bal == 0 || p <= __ffs(bal) - 1);
                if (bal == 0) break;
                const int pf = __ffs(bal) - 1;
                rt.x = __shfl_sync(0xffffffffu, rt.x, pf);
                rt.y = __shfl_sync(0xffffffffu, rt.y, pf);
                sscl.x = __shfl_sync(0xffffffffu, sscl.x, pf);
                sscl.y = __shfl_sync(0xffffffffu, sscl.y, pf);
                const double w = sqrt(cmulc(rt, rt).x);
                ph = cscale(cmul(ph, rt), 1.0 / w);
                if (lane == 0) {
                    acc += 1.0;
                    if (forced) {
                        const double2 l = clog_(rt);
                        lr_re += l.x;
                        lr_im += l.y;
                    }
                    W->sg[r] = sscl;
                    W->pm[r] = pf;
                }
                if (p == pf) { cand = false; cf[j] = nvv; }
                if (p < L) {
                    double2 a = W->gW[pf * UPD_LP + p];          // G'(p, f)
                    double2 b = W->gW[p * UPD_LP + pf];          // G'(f, p)
#pragma unroll 4
                    for (int m = 0; m < r; ++m) {
                        a = cfma(W->bW[m][pf], W->aW[m][p], a);
                        b = cfma(W->aW[m][pf], W->bW[m][p], b);
                    }
                    a = cmul(a, sscl);
                    if (p == pf) b.x -= 1.0;
                    W->aW[r][p] = a;
                    W->bW[r][p] = b;
                    dW = cfma(a, b, dW);
                }
                ++r;
                pc = pf + 1;
                __syncwarp();
                if (k + r == nb) { wend = pc; break; }
            }
            if (lane == 0) { W->r = r; W->wend = wend; }
            nties = warp_sum(nties);
            if (lane == 0 && nties) c.stats[ST_NEAR_TIE] += (double)nties;
        }
        __syncthreads();
        // 3. the window's columns on all rows: column m of this window is
        //    a = s_m (c1_m + sum_{m' < m} a_m' b_m'(f_m)), b = c2_m + sum_{m' < m} b_m' a_m'(f_m)
        //    with c1_m = G'(:,f_m), c2_m = G'(f_m,:)^T - e_f; rows of the delayed
        //    factors at the accepted sites are staged per chunk of UPD_CH columns
        const int r = W->r, wend = W->wend;
        double2* As = (double2*)(W + 1);                // [UPD_CH][nb]: A(f_m, :)
        double2* Bs = As + UPD_CH * nb;                 // [UPD_CH][nb]: B(f_m, :)
        for (int m0 = 0; m0 < r; m0 += UPD_CH) {
            const int mc = min(UPD_CH, r - m0);
            for (int e = tid; e < mc * k; e += nth) {
                const int mm = e % mc, m2 = e / mc, sm = w0 + W->pm[m0 + mm];
                As[mm * nb + m2] = A[MIDX(sm, m2, N)];
                Bs[mm * nb + m2] = B[MIDX(sm, m2, N)];
            }
            __syncthreads();
            for (int i = tid; i < N; i += nth) {
                double2 c1[UPD_CH], c2[UPD_CH];
                int pmm[UPD_CH];
#pragma unroll
                for (int mm = 0; mm < UPD_CH; ++mm) {
                    pmm[mm] = W->pm[m0 + min(mm, mc - 1)];
                    c1[mm] = G[MIDX(i, w0 + pmm[mm], N)];
                    c2[mm] = G[MIDX(w0 + pmm[mm], i, N)];
                }
                // delayed columns since the last flush: G' = G + A B^T
#pragma unroll 4
                for (int m2 = 0; m2 < k; ++m2) {
                    const double2 ai = A[MIDX(i, m2, N)], bi = B[MIDX(i, m2, N)];
#pragma unroll
                    for (int mm = 0; mm < UPD_CH; ++mm) {
                        c1[mm] = cfma(ai, Bs[mm * nb + m2], c1[mm]);
                        c2[mm] = cfma(As[mm * nb + m2], bi, c2[mm]);
                    }
                }
                // this window's earlier chunks
#pragma unroll 2
                for (int m1 = 0; m1 < m0; ++m1) {
                    const double2 a1 = A[MIDX(i, k + m1, N)], b1 = B[MIDX(i, k + m1, N)];
#pragma unroll
                    for (int mm = 0; mm < UPD_CH; ++mm) {
                        c1[mm] = cfma(W->bW[m1][pmm[mm]], a1, c1[mm]);
                        c2[mm] = cfma(W->aW[m1][pmm[mm]], b1, c2[mm]);
                    }
                }
                // this chunk, in order
#pragma unroll
                for (int mm = 0; mm < UPD_CH; ++mm) {
                    if (mm >= mc) break;
#pragma unroll
                    for (int m1 = 0; m1 < mm; ++m1) {
                        c1[mm] = cfma(W->bW[m0 + m1][pmm[mm]], c1[m1], c1[mm]);
                        c2[mm] = cfma(W->aW[m0 + m1][pmm[mm]], c2[m1], c2[mm]);
                    }
                    c1[mm] = cmul(c1[mm], W->sg[m0 + mm]);
                    if (i == w0 + pmm[mm]) c2[mm].x -= 1.0;
                    A[MIDX(i, k + m0 + mm, N)] = c1[mm];
                    B[MIDX(i, k + m0 + mm, N)] = c2[mm];
                }
            }
            __syncthreads();
        }
        k += r;
        s = w0 + wend;
        __syncthreads();
        if (k == nb || (s >= N && k > 0)) {
            flush_addto(G, A, B, N, k, gsm);
            k = 0;
        }
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        if (forced) {
            c.stats[ST_BLK_LR_RE] = lr_re;
            c.stats[ST_BLK_LR_IM] = lr_im;
        } else {
            c.stats[ST_ACC] += acc;
            c.stats[ST_PROP] += N;
        }
    }
}

// The flush alone, G += A B^T over the model's nublock delayed columns, one
// CTA per chain with the staging of k_update_delay: the delayed-update GEMM's
// own rate (dqmc_gpu_time_op 6).  Modifies G.
__global__ void __launch_bounds__(UPD_NT, 2) k_update_flush(const ChainDev* __restrict__ chains) {
    extern __shared__ double2 dsm[];
    const ChainDev& c = chains[blockIdx.x];
    flush_addto(c.G, c.A, c.B, c.N, c.md->nublock, dsm);
}

// The t-V bond field's updates of one family nf at slice nt, delayed
// (src/dqmc_config_v/dqmc_update_delay.f90:30-112): one CTA per chain, the
// bonds in nnlf_list order.  The accepted rank-2 changes are carried as
// columns of (A, B), G' = G + A B^T: bond b's 2 x 2 block of G' is
// G(P,P) + A(P,:) B(P,:)^T (warp 0, lanes over the delayed columns), the ratio
// det(I + (1 - G')(P,P) Delta) and S = Delta (I + ...)^-1 are thread 0's, and an
// accepted bond appends the columns a_q = sum_p G'(:,P_p) S(p,q) and
// b_q = G'(P_q,:)^T - e_(P_q) (whole CTA).  After nublock columns (rounded down
// to even) and at the family's end the factors are flushed, G += A B^T, on the
// FP64 tensor pipe.  Iflip is 1 for the two-valued field; bond k uses the
// words 2k (iflip) and 2k + 1 (accept test) of the family's draws (0b layout:
// families ascending after the plaquette words; b0: descending after the U
// field's).
__global__ void __launch_bounds__(UPD_NT, 2) k_vbond_delay(const ChainDev* __restrict__ chains, int nt, int nf, int visit,
                                                           int dir) {
    extern __shared__ double2 dsm[];                  // flush staging
    __shared__ double2 s_ap[2][64], s_bp[2][64];      // A(P_q, m), B(P_q, m) of the current bond
    __shared__ double2 s_mat[4];
    __shared__ int s_pc[2], s_acc;
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    if (!md.lwrapv || !c.vconf) return;
    const int N = c.N, lf = md.nn_lf, nnf = md.nn_nf, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nbv = min(md.nublock, 64) & ~1;         // delayed columns per flush (even)
    double2 *G = c.G, *A = c.A, *B = c.B;
    int32_t* cf = c.vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    const int* rows = md.vrows + (size_t)(nf - 1) * 2 * lf;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_v[dir] + (size_t)(dir ? nnf - nf : nf - 1) * 2 * lf;
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, nties = 0.0;
    int k = 0;
    for (int b = 0; b < lf; ++b) {
        // every thread is done with the previous bond's shared values
        __syncthreads();
        const int i1 = rows[2 * b], i2 = rows[2 * b + 1];
        if (warp == 0) {
            // the bond's rows of the delayed factors, and G'(P,P)
            double2 g[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};   // (0,0) (1,0) (0,1) (1,1)
            for (int m = lane; m < k; m += 32) {
                const double2 a0 = A[MIDX(i1, m, N)], a1 = A[MIDX(i2, m, N)];
                const double2 b0 = B[MIDX(i1, m, N)], b1 = B[MIDX(i2, m, N)];
                s_ap[0][m] = a0; s_ap[1][m] = a1; s_bp[0][m] = b0; s_bp[1][m] = b1;
                g[0] = cfma(a0, b0, g[0]); g[1] = cfma(a1, b0, g[1]);
                g[2] = cfma(a0, b1, g[2]); g[3] = cfma(a1, b1, g[3]);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                g[e].x = warp_sum(g[e].x);
                g[e].y = warp_sum(g[e].y);
            }
            if (lane == 0) {
                s_pc[0] = i1; s_pc[1] = i2;
                const double2 g11 = cadd(G[MIDX(i1, i1, N)], g[0]), g21 = cadd(G[MIDX(i2, i1, N)], g[1]);
                const double2 g12 = cadd(G[MIDX(i1, i2, N)], g[2]), g22 = cadd(G[MIDX(i2, i2, N)], g[3]);
                const int is = cf[b];
                const double2 d0 = md.vdp[is - 1], d1 = md.vdm[is - 1];
                const double2 v00 = cadd(cmk(1, 0), cmul(cmk(1.0 - g11.x, -g11.y), d0));
                const double2 v10 = cmul(cmk(-g21.x, -g21.y), d0);
                const double2 v01 = cmul(cmk(-g12.x, -g12.y), d1);
                const double2 v11 = cadd(cmk(1, 0), cmul(cmk(1.0 - g22.x, -g22.y), d1));
                const double2 det = csub(cmul(v00, v11), cmul(v01, v10));
                const double2 id = cdiv(cmk(1, 0), det);
                s_mat[0] = cmul(d0, cmul(v11, id));              // S = Delta vukmat^-1, column-major
                s_mat[1] = cmul(d1, cmul(cmk(-v10.x, -v10.y), id));
                s_mat[2] = cmul(d0, cmul(cmk(-v01.x, -v01.y), id));
                s_mat[3] = cmul(d1, cmul(v00, id));
                const double ra = fabs(cmul(det, ph).x / ph.x), r = u32_to_stream(rw[2 * b + 1]);
                if (fabs(ra - r) < DQ_NEAR_TIE) nties += 1.0;
                s_acc = ra > r;
                if (s_acc) {
                    acc += 1.0;
                    ph = cscale(cmul(ph, det), 1.0 / sqrt(cmulc(det, det).x));
                    cf[b] = is % 2 + 1;
                }
            }
        }
        __syncthreads();
        if (s_acc) {
            const int p0 = s_pc[0], p1 = s_pc[1];
            const double2 S00 = s_mat[0], S10 = s_mat[1], S01 = s_mat[2], S11 = s_mat[3];
            for (int i = tid; i < N; i += blockDim.x) {
                double2 c0 = G[MIDX(i, p0, N)], c1 = G[MIDX(i, p1, N)];      // G'(i, P)
                double2 r0 = G[MIDX(p0, i, N)], r1 = G[MIDX(p1, i, N)];      // G'(P, i)
                for (int m = 0; m < k; ++m) {
                    const double2 ai = A[MIDX(i, m, N)], bi = B[MIDX(i, m, N)];
                    c0 = cfma(ai, s_bp[0][m], c0); c1 = cfma(ai, s_bp[1][m], c1);
                    r0 = cfma(s_ap[0][m], bi, r0); r1 = cfma(s_ap[1][m], bi, r1);
                }
                if (i == p0) r0.x -= 1.0;
                if (i == p1) r1.x -= 1.0;
                A[MIDX(i, k, N)] = cadd(cmul(c0, S00), cmul(c1, S10));
                A[MIDX(i, k + 1, N)] = cadd(cmul(c0, S01), cmul(c1, S11));
                B[MIDX(i, k, N)] = r0;
                B[MIDX(i, k + 1, N)] = r1;
            }
            k += 2;
            __syncthreads();
        }
        if (k > 0 && (k + 2 > nbv || b == lf - 1)) {
            flush_addto(G, A, B, N, k, dsm);
            k = 0;
        }
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        c.stats[ST_ACCV] += acc;
        c.stats[ST_PROPV] += lf;
        c.stats[ST_NEAR_TIE] += nties;
    }
}

static int g_vbd_attr = 0;

// the delayed bond updates when the flush depth allows two columns, else the
// rank-2 updates straight on G (kern_plqu.cu)
int launch_vbond_delay(const ChainDev* chains, int nchains, int nublock, int nt, int nf, int visit, int dir,
                       cudaStream_t st) {
    if ((min(nublock, 64) & ~1) < 2) return 0;
    const size_t smem = UpdGemm::SMEM_ELEMS * sizeof(double2);
    if (!g_vbd_attr) {
        cudaFuncSetAttribute(k_vbond_delay, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_vbd_attr = 1;
    }
    k_vbond_delay<<<nchains, UPD_NT, smem, st>>>(chains, nt, nf, visit, dir);
    return 1;
}

static int g_upd_attr = 0;

void launch_update(const ChainDev* chains, int nchains, int nt, int visit, cudaStream_t st, int forced, int dir) {
    size_t smem = UPD_SMEM_BYTES;
    if (!g_upd_attr) {
        cudaFuncSetAttribute(k_update_delay, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_upd_attr = 1;
    }
    k_update_delay<<<nchains, UPD_NT, smem, st>>>(chains, nt, visit, forced, dir);
}

static int g_flush_attr = 0;

void launch_update_flush(const ChainDev* chains, int nchains, cudaStream_t st) {
    size_t smem = UpdGemm::SMEM_ELEMS * sizeof(double2);
    if (!g_flush_attr) {
        cudaFuncSetAttribute(k_update_flush, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_flush_attr = 1;
    }
    k_update_flush<<<nchains, UPD_NT, smem, st>>>(chains);
}
