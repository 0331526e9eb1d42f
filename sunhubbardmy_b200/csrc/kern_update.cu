// Local Hubbard-Stratonovich updates of one time slice, one CTA per chain.
//
// Reference: src/dqmc_config_u/dqmc_update_delay.f90:1-137 (delayed update),
// dqmc_update.f90 (fast update) and dqmc_update_submatrix.f90 (submatrix
// update).  All three visit the sites in order with two SFMT draws per site
// and accept with |Re(R phase)/Re(phase)| > r; they differ only in how the
// accepted rank-1 changes are folded into G.  This kernel runs all of them as
// a delayed update:
//   * every round, all threads evaluate the acceptance test of every
//     remaining site with the current diagonal and phase; the first accepted
//     site is found with a block reduction, so rejected sites cost one
//     parallel pass instead of a sequential step each;
//   * an accepted site s appends a_k = s_k (G(:,s) + A B(s,:)^T) and
//     b_k = G(s,:)^T + B A(s,:)^T - e_s to the N x k factors (A, B) and
//     updates the running diagonal;
//   * after nublock accepted sites (and at the end of the slice) the factors
//     are flushed, G += A B^T, as one DMMA tensor-core GEMM.
// The accept/reject sequence equals the reference's in exact arithmetic.
#include "chain_access.cuh"
#include "kernels.h"
#include "zgemm.cuh"

typedef GemmBig UpdGemm;

struct UpdSmem {
    double red[64];
    int redi[32];
    int first;
    double2 phase;
    double2 sscl;
    double acc;
};

DQ_DEV int block_min_int(int v, int* red) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    int t = (lane < nw) ? red[lane] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = min(t, __shfl_xor_sync(0xffffffffu, t, o));
    return t;
}

DQ_DEV double u32_to_stream(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

// total ratio of flipping site s (dqmc_update_delay.f90:52-60)
DQ_DEV double2 flip_ratio(const ModelDev& md, double2 diag_s, int is, int iflip, double2* sscl_out) {
    int lc = md.lcomp;
    int k = (is - 1) * (lc - 1) + (iflip - 1);
    double2 dlt = md.delta[k];
    double2 ratio1 = cadd(cmul(csub(cmk(1, 0), diag_s), dlt), cmk(1, 0));
    if (sscl_out) *sscl_out = cdiv(dlt, ratio1);
    double2 r = ratio1;
    for (int f = 1; f < md.nflr; ++f) r = cmul(r, ratio1);
    r = cscale(r, md.gam_ratio[k]);
    return cmul(r, md.phase_ratio[k]);
}

// forced = 1: the global block move's forced flips of slice nt (sites with
// blk[i] != 0 go to the next field value, no random test, chains whose block
// did not pass the first stage do nothing); the log of the product of the
// flips' ratios is accumulated in stats[ST_BLK_LR_*].
__global__ void __launch_bounds__(256) k_update_delay(const ChainDev* __restrict__ chains, int nt, int visit, int forced) {
    extern __shared__ double2 dsm[];
    const ChainDev c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, nb = md.nublock, lc = md.lcomp;
    if (forced && c.blk[N] == 0) return;
    const int tid = threadIdx.x, nth = blockDim.x;
    cplx* gsm = dsm;                                   // GEMM staging
    double2* diag = dsm + UpdGemm::SMEM_ELEMS;         // N
    double2* arow = diag + N;                          // nb
    double2* brow = arow + nb;                         // nb
    UpdSmem* S = (UpdSmem*)(brow + nb);
    int32_t* cf = c.conf + (size_t)(nt - 1) * N;
    const uint32_t* rw = c.rnd + (size_t)visit * 2 * N;
    double2* G = c.G;

    for (int i = tid; i < N; i += nth) diag[i] = G[MIDX(i, i, N)];
    if (tid == 0) {
        S->phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
        S->acc = 0.0;
    }
    __syncthreads();

    int ik = 0, s = 0;
    while (s < N) {
        // parallel acceptance test of all remaining sites
        const double2 ph = S->phase;
        int myfirst = N;
        for (int j = s + tid; j < N; j += nth) {
            if (forced) {
                if (c.blk[j]) { myfirst = j; break; }
                continue;
            }
            int is = cf[j];
            int iflip = (int)ceil(u32_to_stream(rw[2 * j]) * (lc - 1));
            double2 rt = flip_ratio(md, diag[j], is, iflip, nullptr);
            double rre = cmul(rt, ph).x / ph.x;
            double rabs = fabs(rre);
            if (rabs > u32_to_stream(rw[2 * j + 1])) { myfirst = j; break; }
        }
        int first = block_min_int(myfirst, S->redi);
        if (first >= N) break;
        // accept site `first`
        if (tid == 0) {
            int is = cf[first];
            int iflip = forced ? 1 : (int)ceil(u32_to_stream(rw[2 * first]) * (lc - 1));
            int isp = (is + iflip - 1) % lc + 1;
            double2 sscl;
            double2 rt = flip_ratio(md, diag[first], is, iflip, &sscl);
            double w = sqrt(cmulc(rt, rt).x);
            S->phase = cscale(cmul(S->phase, rt), 1.0 / w);
            S->sscl = sscl;
            S->acc += 1.0;
            if (forced) {
                double2 l = clog_(rt);
                c.stats[ST_BLK_LR_RE] += l.x;
                c.stats[ST_BLK_LR_IM] += l.y;
            }
            cf[first] = isp;
        }
        for (int m = tid; m < ik; m += nth) {
            arow[m] = c.A[MIDX(first, m, N)];
            brow[m] = c.B[MIDX(first, m, N)];
        }
        __syncthreads();
        const double2 sscl = S->sscl;
        for (int i = tid; i < N; i += nth) {
            double2 a = G[MIDX(i, first, N)];
            double2 b = G[MIDX(first, i, N)];
            for (int m = 0; m < ik; ++m) {
                a = cfma(brow[m], c.A[MIDX(i, m, N)], a);
                b = cfma(arow[m], c.B[MIDX(i, m, N)], b);
            }
            a = cmul(a, sscl);
            if (i == first) b.x -= 1.0;
            c.A[MIDX(i, ik, N)] = a;
            c.B[MIDX(i, ik, N)] = b;
            diag[i] = cfma(a, b, diag[i]);
        }
        ++ik;
        s = first + 1;
        __syncthreads();
        if (ik == nb && s < N) {
            ZGemmArgs g;
            g.M = N; g.N = N; g.K = ik; g.alpha = cmk(1, 0); g.beta = cmk(1, 0);
            g.A = c.A; g.lda = N; g.opA = OP_N; g.B = c.B; g.ldb = N; g.opB = OP_T; g.C = G; g.ldc = N;
            zgemm_cta<UpdGemm>(g, 0, 1, gsm);
            for (int i = tid; i < N; i += nth) diag[i] = G[MIDX(i, i, N)];
            ik = 0;
            __syncthreads();
        }
    }
    if (ik > 0) {
        ZGemmArgs g;
        g.M = N; g.N = N; g.K = ik; g.alpha = cmk(1, 0); g.beta = cmk(1, 0);
        g.A = c.A; g.lda = N; g.opA = OP_N; g.B = c.B; g.ldb = N; g.opB = OP_T; g.C = G; g.ldc = N;
        zgemm_cta<UpdGemm>(g, 0, 1, gsm);
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = S->phase.x;
        c.stats[ST_PHASE_IM] = S->phase.y;
        if (!forced) {
            c.stats[ST_ACC] += S->acc;
            c.stats[ST_PROP] += N;
        }
    }
}

static int g_upd_attr = 0;

void launch_update(const ChainDev* chains, int nchains, int nt, int visit, cudaStream_t st, int forced) {
    size_t smem = UpdGemm::SMEM_ELEMS * sizeof(double2) + (size_t)(512 + 2 * 64) * sizeof(double2) + sizeof(UpdSmem) + 64;
    if (!g_upd_attr) {
        cudaFuncSetAttribute(k_update_delay, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_upd_attr = 1;
    }
    k_update_delay<<<nchains, 256, smem, st>>>(chains, nt, visit, forced);
}
