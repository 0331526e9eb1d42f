// UDV stabilisation and the equal-time Green's function, one CTA per chain.
//
// Reference: src/dqmc_ft_core/dqmc_ft_stablize_0b_qr.f90 / _b0_qr.f90 (1-61),
// green_equaltime.f90 (1-107), green_equaltimebb.f90 (1-84), set_phase.f90,
// and the s_matrix helpers they call (s_z_x_diag_d, s_zmcpt, s_zgeQR_logdetQ,
// s_invdiag_d_x_zr, s_zpm, s_dvec_min_max, s_compare_max_z).
//
// Differences in method, not in result:
//  * the columns are always pre-sorted by norm (s_zmcpt) and factored without
//    pivoting; the reference uses zgeqp3 for its first/last step, where the
//    previous D is 1 and V is the identity, so the same code path applies;
//  * the inverse of the scaled middle matrix M is taken through its QR
//    factors (G = U_L dlmax^-1 R^-1 Q^H drmax^-1 U_R^H, log det M = log det Q +
//    sum log R_ii) instead of an LU factorisation and explicit inverse.
#include "chain_access.cuh"
#include "kernels.h"
#include "linalg.cuh"

struct StabSmem {
    LinalgSmem L;
    double red[64];
};

DQ_DEV LinalgScratch make_scratch(const ChainDev& c) {
    LinalgScratch s;
    s.Vs = c.W[5];
    s.Ws = c.smallw;
    s.Ws2 = c.smallw + (size_t)QR_NB2 * c.N;
    s.T = c.T;
    s.tau = c.tau;
    s.T64 = c.T64;
    return s;
}

static size_t stab_smem_bytes(int maxN) {
    size_t a = QR_PANEL_ELEMS(maxN);
    size_t b = GemmBig::SMEM_ELEMS;
    if ((size_t)GemmWide::SMEM_ELEMS > b) b = GemmWide::SMEM_ELEMS;
    return (a > b ? a : b) * sizeof(double2) + sizeof(StabSmem) + 64;
}

// one UDV step: W0 holds B(slices) * U[src]; writes U/D/V/logdetQ of slot dst.
__global__ void __launch_bounds__(256, 2) k_stab(const ChainDev* __restrict__ chains, int src, int dst) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.x];
    const int N = c.N, tid = threadIdx.x, nth = blockDim.x;
    const size_t NN = (size_t)N * N;
    double2* buf = ssm;
    StabSmem* S = (StabSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = make_scratch(c);
    double2* W0 = c.W[0];
    double2* W2 = c.W[1];
    double2* W3 = c.W[2];
    double2* W4 = c.W[3];
    src = c.slotmap[src];
    dst = c.slotmap[dst];
    const double* Dsrc = c.D + (size_t)src * N;
    double* Ddst = c.D + (size_t)dst * N;
    double* nrm = c.vecs;
    int* perm = c.perm;

    // column norms of B U D (s_z_x_diag_d + s_zmcpt)
    const int lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
    for (int j = warp; j < N; j += nw) {
        double s = 0.0;
        for (int r = lane; r < N; r += 32) s += cabs2(W0[MIDX(r, j, N)]);
        s = warp_sum(s);
        if (lane == 0) nrm[j] = sqrt(s) * fabs(Dsrc[j]);
    }
    __syncthreads();
    // descending stable rank sort
    for (int j = tid; j < N; j += nth) {
        double v = nrm[j];
        int rank = 0;
        for (int k = 0; k < N; ++k) {
            double w = nrm[k];
            rank += (w > v) || (w == v && k < j);
        }
        perm[rank] = j;
    }
    __syncthreads();
    for (size_t e = tid; e < NN; e += nth) {
        int r = (int)(e % N), k = (int)(e / N);
        int j = perm[k];
        W2[e] = cscale(W0[MIDX(r, j, N)], Dsrc[j]);
    }
    __syncthreads();
    cta_qr64(W2, N, sc, buf, buf, &S->L);
    int bad = 0;
    for (int i = tid; i < N; i += nth) {
        const double d = W2[MIDX(i, i, N)].x;
        Ddst[i] = d;
        bad |= (d == 0.0 || !isfinite(d));
    }
    // a zero or non-finite R_ii (the zgeqp3 / zgeqrf step of the reference)
    if (__syncthreads_or(bad) && tid == 0) chain_raise(c, DQ_FAIL_SINGULAR);
    double2 ldq = cta_logdet_q(sc.tau, N, S->red);
    if (tid == 0) c.logdetQ[dst] = ldq;
    __syncthreads();
    // Vt = D^-1 R
    for (size_t e = tid; e < NN; e += nth) {
        int r = (int)(e % N), k = (int)(e / N);
        W3[e] = (r <= k) ? cscale(W2[e], 1.0 / Ddst[r]) : cmk(0, 0);
    }
    // P^T V_src: row k <- row perm[k]
    const double2* Vsrc = c.V + (size_t)src * NN;
    for (size_t e = tid; e < NN; e += nth) {
        int r = (int)(e % N), k = (int)(e / N);
        W4[e] = Vsrc[MIDX(perm[r], k, N)];
    }
    __syncthreads();
    cta_form_q64(W2, N, c.U + (size_t)dst * NN, sc, buf);
    ZGemmArgs g;
    g.M = N; g.N = N; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = W3; g.lda = N; g.opA = OP_N; g.B = W4; g.ldb = N; g.opB = OP_N;
    g.C = c.V + (size_t)dst * NN; g.ldc = N;
    g.triA = 1;                          // D^-1 R is upper triangular
    zgemm_cta<GemmBig>(g, 0, 1, buf);
}

// s_dvec_min_max
DQ_DEV void dminmax(double d, double& dmax, double& dmin) {
    if (fabs(d) > 1.0) { dmax = fabs(d); dmin = copysign(1.0, d); }
    else { dmax = 1.0; dmin = d; }
}

// Green's function into Gnew.  mode 0: green_equaltime(R = slot nr, L = slot nl);
// mode 1: green_equaltimebb (R = slot nr).  New log weight -> stats[ST_LOGDETM_*].
__global__ void __launch_bounds__(256, 2) k_green(const ChainDev* __restrict__ chains, int nr, int nl, int mode) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.x];
    const int N = c.N, tid = threadIdx.x, nth = blockDim.x;
    const size_t NN = (size_t)N * N;
    double2* buf = ssm;
    StabSmem* S = (StabSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = make_scratch(c);
    nr = c.slotmap[nr];
    if (mode == 0) nl = c.slotmap[nl];
    const double2* UR = c.U + (size_t)nr * NN;
    const double2* VR = c.V + (size_t)nr * NN;
    const double* DR = c.D + (size_t)nr * N;
    double* drmax = c.vecs + 0 * N;
    double* drmin = c.vecs + 1 * N;
    double* dlmax = c.vecs + 2 * N;
    double* dlmin = c.vecs + 3 * N;
    double2* M = c.W[0];
    double2* Z = c.W[1];
    double slog = 0.0;
    for (int i = tid; i < N; i += nth) {
        double a, b;
        dminmax(DR[i], a, b);
        drmax[i] = a; drmin[i] = b;
        slog += log(a);
    }
    if (mode == 0) {
        const double2* UL = c.U + (size_t)nl * NN;
        const double2* VL = c.V + (size_t)nl * NN;
        const double* DL = c.D + (size_t)nl * N;
        for (int i = tid; i < N; i += nth) {
            double a, b;
            dminmax(DL[i], a, b);
            dlmax[i] = a; dlmin[i] = b;
            slog += log(a);
        }
        __syncthreads();   // dmax/dmin are read by other threads below
        ZGemmArgs g;
        g.M = N; g.N = N; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
        g.A = UR; g.lda = N; g.opA = OP_C; g.B = UL; g.ldb = N; g.opB = OP_N; g.C = M; g.ldc = N;
        zgemm_cta<GemmBig>(g, 0, 1, buf);
        g.A = VR; g.opA = OP_N; g.B = VL; g.opB = OP_C; g.C = Z;
        zgemm_cta<GemmBig>(g, 0, 1, buf);
        for (size_t e = tid; e < NN; e += nth) {
            int i = (int)(e % N), j = (int)(e / N);
            double2 u = cscale(M[e], 1.0 / (drmax[i] * dlmax[j]));
            M[e] = cadd(u, cscale(Z[e], drmin[i] * dlmin[j]));
        }
    } else {
        __syncthreads();   // drmax/drmin are read by other threads below
        for (size_t e = tid; e < NN; e += nth) {
            int i = (int)(e % N), j = (int)(e / N);
            M[e] = cadd(cscale(cconj(UR[MIDX(j, i, N)]), 1.0 / drmax[i]), cscale(VR[e], drmin[i]));
        }
    }
    slog = block_sum(slog, S->red);
    __syncthreads();
    cta_qr64(M, N, sc, buf, buf, &S->L);
    double2 ldm = cta_logdet_q(sc.tau, N, S->red);
    double2 lr = cmk(0, 0);
    int bad = 0;
    for (int i = tid; i < N; i += nth) {
        double r = M[MIDX(i, i, N)].x;
        bad |= (r == 0.0 || !isfinite(r));
        lr = cadd(lr, cmk(log(fabs(r)), r < 0.0 ? M_PI : 0.0));
    }
    // a zero or non-finite pivot of M: zgetrf's info > 0 in s_inv_logdet_lu_z
    bad = __syncthreads_or(bad);
    lr = block_csum(lr, S->red);
    ldm = cadd(ldm, lr);
    double2* X = (mode == 0) ? Z : c.Gnew;
    for (size_t e = tid; e < NN; e += nth) {
        int i = (int)(e % N), j = (int)(e / N);
        X[e] = cscale(cconj(UR[MIDX(j, i, N)]), 1.0 / drmax[i]);
    }
    __syncthreads();
    cta_apply_qh64(M, N, X, sc, buf);
    cta_trsm_upper64(M, N, X, buf, &S->L);
    if (mode == 0) {
        const double2* UL = c.U + (size_t)nl * NN;
        double2* UL2 = c.W[2];
        for (size_t e = tid; e < NN; e += nth) {
            int j = (int)(e / N);
            UL2[e] = cscale(UL[e], 1.0 / dlmax[j]);
        }
        __syncthreads();
        ZGemmArgs g;
        g.M = N; g.N = N; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
        g.A = UL2; g.lda = N; g.opA = OP_N; g.B = Z; g.ldb = N; g.opB = OP_N; g.C = c.Gnew; g.ldc = N;
        zgemm_cta<GemmBig>(g, 0, 1, buf);
    }
    if (tid == 0) {
        double2 lw = cadd(ldm, cmk(slog, 0.0));
        lw = cadd(lw, c.logdetQ[nr]);
        if (mode == 0) lw = csub(lw, c.logdetQ[nl]);
        c.stats[ST_LOGDETM_RE] = lw.x;
        c.stats[ST_LOGDETM_IM] = lw.y;
        c.stats[ST_GINFO] = (bad || !isfinite(lw.x) || !isfinite(lw.y)) ? (double)DQ_FAIL_SINGULAR : 0.0;
    }
}

// green_tau (src/dqmc_ft_core/green_tau.f90:1-136) at a stabilisation point of
// the unequal-time pass: from the right factors (slot nr: UR DR VR = B(tau,0))
// and the left ones (slot nl: UL DL VL), with d = dmax dmin split as in
// green_equaltime,
//   G(tau,tau) = UL dlmax^-1 M^-1 drmax^-1 UR^H          -> Gnew
//   G(tau,0)   = UL dlmax^-1 M^-1 drmin VR                -> gt0
//   G(0,0)     = VR^-1 drmax^-1 M2^-1 dlmax^-1 (VL^H)^-1  -> g00
//   G(0,tau)   = -VR^-1 drmax^-1 M2^-1 dlmin UL^H         -> g0t
// with M = drmax^-1 UR^H UL dlmax^-1 + drmin VR VL^H dlmin and
// M2 = dlmax^-1 (VR VL^H)^-1 drmax^-1 + dlmin UL^H UR drmin.  Inverses are
// taken through QR factors (solves with Q^H and R), as in k_green, instead of
// LU; log det M (the new log weight) as in k_green.  Scratch W0..W4 (W5 holds
// the reflector blocks of the QR).
__global__ void __launch_bounds__(256, 2) k_green_tau(const ChainDev* __restrict__ chains, int nr, int nl) {
    extern __shared__ double2 ssm[];
    const ChainDev& c = chains[blockIdx.x];
    const int N = c.N, tid = threadIdx.x, nth = blockDim.x;
    const size_t NN = (size_t)N * N;
    double2* buf = ssm;
    StabSmem* S = (StabSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = make_scratch(c);
    nr = c.slotmap[nr];
    nl = c.slotmap[nl];
    const double2* UR = c.U + (size_t)nr * NN;
    const double2* VR = c.V + (size_t)nr * NN;
    const double* DR = c.D + (size_t)nr * N;
    const double2* UL = c.U + (size_t)nl * NN;
    const double2* VL = c.V + (size_t)nl * NN;
    const double* DL = c.D + (size_t)nl * N;
    double* drmax = c.vecs + 0 * N;
    double* drmin = c.vecs + 1 * N;
    double* dlmax = c.vecs + 2 * N;
    double* dlmin = c.vecs + 3 * N;
    double2 *W0 = c.W[0], *W1 = c.W[1], *W2 = c.W[2], *W3 = c.W[3], *W4 = c.W[4];
    double slog = 0.0;
    for (int i = tid; i < N; i += nth) {
        double a, b;
        dminmax(DR[i], a, b);
        drmax[i] = a; drmin[i] = b;
        slog += log(a);
        dminmax(DL[i], a, b);
        dlmax[i] = a; dlmin[i] = b;
        slog += log(a);
    }
    __syncthreads();
    ZGemmArgs g;
    g.M = N; g.N = N; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0); g.lda = N; g.ldb = N; g.ldc = N;
    auto gemm = [&](const double2* A, int opA, const double2* B, int opB, double2* C, double alpha) {
        g.A = A; g.opA = opA; g.B = B; g.opB = opB; g.C = C; g.alpha = cmk(alpha, 0);
        zgemm_cta<GemmBig>(g, 0, 1, buf);
    };
    // uu = UR^H UL (W1, kept for M2), vv = VR VL^H (W2)
    gemm(UR, OP_C, UL, OP_N, W1, 1.0);
    gemm(VR, OP_N, VL, OP_C, W2, 1.0);
    for (size_t e = tid; e < NN; e += nth) {
        const int i = (int)(e % N), j = (int)(e / N);
        W0[e] = cadd(cscale(W1[e], 1.0 / (drmax[i] * dlmax[j])), cscale(W2[e], drmin[i] * dlmin[j]));
    }
    slog = block_sum(slog, S->red);
    __syncthreads();
    cta_qr64(W0, N, sc, buf, buf, &S->L);
    double2 ldm = cta_logdet_q(sc.tau, N, S->red);
    double2 lr = cmk(0, 0);
    int bad = 0;
    for (int i = tid; i < N; i += nth) {
        const double r = W0[MIDX(i, i, N)].x;
        bad |= (r == 0.0 || !isfinite(r));
        lr = cadd(lr, cmk(log(fabs(r)), r < 0.0 ? M_PI : 0.0));
    }
    bad = __syncthreads_or(bad);
    lr = block_csum(lr, S->red);
    ldm = cadd(ldm, lr);
    // X = M^-1 drmax^-1 UR^H (W2), Y = M^-1 drmin VR (W3)
    for (size_t e = tid; e < NN; e += nth) {
        const int i = (int)(e % N), j = (int)(e / N);
        W2[e] = cscale(cconj(UR[MIDX(j, i, N)]), 1.0 / drmax[i]);
        W3[e] = cscale(VR[e], drmin[i]);
    }
    __syncthreads();
    cta_apply_qh64(W0, N, W2, sc, buf);
    cta_trsm_upper64(W0, N, W2, buf, &S->L);
    cta_apply_qh64(W0, N, W3, sc, buf);
    cta_trsm_upper64(W0, N, W3, buf, &S->L);
    // UL dlmax^-1 (W4); G(tau,tau) and G(tau,0)
    for (size_t e = tid; e < NN; e += nth) W4[e] = cscale(UL[e], 1.0 / dlmax[(int)(e / N)]);
    __syncthreads();
    gemm(W4, OP_N, W2, OP_N, c.Gnew, 1.0);
    gemm(W4, OP_N, W3, OP_N, c.gt0, 1.0);
    // VR^-1 (W2) and (VL^H)^-1 (W3) through QR: W0 <- A, W <- I, solve
    for (int pass = 0; pass < 2; ++pass) {
        double2* Xi = pass == 0 ? W2 : W3;
        for (size_t e = tid; e < NN; e += nth) {
            const int i = (int)(e % N), j = (int)(e / N);
            W0[e] = pass == 0 ? VR[e] : cconj(VL[MIDX(j, i, N)]);
            Xi[e] = cmk(i == j ? 1.0 : 0.0, 0.0);
        }
        __syncthreads();
        cta_qr64(W0, N, sc, buf, buf, &S->L);
        cta_apply_qh64(W0, N, Xi, sc, buf);
        cta_trsm_upper64(W0, N, Xi, buf, &S->L);
    }
    // (VR VL^H)^-1 = (VL^H)^-1 VR^-1 (W4); M2 (W0)
    gemm(W3, OP_N, W2, OP_N, W4, 1.0);
    for (size_t e = tid; e < NN; e += nth) {
        const int i = (int)(e % N), j = (int)(e / N);
        W0[e] = cadd(cscale(W4[e], 1.0 / (dlmax[i] * drmax[j])), cscale(cconj(W1[MIDX(j, i, N)]), dlmin[i] * drmin[j]));
    }
    __syncthreads();
    cta_qr64(W0, N, sc, buf, buf, &S->L);
    // Z = M2^-1 dlmax^-1 (VL^H)^-1 (W3), Wm = M2^-1 (-dlmin UL^H) (W4)
    for (size_t e = tid; e < NN; e += nth) {
        const int i = (int)(e % N), j = (int)(e / N);
        W3[e] = cscale(W3[e], 1.0 / dlmax[i]);
        W4[e] = cscale(cconj(UL[MIDX(j, i, N)]), -dlmin[i]);
    }
    __syncthreads();
    cta_apply_qh64(W0, N, W3, sc, buf);
    cta_trsm_upper64(W0, N, W3, buf, &S->L);
    cta_apply_qh64(W0, N, W4, sc, buf);
    cta_trsm_upper64(W0, N, W4, buf, &S->L);
    // VR^-1 drmax^-1 (W2); G(0,0), G(0,tau)
    for (size_t e = tid; e < NN; e += nth) W2[e] = cscale(W2[e], 1.0 / drmax[(int)(e / N)]);
    __syncthreads();
    gemm(W2, OP_N, W3, OP_N, c.g00, 1.0);
    gemm(W2, OP_N, W4, OP_N, c.g0t, 1.0);
    if (tid == 0) {
        double2 lw = cadd(ldm, cmk(slog, 0.0));
        lw = cadd(lw, c.logdetQ[nr]);
        lw = csub(lw, c.logdetQ[nl]);
        c.stats[ST_LOGDETM_RE] = lw.x;
        c.stats[ST_LOGDETM_IM] = lw.y;
        c.stats[ST_GINFO] = (bad || !isfinite(lw.x) || !isfinite(lw.y)) ? (double)DQ_FAIL_SINGULAR : 0.0;
    }
}

// push_stage / pop_stage (src/dqmc_ft_core.f90:290-312): the whole UDV stack
// and G to (dir 0) or from (dir 1) the chain's backup
__global__ void k_stage(const ChainDev* __restrict__ chains, int nslots, int dir) {
    const ChainDev& c = chains[blockIdx.y];
    const size_t NN = (size_t)c.N * c.N, nmat = (size_t)nslots * NN;
    const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double2 *u = c.U, *v = c.V, *ub = c.Ub, *vb = c.Vb, *gg = c.G, *gb = c.Gb, *lq = c.logdetQ, *lb = c.ldqb;
    double *d = c.D, *db = c.Db;
    if (dir == 0) {
        for (size_t e = t0; e < nmat; e += stride) { ub[e] = u[e]; vb[e] = v[e]; }
        for (size_t e = t0; e < NN; e += stride) gb[e] = gg[e];
        for (size_t e = t0; e < (size_t)nslots * c.N; e += stride) db[e] = d[e];
        for (size_t e = t0; e < (size_t)nslots; e += stride) lb[e] = lq[e];
    } else {
        for (size_t e = t0; e < nmat; e += stride) { u[e] = ub[e]; v[e] = vb[e]; }
        for (size_t e = t0; e < NN; e += stride) gg[e] = gb[e];
        for (size_t e = t0; e < (size_t)nslots * c.N; e += stride) d[e] = db[e];
        for (size_t e = t0; e < (size_t)nslots; e += stride) lq[e] = lb[e];
    }
}

// start of the unequal-time pass (dqmc_ft_sweep_0b.f90:39-43): g00 = gt0 = G, g0t = G - I
__global__ void k_dyn_init(const ChainDev* __restrict__ chains) {
    const ChainDev& c = chains[blockIdx.y];
    const int N = c.N;
    const size_t NN = (size_t)N * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < NN; e += (size_t)gridDim.x * blockDim.x) {
        const double2 g = c.G[e];
        c.g00[e] = g;
        c.gt0[e] = g;
        c.g0t[e] = ((int)(e % N) == (int)(e / N)) ? cmk(g.x - 1.0, g.y) : g;
    }
}

// s_compare_max_z + set_phase + replacement of G (dqmc_ft_sweep_b0.f90:145-194).
// Where the reference stops on info /= 0 (188-194), the fresh G is not taken:
// a chain whose Green's function computation hit a singular pivot, or whose
// fresh G is not finite, keeps its propagated G, phase and log weight, and the
// failure is raised (chain_raise) for the host to report.  With a wrap-error
// tolerance ctl[0] > 0, a recorded check above it (or not finite) raises
// DQ_FAIL_WRAP; the fresh G is still taken then.
__global__ void __launch_bounds__(256) k_wrap_check(const ChainDev* __restrict__ chains, int record) {
    __shared__ double red[64];
    const ChainDev c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, tid = threadIdx.x, nth = blockDim.x;
    const size_t NN = (size_t)N * N;
    double mx = 0.0;
    int nonfin = 0, wnan = 0;
    for (size_t e = tid; e < NN; e += nth) {
        const double2 gn = c.Gnew[e];
        nonfin |= !(isfinite(gn.x) && isfinite(gn.y));
        const double a = cabsd(csub(gn, c.G[e]));
        wnan |= !isfinite(a);
        mx = fmax(mx, a);
    }
    nonfin = __syncthreads_or(nonfin);
    wnan = __syncthreads_or(wnan);
    const int ginfo = (int)c.stats[ST_GINFO];
    const bool keep = nonfin || (ginfo & DQ_FAIL_SINGULAR);
    // wrap trace: the fresh G of this check (the reference's -DTEST_LEVEL3
    // print of gf_tmp, dqmc_ft_sweep_b0.f90:160-179)
    const int tslot = (record && c.trace_g) ? *c.trace_n : c.trace_cap;
    if (tslot < c.trace_cap)
        for (size_t e = tid; e < NN; e += nth) c.trace_g[(size_t)tslot * NN + e] = c.Gnew[e];
    if (!keep)
        for (size_t e = tid; e < NN; e += nth) c.G[e] = c.Gnew[e];
    mx = block_max(mx, red);
    double ang = 0.0;
    if (md.plq) {            // set_phase.f90:9-15: the plaquette field's phases
        const size_t nconf = (size_t)md.ltrot * md.lq;
        for (size_t e = tid; e < nconf; e += nth) ang += md.plq_phase_angle[c.conf_plq[e] - 1];
    }
    if (md.phase_on) {
        const size_t nconf = (size_t)md.ltrot * N;
        for (size_t e = tid; e < nconf; e += nth) ang += md.phase_angle[c.conf[e] - 1];
    }
    ang = block_sum(ang, red);
    if (tid == 0) {
        double2 lw = cmk(c.stats[ST_LOGDETM_RE], c.stats[ST_LOGDETM_IM]);
        double2 ph = cexpi(md.nflr * lw.y + ang);
        int code = (ginfo & DQ_FAIL_SINGULAR) | (nonfin ? DQ_FAIL_NONFINITE : 0);
        const double tol = c.ctl ? c.ctl[0] : 0.0;
        if (record && tol > 0.0 && (wnan || mx > tol)) code |= DQ_FAIL_WRAP;
        if (code) chain_raise(c, code);
        if (tslot < c.trace_cap) { c.trace_err[tslot] = mx; *c.trace_n = tslot + 1; }
        if (record) {
            double2 old = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
            double pd = cabsd(csub(old, ph));
            c.stats[ST_MAX_WRAP] = fmax(c.stats[ST_MAX_WRAP], mx);
            c.stats[ST_MAX_PHASEDIFF] = fmax(c.stats[ST_MAX_PHASEDIFF], pd);
            c.stats[ST_LOGCOUNT] += 1.0;
            c.stats[ST_AVGLOG10] += log10(mx);
            c.stats[ST_AVGEXPPD] += exp(pd);
            c.stats[ST_LAST_WRAP] = mx;
        }
        if (!keep) {
            c.stats[ST_PHASE_RE] = ph.x;
            c.stats[ST_PHASE_IM] = ph.y;
            c.stats[ST_LOGW_RE] = lw.x;
            c.stats[ST_LOGW_IM] = lw.y;
        }
    }
}

__global__ void k_copy_mat(const ChainDev* __restrict__ chains, int dst_id, int src_id, int identity) {
    const ChainDev c = chains[blockIdx.y];
    const size_t NN = (size_t)c.N * c.N;
    double2* d = chain_mat(c, dst_id);
    const double2* s = identity ? nullptr : chain_mat(c, src_id);
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < NN; e += (size_t)gridDim.x * blockDim.x) {
        if (identity) d[e] = cmk((e % c.N) == (e / c.N) ? 1.0 : 0.0, 0.0);
        else d[e] = s[e];
    }
}

// identity stack entry: U = V = I, D = 1, logdetQ = 0
__global__ void k_stack_identity(const ChainDev* __restrict__ chains, int slot) {
    const ChainDev c = chains[blockIdx.y];
    slot = c.slotmap[slot];
    const int N = c.N;
    const size_t NN = (size_t)N * N;
    double2* U = c.U + (size_t)slot * NN;
    double2* V = c.V + (size_t)slot * NN;
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < NN; e += (size_t)gridDim.x * blockDim.x) {
        double2 v = cmk((e % N) == (e / N) ? 1.0 : 0.0, 0.0);
        U[e] = v; V[e] = v;
        if (e < (size_t)N) c.D[(size_t)slot * N + e] = 1.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) c.logdetQ[slot] = cmk(0, 0);
}

__global__ void __launch_bounds__(256) k_zgemm_test(const ChainDev* __restrict__ chains, int m, int n, int k, int opa, int opb,
                                                    int a_id, int b_id, int c_id, double beta_re) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.y];
    ZGemmArgs g;
    g.M = m; g.N = n; g.K = k; g.alpha = cmk(1, 0); g.beta = cmk(beta_re, 0);
    g.A = chain_mat(c, a_id); g.lda = c.N; g.opA = opa;
    g.B = chain_mat(c, b_id); g.ldb = c.N; g.opB = opb;
    g.C = chain_mat(c, c_id); g.ldc = c.N;
    zgemm_cta<GemmBig>(g, blockIdx.x, gridDim.x, ssm);
}

// QR of matrix a_id in place; Q into q_id; logdetQ into stats[ST_LOGDETM]
__global__ void __launch_bounds__(256) k_qr_test(const ChainDev* __restrict__ chains, int a_id, int q_id) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.x];
    const int N = c.N;
    StabSmem* S = (StabSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = make_scratch(c);
    double2* A = chain_mat(c, a_id);
    cta_qr64(A, N, sc, ssm, ssm, &S->L);
    double2 ld = cta_logdet_q(sc.tau, N, S->red);
    if (threadIdx.x == 0) { c.stats[ST_LOGDETM_RE] = ld.x; c.stats[ST_LOGDETM_IM] = ld.y; }
    __syncthreads();
    cta_form_q64(A, N, chain_mat(c, q_id), sc, ssm);
}

// swap logical slot n with the spare slot (logical id `spare`)
__global__ void k_swap_slots(int* slotmap, int n, int spare) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int t = slotmap[n]; slotmap[n] = slotmap[spare]; slotmap[spare] = t;
    }
}

static int g_stab_attr = 0;
static void stab_attrs() {
    if (g_stab_attr) return;
    cudaFuncSetAttribute(k_stab, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_green, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_green_tau, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_qr_test, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_zgemm_test, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    g_stab_attr = 1;
}

static int g_maxN = 512;
void set_stab_maxN(int n) { g_maxN = n; }

void launch_stab(const ChainDev* chains, int nchains, int n, int dir, int pivoted, cudaStream_t st) {
    (void)pivoted;
    stab_attrs();
    int src = dir == 0 ? n - 1 : n, dst = dir == 0 ? n : n - 1;
    k_stab<<<nchains, 256, stab_smem_bytes(g_maxN), st>>>(chains, src, dst);
}

void launch_stab_slots(const ChainDev* chains, int nchains, int src, int dst, cudaStream_t st) {
    stab_attrs();
    k_stab<<<nchains, 256, stab_smem_bytes(g_maxN), st>>>(chains, src, dst);
}

void launch_green(const ChainDev* chains, int nchains, int nr, int nl, int rmat_u, int rmat_v,
                  int lmat_u, int lmat_v, int mode, cudaStream_t st) {
    (void)rmat_u; (void)rmat_v; (void)lmat_u; (void)lmat_v;
    stab_attrs();
    k_green<<<nchains, 256, stab_smem_bytes(g_maxN), st>>>(chains, nr, nl, mode);
}

void launch_green_tau(const ChainDev* chains, int nchains, int nr, int nl, cudaStream_t st) {
    stab_attrs();
    k_green_tau<<<nchains, 256, stab_smem_bytes(g_maxN), st>>>(chains, nr, nl);
}

void launch_stage(const ChainDev* chains, int nchains, int nslots, int dir, cudaStream_t st) {
    k_stage<<<dim3(64, nchains), 256, 0, st>>>(chains, nslots, dir);
}

void launch_dyn_init(const ChainDev* chains, int nchains, cudaStream_t st) {
    k_dyn_init<<<dim3(32, nchains), 256, 0, st>>>(chains);
}

void launch_wrap_check(const ChainDev* chains, int nchains, int record, cudaStream_t st) {
    k_wrap_check<<<nchains, 256, 0, st>>>(chains, record);
}

void launch_copy_mat(const ChainDev* chains, int nchains, int dst_id, int src_id, int identity, cudaStream_t st) {
    dim3 grid(8, nchains);
    k_copy_mat<<<grid, 256, 0, st>>>(chains, dst_id, src_id, identity);
}

void launch_swap_slots(int* slotmap, int n, int spare, cudaStream_t st) {
    k_swap_slots<<<1, 32, 0, st>>>(slotmap, n, spare);
}

void launch_stack_identity(const ChainDev* chains, int nchains, int slot, cudaStream_t st) {
    dim3 grid(8, nchains);
    k_stack_identity<<<grid, 256, 0, st>>>(chains, slot);
}

// Dense kinetic step, the zgemm branch of the h0conf props
// (src/dqmc_config_h0/dqmc_left_forward_prop.f90:235-246 and its siblings):
// W4 = K X (left), X K (right) or K^T X (right side on the transposed tall
// UL^T, where (UL K)^T = K^T UL^T), K = urtm1 for the backward ops and urt
// otherwise (urt is Hermitian, so the _hc op uses it too).  The CTAs of a
// chain share its output tiles; k_kin_copy writes the result back.
__global__ void __launch_bounds__(256) k_kin_dense(const ChainDev* __restrict__ chains, int mat_id, int which,
                                                   int right, int tall) {
    extern __shared__ double2 dsm[];
    const ChainDev& c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    const int N = c.N, nv = tall ? md.ne : N;
    const double2* K = (which == PW_INV) ? md.urtm1d : md.urtd;
    const double2* X = chain_mat(c, mat_id);
    ZGemmArgs g;
    g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.C = c.W[4]; g.ldc = N;
    if (right && !tall) {
        g.M = N; g.N = N; g.K = N;
        g.A = X; g.lda = N; g.opA = OP_N;
        g.B = K; g.ldb = N; g.opB = OP_N;
    } else {
        g.M = N; g.N = nv; g.K = N;
        g.A = K; g.lda = N; g.opA = right ? OP_T : OP_N;
        g.B = X; g.ldb = N; g.opB = OP_N;
    }
    zgemm_cta<GemmBig>(g, blockIdx.x, gridDim.x, dsm);
}

// X <- W4 (sub = 0) or X - W4 (sub = 1), X of N x ne (tall) or N x N
__global__ void k_kin_copy(const ChainDev* __restrict__ chains, int mat_id, int tall, int sub) {
    const ChainDev& c = chains[blockIdx.y];
    const int N = c.N, nv = tall ? c.md->ne : N;
    double2* X = chain_mat(c, mat_id);
    const size_t n = (size_t)N * nv;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        X[e] = sub ? csub(X[e], c.W[4][e]) : c.W[4][e];
}

// W4 = A B of two N x N chain matrices (the unequal-time products of
// dqmc_proj_dyn.f90:95-98), output tiles shared by the chain's CTAs
__global__ void __launch_bounds__(256) k_chain_gemm(const ChainDev* __restrict__ chains, int a_id, int b_id) {
    extern __shared__ double2 dsm[];
    const ChainDev& c = chains[blockIdx.y];
    const int N = c.N;
    ZGemmArgs g;
    g.M = N; g.N = N; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = chain_mat(c, a_id); g.lda = N; g.opA = OP_N;
    g.B = chain_mat(c, b_id); g.ldb = N; g.opB = OP_N;
    g.C = c.W[4]; g.ldc = N;
    zgemm_cta<GemmBig>(g, blockIdx.x, gridDim.x, dsm);
}

// s_compare_max_z of the propagated and the fresh G(t,t) into xmax_dyn,
// logdyncount and avglog10dynerror, then G = Gnew (dqmc_proj_dyn.f90:76-94)
__global__ void __launch_bounds__(256) k_dyn_err(const ChainDev* __restrict__ chains) {
    __shared__ double red[64];
    const ChainDev c = chains[blockIdx.x];
    const size_t NN = (size_t)c.N * c.N;
    double mx = 0.0;
    for (size_t e = threadIdx.x; e < NN; e += blockDim.x) {
        mx = fmax(mx, cabsd(csub(c.Gnew[e], c.G[e])));
        c.G[e] = c.Gnew[e];
    }
    mx = block_max(mx, red);
    if (threadIdx.x == 0) {
        c.stats[ST_MAX_DYN] = fmax(c.stats[ST_MAX_DYN], mx);
        c.stats[ST_DYN_LOG10] += log10(mx);
        c.stats[ST_DYN_COUNT] += 1.0;
    }
}

static int g_kin_attr = 0;

void launch_kin_dense(const ChainDev* chains, int nchains, int maxN, int mat_id, int which, int right, int tall,
                      cudaStream_t st) {
    if (!g_kin_attr) {
        cudaFuncSetAttribute(k_kin_dense, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(GemmBig::SMEM_ELEMS * sizeof(double2)));
        g_kin_attr = 1;
    }
    const int tiles = ((maxN + GemmBig::BM - 1) / GemmBig::BM) * ((maxN + GemmBig::BN - 1) / GemmBig::BN);
    k_kin_dense<<<dim3(tiles, nchains), 256, GemmBig::SMEM_ELEMS * sizeof(double2), st>>>(chains, mat_id, which, right, tall);
    k_kin_copy<<<dim3((maxN * maxN + 255) / 256, nchains), 256, 0, st>>>(chains, mat_id, tall, 0);
}

static int g_cg_attr = 0;

void launch_chain_gemm(const ChainDev* chains, int nchains, int maxN, int dst_id, int a_id, int b_id, int sub,
                       cudaStream_t st) {
    if (!g_cg_attr) {
        cudaFuncSetAttribute(k_chain_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(GemmBig::SMEM_ELEMS * sizeof(double2)));
        g_cg_attr = 1;
    }
    const int tiles = ((maxN + GemmBig::BM - 1) / GemmBig::BM) * ((maxN + GemmBig::BN - 1) / GemmBig::BN);
    k_chain_gemm<<<dim3(tiles, nchains), 256, GemmBig::SMEM_ELEMS * sizeof(double2), st>>>(chains, a_id, b_id);
    k_kin_copy<<<dim3((maxN * maxN + 255) / 256, nchains), 256, 0, st>>>(chains, dst_id, 0, sub);
}

void launch_dyn_err(const ChainDev* chains, int nchains, cudaStream_t st) {
    k_dyn_err<<<nchains, 256, 0, st>>>(chains);
}

void launch_zgemm_test(const ChainDev* chains, int nchains, int m, int n, int k, int opa, int opb,
                       int a_id, int b_id, int c_id, double beta_re, cudaStream_t st) {
    stab_attrs();
    dim3 grid(1, nchains);   // one CTA per chain, as in the stabilisation kernels
    k_zgemm_test<<<grid, 256, GemmBig::SMEM_ELEMS * sizeof(double2), st>>>(chains, m, n, k, opa, opb, a_id, b_id, c_id, beta_re);
}

void launch_qr_test(const ChainDev* chains, int nchains, int a_id, int q_id, cudaStream_t st) {
    stab_attrs();
    k_qr_test<<<nchains, 256, stab_smem_bytes(g_maxN), st>>>(chains, a_id, q_id);
}
