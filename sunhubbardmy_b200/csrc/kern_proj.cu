// Projective (ground-state) DQMC: updates, stabilisation and Green's function
// of the projector path, one CTA per walker for the sequential parts.
//
// State per walker: UR = B(tau,0) P (N x ne), UL = P^H B(beta,tau) (ne x N,
// stored transposed as ULT = UL^T, N x ne), ULRINV = (UL UR)^-1 (ne x ne) and
// the stack Ust(0:nst) of N x ne matrices (src/dqmc_proj_core.f90:11-19).
//
// Reference routines:
//  * k_proj_update: dqmc_proj_update_submatrix_LR (src/dqmc_config_v/
//    dqmc_proj_update_submatrix_LR.f90:1-298 for the bond field,
//    src/dqmc_config_u/dqmc_proj_update_submatrix_LR.f90:1-282 for the site
//    field).  Units (bonds of one family, or sites) are visited in order in
//    windows of `wrows` rows (nustock): the window's rows of R = UR ULRINV and
//    of F = R UL are formed by two GEMMs, the accept/reject sequence runs on
//    the F block in shared memory while Gamma^-1 = (I + Delta F_AA)^-1 Delta
//    is bordered one accepted unit at a time, and the window is flushed with
//    ULRINV -= (ULRINV UL_A)(Gamma^-1 R_A) and UR_A <- (I + Delta) UR_A.
//    Instead of re-evaluating F_rr - F_rA Gamma^-1 F_Ar for each unit, the
//    kernel keeps the trailing block of F updated (rank-2 Schur complement
//    per accept), which gives the same numbers in exact arithmetic.
//  * k_proj_qr: s_zgeQR_pqmc (lib/s_matrix.f90:1822-1996) as used by
//    dqmc_proj_stablize_0b_qr / _b0_qr: Q of a tall N x ne matrix with an
//    even number of negative R diagonal entries (else column 1 is negated)
//    and log |det R|.  The wide UL is factored through its transpose, which
//    is the stored layout.
//  * k_proj_ulr: ULR = UL UR and its inverse (s_invlu_z /
//    s_inv_logdet_lu_z); the inverse is taken through a Householder QR, and
//    log det ULR = log det Q + sum log R_ii.
//  * k_proj_t1 + k_proj_gmat: green_equaltime (src/dqmc_proj_core/
//    green_equaltime.f90): G = I - (UR ULRINV) UL, several CTAs per walker.
#include "chain_access.cuh"
#include "kernels.h"
#include "linalg.cuh"

#define PW_MAXR 32          // largest update window (rows)
#define PW_LD (PW_MAXR + 1)

struct ProjSmem {
    LinalgSmem L;
    double red[64];
};

DQ_DEV LinalgScratch proj_scratch(const ChainDev& c) {
    LinalgScratch s;
    s.Vs = c.W[5];
    s.Ws = c.smallw;
    s.Ws2 = c.smallw + (size_t)QR_NB2 * c.N;
    s.T = c.T;
    s.tau = c.tau;
    s.T64 = c.T64;
    return s;
}

static size_t proj_la_smem(int maxN) {
    size_t a = QR_PANEL_ELEMS(maxN);
    size_t b = GemmBig::SMEM_ELEMS;
    if ((size_t)GemmWide::SMEM_ELEMS > b) b = GemmWide::SMEM_ELEMS;
    return (a > b ? a : b) * sizeof(double2) + sizeof(ProjSmem) + 64;
}

// ---------------------------------------------------------------------------
// s_zgeQR_pqmc on the N x ne matrix mat_id, in place (X <- Q); the log of
// |det R| goes to logwDV[dst] = logwDV[add] + log|det R| (add < 0: nothing added;
// dst < 0: not recorded).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_proj_qr(const ChainDev* __restrict__ chains, int mat_id, int dst, int add) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, ne = md.ne, tid = threadIdx.x, nth = blockDim.x;
    double2* buf = ssm;
    ProjSmem* S = (ProjSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = proj_scratch(c);
    double2* X = chain_mat(c, mat_id);
    double2* A = c.W[1];
    for (size_t e = tid; e < (size_t)N * ne; e += nth) A[e] = X[e];
    __syncthreads();
    cta_qr64(A, N, sc, buf, buf, &S->L, ne);
    double lg = 0.0, neg = 0.0;
    for (int i = tid; i < ne; i += nth) {
        double r = A[MIDX(i, i, N)].x;
        lg += log(fabs(r));
        neg += (r < 0.0) ? 1.0 : 0.0;
    }
    lg = block_sum(lg, S->red);
    neg = block_sum(neg, S->red);
    cta_form_q64(A, N, X, sc, buf, ne);
    __syncthreads();
    if (((long long)llround(neg)) & 1)
        for (int i = tid; i < N; i += nth) X[i] = cmk(-X[i].x, -X[i].y);
    if (tid == 0 && dst >= 0) c.logwDV[dst] = (add >= 0 ? c.logwDV[add] : 0.0) + lg;
}

// ---------------------------------------------------------------------------
// out = (ULT^T UR)^-1; with logdet, stats[LOGDETM] = logwDV[ia] (+ logwDV[ib]) +
// log det(UL UR), the logweightf of the sweep routines.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_proj_ulr(const ChainDev* __restrict__ chains, int out_id, int logdet, int ia, int ib) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, ne = md.ne, tid = threadIdx.x, nth = blockDim.x;
    double2* buf = ssm;
    ProjSmem* S = (ProjSmem*)(ssm + ((QR_PANEL_ELEMS(N) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(N) : (size_t)GemmBig::SMEM_ELEMS));
    LinalgScratch sc = proj_scratch(c);
    double2* M = c.W[2];
    ZGemmArgs g;
    g.M = ne; g.N = ne; g.K = N; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = c.ULT; g.lda = N; g.opA = OP_T; g.B = c.UR; g.ldb = N; g.opB = OP_N; g.C = M; g.ldc = ne;
    zgemm_cta<GemmBig>(g, 0, 1, buf);
    cta_qr64(M, ne, sc, buf, buf, &S->L);
    double2 ld = cmk(0, 0);
    int bad = 0;
    for (int i = tid; i < ne; i += nth) {
        const double r = M[MIDX(i, i, ne)].x;
        bad |= (r == 0.0 || !isfinite(r));
    }
    // a zero or non-finite pivot of UL UR: zgetrf's info > 0 in s_inv_logdet_lu_z
    bad = __syncthreads_or(bad);
    if (bad && tid == 0) chain_raise(c, DQ_FAIL_SINGULAR);
    if (logdet) {
        ld = cta_logdet_q(sc.tau, ne, S->red);
        double2 lr = cmk(0, 0);
        for (int i = tid; i < ne; i += nth) {
            double r = M[MIDX(i, i, ne)].x;
            lr = cadd(lr, cmk(log(fabs(r)), r < 0.0 ? M_PI : 0.0));
        }
        lr = block_csum(lr, S->red);
        ld = cadd(ld, lr);
    }
    double2* X = chain_mat(c, out_id);
    for (int e = tid; e < ne * ne; e += nth) X[e] = cmk((e % ne) == (e / ne) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    cta_apply_qh64(M, ne, X, sc, buf);
    cta_trsm_upper(M, ne, X, buf, &S->L);
    if (logdet && tid == 0) {
        double w = c.logwDV[ia] + (ib >= 0 ? c.logwDV[ib] : 0.0);
        c.stats[ST_LOGDETM_RE] = ld.x + w;
        c.stats[ST_LOGDETM_IM] = ld.y;
        c.stats[ST_GINFO] = (bad || !isfinite(ld.x + w) || !isfinite(ld.y)) ? (double)DQ_FAIL_SINGULAR : 0.0;
    }
}

// T1 = UR * INV (N x ne), tiles shared by gridDim.x CTAs per walker
__global__ void __launch_bounds__(256) k_proj_t1(const ChainDev* __restrict__ chains, int inv_id) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.y];
    const int N = c.N, ne = c.md->ne;
    ZGemmArgs g;
    g.M = N; g.N = ne; g.K = ne; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = c.UR; g.lda = N; g.opA = OP_N; g.B = chain_mat(c, inv_id); g.ldb = ne; g.opB = OP_N;
    g.C = c.W[0]; g.ldc = N;
    zgemm_cta<GemmBig>(g, blockIdx.x, gridDim.x, ssm);
}

// dst = I - T1 * ULT^T (N x N)
__global__ void __launch_bounds__(256) k_proj_gmat(const ChainDev* __restrict__ chains, int dst_id) {
    extern __shared__ double2 ssm[];
    const ChainDev c = chains[blockIdx.y];
    const int N = c.N, ne = c.md->ne;
    double2* D = chain_mat(c, dst_id);
    ZGemmArgs g;
    g.M = N; g.N = N; g.K = ne; g.alpha = cmk(-1, 0); g.beta = cmk(0, 0);
    g.A = c.W[0]; g.lda = N; g.opA = OP_N; g.B = c.ULT; g.ldb = N; g.opB = OP_T;
    g.C = D; g.ldc = N;
    zgemm_cta<GemmBig>(g, blockIdx.x, gridDim.x, ssm);
    // the diagonal of the tiles this CTA wrote
    const int tm = (N + GemmBig::BM - 1) / GemmBig::BM, tn = (N + GemmBig::BN - 1) / GemmBig::BN;
    for (int t = blockIdx.x; t < tm * tn; t += gridDim.x) {
        int m0 = (t % tm) * GemmBig::BM, n0 = (t / tm) * GemmBig::BN;
        int lo = max(m0, n0), hi = min(min(m0 + GemmBig::BM, n0 + GemmBig::BN), N);
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) D[MIDX(i, i, N)].x += 1.0;
    }
}

// copy of an N x ne matrix (conj = 1: complex conjugate)
__global__ void k_tall_copy(const ChainDev* __restrict__ chains, int dst_id, int src_id) {
    const ChainDev c = chains[blockIdx.y];
    const size_t n = (size_t)c.N * c.md->ne;
    double2* d = chain_mat(c, dst_id);
    const double2* s = chain_mat(c, src_id);
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) d[e] = s[e];
}

// ---------------------------------------------------------------------------
// projective local update (submatrix-LR), see the file header.  One window of
// one bond family (or of the sites) is three launches:
//   k_pwin_rg    (several CTAs per walker)  Rg = UR(rows,:) ULRINV  [nr x ne]
//                                           Ut = ULRINV UL(:,rows)  [ne x nr]
//   k_pwin_seq   (one CTA per walker)       F = Rg UL(:,rows), the accept /
//                reject sequence with Gamma bordering, Vt = Gamma Rg,
//                UR(A,:) *= 1 + Delta
//   k_pwin_flush (several CTAs per walker)  ULRINV -= Ut Vt
// so the window GEMMs use all SMs while the sequential part runs one CTA per
// walker.  Scratch per walker in pw: Rg (nr x ne), Fg, Gg (nr x nr), Ut, Vt.
// ---------------------------------------------------------------------------
struct PUpdSmem {
    double2 F[PW_MAXR * PW_LD];     // F block of the window (window-start values)
    double2 Pc[PW_MAXR * PW_LD];    // F block with the window's accepted changes folded in
    double2 Gm[PW_MAXR * PW_LD];    // Gamma^-1 in window coordinates (zero off the accepted rows)
    double2 colr[PW_MAXR * 2], rowr[PW_MAXR * 2], ikk[PW_MAXR * 2], kik[PW_MAXR * 2];
    double2 gkk[4];
    double2 dl[PW_MAXR];
    double2 phase;
    int rows[PW_MAXR];
    int accr[PW_MAXR];
    int acc_flag[2], nacc;
    double accm, nties;
    // per-unit proposal, prepared in parallel before the sequential walk
    double2 ud1[PW_MAXR], ud2[PW_MAXR];   // Delta of the unit's rows
    double ur2[PW_MAXR];                  // accept threshold (second draw)
    int uisp[PW_MAXR], ukk[PW_MAXR];      // proposed value, HS-table index (site field)
};

DQ_DEV double u32_stream(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

// window geometry of one walker: returns false when window w is past the end
struct PWin {
    int bond, b, nunits, R, upw, u0, nu, nr;
    const int* rows;     // global row list of the window (bond field), nullptr for sites
};
DQ_DEV bool pwin(const ChainDev& c, int nf, int w, PWin& p) {
    const ModelDev& md = *c.md;
    p.bond = nf > 0;
    p.b = p.bond ? 2 : 1;
    p.nunits = p.bond ? md.nn_lf : c.N;
    int R = min(md.nublock, PW_MAXR);
    R -= R % p.b;
    if (R < p.b) R = p.b;
    p.R = R;
    p.upw = R / p.b;
    p.u0 = w * p.upw;
    if (p.u0 >= p.nunits) return false;
    p.nu = min(p.upw, p.nunits - p.u0);
    p.nr = p.nu * p.b;
    p.rows = p.bond ? md.vrows + (size_t)(nf - 1) * 2 * md.nn_lf + 2 * p.u0 : nullptr;
    return true;
}

DQ_DEV void pw_ptrs(const ChainDev& c, int R, double2*& Rg, double2*& Fg, double2*& Gg, double2*& Ut, double2*& Vt) {
    const int ne = c.md->ne;
    Rg = c.pw;
    Fg = Rg + (size_t)R * ne;
    Gg = Fg + (size_t)R * R;
    Ut = Gg + (size_t)R * R;
    Vt = Ut + (size_t)ne * R;
}

// Rg = UR(rows,:) ULRINV and Ut = ULRINV UL(:,rows) = ULRINV ULT(rows,:)^T
__global__ void __launch_bounds__(256) k_pwin_rg(const ChainDev* __restrict__ chains, int nf, int w) {
    extern __shared__ double2 ssm[];
    const ChainDev& c = chains[blockIdx.y];
    PWin p;
    if (!pwin(c, nf, w, p)) return;
    const int N = c.N, ne = c.md->ne;
    double2 *Rg, *Fg, *Gg, *Ut, *Vt;
    pw_ptrs(c, p.R, Rg, Fg, Gg, Ut, Vt);
    ZGemmArgs ga;   // Rg
    ga.M = p.nr; ga.N = ne; ga.K = ne; ga.alpha = cmk(1, 0); ga.beta = cmk(0, 0);
    ga.A = p.rows ? c.UR : c.UR + p.u0; ga.lda = N; ga.opA = OP_N; ga.arow = p.rows;
    ga.B = c.ULRINV; ga.ldb = ne; ga.opB = OP_N; ga.C = Rg; ga.ldc = p.nr;
    ZGemmArgs gb;   // Ut
    gb.M = ne; gb.N = p.nr; gb.K = ne; gb.alpha = cmk(1, 0); gb.beta = cmk(0, 0);
    gb.A = c.ULRINV; gb.lda = ne; gb.opA = OP_N;
    gb.B = p.rows ? c.ULT : c.ULT + p.u0; gb.ldb = N; gb.opB = OP_T; gb.brow = p.rows;
    gb.C = Ut; gb.ldc = ne;
    const int ca = zt_pick(ga.M, ga.N), cb = zt_pick(gb.M, gb.N);
    const int ta = zt_tiles(ca, ga.M, ga.N), tb = zt_tiles(cb, gb.M, gb.N);
    for (int t = blockIdx.x; t < ta + tb; t += gridDim.x) {
        if (t < ta) zgemm_tile(ga, ca, t, ssm);
        else zgemm_tile(gb, cb, t - ta, ssm);
    }
}

// ULRINV -= Ut Vt (skipped when the window accepted nothing)
__global__ void __launch_bounds__(256) k_pwin_flush(const ChainDev* __restrict__ chains, int nf, int w) {
    extern __shared__ double2 ssm[];
    const ChainDev& c = chains[blockIdx.y];
    PWin p;
    if (!pwin(c, nf, w, p)) return;
    if (c.pw_flag[0] == 0) return;
    const int ne = c.md->ne;
    double2 *Rg, *Fg, *Gg, *Ut, *Vt;
    pw_ptrs(c, p.R, Rg, Fg, Gg, Ut, Vt);
    ZGemmArgs g;
    g.M = ne; g.N = ne; g.K = p.nr; g.alpha = cmk(-1, 0); g.beta = cmk(1, 0);
    g.A = Ut; g.lda = ne; g.opA = OP_N; g.B = Vt; g.ldb = p.nr; g.opB = OP_N; g.C = c.ULRINV; g.ldc = ne;
    const int cl = zt_pick(g.M, g.N), nt = zt_tiles(cl, g.M, g.N);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) zgemm_tile(g, cl, t, ssm);
}

// visit: slices already updated in this half sweep; dir 0 = 0b (bond families
// 1..nn_nf, then sites), 1 = b0 (sites, then families nn_nf..1) fixes where
// this call's draws sit in the half sweep's random words; rnd_off >= 0
// overrides that offset.  last = 1 on the family's last window (statistics).
__global__ void __launch_bounds__(256) k_pwin_seq(const ChainDev* __restrict__ chains, int nt, int nf, int w, int visit,
                                                  int dir, int rnd_off) {
    extern __shared__ double2 ssm[];
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    const int N = c.N, ne = md.ne, tid = threadIdx.x, nth = blockDim.x;
    PWin p;
    if (!pwin(c, nf, w, p)) {
        if (tid == 0) c.pw_flag[0] = 0;
        return;
    }
    double2* buf = ssm;
    PUpdSmem* S = (PUpdSmem*)(ssm + ZT_SMEM_ELEMS);
    const int bond = p.bond, b = p.b, nu = p.nu, nr = p.nr, u0 = p.u0;
    const int lc = bond ? 2 : md.lcomp;
    if (rnd_off < 0) {
        const int vw = md.lwrapv ? 2 * md.nn_lf * md.nn_nf : 0, uw = md.lwrapu ? 2 * N : 0;
        int within;
        if (dir == 0) within = md.rw_pre0 + (bond ? (nf - 1) * 2 * md.nn_lf : vw);
        else within = bond ? uw + (md.nn_nf - nf) * 2 * md.nn_lf : 0;
        rnd_off = visit * md.rps + within;
    }
    const uint32_t* rnd = c.rnd + rnd_off;
    int32_t* cf = bond ? c.vconf + ((size_t)(nt - 1) * md.nn_nf + (nf - 1)) * N : c.conf + (size_t)(nt - 1) * N;
    double2 *Rg, *Fg, *Gg, *Ut, *Vt;
    pw_ptrs(c, p.R, Rg, Fg, Gg, Ut, Vt);
    for (int x = tid; x < nr; x += nth) S->rows[x] = p.rows ? p.rows[x] : u0 + x;
    if (tid == 0) {
        S->phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
        S->accm = 0.0;
        S->nties = 0.0;
        S->nacc = 0;
    }
    {   // F = Rg UL(:,rows) = Rg ULT(rows,:)^T
        ZGemmArgs g;
        g.M = nr; g.N = nr; g.K = ne; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
        g.A = Rg; g.lda = nr; g.opA = OP_N;
        g.B = p.rows ? c.ULT : c.ULT + u0; g.ldb = N; g.opB = OP_T; g.brow = p.rows;
        g.C = Fg; g.ldc = nr;
        zgemm_fit(g, buf);
    }
    for (int e = tid; e < nr * nr; e += nth) {
        int x = e % nr, y = e / nr;
        double2 v = Fg[e];
        S->F[x + y * PW_LD] = v;
        S->Pc[x + y * PW_LD] = v;
        S->Gm[x + y * PW_LD] = cmk(0, 0);
    }
    for (int x = tid; x < nr; x += nth) { S->dl[x] = cmk(0, 0); S->accr[x] = 0; }
    for (int k = tid; k < nu; k += nth) {
        const int u = u0 + k;
        const int is = cf[u];
        const double r1 = u32_stream(rnd[2 * u]);
        const int iflip = (int)ceil(r1 * (lc - 1));
        S->uisp[k] = (is + iflip - 1) % lc + 1;
        S->ur2[k] = u32_stream(rnd[2 * u + 1]);
        if (bond) {
            S->ud1[k] = md.vdp[is - 1];
            S->ud2[k] = md.vdm[is - 1];
            S->ukk[k] = 0;
        } else {
            const int kk = (is - 1) * (lc - 1) + (iflip - 1);
            S->ud1[k] = md.delta[kk];
            S->ud2[k] = cmk(0, 0);
            S->ukk[k] = kk;
        }
    }
    __syncthreads();
    const int warp = tid >> 5;
    for (int k = 0; k < nu; ++k) {
        const int r0 = k * b;
        if (warp == 0) {
            if (tid == 0) {
                double2 ratiotot, g11, g12 = cmk(0, 0), g21 = cmk(0, 0), g22 = cmk(0, 0);
                const double2 d1 = S->ud1[k], d2 = S->ud2[k];
                if (bond) {
                    double2 v11 = cadd(cmk(1, 0), cmul(S->Pc[r0 + r0 * PW_LD], d1));
                    double2 v21 = cmul(S->Pc[r0 + 1 + r0 * PW_LD], d1);
                    double2 v12 = cmul(S->Pc[r0 + (r0 + 1) * PW_LD], d2);
                    double2 v22 = cadd(cmk(1, 0), cmul(S->Pc[r0 + 1 + (r0 + 1) * PW_LD], d2));
                    double2 det = csub(cmul(v11, v22), cmul(v12, v21));
                    ratiotot = det;
                    double2 id = cdiv(cmk(1, 0), det);
                    g11 = cmul(cmul(v22, d1), id);
                    g12 = cmul(cmul(cmk(-v12.x, -v12.y), d1), id);
                    g21 = cmul(cmul(cmk(-v21.x, -v21.y), d2), id);
                    g22 = cmul(cmul(v11, d2), id);
                } else {
                    const int kk = S->ukk[k];
                    double2 ratio1 = cadd(cmk(1, 0), cmul(S->Pc[r0 + r0 * PW_LD], d1));
                    double2 r = ratio1;
                    for (int f = 1; f < md.nflr; ++f) r = cmul(r, ratio1);
                    r = cscale(r, md.gam_ratio[kk]);
                    ratiotot = cmul(r, md.phase_ratio[kk]);
                    g11 = cdiv(d1, ratio1);
                }
                const double2 ph = S->phase;
                double ratio_re = cmul(ratiotot, ph).x / ph.x;
                int acc = fabs(ratio_re) > S->ur2[k];
                if (fabs(fabs(ratio_re) - S->ur2[k]) < DQ_NEAR_TIE) S->nties += 1.0;
                if (acc) {
                    double wgt = sqrt(cmul(ratiotot, cconj(ratiotot)).x);
                    S->phase = cscale(cmul(ph, ratiotot), 1.0 / wgt);
                    cf[u0 + k] = S->uisp[k];
                    S->accm += 1.0;
                    S->gkk[0] = g11; S->gkk[1] = g21; S->gkk[2] = g12; S->gkk[3] = g22;   // column-major b x b
                    S->dl[r0] = d1;
                    S->accr[r0] = 1;
                    if (bond) { S->dl[r0 + 1] = d2; S->accr[r0 + 1] = 1; }
                    S->nacc += b;
                }
                S->acc_flag[k & 1] = acc;
            }
        } else {
            // warps 1..7, while warp 0 decides: columns / rows r of the current
            // block and Gamma F_Ar, F_rA Gamma (four partial sums per product)
            for (int e = tid - 32; e < nr * b; e += nth - 32) {
                int x = e % nr, cc = e / nr;
                S->colr[x + cc * PW_MAXR] = S->Pc[x + (r0 + cc) * PW_LD];
                S->rowr[x + cc * PW_MAXR] = S->Pc[r0 + cc + x * PW_LD];
                double2 a[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
                double2 bb[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
                int y = 0;
                for (; y + 3 < r0; y += 4)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        a[q] = cfma(S->Gm[x + (y + q) * PW_LD], S->F[y + q + (r0 + cc) * PW_LD], a[q]);
                        bb[q] = cfma(S->F[r0 + cc + (y + q) * PW_LD], S->Gm[y + q + x * PW_LD], bb[q]);
                    }
                for (; y < r0; ++y) {
                    a[0] = cfma(S->Gm[x + y * PW_LD], S->F[y + (r0 + cc) * PW_LD], a[0]);
                    bb[0] = cfma(S->F[r0 + cc + y * PW_LD], S->Gm[y + x * PW_LD], bb[0]);
                }
                S->ikk[x + cc * PW_MAXR] = cadd(cadd(a[0], a[1]), cadd(a[2], a[3]));
                S->kik[x + cc * PW_MAXR] = cadd(cadd(bb[0], bb[1]), cadd(bb[2], bb[3]));
            }
        }
        __syncthreads();
        if (!S->acc_flag[k & 1]) continue;
        for (int e = tid; e < nr * nr; e += nth) {
            int x = e % nr, y = e / nr;
            const bool xr = (x >= r0 && x < r0 + b), yr = (y >= r0 && y < r0 + b);
            if (x < r0 && y < r0) {
                double2 sacc = cmk(0, 0);
                for (int pp = 0; pp < b; ++pp)
                    for (int q = 0; q < b; ++q)
                        sacc = cfma(cmul(S->ikk[x + pp * PW_MAXR], S->gkk[pp + q * b]), S->kik[y + q * PW_MAXR], sacc);
                S->Gm[x + y * PW_LD] = cadd(S->Gm[x + y * PW_LD], sacc);
            } else if (xr && y < r0) {
                double2 sacc = cmk(0, 0);
                for (int q = 0; q < b; ++q) sacc = cfma(S->gkk[(x - r0) + q * b], S->kik[y + q * PW_MAXR], sacc);
                S->Gm[x + y * PW_LD] = cmk(-sacc.x, -sacc.y);
            } else if (x < r0 && yr) {
                double2 sacc = cmk(0, 0);
                for (int pp = 0; pp < b; ++pp) sacc = cfma(S->ikk[x + pp * PW_MAXR], S->gkk[pp + (y - r0) * b], sacc);
                S->Gm[x + y * PW_LD] = cmk(-sacc.x, -sacc.y);
            } else if (xr && yr) {
                S->Gm[x + y * PW_LD] = S->gkk[(x - r0) + (y - r0) * b];
            } else if (x >= r0 + b && y >= r0 + b) {
                double2 sacc = cmk(0, 0);
                for (int pp = 0; pp < b; ++pp)
                    for (int q = 0; q < b; ++q)
                        sacc = cfma(cmul(S->colr[x + pp * PW_MAXR], S->gkk[pp + q * b]), S->rowr[y + q * PW_MAXR], sacc);
                S->Pc[x + y * PW_LD] = csub(S->Pc[x + y * PW_LD], sacc);
            }
        }
        __syncthreads();
    }
    const int any = S->nacc > 0;
    if (any) {
        for (int e = tid; e < nr * nr; e += nth) {
            int x = e % nr, y = e / nr;
            Gg[e] = S->Gm[x + y * PW_LD];
        }
        __syncthreads();
        ZGemmArgs g;   // Vt = Gamma Rg
        g.M = nr; g.N = ne; g.K = nr; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
        g.A = Gg; g.lda = nr; g.opA = OP_N; g.B = Rg; g.ldb = nr; g.opB = OP_N; g.C = Vt; g.ldc = nr;
        zgemm_fit(g, buf);
        for (int e = tid; e < nr * ne; e += nth) {
            int x = e % nr, l = e / nr;
            if (S->accr[x]) {
                double2* q = c.UR + MIDX(S->rows[x], l, N);
                double2 v = *q;
                *q = cadd(v, cmul(S->dl[x], v));
            }
        }
    }
    if (tid == 0) {
        c.pw_flag[0] = any;
        c.stats[ST_PHASE_RE] = S->phase.x;
        c.stats[ST_PHASE_IM] = S->phase.y;
        c.stats[bond ? ST_ACCV : ST_ACC] += S->accm;
        c.stats[ST_NEAR_TIE] += S->nties;
        c.stats[bond ? ST_PROPV : ST_PROP] += (double)nu;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int g_proj_attr = 0;
static size_t g_proj_la = 0, g_proj_upd = 0;

void set_proj_maxN(int maxN) {
    g_proj_la = proj_la_smem(maxN);
    g_proj_upd = (size_t)ZT_SMEM_ELEMS * sizeof(double2) + sizeof(PUpdSmem) + 64;
    cudaFuncSetAttribute(k_proj_qr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_proj_la);
    cudaFuncSetAttribute(k_proj_ulr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_proj_la);
    cudaFuncSetAttribute(k_pwin_seq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_proj_upd);
    cudaFuncSetAttribute(k_pwin_rg, cudaFuncAttributeMaxDynamicSharedMemorySize, ZT_SMEM_ELEMS * (int)sizeof(double2));
    cudaFuncSetAttribute(k_pwin_flush, cudaFuncAttributeMaxDynamicSharedMemorySize, ZT_SMEM_ELEMS * (int)sizeof(double2));
    cudaFuncSetAttribute(k_proj_t1, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmBig::SMEM_ELEMS * (int)sizeof(double2));
    cudaFuncSetAttribute(k_proj_gmat, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmBig::SMEM_ELEMS * (int)sizeof(double2));
    g_proj_attr = 1;
}

void launch_proj_qr(const ChainDev* chains, int nchains, int mat_id, int dst, int add, cudaStream_t st) {
    k_proj_qr<<<nchains, 256, g_proj_la, st>>>(chains, mat_id, dst, add);
}

void launch_proj_ulr(const ChainDev* chains, int nchains, int out_id, int logdet, int ia, int ib, cudaStream_t st) {
    k_proj_ulr<<<nchains, 256, g_proj_la, st>>>(chains, out_id, logdet, ia, ib);
}

void launch_proj_green(const ChainDev* chains, int nchains, int inv_id, int dst_id, int ctas, cudaStream_t st) {
    size_t sm = (size_t)GemmBig::SMEM_ELEMS * sizeof(double2);
    k_proj_t1<<<dim3(ctas, nchains), 256, sm, st>>>(chains, inv_id);
    k_proj_gmat<<<dim3(ctas, nchains), 256, sm, st>>>(chains, dst_id);
}

void launch_tall_copy(const ChainDev* chains, int nchains, int dst_id, int src_id, cudaStream_t st) {
    k_tall_copy<<<dim3(8, nchains), 256, 0, st>>>(chains, dst_id, src_id);
}

// one family (nf >= 1) or the site field (nf = 0) of slice nt: nwin windows,
// g_rg / g_fl CTAs per walker for the window GEMMs
void launch_proj_update(const ChainDev* chains, int nchains, int nt, int nf, int visit, int dir, int rnd_off,
                        int nwin, int g_rg, int g_fl, cudaStream_t st) {
    size_t sm = (size_t)ZT_SMEM_ELEMS * sizeof(double2);
    for (int w = 0; w < nwin; ++w) {
        k_pwin_rg<<<dim3(g_rg, nchains), 256, sm, st>>>(chains, nf, w);
        k_pwin_seq<<<nchains, 256, g_proj_upd, st>>>(chains, nt, nf, w, visit, dir, rnd_off);
        k_pwin_flush<<<dim3(g_fl, nchains), 256, sm, st>>>(chains, nf, w);
    }
}
