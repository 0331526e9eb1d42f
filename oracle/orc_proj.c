/* Projective (ground-state) DQMC sweep and the t-V bond field, restated
 * from the Fortran reference.  Test infrastructure only (see dqmc_oracle.h).
 *
 *  - vconf constants, field draw and propagators:
 *      src/dqmc_config_v/dqmc_set_conf.f90:1-79, dqmc_input_conf.f90:36-63,
 *      dqmc_{left,right}_{forward,backward}_prop.f90, _hc
 *  - projective updates (all flavours give the same accept sequence):
 *      src/dqmc_config_v/dqmc_proj_update.f90:1-104 (bond, rank 2, fast)
 *      src/dqmc_config_v/dqmc_proj_update_submatrix_LR.f90:1-298 (bond,
 *        submatrix-LR, selected by update = SUBMATRIX as -DSUBMATRIX does)
 *      src/dqmc_config_u/dqmc_proj_update.f90:1-92  (site, rank 1, fast)
 *  - trial state: src/dqmc_config_h0/set_trial_h0.f90:1-29,
 *      src/dqmc_proj_core/dqmc_set_proj.f90:1-78
 *  - core: src/dqmc_proj_core/dqmc_proj_sweep_start_0b.f90:1-48,
 *      dqmc_proj_sweep_b0.f90:1-220, dqmc_proj_sweep_0b.f90:1-235,
 *      dqmc_proj_stablize_{0b,b0}_qr.f90, green_equaltime.f90, set_phase.f90
 *
 * Layouts follow the reference: UR is ndim x ne, UL is ne x ndim, both
 * column-major; the stack keeps Ust(n) as ndim x ne.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

static zc *zalloc(size_t n) { return calloc(n ? n : 1, sizeof(zc)); }

/* ------------------------------------------------------------------ */
/* vconf constants (src/dqmc_config_v/dqmc_set_conf.f90:1-79)          */
/* ------------------------------------------------------------------ */
void orc_set_vconf(orc_model *m) {
    const orc_params *p = &m->p;
    m->lwrapv = (p->rv != 0.0);
    if (!m->lwrapv) return;
    const double etal[2] = {-1.0, 1.0};
    double al = acosh(exp(p->dtau * p->rv * 0.5));
    m->v_alpha = al;
    for (int is = 1; is <= 2; ++is) {
        if (p->lprojv) {
            zc z = cexp(I * (M_PI * 2.0 * is / 2.0));
            m->vbp[is - 1] = z; m->vbm[is - 1] = z;
            m->vbpi[is - 1] = conj(z); m->vbmi[is - 1] = conj(z);
        } else {
            m->vbp[is - 1] = exp(al * etal[is - 1]);
            m->vbpi[is - 1] = exp(-al * etal[is - 1]);
            m->vbm[is - 1] = exp(-al * etal[is - 1]);
            m->vbmi[is - 1] = exp(al * etal[is - 1]);
        }
        int isp = is % 2 + 1;   /* mod(is+iflip-1, lcomp)+1 with iflip = 1 */
        if (p->lprojv) {
            m->vdp[is - 1] = cexp(I * (M_PI * (2.0 * isp - 2.0 * is) / 2.0)) - 1.0;
            m->vdm[is - 1] = exp(al * (etal[isp - 1] - etal[is - 1])) - 1.0;
        } else {
            m->vdp[is - 1] = exp(al * (etal[isp - 1] - etal[is - 1])) - 1.0;
            m->vdm[is - 1] = exp(-al * (etal[isp - 1] - etal[is - 1])) - 1.0;
        }
    }
}

/* ------------------------------------------------------------------ */
/* vconf props: B_nf = U diag(bmat_p, bmat_m) U^T per bond, U the 2x2   */
/* Hadamard; nflag 2 and 1 are the two halves around the update.       */
/* ------------------------------------------------------------------ */
void orc_v_prop(const orc_model *m, const int32_t *vconf, int op, int nt, int nf, int nflag, zc *g, int n2) {
    const orc_latt *L = &m->L;
    int N = m->ndim, lf = L->nn_lf, nnf = L->nn_nf;
    const double h = 1.0 / sqrt(2.0);
    const zc u11 = h, u12 = h, u21 = h, u22 = -h;   /* u = ut (dqmc_config_v.f90:20-21) */
    const int32_t *cf = vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    int left = (op == ORC_LEFT_FORWARD || op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC);
    for (int b = 0; b < lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b] - 1;
        if (left) {
            /* rows i1, i2 of an N x n2 matrix */
            for (int j = 0; j < n2; ++j) {
                zc x1 = g[ZIDX(i1, j, N)], x2 = g[ZIDX(i2, j, N)];
                if (op == ORC_LEFT_FORWARD || op == ORC_LEFT_FORWARD_HC) {
                    if (nflag == 2) {
                        zc v1 = u11 * x1 + u12 * x2, v2 = u21 * x1 + u22 * x2;
                        x1 = m->vbp[is] * v1; x2 = m->vbm[is] * v2;
                    } else {
                        zc v1 = u11 * x1 + u12 * x2, v2 = u21 * x1 + u22 * x2;
                        x1 = v1; x2 = v2;
                    }
                } else {   /* LEFT_BACKWARD */
                    if (nflag == 2) {
                        zc v1 = u11 * x1 + u12 * x2, v2 = u21 * x1 + u22 * x2;
                        x1 = v1; x2 = v2;
                    } else {
                        x1 = m->vbpi[is] * x1; x2 = m->vbmi[is] * x2;
                        zc v1 = u11 * x1 + u12 * x2, v2 = u21 * x1 + u22 * x2;
                        x1 = v1; x2 = v2;
                    }
                }
                g[ZIDX(i1, j, N)] = x1; g[ZIDX(i2, j, N)] = x2;
            }
        } else {
            /* columns i1, i2 of an n2 x N matrix */
            for (int j = 0; j < n2; ++j) {
                zc x1 = g[ZIDX(j, i1, n2)], x2 = g[ZIDX(j, i2, n2)];
                if (op == ORC_RIGHT_FORWARD) {
                    if (nflag == 2) {
                        zc v1 = x1 * u11 + x2 * u21, v2 = x1 * u12 + x2 * u22;
                        x1 = v1; x2 = v2;
                    } else {
                        x1 = m->vbp[is] * x1; x2 = m->vbm[is] * x2;
                        zc v1 = x1 * u11 + x2 * u21, v2 = x1 * u12 + x2 * u22;
                        x1 = v1; x2 = v2;
                    }
                } else {   /* RIGHT_BACKWARD */
                    if (nflag == 2) {
                        zc v1 = x1 * u11 + x2 * u21, v2 = x1 * u12 + x2 * u22;
                        x1 = m->vbpi[is] * v1; x2 = m->vbmi[is] * v2;
                    } else {
                        zc v1 = x1 * u11 + x2 * u21, v2 = x1 * u12 + x2 * u22;
                        x1 = v1; x2 = v2;
                    }
                }
                g[ZIDX(j, i1, n2)] = x1; g[ZIDX(j, i2, n2)] = x2;
            }
        }
    }
}

void orc_vconf_prop(const orc_model *m, const int32_t *vconf, int op, int nt, int nf, int nflag, double *g, int n2) {
    orc_v_prop(m, vconf, op, nt, nf, nflag, (zc *)g, n2);
}

/* ------------------------------------------------------------------ */
/* chain state                                                         */
/* ------------------------------------------------------------------ */

/* set_trial_h0 (src/dqmc_config_h0/set_trial_h0.f90:1-29) + dqmc_set_proj */
static void set_proj(orc_chain *c) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    const orc_params *p = &m->p;
    int N = m->ndim, nnf = L->nn_nf;
    zc *h = zalloc((size_t)N * N);
    for (int b = 0; b < L->nn_lf; ++b) {
        int i0 = L->nnlf_list[b] - 1;
        for (int nf = 1; nf <= nnf; ++nf) {
            int in = L->nnlist[i0 * nnf + nf - 1] - 1;
            double r = orc_sfmt_stream(&c->rng);
            zc z1 = (-p->rt + p->rndness * (r - 1.0)) * orc_expar(L, i0, nf, p->xmag, p->flux_x, p->flux_y, p->dimer);
            h[ZIDX(i0, in, N)] += z1;
            h[ZIDX(in, i0, N)] += conj(z1);
        }
    }
    for (int i = 0; i < N; ++i) h[ZIDX(i, i, N)] -= p->mu;
    orc_eig_he(N, h, c->trial_w, c->projR);
    memcpy(c->projL, c->projR, sizeof(zc) * (size_t)N * N);
    free(h);
}

void orc_proj_chain_init(orc_chain *c, int draw_conf) {
    const orc_model *m = c->m;
    int N = m->ndim, lt = m->ltrot, nnf = m->L.nn_nf, ne = m->ne, nst = m->nst;
    if (m->lwrapv) {
        c->vconf = calloc((size_t)lt * nnf * N, sizeof(int32_t));
        for (size_t e = 0; e < (size_t)lt * nnf * N; ++e) c->vconf[e] = 1;
        if (draw_conf)   /* dqmc_config_v/dqmc_input_conf.f90:55-63: nt, site, family */
            for (int nt = 0; nt < lt; ++nt)
                for (int i = 0; i < N; ++i)
                    for (int nf = 0; nf < nnf; ++nf)
                        c->vconf[((size_t)nt * nnf + nf) * N + i] = (int32_t)ceil(orc_sfmt_stream(&c->rng) * 2);
    }
    if (!m->proj) return;
    c->projR = zalloc((size_t)N * N);
    c->projL = zalloc((size_t)N * N);
    c->trial_w = calloc(N, sizeof(double));
    c->UR = zalloc((size_t)N * ne);
    c->UL = zalloc((size_t)N * ne);
    c->ULRINV = zalloc((size_t)ne * ne);
    c->Pst = calloc(nst + 1, sizeof(zc *));
    for (int n = 0; n <= nst; ++n) c->Pst[n] = zalloc((size_t)N * ne);
    c->logwDV = calloc(nst + 1, sizeof(double));
    set_proj(c);
}

void orc_proj_chain_free(orc_chain *c) {
    free(c->vconf);
    if (!c->m->proj) return;
    for (int n = 0; n <= c->m->nst; ++n) free(c->Pst[n]);
    free(c->Pst); free(c->logwDV);
    free(c->projR); free(c->projL); free(c->trial_w);
    free(c->UR); free(c->UL); free(c->ULRINV);
}

void orc_proj_get_trial(const orc_chain *c, double *proj, double *w) {
    int N = c->m->ndim;
    if (proj) memcpy(proj, c->projR, sizeof(zc) * (size_t)N * N);
    if (w) memcpy(w, c->trial_w, sizeof(double) * N);
}
void orc_proj_set_trial(orc_chain *c, const double *proj) {
    int N = c->m->ndim;
    memcpy(c->projR, proj, sizeof(zc) * (size_t)N * N);
    memcpy(c->projL, proj, sizeof(zc) * (size_t)N * N);
}
void orc_proj_get(const orc_chain *c, double *ur, double *ul, double *ulrinv) {
    int N = c->m->ndim, ne = c->m->ne;
    if (ur) memcpy(ur, c->UR, sizeof(zc) * (size_t)N * ne);
    if (ul) memcpy(ul, c->UL, sizeof(zc) * (size_t)N * ne);
    if (ulrinv) memcpy(ulrinv, c->ULRINV, sizeof(zc) * (size_t)ne * ne);
}
void orc_proj_set(orc_chain *c, const double *ur, const double *ul, const double *ulrinv) {
    int N = c->m->ndim, ne = c->m->ne;
    if (ur) memcpy(c->UR, ur, sizeof(zc) * (size_t)N * ne);
    if (ul) memcpy(c->UL, ul, sizeof(zc) * (size_t)N * ne);
    if (ulrinv) memcpy(c->ULRINV, ulrinv, sizeof(zc) * (size_t)ne * ne);
}
void orc_vconf_get(const orc_chain *c, int32_t *v) {
    const orc_model *m = c->m;
    if (c->vconf) memcpy(v, c->vconf, sizeof(int32_t) * (size_t)m->ltrot * m->L.nn_nf * m->ndim);
}
void orc_vconf_set(orc_chain *c, const int32_t *v) {
    const orc_model *m = c->m;
    if (c->vconf) memcpy(c->vconf, v, sizeof(int32_t) * (size_t)m->ltrot * m->L.nn_nf * m->ndim);
}

/* ------------------------------------------------------------------ */
/* core helpers                                                        */
/* ------------------------------------------------------------------ */

/* green_equaltime (src/dqmc_proj_core/green_equaltime.f90): gr = I - UR ULRINV UL */
static void proj_green(int N, int ne, const zc *ul, const zc *ur, const zc *ulrinv, zc *gr) {
    zc *t = zalloc((size_t)N * ne);
    orc_zgemm('N', 'N', N, ne, ne, 1.0, ur, N, ulrinv, ne, 0.0, t, N);
    orc_zgemm('N', 'N', N, N, ne, -1.0, t, N, ul, ne, 0.0, gr, N);
    for (int i = 0; i < N; ++i) gr[ZIDX(i, i, N)] += 1.0;
    free(t);
}

void orc_proj_green(orc_chain *c) {
    proj_green(c->m->ndim, c->m->ne, c->UL, c->UR, c->ULRINV, c->gf);
}

/* ULR = UL UR; inverse (s_invlu_z or s_inv_logdet_lu_z) into out */
static void ulr_inverse(int N, int ne, const zc *ul, const zc *ur, zc *out, zc *logdet) {
    orc_zgemm('N', 'N', ne, ne, N, 1.0, ul, ne, ur, N, 0.0, out, ne);
    if (logdet) orc_zinv_logdet(ne, out, logdet);
    else orc_zinv(ne, out);
}

/* dqmc_proj_update, bond field (src/dqmc_config_v/dqmc_proj_update.f90:1-104) */
static void proj_update_v(orc_chain *c, int nt, int nf) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, ne = m->ne, nnf = L->nn_nf;
    int32_t *cf = c->vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    zc *vk_tmp = zalloc(2 * (size_t)ne), *vk = zalloc(2 * (size_t)ne), *uk = zalloc(2 * (size_t)ne);
    zc *lruk = zalloc(2 * (size_t)ne), *vuvk = zalloc(2 * (size_t)ne);
    double accm = 0.0;
    for (int b = 0; b < L->nn_lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * 1);
        int isp = (is + iflip - 1) % 2 + 1;
        zc dp = m->vdp[is - 1], dm = m->vdm[is - 1];
        for (int l = 0; l < ne; ++l) {
            vk_tmp[2 * l] = dp * c->UR[ZIDX(i1, l, N)];        /* D * vuvkmat, 2 x ne */
            vk_tmp[2 * l + 1] = dm * c->UR[ZIDX(i2, l, N)];
            uk[l] = c->UL[ZIDX(l, i1, ne)];                    /* ukmat, ne x 2 */
            uk[ne + l] = c->UL[ZIDX(l, i2, ne)];
        }
        orc_zgemm('N', 'N', 2, ne, ne, 1.0, vk_tmp, 2, c->ULRINV, ne, 0.0, vk, 2);
        zc vuk[4] = {1.0, 0.0, 0.0, 1.0};
        orc_zgemm('N', 'N', 2, 2, ne, 1.0, vk, 2, uk, ne, 1.0, vuk, 2);
        zc det = vuk[0] * vuk[3] - vuk[2] * vuk[1];
        zc inv[4] = {vuk[3] / det, -vuk[1] / det, -vuk[2] / det, vuk[0] / det};
        zc ratiotot = det;
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            for (int l = 0; l < ne; ++l) {
                c->UR[ZIDX(i1, l, N)] += vk_tmp[2 * l];
                c->UR[ZIDX(i2, l, N)] += vk_tmp[2 * l + 1];
            }
            orc_zgemm('N', 'N', 2, ne, 2, 1.0, inv, 2, vk, 2, 0.0, vuvk, 2);
            orc_zgemm('N', 'N', ne, 2, ne, 1.0, c->ULRINV, ne, uk, ne, 0.0, lruk, ne);
            orc_zgemm('N', 'N', ne, ne, 2, -1.0, lruk, ne, vuvk, 2, 1.0, c->ULRINV, ne);
            cf[b] = isp;
        }
    }
    c->acc_v += accm;
    c->prop_v += L->nn_lf;
    free(vk_tmp); free(vk); free(uk); free(lruk); free(vuvk);
}

/* The finite-temperature bond-field update on the equal-time G
 * (src/dqmc_config_v/dqmc_update.f90:1-119; the delayed variant
 * dqmc_update_delay.f90 makes the same draws and decisions): per bond of family
 * nf, in nnlf_list order, iflip and then the accept word; Delta = diag(dp, dm),
 * vukmat = I + (1 - G)(P,P) Delta, ratiotot = det vukmat (no flavour power);
 * on acceptance G <- G - G(:,P) Delta vukmat^-1 (delta(P,:) - G(P,:)). */
void orc_ft_update_v(orc_chain *c, int nt, int nf) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, nnf = L->nn_nf;
    int32_t *cf = c->vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    zc *gc = zalloc(2 * (size_t)N), *vr = zalloc(2 * (size_t)N);
    zc *g = c->gf;
    double accm = 0.0;
    for (int b = 0; b < L->nn_lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * 1);
        int isp = (is + iflip - 1) % 2 + 1;
        zc d[2] = {m->vdp[is - 1], m->vdm[is - 1]};
        int pc[2] = {i1, i2};
        zc vu[4];                                   /* column-major 2 x 2 */
        for (int a = 0; a < 2; ++a)
            for (int q = 0; q < 2; ++q)
                vu[a + 2 * q] = (a == q ? 1.0 : 0.0) + ((pc[a] == pc[q] ? 1.0 : 0.0) - g[ZIDX(pc[a], pc[q], N)]) * d[q];
        zc det = vu[0] * vu[3] - vu[2] * vu[1];
        zc inv[4] = {vu[3] / det, -vu[1] / det, -vu[2] / det, vu[0] / det};
        zc ratiotot = det;
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            zc s[4];                                /* smat = Delta vukmat^-1 */
            for (int a = 0; a < 2; ++a)
                for (int q = 0; q < 2; ++q) s[a + 2 * q] = d[a] * inv[a + 2 * q];
            for (int j = 0; j < N; ++j) {           /* vr = smat (delta(P,:) - G(P,:)), gc = G(:,P) */
                zc v0 = (j == i1 ? 1.0 : 0.0) - g[ZIDX(i1, j, N)];
                zc v1 = (j == i2 ? 1.0 : 0.0) - g[ZIDX(i2, j, N)];
                vr[2 * j] = s[0] * v0 + s[2] * v1;
                vr[2 * j + 1] = s[1] * v0 + s[3] * v1;
                gc[j] = g[ZIDX(j, i1, N)];
                gc[N + j] = g[ZIDX(j, i2, N)];
            }
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i)
                    g[ZIDX(i, j, N)] -= gc[i] * vr[2 * j] + gc[N + i] * vr[2 * j + 1];
            cf[b] = isp;
        }
    }
    c->acc_v += accm;
    c->prop_v += L->nn_lf;
    free(gc); free(vr);
}

/* dqmc_proj_update, bond field, submatrix-LR flavour
 * (src/dqmc_config_v/dqmc_proj_update_submatrix_LR.f90:1-298): windows of
 * nustock = nublock rows; per window Rrows = UR(rows,:) ULRINV and
 * Felms = Rrows UL(:,rows) by GEMM, the accept test on
 * F_rr - F_rA Gamma F_Ar with Gamma bordered per accepted bond, and the flush
 * ULRINV -= (ULRINV UL(:,A)) (Gamma Rrows(A,:)), UR(A,:) *= 1 + Delta. */
static void proj_update_v_lr(orc_chain *c, int nt, int nf) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, ne = m->ne, nnf = L->nn_nf, lf = L->nn_lf;
    int nus = m->nublock > 1 ? m->nublock : 2;
    nus -= nus % 2;
    int32_t *cf = c->vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    zc *urP = zalloc((size_t)nus * ne), *ulP = zalloc((size_t)ne * nus), *Rrows = zalloc((size_t)nus * ne);
    zc *Felms = zalloc((size_t)nus * nus), *Gam = zalloc((size_t)nus * nus);
    zc *Vmat = zalloc((size_t)nus * ne), *Umat = zalloc((size_t)ne * nus);
    zc *Vtmp = zalloc((size_t)nus * ne), *Utmp = zalloc((size_t)ne * nus);
    zc *ikk = zalloc((size_t)nus * 2), *kik = zalloc((size_t)2 * nus), *Gtmp = zalloc((size_t)nus * nus);
    int *xvec = calloc(nus, sizeof(int)), *svec = calloc(nus, sizeof(int));
    zc *dvec = zalloc(nus);
    double accm = 0.0;
    int ik = 0, istk_s = 0, istk_e = -1, nstk = 0;
    for (int b = 0; b < lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * 1);
        int isp = (is + iflip - 1) % 2 + 1;
        if (nstk == 0) {
            int nup = nus < (lf - b) * 2 ? nus : (lf - b) * 2;
            for (int k = 0; k < nup / 2; ++k) {
                int j1 = L->nnlf_list[b + k] - 1, j2 = L->nnlist[j1 * nnf + nf - 1] - 1;
                for (int l = 0; l < ne; ++l) {
                    ulP[ZIDX(l, 2 * k, ne)] = c->UL[ZIDX(l, j1, ne)];
                    ulP[ZIDX(l, 2 * k + 1, ne)] = c->UL[ZIDX(l, j2, ne)];
                    urP[ZIDX(2 * k, l, nus)] = c->UR[ZIDX(j1, l, N)];
                    urP[ZIDX(2 * k + 1, l, nus)] = c->UR[ZIDX(j2, l, N)];
                }
            }
            orc_zgemm('N', 'N', nup, ne, ne, 1.0, urP, nus, c->ULRINV, ne, 0.0, Rrows, nus);
            orc_zgemm('N', 'N', nup, nup, ne, 1.0, Rrows, nus, ulP, ne, 0.0, Felms, nus);
            istk_s = b; istk_e = b + nup / 2 - 1; nstk = nup / 2;
        }
        int s1 = (b - istk_s) * 2, s2 = s1 + 1;
        zc v[4];   /* vukmat column-major: v[0]=(1,1) v[1]=(2,1) v[2]=(1,2) v[3]=(2,2) */
        v[0] = Felms[ZIDX(s1, s1, nus)]; v[1] = Felms[ZIDX(s2, s1, nus)];
        v[2] = Felms[ZIDX(s1, s2, nus)]; v[3] = Felms[ZIDX(s2, s2, nus)];
        if (ik > 0) {
            /* ikktmp = Gamma F(A, r) ; vukmat -= F(r, A) ikktmp */
            for (int cc = 0; cc < 2; ++cc)
                for (int x = 0; x < ik; ++x) {
                    zc sacc = 0;
                    for (int y = 0; y < ik; ++y) sacc += Gam[ZIDX(x, y, nus)] * Felms[ZIDX(svec[y], s1 + cc, nus)];
                    ikk[ZIDX(x, cc, nus)] = sacc;
                }
            for (int rr = 0; rr < 2; ++rr)
                for (int cc = 0; cc < 2; ++cc) {
                    zc sacc = 0;
                    for (int x = 0; x < ik; ++x) sacc += Felms[ZIDX(s1 + rr, svec[x], nus)] * ikk[ZIDX(x, cc, nus)];
                    v[rr + 2 * cc] -= sacc;
                }
        }
        zc dp = m->vdp[is - 1], dm = m->vdm[is - 1];
        v[0] = 1.0 + v[0] * dp; v[1] = v[1] * dp; v[2] = v[2] * dm; v[3] = 1.0 + v[3] * dm;
        zc ratio1 = v[0] * v[3] - v[2] * v[1];
        zc ratiotot = ratio1;
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            zc gk[4];   /* Gammainv_kk column-major */
            gk[0] = v[3] * dp / ratio1; gk[2] = -v[2] * dp / ratio1;
            gk[1] = -v[1] * dm / ratio1; gk[3] = v[0] * dm / ratio1;
            if (ik > 0) {
                /* kiktmp = F(r, A) Gamma */
                for (int rr = 0; rr < 2; ++rr)
                    for (int y = 0; y < ik; ++y) {
                        zc sacc = 0;
                        for (int x = 0; x < ik; ++x) sacc += Felms[ZIDX(s1 + rr, svec[x], nus)] * Gam[ZIDX(x, y, nus)];
                        kik[ZIDX(rr, y, 2)] = sacc;
                    }
                /* new row block -gk kik, new column block -ikk gk, Gamma_AA += ikk gk kik */
                for (int rr = 0; rr < 2; ++rr)
                    for (int y = 0; y < ik; ++y)
                        Gam[ZIDX(ik + rr, y, nus)] = -(gk[rr] * kik[ZIDX(0, y, 2)] + gk[rr + 2] * kik[ZIDX(1, y, 2)]);
                for (int x = 0; x < ik; ++x)
                    for (int cc = 0; cc < 2; ++cc)
                        Gam[ZIDX(x, ik + cc, nus)] = -(ikk[ZIDX(x, 0, nus)] * gk[2 * cc] + ikk[ZIDX(x, 1, nus)] * gk[1 + 2 * cc]);
                for (int y = 0; y < ik; ++y)
                    for (int x = 0; x < ik; ++x)
                        Gam[ZIDX(x, y, nus)] -= ikk[ZIDX(x, 0, nus)] * Gam[ZIDX(ik, y, nus)] + ikk[ZIDX(x, 1, nus)] * Gam[ZIDX(ik + 1, y, nus)];
            }
            Gam[ZIDX(ik, ik, nus)] = gk[0]; Gam[ZIDX(ik + 1, ik, nus)] = gk[1];
            Gam[ZIDX(ik, ik + 1, nus)] = gk[2]; Gam[ZIDX(ik + 1, ik + 1, nus)] = gk[3];
            xvec[ik] = i1; xvec[ik + 1] = i2;
            svec[ik] = s1; svec[ik + 1] = s2;
            dvec[ik] = dp; dvec[ik + 1] = dm;
            for (int l = 0; l < ne; ++l) {
                Vmat[ZIDX(ik, l, nus)] = Rrows[ZIDX(s1, l, nus)];
                Vmat[ZIDX(ik + 1, l, nus)] = Rrows[ZIDX(s2, l, nus)];
                Umat[ZIDX(l, ik, ne)] = ulP[ZIDX(l, s1, ne)];
                Umat[ZIDX(l, ik + 1, ne)] = ulP[ZIDX(l, s2, ne)];
            }
            ik += 2;
            cf[b] = isp;
        }
        if (b == istk_e || b == lf - 1) {
            if (ik > 0) {
                orc_zgemm('N', 'N', ik, ne, ik, 1.0, Gam, nus, Vmat, nus, 0.0, Vtmp, nus);
                orc_zgemm('N', 'N', ne, ik, ne, 1.0, c->ULRINV, ne, Umat, ne, 0.0, Utmp, ne);
                orc_zgemm('N', 'N', ne, ne, ik, -1.0, Utmp, ne, Vtmp, nus, 1.0, c->ULRINV, ne);
                for (int k = 0; k < ik; ++k)
                    for (int l = 0; l < ne; ++l)
                        c->UR[ZIDX(xvec[k], l, N)] += dvec[k] * c->UR[ZIDX(xvec[k], l, N)];
            }
            ik = 0; nstk = 0;
            memset(Gam, 0, sizeof(zc) * (size_t)nus * nus);
        }
    }
    c->acc_v += accm;
    c->prop_v += lf;
    free(urP); free(ulP); free(Rrows); free(Felms); free(Gam); free(Vmat); free(Umat); free(Vtmp); free(Utmp);
    free(ikk); free(kik); free(Gtmp); free(xvec); free(svec); free(dvec);
}

/* dqmc_proj_update, site field (src/dqmc_config_u/dqmc_proj_update.f90:1-92) */
static void proj_update_u(orc_chain *c, int nt) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, lc = m->lcomp;
    int32_t *cf = c->conf + (size_t)(nt - 1) * N;
    zc *vk_tmp = zalloc(ne), *vk = zalloc(ne), *uk = zalloc(ne), *lruk = zalloc(ne);
    double accm = 0.0;
    for (int i = 0; i < N; ++i) {
        int is = cf[i];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        zc d = m->delta[(is - 1) * (lc - 1) + iflip - 1];
        for (int l = 0; l < ne; ++l) { vk_tmp[l] = d * c->UR[ZIDX(i, l, N)]; uk[l] = c->UL[ZIDX(l, i, ne)]; }
        for (int l = 0; l < ne; ++l) {
            zc s = 0;
            for (int k = 0; k < ne; ++k) s += vk_tmp[k] * c->ULRINV[ZIDX(k, l, ne)];
            vk[l] = s;
        }
        zc ratio1 = 1.0;
        for (int l = 0; l < ne; ++l) ratio1 += vk[l] * uk[l];
        zc sscl = 1.0 / ratio1;
        zc ratiotot = orc_total_ratio(m, ratio1, is, iflip, isp);
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            for (int l = 0; l < ne; ++l) c->UR[ZIDX(i, l, N)] += vk_tmp[l];
            for (int l = 0; l < ne; ++l) {
                zc s = 0;
                for (int k = 0; k < ne; ++k) s += c->ULRINV[ZIDX(l, k, ne)] * uk[k];
                lruk[l] = s;
            }
            for (int k = 0; k < ne; ++k) {
                zc w = sscl * vk[k];
                for (int l = 0; l < ne; ++l) c->ULRINV[ZIDX(l, k, ne)] -= lruk[l] * w;
            }
            cf[i] = isp;
        }
    }
    c->acc_u += accm;
    c->prop_u += N;
    free(vk_tmp); free(vk); free(uk); free(lruk);
}

/* G = I - UR (ULRINV UL) of the current walker (gmmat of the delayed updates) */
static void proj_gmat(const orc_chain *c, zc *gm) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne;
    zc *lu = zalloc((size_t)ne * N);
    orc_zgemm('N', 'N', ne, N, ne, 1.0, c->ULRINV, ne, c->UL, ne, 0.0, lu, ne);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) gm[ZIDX(i, j, N)] = (i == j) ? 1.0 : 0.0;
    orc_zgemm('N', 'N', N, N, ne, -1.0, c->UR, N, lu, ne, 1.0, gm, N);
    free(lu);
}

/* end of a delayed or submatrix-G sweep over one family: UR = urrecord and
 * ULRINV = (UL UR)^-1 by LU (s_invlu_z) */
static void proj_close(orc_chain *c, const zc *urrecord) {
    const orc_model *m = c->m;
    memcpy(c->UR, urrecord, sizeof(zc) * (size_t)m->ndim * m->ne);
    ulr_inverse(m->ndim, m->ne, c->UL, c->UR, c->ULRINV, NULL);
}

/* dqmc_proj_update, site field, delayed flavour
 * (src/dqmc_config_u/dqmc_proj_update_delay.f90): rank-1 changes of G are
 * carried in avec/bvec and flushed every nublock accepts, the diagonal of G
 * is tracked, UR rows are scaled per accept, and ULRINV is rebuilt at the end */
static void proj_update_u_delay(orc_chain *c, int nt) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, lc = m->lcomp, nb = m->nublock > 0 ? m->nublock : 1;
    int32_t *cf = c->conf + (size_t)(nt - 1) * N;
    zc *gm = zalloc((size_t)N * N), *av = zalloc((size_t)N * nb), *bv = zalloc((size_t)N * nb);
    zc *dg = zalloc(N), *urr = zalloc((size_t)N * ne);
    memcpy(urr, c->UR, sizeof(zc) * (size_t)N * ne);
    proj_gmat(c, gm);
    for (int i = 0; i < N; ++i) dg[i] = gm[ZIDX(i, i, N)];
    double accm = 0.0;
    int ik = 0;
    for (int i = 0; i < N; ++i) {
        int is = cf[i];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        zc d = m->delta[(is - 1) * (lc - 1) + iflip - 1];
        zc ratio1 = (1.0 - dg[i]) * d + 1.0;
        zc sscl = d / ratio1;
        zc ratiotot = orc_total_ratio(m, ratio1, is, iflip, isp);
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            zc *a = av + (size_t)ik * N, *b = bv + (size_t)ik * N;
            for (int r = 0; r < N; ++r) { a[r] = gm[ZIDX(r, i, N)]; b[r] = gm[ZIDX(i, r, N)]; }
            for (int q = 0; q < ik; ++q) {
                zc bq = bv[(size_t)q * N + i], aq = av[(size_t)q * N + i];
                for (int r = 0; r < N; ++r) {
                    a[r] += bq * av[(size_t)q * N + r];
                    b[r] += aq * bv[(size_t)q * N + r];
                }
            }
            for (int r = 0; r < N; ++r) a[r] *= sscl;
            b[i] -= 1.0;
            for (int r = 0; r < N; ++r) dg[r] += a[r] * b[r];
            for (int l = 0; l < ne; ++l) urr[ZIDX(i, l, N)] += d * urr[ZIDX(i, l, N)];
            cf[i] = isp;
            ++ik;
        }
        if (ik == nb && i < N - 1) {
            orc_zgemm('N', 'T', N, N, nb, 1.0, av, N, bv, N, 1.0, gm, N);
            for (int r = 0; r < N; ++r) dg[r] = gm[ZIDX(r, r, N)];
            memset(av, 0, sizeof(zc) * (size_t)N * nb);
            memset(bv, 0, sizeof(zc) * (size_t)N * nb);
            ik = 0;
        }
    }
    proj_close(c, urr);
    c->acc_u += accm;
    c->prop_u += N;
    free(gm); free(av); free(bv); free(dg); free(urr);
}

/* dqmc_proj_update, bond field, delayed flavour
 * (src/dqmc_config_v/dqmc_proj_update_delay.f90): per accepted bond two
 * delayed columns avec = [G(:,i1) G(:,i2)] S and bvec = [G(i1,:) G(i2,:)]^T - e,
 * S = diag(dp, dm) (I + vukmat)^-1, flushed every nublock columns */
static void proj_update_v_delay(orc_chain *c, int nt, int nf) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, ne = m->ne, nnf = L->nn_nf, lf = L->nn_lf;
    int nb = m->nublock > 1 ? m->nublock : 2;
    nb -= nb % 2;
    int32_t *cf = c->vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    zc *gm = zalloc((size_t)N * N), *av = zalloc((size_t)N * nb), *bv = zalloc((size_t)N * nb);
    zc *g1 = zalloc(N), *g2 = zalloc(N), *urr = zalloc((size_t)N * ne);
    memcpy(urr, c->UR, sizeof(zc) * (size_t)N * ne);
    proj_gmat(c, gm);
    double accm = 0.0;
    int ik = 0;
    for (int b = 0; b < lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * 1);
        int isp = (is + iflip - 1) % 2 + 1;
        zc gp[4];   /* gpart column-major: (1,1) (2,1) (1,2) (2,2) */
        gp[0] = gm[ZIDX(i1, i1, N)]; gp[1] = gm[ZIDX(i2, i1, N)];
        gp[2] = gm[ZIDX(i1, i2, N)]; gp[3] = gm[ZIDX(i2, i2, N)];
        for (int q = 0; q < ik; ++q) {
            const zc *a = av + (size_t)q * N, *bb = bv + (size_t)q * N;
            gp[0] += a[i1] * bb[i1]; gp[2] += a[i1] * bb[i2];
            gp[1] += a[i2] * bb[i1]; gp[3] += a[i2] * bb[i2];
        }
        zc dp = m->vdp[is - 1], dm = m->vdm[is - 1];
        zc v[4];
        v[0] = (1.0 - gp[0]) * dp + 1.0; v[2] = -gp[2] * dm;
        v[1] = -gp[1] * dp;              v[3] = (1.0 - gp[3]) * dm + 1.0;
        zc ratio1 = v[0] * v[3] - v[2] * v[1];
        zc inv[4] = {v[3] / ratio1, -v[1] / ratio1, -v[2] / ratio1, v[0] / ratio1};
        zc sm[4];   /* smat = diag(dp, dm) inv */
        sm[0] = dp * inv[0]; sm[2] = dp * inv[2];
        sm[1] = dm * inv[1]; sm[3] = dm * inv[3];
        zc ratiotot = ratio1;
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            zc *b1 = bv + (size_t)ik * N, *b2 = bv + (size_t)(ik + 1) * N;
            for (int r = 0; r < N; ++r) {
                g1[r] = gm[ZIDX(r, i1, N)]; g2[r] = gm[ZIDX(r, i2, N)];
                b1[r] = gm[ZIDX(i1, r, N)]; b2[r] = gm[ZIDX(i2, r, N)];
            }
            b1[i1] = gm[ZIDX(i1, i1, N)] - 1.0;
            b2[i2] = gm[ZIDX(i2, i2, N)] - 1.0;
            for (int q = 0; q < ik; ++q) {
                const zc *a = av + (size_t)q * N, *bb = bv + (size_t)q * N;
                zc bq1 = bb[i1], bq2 = bb[i2], aq1 = a[i1], aq2 = a[i2];
                for (int r = 0; r < N; ++r) {
                    g1[r] += a[r] * bq1;
                    g2[r] += a[r] * bq2;
                    b1[r] += aq1 * bb[r];
                    b2[r] += aq2 * bb[r];
                }
            }
            zc *a1 = av + (size_t)ik * N, *a2 = av + (size_t)(ik + 1) * N;
            for (int r = 0; r < N; ++r) {
                a1[r] = g1[r] * sm[0] + g2[r] * sm[1];
                a2[r] = g1[r] * sm[2] + g2[r] * sm[3];
            }
            for (int l = 0; l < ne; ++l) {
                urr[ZIDX(i1, l, N)] += dp * urr[ZIDX(i1, l, N)];
                urr[ZIDX(i2, l, N)] += dm * urr[ZIDX(i2, l, N)];
            }
            cf[b] = isp;
            ik += 2;
        }
        if (ik == nb && b < lf - 1) {
            orc_zgemm('N', 'T', N, N, nb, 1.0, av, N, bv, N, 1.0, gm, N);
            memset(av, 0, sizeof(zc) * (size_t)N * nb);
            memset(bv, 0, sizeof(zc) * (size_t)N * nb);
            ik = 0;
        }
    }
    proj_close(c, urr);
    c->acc_v += accm;
    c->prop_v += lf;
    free(gm); free(av); free(bv); free(g1); free(g2); free(urr);
}

/* dqmc_proj_update, site field, submatrix-G flavour
 * (src/dqmc_config_u/dqmc_proj_update_submatrix_G.f90): F = UR ULRINV UL,
 * the ratio from F(i,i) - F(i,A) Gammainv F(A,i), Gammainv bordered per accept,
 * F -= F(:,A) Gammainv F(A,:) every nublock accepts */
static void proj_update_u_subg(orc_chain *c, int nt) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, lc = m->lcomp, nb = m->nublock > 0 ? m->nublock : 1;
    int32_t *cf = c->conf + (size_t)(nt - 1) * N;
    zc *F = zalloc((size_t)N * N), *gi = zalloc((size_t)nb * nb), *cv = zalloc(nb), *bvv = zalloc(nb);
    zc *v1 = zalloc(nb), *v4 = zalloc(nb), *t1 = zalloc((size_t)N * nb), *t2 = zalloc((size_t)nb * N);
    zc *G1 = zalloc((size_t)N * nb), *urr = zalloc((size_t)N * ne);
    int *pv = calloc(nb, sizeof(int));
    memcpy(urr, c->UR, sizeof(zc) * (size_t)N * ne);
    proj_gmat(c, F);
    for (int j = 0; j < N; ++j)          /* F = I - G */
        for (int i = 0; i < N; ++i) F[ZIDX(i, j, N)] = (i == j ? 1.0 : 0.0) - F[ZIDX(i, j, N)];
    double accm = 0.0;
    int ik = 0;
    for (int i = 0; i < N; ++i) {
        int is = cf[i];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        zc d = m->delta[(is - 1) * (lc - 1) + iflip - 1];
        for (int q = 0; q < ik; ++q) { cv[q] = F[ZIDX(i, pv[q], N)]; bvv[q] = F[ZIDX(pv[q], i, N)]; }
        zc v = 0.0;
        for (int q = 0; q < ik; ++q) {
            zc s2 = 0.0;
            for (int r = 0; r < ik; ++r) s2 += cv[r] * gi[ZIDX(r, q, nb)];
            v1[q] = s2;
        }
        for (int q = 0; q < ik; ++q) v += v1[q] * bvv[q];
        zc v2 = F[ZIDX(i, i, N)] - v;
        zc ratio1 = v2 * d + 1.0;
        zc ratiotot = orc_total_ratio(m, ratio1, is, iflip, isp);
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            zc v3 = 1.0 / (-v + 1.0 / d + F[ZIDX(i, i, N)]);
            for (int q = 0; q < ik; ++q) {
                zc s2 = 0.0;
                for (int r = 0; r < ik; ++r) s2 += gi[ZIDX(q, r, nb)] * bvv[r];
                v4[q] = s2;
            }
            for (int q = 0; q < ik; ++q) {
                gi[ZIDX(ik, q, nb)] = -v3 * v1[q];
                gi[ZIDX(q, ik, nb)] = -v4[q] * v3;
            }
            for (int r = 0; r < ik; ++r)
                for (int q = 0; q < ik; ++q) gi[ZIDX(q, r, nb)] += v4[q] * v3 * v1[r];
            gi[ZIDX(ik, ik, nb)] = v3;
            pv[ik] = i;
            for (int l = 0; l < ne; ++l) urr[ZIDX(i, l, N)] += d * urr[ZIDX(i, l, N)];
            for (int r = 0; r < N; ++r) { t1[ZIDX(r, ik, N)] = F[ZIDX(r, i, N)]; t2[ZIDX(ik, r, nb)] = F[ZIDX(i, r, N)]; }
            cf[i] = isp;
            ++ik;
        }
        if (ik == nb && i < N - 1) {
            orc_zgemm('N', 'N', N, nb, ik, 1.0, t1, N, gi, nb, 0.0, G1, N);
            orc_zgemm('N', 'N', N, N, ik, -1.0, G1, N, t2, nb, 1.0, F, N);
            memset(gi, 0, sizeof(zc) * (size_t)nb * nb);
            ik = 0;
        }
    }
    proj_close(c, urr);
    c->acc_u += accm;
    c->prop_u += N;
    free(F); free(gi); free(cv); free(bvv); free(v1); free(v4); free(t1); free(t2); free(G1); free(urr); free(pv);
}

/* dqmc_proj_update, bond field, submatrix-G flavour
 * (src/dqmc_config_v/dqmc_proj_update_submatrix_G.f90): the site-field scheme
 * with 2 x 2 blocks per bond (rows/columns i1, i2).  exact = 0 inverts the
 * accepted bond's 2 x 2 block v5 = [[a, b], [c, d]] with the reference's
 * expressions (submatrix_G.f90 v3(:,:)), whose (2,1) entry
 * -(1/a) c / (a - c b / d) equals the true -c / (ad - bc) only when a = d;
 * exact = 1 uses the true inverse, which is what the fast, delayed and
 * submatrix-LR flavours (and the GPU) amount to. */
static void proj_update_v_subg(orc_chain *c, int nt, int nf, int exact) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, ne = m->ne, nnf = L->nn_nf, lf = L->nn_lf;
    int nb = m->nublock > 1 ? m->nublock : 2;
    nb -= nb % 2;
    int32_t *cf = c->vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    zc *F = zalloc((size_t)N * N), *gi = zalloc((size_t)nb * nb), *cv = zalloc(2 * (size_t)nb), *bvv = zalloc(2 * (size_t)nb);
    zc *v1 = zalloc(2 * (size_t)nb), *v4 = zalloc(2 * (size_t)nb), *t1 = zalloc((size_t)N * nb), *t2 = zalloc((size_t)nb * N);
    zc *G1 = zalloc((size_t)N * nb), *urr = zalloc((size_t)N * ne);
    int *pv = calloc(nb, sizeof(int));
    memcpy(urr, c->UR, sizeof(zc) * (size_t)N * ne);
    proj_gmat(c, F);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) F[ZIDX(i, j, N)] = (i == j ? 1.0 : 0.0) - F[ZIDX(i, j, N)];
    double accm = 0.0;
    int ik = 0;
    for (int b = 0; b < lf; ++b) {
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * nnf + nf - 1] - 1;
        int is = cf[b];
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * 1);
        int isp = (is + iflip - 1) % 2 + 1;
        const int ii[2] = {i1, i2};
        /* cvec (2 x ik) = F(ii, A), bvec (ik x 2) = F(A, ii) */
        for (int q = 0; q < ik; ++q)
            for (int x = 0; x < 2; ++x) { cv[ZIDX(x, q, 2)] = F[ZIDX(ii[x], pv[q], N)]; bvv[ZIDX(q, x, nb)] = F[ZIDX(pv[q], ii[x], N)]; }
        /* v1 = cvec Gammainv (2 x ik), v = v1 bvec (2 x 2) */
        for (int q = 0; q < ik; ++q)
            for (int x = 0; x < 2; ++x) {
                zc s2 = 0.0;
                for (int r = 0; r < ik; ++r) s2 += cv[ZIDX(x, r, 2)] * gi[ZIDX(r, q, nb)];
                v1[ZIDX(x, q, 2)] = s2;
            }
        zc v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int y = 0; y < 2; ++y)
            for (int x = 0; x < 2; ++x)
                for (int q = 0; q < ik; ++q) v[x + 2 * y] += v1[ZIDX(x, q, 2)] * bvv[ZIDX(q, y, nb)];
        zc dp = m->vdp[is - 1], dm = m->vdm[is - 1];
        zc w2[4];
        w2[0] = dp * (-v[0] + F[ZIDX(i1, i1, N)]) + 1.0; w2[2] = dm * (-v[2] + F[ZIDX(i1, i2, N)]);
        w2[1] = dp * (-v[1] + F[ZIDX(i2, i1, N)]);       w2[3] = dm * (-v[3] + F[ZIDX(i2, i2, N)]) + 1.0;
        zc ratio1 = w2[0] * w2[3] - w2[2] * w2[1];
        zc ratiotot = ratio1;
        double ratio_re = creal(ratiotot * c->phase) / creal(c->phase);
        double ratio_abs = ratio_re < 0 ? -ratio_re : ratio_re;
        double random = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, ratio_abs, random);
        if (ratio_abs > random) {
            accm += 1.0;
            double weight = sqrt(creal(ratiotot * conj(ratiotot)));
            c->phase = c->phase * ratiotot / weight;
            /* v5 = diag(1/dp, 1/dm) + F(ii,ii) - v; v3 = v5^-1 by the reference's
             * block formulas */
            zc v5[4];
            v5[0] = 1.0 / dp + F[ZIDX(i1, i1, N)] - v[0]; v5[2] = F[ZIDX(i1, i2, N)] - v[2];
            v5[1] = F[ZIDX(i2, i1, N)] - v[1];           v5[3] = 1.0 / dm + F[ZIDX(i2, i2, N)] - v[3];
            zc v3[4];
            zc s11 = 1.0 / v5[0], s22 = 1.0 / v5[3];
            zc sc1 = 1.0 / (v5[3] - s11 * v5[2] * v5[1]);
            zc sc2 = 1.0 / (v5[0] - s22 * v5[1] * v5[2]);
            v3[0] = s11 + s11 * v5[2] * sc1 * s11 * v5[1];
            v3[2] = -s11 * v5[2] * sc1;
            v3[1] = -s11 * v5[1] * sc2;
            v3[3] = sc1;
            if (exact) {
                zc det5 = v5[0] * v5[3] - v5[2] * v5[1];
                v3[0] = v5[3] / det5; v3[2] = -v5[2] / det5;
                v3[1] = -v5[1] / det5; v3[3] = v5[0] / det5;
            }
            /* v4 = Gammainv bvec (ik x 2) with the old Gammainv */
            for (int y = 0; y < 2; ++y)
                for (int q = 0; q < ik; ++q) {
                    zc s2 = 0.0;
                    for (int r = 0; r < ik; ++r) s2 += gi[ZIDX(q, r, nb)] * bvv[ZIDX(r, y, nb)];
                    v4[ZIDX(q, y, nb)] = s2;
                }
            const int n0 = ik;
            for (int y = 0; y < 2; ++y)
                for (int x = 0; x < 2; ++x) gi[ZIDX(n0 + x, n0 + y, nb)] = v3[x + 2 * y];
            for (int q = 0; q < n0; ++q)
                for (int x = 0; x < 2; ++x) {
                    gi[ZIDX(n0 + x, q, nb)] = -(v3[x] * v1[ZIDX(0, q, 2)] + v3[x + 2] * v1[ZIDX(1, q, 2)]);
                    gi[ZIDX(q, n0 + x, nb)] = -(v4[ZIDX(q, 0, nb)] * v3[2 * x] + v4[ZIDX(q, 1, nb)] * v3[1 + 2 * x]);
                }
            for (int r = 0; r < n0; ++r)
                for (int q = 0; q < n0; ++q)
                    gi[ZIDX(q, r, nb)] -= v4[ZIDX(q, 0, nb)] * gi[ZIDX(n0, r, nb)] + v4[ZIDX(q, 1, nb)] * gi[ZIDX(n0 + 1, r, nb)];
            pv[n0] = i1; pv[n0 + 1] = i2;
            for (int l = 0; l < ne; ++l) {
                urr[ZIDX(i1, l, N)] += dp * urr[ZIDX(i1, l, N)];
                urr[ZIDX(i2, l, N)] += dm * urr[ZIDX(i2, l, N)];
            }
            for (int r = 0; r < N; ++r)
                for (int x = 0; x < 2; ++x) {
                    t1[ZIDX(r, n0 + x, N)] = F[ZIDX(r, ii[x], N)];
                    t2[ZIDX(n0 + x, r, nb)] = F[ZIDX(ii[x], r, N)];
                }
            cf[b] = isp;
            ik += 2;
        }
        if (ik == nb && b < lf - 1) {
            orc_zgemm('N', 'N', N, nb, ik, 1.0, t1, N, gi, nb, 0.0, G1, N);
            orc_zgemm('N', 'N', N, N, ik, -1.0, G1, N, t2, nb, 1.0, F, N);
            memset(gi, 0, sizeof(zc) * (size_t)nb * nb);
            ik = 0;
        }
    }
    proj_close(c, urr);
    c->acc_v += accm;
    c->prop_v += lf;
    free(F); free(gi); free(cv); free(bvv); free(v1); free(v4); free(t1); free(t2); free(G1); free(urr); free(pv);
}

/* the build's update flavour: -DSUBMATRIX selects the submatrix-LR bond
 * update, every other flavour the fast one (same accept sequence) */
static void proj_update_bond(orc_chain *c, int nt, int nf) {
    if (c->m->p.update == ORC_SUBMATRIX) proj_update_v_lr(c, nt, nf);
    else proj_update_v(c, nt, nf);
}

void orc_proj_update(orc_chain *c, int nt, int nf) {
    if (nf > 0) proj_update_bond(c, nt, nf);
    else proj_update_u(c, nt);
}

void orc_proj_update_flavour(orc_chain *c, int nt, int nf, int flavour) {
    if (nf > 0) {
        if (flavour == ORC_SUBMATRIX) proj_update_v_lr(c, nt, nf);
        else if (flavour == ORC_DELAY) proj_update_v_delay(c, nt, nf);
        else if (flavour == ORC_SUBMATRIX_G) proj_update_v_subg(c, nt, nf, 0);
        else if (flavour == ORC_SUBMATRIX_G_EXACT) proj_update_v_subg(c, nt, nf, 1);
        else proj_update_v(c, nt, nf);
    } else {
        if (flavour == ORC_DELAY) proj_update_u_delay(c, nt);
        else if (flavour == ORC_SUBMATRIX_G || flavour == ORC_SUBMATRIX_G_EXACT) proj_update_u_subg(c, nt);
        else proj_update_u(c, nt);
    }
}

/* h0 half step on UR (left op) and UL (right op), families in order or reversed */
static void h0_pair(orc_chain *c, int lop, int rop, int reversed) {
    const orc_model *m = c->m;
    int ne = m->ne, nnf = m->L.nn_nf;
    if (!m->lwrapT) return;
    if (m->p.kinetic == ORC_CHECKERBOARD) {
        for (int k = 1; k <= nnf; ++k) {
            int nf = reversed ? nnf + 1 - k : k;
            /* the reference applies the UL side first in the b0 sweep and the
             * UR side first in the 0b sweep; the two act on different matrices */
            orc_h0_prop(m, lop, nf, (double *)c->UR, ne);
            orc_h0_prop(m, rop, nf, (double *)c->UL, ne);
        }
    } else {
        orc_h0_prop(m, lop, 0, (double *)c->UR, ne);
        orc_h0_prop(m, rop, 0, (double *)c->UL, ne);
    }
}

/* Bmat_left_forward over slices nt2..nt1 (src/dqmc_proj_core.f90:61-104) on an N x ne matrix */
static void bmat_left_forward_proj(const orc_chain *c, int nt1, int nt2, zc *x) {
    const orc_model *m = c->m;
    int ne = m->ne, nnf = m->L.nn_nf;
    for (int nt = nt2; nt <= nt1; ++nt) {
        if (m->lwrapT) {
            if (m->p.kinetic == ORC_CHECKERBOARD)
                for (int nf = 1; nf <= nnf; ++nf) orc_h0_prop(m, ORC_LEFT_FORWARD, nf, (double *)x, ne);
            else orc_h0_prop(m, ORC_LEFT_FORWARD, 0, (double *)x, ne);
        }
        if (m->lwrapplqu)      /* dqmc_proj_core.f90:89-94 */
            for (int i = 0; i < m->lq; ++i) orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD, i, nt, x, ne);
        if (m->lwrapv)
            for (int nf = 1; nf <= nnf; ++nf) {
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 2, x, ne);
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 1, x, ne);
            }
        if (m->lwrapu) orc_u_prop(m, c->conf, ORC_LEFT_FORWARD, nt, (double *)x, ne);
        if (m->lwrapT) {
            if (m->p.kinetic == ORC_CHECKERBOARD)
                for (int nf = nnf; nf >= 1; --nf) orc_h0_prop(m, ORC_LEFT_FORWARD, nf, (double *)x, ne);
            else orc_h0_prop(m, ORC_LEFT_FORWARD, 0, (double *)x, ne);
        }
    }
}

static int in_mid(const orc_model *m, int nt) {
    int lt = m->ltrot, len = m->obs_mid_len;
    return nt > (lt / 2 - (len + 1) / 2) && nt <= (lt / 2 + len / 2);
}

static void measure_here(orc_chain *c, int nt) {
    const orc_model *m = c->m;
    ulr_inverse(m->ndim, m->ne, c->UL, c->UR, c->ULRINV, NULL);
    orc_proj_green(c);
    orc_measure(c, nt);
}

/* wrap-error bookkeeping of the WRAPERROR blocks, then adopt the new weight */
static void record_proj_wrap(orc_chain *c, const zc *ultmp, const zc *urtmp, zc lw) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne;
    zc *inv = zalloc((size_t)ne * ne), *gtmp = zalloc((size_t)N * N);
    ulr_inverse(N, ne, ultmp, urtmp, inv, NULL);
    proj_green(N, ne, ultmp, urtmp, inv, gtmp);
    double err = orc_compare_max(N, gtmp, c->gf);
    if (err > c->max_wrap_error) c->max_wrap_error = err;
    if (c->trace_g && c->trace_n < c->trace_cap) {
        memcpy(c->trace_g + (size_t)c->trace_n * N * N, gtmp, sizeof(zc) * (size_t)N * N);
        c->trace_err[c->trace_n++] = err;
    }
    zc ph = orc_set_phase(c, lw);
    double pd = cabs(c->phase - ph);
    if (pd > c->max_phasediff) c->max_phasediff = pd;
    c->logcount += 1.0;
    c->avglog10error += log10(err);
    c->avgexpphasediff += exp(pd);
    c->phase = ph;
    c->logweightf = lw;
    free(inv); free(gtmp);
}

/* ------------------------------------------------------------------ */
/* sweeps                                                              */
/* ------------------------------------------------------------------ */

/* dqmc_proj_sweep_start_0b (src/dqmc_proj_core/dqmc_proj_sweep_start_0b.f90:1-48) */
int orc_proj_sweep_start_0b(orc_chain *c) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, nst = m->nst;
    for (int l = 0; l < ne; ++l)
        for (int i = 0; i < N; ++i) {
            c->UR[ZIDX(i, l, N)] = c->projR[ZIDX(i, l, N)];
            c->Pst[nst][ZIDX(i, l, N)] = conj(c->projL[ZIDX(i, l, N)]);
        }
    c->logweightf = 0;
    c->logwDV[0] = 0.0;
    zc *tmp = zalloc((size_t)N * ne);
    for (int n = 1; n <= nst; ++n) {
        bmat_left_forward_proj(c, m->wrap_step[(n - 1) * 2 + 1], m->wrap_step[(n - 1) * 2], c->UR);
        double lw = orc_qr_pqmc(N, ne, c->UR, tmp);
        memcpy(c->UR, tmp, sizeof(zc) * (size_t)N * ne);
        memcpy(c->Pst[n], c->UR, sizeof(zc) * (size_t)N * ne);
        c->logwDV[n] = c->logwDV[n - 1] + lw;
    }
    for (int l = 0; l < ne; ++l)
        for (int i = 0; i < N; ++i) c->UL[ZIDX(l, i, ne)] = conj(c->projL[ZIDX(i, l, N)]);
    zc zlogw;
    ulr_inverse(N, ne, c->UL, c->UR, c->ULRINV, &zlogw);
    c->phase = orc_set_phase(c, zlogw);
    c->logweightf = c->logwDV[nst] + zlogw;
    free(tmp);
    return 0;
}

/* dqmc_proj_sweep_b0 (src/dqmc_proj_core/dqmc_proj_sweep_b0.f90:1-220); nslices
 * limits the sweep to its first nslices time slices (bounded CPU samples). */
int orc_proj_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices);
int orc_proj_sweep_b0(orc_chain *c, int lupdate, int lmeasure) {
    return orc_proj_sweep_b0_slices(c, lupdate, lmeasure, c->m->ltrot);
}
int orc_proj_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, nst = m->nst, nnf = m->L.nn_nf;
    zc *ultmp = zalloc((size_t)N * ne), *urtmp = zalloc((size_t)N * ne), *q = zalloc((size_t)N * ne);
    for (int l = 0; l < ne; ++l)
        for (int i = 0; i < N; ++i) {
            c->UL[ZIDX(l, i, ne)] = conj(c->projL[ZIDX(i, l, N)]);
            c->Pst[0][ZIDX(i, l, N)] = c->projR[ZIDX(i, l, N)];
        }
    for (int nt = m->ltrot; nt >= 1 && nt > m->ltrot - nslices; --nt) {
        if (lmeasure && in_mid(m, nt)) measure_here(c, nt);
        h0_pair(c, ORC_LEFT_BACKWARD, ORC_RIGHT_FORWARD, 0);
        if (m->lwrapu) {
            if (lupdate) proj_update_u(c, nt);
            orc_u_prop(m, c->conf, ORC_RIGHT_FORWARD, nt, (double *)c->UL, ne);
            orc_u_prop(m, c->conf, ORC_LEFT_BACKWARD, nt, (double *)c->UR, ne);
        }
        if (m->lwrapv)
            for (int nf = nnf; nf >= 1; --nf) {
                orc_v_prop(m, c->vconf, ORC_RIGHT_FORWARD, nt, nf, 2, c->UL, ne);
                orc_v_prop(m, c->vconf, ORC_LEFT_BACKWARD, nt, nf, 2, c->UR, ne);
                if (lupdate) proj_update_bond(c, nt, nf);
                orc_v_prop(m, c->vconf, ORC_RIGHT_FORWARD, nt, nf, 1, c->UL, ne);
                orc_v_prop(m, c->vconf, ORC_LEFT_BACKWARD, nt, nf, 1, c->UR, ne);
            }
        if (m->lwrapplqu)      /* dqmc_proj_sweep_b0.f90:91-99 */
            for (int i = m->lq - 1; i >= 0; --i) {
                if (lupdate) orc_plq_proj_update(c, i, nt);
                orc_plq_prop(m, c->conf_plq, ORC_RIGHT_FORWARD, i, nt, c->UL, ne);
                orc_plq_prop(m, c->conf_plq, ORC_LEFT_BACKWARD, i, nt, c->UR, ne);
            }
        h0_pair(c, ORC_LEFT_BACKWARD, ORC_RIGHT_FORWARD, 1);
        if ((m->iwrap_nt[nt - 1] > 0 || m->p.nwrap == 1) || nt == 1) {
            int n = m->iwrap_nt[nt - 1];
            memcpy(urtmp, c->UR, sizeof(zc) * (size_t)N * ne);
            memcpy(ultmp, c->UL, sizeof(zc) * (size_t)N * ne);
            memcpy(c->UR, c->Pst[n], sizeof(zc) * (size_t)N * ne);
            double lwt = orc_qr_pqmc(ne, N, c->UL, q);       /* stablize_b0_qr */
            memcpy(c->UL, q, sizeof(zc) * (size_t)N * ne);
            c->logwDV[n + 1] = (n + 1 == nst) ? lwt : c->logwDV[n + 2] + lwt;
            zc zlogw;
            ulr_inverse(N, ne, c->UL, c->UR, c->ULRINV, &zlogw);
            zc lw = (n == 0) ? c->logwDV[n + 1] + zlogw : c->logwDV[n + 1] + c->logwDV[n] + zlogw;
            orc_proj_green(c);
            record_proj_wrap(c, ultmp, urtmp, lw);
            for (int l = 0; l < ne; ++l)
                for (int i = 0; i < N; ++i) c->Pst[n][ZIDX(i, l, N)] = c->UL[ZIDX(l, i, ne)];
        }
    }
    free(ultmp); free(urtmp); free(q);
    return 0;
}

/* Bmat_left_forward / Bmat_right_backward (src/dqmc_ft_core.f90:70-121, 234-288)
 * over slice nt on an N x N matrix, with the projective runs' bond field
 * (nflag 2, then 1, per family) */
static void bmat_nn(const orc_chain *c, int nt, int left, zc *x) {
    const orc_model *m = c->m;
    int N = m->ndim, nnf = m->L.nn_nf, cb = (m->p.kinetic == ORC_CHECKERBOARD);
    int op = left ? ORC_LEFT_FORWARD : ORC_RIGHT_BACKWARD;
    if (m->lwrapT) {
        if (cb) for (int nf = 1; nf <= nnf; ++nf) orc_h0_prop(m, op, nf, (double *)x, N);
        else orc_h0_prop(m, op, 0, (double *)x, N);
    }
    if (m->lwrapplqu)          /* Bmat_left_forward / Bmat_right_backward: plaquettes ascending */
        for (int i = 0; i < m->lq; ++i) orc_plq_prop(m, c->conf_plq, op, i, nt, x, N);
    if (m->lwrapv)
        for (int nf = 1; nf <= nnf; ++nf) {
            orc_v_prop(m, c->vconf, op, nt, nf, 2, x, N);
            orc_v_prop(m, c->vconf, op, nt, nf, 1, x, N);
        }
    if (m->lwrapu) orc_u_prop(m, c->conf, op, nt, (double *)x, N);
    if (m->lwrapT) {
        if (cb) for (int nf = nnf; nf >= 1; --nf) orc_h0_prop(m, op, nf, (double *)x, N);
        else orc_h0_prop(m, op, 0, (double *)x, N);
    }
}

/* c = a b (N x N) */
static void zmm(int N, const zc *a, const zc *b, zc *c) {
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            zc acc = 0;
            for (int k = 0; k < N; ++k) acc += a[ZIDX(i, k, N)] * b[ZIDX(k, j, N)];
            c[ZIDX(i, j, N)] = acc;
        }
}

/* dqmc_proj_dyn (src/dqmc_proj_core/dqmc_proj_dyn.f90:1-128), called by the 0b
 * sweep at nt = ntauin on copies of UL and UR; Pst holds the b0 sweep's UL^T at
 * the stabilisation points after ntauin.  The reference assumes that ntauin is
 * a stabilisation point; G is computed fresh at ntauin in either case. */
static void proj_dyn(orc_chain *c) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, t0 = m->ntauin, ntdm = m->ntdm;
    size_t NN = (size_t)N * N;
    zc *ul = zalloc((size_t)N * ne), *ur = zalloc((size_t)N * ne), *q = zalloc((size_t)N * ne);
    zc *inv = zalloc((size_t)ne * ne), *gf = zalloc(NN), *gtt = zalloc(NN), *tmp = zalloc(NN);
    memcpy(ul, c->UL, sizeof(zc) * (size_t)N * ne);
    memcpy(ur, c->UR, sizeof(zc) * (size_t)N * ne);
    for (int nt = t0; nt <= t0 + ntdm - 1; ++nt) {
        int ntau = nt - t0;
        if (m->iwrap_nt[nt] > 0 || ntau == 0) {
            if (ntau > 0) {
                int n = m->iwrap_nt[nt];
                for (int l = 0; l < ne; ++l)
                    for (int i = 0; i < N; ++i) ul[ZIDX(l, i, ne)] = c->Pst[n][ZIDX(i, l, N)];
            }
            ulr_inverse(N, ne, ul, ur, inv, NULL);
            proj_green(N, ne, ul, ur, inv, gf);
            if (ntau == 0) {
                memcpy(c->g00, gf, sizeof(zc) * NN);
                memcpy(gtt, gf, sizeof(zc) * NN);
                memcpy(c->gt0, gf, sizeof(zc) * NN);
                memcpy(c->g0t, gf, sizeof(zc) * NN);
                for (int i = 0; i < N; ++i) c->g0t[ZIDX(i, i, N)] -= 1.0;      /* -(1 - G) */
                orc_dyn_measure(c, 1, c->gt0, c->g0t, gtt, c->g00);
            } else {
                double err = orc_compare_max(N, gtt, gf);
                if (err > c->max_dyn_error) c->max_dyn_error = err;
                memcpy(gtt, gf, sizeof(zc) * NN);
                zmm(N, gf, c->gt0, tmp);                                        /* gt0 = G gt0 */
                memcpy(c->gt0, tmp, sizeof(zc) * NN);
                for (size_t e = 0; e < NN; ++e) gf[e] = -gf[e];
                for (int i = 0; i < N; ++i) gf[ZIDX(i, i, N)] += 1.0;           /* 1 - G */
                zmm(N, c->g0t, gf, tmp);                                        /* g0t = g0t (1 - G) */
                memcpy(c->g0t, tmp, sizeof(zc) * NN);
            }
        }
        int nt1 = nt + 1;
        bmat_nn(c, nt1, 1, c->gt0);
        bmat_nn(c, nt1, 0, c->g0t);
        bmat_nn(c, nt1, 0, gtt);
        bmat_nn(c, nt1, 1, gtt);
        orc_dyn_measure(c, nt1 - t0 + 1, c->gt0, c->g0t, gtt, c->g00);
        bmat_left_forward_proj(c, nt1, nt1, ur);
        if (m->iwrap_nt[nt] > 0 && nt1 != t0 + ntdm) {
            orc_qr_pqmc(N, ne, ur, q);                                          /* stablize_0b_qr */
            memcpy(ur, q, sizeof(zc) * (size_t)N * ne);
        }
    }
    free(ul); free(ur); free(q); free(inv); free(gf); free(gtt); free(tmp);
}

/* dqmc_proj_sweep_0b (src/dqmc_proj_core/dqmc_proj_sweep_0b.f90:1-235); with
 * ltau the measured sweep runs the unequal-time pass at nt = ntauin (206-211) */
int orc_proj_sweep_0b(orc_chain *c, int lupdate, int lmeasure) {
    const orc_model *m = c->m;
    int N = m->ndim, ne = m->ne, nst = m->nst, nnf = m->L.nn_nf;
    zc *ultmp = zalloc((size_t)N * ne), *urtmp = zalloc((size_t)N * ne), *q = zalloc((size_t)N * ne);
    for (int l = 0; l < ne; ++l)
        for (int i = 0; i < N; ++i) {
            c->UR[ZIDX(i, l, N)] = c->projR[ZIDX(i, l, N)];
            c->Pst[nst][ZIDX(i, l, N)] = conj(c->projL[ZIDX(i, l, N)]);
        }
    c->logwDV[0] = 0.0;
    for (int nt = 1; nt <= m->ltrot; ++nt) {
        h0_pair(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 0);
        if (m->lwrapplqu)      /* dqmc_proj_sweep_0b.f90:61-68 */
            for (int i = 0; i < m->lq; ++i) {
                orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD, i, nt, c->UR, ne);
                orc_plq_prop(m, c->conf_plq, ORC_RIGHT_BACKWARD, i, nt, c->UL, ne);
                if (lupdate) orc_plq_proj_update(c, i, nt);
            }
        if (m->lwrapv)
            for (int nf = 1; nf <= nnf; ++nf) {
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 2, c->UR, ne);
                orc_v_prop(m, c->vconf, ORC_RIGHT_BACKWARD, nt, nf, 2, c->UL, ne);
                if (lupdate) proj_update_bond(c, nt, nf);
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 1, c->UR, ne);
                orc_v_prop(m, c->vconf, ORC_RIGHT_BACKWARD, nt, nf, 1, c->UL, ne);
            }
        if (m->lwrapu) {
            orc_u_prop(m, c->conf, ORC_LEFT_FORWARD, nt, (double *)c->UR, ne);
            orc_u_prop(m, c->conf, ORC_RIGHT_BACKWARD, nt, (double *)c->UL, ne);
            if (lupdate) proj_update_u(c, nt);
        }
        h0_pair(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 1);
        if (lmeasure && in_mid(m, nt)) measure_here(c, nt);
        if (m->iwrap_nt[nt] > 0) {
            int n = m->iwrap_nt[nt];
            memcpy(ultmp, c->UL, sizeof(zc) * (size_t)N * ne);
            memcpy(urtmp, c->UR, sizeof(zc) * (size_t)N * ne);
            for (int l = 0; l < ne; ++l)
                for (int i = 0; i < N; ++i) c->UL[ZIDX(l, i, ne)] = c->Pst[n][ZIDX(i, l, N)];
            double lwt = orc_qr_pqmc(N, ne, c->UR, q);       /* stablize_0b_qr */
            memcpy(c->UR, q, sizeof(zc) * (size_t)N * ne);
            c->logwDV[n] = c->logwDV[n - 1] + lwt;
            zc zlogw;
            ulr_inverse(N, ne, c->UL, c->UR, c->ULRINV, &zlogw);
            zc lw = (n == nst) ? c->logwDV[n] + zlogw : c->logwDV[n] + c->logwDV[n + 1] + zlogw;
            orc_proj_green(c);
            record_proj_wrap(c, ultmp, urtmp, lw);
            memcpy(c->Pst[n], c->UR, sizeof(zc) * (size_t)N * ne);
        }
        if (m->p.ltau && lmeasure && nt == m->ntauin) proj_dyn(c);
    }
    free(ultmp); free(urtmp); free(q);
    return 0;
}

double orc_qr_pqmc_d(int rdim, int cdim, const double *a, double *q) {
    return orc_qr_pqmc(rdim, cdim, (const zc *)a, (zc *)q);
}
void orc_eig_he_d(int n, const double *h, double *w, double *v) {
    orc_eig_he(n, (const zc *)h, w, (zc *)v);
}
