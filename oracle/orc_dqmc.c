/* Finite-temperature DQMC sweep restated from the Fortran reference.
 * Test infrastructure only (see dqmc_oracle.h).  Each function cites the
 * reference routine it follows. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

static zc *zalloc(size_t n) { zc *p = calloc(n ? n : 1, sizeof(zc)); return p; }

/* ------------------------------------------------------------------ */
/* model: src/model_para.f90:129-474 (make_tables)                     */
/* ------------------------------------------------------------------ */

/* dqmc_set_conf (src/dqmc_config_u/dqmc_set_conf.f90:1-176) */
static void set_hs(orc_model *m) {
    const orc_params *p = &m->p;
    int nflr = p->nflr;
    double u = p->rhub, dtau = p->dtau, nu = p->nu;
    int exact = (p->hs == ORC_HS_EXACT);
    if (p->lproju) {
        m->lcomp = nflr / 2 + 1 + (int)(0.5 * fabs(nu));
    } else if (exact && nflr == 2) {
        m->lcomp = 2;
    } else {
        m->lcomp = 4;
    }
    int use_general = !exact || (nflr != 2 && nflr != 4 && nflr != 6);
    if (!use_general && nflr == 2) {
        m->etal[0] = -1.0; m->etal[1] = 1.0;
        m->hs_alpha = (u >= 0) ? acos(exp(-dtau * fabs(u) * 0.5)) : acosh(exp(dtau * fabs(u) * 0.5));
        m->gaml[0] = m->gaml[1] = 1.0;
    } else if (!use_general) {
        double a = exp(-0.5 * dtau * u);
        double d = sqrt(8.0 + a * a * (3.0 + a * a) * (3.0 + a * a));
        double xp = (a + 2 * a * a * a + a * a * a * a * a + (a * a - 1.0) * d) / 4.0;
        double xm = (a + 2 * a * a * a + a * a * a * a * a - (a * a - 1.0) * d) / 4.0;
        if (u >= 0) { m->etal[0] = -acos(xm); m->etal[1] = -acos(xp); m->etal[2] = acos(xp); m->etal[3] = acos(xm); }
        else { m->etal[0] = -acosh(xm); m->etal[1] = -acosh(xp); m->etal[2] = acosh(xp); m->etal[3] = acosh(xm); }
        m->hs_alpha = 1.0;
        double t = a * (3.0 + a * a);
        m->gaml[0] = (t + d) / d; m->gaml[1] = (-t + d) / d; m->gaml[2] = (-t + d) / d; m->gaml[3] = (t + d) / d;
    } else {
        double s6 = sqrt(6.0);
        m->etal[0] = -sqrt(2.0 * (3.0 + s6)); m->etal[1] = -sqrt(2.0 * (3.0 - s6));
        m->etal[2] = sqrt(2.0 * (3.0 - s6)); m->etal[3] = sqrt(2.0 * (3.0 + s6));
        m->hs_alpha = sqrt(dtau * fabs(u) * 0.5);
        m->gaml[0] = 1.0 - s6 / 3.0; m->gaml[1] = 1.0 + s6 / 3.0; m->gaml[2] = 1.0 + s6 / 3.0; m->gaml[3] = 1.0 - s6 / 3.0;
    }
    int lc = m->lcomp;
    double al = m->hs_alpha;
    for (int is = 1; is <= lc; ++is) {
        if (p->lproju) {
            m->phase[is - 1] = cexp(I * (M_PI * (-2.0 * is) * 0.5 * (nflr + nu) / lc));
            m->bmat[is - 1] = cexp(I * (M_PI * 2.0 * is / lc));
            m->bmat_inv[is - 1] = cexp(-I * (M_PI * 2.0 * is / lc));
        } else if (u >= 0) {
            m->phase[is - 1] = cexp(I * (al * (-m->etal[is - 1]) * 0.5 * (nflr + nu)));
            m->bmat[is - 1] = cexp(I * (al * m->etal[is - 1]));
            m->bmat_inv[is - 1] = cexp(-I * (al * m->etal[is - 1]));
        } else {
            m->phase[is - 1] = exp(al * (-m->etal[is - 1]) * 0.5 * (nflr + nu));
            m->bmat[is - 1] = exp(al * m->etal[is - 1]);
            m->bmat_inv[is - 1] = exp(-al * m->etal[is - 1]);
        }
    }
    for (int is = 1; is <= lc; ++is)
        for (int iflip = 1; iflip <= lc - 1; ++iflip) {
            int isp = (is + iflip - 1) % lc + 1;
            int k = (is - 1) * (lc - 1) + (iflip - 1);
            if (p->lproju) {
                m->phase_ratio[k] = cexp(I * (M_PI * (2.0 * is - 2.0 * isp) * 0.5 * (nflr + nu) / lc));
                m->delta[k] = cexp(I * (M_PI * (2.0 * isp - 2.0 * is) / lc)) - 1.0;
            } else if (u >= 0) {
                m->phase_ratio[k] = cexp(I * (al * (m->etal[is - 1] - m->etal[isp - 1]) * 0.5 * (nflr + nu)));
                m->delta[k] = cexp(I * (al * (m->etal[isp - 1] - m->etal[is - 1]))) - 1.0;
            } else {
                m->phase_ratio[k] = exp(al * (m->etal[is - 1] - m->etal[isp - 1]) * 0.5 * (nflr + nu));
                m->delta[k] = exp(al * (m->etal[isp - 1] - m->etal[is - 1])) - 1.0;
            }
        }
}

/* exp(-s h) for h = [[d, z],[conj z, d]], the closed form of the 2x2
 * eigen-decomposition used by dqmc_set_h0conf.f90:76-123 */
static void exp2x2(double d, zc z, double s, zc out[4]) {
    double az = cabs(z);
    double e = exp(-s * d);
    double ch = cosh(s * az), sh = (az > 0) ? sinh(s * az) / az : 0.0;
    out[0] = e * ch;          /* (1,1) */
    out[1] = -e * sh * z;     /* (1,2) */
    out[2] = -e * sh * conj(z); /* (2,1) */
    out[3] = e * ch;          /* (2,2) */
}

/* In-place 1D DFT of n points with stride st: radix-2 for powers of two,
 * direct sum otherwise; tw[k] = exp(-2 pi i k / n), sign -1 forward. */
static void dft1(zc *x, int n, int st, const zc *tw, int sign, zc *tmp) {
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { zc t = x[i * st]; x[i * st] = x[j * st]; x[j * st] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int s0 = 0; s0 < n; s0 += len)
                for (int k = 0; k < half; ++k) {
                    zc w = tw[k * step];
                    if (sign > 0) w = conj(w);
                    zc u = x[(s0 + k) * st], v = w * x[(s0 + k + half) * st];
                    x[(s0 + k) * st] = u + v;
                    x[(s0 + k + half) * st] = u - v;
                }
        }
    } else {
        for (int k = 0; k < n; ++k) {
            zc acc = 0;
            for (int j = 0; j < n; ++j) {
                zc w = tw[(j * k) % n];
                acc += (sign > 0 ? conj(w) : w) * x[j * st];
            }
            tmp[k] = acc;
        }
        for (int k = 0; k < n; ++k) x[k * st] = tmp[k];
    }
}

/* 2D DFT over (l1, l2) of a length-lq vector, index j1 + l1*j2, scale 1/sqrt(lq) */
static void dft2(const orc_model *m, zc *x, int sign) {
    int l1 = m->p.l1, l2 = m->p.l2, lq = l1 * l2;
    zc tmp[512];
    for (int j2 = 0; j2 < l2; ++j2) dft1(x + l1 * j2, l1, 1, m->tw1, sign, tmp);
    for (int j1 = 0; j1 < l1; ++j1) dft1(x + j1, l2, l1, m->tw2, sign, tmp);
    double sc = 1.0 / sqrt((double)lq);
    for (int k = 0; k < lq; ++k) x[k] *= sc;
}

/* dqmc_set_h0conf.f90 + seth0.f90 */
static void set_h0(orc_model *m) {
    const orc_params *p = &m->p;
    const orc_latt *L = &m->L;
    int N = m->ndim, nf_n = L->nn_nf, lf = L->nn_lf;
    m->h0mat = zalloc((size_t)N * N);
    m->expar_nn = zalloc((size_t)L->nsites * nf_n);
    for (int i = 0; i < L->nsites; ++i)
        for (int nf = 1; nf <= nf_n; ++nf)
            m->expar_nn[i * nf_n + nf - 1] = orc_expar(L, i, nf, p->xmag, p->flux_x, p->flux_y, p->dimer);
    for (int b = 0; b < lf; ++b) {
        int i0 = L->nnlf_list[b] - 1;
        for (int nf = 1; nf <= nf_n; ++nf) {
            int in = L->nnlist[i0 * nf_n + nf - 1] - 1;
            zc z1 = -p->rt * m->expar_nn[i0 * nf_n + nf - 1];
            m->h0mat[ZIDX(i0, in, N)] += z1;
            m->h0mat[ZIDX(in, i0, N)] += conj(z1);
        }
    }
    for (int i = 0; i < L->nsites; ++i) m->h0mat[ZIDX(i, i, N)] -= p->mu;

    if (p->kinetic == ORC_CHECKERBOARD) {
        m->urt = zalloc((size_t)nf_n * lf * 4);
        m->urtm1 = zalloc((size_t)nf_n * lf * 4);
        for (int nf = 1; nf <= nf_n; ++nf)
            for (int iu = 0; iu < lf; ++iu) {
                int ist = iu + (nf - 1) * lf;
                int i0 = L->nnlf_list[iu] - 1;
                /* r_cubic: family 4 hops rtd between the layers (dqmc_set_h0conf.f90:22-73) */
                const double t = (L->kind == ORC_R_CUBIC && nf == 4) ? p->rtd : p->rt;
                zc z = -t * m->expar_nn[i0 * nf_n + nf - 1];
                double d = -p->mu / nf_n;
                exp2x2(d, z, 0.5 * p->dtau, &m->urt[ist * 4]);
                exp2x2(d, z, -0.5 * p->dtau, &m->urtm1[ist * 4]);
            }
    } else if (p->kinetic == ORC_DENSE) {
        /* urt = U exp(-dtau e / 2) U^H, urtm1 = U exp(+dtau e / 2) U^H from the
         * eigen-decomposition of h0mat (dqmc_set_h0conf.f90:484-509) */
        m->urtd = zalloc((size_t)N * N);
        m->urtm1d = zalloc((size_t)N * N);
        double *w = (double *)malloc(sizeof(double) * N);
        zc *u = zalloc((size_t)N * N);
        orc_eig_he(N, m->h0mat, w, u);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                zc z0 = 0, z1 = 0;
                for (int k = 0; k < N; ++k) {
                    zc t = u[ZIDX(i, k, N)] * conj(u[ZIDX(j, k, N)]);
                    z0 += t * exp(-0.5 * p->dtau * w[k]);
                    z1 += t * exp(0.5 * p->dtau * w[k]);
                }
                m->urtd[ZIDX(i, j, N)] = z0;
                m->urtm1d[ZIDX(i, j, N)] = z1;
            }
        free(w); free(u);
    } else {
        /* h0k = diag(F H F^-1) with F the scaled forward DFT over (l1, l2) */
        int lq = m->lq;
        m->tw1 = zalloc(p->l1);
        m->tw2 = zalloc(p->l2);
        for (int k = 0; k < p->l1; ++k) m->tw1[k] = cexp(-I * 2.0 * M_PI * k / p->l1);
        for (int k = 0; k < p->l2; ++k) m->tw2[k] = cexp(-I * 2.0 * M_PI * k / p->l2);
        m->exph0k = zalloc(lq);
        m->exph0kinv = zalloc(lq);
        zc *tmp = zalloc((size_t)lq * lq);
        memcpy(tmp, m->h0mat, sizeof(zc) * lq * lq);
        for (int j = 0; j < lq; ++j) dft2(m, tmp + (size_t)j * lq, -1);     /* F H (columns) */
        zc *row = zalloc(lq);
        for (int i = 0; i < lq; ++i) {                                    /* (F H) F^-1 on rows */
            for (int j = 0; j < lq; ++j) row[j] = tmp[ZIDX(i, j, lq)];
            dft2(m, row, +1);
            for (int j = 0; j < lq; ++j) tmp[ZIDX(i, j, lq)] = row[j];
        }
        for (int i = 0; i < lq; ++i) {
            zc h = tmp[ZIDX(i, i, lq)];
            m->exph0k[i] = cexp(-0.5 * p->dtau * h);
            m->exph0kinv[i] = cexp(0.5 * p->dtau * h);
        }
        free(row); free(tmp);
    }
}

orc_model *orc_model_new(const orc_params *pin) {
    orc_model *m = calloc(1, sizeof(orc_model));
    m->p = *pin;
    orc_params *p = &m->p;
    if (p->lattice != ORC_CUBIC && p->lattice != ORC_R_CUBIC) p->l3 = 1;
    if (orc_latt_build(&m->L, p->lattice, p->l1, p->l2, p->l3) != 0) { free(m); return NULL; }
    p->theta = p->theta * M_PI;
    m->lq = m->L.ncell;
    m->ndim = m->L.nsites;
    m->ne = m->ndim / 2 + (int)(p->nu * m->ndim / 8.0);
    m->ltrot = (int)lround(p->beta / p->dtau);
    m->ntdm = p->ltau ? (int)lround(p->dyntau / p->dtau) : 0;
    if (m->ntdm < 0) m->ntdm = 0;
    m->ntauin = (m->ltrot - m->ntdm) / 2;
    m->lwrapT = (p->rt != 0.0);
    m->lwrapu = (p->rhub != 0.0);
    int N = m->ndim;
    if (p->nublock == 0) {
        if (p->update == ORC_DELAY) {
            int q = N / 5;
            p->nublock = q < 16 ? 4 : q < 32 ? 8 : q < 64 ? 16 : q < 256 ? 32 : 64;
        } else if (p->update == ORC_SUBMATRIX) {
            int q = N / 20;
            p->nublock = q < 32 ? 32 : q < 64 ? 64 : q < 128 ? 16 : q < 256 ? 256 : q < 512 ? 512 : 1024;
        }
    }
    m->nublock = p->nublock;
    int lt = m->ltrot;
    m->iwrap_nt = calloc(lt + 1, sizeof(int));
    if (lt < p->nwrap) p->nwrap = lt;
    if (lt < p->nwrap || !p->lstabilize) {
        m->nst = 0;
    } else if (lt % p->nwrap == 0) {
        m->nst = lt / p->nwrap;
        m->wrap_step = calloc(2 * m->nst, sizeof(int));
        for (int i = 1; i <= m->nst; ++i) {
            m->iwrap_nt[i * p->nwrap] = i;
            m->wrap_step[(i - 1) * 2] = 1 + (i - 1) * p->nwrap;
            m->wrap_step[(i - 1) * 2 + 1] = i * p->nwrap;
        }
    } else {
        m->nst = lt / p->nwrap + 1;
        m->wrap_step = calloc(2 * m->nst, sizeof(int));
        for (int i = 1; i <= m->nst - 1; ++i) {
            m->iwrap_nt[i * p->nwrap] = i;
            m->wrap_step[(i - 1) * 2] = 1 + (i - 1) * p->nwrap;
            m->wrap_step[(i - 1) * 2 + 1] = i * p->nwrap;
        }
        int i = m->nst;
        m->iwrap_nt[lt] = i;
        m->wrap_step[(i - 1) * 2] = (i - 1) * p->nwrap + 1;
        m->wrap_step[(i - 1) * 2 + 1] = lt;
    }
    set_hs(m);
    set_h0(m);
    /* the plaquette field (dqmc_ft_ctrl.f90:19-23, dqmc_proj_ctrl.f90:21-24) */
    m->lwrapplqu = p->rhub_plq != 0.0;
    if (m->lwrapplqu && orc_plq_setup(m) != 0) { orc_model_free(m); return NULL; }
    m->proj = p->proj != 0;
    m->obs_mid_len = p->obs_mid_len > 0 ? p->obs_mid_len : 1;
    orc_set_vconf(m);
    return m;
}

void orc_model_free(orc_model *m) {
    if (!m) return;
    orc_latt_free(&m->L);
    free(m->iwrap_nt); free(m->wrap_step); free(m->urt); free(m->urtm1);
    free(m->exph0k); free(m->exph0kinv); free(m->urtd); free(m->urtm1d); free(m->tw1); free(m->tw2); free(m->h0mat); free(m->expar_nn);
    orc_plq_free(m);
    free(m);
}

void orc_model_dims(const orc_model *m, int32_t out[10]) {
    out[0] = m->ndim; out[1] = m->lq; out[2] = m->ltrot; out[3] = m->nst; out[4] = m->nublock;
    out[5] = m->lcomp; out[6] = m->L.nn_nf; out[7] = m->L.nn_lf; out[8] = m->L.nsub; out[9] = m->L.z_plq;
}

void orc_model_tables(const orc_model *m, int32_t *nnlist, int32_t *nnlf_list, int32_t *list,
                      int32_t *imj, int32_t *plq_cord, int32_t *snlist) {
    const orc_latt *L = &m->L;
    if (nnlist) for (int i = 0; i < L->nsites * L->nn_nf; ++i) nnlist[i] = L->nnlist[i];
    if (nnlf_list) for (int i = 0; i < L->nn_lf; ++i) nnlf_list[i] = L->nnlf_list[i];
    if (list) for (int i = 0; i < L->nsites * 2; ++i) list[i] = L->list[i];
    if (imj) for (int i = 0; i < L->ncell * L->ncell; ++i) imj[i] = L->imj[i];
    if (plq_cord) for (int i = 0; i < L->ncell * L->z_plq; ++i) plq_cord[i] = L->plq_cord[i];
    if (snlist) for (int i = 0; i < L->nsites * L->nsn; ++i) snlist[i] = L->snlist[i];
}

void orc_model_hs(const orc_model *m, double *bmat, double *bmat_inv, double *delta,
                  double *phase, double *phase_ratio, double *gaml, double *etal, double *alpha) {
    int lc = m->lcomp;
    memcpy(bmat, m->bmat, sizeof(zc) * lc);
    memcpy(bmat_inv, m->bmat_inv, sizeof(zc) * lc);
    memcpy(delta, m->delta, sizeof(zc) * lc * (lc - 1));
    memcpy(phase, m->phase, sizeof(zc) * lc);
    memcpy(phase_ratio, m->phase_ratio, sizeof(zc) * lc * (lc - 1));
    memcpy(gaml, m->gaml, sizeof(double) * lc);
    memcpy(etal, m->etal, sizeof(double) * lc);
    *alpha = m->hs_alpha;
}

void orc_model_kinetic(const orc_model *m, double *urt, double *urtm1, double *exph0k, double *exph0kinv) {
    size_t nb = (size_t)m->L.nn_nf * m->L.nn_lf;
    if (m->urt && urt) memcpy(urt, m->urt, sizeof(zc) * nb * 4);
    if (m->urtm1 && urtm1) memcpy(urtm1, m->urtm1, sizeof(zc) * nb * 4);
    if (m->exph0k && exph0k) memcpy(exph0k, m->exph0k, sizeof(zc) * m->lq);
    if (m->exph0kinv && exph0kinv) memcpy(exph0kinv, m->exph0kinv, sizeof(zc) * m->lq);
}

void orc_model_h0mat(const orc_model *m, double *h0) {
    memcpy(h0, m->h0mat, sizeof(zc) * (size_t)m->ndim * m->ndim);
}

/* ------------------------------------------------------------------ */
/* chain                                                               */
/* ------------------------------------------------------------------ */
orc_chain *orc_chain_new(const orc_model *m, int32_t seed, int draw_conf) {
    orc_chain *c = calloc(1, sizeof(orc_chain));
    c->m = m;
    int N = m->ndim, lt = m->ltrot, nst = m->nst, lq = m->lq;
    orc_sfmt_init(&c->rng, seed);
    if (m->lwrapplqu) {       /* dqmc_input_plqconf.f90:53-60, before the U field: nt outer, plaquette inner */
        c->conf_plq = calloc((size_t)lq * lt, sizeof(int32_t));
        for (size_t e = 0; e < (size_t)lq * lt; ++e)
            c->conf_plq[e] = draw_conf ? (int32_t)ceil(orc_sfmt_stream(&c->rng) * m->plq_lcomp) : 1;
    }
    c->conf = calloc((size_t)N * lt, sizeof(int32_t));
    if (draw_conf && m->lwrapu) {  /* dqmc_input_conf.f90:55-63: nt outer, site inner */
        for (int nt = 0; nt < lt; ++nt)
            for (int i = 0; i < N; ++i)
                c->conf[nt * N + i] = (int32_t)ceil(orc_sfmt_stream(&c->rng) * m->lcomp);
    } else {
        for (int i = 0; i < N * lt; ++i) c->conf[i] = 1;
    }
    c->gf = zalloc((size_t)N * N);
    c->gfc = zalloc((size_t)N * N);
    c->Ust = calloc(nst + 1, sizeof(zc *));
    c->Vst = calloc(nst + 1, sizeof(zc *));
    c->Dst = calloc(nst + 1, sizeof(double *));
    c->logdetQst = zalloc(nst + 1);
    for (int n = 0; n <= nst; ++n) {
        c->Ust[n] = zalloc((size_t)N * N);
        c->Vst[n] = zalloc((size_t)N * N);
        c->Dst[n] = calloc(N, sizeof(double));
    }
    c->phase = 1.0;
    if (m->p.ltau) {
        c->g00 = zalloc((size_t)N * N); c->gt0 = zalloc((size_t)N * N); c->g0t = zalloc((size_t)N * N);
        c->znn_tau_bin = zalloc((size_t)lq * 4 * (m->ntdm + 1));
        c->gf_b = zalloc((size_t)N * N);
        c->Ust_b = calloc(nst + 1, sizeof(zc *)); c->Vst_b = calloc(nst + 1, sizeof(zc *));
        c->Dst_b = calloc(nst + 1, sizeof(double *)); c->logdetQst_b = zalloc(nst + 1);
        for (int n = 0; n <= nst; ++n) {
            c->Ust_b[n] = zalloc((size_t)N * N); c->Vst_b[n] = zalloc((size_t)N * N);
            c->Dst_b[n] = calloc(N, sizeof(double));
        }
    }
    c->zcpcm_bin = zalloc(lq * 4); c->zspsm_bin = zalloc(lq * 4);
    c->znn_bin = zalloc(lq * 4); c->pair_onsite_bin = zalloc(lq * 4);
    c->zjj_bin = zalloc(lq); c->zbb_bin = zalloc(lq);
    c->pair_nn_bin = zalloc(lq); c->pair_sn_bin = zalloc(lq);
    orc_proj_chain_init(c, draw_conf);
    return c;
}

void orc_chain_free(orc_chain *c) {
    if (!c) return;
    for (int n = 0; n <= c->m->nst; ++n) { free(c->Ust[n]); free(c->Vst[n]); free(c->Dst[n]); }
    free(c->Ust); free(c->Vst); free(c->Dst); free(c->logdetQst);
    free(c->conf); free(c->conf_plq); free(c->gf); free(c->gfc);
    if (c->m->p.ltau) {
        for (int n = 0; n <= c->m->nst; ++n) { free(c->Ust_b[n]); free(c->Vst_b[n]); free(c->Dst_b[n]); }
        free(c->Ust_b); free(c->Vst_b); free(c->Dst_b); free(c->logdetQst_b); free(c->gf_b);
        free(c->g00); free(c->gt0); free(c->g0t); free(c->znn_tau_bin);
    }
    free(c->zcpcm_bin); free(c->zspsm_bin); free(c->znn_bin); free(c->pair_onsite_bin);
    free(c->zjj_bin); free(c->zbb_bin); free(c->pair_nn_bin); free(c->pair_sn_bin);
    orc_proj_chain_free(c);
    free(c->trace_g); free(c->trace_err);
    free(c);
}

void orc_chain_set_conf(orc_chain *c, const int32_t *conf) {
    memcpy(c->conf, conf, sizeof(int32_t) * (size_t)c->m->ndim * c->m->ltrot);
}
void orc_chain_get_conf(const orc_chain *c, int32_t *conf) {
    memcpy(conf, c->conf, sizeof(int32_t) * (size_t)c->m->ndim * c->m->ltrot);
}
void orc_chain_set_green(orc_chain *c, const double *g) {
    memcpy(c->gf, g, sizeof(zc) * (size_t)c->m->ndim * c->m->ndim);
}
void orc_chain_get_green(const orc_chain *c, double *g) {
    memcpy(g, c->gf, sizeof(zc) * (size_t)c->m->ndim * c->m->ndim);
}
void orc_chain_set_phase(orc_chain *c, double re, double im) { c->phase = re + I * im; }
double orc_chain_uniform(orc_chain *c) { return orc_sfmt_stream(&c->rng); }

void orc_chain_get_diag(const orc_chain *c, double *out) {
    out[0] = creal(c->phase); out[1] = cimag(c->phase);
    out[2] = creal(c->logweightf); out[3] = cimag(c->logweightf);
    out[4] = c->max_wrap_error; out[5] = c->max_phasediff;
    out[6] = c->avglog10error; out[7] = c->logcount;
    out[8] = c->acc_u; out[9] = c->prop_u;
    out[10] = c->acc_v; out[11] = c->prop_v;
    out[12] = c->near_ties;
    out[13] = c->plq_accepted; out[14] = c->plq_proposed;
}

void orc_chain_set_conf_plq(orc_chain *c, const int32_t *conf) {
    if (c->conf_plq) memcpy(c->conf_plq, conf, sizeof(int32_t) * (size_t)c->m->lq * c->m->ltrot);
}
void orc_chain_get_conf_plq(const orc_chain *c, int32_t *conf) {
    if (c->conf_plq) memcpy(conf, c->conf_plq, sizeof(int32_t) * (size_t)c->m->lq * c->m->ltrot);
}

/* trace of (fresh G, wrap error) at the next `cap` recorded wrap checks
 * (cap = 0 stops and frees it) */
void orc_chain_trace(orc_chain *c, int cap) {
    free(c->trace_g); free(c->trace_err);
    c->trace_g = NULL; c->trace_err = NULL; c->trace_cap = 0; c->trace_n = 0;
    if (cap <= 0) return;
    size_t NN = (size_t)c->m->ndim * c->m->ndim;
    c->trace_g = calloc(NN * (size_t)cap, sizeof(zc));
    c->trace_err = calloc((size_t)cap, sizeof(double));
    c->trace_cap = (c->trace_g && c->trace_err) ? cap : 0;
}
int orc_chain_trace_count(const orc_chain *c) { return c->trace_n; }
void orc_chain_trace_get(const orc_chain *c, int i, double *g, double *err) {
    size_t NN = (size_t)c->m->ndim * c->m->ndim;
    if (i < 0 || i >= c->trace_n) return;
    if (g) memcpy(g, c->trace_g + (size_t)i * NN, sizeof(zc) * NN);
    if (err) *err = c->trace_err[i];
}

/* ------------------------------------------------------------------ */
/* propagators                                                         */
/* ------------------------------------------------------------------ */

/* checkerboard h0conf props (dqmc_config_h0/dqmc_{left,right}_{forward,backward}_prop.f90
 * BREAKUP_T branches, and _hc which uses urt since urt is Hermitian) */
static void h0_cb(const orc_model *m, int op, int nf, zc *g, int n2) {
    const orc_latt *L = &m->L;
    int N = m->ndim, lf = L->nn_lf;
    if (m->p.rt <= 0.0) return;
    const zc *U = (op == ORC_LEFT_BACKWARD || op == ORC_RIGHT_BACKWARD) ? m->urtm1 : m->urt;
    for (int b = 0; b < lf; ++b) {
        int ist = b + (nf - 1) * lf;
        int i1 = L->nnlf_list[b] - 1;
        int i2 = L->nnlist[i1 * L->nn_nf + nf - 1] - 1;
        const zc *u = &U[ist * 4];
        if (op == ORC_LEFT_FORWARD || op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC) {
            for (int j = 0; j < n2; ++j) {
                zc a = g[ZIDX(i1, j, N)], bb = g[ZIDX(i2, j, N)];
                g[ZIDX(i1, j, N)] = u[0] * a + u[1] * bb;
                g[ZIDX(i2, j, N)] = u[2] * a + u[3] * bb;
            }
        } else {
            for (int j = 0; j < n2; ++j) {   /* here n2 is the row count */
                zc a = g[ZIDX(j, i1, n2)], bb = g[ZIDX(j, i2, n2)];
                g[ZIDX(j, i1, n2)] = a * u[0] + bb * u[2];
                g[ZIDX(j, i2, n2)] = a * u[1] + bb * u[3];
            }
        }
    }
}

/* FFT h0conf props (-DFFT, square): B_K = F^-1 diag(exph0k) F */
/* dense kinetic step, the zgemm branch of the h0conf props
 * (src/dqmc_config_h0/dqmc_left_forward_prop.f90:235-246, _hc.f90:240,
 * dqmc_left_backward_prop.f90:236, dqmc_right_forward_prop.f90:276,
 * dqmc_right_backward_prop.f90:268): left ops g (N x n2) <- K g, right ops
 * g (n2 x N) <- g K, K = urtm1 for the backward ops and urt otherwise (urt is
 * Hermitian, so the _hc op uses it as well) */
static void h0_dense(const orc_model *m, int op, zc *g, int n2) {
    int N = m->ndim;
    zc *t = zalloc((size_t)N * n2);
    if (op == ORC_LEFT_FORWARD || op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC) {
        const zc *K = (op == ORC_LEFT_BACKWARD) ? m->urtm1d : m->urtd;
        for (int j = 0; j < n2; ++j)
            for (int i = 0; i < N; ++i) {
                zc acc = 0;
                for (int k = 0; k < N; ++k) acc += K[ZIDX(i, k, N)] * g[ZIDX(k, j, N)];
                t[ZIDX(i, j, N)] = acc;
            }
    } else {
        const zc *K = (op == ORC_RIGHT_BACKWARD) ? m->urtm1d : m->urtd;
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < n2; ++i) {
                zc acc = 0;
                for (int k = 0; k < N; ++k) acc += g[ZIDX(i, k, n2)] * K[ZIDX(k, j, N)];
                t[ZIDX(i, j, n2)] = acc;
            }
    }
    memcpy(g, t, sizeof(zc) * (size_t)N * n2);
    free(t);
}

/* the whole kinetic half step as one operator: FFT, or the dense matrix */
static void h0_fft(const orc_model *m, int op, zc *g, int n2) {
    if (m->p.kinetic == ORC_DENSE) { h0_dense(m, op, g, n2); return; }
    int lq = m->lq;
    zc *v = zalloc(lq);
    if (op == ORC_LEFT_FORWARD || op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC) {
        const zc *d = (op == ORC_LEFT_BACKWARD) ? m->exph0kinv : m->exph0k;
        for (int j = 0; j < n2; ++j) {
            zc *col = g + (size_t)j * lq;
            dft2(m, col, -1);
            for (int k = 0; k < lq; ++k) col[k] *= (op == ORC_LEFT_FORWARD_HC) ? conj(d[k]) : d[k];
            dft2(m, col, +1);
        }
    } else {
        /* rows r: (r B)^T = F D F^-1 r^T since F is symmetric */
        const zc *d = (op == ORC_RIGHT_BACKWARD) ? m->exph0kinv : m->exph0k;
        for (int i = 0; i < n2; ++i) {
            for (int k = 0; k < lq; ++k) v[k] = g[ZIDX(i, k, n2)];
            dft2(m, v, +1);
            for (int k = 0; k < lq; ++k) v[k] *= d[k];
            dft2(m, v, -1);
            for (int k = 0; k < lq; ++k) g[ZIDX(i, k, n2)] = v[k];
        }
    }
    free(v);
}

void orc_h0_prop(const orc_model *m, int op, int nf, double *g, int n2) {
    if (m->p.kinetic == ORC_CHECKERBOARD) h0_cb(m, op, nf, (zc *)g, n2);
    else h0_fft(m, op, (zc *)g, n2);
}

/* uconf props (src/dqmc_config_u/dqmc_*_prop.f90): diagonal exp(+-V) scaling */
static void u_prop(const orc_model *m, const int32_t *conf, int op, int nt, zc *g, int n2) {
    int N = m->ndim;
    const int32_t *cf = conf + (size_t)(nt - 1) * N;
    if (op == ORC_LEFT_FORWARD || op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC) {
        for (int i = 0; i < N; ++i) {
            int is = cf[i] - 1;
            zc b = (op == ORC_LEFT_FORWARD) ? m->bmat[is] : (op == ORC_LEFT_BACKWARD) ? m->bmat_inv[is] : conj(m->bmat[is]);
            for (int j = 0; j < n2; ++j) g[ZIDX(i, j, N)] *= b;
        }
    } else {
        for (int j = 0; j < N; ++j) {
            int is = cf[j] - 1;
            zc b = (op == ORC_RIGHT_FORWARD) ? m->bmat[is] : m->bmat_inv[is];
            for (int i = 0; i < n2; ++i) g[ZIDX(i, j, n2)] *= b;
        }
    }
}

void orc_u_prop(const orc_model *m, const int32_t *conf, int op, int nt, double *g, int n2) {
    u_prop(m, conf, op, nt, (zc *)g, n2);
}

/* Bmat_left_forward (src/dqmc_ft_core.f90:70-121): B(nt1,nt2) * g */
/* the bond field of slice nt in a B product: per family (1..nnf, or nnf..1
 * when desc) the nflag = 2 step, then nflag = 1 (src/dqmc_ft_core.f90:98-104,
 * 150-156, 264-270) */
static void v_slice(const orc_chain *c, int op, int nt, int desc, zc *g) {
    const orc_model *m = c->m;
    if (!m->lwrapv) return;
    int nnf = m->L.nn_nf;
    for (int k = 1; k <= nnf; ++k) {
        int nf = desc ? nnf + 1 - k : k;
        orc_v_prop(m, c->vconf, op, nt, nf, 2, g, m->ndim);
        orc_v_prop(m, c->vconf, op, nt, nf, 1, g, m->ndim);
    }
}

static void bmat_left_forward(const orc_chain *c, int nt1, int nt2, zc *g) {
    const orc_model *m = c->m;
    int N = m->ndim, nnf = m->L.nn_nf;
    int cb = (m->p.kinetic == ORC_CHECKERBOARD);
    for (int nt = nt2; nt <= nt1; ++nt) {
        if (m->lwrapT) {
            if (cb) for (int nf = 1; nf <= nnf; ++nf) h0_cb(m, ORC_LEFT_FORWARD, nf, g, N);
            else h0_fft(m, ORC_LEFT_FORWARD, g, N);
        }
        if (m->lwrapplqu)
            for (int i = 0; i < m->lq; ++i) orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD, i, nt, g, N);
        v_slice(c, ORC_LEFT_FORWARD, nt, 0, g);
        if (m->lwrapu) u_prop(m, c->conf, ORC_LEFT_FORWARD, nt, g, N);
        if (m->lwrapT) {
            if (cb) for (int nf = nnf; nf >= 1; --nf) h0_cb(m, ORC_LEFT_FORWARD, nf, g, N);
            else h0_fft(m, ORC_LEFT_FORWARD, g, N);
        }
    }
}

/* Bmat_left_forward_hc (src/dqmc_ft_core.f90:123-175): B(nt1,nt2)^H * g */
static void bmat_left_forward_hc(const orc_chain *c, int nt1, int nt2, zc *g) {
    const orc_model *m = c->m;
    int N = m->ndim, nnf = m->L.nn_nf;
    int cb = (m->p.kinetic == ORC_CHECKERBOARD);
    for (int nt = nt1; nt >= nt2; --nt) {
        if (m->lwrapT) {
            if (cb) for (int nf = 1; nf <= nnf; ++nf) h0_cb(m, ORC_LEFT_FORWARD_HC, nf, g, N);
            else h0_fft(m, ORC_LEFT_FORWARD_HC, g, N);
        }
        if (m->lwrapu) u_prop(m, c->conf, ORC_LEFT_FORWARD_HC, nt, g, N);
        v_slice(c, ORC_LEFT_FORWARD_HC, nt, 1, g);
        if (m->lwrapplqu)
            for (int i = m->lq - 1; i >= 0; --i) orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD_HC, i, nt, g, N);
        if (m->lwrapT) {
            if (cb) for (int nf = nnf; nf >= 1; --nf) h0_cb(m, ORC_LEFT_FORWARD_HC, nf, g, N);
            else h0_fft(m, ORC_LEFT_FORWARD_HC, g, N);
        }
    }
}

void orc_bmat_left_forward(const orc_chain *c, int nt1, int nt2, double *g) { bmat_left_forward(c, nt1, nt2, (zc *)g); }
void orc_bmat_left_forward_hc(const orc_chain *c, int nt1, int nt2, double *g) { bmat_left_forward_hc(c, nt1, nt2, (zc *)g); }

/* ------------------------------------------------------------------ */
/* local updates                                                       */
/* ------------------------------------------------------------------ */

static zc zpow(zc z, int n) { zc r = 1; for (int i = 0; i < n; ++i) r *= z; return r; }

/* ratio of the flip (is -> isp) given the fermion part ratio1;
 * dqmc_update.f90:52-60 */
zc orc_total_ratio(const orc_model *m, zc ratio1, int is, int iflip, int isp) {
    int lc = m->lcomp;
    zc r = zpow(ratio1, m->p.nflr);
    zc pr = m->phase_ratio[(is - 1) * (lc - 1) + (iflip - 1)];
    if (m->p.lproju) r *= pr;
    else r *= (m->gaml[isp - 1] / m->gaml[is - 1]) * pr;
    return r;
}

/* fast update (src/dqmc_config_u/dqmc_update.f90:1-92) */
static void update_fast(orc_chain *c, int nt, int32_t *acc) {
    const orc_model *m = c->m;
    int N = m->ndim, lc = m->lcomp;
    zc *g = c->gf;
    zc *uk = zalloc(N), *vk = zalloc(N);
    double accm = 0;
    for (int is_ = 0; is_ < N; ++is_) {
        int32_t *cf = &c->conf[(size_t)(nt - 1) * N + is_];
        int is = *cf;
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        for (int j = 0; j < N; ++j) vk[j] = -g[ZIDX(is_, j, N)];
        vk[is_] = 1.0 - g[ZIDX(is_, is_, N)];
        zc dlt = m->delta[(is - 1) * (lc - 1) + (iflip - 1)];
        zc ratio1 = vk[is_] * dlt + 1.0;
        zc sscl = dlt / ratio1;
        zc rt = orc_total_ratio(m, ratio1, is, iflip, isp);
        double rre = creal(rt * c->phase) / creal(c->phase);
        double rabs = rre < 0 ? -rre : rre;
        double rnd = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, rabs, rnd);
        int a = rabs > rnd;
        if (acc) acc[is_] = a;
        if (a) {
            accm += 1;
            double w = sqrt(creal(rt * conj(rt)));
            c->phase = c->phase * rt / w;
            for (int i = 0; i < N; ++i) uk[i] = g[ZIDX(i, is_, N)];
            for (int i2 = 0; i2 < N; ++i2)
                for (int i1 = 0; i1 < N; ++i1) g[ZIDX(i1, i2, N)] -= sscl * uk[i1] * vk[i2];
            *cf = isp;
        }
    }
    c->acc_u += accm; c->prop_u += N;
    free(uk); free(vk);
}

/* delay update (src/dqmc_config_u/dqmc_update_delay.f90:1-137) */
static void update_delay(orc_chain *c, int nt, int32_t *acc) {
    const orc_model *m = c->m;
    int N = m->ndim, lc = m->lcomp, nb = m->nublock;
    zc *g = c->gf;
    zc *diag = zalloc(N), *av = zalloc((size_t)N * nb), *bv = zalloc((size_t)N * nb);
    double accm = 0;
    int ik = 0;
    for (int i = 0; i < N; ++i) diag[i] = g[ZIDX(i, i, N)];
    for (int s = 0; s < N; ++s) {
        int32_t *cf = &c->conf[(size_t)(nt - 1) * N + s];
        int is = *cf;
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        zc dlt = m->delta[(is - 1) * (lc - 1) + (iflip - 1)];
        zc ratio1 = (1.0 - diag[s]) * dlt + 1.0;
        zc sscl = dlt / ratio1;
        zc rt = orc_total_ratio(m, ratio1, is, iflip, isp);
        double rre = creal(rt * c->phase) / creal(c->phase);
        double rabs = rre < 0 ? -rre : rre;
        double rnd = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, rabs, rnd);
        int a = rabs > rnd;
        if (acc) acc[s] = a;
        if (a) {
            accm += 1;
            double w = sqrt(creal(rt * conj(rt)));
            c->phase = c->phase * rt / w;
            ik += 1;
            zc *ak = av + (size_t)(ik - 1) * N, *bk = bv + (size_t)(ik - 1) * N;
            for (int i = 0; i < N; ++i) { ak[i] = g[ZIDX(i, s, N)]; bk[i] = g[ZIDX(s, i, N)]; }
            for (int mm = 0; mm < ik - 1; ++mm) {
                zc bsm = bv[(size_t)mm * N + s], asm_ = av[(size_t)mm * N + s];
                for (int i = 0; i < N; ++i) {
                    ak[i] += bsm * av[(size_t)mm * N + i];
                    bk[i] += asm_ * bv[(size_t)mm * N + i];
                }
            }
            for (int i = 0; i < N; ++i) ak[i] *= sscl;
            bk[s] -= 1.0;
            for (int i = 0; i < N; ++i) diag[i] += ak[i] * bk[i];
            *cf = isp;
        }
        if (ik == nb || s == N - 1) {
            ik = 0;
            orc_zgemm('N', 'T', N, N, nb, 1.0, av, N, bv, N, 1.0, g, N);
            if (s < N - 1) {
                for (int i = 0; i < N; ++i) diag[i] = g[ZIDX(i, i, N)];
                memset(av, 0, sizeof(zc) * (size_t)N * nb);
                memset(bv, 0, sizeof(zc) * (size_t)N * nb);
            }
        }
    }
    c->acc_u += accm; c->prop_u += N;
    free(diag); free(av); free(bv);
}

/* submatrix update (src/dqmc_config_u/dqmc_update_submatrix.f90:1-180) */
static void update_submatrix(orc_chain *c, int nt, int32_t *acc) {
    const orc_model *m = c->m;
    int N = m->ndim, lc = m->lcomp, nb = m->nublock;
    zc *g = c->gf;
    int *pvec = calloc(nb, sizeof(int));
    zc *gam = zalloc((size_t)nb * nb), *gcut = zalloc((size_t)N * N);
    zc *cvec = zalloc(nb), *bvec = zalloc(nb), *v1 = zalloc(nb), *v4 = zalloc(nb);
    zc *gt1 = zalloc((size_t)N * nb), *gt2 = zalloc((size_t)nb * N), *gm1 = zalloc((size_t)N * nb);
    double accm = 0;
    int ik = 0;
    memcpy(gcut, g, sizeof(zc) * (size_t)N * N);
#define GAM(i, j) gam[(i) + (size_t)(j) * nb]
    for (int s = 0; s < N; ++s) {
        int32_t *cf = &c->conf[(size_t)(nt - 1) * N + s];
        int is = *cf;
        int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
        int isp = (is + iflip - 1) % lc + 1;
        for (int i = 0; i < nb; ++i) { cvec[i] = 0; bvec[i] = 0; v1[i] = 0; }
        for (int i = 0; i < ik; ++i) {
            int isf = pvec[i];
            cvec[i] = g[ZIDX(s, isf, N)];
            bvec[i] = g[ZIDX(isf, s, N)];
        }
        for (int i = 0; i < ik; ++i)
            for (int mm = 0; mm < ik; ++mm) v1[i] += cvec[mm] * GAM(mm, i);
        zc v = 0;
        for (int i = 0; i < ik; ++i) v += v1[i] * bvec[i];
        zc v2 = v + g[ZIDX(s, s, N)] - 1.0;
        zc dlt = m->delta[(is - 1) * (lc - 1) + (iflip - 1)];
        zc ratio1 = -v2 * dlt + 1.0;
        zc rt = orc_total_ratio(m, ratio1, is, iflip, isp);
        double rre = creal(rt * c->phase) / creal(c->phase);
        double rabs = rre < 0 ? -rre : rre;
        double rnd = orc_sfmt_stream(&c->rng);
        ORC_COUNT_TIE(c, rabs, rnd);
        int a = rabs > rnd;
        if (acc) acc[s] = a;
        if (a) {
            accm += 1;
            double w = sqrt(creal(rt * conj(rt)));
            c->phase = c->phase * rt / w;
            ik += 1;
            pvec[ik - 1] = s;
            zc v3 = 1.0 / (-v + 1.0 + 1.0 / dlt - g[ZIDX(s, s, N)]);
            GAM(ik - 1, ik - 1) = v3;
            for (int i = 0; i < nb; ++i) v4[i] = 0;
            for (int i = 0; i < ik - 1; ++i)
                for (int mm = 0; mm < ik - 1; ++mm) v4[i] += GAM(i, mm) * bvec[mm];
            for (int i = 0; i < ik - 1; ++i) {
                GAM(ik - 1, i) = v3 * v1[i];
                GAM(i, ik - 1) = v4[i] * v3;
            }
            for (int mm = 0; mm < ik - 1; ++mm)
                for (int i = 0; i < ik - 1; ++i) GAM(i, mm) += v4[i] * v3 * v1[mm];
            zc f = dlt / (1.0 + dlt);
            for (int i = 0; i < N; ++i) gcut[ZIDX(i, s, N)] -= f * gcut[ZIDX(i, s, N)];
            for (int i = 0; i < N; ++i) gt1[ZIDX(i, ik - 1, N)] = g[ZIDX(i, s, N)];
            *cf = isp;
        }
        if (ik == nb || s == N - 1) {
            for (int i = 0; i < ik; ++i) {
                int isf = pvec[i];
                for (int j = 0; j < N; ++j) gt2[ZIDX(i, j, nb)] = gcut[ZIDX(isf, j, N)];
            }
            if (ik > 0) {
                orc_zgemm('N', 'N', N, nb, ik, 1.0, gt1, N, gam, nb, 0.0, gm1, N);
                orc_zgemm('N', 'N', N, N, ik, 1.0, gm1, N, gt2, nb, 1.0, gcut, N);
            }
            memcpy(g, gcut, sizeof(zc) * (size_t)N * N);
            ik = 0;
        }
    }
#undef GAM
    c->acc_u += accm; c->prop_u += N;
    free(pvec); free(gam); free(gcut); free(cvec); free(bvec); free(v1); free(v4);
    free(gt1); free(gt2); free(gm1);
}

void orc_update(orc_chain *c, int nt, int32_t *acc) {
    switch (c->m->p.update) {
    case ORC_FAST: update_fast(c, nt, acc); break;
    case ORC_DELAY: update_delay(c, nt, acc); break;
    default: update_submatrix(c, nt, acc); break;
    }
}

/* ------------------------------------------------------------------ */
/* stabilisation (src/dqmc_ft_core/dqmc_ft_stablize_{0b,b0}_qr.f90)    */
/* ------------------------------------------------------------------ */

/* s_zpm (s_matrix.f90:864-930), transcribed: row permutation by jpv */
static void zpm(int rdim, int cdim, int32_t *jpv, zc *a) {
    int *jpvt = malloc(sizeof(int) * rdim);
    for (int k = 0; k < rdim; ++k) jpvt[k] = k + 1;
    for (;;) {
        int npt = 0;
        for (int k = 1; k <= rdim; ++k) {
            int pv = jpv[k - 1];
            if (pv != k) {
                ++npt;
                int t = jpv[pv - 1]; jpv[pv - 1] = jpv[k - 1]; jpv[k - 1] = t;
                t = jpvt[pv - 1]; jpvt[pv - 1] = jpvt[k - 1]; jpvt[k - 1] = t;
            }
        }
        if (!npt) break;
    }
    for (;;) {
        int npt = 0;
        for (int k = 1; k <= rdim; ++k) {
            int pv = jpvt[k - 1];
            if (pv != k) {
                ++npt;
                for (int c2 = 0; c2 < cdim; ++c2) {
                    zc t = a[ZIDX(pv - 1, c2, rdim)]; a[ZIDX(pv - 1, c2, rdim)] = a[ZIDX(k - 1, c2, rdim)]; a[ZIDX(k - 1, c2, rdim)] = t;
                }
                int t = jpvt[pv - 1]; jpvt[pv - 1] = jpvt[k - 1]; jpvt[k - 1] = t;
            }
        }
        if (!npt) break;
    }
    free(jpvt);
}

/* s_zmp (s_matrix.f90:1059-1087), transcribed: column permutation */
static void zmp(int rdim, int cdim, zc *a, int32_t *jpv) {
    for (;;) {
        int npt = 0;
        for (int k = 1; k <= cdim; ++k) {
            int pv = jpv[k - 1];
            if (pv != k) {
                ++npt;
                for (int r = 0; r < rdim; ++r) {
                    zc t = a[ZIDX(r, pv - 1, rdim)]; a[ZIDX(r, pv - 1, rdim)] = a[ZIDX(r, k - 1, rdim)]; a[ZIDX(r, k - 1, rdim)] = t;
                }
                int t = jpv[pv - 1]; jpv[pv - 1] = jpv[k - 1]; jpv[k - 1] = t;
            }
        }
        if (!npt) break;
    }
}

/* shared body of the two stabilisation routines.  Input b = propagated U;
 * d1/v1 = previous D/V (ignored if pivoted). */
static void stab_step(int N, int pivoted, zc *b, const double *d1, const zc *v1,
                      zc *uo, double *dout, zc *vo, zc *logdet) {
    zc *btmp = zalloc((size_t)N * N), *r = zalloc((size_t)N * N), *vt = zalloc((size_t)N * N);
    int32_t *jpvt = malloc(sizeof(int32_t) * N);
    if (pivoted) {
        orc_qrpt_logdet(N, b, uo, r, jpvt, logdet);
        for (int i = 0; i < N; ++i) dout[i] = creal(r[ZIDX(i, i, N)]);
        memset(vo, 0, sizeof(zc) * (size_t)N * N);
        for (int j = 0; j < N; ++j)
            for (int i = 0; i <= j; ++i) vo[ZIDX(i, j, N)] = r[ZIDX(i, j, N)] / dout[i];
        zmp(N, N, vo, jpvt);
    } else {
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) btmp[ZIDX(i, j, N)] = d1[j] * b[ZIDX(i, j, N)];
        orc_zmcpt(N, N, (double *)btmp, jpvt);
        orc_qr_logdet(N, btmp, uo, r, logdet);
        for (int i = 0; i < N; ++i) dout[i] = creal(r[ZIDX(i, i, N)]);
        for (int j = 0; j < N; ++j)
            for (int i = 0; i <= j; ++i) vt[ZIDX(i, j, N)] = r[ZIDX(i, j, N)] / dout[i];
        zc *vm1 = zalloc((size_t)N * N);
        memcpy(vm1, v1, sizeof(zc) * (size_t)N * N);
        zpm(N, N, jpvt, vm1);
        orc_zgemm('N', 'N', N, N, N, 1.0, vt, N, vm1, N, 0.0, vo, N);
        free(vm1);
    }
    free(btmp); free(r); free(vt); free(jpvt);
}

void orc_stablize_0b(orc_chain *c, int n) {
    const orc_model *m = c->m;
    int N = m->ndim;
    zc *b = zalloc((size_t)N * N);
    memcpy(b, c->Ust[n - 1], sizeof(zc) * (size_t)N * N);
    bmat_left_forward(c, m->wrap_step[(n - 1) * 2 + 1], m->wrap_step[(n - 1) * 2], b);
    stab_step(N, n == 1, b, c->Dst[n - 1], c->Vst[n - 1], c->Ust[n], c->Dst[n], c->Vst[n], &c->logdetQst[n]);
    free(b);
}

void orc_stablize_b0(orc_chain *c, int n) {
    const orc_model *m = c->m;
    int N = m->ndim;
    zc *b = zalloc((size_t)N * N);
    memcpy(b, c->Ust[n], sizeof(zc) * (size_t)N * N);
    bmat_left_forward_hc(c, m->wrap_step[(n - 1) * 2 + 1], m->wrap_step[(n - 1) * 2], b);
    zc *uo = zalloc((size_t)N * N), *vo = zalloc((size_t)N * N);
    double *dout = calloc(N, sizeof(double));
    zc ld;
    stab_step(N, n == m->nst, b, c->Dst[n], c->Vst[n], uo, dout, vo, &ld);
    memcpy(c->Ust[n - 1], uo, sizeof(zc) * (size_t)N * N);
    memcpy(c->Vst[n - 1], vo, sizeof(zc) * (size_t)N * N);
    memcpy(c->Dst[n - 1], dout, sizeof(double) * N);
    c->logdetQst[n - 1] = ld;
    free(b); free(uo); free(vo); free(dout);
}

void orc_stack_get(const orc_chain *c, int n, double *u, double *d, double *v, double *logdetq) {
    int N = c->m->ndim;
    if (u) memcpy(u, c->Ust[n], sizeof(zc) * (size_t)N * N);
    if (v) memcpy(v, c->Vst[n], sizeof(zc) * (size_t)N * N);
    if (d) memcpy(d, c->Dst[n], sizeof(double) * N);
    if (logdetq) { logdetq[0] = creal(c->logdetQst[n]); logdetq[1] = cimag(c->logdetQst[n]); }
}

void orc_stack_set(orc_chain *c, int n, const double *u, const double *d, const double *v, const double *logdetq) {
    int N = c->m->ndim;
    if (u) memcpy(c->Ust[n], u, sizeof(zc) * (size_t)N * N);
    if (v) memcpy(c->Vst[n], v, sizeof(zc) * (size_t)N * N);
    if (d) memcpy(c->Dst[n], d, sizeof(double) * N);
    if (logdetq) c->logdetQst[n] = logdetq[0] + I * logdetq[1];
}

/* s_dvec_min_max (s_matrix.f90:752-783) */
static void dvec_min_max(int n, const double *d, double *dmax, double *dmin) {
    for (int i = 0; i < n; ++i) {
        if (fabs(d[i]) > 1.0) { dmax[i] = fabs(d[i]); dmin[i] = copysign(1.0, d[i]); }
        else { dmax[i] = 1.0; dmin[i] = d[i]; }
    }
}

/* green_equaltime (src/dqmc_ft_core/green_equaltime.f90:1-107) */
static int green_equaltime(int N, const zc *ure, const double *dre, const zc *vre, const zc *vle,
                           const double *dle, const zc *ule, zc *gtt, zc logdetqr, zc logdetql, zc *logw) {
    double *drmax = malloc(sizeof(double) * N), *drmin = malloc(sizeof(double) * N);
    double *dlmax = malloc(sizeof(double) * N), *dlmin = malloc(sizeof(double) * N);
    zc *uu = zalloc((size_t)N * N), *vv = zalloc((size_t)N * N), *dvvd = zalloc((size_t)N * N), *bt = zalloc((size_t)N * N);
    dvec_min_max(N, dre, drmax, drmin);
    dvec_min_max(N, dle, dlmax, dlmin);
    orc_zgemm('C', 'N', N, N, N, 1.0, ure, N, ule, N, 0.0, uu, N);
    orc_zgemm('N', 'C', N, N, N, 1.0, vre, N, vle, N, 0.0, vv, N);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
            dvvd[ZIDX(i, j, N)] = uu[ZIDX(i, j, N)] / (drmax[i] * dlmax[j]) + vv[ZIDX(i, j, N)] * drmin[i] * dlmin[j];
    zc zl;
    orc_zinv_logdet(N, dvvd, &zl);
    /* s_v_invd_u(ule, dlmax, dvvd) -> bt ; s_v_invd_uH(bt, drmax, ure) -> gtt */
    zc *vi = zalloc((size_t)N * N);
    for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) vi[ZIDX(i, j, N)] = ule[ZIDX(i, j, N)] / dlmax[j];
    orc_zgemm('N', 'N', N, N, N, 1.0, vi, N, dvvd, N, 0.0, bt, N);
    for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) vi[ZIDX(i, j, N)] = bt[ZIDX(i, j, N)] / drmax[j];
    orc_zgemm('N', 'C', N, N, N, 1.0, vi, N, ure, N, 0.0, gtt, N);
    double r1 = 0, r2 = 0;
    for (int i = 0; i < N; ++i) r1 += log(dlmax[i]);
    for (int i = 0; i < N; ++i) r2 += log(drmax[i]);
    *logw = -logdetql + logdetqr + zl + (r1 + r2);
    free(drmax); free(drmin); free(dlmax); free(dlmin); free(uu); free(vv); free(dvvd); free(bt); free(vi);
    return 0;
}

int orc_green_equaltime(int n, const double *ur, const double *dr, const double *vr,
                        const double *vl, const double *dl, const double *ul,
                        double *g, const double *logdetqr, const double *logdetql, double *logw) {
    zc lw;
    int info = green_equaltime(n, (const zc *)ur, dr, (const zc *)vr, (const zc *)vl, dl, (const zc *)ul,
                               (zc *)g, logdetqr[0] + I * logdetqr[1], logdetql[0] + I * logdetql[1], &lw);
    logw[0] = creal(lw); logw[1] = cimag(lw);
    return info;
}

/* green_equaltimebb (src/dqmc_ft_core/green_equaltimebb.f90:1-84) */
static int green_equaltimebb(int N, const zc *ure, const double *dre, const zc *vre, zc *gtt, zc logdetqr, zc *logw) {
    double *drmax = malloc(sizeof(double) * N), *drmin = malloc(sizeof(double) * N);
    zc *dvvd = zalloc((size_t)N * N), *vi = zalloc((size_t)N * N);
    dvec_min_max(N, dre, drmax, drmin);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
            dvvd[ZIDX(i, j, N)] = conj(ure[ZIDX(j, i, N)]) / drmax[i] + vre[ZIDX(i, j, N)] * drmin[i];
    zc zl;
    orc_zinv_logdet(N, dvvd, &zl);
    for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) vi[ZIDX(i, j, N)] = dvvd[ZIDX(i, j, N)] / drmax[j];
    orc_zgemm('N', 'C', N, N, N, 1.0, vi, N, ure, N, 0.0, gtt, N);
    double r = 0;
    for (int i = 0; i < N; ++i) r += log(drmax[i]);
    *logw = logdetqr + zl + r;
    free(drmax); free(drmin); free(dvvd); free(vi);
    return 0;
}

/* set_phase (src/dqmc_ft_core/set_phase.f90:1-24) */
zc orc_set_phase(const orc_chain *c, zc logw) {
    const orc_model *m = c->m;
    zc ph = cexp(I * (m->p.nflr * cimag(logw)));
    if (m->lwrapplqu)
        for (int nt = 0; nt < m->ltrot; ++nt)
            for (int i = 0; i < m->lq; ++i) ph *= m->plq_phase[c->conf_plq[(size_t)nt * m->lq + i] - 1];
    if (m->lwrapu && m->p.rhub > 0.0) {
        int N = m->ndim;
        for (int nt = 0; nt < m->ltrot; ++nt)
            for (int i = 0; i < N; ++i) ph *= m->phase[c->conf[(size_t)nt * N + i] - 1];
    }
    return ph;
}

double orc_compare_max(int N, const zc *a, const zc *b) {   /* s_compare_max_z */
    double mx = 0;
    for (size_t k = 0; k < (size_t)N * N; ++k) { double t = cabs(a[k] - b[k]); if (t > mx) mx = t; }
    return mx;
}

/* dqmc_ft_sweep_start_0b (src/dqmc_ft_core/dqmc_ft_sweep_start_0b.f90:1-71) */
int orc_sweep_start_0b(orc_chain *c) {
    const orc_model *m = c->m;
    int N = m->ndim;
    if (m->nst > 0) {
        memset(c->Ust[0], 0, sizeof(zc) * (size_t)N * N);
        memset(c->Vst[0], 0, sizeof(zc) * (size_t)N * N);
        for (int i = 0; i < N; ++i) { c->Ust[0][ZIDX(i, i, N)] = 1; c->Vst[0][ZIDX(i, i, N)] = 1; c->Dst[0][i] = 1; }
        c->logdetQst[0] = 0;
        for (int n = 1; n <= m->nst; ++n) orc_stablize_0b(c, n);
        green_equaltimebb(N, c->Ust[m->nst], c->Dst[m->nst], c->Vst[m->nst], c->gf, c->logdetQst[m->nst], &c->logweightf);
        c->phase = orc_set_phase(c, c->logweightf);
    } else {
        memset(c->gf, 0, sizeof(zc) * (size_t)N * N);
        for (int i = 0; i < N; ++i) c->gf[ZIDX(i, i, N)] = 1;
        bmat_left_forward(c, m->ltrot, 1, c->gf);
        for (int i = 0; i < N; ++i) c->gf[ZIDX(i, i, N)] += 1;
        orc_zinv(N, c->gf);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* equal-time measurement (src/dqmc_measure/equaltime_measure.f90)     */
/* ------------------------------------------------------------------ */
void orc_obser_init(orc_chain *c) {   /* dqmc_measure_2d.f90:105-130 */
    int lq = c->m->lq;
    c->nobs = 0;
    memset(c->energy_bin, 0, sizeof(c->energy_bin));
    memset(c->zcpcm_bin, 0, sizeof(zc) * lq * 4); memset(c->zspsm_bin, 0, sizeof(zc) * lq * 4);
    memset(c->znn_bin, 0, sizeof(zc) * lq * 4); memset(c->pair_onsite_bin, 0, sizeof(zc) * lq * 4);
    memset(c->zjj_bin, 0, sizeof(zc) * lq); memset(c->zbb_bin, 0, sizeof(zc) * lq);
    memset(c->pair_nn_bin, 0, sizeof(zc) * lq); memset(c->pair_sn_bin, 0, sizeof(zc) * lq);
    c->zn_bin[0] = c->zn_bin[1] = 0; c->zj_bin = 0; c->zb_bin = 0;
    if (c->m->p.ltau) memset(c->znn_tau_bin, 0, sizeof(zc) * (size_t)lq * 4 * (c->m->ntdm + 1));
}

static int npbc_cyc(int nr, int l) { if (nr > l) return nr - l; if (nr < 1) return nr + l; return nr; }

/* equaltime_measure of the cubic and r_cubic lattices after energy_bin(1:2)
 * (src/dqmc_measure/equaltime_measure3d.f90:43-179): zkint over the bond
 * families of the A sites (no rt, no t2 term), zint_u, and cpcm, spsm, nn (+ zn)
 * binned by the cell distance imj(list(i,1), list(j,1)) over all orbital
 * pairs, bondcorr (+ zb) over the pairs (nu, nnlist(nu, 1)) for nu = 1..lq,
 * a cell index used as a site index as the reference does.  The bins are the
 * (no_i, no_j) = (1, 1) block of the 2D layout; pair_onsite, jj, pair_nn,
 * pair_sn, zj and energy_bin(5:10) do not exist here and stay 0.  c->gfc
 * already holds Gc. */
static void measure_3d(orc_chain *c, zc zphi) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    const int N = m->ndim, lq = m->lq, nnf = L->nn_nf, nflr = m->p.nflr;
    const zc *g = c->gf, *gc = c->gfc;
#define GC3(i, j) gc[ZIDX((i), (j), N)]
#define GF3(i, j) g[ZIDX((i), (j), N)]
    zc zk = 0;
    for (int b = 0; b < L->nn_lf; ++b) {
        const int i0 = L->nnlf_list[b] - 1;
        for (int nf = 1; nf <= nnf; ++nf) {
            const int in = L->nnlist[i0 * nnf + nf - 1] - 1;
            zk += -2.0 * creal(GC3(i0, in) * m->expar_nn[i0 * nnf + nf - 1]);
        }
    }
    c->energy_bin[2] += zk * zphi;
    zc zu = 0;
    for (int i = 0; i < L->nsites; ++i) zu += GC3(i, i) * GC3(i, i);
    c->energy_bin[3] += zu * zphi;
    const double fsp = 1.0 - 1.0 / (double)(nflr * nflr), fn = 1.0 / (double)nflr;
    zc *cp = zalloc(lq), *sp = zalloc(lq), *nn = zalloc(lq), *bb = zalloc(lq);
    zc zn = 0, zb = 0;
    for (int j = 0; j < N; ++j) {
        const int nuj = L->list[j * 2] - 1;
        zn += GC3(j, j);
        for (int i = 0; i < N; ++i) {
            const int k = L->imj[(L->list[i * 2] - 1) * lq + nuj] - 1;
            cp[k] += GC3(i, j);
            sp[k] += GC3(i, j) * GF3(i, j) * fsp;
            nn[k] += GC3(i, i) * GC3(j, j) + fn * GC3(i, j) * GF3(i, j);
        }
    }
    for (int nuj = 0; nuj < lq; ++nuj) {
        const int j0 = nuj, jn = L->nnlist[j0 * nnf] - 1;
        const zc zj = m->expar_nn[j0 * nnf];
        zb += zj * GC3(j0, jn) + conj(zj) * GC3(jn, j0);
        for (int nui = 0; nui < lq; ++nui) {
            const int i0 = nui, in = L->nnlist[i0 * nnf] - 1;
            const zc zi = m->expar_nn[i0 * nnf];
            const int k = L->imj[nui * lq + nuj] - 1;
            bb[k] += (zj * GC3(j0, jn) + conj(zj) * GC3(jn, j0)) * (zi * GC3(i0, in) + conj(zi) * GC3(in, i0)) +
                     (zi * zj * GC3(i0, jn) * GF3(in, j0) + conj(zi) * conj(zj) * GC3(in, j0) * GF3(i0, jn) +
                      zi * conj(zj) * GC3(i0, j0) * GF3(in, jn) + conj(zi) * zj * GC3(in, jn) * GF3(i0, j0)) * fn;
        }
    }
    for (int k = 0; k < lq; ++k) {
        c->zcpcm_bin[k] += cp[k] * zphi;
        c->zspsm_bin[k] += sp[k] * zphi;
        c->znn_bin[k] += nn[k] * zphi;
        c->zbb_bin[k] += bb[k] * zphi;
    }
    c->zn_bin[0] += zn * zphi;
    c->zb_bin += zb * zphi;
    free(cp); free(sp); free(nn); free(bb);
#undef GC3
#undef GF3
}

void orc_measure(orc_chain *c, int nt) {
    (void)nt;
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    const orc_params *p = &m->p;
    int N = m->ndim, lq = m->lq, nnf = L->nn_nf, zp = L->z_plq, nflr = p->nflr;
    const zc *g = c->gf;
    zc *gc = c->gfc;
    c->nobs += 1;
    double sgn = creal(c->phase) < 0 ? -1.0 : 1.0;
    zc zphi = (sgn / creal(c->phase)) * c->phase;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) gc[ZIDX(j, i, N)] = (i == j ? 1.0 : 0.0) - g[ZIDX(i, j, N)];
#define GC(i, j) gc[ZIDX((i), (j), N)]
#define GF(i, j) g[ZIDX((i), (j), N)]
    c->energy_bin[0] += sgn;
    zc zne = 0;
    for (int i = 0; i < N; ++i) zne += GC(i, i);
    c->energy_bin[1] += zne * zphi / (double)lq;
    if (L->kind == ORC_CUBIC || L->kind == ORC_R_CUBIC) { measure_3d(c, zphi); return; }
    /* zkint; the chain's (equaltime_measure1d.f90) carries the factor nflr rt on
     * the bonds and 2 t2 on the two second neighbours */
    const int chain = (L->kind == ORC_CHAIN);
    zc zk = 0;
    for (int b = 0; b < L->nn_lf; ++b) {
        int i0 = L->nnlf_list[b] - 1;
        for (int nf = 1; nf <= nnf; ++nf) {
            int in = L->nnlist[i0 * nnf + nf - 1] - 1;
            zk += (chain ? -2.0 * nflr * p->rt : -2.0) * creal(GC(i0, in) * m->expar_nn[i0 * nnf + nf - 1]);
        }
    }
    if (p->t2 != 0.0) {
        int ns = chain ? 2 : (L->kind == ORC_SQUARE) ? 4 : 6;
        for (int i0 = 0; i0 < L->nsites; ++i0)
            for (int nf = 0; nf < ns; ++nf)
                zk += (chain ? -2.0 * p->t2 : -p->t2) * creal(GC(i0, L->snlist[i0 * L->nsn + nf] - 1));
    }
    c->energy_bin[2] += zk * zphi;
    /* zint_u */
    zc zu = 0;
    for (int i = 0; i < L->nsites; ++i) zu += GC(i, i) * GC(i, i);
    c->energy_bin[3] += zu * zphi;
    /* zqsq, ztsq, ztq (2D only) */
    zc zq = 0, zt = 0, ztq = 0;
    zc e_m = cexp(-I * p->theta), e_p = cexp(I * p->theta);
    for (int q = 0; q < (chain ? 0 : lq); ++q) {
        const int *pc = &L->plq_cord[q * zp];
        zc tmp = 0;
        for (int a = 0; a < zp; ++a) tmp += GC(pc[a] - 1, pc[a] - 1);
        zq += tmp * tmp * (double)nflr;
        for (int a = 0; a < zp; ++a)
            for (int b = 0; b < zp; ++b) zq += GC(pc[a] - 1, pc[b] - 1) * GF(pc[a] - 1, pc[b] - 1);
        /* T^2 */
        zc tt = 0;
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1] - 1, i1a = pc[npbc_cyc(a + 1, zp) - 1] - 1;
            zc z1 = (a % 2 == 0) ? -e_p : e_m;
            tt += 2.0 * creal(z1 * GC(i1, i1a));
        }
        zt += tt * tt * (double)nflr;
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1] - 1, i1a = pc[npbc_cyc(a + 1, zp) - 1] - 1;
            zc z1 = (a % 2 == 0) ? -e_p : e_m, z2 = conj(z1);
            for (int b = 1; b <= zp; ++b) {
                int i2 = pc[b - 1] - 1, i2a = pc[npbc_cyc(b + 1, zp) - 1] - 1;
                zc z3 = (b % 2 == 0) ? -e_p : e_m, z4 = conj(z3);
                zt += z1 * z3 * (GC(i1, i2a) * GF(i1a, i2)) + z1 * z4 * (GC(i1, i2) * GF(i1a, i2a)) +
                      z2 * z3 * (GC(i1a, i2a) * GF(i1, i2)) + z2 * z4 * (GC(i1a, i2) * GF(i1, i2a));
            }
        }
        /* TQ */
        zc t1 = 0, t2 = 0;
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1] - 1, i1a = pc[npbc_cyc(a + 1, zp) - 1] - 1;
            zc z1 = (a % 2 == 0) ? -e_p : e_m;
            t1 += 2.0 * creal(z1 * GC(i1, i1a));
            t2 += (1.0 / 3.0) * GC(i1, i1);
        }
        ztq += t1 * t2 * (double)nflr;
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1] - 1, i1a = pc[npbc_cyc(a + 1, zp) - 1] - 1;
            zc z1 = ((a % 2 == 0) ? -e_p : e_m) / 3.0, z2 = conj(z1);
            for (int b = 1; b <= zp; ++b) {
                int i2 = pc[b - 1] - 1;
                ztq += z1 * (GC(i1, i2) * GF(i1a, i2)) + z2 * (GC(i1a, i2) * GF(i1, i2));
            }
        }
    }
    /* zint_v */
    zc zv = 0;
    for (int b = 0; b < L->nn_lf; ++b) {
        int i0 = L->nnlf_list[b] - 1;
        for (int nf = 1; nf <= nnf; ++nf) zv += creal(GC(i0, L->nnlist[i0 * nnf + nf - 1] - 1));
    }
    if (chain) {
        c->energy_bin[4] += zv * zphi;                /* energy_bin(5), without rv */
    } else {
        c->energy_bin[4] += zq * (1.0 / 9.0) * zphi;
        c->energy_bin[5] += zt * zphi;
        c->energy_bin[6] += ztq * zphi;
        c->energy_bin[7] += zv * p->rv * zphi;
    }
    /* cpcm, spsm, nn, pair_onsite: [imj][no_i][no_j], index (imj-1) + lq*((no_i-1) + 2*(no_j-1)) */
    double fsp = 1.0 - 1.0 / (double)(nflr * nflr), fn = 1.0 / (double)nflr;
    zc zn[2] = {0, 0};
    for (int j = 0; j < N; ++j) {
        int nuj = L->list[j * 2] - 1, noj = L->list[j * 2 + 1] - 1;
        zn[noj] += GC(j, j);
        for (int i = 0; i < N; ++i) {
            int nui = L->list[i * 2] - 1, noi = L->list[i * 2 + 1] - 1;
            int k = (L->imj[nui * lq + nuj] - 1) + lq * (noi + 2 * noj);
            c->zcpcm_bin[k] += GC(i, j) * zphi;
            c->zspsm_bin[k] += GC(i, j) * GF(i, j) * fsp * zphi;
            c->znn_bin[k] += (GC(i, i) * GC(j, j) + fn * GC(i, j) * GF(i, j)) * zphi;
            c->pair_onsite_bin[k] += GF(i, j) * GF(i, j) * zphi;
        }
    }
    c->zn_bin[0] += zn[0] * zphi; c->zn_bin[1] += zn[1] * zphi;
    /* jj, bb, pair_nn, pair_sn over unit cells */
    int hc = (L->kind == ORC_HONEYCOMB);
    zc zj = 0, zb = 0;
    for (int nuj = 0; nuj < lq; ++nuj) {
        int j0 = hc ? 2 * nuj : nuj;
        int jn_j = hc ? L->snlist[j0 * L->nsn] - 1 : L->nnlist[j0 * nnf] - 1;   /* jj partner */
        int jn_b = L->nnlist[j0 * nnf] - 1;                                      /* bond partner */
        int jn_s = L->snlist[j0 * L->nsn] - 1;
        zc zjb = m->expar_nn[j0 * nnf + 0];
        zb += zjb * GC(j0, jn_b) + conj(zjb) * GC(jn_b, j0);
        zj += I * (GC(j0, jn_j) - GC(jn_j, j0));
        for (int nui = 0; nui < lq; ++nui) {
            int i0 = hc ? 2 * nui : nui;
            int in_j = hc ? L->snlist[i0 * L->nsn] - 1 : L->nnlist[i0 * nnf] - 1;
            int in_b = L->nnlist[i0 * nnf] - 1;
            int in_s = L->snlist[i0 * L->nsn] - 1;
            int k = L->imj[nui * lq + nuj] - 1;
            zc z1 = (GC(i0, in_j) - GC(in_j, i0)) * (GC(j0, jn_j) - GC(jn_j, j0));
            zc z3 = GC(i0, jn_j) * GF(in_j, j0) + GC(in_j, j0) * GF(i0, jn_j) - GC(i0, j0) * GF(in_j, jn_j) - GC(in_j, jn_j) * GF(i0, j0);
            c->zjj_bin[k] += (-z1 - fn * z3) * zphi;
            zc zi = m->expar_nn[i0 * nnf + 0];
            zc bbv = (zjb * GC(j0, jn_b) + conj(zjb) * GC(jn_b, j0)) * (zi * GC(i0, in_b) + conj(zi) * GC(in_b, i0)) +
                     (zi * zjb * GC(i0, jn_b) * GF(in_b, j0) + conj(zi) * conj(zjb) * GC(in_b, j0) * GF(i0, jn_b) +
                      zi * conj(zjb) * GC(i0, j0) * GF(in_b, jn_b) + conj(zi) * zjb * GC(in_b, jn_b) * GF(i0, j0)) * fn;
            c->zbb_bin[k] += bbv * zphi;
            c->pair_nn_bin[k] += GF(i0, j0) * GF(in_b, jn_b) * zphi;
            c->pair_sn_bin[k] += GF(i0, j0) * GF(in_s, jn_s) * zphi;
        }
    }
    c->zj_bin += zj * zphi;
    c->zb_bin += zb * zphi;
#undef GC
#undef GF
}

int orc_bins_size(const orc_model *m) {
    /* complex entries: energy 10 + 4 arrays lq*4 + 4 arrays lq + zn 2 + zj + zb ; plus nobs */
    return 2 * (10 + 16 * m->lq + 4 * m->lq + 4) + 1;
}

void orc_get_bins(const orc_chain *c, double *out) {
    int lq = c->m->lq;
    zc *o = (zc *)out;
    size_t k = 0;
    for (int i = 0; i < 10; ++i) o[k++] = c->energy_bin[i];
    memcpy(o + k, c->zcpcm_bin, sizeof(zc) * lq * 4); k += lq * 4;
    memcpy(o + k, c->zspsm_bin, sizeof(zc) * lq * 4); k += lq * 4;
    memcpy(o + k, c->znn_bin, sizeof(zc) * lq * 4); k += lq * 4;
    memcpy(o + k, c->pair_onsite_bin, sizeof(zc) * lq * 4); k += lq * 4;
    memcpy(o + k, c->zjj_bin, sizeof(zc) * lq); k += lq;
    memcpy(o + k, c->zbb_bin, sizeof(zc) * lq); k += lq;
    memcpy(o + k, c->pair_nn_bin, sizeof(zc) * lq); k += lq;
    memcpy(o + k, c->pair_sn_bin, sizeof(zc) * lq); k += lq;
    o[k++] = c->zn_bin[0]; o[k++] = c->zn_bin[1]; o[k++] = c->zj_bin; o[k++] = c->zb_bin;
    out[2 * k] = c->nobs;
}

/* ------------------------------------------------------------------ */
/* sweeps                                                              */
/* ------------------------------------------------------------------ */
static void h0_half(orc_chain *c, int left_op, int right_op, int reversed) {
    const orc_model *m = c->m;
    int N = m->ndim, nnf = m->L.nn_nf;
    if (!m->lwrapT) return;
    if (m->p.kinetic == ORC_CHECKERBOARD) {
        for (int k = 1; k <= nnf; ++k) {
            int nf = reversed ? nnf + 1 - k : k;
            h0_cb(m, right_op, nf, c->gf, N);
            h0_cb(m, left_op, nf, c->gf, N);
        }
    } else {
        h0_fft(m, right_op, c->gf, N);
        h0_fft(m, left_op, c->gf, N);
    }
}

static void record_wrap(orc_chain *c, const zc *gtmp, zc logw) {
    int N = c->m->ndim;
    double err = orc_compare_max(N, gtmp, c->gf);
    if (c->trace_g && c->trace_n < c->trace_cap) {
        memcpy(c->trace_g + (size_t)c->trace_n * N * N, gtmp, sizeof(zc) * (size_t)N * N);
        c->trace_err[c->trace_n++] = err;
    }
    if (err > c->max_wrap_error) c->max_wrap_error = err;
    zc ph = orc_set_phase(c, logw);
    double pd = cabs(c->phase - ph);
    if (pd > c->max_phasediff) c->max_phasediff = pd;
    c->logcount += 1.0;
    c->avglog10error += log10(err);
    c->avgexpphasediff += exp(pd);
    memcpy(c->gf, gtmp, sizeof(zc) * (size_t)N * N);
    c->logweightf = logw;
    c->phase = ph;
}

/* dqmc_ft_sweep_b0 (src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:1-216); nslices
 * limits the sweep to its first nslices time slices (bounded CPU samples). */
int orc_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices);
int orc_sweep_b0(orc_chain *c, int lupdate, int lmeasure) { return orc_sweep_b0_slices(c, lupdate, lmeasure, c->m->ltrot); }
int orc_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices) {
    const orc_model *m = c->m;
    int N = m->ndim, nst = m->nst;
    zc *gtmp = zalloc((size_t)N * N), *ur = zalloc((size_t)N * N), *vr = zalloc((size_t)N * N);
    double *dr = calloc(N, sizeof(double));
    if (nst > 0) {
        memset(c->Ust[nst], 0, sizeof(zc) * (size_t)N * N);
        memset(c->Vst[nst], 0, sizeof(zc) * (size_t)N * N);
        for (int i = 0; i < N; ++i) { c->Ust[nst][ZIDX(i, i, N)] = 1; c->Vst[nst][ZIDX(i, i, N)] = 1; c->Dst[nst][i] = 1; }
        c->logdetQst[nst] = 0;
    }
    for (int nt = m->ltrot; nt >= 1 && nt > m->ltrot - nslices; --nt) {
        if (lmeasure) orc_measure(c, nt);
        h0_half(c, ORC_LEFT_BACKWARD, ORC_RIGHT_FORWARD, 0);
        if (m->lwrapu) {
            if (lupdate) orc_update(c, nt, NULL);
            u_prop(m, c->conf, ORC_RIGHT_FORWARD, nt, c->gf, N);
            u_prop(m, c->conf, ORC_LEFT_BACKWARD, nt, c->gf, N);
        }
        if (m->lwrapv)          /* dqmc_ft_sweep_b0.f90:79-90 */
            for (int nf = m->L.nn_nf; nf >= 1; --nf) {
                orc_v_prop(m, c->vconf, ORC_RIGHT_FORWARD, nt, nf, 2, c->gf, N);
                orc_v_prop(m, c->vconf, ORC_LEFT_BACKWARD, nt, nf, 2, c->gf, N);
                if (lupdate) orc_ft_update_v(c, nt, nf);
                orc_v_prop(m, c->vconf, ORC_RIGHT_FORWARD, nt, nf, 1, c->gf, N);
                orc_v_prop(m, c->vconf, ORC_LEFT_BACKWARD, nt, nf, 1, c->gf, N);
            }
        if (m->lwrapplqu)       /* dqmc_ft_sweep_b0.f90:91-101 */
            for (int i = m->lq - 1; i >= 0; --i) {
                if (lupdate) orc_plq_update(c, i, nt);
                orc_plq_prop(m, c->conf_plq, ORC_RIGHT_FORWARD, i, nt, c->gf, N);
                orc_plq_prop(m, c->conf_plq, ORC_LEFT_BACKWARD, i, nt, c->gf, N);
            }
        h0_half(c, ORC_LEFT_BACKWARD, ORC_RIGHT_FORWARD, 1);
        if ((m->iwrap_nt[nt - 1] > 0 || m->p.nwrap == 1) || nt == 1) {
            int n = m->iwrap_nt[nt - 1];
            memcpy(ur, c->Ust[n], sizeof(zc) * (size_t)N * N);
            memcpy(vr, c->Vst[n], sizeof(zc) * (size_t)N * N);
            memcpy(dr, c->Dst[n], sizeof(double) * N);
            zc ldr = c->logdetQst[n];
            orc_stablize_b0(c, n + 1);
            zc lw;
            green_equaltime(N, ur, dr, vr, c->Vst[n], c->Dst[n], c->Ust[n], gtmp, ldr, c->logdetQst[n], &lw);
            record_wrap(c, gtmp, lw);
        }
    }
    free(gtmp); free(ur); free(vr); free(dr);
    return 0;
}

/* Bmat_right_backward (src/dqmc_ft_core.f90:234-288): g * B(nt1,nt2)^-1 */
static void bmat_right_backward(const orc_chain *c, int nt1, int nt2, zc *g) {
    const orc_model *m = c->m;
    int N = m->ndim, nnf = m->L.nn_nf;
    int cb = (m->p.kinetic == ORC_CHECKERBOARD);
    for (int nt = nt2; nt <= nt1; ++nt) {
        if (m->lwrapT) {
            if (cb) for (int nf = 1; nf <= nnf; ++nf) h0_cb(m, ORC_RIGHT_BACKWARD, nf, g, N);
            else h0_fft(m, ORC_RIGHT_BACKWARD, g, N);
        }
        if (m->lwrapplqu)
            for (int i = 0; i < m->lq; ++i) orc_plq_prop(m, c->conf_plq, ORC_RIGHT_BACKWARD, i, nt, g, N);
        v_slice(c, ORC_RIGHT_BACKWARD, nt, 0, g);
        if (m->lwrapu) u_prop(m, c->conf, ORC_RIGHT_BACKWARD, nt, g, N);
        if (m->lwrapT) {
            if (cb) for (int nf = nnf; nf >= 1; --nf) h0_cb(m, ORC_RIGHT_BACKWARD, nf, g, N);
            else h0_fft(m, ORC_RIGHT_BACKWARD, g, N);
        }
    }
}

/* z = v diag(d or 1/d) u  (or u^H): s_v_d_u, s_v_invd_u, s_v_d_uH, s_v_invd_uH
 * (lib/s_matrix.f90:597-719) */
static void v_d_u(int N, const zc *v, const double *d, int inv, const zc *u, char tu, zc *z) {
    zc *vd = zalloc((size_t)N * N);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) vd[ZIDX(i, j, N)] = inv ? v[ZIDX(i, j, N)] / d[j] : v[ZIDX(i, j, N)] * d[j];
    orc_zgemm('N', tu, N, N, N, 1.0, vd, N, u, N, 0.0, z, N);
    free(vd);
}

/* green_tau (src/dqmc_ft_core/green_tau.f90:1-136): G(tau,tau), G(tau,0),
 * G(0,tau), G(0,0) from the right (ure, dre, vre) and left (ule, dle, vle)
 * factors */
static int green_tau(int N, const zc *ure, const double *dre, const zc *vre, const zc *vle, const double *dle,
                     const zc *ule, zc *g00, zc *gt0, zc *g0t, zc *gtt, zc logdetqr, zc logdetql, zc *logw) {
    double *drmax = malloc(sizeof(double) * N), *drmin = malloc(sizeof(double) * N);
    double *dlmax = malloc(sizeof(double) * N), *dlmin = malloc(sizeof(double) * N);
    size_t NN = (size_t)N * N;
    zc *vlh = zalloc(NN), *uu = zalloc(NN), *vv = zalloc(NN), *dvvd = zalloc(NN), *bt = zalloc(NN), *vri = zalloc(NN);
    dvec_min_max(N, dre, drmax, drmin);
    dvec_min_max(N, dle, dlmax, dlmin);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) vlh[ZIDX(i, j, N)] = conj(vle[ZIDX(j, i, N)]);
    orc_zgemm('C', 'N', N, N, N, 1.0, ure, N, ule, N, 0.0, uu, N);     /* uutmp = ure^H ule */
    orc_zgemm('N', 'C', N, N, N, 1.0, vre, N, vle, N, 0.0, vv, N);     /* vvtmp = vre vle^H */
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
            dvvd[ZIDX(i, j, N)] = uu[ZIDX(i, j, N)] / (drmax[i] * dlmax[j]) + vv[ZIDX(i, j, N)] * drmin[i] * dlmin[j];
    zc zl;
    orc_zinv_logdet(N, dvvd, &zl);
    v_d_u(N, ule, dlmax, 1, dvvd, 'N', bt);
    v_d_u(N, bt, drmax, 1, ure, 'C', gtt);
    double r1 = 0, r2 = 0;
    for (int i = 0; i < N; ++i) r1 += log(dlmax[i]);
    for (int i = 0; i < N; ++i) r2 += log(drmax[i]);
    *logw = -logdetql + logdetqr + zl + (r1 + r2);
    v_d_u(N, bt, drmin, 0, vre, 'N', gt0);                             /* g(t,0) */
    memcpy(vri, vre, sizeof(zc) * NN);
    orc_zinv(N, vri);                                                  /* vre^-1 */
    orc_zinv(N, vlh);                                                  /* (vle^H)^-1 */
    orc_zgemm('N', 'N', N, N, N, 1.0, vlh, N, vri, N, 0.0, vv, N);     /* (vre vle^H)^-1 */
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
            dvvd[ZIDX(i, j, N)] = vv[ZIDX(i, j, N)] / (dlmax[i] * drmax[j]) + conj(uu[ZIDX(j, i, N)]) * dlmin[i] * drmin[j];
    orc_zinv(N, dvvd);
    v_d_u(N, vri, drmax, 1, dvvd, 'N', bt);
    v_d_u(N, bt, dlmax, 1, vlh, 'N', g00);                             /* g(0,0) */
    for (int i = 0; i < N; ++i) dlmin[i] = -dlmin[i];
    v_d_u(N, bt, dlmin, 0, ule, 'C', g0t);                             /* g(0,t) */
    free(drmax); free(drmin); free(dlmax); free(dlmin);
    free(vlh); free(uu); free(vv); free(dvvd); free(bt); free(vri);
    return 0;
}

/* dyn_measure (src/dqmc_measure/dyn_measure.f90:1-101): the density-density
 * correlation znn_tau(imj, no_i, no_j, nt), the only active observable.  On
 * the cubic lattice (dyn_measure3d.f90:44-66) also zspsm_tau(imj, nt) +=
 * -G(0,t)_ji G(t,0)_ij (1 - 1/nflr^2) and gtau0(imj, nt) += G(t,0)_ij, kept in
 * the (no_i, no_j) = (2, 1) and (1, 2) slots of the 2D layout. */
static void dyn_measure(orc_chain *c, int nt, const zc *gt0, const zc *g0t, const zc *gtt, const zc *g00) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    int N = m->ndim, lq = m->lq;
    if (nt > m->ntdm + 1) return;     /* outside znn_tau's nt range (dyntau < beta) */
    double sgn = creal(c->phase) < 0.0 ? -1.0 : 1.0;
    zc zphi = (sgn / creal(c->phase)) * c->phase;
    zc *z = zalloc((size_t)lq * 4);
    for (int j = 0; j < N; ++j) {
        int nu_j = L->list[j * 2 + 0], no_j = L->list[j * 2 + 1];
        for (int i = 0; i < N; ++i) {
            int nu_i = L->list[i * 2 + 0], no_i = L->list[i * 2 + 1];
            int imj = L->imj[(nu_i - 1) * L->ncell + (nu_j - 1)];
            const int d3 = L->kind == ORC_CUBIC || L->kind == ORC_R_CUBIC;   /* orbital pairs summed */
            z[(imj - 1) + (d3 ? 0 : lq * (no_i - 1) + 2 * lq * (no_j - 1))] +=
                (0.5 - creal(gtt[ZIDX(i, i, N)])) * (0.5 - creal(g00[ZIDX(j, j, N)]))
                - (1.0 / m->p.nflr) * g0t[ZIDX(j, i, N)] * gt0[ZIDX(i, j, N)];
            if (d3) {
                const double fsp = 1.0 - 1.0 / (double)(m->p.nflr * m->p.nflr);
                z[(imj - 1) + lq] += -g0t[ZIDX(j, i, N)] * gt0[ZIDX(i, j, N)] * fsp;
                z[(imj - 1) + 2 * lq] += gt0[ZIDX(i, j, N)];
            }
        }
    }
    zc *bin = c->znn_tau_bin + (size_t)4 * lq * (nt - 1);
    for (int k = 0; k < 4 * lq; ++k) bin[k] += z[k] * zphi;
    free(z);
}

/* The unequal-time pass of dqmc_sweep (src/dqmc_ft_ctrl.f90:97-101):
 * push_stage, dqmc_ft_sweep_0b(lupdate = F, lmeasure_equaltime = F,
 * lmeasure_dyn = T) with dyn.f90 and green_tau at the stabilisation points,
 * pop_stage (src/dqmc_ft_core.f90:290-312). */
int orc_sweep_dyn(orc_chain *c) {
    const orc_model *m = c->m;
    int N = m->ndim, nst = m->nst;
    size_t NN = (size_t)N * N;
    if (!m->p.ltau) return -1;
    for (int n = 0; n <= nst; ++n) {   /* push_stage */
        memcpy(c->Ust_b[n], c->Ust[n], sizeof(zc) * NN);
        memcpy(c->Vst_b[n], c->Vst[n], sizeof(zc) * NN);
        memcpy(c->Dst_b[n], c->Dst[n], sizeof(double) * N);
        c->logdetQst_b[n] = c->logdetQst[n];
    }
    memcpy(c->gf_b, c->gf, sizeof(zc) * NN);
    zc *gtmp = zalloc(NN), *ul = zalloc(NN), *vl = zalloc(NN);
    double *dl = calloc(N, sizeof(double));
    if (nst > 0) {
        memset(c->Ust[0], 0, sizeof(zc) * NN);
        memset(c->Vst[0], 0, sizeof(zc) * NN);
        for (int i = 0; i < N; ++i) { c->Ust[0][ZIDX(i, i, N)] = 1; c->Vst[0][ZIDX(i, i, N)] = 1; c->Dst[0][i] = 1; }
        c->logdetQst[0] = 0;
    }
    memcpy(c->g00, c->gf, sizeof(zc) * NN);
    memcpy(c->gt0, c->gf, sizeof(zc) * NN);
    memcpy(c->g0t, c->gf, sizeof(zc) * NN);
    for (int i = 0; i < N; ++i) c->g0t[ZIDX(i, i, N)] -= 1.0;
    dyn_measure(c, 1, c->gt0, c->g0t, c->gf, c->g00);
    for (int nt = 1; nt <= m->ltrot; ++nt) {
        h0_half(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 0);
        if (m->lwrapplqu)       /* dqmc_ft_sweep_0b.f90:82-93 without updates */
            for (int i = 0; i < m->lq; ++i) {
                orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD, i, nt, c->gf, N);
                orc_plq_prop(m, c->conf_plq, ORC_RIGHT_BACKWARD, i, nt, c->gf, N);
            }
        if (m->lwrapv)          /* dqmc_ft_sweep_0b.f90:96-106 without updates */
            for (int nf = 1; nf <= m->L.nn_nf; ++nf)
                for (int nflag = 2; nflag >= 1; --nflag) {
                    orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, nflag, c->gf, N);
                    orc_v_prop(m, c->vconf, ORC_RIGHT_BACKWARD, nt, nf, nflag, c->gf, N);
                }
        if (m->lwrapu) {
            u_prop(m, c->conf, ORC_LEFT_FORWARD, nt, c->gf, N);
            u_prop(m, c->conf, ORC_RIGHT_BACKWARD, nt, c->gf, N);
        }
        h0_half(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 1);
        if (m->iwrap_nt[nt] > 0) {
            int n = m->iwrap_nt[nt];
            memcpy(vl, c->Vst[n], sizeof(zc) * NN);
            memcpy(dl, c->Dst[n], sizeof(double) * N);
            memcpy(ul, c->Ust[n], sizeof(zc) * NN);
            zc ldl = c->logdetQst[n];
            orc_stablize_0b(c, n);
            zc lw;
            green_tau(N, c->Ust[n], c->Dst[n], c->Vst[n], vl, dl, ul, c->g00, c->gt0, c->g0t, gtmp,
                      c->logdetQst[n], ldl, &lw);
            record_wrap(c, gtmp, lw);
        } else {
            bmat_left_forward(c, nt, nt, c->gt0);
            bmat_right_backward(c, nt, nt, c->g0t);
        }
        dyn_measure(c, nt + 1, c->gt0, c->g0t, c->gf, c->g00);
    }
    for (int n = 0; n <= nst; ++n) {   /* pop_stage */
        memcpy(c->Ust[n], c->Ust_b[n], sizeof(zc) * NN);
        memcpy(c->Vst[n], c->Vst_b[n], sizeof(zc) * NN);
        memcpy(c->Dst[n], c->Dst_b[n], sizeof(double) * N);
        c->logdetQst[n] = c->logdetQst_b[n];
    }
    memcpy(c->gf, c->gf_b, sizeof(zc) * NN);
    free(gtmp); free(ul); free(vl); free(dl);
    return 0;
}

void orc_dyn_measure(orc_chain *c, int nt, const zc *gt0, const zc *g0t, const zc *gtt, const zc *g00) {
    dyn_measure(c, nt, gt0, g0t, gtt, g00);
}

double orc_chain_max_dyn_error(const orc_chain *c) { return c->max_dyn_error; }

/* znn_tau_bin (lq, 2, 2, ntdm+1), Fortran order, complex as re/im pairs */
int orc_dyn_bins(const orc_chain *c, double *out) {
    if (!c->m->p.ltau) return -1;
    memcpy(out, c->znn_tau_bin, sizeof(zc) * (size_t)c->m->lq * 4 * (c->m->ntdm + 1));
    return 0;
}

/* G(0,0), G(tau,0), G(0,tau) of the last unequal-time pass (any may be NULL) */
int orc_dyn_mats(const orc_chain *c, double *g00, double *gt0, double *g0t) {
    if (!c->m->p.ltau) return -1;
    size_t b = sizeof(zc) * (size_t)c->m->ndim * c->m->ndim;
    if (g00) memcpy(g00, c->g00, b);
    if (gt0) memcpy(gt0, c->gt0, b);
    if (g0t) memcpy(g0t, c->g0t, b);
    return 0;
}

/* green_tau on given factors (for tests) */
int orc_green_tau(int n, const double *ur, const double *dr, const double *vr, const double *vl, const double *dl,
                  const double *ul, double *g00, double *gt0, double *g0t, double *gtt, const double *logdetqr,
                  const double *logdetql, double *logw) {
    zc lw;
    int info = green_tau(n, (const zc *)ur, dr, (const zc *)vr, (const zc *)vl, dl, (const zc *)ul, (zc *)g00,
                         (zc *)gt0, (zc *)g0t, (zc *)gtt, logdetqr[0] + I * logdetqr[1],
                         logdetql[0] + I * logdetql[1], &lw);
    logw[0] = creal(lw); logw[1] = cimag(lw);
    return info;
}

/* dqmc_ft_sweep_0b (src/dqmc_ft_core/dqmc_ft_sweep_0b.f90:1-288), ltau off */
int orc_sweep_0b(orc_chain *c, int lupdate, int lmeasure) {
    const orc_model *m = c->m;
    int N = m->ndim, nst = m->nst;
    zc *gtmp = zalloc((size_t)N * N), *ul = zalloc((size_t)N * N), *vl = zalloc((size_t)N * N);
    double *dl = calloc(N, sizeof(double));
    if (nst > 0) {
        memset(c->Ust[0], 0, sizeof(zc) * (size_t)N * N);
        memset(c->Vst[0], 0, sizeof(zc) * (size_t)N * N);
        for (int i = 0; i < N; ++i) { c->Ust[0][ZIDX(i, i, N)] = 1; c->Vst[0][ZIDX(i, i, N)] = 1; c->Dst[0][i] = 1; }
        c->logdetQst[0] = 0;
    }
    for (int nt = 1; nt <= m->ltrot; ++nt) {
        h0_half(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 0);
        if (m->lwrapplqu)       /* dqmc_ft_sweep_0b.f90:82-93 */
            for (int i = 0; i < m->lq; ++i) {
                orc_plq_prop(m, c->conf_plq, ORC_LEFT_FORWARD, i, nt, c->gf, N);
                orc_plq_prop(m, c->conf_plq, ORC_RIGHT_BACKWARD, i, nt, c->gf, N);
                if (lupdate) orc_plq_update(c, i, nt);
            }
        if (m->lwrapv)          /* dqmc_ft_sweep_0b.f90:96-106 */
            for (int nf = 1; nf <= m->L.nn_nf; ++nf) {
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 2, c->gf, N);
                orc_v_prop(m, c->vconf, ORC_RIGHT_BACKWARD, nt, nf, 2, c->gf, N);
                if (lupdate) orc_ft_update_v(c, nt, nf);
                orc_v_prop(m, c->vconf, ORC_LEFT_FORWARD, nt, nf, 1, c->gf, N);
                orc_v_prop(m, c->vconf, ORC_RIGHT_BACKWARD, nt, nf, 1, c->gf, N);
            }
        if (m->lwrapu) {
            u_prop(m, c->conf, ORC_LEFT_FORWARD, nt, c->gf, N);
            u_prop(m, c->conf, ORC_RIGHT_BACKWARD, nt, c->gf, N);
            if (lupdate) orc_update(c, nt, NULL);
        }
        h0_half(c, ORC_LEFT_FORWARD, ORC_RIGHT_BACKWARD, 1);
        if (lmeasure) orc_measure(c, nt);
        if (m->iwrap_nt[nt] > 0) {
            int n = m->iwrap_nt[nt];
            memcpy(vl, c->Vst[n], sizeof(zc) * (size_t)N * N);
            memcpy(dl, c->Dst[n], sizeof(double) * N);
            memcpy(ul, c->Ust[n], sizeof(zc) * (size_t)N * N);
            zc ldl = c->logdetQst[n];
            orc_stablize_0b(c, n);
            zc lw;
            green_equaltime(N, c->Ust[n], c->Dst[n], c->Vst[n], vl, dl, ul, gtmp, c->logdetQst[n], ldl, &lw);
            record_wrap(c, gtmp, lw);
        }
    }
    free(gtmp); free(ul); free(vl); free(dl);
    return 0;
}
