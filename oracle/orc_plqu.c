/* The plaquette Hubbard-Stratonovich field (hconf), restated from
 * src/dqmc_config_plqu.f90 and src/dqmc_config_plqu/: dqmc_set_plqconf.f90
 * (constants), dqmc_input_plqconf.f90 (the fresh-start draws), the five
 * *_prop.f90 files (one plaquette's z x z block applied to its rows or
 * columns) and dqmc_update_plqu.f90 (the rank-z local update).  Test
 * infrastructure only.
 *
 * One field per plaquette and time slice, conf_plq[(nt-1) lq + i], values
 * 1..lcomp.  The block of plaquette i at field value is is
 * bmat(is) = U exp(i alpha_p eta(is) e) U^H with U, e the eigen-decomposition
 * of the plaquette matrix vstmat (diagonal 1/nn_nf, alpha exp(-+i theta)
 * around the plaquette), alpha_p = sqrt(dtau rhub_plq); under lprojplqu the
 * phases are pi 2 nn_nf is / lcomp instead. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

static zc *zal(size_t n) { return calloc(n ? n : 1, sizeof(zc)); }

/* module parameters etal, gaml of dqmc_config_plqu.f90:44-52 (fields -2, -1, 1, 2) */
static double plq_eta(int is) { return is == 1 ? -sqrt(2.0 * (3.0 + sqrt(6.0))) : is == 2 ? -sqrt(2.0 * (3.0 - sqrt(6.0)))
                                      : is == 3 ? sqrt(2.0 * (3.0 - sqrt(6.0))) : sqrt(2.0 * (3.0 + sqrt(6.0))); }
static double plq_gam(int is) { return (is == 1 || is == 4) ? 1.0 - sqrt(6.0) / 3.0 : 1.0 + sqrt(6.0) / 3.0; }

/* dqmc_set_plqconf (dqmc_set_plqconf.f90:1-200) */
int orc_plq_setup(orc_model *m) {
    const orc_params *p = &m->p;
    const orc_latt *L = &m->L;
    const int z = L->z_plq, nnf = L->nn_nf;
    if (z != 4 && z != 6) return -1;                       /* square and honeycomb plaquettes only */
    int lproj = p->lprojplqu && (double)(int)p->nu == p->nu;  /* model_para.f90:266-272 */
    m->plq_proj = lproj;
    if (lproj) {
        if (L->kind == ORC_HONEYCOMB) m->plq_lcomp = nnf * (int)(p->nflr + fabs(p->nu)) + 1;
        else m->plq_lcomp = (int)(nnf * (0.5 * p->nflr + fabs(p->nu))) + 1;
    } else {
        m->plq_lcomp = 4;
    }
    const int lc = m->plq_lcomp;
    const double ap = sqrt(p->dtau * p->rhub_plq);
    m->plq_alpha = ap;
    /* vstmat: Fortran reshape of the listed values, column by column */
    const zc z0 = 1.0 / nnf, z1 = p->alpha * cexp(-I * p->theta), z1h = p->alpha * cexp(I * p->theta);
    zc v[36];
    if (z == 6) {
        const zc c[36] = {z0, z1, 0, 0, 0, -z1,    z1h, z0, -z1h, 0, 0, 0,   0, -z1, z0, z1, 0, 0,
                          0, 0, z1h, z0, -z1h, 0,   0, 0, 0, -z1, z0, z1,    -z1h, 0, 0, 0, z1h, z0};
        memcpy(v, c, sizeof(c));
    } else {
        const zc c[16] = {z0, z1, 0, -z1,   z1h, z0, -z1h, 0,   0, -z1, z0, z1,   -z1h, 0, z1h, z0};
        memcpy(v, c, sizeof(c));
    }
    double e[6];
    zc u[36];
    orc_eig_he(z, v, e, u);          /* v column-major: v[i + z j] = vstmat(i+1, j+1) */
    m->plq_bmat = zal((size_t)lc * z * z);
    m->plq_bmat_inv = zal((size_t)lc * z * z);
    m->plq_delta = zal((size_t)lc * (lc - 1) * z * z);
    m->plq_phase = zal(lc);
    m->plq_phase_ratio = zal((size_t)lc * (lc - 1));
    m->plq_gam_ratio = calloc((size_t)lc * (lc - 1), sizeof(double));
    const double fac = (L->kind == ORC_HONEYCOMB) ? 1.0 : 0.5;
    for (int is = 1; is <= lc; ++is) {
        const double a = lproj ? M_PI * 2.0 * nnf * is / lc : ap * plq_eta(is);
        zc *b = m->plq_bmat + (size_t)(is - 1) * z * z, *bi = m->plq_bmat_inv + (size_t)(is - 1) * z * z;
        for (int j = 0; j < z; ++j)
            for (int i = 0; i < z; ++i) {
                zc s0 = 0, s2 = 0;
                for (int k = 0; k < z; ++k) {
                    s0 += u[i + z * k] * cexp(I * e[k] * a) * conj(u[j + z * k]);
                    s2 += u[i + z * k] * cexp(-I * e[k] * a) * conj(u[j + z * k]);
                }
                b[i + z * j] = s0;
                bi[i + z * j] = s2;
            }
        m->plq_phase[is - 1] = lproj ? cexp(I * M_PI * (-2.0 * nnf * is) * fac * (p->nflr + p->nu) / lc)
                                     : cexp(I * ap * (-plq_eta(is)) * fac * (p->nflr + p->nu));
    }
    for (int is = 1; is <= lc; ++is)
        for (int iflip = 1; iflip <= lc - 1; ++iflip) {
            const int isp = (is + iflip - 1) % lc + 1;
            const double a = lproj ? M_PI * (2.0 * nnf * isp - 2.0 * nnf * is) / lc : ap * (plq_eta(isp) - plq_eta(is));
            zc *d = m->plq_delta + ((size_t)(is - 1) * (lc - 1) + (iflip - 1)) * z * z;
            for (int j = 0; j < z; ++j)
                for (int i = 0; i < z; ++i) {
                    zc s0 = 0;
                    for (int k = 0; k < z; ++k) s0 += u[i + z * k] * cexp(I * e[k] * a) * conj(u[j + z * k]);
                    d[i + z * j] = (i == j) ? s0 - 1.0 : s0;
                }
            const size_t k2 = (size_t)(is - 1) * (lc - 1) + (iflip - 1);
            m->plq_phase_ratio[k2] = lproj ? cexp(I * M_PI * (2.0 * nnf * is - 2.0 * nnf * isp) * fac * (p->nflr + p->nu) / lc)
                                           : cexp(I * ap * (plq_eta(is) - plq_eta(isp)) * fac * (p->nflr + p->nu));
            m->plq_gam_ratio[k2] = lproj ? 1.0 : plq_gam(isp) / plq_gam(is);
        }
    return 0;
}

void orc_plq_free(orc_model *m) {
    free(m->plq_bmat); free(m->plq_bmat_inv); free(m->plq_delta); free(m->plq_phase);
    free(m->plq_phase_ratio); free(m->plq_gam_ratio);
}

/* one plaquette's block on its rows (left ops, g N x n2, ld N) or columns
 * (right ops, g n2 x N, ld n2):
 *   left_forward: rows <- bmat rows;  left_backward, left_forward_hc: rows <- bmat_inv rows
 *   right_forward: cols <- cols bmat; right_backward: cols <- cols bmat_inv */
void orc_plq_prop(const orc_model *m, const int32_t *conf_plq, int op, int isite, int nt, zc *g, int n2) {
    const orc_latt *L = &m->L;
    const int z = L->z_plq, N = m->ndim;
    const int is = conf_plq[(size_t)(nt - 1) * m->lq + isite];
    const int *pc = &L->plq_cord[isite * z];
    const int inv = (op == ORC_LEFT_BACKWARD || op == ORC_LEFT_FORWARD_HC || op == ORC_RIGHT_BACKWARD);
    const zc *b = (inv ? m->plq_bmat_inv : m->plq_bmat) + (size_t)(is - 1) * z * z;
    zc x[6], y[6];
    if (op == ORC_RIGHT_FORWARD || op == ORC_RIGHT_BACKWARD) {
        for (int r = 0; r < n2; ++r) {
            for (int a = 0; a < z; ++a) x[a] = g[r + (size_t)n2 * (pc[a] - 1)];
            for (int a = 0; a < z; ++a) {
                zc s = 0;
                for (int k = 0; k < z; ++k) s += x[k] * b[k + z * a];
                y[a] = s;
            }
            for (int a = 0; a < z; ++a) g[r + (size_t)n2 * (pc[a] - 1)] = y[a];
        }
    } else {
        for (int col = 0; col < n2; ++col) {
            for (int a = 0; a < z; ++a) x[a] = g[(pc[a] - 1) + (size_t)N * col];
            for (int a = 0; a < z; ++a) {
                zc s = 0;
                for (int k = 0; k < z; ++k) s += b[a + z * k] * x[k];
                y[a] = s;
            }
            for (int a = 0; a < z; ++a) g[(pc[a] - 1) + (size_t)N * col] = y[a];
        }
    }
}

/* dqmc_update_plqu (dqmc_update_plqu.f90:1-86): one plaquette's flip with the
 * rank-z change of G on acceptance */
void orc_plq_update(orc_chain *c, int isite, int nt) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    const int z = L->z_plq, N = m->ndim, lc = m->plq_lcomp;
    const int *pc = &L->plq_cord[isite * z];
    int32_t *cf = &c->conf_plq[(size_t)(nt - 1) * m->lq + isite];
    const int is = *cf;
    const int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
    const int isp = (is + iflip - 1) % lc + 1;
    const size_t k2 = (size_t)(is - 1) * (lc - 1) + (iflip - 1);
    const zc *dl = m->plq_delta + k2 * z * z;
    zc *g = c->gf;
    /* vkmat(i0, :) = -G(P(i0), :) + e_P(i0); vukmat = I + vkmat(:, P) delta */
    zc vpp[36], vu[36], sm[36];
    for (int a = 0; a < z; ++a)
        for (int b = 0; b < z; ++b) vpp[a + z * b] = (a == b ? 1.0 : 0.0) - g[(pc[a] - 1) + (size_t)N * (pc[b] - 1)];
    for (int a = 0; a < z; ++a)
        for (int b = 0; b < z; ++b) {
            zc s = (a == b) ? 1.0 : 0.0;
            for (int k = 0; k < z; ++k) s += vpp[a + z * k] * dl[k + z * b];
            vu[a + z * b] = s;
        }
    zc ld;
    orc_zinv_logdet(z, vu, &ld);               /* vu <- (I + V U)^-1, ld = log det */
    const zc ratio1 = cexp(ld);
    for (int a = 0; a < z; ++a)                /* smat = delta (I + V U)^-1 */
        for (int b = 0; b < z; ++b) {
            zc s = 0;
            for (int k = 0; k < z; ++k) s += dl[a + z * k] * vu[k + z * b];
            sm[a + z * b] = s;
        }
    zc rt = 1.0;
    for (int f = 0; f < m->p.nflr; ++f) rt *= ratio1;
    rt *= m->plq_gam_ratio[k2] * m->plq_phase_ratio[k2];
    const double rre = creal(rt * c->phase) / creal(c->phase);
    const double r = orc_sfmt_stream(&c->rng);
    c->plq_proposed += 1.0;
    if (fabs(rre) > r) {
        c->plq_accepted += 1.0;
        const double w = sqrt(creal(rt * conj(rt)));
        c->phase = c->phase * rt / w;
        /* G <- G - G(:, P) smat V, V(j0, :) = vkmat(j0, :) */
        zc *gp = zal((size_t)N * z), *sv = zal((size_t)z * N);
        for (int a = 0; a < z; ++a)
            for (int i = 0; i < N; ++i) gp[i + (size_t)N * a] = g[i + (size_t)N * (pc[a] - 1)];
        for (int col = 0; col < N; ++col)
            for (int a = 0; a < z; ++a) {
                zc s = 0;
                for (int k = 0; k < z; ++k) {
                    zc vk = -g[(pc[k] - 1) + (size_t)N * col];
                    if (pc[k] - 1 == col) vk += 1.0;
                    s += sm[a + z * k] * vk;
                }
                sv[a + (size_t)z * col] = s;
            }
        for (int col = 0; col < N; ++col)
            for (int i = 0; i < N; ++i) {
                zc s = 0;
                for (int a = 0; a < z; ++a) s += gp[i + (size_t)N * a] * sv[a + (size_t)z * col];
                g[i + (size_t)N * col] -= s;
            }
        free(gp); free(sv);
        *cf = isp;
    }
}

/* dqmc_proj_update_plqu (dqmc_proj_update_plqu.f90:1-90): the projective
 * flip of one plaquette.  UR (N x ne), UL (ne x N), ULRINV = (UL UR)^-1:
 * vkt = delta UR(P,:), vk = vkt ULRINV, ratio det(I + vk UL(:,P)); on
 * acceptance UR(P,:) += vkt and ULRINV -= ULRINV UL(:,P) (I + vk UL(:,P))^-1 vk. */
void orc_plq_proj_update(orc_chain *c, int isite, int nt) {
    const orc_model *m = c->m;
    const orc_latt *L = &m->L;
    const int z = L->z_plq, N = m->ndim, ne = m->ne, lc = m->plq_lcomp;
    const int *pc = &L->plq_cord[isite * z];
    int32_t *cf = &c->conf_plq[(size_t)(nt - 1) * m->lq + isite];
    const int is = *cf;
    const int iflip = (int)ceil(orc_sfmt_stream(&c->rng) * (lc - 1));
    const int isp = (is + iflip - 1) % lc + 1;
    const size_t k2 = (size_t)(is - 1) * (lc - 1) + (iflip - 1);
    const zc *dl = m->plq_delta + k2 * z * z;
    zc *vkt = zal((size_t)z * ne), *vk = zal((size_t)z * ne), vu[36];
    for (int l = 0; l < ne; ++l)
        for (int a = 0; a < z; ++a) {
            zc s = 0;
            for (int k = 0; k < z; ++k) s += dl[a + z * k] * c->UR[(pc[k] - 1) + (size_t)N * l];
            vkt[a + (size_t)z * l] = s;
        }
    for (int l = 0; l < ne; ++l)
        for (int a = 0; a < z; ++a) {
            zc s = 0;
            for (int q = 0; q < ne; ++q) s += vkt[a + (size_t)z * q] * c->ULRINV[q + (size_t)ne * l];
            vk[a + (size_t)z * l] = s;
        }
    for (int a = 0; a < z; ++a)
        for (int b = 0; b < z; ++b) {
            zc s = (a == b) ? 1.0 : 0.0;
            for (int l = 0; l < ne; ++l) s += vk[a + (size_t)z * l] * c->UL[l + (size_t)ne * (pc[b] - 1)];
            vu[a + z * b] = s;
        }
    zc ld;
    orc_zinv_logdet(z, vu, &ld);
    const zc ratio1 = cexp(ld);
    zc rt = 1.0;
    for (int f = 0; f < m->p.nflr; ++f) rt *= ratio1;
    rt *= m->plq_gam_ratio[k2] * m->plq_phase_ratio[k2];
    const double rre = creal(rt * c->phase) / creal(c->phase);
    const double r = orc_sfmt_stream(&c->rng);
    c->plq_proposed += 1.0;
    if (fabs(rre) > r) {
        c->plq_accepted += 1.0;
        const double w = sqrt(creal(rt * conj(rt)));
        c->phase = c->phase * rt / w;
        for (int l = 0; l < ne; ++l)
            for (int a = 0; a < z; ++a) c->UR[(pc[a] - 1) + (size_t)N * l] += vkt[a + (size_t)z * l];
        zc *w2 = zal((size_t)z * ne), *lru = zal((size_t)ne * z);
        for (int l = 0; l < ne; ++l)
            for (int a = 0; a < z; ++a) {
                zc s = 0;
                for (int b = 0; b < z; ++b) s += vu[a + z * b] * vk[b + (size_t)z * l];
                w2[a + (size_t)z * l] = s;
            }
        for (int b = 0; b < z; ++b)
            for (int q = 0; q < ne; ++q) {
                zc s = 0;
                for (int l = 0; l < ne; ++l) s += c->ULRINV[q + (size_t)ne * l] * c->UL[l + (size_t)ne * (pc[b] - 1)];
                lru[q + (size_t)ne * b] = s;
            }
        for (int l = 0; l < ne; ++l)
            for (int q = 0; q < ne; ++q) {
                zc s = 0;
                for (int b = 0; b < z; ++b) s += lru[q + (size_t)ne * b] * w2[b + (size_t)z * l];
                c->ULRINV[q + (size_t)ne * l] -= s;
            }
        free(w2); free(lru);
        *cf = isp;
    }
    free(vkt); free(vk);
}
