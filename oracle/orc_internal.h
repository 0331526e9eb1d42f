/* Internal declarations shared by the oracle's C files.  Test infrastructure
 * only (see dqmc_oracle.h). */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H
#include <complex.h>
#include <stdint.h>
#include "dqmc_oracle.h"

typedef double _Complex zc;
#define ZIDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

typedef struct {
    int kind, l1, l2, l3, ncell, nsub, nsites, z_plq, nn_nf, nn_lf, nsn;
    double a1[2], a2[2], b1[2], b2[2];
    int *ulist;      /* [ncell][2] 1-based cell coordinates, ulist[c*2+d]        */
    int *ulist3;     /* cubic: [ncell][3] (i1, i2, i3), ulist3[c*3+d]             */
    int *list;       /* [nsites][2] (cell, orb), 1-based values                  */
    int *cord;       /* [nsites][2] cell coordinates                              */
    double *rcord;   /* [nsites][2]                                               */
    int *nnlist;     /* [nsites][nn_nf] 1-based neighbour (nnlist[i*nn_nf+nf])    */
    int *snlist;     /* [nsites][nsn]                                             */
    int *nnlf_list;  /* [nn_lf] 1-based A sites                                   */
    int *nnveci;     /* [nsites][nn_nf][2]                                        */
    double *nnvecr;  /* [nsites][nn_nf][2]                                        */
    int *imj;        /* [ncell][ncell] imj[i*ncell+j] = imj(i,j), 1-based         */
    int *plq_cord;   /* [ncell][z_plq] plq_cord[id*z_plq+k] = plq_cord(k,id)      */
    int *listk;      /* [ncell][2]                                                */
    zc *zexpiqr;     /* [ncell(site)][ncell(k)] zexpiqr(nk,i) at [i*ncell+nk]    */
} orc_latt;

int  orc_latt_build(orc_latt *L, int kind, int l1, int l2, int l3);
void orc_latt_free(orc_latt *L);
zc   orc_expar(const orc_latt *L, int i, int nf, double xmag, double fx, double fy, double dimer);

struct orc_model {
    orc_params p;
    orc_latt L;
    int ndim, lq, ltrot, nst, nublock, ne;
    int ntdm;        /* nint(dyntau / dtau) when ltau (src/model_para.f90:455-459) */
    int ntauin;      /* (ltrot - ntdm) / 2: first slice of the projective unequal-time window */
    int lwrapT, lwrapu;
    int *iwrap_nt;   /* [ltrot+1] */
    int *wrap_step;  /* [nst][2] 1-based slice range */
    /* HS constants */
    int lcomp;
    double hs_alpha;
    double etal[4], gaml[4];
    zc bmat[4], bmat_inv[4], phase[4];
    zc delta[3 * 4], phase_ratio[3 * 4];   /* [(is-1)*(lcomp-1) + (iflip-1)] */
    /* kinetic */
    zc *urt, *urtm1;          /* [ist][2][2] with urt[ist*4 + (i-1)*2 + (j-1)] */
    zc *exph0k, *exph0kinv;   /* [lq] */
    zc *urtd, *urtm1d;        /* [N*N] dense exp(-+dtau h0mat / 2) */
    zc *tw1, *tw2;            /* DFT twiddles exp(-2 pi i k / l) */
    zc *h0mat;                /* [N*N] */
    zc *expar_nn;             /* [nsites][nn_nf] */
    /* plaquette field (src/dqmc_config_plqu/dqmc_set_plqconf.f90), when rhub_plq != 0 */
    int lwrapplqu, plq_proj, plq_lcomp;
    double plq_alpha;
    zc *plq_bmat, *plq_bmat_inv;   /* [lcomp][z][z] column-major blocks */
    zc *plq_delta;                  /* [lcomp][lcomp-1][z][z]: bmat(isp) bmat(is)^-1 - I */
    zc *plq_phase;                  /* [lcomp] */
    zc *plq_phase_ratio;            /* [(is-1)(lcomp-1) + iflip-1] */
    double *plq_gam_ratio;          /* gaml(isp)/gaml(is), or 1 under lprojplqu */
    /* projective path and the t-V bond field (src/dqmc_config_v/dqmc_set_conf.f90) */
    int proj, lwrapv, obs_mid_len;
    double v_alpha;
    zc vbp[2], vbm[2], vbpi[2], vbmi[2];   /* bmat_p, bmat_m, bmat_p_inv, bmat_m_inv */
    zc vdp[2], vdm[2];                     /* delta_bmat_p(1,is), delta_bmat_m(1,is) */
};

struct orc_chain {
    const orc_model *m;
    orc_sfmt rng;
    int32_t *conf;            /* [ltrot][nsites], site fastest */
    int32_t *conf_plq;        /* [ltrot][lq] plaquette field, plaquette fastest (hconf%conf_plqu) */
    double plq_accepted, plq_proposed;   /* main_obs(2) */
    zc *gf, *gfc;             /* N*N */
    zc **Ust, **Vst;          /* (nst+1) of N*N */
    double **Dst;
    zc *logdetQst;
    zc phase, logweightf;
    double max_wrap_error, max_phasediff, avglog10error, avgexpphasediff, logcount;
    double max_dyn_error;     /* xmax_dyn of the projective unequal-time pass */
    double acc_u, prop_u;
    /* bins */
    int nobs;
    zc energy_bin[10];
    zc *zcpcm_bin, *zspsm_bin, *znn_bin, *pair_onsite_bin;  /* [lq][2][2] */
    zc *zjj_bin, *zbb_bin, *pair_nn_bin, *pair_sn_bin;       /* [lq] */
    zc zn_bin[2], zj_bin, zb_bin;
    /* projective path (src/dqmc_proj_core.f90:11-19) */
    int32_t *vconf;           /* [ltrot][nn_nf][nsites]: vconf%conf(nsites, nn_nf, ltrot) */
    zc *projR, *projL;        /* N x N trial eigenvectors, first ne columns used */
    double *trial_w;          /* trial eigenvalues */
    zc *UR, *UL, *ULRINV;     /* N x ne, ne x N, ne x ne */
    zc **Pst;                 /* Ust(0:nst) of the projective stack, N x ne */
    double *logwDV;           /* logwDV(0:nst) */
    double acc_v, prop_v;     /* main_obs(4) */
    /* unequal-time measurement (ltau): G(0,0), G(tau,0), G(0,tau), the
     * znn_tau_bin(lq,2,2,ntdm+1) bins and the push_stage copies */
    zc *g00, *gt0, *g0t;
    zc *znn_tau_bin;
    zc **Ust_b, **Vst_b, *gf_b, *logdetQst_b;
    double **Dst_b;
    /* test instrumentation: accept tests decided within ORC_NEAR_TIE of the
     * random number, and a trace of (fresh G, wrap error) at every recorded
     * wrap check (the reference's -DTEST_LEVEL3 print of gf_tmp) */
    double near_ties;
    zc *trace_g;
    double *trace_err;
    int trace_cap, trace_n;
};

#define ORC_NEAR_TIE 1e-12
#define ORC_COUNT_TIE(c, ratio_abs, random) \
    do { if (fabs((ratio_abs) - (random)) < ORC_NEAR_TIE) (c)->near_ties += 1.0; } while (0)

/* linear algebra helpers (orc_linalg.c) */
void orc_zgemm(char ta, char tb, int m, int n, int k, zc alpha, const zc *a, int lda,
               const zc *b, int ldb, zc beta, zc *c, int ldc);
void orc_qr_logdet(int n, zc *a, zc *q, zc *r, zc *logdet);                 /* s_zgeQR_logdetQ */
void orc_qrpt_logdet(int n, zc *a, zc *q, zc *r, int32_t *jpvt, zc *logdet); /* s_zgeQRPT_logdetQ */
void orc_zinv_logdet(int n, zc *a, zc *logdet);                              /* s_inv_logdet_lu_z */
void orc_zinv(int n, zc *a);                                                 /* s_invlu_z */
double orc_dznrm2(int n, const zc *x, int incx);
double orc_qr_pqmc(int rdim, int cdim, const zc *amat, zc *qmat);             /* s_zgeQR_pqmc */
void orc_eig_he(int n, const zc *h, double *w, zc *v);                       /* s_eig_he */
/* plaquette field (orc_plqu.c) */
int  orc_plq_setup(orc_model *m);
void orc_plq_free(orc_model *m);
void orc_plq_prop(const orc_model *m, const int32_t *conf_plq, int op, int isite, int nt, zc *g, int n2);
void orc_plq_update(orc_chain *c, int isite, int nt);
void orc_plq_proj_update(orc_chain *c, int isite, int nt);

/* shared with the projective path (orc_dqmc.c) */
zc orc_total_ratio(const orc_model *m, zc ratio1, int is, int iflip, int isp);
zc orc_set_phase(const orc_chain *c, zc logw);
double orc_compare_max(int N, const zc *a, const zc *b);
void orc_dyn_measure(orc_chain *c, int nt, const zc *gt0, const zc *g0t, const zc *gtt, const zc *g00);

/* projective path (orc_proj.c) */
void orc_set_vconf(orc_model *m);
void orc_proj_chain_init(orc_chain *c, int draw_conf);
void orc_proj_chain_free(orc_chain *c);
void orc_v_prop(const orc_model *m, const int32_t *vconf, int op, int nt, int nf, int nflag, zc *g, int n2);
void orc_ft_update_v(orc_chain *c, int nt, int nf);

#endif
