/*
 * CPU oracle for the DQMC sweep of sun-hubbard (YuanyueChen/sunhubbardmy).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against, and the timed CPU baseline.  Only tests/, the smoke
 * check and the cpu_baseline / reference arm of bench.py may load it.  The
 * product library (sunhubbardmy_b200) never links, loads or calls it.
 *
 * It restates, in plain C99, the Fortran reference's hot path: SFMT RNG
 * (lib/m_spring.f90), square/honeycomb/chain/cubic lattice tables (src/lattice.f90),
 * HS constants (src/dqmc_config_u/dqmc_set_conf.f90), kinetic propagators
 * (checkerboard, FFT and dense; src/dqmc_config_h0/ directory), local updates
 * (src/dqmc_config_u/dqmc_update*.f90), the UDV stack
 * (src/dqmc_ft_core/dqmc_ft_stablize_*.f90, lib/s_matrix.f90), the Green's
 * functions (src/dqmc_ft_core/green_equaltime*.f90, green_tau.f90), the
 * equal-time and unequal-time measurements (src/dqmc_measure/
 * equaltime_measure.f90, equaltime_measure1d.f90, dyn_measure.f90) and the
 * projective core with its unequal-time pass (src/dqmc_proj_core/, in
 * orc_proj.c).
 *
 * Parity status: UNPINNED against reference output.  The reference is Fortran
 * + MPI + MKL; none of the three exist on either machine, and the reference
 * ships no golden vectors or stored outputs.  The oracle is pinned instead by
 * known answers (free-fermion Green's function, atomic limit, an independent
 * SFMT restatement, scipy LAPACK for the linear-algebra kernels, expm for the
 * dense kinetic operators).
 *
 * Matrices are column-major complex128 (Fortran layout), indices 0-based
 * internally; HS-field values are 1..lcomp exactly as in the reference.
 */
#ifndef DQMC_ORACLE_H
#define DQMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------- SFMT-19937 (lib/m_spring.f90:187-379) ---------- */
typedef struct { uint32_t st[624]; int idx; } orc_sfmt;
void     orc_sfmt_init(orc_sfmt *s, int32_t seed);
uint32_t orc_sfmt_u32(orc_sfmt *s);
double   orc_sfmt_stream(orc_sfmt *s);
int32_t  orc_test_seed(int32_t irank);   /* src/dqmc_util.f90:72 under -DTEST */

/* ---------- parameters (src/model_para.f90 &model_para/&ctrl_para) ---------- */
enum { ORC_SQUARE = 1, ORC_HONEYCOMB = 2, ORC_CHAIN = 3, ORC_CUBIC = 4, ORC_R_CUBIC = 5 };
enum { ORC_FAST = 0, ORC_DELAY = 1, ORC_SUBMATRIX = 2, ORC_SUBMATRIX_G = 3, ORC_SUBMATRIX_G_EXACT = 4 };
enum { ORC_CHECKERBOARD = 0, ORC_FFT = 1, ORC_DENSE = 2 };
enum { ORC_HS_EXACT = 0, ORC_HS_GENERAL4 = 1 };

typedef struct {
    int32_t lattice, l1, l2;
    double beta, dtau, rt, t2, t3, nu, mu, rhub, rv, alpha, theta;
    double xmag, flux_x, flux_y, dimer, rndness;
    int32_t nflr, lproju, lstabilize;
    int32_t nwrap, nsweep, nbin, nublock;
    int32_t update, kinetic, hs;
    /* projective run (dqmc_proj_ctrl), lprojv and obs_eqt_mid_len of &ctrl_para */
    int32_t proj, lprojv, obs_mid_len;
    /* unequal-time measurement: ltau and dyntau of &ctrl_para */
    int32_t ltau;
    double dyntau;
    /* lc of &model_para: the 3D lattices' length along a3; rtd: the r_cubic
     * interlayer hopping */
    int32_t l3;
    double rtd;
    /* rhub_plq and lprojplqu of &model_para: the plaquette field */
    double rhub_plq;
    int32_t lprojplqu;
} orc_params;

typedef struct orc_model orc_model;
typedef struct orc_chain orc_chain;

/* Function-pointer hooks for BLAS/LAPACK (Fortran calling convention, no
 * hidden string lengths, e.g. scipy.linalg.cython_* capsules).  Any NULL
 * entry falls back to the oracle's own unblocked restatement. */
typedef void (*orc_zgemm_fn)(const char*, const char*, const int*, const int*, const int*,
                             const void*, const void*, const int*, const void*, const int*,
                             const void*, void*, const int*);
typedef void (*orc_zgeqrf_fn)(const int*, const int*, void*, const int*, void*, void*, const int*, int*);
typedef void (*orc_zgeqp3_fn)(const int*, const int*, void*, const int*, int*, void*, void*, const int*, double*, int*);
typedef void (*orc_zungqr_fn)(const int*, const int*, const int*, void*, const int*, const void*, void*, const int*, int*);
typedef void (*orc_zgetrf_fn)(const int*, const int*, void*, const int*, int*, int*);
typedef void (*orc_ztrtri_fn)(const char*, const char*, const int*, void*, const int*, int*);
void orc_set_lapack(orc_zgemm_fn, orc_zgeqrf_fn, orc_zgeqp3_fn, orc_zungqr_fn, orc_zgetrf_fn, orc_ztrtri_fn);
typedef void (*orc_zheev_fn)(const char*, const char*, const int*, void*, const int*, double*, void*,
                             const int*, double*, int*);
void orc_set_zheev(orc_zheev_fn);

/* ---------- model / chain ---------- */
orc_model *orc_model_new(const orc_params *p);
void       orc_model_free(orc_model *m);
/* derived: ndim, lq, ltrot, nst, nublock, lcomp, nn_nf, nn_lf, nsub, z_plq */
void orc_model_dims(const orc_model *m, int32_t out[10]);
/* lattice tables, 1-based values as in src/lattice.f90 (sizes from dims) */
void orc_model_tables(const orc_model *m, int32_t *nnlist, int32_t *nnlf_list, int32_t *list,
                      int32_t *imj, int32_t *plq_cord, int32_t *snlist);
/* HS constants: bmat[lcomp], bmat_inv[lcomp], delta[(lcomp-1)*lcomp], phase[lcomp],
 * phase_ratio[(lcomp-1)*lcomp], gaml[lcomp], etal[lcomp], alpha */
void orc_model_hs(const orc_model *m, double *bmat, double *bmat_inv, double *delta,
                  double *phase, double *phase_ratio, double *gaml, double *etal, double *alpha);
/* kinetic: urt/urtm1 [nn_nf*nn_lf][2][2] complex (bond-major, Fortran (ist,i,j)) or exph0k */
void orc_model_kinetic(const orc_model *m, double *urt, double *urtm1, double *exph0k, double *exph0kinv);
/* dense hopping matrix h0mat (seth0) */
void orc_model_h0mat(const orc_model *m, double *h0);

orc_chain *orc_chain_new(const orc_model *m, int32_t seed, int draw_conf);
void       orc_chain_free(orc_chain *c);
void orc_chain_set_conf(orc_chain *c, const int32_t *conf);
void orc_chain_get_conf(const orc_chain *c, int32_t *conf);
/* plaquette field conf_plqu(lq, ltrot), plaquette fastest (rhub_plq != 0) */
void orc_chain_set_conf_plq(orc_chain *c, const int32_t *conf);
void orc_chain_get_conf_plq(const orc_chain *c, int32_t *conf);
void orc_chain_set_green(orc_chain *c, const double *g);
void orc_chain_get_green(const orc_chain *c, double *g);
void orc_chain_set_phase(orc_chain *c, double re, double im);
/* diag: [0]=phase.re [1]=phase.im [2]=logw.re [3]=logw.im [4]=max_wrap_error
 * [5]=max_phasediff [6]=avglog10error [7]=logcount [8]=accepted [9]=proposed
 * [10]=accepted bond-field [11]=proposed bond-field */
void orc_chain_get_diag(const orc_chain *c, double *out);   /* 15 doubles; out[12] = near ties, out[13:15] plaquette accepts/proposals */
void orc_chain_trace(orc_chain *c, int cap);
int orc_chain_trace_count(const orc_chain *c);
void orc_chain_trace_get(const orc_chain *c, int i, double *g, double *err);
double orc_chain_uniform(orc_chain *c);

/* drivers (src/dqmc_ft_core/ directory) */
int  orc_sweep_start_0b(orc_chain *c);
int  orc_sweep_b0(orc_chain *c, int lupdate, int lmeasure);
int  orc_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices);
int  orc_sweep_0b(orc_chain *c, int lupdate, int lmeasure);
/* unequal-time pass of dqmc_sweep (push_stage, 0b sweep with dyn_measure, pop_stage) */
int  orc_sweep_dyn(orc_chain *c);
int  orc_dyn_bins(const orc_chain *c, double *out);
int  orc_dyn_mats(const orc_chain *c, double *g00, double *gt0, double *g0t);
int  orc_green_tau(int n, const double *ur, const double *dr, const double *vr, const double *vl, const double *dl,
                   const double *ul, double *g00, double *gt0, double *g0t, double *gtt, const double *logdetqr,
                   const double *logdetql, double *logw);
void orc_obser_init(orc_chain *c);

/* operator-level entry points acting on an explicit N x N matrix */
enum { ORC_LEFT_FORWARD = 0, ORC_LEFT_BACKWARD = 1, ORC_RIGHT_FORWARD = 2,
       ORC_RIGHT_BACKWARD = 3, ORC_LEFT_FORWARD_HC = 4 };
void orc_h0_prop(const orc_model *m, int op, int nf, double *g, int n2);
void orc_u_prop(const orc_model *m, const int32_t *conf, int op, int nt, double *g, int n2);
void orc_bmat_left_forward(const orc_chain *c, int nt1, int nt2, double *g);
void orc_bmat_left_forward_hc(const orc_chain *c, int nt1, int nt2, double *g);
/* one local update of slice nt (1-based) on the chain's G with its RNG;
 * writes the accept flags of each site to acc (may be NULL) */
void orc_update(orc_chain *c, int nt, int32_t *acc);
/* one equal-time measurement of the chain's current G */
void orc_measure(orc_chain *c, int nt);
/* stack access: which=0 U, 1 V; D and logdetQ */
void orc_stack_get(const orc_chain *c, int n, double *u, double *d, double *v, double *logdetq);
void orc_stack_set(orc_chain *c, int n, const double *u, const double *d, const double *v, const double *logdetq);
void orc_stablize_0b(orc_chain *c, int n);
void orc_stablize_b0(orc_chain *c, int n);
/* green_equaltime with explicit operands */
int  orc_green_equaltime(int n, const double *ur, const double *dr, const double *vr,
                         const double *vl, const double *dl, const double *ul,
                         double *g, const double *logdetqr, const double *logdetql, double *logw);

/* bins: energy[20] (10 complex), nobs, then the per-array bins */
int  orc_bins_size(const orc_model *m);
void orc_get_bins(const orc_chain *c, double *out);

/* ---------- projective path (src/dqmc_proj_core/ directory) ----------
 * The chain of a model with proj = 1 holds UR (N x ne), UL (ne x N), (UL UR)^-1
 * and the stack Ust(0:nst) of N x ne matrices; the t-V bond field (rv != 0)
 * is int32 [ltrot][nn_nf][nsites], values 1..2. */
int  orc_proj_sweep_start_0b(orc_chain *c);
int  orc_proj_sweep_b0(orc_chain *c, int lupdate, int lmeasure);
int  orc_proj_sweep_b0_slices(orc_chain *c, int lupdate, int lmeasure, int nslices);
int  orc_proj_sweep_0b(orc_chain *c, int lupdate, int lmeasure);
/* trial state: proj (N x N, ascending eigenvectors of set_trial_h0) and its eigenvalues */
void orc_proj_get_trial(const orc_chain *c, double *proj, double *w);
void orc_proj_set_trial(orc_chain *c, const double *proj);
void orc_proj_get(const orc_chain *c, double *ur, double *ul, double *ulrinv);
void orc_proj_set(orc_chain *c, const double *ur, const double *ul, const double *ulrinv);
void orc_proj_green(orc_chain *c);                  /* gf from UR, UL, ULRINV */
void orc_vconf_get(const orc_chain *c, int32_t *v);
void orc_vconf_set(orc_chain *c, const int32_t *v);
/* one projective update of slice nt (family nf for the bond field, nf = 0 for the site field) */
void orc_proj_update(orc_chain *c, int nt, int nf);
/* explicit flavour of one projective update: ORC_FAST (dqmc_proj_update.f90),
 * ORC_DELAY (dqmc_proj_update_delay.f90), ORC_SUBMATRIX (submatrix-LR, bond
 * field; the site field runs fast), ORC_SUBMATRIX_G (-DDELAYG,
 * dqmc_proj_update_submatrix_G.f90) or ORC_SUBMATRIX_G_EXACT (the same with
 * the exact inverse of the bond's 2 x 2 block) */
void orc_proj_update_flavour(orc_chain *c, int nt, int nf, int flavour);
/* vconf props on an explicit matrix: left ops on N x n2, right ops on n2 x N */
void orc_vconf_prop(const orc_model *m, const int32_t *vconf, int op, int nt, int nf, int nflag, double *g, int n2);
double orc_qr_pqmc_d(int rdim, int cdim, const double *a, double *q);
void orc_eig_he_d(int n, const double *h, double *w, double *v);

/* linear-algebra restatements exposed for pinning against LAPACK */
void   orc_zgeqr2(int m, int n, double *a, int lda, double *tau);
void   orc_zgeqp2(int m, int n, double *a, int lda, int32_t *jpvt, double *tau);
void   orc_zung2r(int m, int n, int k, double *a, int lda, const double *tau);
int    orc_zgetf2(int m, int n, double *a, int lda, int32_t *ipiv);
void   orc_zmcpt(int rdim, int cdim, double *a, int32_t *jpvt);
void   orc_inv_logdet_lu(int n, double *a, double *logdet);

#ifdef __cplusplus
}
#endif
/* xmax_dyn: largest |G(t,t) propagated - G(t,t) fresh| of the projective unequal-time pass */
double orc_chain_max_dyn_error(const orc_chain *c);

#endif
