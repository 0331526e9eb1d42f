/*
 * dqmc_gpu.h -- C ABI of the B200 (sm_100a) DQMC sweep library
 * (sunhubbardmy_b200/_lib/libdqmc_gpu.so).
 *
 * Drop-in boundary for the finite-temperature sweep of sun-hubbard
 * (YuanyueChen/sunhubbardmy).  In the reference the path is reached through
 * Fortran module procedures (no FFI exists); each entry point below names the
 * reference routine whose effect it reproduces, so a Fortran iso_c_binding
 * shim (include/dqmc_gpu_f.f90) can replace them one by one.
 *
 * Conventions
 *  - Matrices are complex128, column-major (Fortran layout), passed as
 *    interleaved double (re, im) arrays of 2*N*N doubles.
 *  - The HS field conf is int32 [ltrot][nsites] with the site index fastest
 *    and values 1..lcomp, i.e. the memory of uconf%conf(nsites, ltrot)
 *    (src/dqmc_config_u.f90:11).
 *  - Every function returns 0 on success and a negative DQMC_E* code on
 *    failure; dqmc_gpu_last_error() describes the last failure.  Calls on one
 *    handle are synchronous and not thread-safe; use one handle per host
 *    thread.  The caller owns every host buffer; the library owns all device
 *    state.
 *  - A handle holds n_chains independent Markov chains (the reference's MPI
 *    ranks) that are advanced together, one CTA per chain.
 */
#ifndef DQMC_GPU_H
#define DQMC_GPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define DQMC_OK 0
#define DQMC_EINVAL (-1)     /* invalid argument / unsupported parameter set */
#define DQMC_ECUDA (-2)      /* CUDA runtime error */
#define DQMC_ENOMEM (-3)     /* device allocation failed */
#define DQMC_ESTATE (-4)     /* call out of order (e.g. sweep before sweep_start) */
/* numerical failure: a zero or non-finite pivot in the QR of a UDV step, of the
 * middle matrix of green_equaltime / green_tau or of UL UR, or a freshly
 * computed Green's function that is not finite.  The reference stops the run
 * there (the LAPACK info /= 0 stops of lib/s_matrix.f90:1260-1267 and
 * src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:188-194); the chain keeps its
 * propagated G, and dqmc_diag.info holds the DQMC_FAIL_* bits per chain. */
#define DQMC_ENUMERIC (-5)
/* a wrap check exceeded the tolerance set by dqmc_gpu_set_checks */
#define DQMC_EWRAP (-6)

/* dqmc_diag.info bits */
#define DQMC_FAIL_SINGULAR 1
#define DQMC_FAIL_NONFINITE 2
#define DQMC_FAIL_WRAP 4

/* enums (compile-time RUNMODE flags of src/make.sys.* turned into values) */
#define DQMC_LATT_SQUARE 1     /* -DSQUARE */
#define DQMC_LATT_HONEYCOMB 2  /* -DHONEYCOMB */
#define DQMC_LATT_CHAIN 3      /* -DCHAIN: l2 = 1, even l1; checkerboard or dense kinetic term */
#define DQMC_LATT_CUBIC 4      /* -DCUBIC: l1 x l2 x l3 (la, lb, lc); checkerboard (even lengths) or dense kinetic term */
#define DQMC_LATT_R_CUBIC 5    /* -DR_CUBIC: rhombohedral stack, six orbitals per cell, interlayer hopping rtd */
#define DQMC_UPD_FAST 0        /* default (no flag) */
#define DQMC_UPD_DELAY 1       /* -DDELAY */
#define DQMC_UPD_SUBMATRIX 2   /* -DSUBMATRIX */
#define DQMC_KIN_CHECKERBOARD 0 /* -DBREAKUP_T */
#define DQMC_KIN_FFT 1          /* -DFFT (square lattice, l1 == l2) */
#define DQMC_KIN_DENSE 2        /* neither: zgemm with the dense exp(-+dtau H0 / 2) */
#define DQMC_HS_EXACT 0        /* -DEXACTHS */
#define DQMC_HS_GENERAL4 1     /* no -DEXACTHS */

/* &model_para and &ctrl_para of dqmc.in (src/model_para.f90:155-218) plus the
 * compile-time choices.  dqmc_params_derive fills the derived fields. */
typedef struct dqmc_params {
    int32_t lattice, l1, l2;
    double beta, dtau, rt, t2, t3, nu, mu, rhub, rv, alpha, theta;
    double xmag, flux_x, flux_y, dimer, rndness;
    int32_t nflr, lproju, lstabilize;
    int32_t nwrap, nsweep, nbin, nublock;
    int32_t update, kinetic, hs;
    /* projective run (dqmc_proj_ctrl instead of dqmc_ft_ctrl), lprojv of
     * &model_para and obs_eqt_mid_len of &ctrl_para (0 = default 1) */
    int32_t proj, lprojv, obs_mid_len;
    /* derived (src/model_para.f90:334-453) */
    int32_t ndim, lq, ltrot, nst, ne, lcomp;
    /* unequal-time measurement: ltau and dyntau of &ctrl_para; ntdm =
     * nint(dyntau / dtau) is derived (src/model_para.f90:455-459) */
    int32_t ltau, ntdm;
    double dyntau;
    /* lc of &model_para: the length along a3 of the cubic and r_cubic
     * lattices (set to 1 on the other lattices by dqmc_params_derive) */
    int32_t l3;
    /* rtd of &model_para (-DR_CUBIC): the hopping of bond family 4 between
     * the layers of the r_cubic lattice (the reference's default is 1) */
    double rtd;
    /* rhub_plq and lprojplqu of &model_para: the plaquette interaction, one
     * HS field per plaquette and slice (hconf, src/dqmc_config_plqu.f90);
     * finite temperature on the square and honeycomb lattices, without the
     * unequal-time pass */
    double rhub_plq;
    int32_t lprojplqu;
} dqmc_params;

/* per-chain diagnostics (src/dqmc_util.f90:15-57, 287-299) */
typedef struct dqmc_diag {
    double phase_re, phase_im;          /* phase of the determinant weight */
    double logweight_re, logweight_im;  /* logweightf */
    double max_wrap_error;              /* max |G_scratch - G_wrapped| */
    double max_phasediff;
    double avglog10error_sum;           /* sum of log10(wrap error) */
    double logcount;                    /* number of wrap checks */
    double avgexpphasediff_sum;
    double accepted, proposed;          /* main_obs(3): site (U) field */
    double nobs;                        /* measurements in the current bin */
    double accepted_v, proposed_v;      /* main_obs(4): bond (t-V) field */
    double blk_proposed, blk_stage1, blk_accepted;   /* global block moves (dqmc_gpu_sweep_learned) */
    double blk_sum_logratio;            /* sum of Re log R over the accepted blocks */
    double blk_err_learned, blk_err_zero;   /* sums over second-stage blocks of (log|R| + dS)^2 and (log|R|)^2 */
    double max_dyn_error;               /* xmax_dyn: projective unequal-time pass, max |G(t,t) propagated - fresh| */
    double dyn_log10_sum, dyn_count;    /* sum of log10 of those checks (avglog10dynerror) and their number */
    double info;                        /* OR of the DQMC_FAIL_* codes this chain raised since reset_diag */
    double restabilized;                /* re-stabilisations of the handle (dqmc_gpu_set_checks) since reset_diag */
    double near_ties;                   /* accept tests with | |Re(R phase)/Re(phase)| - r | < 1e-12: their
                                           outcome may depend on rounding (logged, not altered) */
    double accepted_plq, proposed_plq;  /* main_obs(2): plaquette field */
} dqmc_diag;

typedef struct dqmc_handle dqmc_handle;

/* Host-only: the lattice and kinetic tables the library builds for p, in the
 * reference's 1-based conventions (src/lattice.f90, dqmc_set_h0conf.f90):
 * nnlist[ndim][nn_nf], nnlf_list[nn_lf], list[ndim][2], imj[lq][lq],
 * plq_cord[lq][z_plq], snlist[ndim][nsn] (nsn = 2 chain, 4 square, 6
 * honeycomb, 12 cubic and r_cubic; z_plq = 8 on both 3D lattices, the
 * r_cubic tables of snlist and plq_cord being zeros as the reference leaves
 * them), urt[nn_nf*nn_lf][2][2] complex,
 * exph0k[lq] complex (FFT only).  Any pointer may be NULL.  Needs no GPU. */
int dqmc_model_tables(const dqmc_params* p, int32_t* nnlist, int32_t* nnlf_list, int32_t* list,
                      int32_t* imj, int32_t* plq_cord, int32_t* snlist, double* urt, double* exph0k);

/* Derive ndim, lq, ltrot, nst, ne, lcomp and the default nublock exactly as
 * make_tables does (src/model_para.f90:334-453). */
int dqmc_params_derive(dqmc_params* p);

/* Create n_chains chains on the current CUDA device.  params points to
 * n_params parameter sets; chain c uses params[c % n_params] (all sets must
 * share beta, dtau and nwrap; lattice sizes may differ, and identical sets
 * share one copy of the model tables).  seeds[c] seeds chain c's SFMT generator
 * (spring_sfmt_init, lib/m_spring.f90:187); if draw_conf is nonzero the HS
 * field is drawn from it as dqmc_input_conf does for a fresh start
 * (src/dqmc_config_u/dqmc_input_conf.f90:55-63).  Replaces dqmc_start's
 * set_h0conf / set_conf / input_conf / allocate_core (src/dqmc_ft_ctrl.f90:9-45). */
int dqmc_gpu_create(const dqmc_params* params, int n_params, int n_chains, const int32_t* seeds,
                    int draw_conf, dqmc_handle** out);
int dqmc_gpu_destroy(dqmc_handle* h);
const char* dqmc_gpu_last_error(void);

/* HS field of one chain (uconf%conf; input_conf / output_conf). */
int dqmc_gpu_set_conf(dqmc_handle* h, int chain, const int32_t* conf);
int dqmc_gpu_get_conf(dqmc_handle* h, int chain, int32_t* conf);
/* all chains at once: conf arrays concatenated chain after chain */
int dqmc_gpu_set_conf_all(dqmc_handle* h, const int32_t* conf);
int dqmc_gpu_get_conf_all(dqmc_handle* h, int32_t* conf);

/* Equal-time Green's function G = <c c^+> of one chain (gf%blk1). */
int dqmc_gpu_get_green(dqmc_handle* h, int chain, double* g);
int dqmc_gpu_set_green(dqmc_handle* h, int chain, const double* g);

/* Wrap trace of one chain, the counterpart of the reference's -DTEST_LEVEL3
 * print of the scratch Green's function at every stabilisation
 * (src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:160-179): the next `capacity`
 * recorded wrap checks store the freshly computed G (N x N complex) and the
 * wrap error max|G_fresh - G_propagated|.  capacity 0 stops and frees it. */
int dqmc_gpu_trace_wraps(dqmc_handle* h, int chain, int capacity);
int dqmc_gpu_trace_count(dqmc_handle* h, int chain);
int dqmc_gpu_trace_get(dqmc_handle* h, int chain, int i, double* g, double* err);

/* Entry n = 0..nst of the finite-temperature UDV stack of one chain: Ust(n)
 * and Vst(n) (N x N complex), Dst(n) (N doubles) and logdetQst(n) (one
 * complex), the module arrays of src/dqmc_ft_core.f90:11-19.  Any pointer may
 * be NULL.  DQMC_ESTATE on a projective handle. */
int dqmc_gpu_get_stack(dqmc_handle* h, int chain, int n, double* u, double* d, double* v, double* logdetq);
int dqmc_gpu_set_stack(dqmc_handle* h, int chain, int n, const double* u, const double* d, const double* v,
                       const double* logdetq);

/* Numerical checks of the sweep entry points (sweep_start, sweep_b0/_0b,
 * sweeps, sweeps_multi, sweep_dyn, sweep_learned).  Singular and non-finite
 * Green's functions are always reported (DQMC_ENUMERIC).  wrap_tol > 0 also
 * reports a wrap check (s_compare_max_z at a stabilisation) above wrap_tol, or
 * not finite, as DQMC_EWRAP (0 = no tolerance, the default).  restabilize != 0:
 * instead of returning either code, a call that ends at tau = beta (sweep_0b,
 * sweeps, sweeps_multi, sweep_learned) rebuilds every chain's stack and G
 * from its HS field (dqmc_ft_sweep_start_0b / dqmc_proj_sweep_start_0b) and
 * returns 0 if the rebuilt G is sound; dqmc_diag.restabilized counts these.
 * A call always runs all its sweeps; the status is read at its end. */
int dqmc_gpu_set_checks(dqmc_handle* h, double wrap_tol, int restabilize);

/* dqmc_ft_sweep_start_0b (src/dqmc_ft_core/dqmc_ft_sweep_start_0b.f90): UDV
 * stack 0 -> beta and G(beta, beta). */
int dqmc_gpu_sweep_start(dqmc_handle* h);
/* dqmc_ft_sweep_b0 / dqmc_ft_sweep_0b (src/dqmc_ft_core/dqmc_ft_sweep_*.f90)
 * with lupdate / lmeasure_equaltime (lmeasure_dyn = .false.). */
int dqmc_gpu_sweep_b0(dqmc_handle* h, int lupdate, int lmeasure);
int dqmc_gpu_sweep_0b(dqmc_handle* h, int lupdate, int lmeasure);
/* n x (sweep_b0 + sweep_0b) with updates, the body of dqmc_sweep
 * (src/dqmc_ft_ctrl.f90:80-126) without the bin output. */
int dqmc_gpu_sweeps(dqmc_handle* h, int n, int lmeasure);

/* obser_init (src/dqmc_measure_2d.f90:105-130) and the per-chain bin sums of
 * equaltime_measure before the MPI reduction of equaltime_output.  Layout of
 * out (complex, 2 doubles each): energy_bin[10], zcpcm, zspsm, znn,
 * pair_onsite [lq*4 each, index d + lq*(no_i + 2*no_j), d = imj - 1],
 * zjj, zbb, pair_nn, pair_sn [lq each], zn[2], zj, zb; nbins() complex. */
int dqmc_gpu_obser_init(dqmc_handle* h);
int dqmc_gpu_nbins(dqmc_handle* h, int chain);
int dqmc_gpu_get_bins(dqmc_handle* h, int chain, double* out);
int dqmc_gpu_get_diag(dqmc_handle* h, int chain, dqmc_diag* out);
/* energy_bin(1:10) of every chain (10 complex per chain, chain after chain):
 * the per-sweep series of sign, density, energies and double occupancy. */
int dqmc_gpu_get_energy_all(dqmc_handle* h, double* out);
int dqmc_gpu_reset_diag(dqmc_handle* h);

/* Operator-level entry points of the reference's type-bound procedures
 * (h0conf / uconf, src/dqmc_config_h0.f90:6-31, src/dqmc_config_u.f90:5-29),
 * acting on each chain's current G.  op: 0 left_forward, 1 left_backward,
 * 2 right_forward, 3 right_backward, 4 left_forward_hc; nf: bond family
 * (checkerboard, 1-based; ignored for FFT); nt: time slice (1-based). */
int dqmc_gpu_h0_prop(dqmc_handle* h, int op, int nf);
int dqmc_gpu_u_prop(dqmc_handle* h, int op, int nt);
/* uconf%update(gf, nt): local updates of slice nt on each chain's G
 * (dqmc_update*.f90).  Consumes 2*nsites draws per chain. */
int dqmc_gpu_update(dqmc_handle* h, int nt);
/* equaltime_measure(nt, gf, gfc) on each chain's current G. */
int dqmc_gpu_measure(dqmc_handle* h);
/* set the determinant phase of a chain (global `phase` of model_para) */
int dqmc_gpu_set_phase(dqmc_handle* h, int chain, double re, double im);
/* raw SFMT draws (spring_sfmt_source) of a chain, advancing its generator */
int dqmc_gpu_draw_u32(dqmc_handle* h, int chain, int count, uint32_t* out);
/* SFMT-19937 state of one chain as the reference holds it (lib/m_spring.f90:66-71):
 * 625 int32 words, pt32(0:623) then the read index idx (0..624; 624 = the next
 * draw regenerates the block).  set_rng continues a caller's stream (e.g. a
 * Fortran rank's generator after spring_sfmt_init and its own draws). */
int dqmc_gpu_get_rng(dqmc_handle* h, int chain, int32_t* state);
int dqmc_gpu_set_rng(dqmc_handle* h, int chain, const int32_t* state);

/* Diagnostics: batched complex GEMM C = op(A) op(B) + beta C on per-chain
 * N x N work matrices, and a QR factorisation (R, Q, log det Q) of one; used
 * by the parity tests of the tensor-core kernels.  Matrices are uploaded and
 * downloaded through the work-matrix accessors. */
int dqmc_gpu_set_work(dqmc_handle* h, int chain, int which, const double* m);
int dqmc_gpu_get_work(dqmc_handle* h, int chain, int which, double* m);
int dqmc_gpu_test_zgemm(dqmc_handle* h, int m, int n, int k, int opa, int opb, int a, int b, int c, double beta);
int dqmc_gpu_test_qr(dqmc_handle* h, int a, int q, double* logdetq /* 2 per chain */);

/* Stream-ordered timing helper: average device time (ms) of the last
 * dqmc_gpu_sweeps call, measured with CUDA events on the library's stream. */
double dqmc_gpu_last_sweeps_ms(dqmc_handle* h);
/* n whole sweeps of several handles at once (every handle as in
 * dqmc_gpu_sweeps): each handle's captured sweep runs on its own stream,
 * forked from and joined to the first handle's stream, so that kernels of
 * different handles -- different phases of independent chains -- share the SMs.
 * *ms_out (may be NULL): device ms per sweep between fork and join.  The
 * reference's counterpart is several MPI ranks sharing a node. */
int dqmc_gpu_sweeps_multi(dqmc_handle* const* hs, int nh, int n, int lmeasure, double* ms_out);
/* dqmc_gpu_sweep_start of n handles (1..16) at once
 * (src/dqmc_ft_core/dqmc_ft_sweep_start_0b.f90, dqmc_proj_sweep_start_0b.f90 per
 * handle): every handle's start-up is enqueued on its own stream before any is
 * waited for, so they run concurrently; then each handle's failure status is
 * read as dqmc_gpu_sweep_start reads it. */
int dqmc_gpu_sweep_start_multi(dqmc_handle* const* hs, int n);
/* Number of kernel launches in one captured sweep (b0 + 0b) of dqmc_gpu_sweeps. */
int dqmc_gpu_sweep_kernels(dqmc_handle* h);
/* Average device time (ms) of `reps` back-to-back launches of one sweep kernel
 * over all chains, timed with CUDA events on the library's stream.  op: 0
 * update of slice 1, 1 UDV stabilisation step, 2 equal-time Green's function,
 * 3 kinetic + HS column pass, 4 equal-time measurement, 5 row pass.  Modifies
 * chain state; intended for benchmarks after the timed sweeps. */
int dqmc_gpu_time_op(dqmc_handle* h, int op, int reps, double* ms_out);

/* Unequal-time measurement (params.ltau = 1, finite temperature): the pass
 * dqmc_sweep runs between the b0 and the 0b sweep (src/dqmc_ft_ctrl.f90:97-101):
 * push_stage, dqmc_ft_sweep_0b(lupdate = F, lmeasure_equaltime = F,
 * lmeasure_dyn = T) -- G(tau,0) and G(0,tau) propagated slice by slice
 * (src/dqmc_ft_core/dyn.f90) and recomputed by green_tau at every
 * stabilisation (src/dqmc_ft_core/green_tau.f90), dyn_measure at every time
 * index (src/dqmc_measure/dyn_measure.f90) -- then pop_stage
 * (src/dqmc_ft_core.f90:290-312).  It must follow a b0 sweep, whose left
 * factors it needs (DQMC_ESTATE otherwise); dqmc_gpu_sweeps runs it between the
 * b0 and the 0b sweep of every measured sweep when ltau = 1. */
int dqmc_gpu_sweep_dyn(dqmc_handle* h);
/* znn_tau_bin(lq, 2, 2, ntdm+1) of one chain, Fortran order, complex as
 * (re, im) pairs: 8 lq (ntdm+1) doubles; obser_init clears it. */
int dqmc_gpu_get_dyn_bins(dqmc_handle* h, int chain, double* out);
/* G(0,0), G(tau,0), G(0,tau) (N x N complex, column-major) after the last
 * unequal-time pass, tau = beta; any pointer may be NULL. */
int dqmc_gpu_get_dyn_mats(dqmc_handle* h, int chain, double* g00, double* gt0, double* g0t);

/* Per-kind device time of whole sweeps, the counterpart of the reference's
 * -DTIMING breakdown (src/dqmc_util.f90:287-369, dqmc_timing).  Runs `nsweeps`
 * sweeps (b0 + 0b, updates on, measurement if lmeasure) launch by launch, not
 * as a graph, with a CUDA event after every launch group; the time between
 * consecutive events is charged to the group's kind.  ms[k] receives the total
 * device ms and groups[k] the number of launch groups of kind k, for
 * k < DQMC_PROF_KINDS.  Advances the chains like dqmc_gpu_sweeps. */
#define DQMC_PROF_UPDATE 0    /* local updates (k_update_delay; projective: one window sequence) */
#define DQMC_PROF_STAB 1      /* UDV stabilisation step (k_stab; projective: tall QR) */
#define DQMC_PROF_GREEN 2     /* Green's function (k_green; projective: (UL UR)^-1 and G) */
#define DQMC_PROF_PROP_L 3    /* propagation from the left (G columns; projective: UR) */
#define DQMC_PROF_MEASURE 4   /* equal-time measurement (transpose + k_measure) */
#define DQMC_PROF_PROP_R 5    /* propagation from the right (G rows; projective: UL^T) */
#define DQMC_PROF_BPROD 6     /* B(tau2, tau1) product of a stabilisation */
#define DQMC_PROF_OTHER 7     /* copies, wrap checks, random numbers, recording */
#define DQMC_PROF_KINDS 8
int dqmc_gpu_sweep_profile(dqmc_handle* h, int nsweeps, int lmeasure, double* ms, int* groups);

/* ---------------------------------------------------------------------------
 * Projective (ground-state) path, params.proj = 1 (src/dqmc_proj_ctrl.f90,
 * src/dqmc_proj_core/).  A walker holds UR = B(tau,0) P (ndim x ne),
 * UL = P^H B(beta,tau) (ne x ndim), (UL UR)^-1 and the stack Ust(0:nst).
 * dqmc_gpu_create draws, per walker and in the reference's order, the U field
 * (if rhub != 0), the t-V bond field (if rv != 0;
 * src/dqmc_config_v/dqmc_input_conf.f90:55-63) and the nn_lf*nn_nf hopping
 * perturbations of set_trial_h0 (src/dqmc_config_h0/set_trial_h0.f90), and
 * takes the ne lowest eigenvectors of that trial Hamiltonian as projL = projR
 * (dqmc_set_proj, src/dqmc_proj_core/dqmc_set_proj.f90:1-78).
 * dqmc_gpu_sweep_start / _sweep_b0 / _sweep_0b / _sweeps then run
 * dqmc_proj_sweep_start_0b / dqmc_proj_sweep_b0 / dqmc_proj_sweep_0b, with the
 * equal-time measurement on the obs_eqt_mid_len middle slices.
 * --------------------------------------------------------------------------- */

/* t-V bond field vconf%conf(nsites, nn_nf, ltrot) of one walker: int32
 * [ltrot][nn_nf][ndim], values 1..2; entries with bond index >= nn_lf are kept
 * but unused, as in the reference. */
int dqmc_gpu_set_vconf(dqmc_handle* h, int chain, const int32_t* vconf);
int dqmc_gpu_get_vconf(dqmc_handle* h, int chain, int32_t* vconf);

/* plaquette field hconf%conf_plqu(lq, ltrot) of one chain: int32 [ltrot][lq],
 * plaquette fastest, values 1..lcomp (dqmc_input_plqconf / dqmc_output_plqconf).
 * DQMC_ESTATE when the chain's model has rhub_plq = 0. */
int dqmc_gpu_set_conf_plq(dqmc_handle* h, int chain, const int32_t* conf);
int dqmc_gpu_get_conf_plq(dqmc_handle* h, int chain, int32_t* conf);
/* trial state of one walker: proj (ndim x ndim complex, ascending eigenvectors
 * of the trial Hamiltonian, first ne columns used), w (ndim eigenvalues; may be
 * NULL).  set_trial replaces projL = projR (e.g. with a caller's eigenvectors). */
int dqmc_gpu_get_trial(dqmc_handle* h, int chain, double* proj, double* w);
int dqmc_gpu_set_trial(dqmc_handle* h, int chain, const double* proj);
/* UR (ndim x ne), UL (ne x ndim) and ULRINV (ne x ne) of one walker, column-major
 * complex; any pointer may be NULL. */
int dqmc_gpu_get_proj(dqmc_handle* h, int chain, double* ur, double* ul, double* ulrinv);
int dqmc_gpu_set_proj(dqmc_handle* h, int chain, const double* ur, const double* ul, const double* ulrinv);
/* proj_update(nt, nf, UL, UR, ULRINV) of every walker (nf = 1..nn_nf: bond
 * family of vconf; nf = 0: the U field of uconf), consuming two draws per bond
 * or site (src/dqmc_config_v/dqmc_proj_update_submatrix_LR.f90,
 * src/dqmc_config_u/dqmc_proj_update_submatrix_LR.f90). */
int dqmc_gpu_proj_update(dqmc_handle* h, int nt, int nf);
/* green_equaltime of the projective core (src/dqmc_proj_core/green_equaltime.f90)
 * after a fresh ULRINV = (UL UR)^-1, into each walker's G. */
int dqmc_gpu_proj_green(dqmc_handle* h);
/* Host-only: the trial state dqmc_gpu_create computes for a walker seeded
 * with `seed` (draws the fields first when draw_conf is nonzero, as create
 * does).  proj: ndim x ndim complex; w: ndim.  Needs no GPU. */
int dqmc_trial_state(const dqmc_params* p, int32_t seed, int draw_conf, double* proj, double* w);

/* ---------------------------------------------------------------------------
 * Learned effective action and global block moves.  No counterpart in the
 * reference: an extra Monte Carlo move beside its local updates, which stay
 * the arbiter of every proposal (delayed-acceptance Metropolis-Hastings with the
 * exact determinant ratio as the second stage).
 *
 * The effective action is a 3-layer periodic convolutional network over the
 * (ltrot x L x L) HS field s = +-1 of the square lattice:
 *   h1 = tanh(W1 * s + b1), h2 = tanh(W2 * h1 + b2)  (3x3x3 convolutions over
 *   (t, y, x), 32 channels), S = sum over space-time of w3 . h2 + b3 V.
 * BF16 weights and activations in the tensor-core kernels, FP32 accumulation
 * and FP32 master weights (Adam).  Parameters, flat FP32: W1[27][32], b1[32],
 * W2[27][32 in][32 out], b2[32], w3[32], b3 (tap = 9 (dt+1) + 3 (dy+1) + (dx+1)
 * for the offsets dt, dy, dx in -1..1; a correlation, out(v) = sum W in(v+off)).
 * Fields are int8 +-1 arrays [ltrot][L][L] (x fastest: the site order of conf).
 * --------------------------------------------------------------------------- */
typedef struct dqmc_nn dqmc_nn;
int dqmc_nn_create(int ltrot, int l, int max_batch, uint64_t seed, dqmc_nn** out);
int dqmc_nn_destroy(dqmc_nn* nn);
int dqmc_nn_nparams(void);
int dqmc_nn_set_params(dqmc_nn* nn, const float* theta);
int dqmc_nn_get_params(dqmc_nn* nn, float* theta);
/* S of B host fields */
int dqmc_nn_forward(dqmc_nn* nn, const int8_t* fields, int B, double* S);
/* S of B fields and the gradient of sum_b r_b S_b with respect to the parameters */
int dqmc_nn_gradient(dqmc_nn* nn, const int8_t* fields, int B, const double* r, double* S, float* grad);
/* one Adam step on the centred squared error mean_b (S_b - y_b - mean(S - y))^2 */
int dqmc_nn_train_step(dqmc_nn* nn, const int8_t* fields, const double* y, int B, double lr, double* loss);
/* the same on pairs recorded by the handle (indices idx, targets y) */
int dqmc_nn_train_recorded(dqmc_nn* nn, dqmc_handle* h, const int32_t* idx, const double* y, int B, double lr,
                           double* loss);
/* One Adam step on differences of recorded pairs: minimises the mean of
 * ((S(record idx_b[b]) - S(record idx_a[b])) - dy[b])^2 over the B pairs
 * (2 B <= max_batch).  With idx_b = idx_a + n_chains (the same chain one
 * stabilisation later) and dy the difference of the recorded values, the
 * network learns how the weight changes under one interval of local updates,
 * the scale of a block proposal; no counterpart in the reference. */
int dqmc_nn_train_recorded_pairs(dqmc_nn* nn, dqmc_handle* h, const int32_t* idx_a, const int32_t* idx_b,
                                 const double* dy, int B, double lr, double* loss);

/* Record (HS field as int8 +-1, nflr Re log W) of every chain at every
 * stabilisation of the finite-temperature sweeps into a ring of `capacity`
 * pairs (capacity 0 stops recording).  All chains must have one size. */
int dqmc_gpu_record(dqmc_handle* h, int capacity);
int dqmc_gpu_record_count(dqmc_handle* h);
int dqmc_gpu_record_get(dqmc_handle* h, int i, int8_t* field, double* value);
int dqmc_gpu_record_values(dqmc_handle* h, double* values /* capacity */);

/* n learned sweeps: b0 as dqmc_gpu_sweep_b0 (local updates if lupdate), then 0b with one proposal of an
 * 8 x 4 x 4 block flip (slices x y x x) at the first slice of every other
 * stabilisation interval (which ones alternates at random), each walker at its
 * own random spatial origin.  Square lattice, two-valued HS field (lcomp = 2).
 * seed != 0 reseeds the block-move generator.  Block statistics go to
 * dqmc_diag.blk_*.  Device time per sweep: dqmc_gpu_last_sweeps_ms. */
int dqmc_gpu_sweep_learned(dqmc_handle* h, dqmc_nn* nn, int n, int lupdate, int lmeasure, uint64_t seed);

/* Allocation-free QR factorisation with log det Q.  No counterpart in the
 * reference: it is an extra entry point for host codes that cannot allocate
 * device memory themselves (their device memory comes from a pool they do not
 * control, or they must not allocate once a run has started).  It allocates
 * nothing: the caller passes device pointers to its own buffers and the
 * library uses a fixed scratch area compiled into it (about 0.55 MB, held on
 * every GPU that loads the library until the process exits).
 *   a        device, n x n complex (2*n*n doubles), column-major.  In: the
 *            matrix.  Out: R in the upper triangle (real diagonal) and the
 *            Householder vectors below it (zgeqrf layout, tau not returned).
 *   q        device, n x n complex out: the explicit unitary factor Q.
 *   logdetq  device, one complex (2 doubles) out: log det Q.
 *   stream   cudaStream_t to launch on (NULL = legacy default stream).
 * n must be 1..512; larger n returns DQMC_EINVAL.  The call is asynchronous on
 * `stream`.  The first call on each device looks up the scratch address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the scratch, so calls whose kernels overlap on the GPU
 * (other streams, other host threads) race; serialise them.  Errors are
 * described by dqmc_gpu_noalloc_error(). */
int dqmc_gpu_qr_logdet_noalloc(int n, double* a, double* q, double* logdetq, void* stream);
const char* dqmc_gpu_noalloc_error(void);

#ifdef __cplusplus
}
#endif
#endif
