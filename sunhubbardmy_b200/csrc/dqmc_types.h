// Device-side descriptors shared by the host code and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DQ_MAX_LCOMP 4
#define DQ_MAX_NNF 8      // bond families
#define DQ_MAX_PLQ_LCOMP 8  // field values of the plaquette field
#define DQ_MAX_PROG 256   // propagation ops per pass (nwrap slices x ops per slice)

// Model tables for one lattice/parameter set (read-only during a sweep).
struct ModelDev {
    int N, lq, nsub, l1, l2, nn_nf, nn_lf, z_plq, nsn;
    int lcomp, nflr, lproju, kinetic, update, nublock, ltrot, nst, nwrap;
    int ntdm;                            // unequal-time bins cover nt = 1 .. ntdm+1 (-1: ltau off)
    int lwrapT, lwrapu, phase_on;        // phase_on: rhub > 0 (set_phase multiplies conf phases)
    double rt, rv, t2, theta;
    int chain;                 // 1D chain: the energy terms of equaltime_measure1d.f90
    int cubic, l3;             // cubic or r_cubic lattice (l3 = 1 otherwise): the observables of equaltime_measure3d.f90
    int cb_split[DQ_MAX_NNF];  // bonds of each family's first disjoint phase (the device bond order)
    // plaquette field (src/dqmc_config_plqu/dqmc_set_plqconf.f90): z x z blocks per field value
    int plq, plq_z, plq_lcomp;
    int rw_u[2], rw_plq[2];    // offsets of the U-field and plaquette words in a slice's draws (0: 0b, 1: b0)
    int rw_pre0;               // words ahead of the U and bond fields' in the 0b layout (the plaquettes')
    int rw_v[2];               // first bond-field word of a slice (0b: family 1 first; b0: family nn_nf first)
    const double2* plq_bmat;   // [lcomp][z*z] column-major
    const double2* plq_bmat_inv;
    const double2* plq_delta;  // [(is-1)(lcomp-1) + iflip-1][z*z]: bmat(isp) bmat(is)^-1 - I
    const double2* plq_phase_ratio;   // [(is-1)(lcomp-1) + iflip-1]
    const double* plq_gam_ratio;
    double plq_phase_angle[DQ_MAX_PLQ_LCOMP];   // arg(phase(is)) for set_phase
    // HS constants (src/dqmc_config_u/dqmc_set_conf.f90)
    double2 bmat[DQ_MAX_LCOMP], bmat_inv[DQ_MAX_LCOMP], phase[DQ_MAX_LCOMP];
    double2 delta[DQ_MAX_LCOMP * (DQ_MAX_LCOMP - 1)];        // [(is-1)*(lc-1) + iflip-1]
    double2 phase_ratio[DQ_MAX_LCOMP * (DQ_MAX_LCOMP - 1)];
    double gam_ratio[DQ_MAX_LCOMP * (DQ_MAX_LCOMP - 1)];     // gaml(isp)/gaml(is) or 1 (lproju)
    double phase_angle[DQ_MAX_LCOMP];                        // arg(phase(is)) for set_phase
    // kinetic
    const int* bond_i1;        // [nn_nf * nn_lf] 0-based (A site)
    const int* bond_i2;        // [nn_nf * nn_lf] 0-based (B site)
    const double2* urt;        // [nn_nf*nn_lf][4]
    const double2* urtm1;
    const double2* exph0k;     // [lq], already divided by lq (FFT normalisation)
    const double2* exph0kinv;
    const double2* exph0kT;    // the same, index k2 + l1 k1 (l1 == l2): rows on adjacent lanes
    const double2* exph0kinvT;
    const double2* urtd;       // dense kinetic: exp(-dtau H0 / 2), N x N (column-major)
    const double2* urtm1d;     // exp(+dtau H0 / 2)
    const double2* tw1;        // [l1] exp(-2 pi i k / l1)
    const double2* tw2;        // [l2]
    // measurement tables (0-based)
    const int* cell_plus;      // [lq][lq]: cell i with imj(i, j) = d, at [d*lq + j]
    const int* nnlist;         // [N][nn_nf]
    const int* snlist;         // [N][nsn]
    const int* plq_cord;       // [lq][z_plq]
    const double2* expar_nn;   // [N][nn_nf]
    // projective path and the t-V bond field (src/dqmc_config_v/dqmc_set_conf.f90)
    int proj, ne, lwrapv, rps;         // rps: random words drawn per time slice by the updates
    double2 vbp[2], vbm[2], vbpi[2], vbmi[2];   // bmat_p, bmat_m and inverses, by field value
    double2 vdp[2], vdm[2];                     // delta_bmat_p(1,is), delta_bmat_m(1,is)
    const int* vrows;          // [nn_nf][2 nn_lf]: rows (i1, i2) of each bond, bonds in order
};

// Per-chain state.  All pointers are device memory.
struct ChainDev {
    const ModelDev* md;        // device pointer to this chain's model
    int N;
    double2* G;                // current equal-time Green's function
    double2* Gnew;             // scratch Green's function
    double2* GT;               // G transposed (written before each measurement)
    double2* W[6];             // N x N work matrices
    double2* U;                // stack (nst+1) x N x N
    double2* V;
    double* D;                 // (nst+1) x N
    double2* logdetQ;          // nst+1
    double2* A;                // delay / submatrix factors N x nublock
    double2* B;
    double2* tau;              // N (Householder scalars)
    double2* T;                // (N/16+1) x 16 x 16 block-reflector factors
    double2* T64;              // (N/64+1) x 64 x 64 factors of the 64-wide blocks
    double2* smallw;           // 128 x N scratch
    double* vecs;              // 8 x N real scratch (norms, dmax/dmin)
    int* perm;                 // N
    int32_t* conf;             // ltrot x N (site fastest), values 1..lcomp
    int32_t* conf_plq;         // ltrot x lq (plaquette fastest): the plaquette field, or null
    uint32_t* sfmt;            // 624 words + index
    uint32_t* rnd;             // random words for the current half sweep
    double2* bins;             // measurement bins (layout: see kern_measure.cu)
    const int* slotmap;        // logical stack slot -> physical slot (shared by all chains)
    double* stats;             // per-chain scalars, see ST_* below
    // projective path (src/dqmc_proj_core.f90:11-19); N x ne matrices have ld N
    double2* UR;               // N x ne
    double2* ULT;              // N x ne, the transpose of UL (ne x N)
    double2* ULRINV;           // ne x ne, (UL UR)^-1
    double2* Pst;              // (nst+1) x N x ne: Ust(0:nst)
    double2* projR;            // N x ne: first ne trial vectors
    double2* projLc;           // N x ne: conj(projL), i.e. UL^T of the left trial state
    double* logwDV;            // nst+2
    int32_t* vconf;            // ltrot x nn_nf x N (bond index fastest), values 1..2
    double2* pw;               // update window scratch
    int* pw_flag;              // per-walker flag: the current window accepted something
    // global block proposals (learned effective action): [0, N) site mask of the
    // block's spatial patch, [N] stage-1 passed, [N+1] accepted, [N+4..N+6]
    // block origin (t, y, x), 0-based
    int* blk;
    double2* Gsave;            // G at the block's first slice
    int32_t* confsave;         // HS field of the block's slices
    // unequal-time measurement (params.ltau): G(tau,0), G(0,tau), G(0,0), the
    // znn_tau bins (lq, 2, 2, ntdm+1) and push_stage copies of the stack and G
    double2* gt0;
    double2* g0t;
    double2* g00;
    double2* dynbins;
    double2* Ub;
    double2* Vb;
    double* Db;
    double2* ldqb;
    double2* Gb;
    double2* URs;              // projective unequal-time pass: the sweep's UR and UL^T, kept aside
    double2* ULTs;
    // numerical-failure reporting (shared by the handle's chains): fail[0] is
    // the OR of the DQ_FAIL_* codes raised since the host last cleared it;
    // ctl[0] is the wrap-error tolerance (0 = none)
    int* fail;
    const double* ctl;
    // wrap trace (dqmc_gpu_trace_wraps): the fresh G and the wrap error of
    // each recorded wrap check, up to trace_cap of them (null: off)
    double2* trace_g;
    double* trace_err;
    int* trace_n;
    int trace_cap;
};

// an accept test |Re(R phase)/Re(phase)| > r whose two sides differ by less than
// this is counted in stats[ST_NEAR_TIE]: its outcome may depend on rounding
#define DQ_NEAR_TIE 1e-12

// numerical-failure codes (stats[ST_INFO] per chain, fail[0] per handle)
enum {
    DQ_FAIL_SINGULAR = 1,      // zero or non-finite pivot: QR of the UDV step, of M in green_equaltime, of UL UR
    DQ_FAIL_NONFINITE = 2,     // the freshly computed Green's function is not finite
    DQ_FAIL_WRAP = 4           // wrap error above the tolerance ctl[0] (or not finite while a tolerance is set)
};

// indices into ChainDev::stats
enum {
    ST_PHASE_RE = 0, ST_PHASE_IM, ST_LOGW_RE, ST_LOGW_IM,
    ST_MAX_WRAP, ST_MAX_PHASEDIFF, ST_AVGLOG10, ST_LOGCOUNT, ST_AVGEXPPD,
    ST_ACC, ST_PROP, ST_NOBS, ST_INFO, ST_LOGDETM_RE, ST_LOGDETM_IM, ST_LAST_WRAP,
    ST_ACCV, ST_PROPV,
    ST_BLK_LR_RE, ST_BLK_LR_IM, ST_BLK_PH_RE, ST_BLK_PH_IM, ST_BLK_PROP, ST_BLK_S1, ST_BLK_ACC,
    ST_BLK_DS, ST_BLK_U2, ST_BLK_SUMLR, ST_BLK_ERR1, ST_BLK_ERR0,
    ST_MAX_DYN,                // xmax_dyn of the projective unequal-time pass
    ST_DYN_LOG10,              // its sum of log10 over the checks (avglog10dynerror) ...
    ST_DYN_COUNT,              // ... and the number of checks (logdyncount)
    ST_GINFO,                  // DQ_FAIL_SINGULAR of the latest Green's-function computation (overwritten by each)
    ST_NEAR_TIE,               // accept tests decided with | |ratio| - r | < DQ_NEAR_TIE
    ST_ACCP, ST_PROPP,         // plaquette field: accepted flips, proposals
    ST_COUNT = 40
};

// propagation op encoding: kind | which << 4 | nf << 8 | nt << 16
enum { PK_CB = 1, PK_FFT = 2, PK_DIAG = 3, PK_VMIX = 4, PK_VSCALE = 5, PK_DENSE = 6,
       PK_PLQ = 7 };    // PK_PLQ: every plaquette's block in turn, nf = 0 ascending, 1 descending
enum { PW_FWD = 0, PW_INV = 1, PW_CONJ = 2 };   // urt/bmat/exph0k, urtm1/bmat_inv/exph0kinv, conj(...)
struct PropProg {
    int n;
    int op[DQ_MAX_PROG];
};
