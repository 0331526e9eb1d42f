// Host-side launch wrappers of the CUDA kernels (one CTA or a few CTAs per
// Markov chain; blockIdx.y / blockIdx.x selects the chain).
#pragma once
#include <cuda_runtime.h>
#include "dqmc_types.h"

void launch_prop(const ChainDev* chains, int nchains, int maxN, int mat_id, const PropProg& prog,
                 int right, int ctas_per_chain, cudaStream_t st);
// register-resident FFT pass (square l x l lattice, one site per cell, l = 4, 8, 16) for
// programs of PK_FFT and PK_DIAG ops only; rows = 1: the vectors are the rows of an
// N x N matrix, else its columns (nvec of them)
int prop_fft_eligible(const PropProg& prog);
void launch_prop_fft(const ChainDev* chains, int nchains, int L, int nvec, int mat_id, const PropProg& prog,
                     int rows, int right, int tall, cudaStream_t st);
void launch_sfmt(const ChainDev* chains, int nchains, int slices, cudaStream_t st);
void launch_sfmt_raw(const ChainDev* chains, int chain, int count, cudaStream_t st);
// dir: the sweep direction of the slice's draws (0: 0b, 1: b0; ModelDev::rw_u)
void launch_update(const ChainDev* chains, int nchains, int nt, int visit, cudaStream_t st, int forced = 0, int dir = 0);
// one slice of plaquette-field props and updates (dir 0: the 0b order, 1: the b0 order)
void launch_plq_slice(const ChainDev* chains, int nchains, int maxN, int nt, int visit, int dir, int lupdate,
                      cudaStream_t st);
// the finite-temperature bond-field updates of one family nf at slice nt (dir 0: 0b draws, 1: b0)
void launch_vbond_slice(const ChainDev* chains, int nchains, int maxN, int nt, int nf, int visit, int dir,
                        cudaStream_t st);
// the same, delayed (rank-2 columns flushed by a DMMA GEMM); returns 0 without
// launching when nublock leaves fewer than two delayed columns
int launch_vbond_delay(const ChainDev* chains, int nchains, int nublock, int nt, int nf, int visit, int dir,
                       cudaStream_t st);
// the same delayed (lupdate = 1; the accepted changes flushed by a DMMA GEMM);
// returns 0 without launching when nublock < z
int launch_plq_delay(const ChainDev* chains, int nchains, int nublock, int z, int nt, int visit, int dir,
                     cudaStream_t st);
// the same on the projective path (UR, UL^T, ULRINV)
void launch_plq_proj_slice(const ChainDev* chains, int nchains, int maxNe, int nt, int visit, int dir, int lupdate,
                           cudaStream_t st);
void launch_update_flush(const ChainDev* chains, int nchains, cudaStream_t st);   // G += A B^T alone
// equal-time measurement: G^T into GT (tiled transpose), then the observables
enum { MEAS_ONE_ORBITAL = 0, MEAS_HONEYCOMB = 1, MEAS_CUBIC = 2, MEAS_R_CUBIC = 3 };
void launch_measure(const ChainDev* chains, int nchains, int maxN, int kind, int maxlq, cudaStream_t st);
void launch_bins_clear(const ChainDev* chains, int nchains, int nbins, cudaStream_t st);
void launch_stab_slots(const ChainDev* chains, int nchains, int src, int dst, cudaStream_t st);
void launch_swap_slots(int* slotmap, int n, int spare, cudaStream_t st);
void launch_stack_identity(const ChainDev* chains, int nchains, int slot, cudaStream_t st);
void set_stab_maxN(int n);
void launch_copy_mat(const ChainDev* chains, int nchains, int dst_id, int src_id, int identity, cudaStream_t st);
// stabilisation step: dir 0 = 0b (writes stack n from n-1), 1 = b0 (writes n-1 from n);
// pivoted selects the QR with column pivoting of the first/last step.
void launch_stab(const ChainDev* chains, int nchains, int n, int dir, int pivoted, cudaStream_t st);
// Green's function from the stack entries (r side, l side) into Gnew; mode 0 =
// green_equaltime, 1 = green_equaltimebb (l side = identity)
void launch_green(const ChainDev* chains, int nchains, int nr, int nl, int rmat_u, int rmat_v,
                  int lmat_u, int lmat_v, int mode, cudaStream_t st);
// green_tau: G(tau,tau) into Gnew, G(tau,0), G(0,tau), G(0,0) into gt0, g0t, g00
// (R = slot nr, L = slot nl); new log weight -> stats[ST_LOGDETM_*]
void launch_green_tau(const ChainDev* chains, int nchains, int nr, int nl, cudaStream_t st);
// push_stage (dir 0) / pop_stage (dir 1) of nslots stack slots and G
void launch_stage(const ChainDev* chains, int nchains, int nslots, int dir, cudaStream_t st);
void launch_dyn_init(const ChainDev* chains, int nchains, cudaStream_t st);
// unequal-time measurement of time index nt (1-based): znn_tau
void launch_dyn_measure(const ChainDev* chains, int nchains, int maxN, int nt, cudaStream_t st);
// wrap check: compare Gnew with G, recompute the phase, replace G (record = 0: just replace)
void launch_wrap_check(const ChainDev* chains, int nchains, int record, cudaStream_t st);
// generic batched complex GEMM on per-chain matrices (diagnostics)
// dense kinetic step on matrix mat_id: X <- K X (left), X K (right) or K^T X
// (right side of the transposed tall UL^T), K = urt (which != PW_INV) or urtm1
void launch_kin_dense(const ChainDev* chains, int nchains, int maxN, int mat_id, int which, int right, int tall,
                      cudaStream_t st);
// dst = A B (sub = 0) or dst - A B (sub = 1) for N x N chain matrices (W4 is the scratch)
void launch_chain_gemm(const ChainDev* chains, int nchains, int maxN, int dst_id, int a_id, int b_id, int sub,
                       cudaStream_t st);
// xmax_dyn of |Gnew - G|, then G = Gnew
void launch_dyn_err(const ChainDev* chains, int nchains, cudaStream_t st);
void launch_zgemm_test(const ChainDev* chains, int nchains, int m, int n, int k, int opa, int opb,
                       int a_id, int b_id, int c_id, double beta_re, cudaStream_t st);
void launch_qr_test(const ChainDev* chains, int nchains, int a_id, int q_id, cudaStream_t st);

// projective path (kern_proj.cu, kern_prop.cu)
void set_proj_maxN(int maxN);
// one pass of prog over the N x ne matrix mat_id (right = 1: right multiplications of UL, stored as UL^T)
void launch_prop_tall(const ChainDev* chains, int nchains, int maxN, int mat_id, const PropProg& prog,
                      int right, int ctas_per_chain, cudaStream_t st);
void launch_proj_qr(const ChainDev* chains, int nchains, int mat_id, int dst, int add, cudaStream_t st);
void launch_proj_ulr(const ChainDev* chains, int nchains, int out_id, int logdet, int ia, int ib, cudaStream_t st);
void launch_proj_green(const ChainDev* chains, int nchains, int inv_id, int dst_id, int ctas, cudaStream_t st);
void launch_tall_copy(const ChainDev* chains, int nchains, int dst_id, int src_id, cudaStream_t st);
void launch_proj_update(const ChainDev* chains, int nchains, int nt, int nf, int visit, int dir, int rnd_off,
                        int nwin, int g_rg, int g_fl, cudaStream_t st);

// global block moves and training-pair recording (kern_block.cu)
void launch_blk_setup(const ChainDev* chains, int nchains, const int* org, int L, cudaStream_t st);
void launch_blk_begin(const ChainDev* chains, int nchains, const double* S, const double* u, int t0, int nsl, cudaStream_t st);
void launch_blk_decide(const ChainDev* chains, int nchains, cudaStream_t st);
void launch_blk_end(const ChainDev* chains, int nchains, int t0, int nsl, cudaStream_t st);
void launch_record(const ChainDev* chains, int nchains, int8_t* fields, double* vals, int* count, int capacity, int V,
                   cudaStream_t st);

// set-up eigenproblems on the device (kern_eig.cu): batched cyclic Jacobi of
// Hermitian matrices; return the sweep count, -1 on a CUDA error, -2 without
// convergence
int eig_herm_device(const double2* Hh, int N, int nmat, double2* Vh, double* wh, cudaStream_t st);
int dense_kinetic_device(const double2* Hh, int N, double dtau, double2* d_urt, double2* d_urtm1, cudaStream_t st);
