// Time-slice propagation: the kinetic factor exp(-dtau K/2) (checkerboard
// bond families or FFT) and the diagonal HS factor exp(+-V), applied from the
// left (column pass) or from the right (row pass) to a per-chain N x N matrix.
//
// Reference operators: src/dqmc_config_h0/dqmc_{left,right}_{forward,backward}_prop.f90
// and _hc (checkerboard 18-44, FFT 95-134), src/dqmc_config_u/dqmc_*_prop.f90 (27-32),
// src/dqmc_config_v/dqmc_*_prop.f90 (t-V bond field: per bond U diag(bp, bm) U^T with
// U the 2x2 Hadamard, split at nflag into a mix op PK_VMIX and a scale op PK_VSCALE).
// The projective path propagates UR (N x ne) from the left and UL (ne x N) from the
// right; UL is stored transposed (N x ne), so both are passes over site vectors.
// A pass streams each column (row) of the matrix through shared memory once and
// applies a whole program of such operators to it, so a full slice wrap (or
// an nwrap-slice B product for the stabilisation) costs one read and one write
// of the matrix per side: the pass is HBM/L2-bandwidth bound.
#include "chain_access.cuh"
#include "kernels.h"
#include <cmath>

#define PLQ_ZMAX 6   // sites of a plaquette (honeycomb)

// The PK_PLQ op (the plaquette field, src/dqmc_config_plqu/dqmc_*_prop.f90):
// x <- P_p x (left, vectors are columns) or x <- x P_p (right, vectors are
// rows) for p over the plaquettes in the op's order, P_p the block bmat
// (which = PW_FWD) or bmat_inv of the plaquette's field at slice nt.  The
// plaquettes share sites, so each vector's thread applies them in turn.
DQ_DEV void plq_apply(const ModelDev& md, const int32_t* conf_plq, int which, int desc, int nt, int right,
                      double2* S, int nv, int vs) {
    const int z = md.plq_z, lq = md.lq;
    const double2* Mb = which == PW_INV ? md.plq_bmat_inv : md.plq_bmat;
    const int32_t* cf = conf_plq + (size_t)(nt - 1) * lq;
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        double2* x = S + (size_t)v * vs;
        for (int k = 0; k < lq; ++k) {
            const int p = desc ? lq - 1 - k : k;
            const int* pc = md.plq_cord + p * z;
            const double2* M = Mb + (size_t)(cf[p] - 1) * z * z;
            double2 a[PLQ_ZMAX], y[PLQ_ZMAX];
#pragma unroll
            for (int i = 0; i < PLQ_ZMAX; ++i) if (i < z) a[i] = x[pc[i]];
#pragma unroll
            for (int i = 0; i < PLQ_ZMAX; ++i) {
                if (i >= z) break;
                double2 s = cmk(0, 0);
#pragma unroll
                for (int j = 0; j < PLQ_ZMAX; ++j) {
                    if (j >= z) break;
                    s = right ? cfma(a[j], __ldg(&M[j + z * i]), s) : cfma(__ldg(&M[i + z * j]), a[j], s);
                }
                y[i] = s;
            }
#pragma unroll
            for (int i = 0; i < PLQ_ZMAX; ++i) if (i < z) x[pc[i]] = y[i];
        }
    }
}

// One operator applied to `nv` vectors held in shared memory (vector v at
// S + v*vs, element stride 1).  right = 0: vectors are columns and the operator
// multiplies from the left; right = 1: vectors are rows (x -> x * Op).
__device__ void apply_op(const ModelDev& md, const int32_t* conf, const int32_t* vconf, const int32_t* conf_plq,
                         int code, int right, double2* S, int nv, int vs) {
    const int kind = code & 15, which = (code >> 4) & 15, nf = (code >> 8) & 255, nt = code >> 16;
    const int N = md.N, tid = threadIdx.x, nth = blockDim.x;
    // CB, DIAG and bond-field ops: a thread owns one bond (or site) and applies
    // it to a group of the nv vectors, so the bond's indices and coefficients
    // are loaded once per op instead of once per vector
    if (kind == PK_CB || kind == PK_VMIX || kind == PK_VSCALE) {
        const int lf = md.nn_lf;
        const int ngrp = max(1, min(nv, nth / lf));
        const int per = (nv + ngrp - 1) / ngrp;
        const double h = 1.0 / sqrt(2.0);
        const double2* U = (which == PW_INV) ? md.urtm1 : md.urt;
        const int32_t* vc = (kind == PK_VSCALE) ? vconf + ((size_t)(nt - 1) * md.nn_nf + (nf - 1)) * N : nullptr;
        // a family's bonds come in two phases of disjoint bonds, the second
        // applied after the first (the second is empty unless bonds of the
        // family share a site, as on the r_cubic lattice)
        const int sp = md.cb_split[nf - 1];
        for (int ph = 0; ph < 2; ++ph) {
        const int b0 = ph ? sp : 0, nbp = ph ? lf - sp : sp;
        if (ph) {
            if (nbp == 0) break;
            __syncthreads();
        }
        for (int w = tid; w < nbp * ngrp; w += nth) {
            const int b = b0 + w % nbp, g = w / nbp;
            const int v0 = g * per, v1 = min(nv, v0 + per);
            const int ist = (nf - 1) * lf + b;
            const int i1 = __ldg(&md.bond_i1[ist]), i2 = __ldg(&md.bond_i2[ist]);
            double2 c0, c1, c2, c3;   // x1' = c0 x1 + c1 x2, x2' = c2 x1 + c3 x2
            if (kind == PK_CB) {
                const double2* u = U + 4 * ist;   // u[0]=(1,1) u[1]=(1,2) u[2]=(2,1) u[3]=(2,2)
                if (!right) { c0 = __ldg(&u[0]); c1 = __ldg(&u[1]); c2 = __ldg(&u[2]); c3 = __ldg(&u[3]); }
                else { c0 = __ldg(&u[0]); c1 = __ldg(&u[2]); c2 = __ldg(&u[1]); c3 = __ldg(&u[3]); }
                for (int v = v0; v < v1; ++v) {
                    double2* x = S + (size_t)v * vs;
                    double2 a = x[i1], c = x[i2];
                    if (!right) {
                        x[i1] = cadd(cmul(c0, a), cmul(c1, c));
                        x[i2] = cadd(cmul(c2, a), cmul(c3, c));
                    } else {
                        x[i1] = cadd(cmul(a, c0), cmul(c, c1));
                        x[i2] = cadd(cmul(a, c2), cmul(c, c3));
                    }
                }
            } else if (kind == PK_VMIX) {
                // x <- H x, H = H^T = [[1,1],[1,-1]]/sqrt2 (the same from either side)
                for (int v = v0; v < v1; ++v) {
                    double2* x = S + (size_t)v * vs;
                    double2 a = x[i1], c = x[i2];
                    x[i1] = cadd(cscale(a, h), cscale(c, h));
                    x[i2] = cadd(cscale(a, h), cscale(c, -h));
                }
            } else {
                // x_i1 *= s1(is), x_i2 *= s2(is)
                const int is = __ldg(&vc[b]) - 1;
                const double2 s1 = (which == PW_INV) ? md.vbpi[is] : md.vbp[is];
                const double2 s2 = (which == PW_INV) ? md.vbmi[is] : md.vbm[is];
                for (int v = v0; v < v1; ++v) {
                    double2* x = S + (size_t)v * vs;
                    x[i1] = cmul(s1, x[i1]);
                    x[i2] = cmul(s2, x[i2]);
                }
            }
        }
        }
    } else if (kind == PK_PLQ) {
        plq_apply(md, conf_plq, which, nf, nt, right, S, nv, vs);
    } else if (kind == PK_DIAG) {
        const int32_t* cf = conf + (size_t)(nt - 1) * N;
        const int ngrp = max(1, min(nv, nth / N));
        const int per = (nv + ngrp - 1) / ngrp;
        for (int w = tid; w < N * ngrp; w += nth) {
            const int i = w % N, g = w / N;
            const int v0 = g * per, v1 = min(nv, v0 + per);
            const int is = __ldg(&cf[i]) - 1;
            double2 b = (which == PW_INV) ? md.bmat_inv[is] : md.bmat[is];
            if (which == PW_CONJ) b.y = -b.y;
            for (int v = v0; v < v1; ++v) {
                double2* x = S + (size_t)v * vs;
                x[i] = cmul(x[i], b);
            }
        }
    } else if (kind == PK_FFT) {
        // left:  x <- F^-1 D F x ; right (row r): r <- F D F^-1 r  (F symmetric)
        const int l1 = md.l1, l2 = md.l2, lq = md.lq;
        const double2* d = (which == PW_INV) ? md.exph0kinv : md.exph0k;
        const int s1 = right ? +1 : -1;
        // dim 1: nv*l2 contiguous lines; consecutive threads take different
        // vectors (vector stride vs is odd, so their lines sit in different banks)
        for (int w = tid; w < nv * l2; w += nth) {
            int v = w % nv, j2 = w / nv;
            line_dft(S + (size_t)v * vs + j2 * l1, l1, 1, md.tw1, s1);
        }
        __syncthreads();
        // dim 2: nv*l1 lines of stride l1; consecutive threads take consecutive j1
        for (int w = tid; w < nv * l1; w += nth) {
            int j1 = w % l1, v = w / l1;
            line_dft(S + (size_t)v * vs + j1, l2, l1, md.tw2, s1);
        }
        __syncthreads();
        for (int w = tid; w < nv * lq; w += nth) {
            int v = w / lq, k = w % lq;
            double2 dk = d[k];
            if (which == PW_CONJ) dk.y = -dk.y;
            double2* x = S + (size_t)v * vs;
            x[k] = cmul(x[k], dk);
        }
        __syncthreads();
        for (int w = tid; w < nv * l2; w += nth) {
            int v = w % nv, j2 = w / nv;
            line_dft(S + (size_t)v * vs + j2 * l1, l1, 1, md.tw1, -s1);
        }
        __syncthreads();
        for (int w = tid; w < nv * l1; w += nth) {
            int j1 = w % l1, v = w / l1;
            line_dft(S + (size_t)v * vs + j1, l2, l1, md.tw2, -s1);
        }
    }
    __syncthreads();
}

// Column pass: X <- Op_k ... Op_1 X for the program prog.  tall = 1: X is one
// of the N x ne matrices of the projective path; right = 1 applies the
// operators as right multiplications of the transposed matrix (UL^T).
__global__ void __launch_bounds__(256, 2) k_prop_cols(const ChainDev* __restrict__ chains, int mat_id, PropProg prog, int cb,
                                                      int tall, int right) {
    extern __shared__ double2 sm[];
    const ChainDev c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    const int N = c.N;
    const int ncol = tall ? md.ne : N;
    double2* X = chain_mat(c, mat_id);
    const int vs = N + 1;   // odd vector stride: conflict-free strided lines
    for (int c0 = blockIdx.x * cb; c0 < ncol; c0 += gridDim.x * cb) {
        int nv = min(cb, ncol - c0);
        for (int e = threadIdx.x; e < nv * N; e += blockDim.x) sm[(e / N) * vs + e % N] = X[(size_t)c0 * N + e];
        __syncthreads();
        for (int k = 0; k < prog.n; ++k) apply_op(md, c.conf, c.vconf, c.conf_plq, prog.op[k], right, sm, nv, vs);
        for (int e = threadIdx.x; e < nv * N; e += blockDim.x) X[(size_t)c0 * N + e] = sm[(e / N) * vs + e % N];
        __syncthreads();
    }
}

// Row pass: X <- X Op_1 ... Op_k.  Rows are staged with a padded stride.
__global__ void __launch_bounds__(256, 2) k_prop_rows(const ChainDev* __restrict__ chains, int mat_id, PropProg prog, int rb) {
    extern __shared__ double2 sm[];
    const ChainDev c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    const int N = c.N, vs = N + 1;
    double2* X = chain_mat(c, mat_id);
    for (int r0 = blockIdx.x * rb; r0 < N; r0 += gridDim.x * rb) {
        int nv = min(rb, N - r0);
        for (int e = threadIdx.x; e < nv * N; e += blockDim.x) {
            int r = e % nv, j = e / nv;
            sm[r * vs + j] = X[MIDX(r0 + r, j, N)];
        }
        __syncthreads();
        for (int k = 0; k < prog.n; ++k) apply_op(md, c.conf, c.vconf, c.conf_plq, prog.op[k], 1, sm, nv, vs);
        for (int e = threadIdx.x; e < nv * N; e += blockDim.x) {
            int r = e % nv, j = e / nv;
            X[MIDX(r0 + r, j, N)] = sm[r * vs + j];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// FFT kinetic term with register-resident vectors.  For a square l x l lattice
// with one site per cell (l = 4, 8, 16; site i = j1 + l j2), a group of l
// threads owns one vector: thread g holds the dim-2 line j1 = g (l values) in
// registers.  A PK_FFT op is   dim-2 DFT -> transpose (shared memory, within
// the warp) -> dim-1 DFT -> x exph0k(k) -> inverse dim-1 -> transpose back ->
// inverse dim-2, and a PK_DIAG op scales the registers by the HS factor of its
// sites, so a whole program (an nwrap-slice B product included) costs one read
// and one write of the matrix and two shared-memory transposes per FFT op.
// Columns (rows = 0) are loaded with consecutive threads on consecutive sites;
// rows (rows = 1) with the two rows of a warp on adjacent addresses.
// ---------------------------------------------------------------------------

// x * w with w = exp(-SG 2 pi i m / 16) (SG = +1: forward sign, -1: backward),
// the trivial angles folded at compile time; c1 = cos(pi/8), s1 = sin(pi/8),
// h = cos(pi/4)
template <int SG>
DQ_DEV double2 tw_mul(int m, double2 x, double c1, double s1, double h) {
    double wr, wi;   // forward twiddle exp(-2 pi i m / 16)
    switch (m) {
    case 0: return x;
    case 4: return SG > 0 ? cmk(x.y, -x.x) : cmk(-x.y, x.x);
    case 2: return SG > 0 ? cmk(h * (x.x + x.y), h * (x.y - x.x)) : cmk(h * (x.x - x.y), h * (x.y + x.x));
    case 6: return SG > 0 ? cmk(h * (x.y - x.x), -h * (x.x + x.y)) : cmk(-h * (x.x + x.y), h * (x.x - x.y));
    case 1: wr = c1; wi = -s1; break;
    case 3: wr = s1; wi = -c1; break;
    case 5: wr = -s1; wi = -c1; break;
    default: wr = -c1; wi = -s1; break;   // 7
    }
    if (SG < 0) wi = -wi;
    return cmk(wr * x.x - wi * x.y, wr * x.y + wi * x.x);
}

// unnormalised radix-2 DFT of n <= 16 values in registers, natural order in
// and out; SG = +1: exp(-2 pi i jk/n), SG = -1: exp(+2 pi i jk/n)
template <int n>
DQ_DEV constexpr int bit_reverse(int i) {
    int j = 0;
    for (int b = 1; b < n; b <<= 1, i >>= 1) j = (j << 1) | (i & 1);
    return j;
}

// one radix-2 stage of butterflies of length LEN over n registers
template <int n, int LEN, int SG>
DQ_DEV void fft_stage(double2 (&r)[n], double c1, double s1, double h) {
    constexpr int half = LEN / 2;
#pragma unroll
    for (int s0 = 0; s0 < n; s0 += LEN)
#pragma unroll
        for (int k = 0; k < half; ++k) {
            double2 u = r[s0 + k], v = tw_mul<SG>(k * (16 / LEN), r[s0 + k + half], c1, s1, h);
            r[s0 + k] = cadd(u, v);
            r[s0 + k + half] = csub(u, v);
        }
}

template <int n, int SG>
DQ_DEV void fft_reg(double2 (&x)[n], double c1, double s1, double h) {
    double2 r[n];
#pragma unroll
    for (int i = 0; i < n; ++i) r[bit_reverse<n>(i)] = x[i];
    fft_stage<n, 2, SG>(r, c1, s1, h);
    if constexpr (n >= 4) fft_stage<n, 4, SG>(r, c1, s1, h);
    if constexpr (n >= 8) fft_stage<n, 8, SG>(r, c1, s1, h);
    if constexpr (n >= 16) fft_stage<n, 16, SG>(r, c1, s1, h);
#pragma unroll
    for (int i = 0; i < n; ++i) x[i] = r[i];
}

// SG = +1 for the forward sign exp(-2 pi i jk/n)
template <int L>
DQ_DEV void fft_dir(double2 (&x)[L], int sg, double c1, double s1, double h) {
    if (sg > 0) fft_reg<L, 1>(x, c1, s1, h);
    else fft_reg<L, -1>(x, c1, s1, h);
}

template <int L, bool ROWS>
__global__ void __launch_bounds__(128, 4) k_prop_fft(const ChainDev* __restrict__ chains, int mat_id, PropProg prog,
                                                     int right, int tall, double c1, double s1, double h) {
    constexpr bool rows = ROWS;
    constexpr int VPC = 128 / L;    // vectors per CTA
    constexpr int LD = L + 1;       // odd row pitch: conflict-free transposes
    constexpr int TS = L * LD + 1;  // per-vector region; the +1 spreads the row-tile stores over the banks
    __shared__ double2 tb[VPC * TS];
    const ChainDev& c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    const int N = c.N;
    const int nvec = (tall && !rows) ? md.ne : N;
    double2* X = chain_mat(c, mat_id);
    const int g = threadIdx.x % L, vl = threadIdx.x / L;
    double2* T = tb + vl * TS;
    // left multiplication: F^-1 D F (forward sign first); right: F D F^-1
    const int sg = right ? -1 : 1;
    for (int v0 = blockIdx.x * VPC; v0 < nvec; v0 += gridDim.x * VPC) {
        const int v = v0 + vl;
        const bool act = v < nvec;      // uniform over the l threads of a vector
        double2 x[L];
        if (rows) {
            // Rows are strided by N: stage the (L*L) x VPC tile through shared
            // memory with consecutive threads on consecutive vectors.
            // L * L * VPC = 128 * L: L elements per thread, all loads in flight
#pragma unroll
            for (int k = 0; k < L; ++k) {
                const int e = threadIdx.x + 128 * k, vv = e % VPC, i = e / VPC;
                x[k] = (v0 + vv < nvec) ? X[(size_t)i * N + v0 + vv] : cmk(0, 0);
            }
#pragma unroll
            for (int k = 0; k < L; ++k) {
                const int e = threadIdx.x + 128 * k, vv = e % VPC, i = e / VPC;
                tb[vv * TS + (i / L) * LD + (i % L)] = x[k];
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < L; ++j) x[j] = act ? T[j * LD + g] : cmk(0, 0);
        } else {
#pragma unroll
            for (int j = 0; j < L; ++j) x[j] = act ? X[(size_t)v * N + g + L * j] : cmk(0, 0);
        }
        for (int k = 0; k < prog.n; ++k) {
            const int code = prog.op[k];
            const int kind = code & 15, which = (code >> 4) & 15, nt = code >> 16;
            if (kind == PK_DIAG) {
                const int32_t* cf = c.conf + (size_t)(nt - 1) * N;
                const double2* bt = (which == PW_INV) ? md.bmat_inv : md.bmat;
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    double2 b = bt[__ldg(&cf[g + L * j]) - 1];
                    if (which == PW_CONJ) b.y = -b.y;
                    x[j] = cmul(x[j], b);
                }
                continue;
            }
            // PK_FFT
            const double2* d = (which == PW_INV) ? md.exph0kinvT : md.exph0kT;
            fft_dir<L>(x, sg, c1, s1, h);                 // dim 2: x[k2] at j1 = g
#pragma unroll
            for (int j = 0; j < L; ++j) T[j * LD + g] = x[j];
            __syncwarp();
#pragma unroll
            for (int j = 0; j < L; ++j) x[j] = T[g * LD + j];   // k2 = g, j1 = j
            __syncwarp();
            fft_dir<L>(x, sg, c1, s1, h);                 // dim 1: x[k1] at k2 = g
#pragma unroll
            for (int j = 0; j < L; ++j) {
                double2 dk = __ldg(&d[g + L * j]);       // exph0k(k1 = j, k2 = g)
                if (which == PW_CONJ) dk.y = -dk.y;
                x[j] = cmul(x[j], dk);
            }
            fft_dir<L>(x, -sg, c1, s1, h);                // inverse dim 1
#pragma unroll
            for (int j = 0; j < L; ++j) T[g * LD + j] = x[j];
            __syncwarp();
#pragma unroll
            for (int j = 0; j < L; ++j) x[j] = T[j * LD + g];   // j1 = g, k2 = j
            __syncwarp();
            fft_dir<L>(x, -sg, c1, s1, h);                // inverse dim 2
        }
        if (rows) {
            __syncthreads();            // all warps are done with their transposes
#pragma unroll
            for (int j = 0; j < L; ++j) T[j * LD + g] = x[j];
            __syncthreads();
#pragma unroll
            for (int k = 0; k < L; ++k) {
                const int e = threadIdx.x + 128 * k, vv = e % VPC, i = e / VPC;
                if (v0 + vv < nvec) X[(size_t)i * N + v0 + vv] = tb[vv * TS + (i / L) * LD + (i % L)];
            }
            __syncthreads();            // the tile is free for the next vectors
        } else if (act) {
#pragma unroll
            for (int j = 0; j < L; ++j) X[(size_t)v * N + g + L * j] = x[j];
        }
    }
}

int prop_fft_eligible(const PropProg& prog) {
    for (int k = 0; k < prog.n; ++k) {
        const int kind = prog.op[k] & 15;
        if (kind != PK_FFT && kind != PK_DIAG) return 0;
    }
    return prog.n > 0;
}

void launch_prop_fft(const ChainDev* chains, int nchains, int L, int nvec, int mat_id, const PropProg& prog,
                     int rows, int right, int tall, cudaStream_t st) {
    const double c1 = std::cos(M_PI / 8), s1 = std::sin(M_PI / 8), h = std::sqrt(0.5);
    const int vpc = 128 / L;
    dim3 grid((nvec + vpc - 1) / vpc, nchains);
#define PROP_FFT_CASE(LL)                                                                        \
    if (rows) k_prop_fft<LL, true><<<grid, 128, 0, st>>>(chains, mat_id, prog, right, tall, c1, s1, h); \
    else k_prop_fft<LL, false><<<grid, 128, 0, st>>>(chains, mat_id, prog, right, tall, c1, s1, h);
    switch (L) {
    case 16: PROP_FFT_CASE(16) break;
    case 8: PROP_FFT_CASE(8) break;
    default: PROP_FFT_CASE(4) break;
    }
#undef PROP_FFT_CASE
}

static int g_prop_smem_ok = 0;

void launch_prop(const ChainDev* chains, int nchains, int maxN, int mat_id, const PropProg& prog,
                 int right, int ctas_per_chain, cudaStream_t st) {
    const int nb = 16;
    size_t smem = (size_t)nb * (maxN + 1) * sizeof(double2);
    if (!g_prop_smem_ok) {
        cudaFuncSetAttribute(k_prop_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_prop_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_prop_smem_ok = 1;
    }
    dim3 grid(ctas_per_chain, nchains);
    if (right) k_prop_rows<<<grid, 256, smem, st>>>(chains, mat_id, prog, nb);
    else k_prop_cols<<<grid, 256, smem, st>>>(chains, mat_id, prog, nb, 0, 0);
}

void launch_prop_tall(const ChainDev* chains, int nchains, int maxN, int mat_id, const PropProg& prog,
                      int right, int ctas_per_chain, cudaStream_t st) {
    const int nb = 16;
    size_t smem = (size_t)nb * (maxN + 1) * sizeof(double2);
    if (!g_prop_smem_ok) {
        cudaFuncSetAttribute(k_prop_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_prop_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_prop_smem_ok = 1;
    }
    dim3 grid(ctas_per_chain, nchains);
    k_prop_cols<<<grid, 256, smem, st>>>(chains, mat_id, prog, nb, 1, right);
}
