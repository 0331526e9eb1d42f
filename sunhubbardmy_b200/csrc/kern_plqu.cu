// The plaquette Hubbard-Stratonovich field (hconf): one field per plaquette and
// time slice whose factor is a dense z x z block on the plaquette's z sites
// (z = 4 square, 6 honeycomb).
//
// Reference: src/dqmc_config_plqu/ -- dqmc_left_forward_prop.f90 and its four
// siblings (the block on a plaquette's rows or columns) and
// dqmc_update_plqu.f90 (the flip of one plaquette: ratio det(I + V U) from a
// z x z matrix, G <- G - G(:,P) S V on acceptance), called plaquette by
// plaquette in dqmc_ft_sweep_0b.f90:82-93 (ascending: props, then update) and
// dqmc_ft_sweep_b0.f90:91-101 (descending: update, then props).
//
// Plaquettes share sites, so the blocks of one slice are applied one after the
// other.  In a B product (the PK_PLQ op of kern_prop.cu) every vector of the
// pass walks the plaquettes sequentially in its own thread; in the sweep,
// k_plq_slice runs the interleaved props and updates of one slice for one
// chain per CTA.
#include "chain_access.cuh"
#include "flush.cuh"
#include "kernels.h"

#define PLQ_NT 256
#define PLQ_ZMAX 6

DQ_DEV double plq_stream(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

// rows P of X (ld rows, ncol columns) <- M rows P, or M^T rows P when trans
// (M z x z, column-major)
DQ_DEV void plq_rows(double2* X, int ld, int ncol, const int* pc, int z, const double2* M, bool trans = false) {
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
        double2 a[PLQ_ZMAX];
#pragma unroll
        for (int i = 0; i < PLQ_ZMAX; ++i) if (i < z) a[i] = X[(size_t)pc[i] + (size_t)ld * col];
#pragma unroll
        for (int i = 0; i < PLQ_ZMAX; ++i) {
            if (i >= z) break;
            double2 s = cmk(0, 0);
#pragma unroll
            for (int j = 0; j < PLQ_ZMAX; ++j) if (j < z) s = cfma(trans ? M[j + z * i] : M[i + z * j], a[j], s);
            X[(size_t)pc[i] + (size_t)ld * col] = s;
        }
    }
    __syncthreads();
}

// columns P of G <- columns P M
DQ_DEV void plq_cols(double2* G, int N, const int* pc, int z, const double2* M) {
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        double2 a[PLQ_ZMAX];
#pragma unroll
        for (int i = 0; i < PLQ_ZMAX; ++i) if (i < z) a[i] = G[MIDX(r, pc[i], N)];
#pragma unroll
        for (int i = 0; i < PLQ_ZMAX; ++i) {
            if (i >= z) break;
            double2 s = cmk(0, 0);
#pragma unroll
            for (int j = 0; j < PLQ_ZMAX; ++j) if (j < z) s = cfma(a[j], M[j + z * i], s);
            G[MIDX(r, pc[i], N)] = s;
        }
    }
    __syncthreads();
}

// In-place inverse of the n x n (column-major) matrix a by Gauss-Jordan
// elimination with partial pivoting; returns det(a).
DQ_DEV double2 small_inv_det(double2* a, int n) {
    int piv[PLQ_ZMAX];
    double2 det = cmk(1, 0);
    for (int k = 0; k < n; ++k) {
        int pr = k;
        double best = cabsd(a[k + n * k]);
        for (int i = k + 1; i < n; ++i) {
            const double v = cabsd(a[i + n * k]);
            if (v > best) { best = v; pr = i; }
        }
        piv[k] = pr;
        if (pr != k) {
            for (int j = 0; j < n; ++j) { const double2 t = a[k + n * j]; a[k + n * j] = a[pr + n * j]; a[pr + n * j] = t; }
            det = cmk(-det.x, -det.y);
        }
        const double2 d = a[k + n * k];
        det = cmul(det, d);
        const double2 di = cdiv(cmk(1, 0), d);
        a[k + n * k] = cmk(1, 0);
        for (int j = 0; j < n; ++j) a[k + n * j] = cmul(a[k + n * j], di);
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            const double2 f = a[i + n * k];
            a[i + n * k] = cmk(0, 0);
            for (int j = 0; j < n; ++j) a[i + n * j] = csub(a[i + n * j], cmul(f, a[k + n * j]));
        }
    }
    for (int k = n - 1; k >= 0; --k)          // undo the row swaps as column swaps
        if (piv[k] != k)
            for (int i = 0; i < n; ++i) { const double2 t = a[i + n * k]; a[i + n * k] = a[i + n * piv[k]]; a[i + n * piv[k]] = t; }
    return det;
}

// G <- G - G(:, P) S V with V(q, col) = delta(P_q, col) - G(P_q, col), S the
// z x z matrix s_mat (column-major); wsm holds W = S V (z x N)
DQ_DEV void rankz_green(double2* G, int N, const int* pc, int z, const double2* s_mat, double2* wsm) {
    const int tid = threadIdx.x;
    for (int col = tid; col < N; col += blockDim.x) {
        double2 v[PLQ_ZMAX];
#pragma unroll
        for (int q = 0; q < PLQ_ZMAX; ++q)
            if (q < z) {
                const double2 g = G[MIDX(pc[q], col, N)];
                v[q] = cmk((pc[q] == col ? 1.0 : 0.0) - g.x, -g.y);
            }
        for (int a = 0; a < z; ++a) {
            double2 s = cmk(0, 0);
#pragma unroll
            for (int q = 0; q < PLQ_ZMAX; ++q) if (q < z) s = cfma(s_mat[a + z * q], v[q], s);
            wsm[(size_t)a * N + col] = s;
        }
    }
    __syncthreads();
    // a thread owns whole rows
    for (int r = tid; r < N; r += blockDim.x) {
        double2 gp[PLQ_ZMAX];
#pragma unroll
        for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) gp[a] = G[MIDX(r, pc[a], N)];
        for (int col = 0; col < N; ++col) {
            double2 s = cmk(0, 0);
#pragma unroll
            for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) s = cfma(gp[a], wsm[(size_t)a * N + col], s);
            G[MIDX(r, col, N)] = csub(G[MIDX(r, col, N)], s);
        }
    }
    __syncthreads();
}

// One slice of plaquette props and updates for one chain (one CTA per chain).
// dir = 0: the 0b order, plaquettes ascending, bmat on the rows and bmat_inv
// on the columns, then the update; dir = 1: the b0 order, plaquettes
// descending, the update, then bmat on the columns and bmat_inv on the rows.
// The k-th visited plaquette uses the random words 2k, 2k + 1 of the slice's
// plaquette draws (iflip, then the accept test).
__global__ void __launch_bounds__(PLQ_NT) k_plq_slice(const ChainDev* __restrict__ chains, int nt, int visit, int dir,
                                                     int lupdate) {
    extern __shared__ double2 wsm[];           // S V, z x N (row a at wsm + a N)
    __shared__ double2 s_mat[PLQ_ZMAX * PLQ_ZMAX];
    __shared__ int s_acc;
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    if (!md.plq) return;
    const int N = c.N, z = md.plq_z, lq = md.lq, lc = md.plq_lcomp, tid = threadIdx.x;
    double2* G = c.G;
    int32_t* cf = c.conf_plq + (size_t)(nt - 1) * lq;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_plq[dir];
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, nties = 0.0;
    for (int k = 0; k < lq; ++k) {
        const int p = dir ? lq - 1 - k : k;
        const int* pc = md.plq_cord + p * z;
        if (!dir) {
            plq_rows(G, N, N, pc, z, md.plq_bmat + (size_t)(cf[p] - 1) * z * z);
            plq_cols(G, N, pc, z, md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z);
        }
        if (lupdate) {
            if (tid == 0) {
                const int is = cf[p];
                const int iflip = (int)ceil(plq_stream(rw[2 * k]) * (lc - 1));
                const int isp = (is + iflip - 1) % lc + 1;
                const int k2 = (is - 1) * (lc - 1) + (iflip - 1);
                const double2* dl = md.plq_delta + (size_t)k2 * z * z;
                double2 vpp[PLQ_ZMAX * PLQ_ZMAX], vu[PLQ_ZMAX * PLQ_ZMAX];
                for (int a = 0; a < z; ++a)
                    for (int b = 0; b < z; ++b) {
                        const double2 g = G[MIDX(pc[a], pc[b], N)];
                        vpp[a + z * b] = cmk((a == b ? 1.0 : 0.0) - g.x, -g.y);
                    }
                for (int a = 0; a < z; ++a)            // vukmat = I + V(:, P) delta
                    for (int b = 0; b < z; ++b) {
                        double2 s = cmk(a == b ? 1.0 : 0.0, 0.0);
                        for (int q = 0; q < z; ++q) s = cfma(vpp[a + z * q], dl[q + z * b], s);
                        vu[a + z * b] = s;
                    }
                const double2 ratio1 = small_inv_det(vu, z);
                for (int a = 0; a < z; ++a)            // smat = delta (I + V U)^-1
                    for (int b = 0; b < z; ++b) {
                        double2 s = cmk(0, 0);
                        for (int q = 0; q < z; ++q) s = cfma(dl[a + z * q], vu[q + z * b], s);
                        s_mat[a + z * b] = s;
                    }
                double2 rt = ratio1;
                for (int f = 1; f < md.nflr; ++f) rt = cmul(rt, ratio1);
                rt = cmul(cscale(rt, md.plq_gam_ratio[k2]), md.plq_phase_ratio[k2]);
                const double ra = fabs(cmul(rt, ph).x / ph.x), r = plq_stream(rw[2 * k + 1]);
                if (fabs(ra - r) < DQ_NEAR_TIE) nties += 1.0;
                s_acc = ra > r;
                if (s_acc) {
                    acc += 1.0;
                    ph = cscale(cmul(ph, rt), 1.0 / sqrt(cmulc(rt, rt).x));
                    cf[p] = isp;
                }
            }
            __syncthreads();
            if (s_acc) rankz_green(G, N, pc, z, s_mat, wsm);
        }
        if (dir) {
            plq_cols(G, N, pc, z, md.plq_bmat + (size_t)(cf[p] - 1) * z * z);
            plq_rows(G, N, N, pc, z, md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z);
        }
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        if (lupdate) {
            c.stats[ST_ACCP] += acc;
            c.stats[ST_PROPP] += lq;
            c.stats[ST_NEAR_TIE] += nties;
        }
    }
}

// One slice of plaquette props and updates for one chain (one CTA per chain),
// delayed: G' = G + A B^T with the accepted rank-z changes as columns of
// (A, B), flushed by the DMMA GEMM after nublock columns and at the slice's
// end (the plaquette counterpart of dqmc_update_delay.f90).  A block on the
// rows P of G' acts on the rows P of G and of A; a block on its columns P acts
// on the columns P of G and, transposed, on the rows P of B.  Plaquette p's
// z x z block of G' is G(P,P) + A(P,:) B(P,:)^T; an accepted plaquette appends
// a_q = sum_p G'(:,P_p) S(p,q) and b_q = G'(P_q,:)^T - e_(P_q).  Order, draws
// and decisions as k_plq_slice (lupdate = 1).
__global__ void __launch_bounds__(PLQ_NT, 2) k_plq_delay(const ChainDev* __restrict__ chains, int nt, int visit, int dir) {
    extern __shared__ double2 dsm[];                   // flush staging
    __shared__ double2 s_ap[PLQ_ZMAX][64], s_bp[PLQ_ZMAX][64];   // A(P_a, m), B(P_a, m)
    __shared__ double2 s_g[PLQ_ZMAX * PLQ_ZMAX];       // G'(P,P), column-major
    __shared__ double2 s_mat[PLQ_ZMAX * PLQ_ZMAX];
    __shared__ double2 s_vu[PLQ_ZMAX * PLQ_ZMAX];     // thread 0's z x z work matrix
    __shared__ int s_acc;
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    if (!md.plq) return;
    const int N = c.N, z = md.plq_z, lq = md.lq, lc = md.plq_lcomp, tid = threadIdx.x;
    const int nbv = min(md.nublock, 64);
    double2 *G = c.G, *A = c.A, *B = c.B;
    int32_t* cf = c.conf_plq + (size_t)(nt - 1) * lq;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_plq[dir];
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, nties = 0.0;
    int k = 0;
    for (int kp = 0; kp < lq; ++kp) {
        const int p = dir ? lq - 1 - kp : kp;
        const int* pc = md.plq_cord + p * z;
        __syncthreads();
        if (!dir) {
            const double2* M = md.plq_bmat + (size_t)(cf[p] - 1) * z * z;
            const double2* Mi = md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z;
            plq_rows(G, N, N, pc, z, M);
            if (k) plq_rows(A, N, k, pc, z, M);
            plq_cols(G, N, pc, z, Mi);
            if (k) plq_rows(B, N, k, pc, z, Mi, true);
        }
        // the plaquette's rows of the delayed factors and its block of G'
        for (int e = tid; e < z * k; e += blockDim.x) {
            const int a = e % z, m = e / z;
            s_ap[a][m] = A[MIDX(pc[a], m, N)];
            s_bp[a][m] = B[MIDX(pc[a], m, N)];
        }
        __syncthreads();
        if (tid < z * z) {
            const int a = tid % z, b = tid / z;
            double2 g = G[MIDX(pc[a], pc[b], N)];
            for (int m = 0; m < k; ++m) g = cfma(s_ap[a][m], s_bp[b][m], g);
            s_g[tid] = g;
        }
        __syncthreads();
        if (tid == 0) {
            const int is = cf[p];
            const int iflip = (int)ceil(plq_stream(rw[2 * kp]) * (lc - 1));
            const int isp = (is + iflip - 1) % lc + 1;
            const int k2 = (is - 1) * (lc - 1) + (iflip - 1);
            const double2* dl = md.plq_delta + (size_t)k2 * z * z;
            double2* vu = s_vu;
            for (int a = 0; a < z; ++a)                  // I + (1 - G')(P,P) delta
                for (int b = 0; b < z; ++b) {
                    double2 sv = cmk(a == b ? 1.0 : 0.0, 0.0);
                    for (int q = 0; q < z; ++q) {
                        const double2 g = s_g[a + z * q];
                        sv = cfma(cmk((a == q ? 1.0 : 0.0) - g.x, -g.y), dl[q + z * b], sv);
                    }
                    vu[a + z * b] = sv;
                }
            const double2 ratio1 = small_inv_det(vu, z);
            for (int a = 0; a < z; ++a)                  // S = delta (I + ...)^-1
                for (int b = 0; b < z; ++b) {
                    double2 sv = cmk(0, 0);
                    for (int q = 0; q < z; ++q) sv = cfma(dl[a + z * q], vu[q + z * b], sv);
                    s_mat[a + z * b] = sv;
                }
            double2 rt = ratio1;
            for (int f = 1; f < md.nflr; ++f) rt = cmul(rt, ratio1);
            rt = cmul(cscale(rt, md.plq_gam_ratio[k2]), md.plq_phase_ratio[k2]);
            const double ra = fabs(cmul(rt, ph).x / ph.x), r = plq_stream(rw[2 * kp + 1]);
            if (fabs(ra - r) < DQ_NEAR_TIE) nties += 1.0;
            s_acc = ra > r;
            if (s_acc) {
                acc += 1.0;
                ph = cscale(cmul(ph, rt), 1.0 / sqrt(cmulc(rt, rt).x));
                cf[p] = isp;
            }
        }
        __syncthreads();
        if (s_acc) {
            int pcs[PLQ_ZMAX];
#pragma unroll
            for (int a = 0; a < PLQ_ZMAX; ++a) pcs[a] = a < z ? pc[a] : 0;
            for (int i = tid; i < N; i += blockDim.x) {
                double2 cc[PLQ_ZMAX], rr[PLQ_ZMAX];
#pragma unroll
                for (int a = 0; a < PLQ_ZMAX; ++a)
                    if (a < z) { cc[a] = G[MIDX(i, pcs[a], N)]; rr[a] = G[MIDX(pcs[a], i, N)]; }
                for (int m = 0; m < k; ++m) {
                    const double2 ai = A[MIDX(i, m, N)], bi = B[MIDX(i, m, N)];
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a)
                        if (a < z) { cc[a] = cfma(ai, s_bp[a][m], cc[a]); rr[a] = cfma(s_ap[a][m], bi, rr[a]); }
                }
#pragma unroll
                for (int q = 0; q < PLQ_ZMAX; ++q) {
                    if (q >= z) break;
                    double2 sv = cmk(0, 0);
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) sv = cfma(cc[a], s_mat[a + z * q], sv);
                    double2 r = rr[q];
                    if (i == pcs[q]) r.x -= 1.0;
                    A[MIDX(i, k + q, N)] = sv;
                    B[MIDX(i, k + q, N)] = r;
                }
            }
            k += z;
            __syncthreads();
        }
        if (dir) {
            const double2* M = md.plq_bmat + (size_t)(cf[p] - 1) * z * z;
            const double2* Mi = md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z;
            plq_cols(G, N, pc, z, M);
            if (k) plq_rows(B, N, k, pc, z, M, true);
            plq_rows(G, N, N, pc, z, Mi);
            if (k) plq_rows(A, N, k, pc, z, Mi);
        }
        if (k > 0 && (k + z > nbv || kp == lq - 1)) {
            flush_addto(G, A, B, N, k, dsm);
            k = 0;
        }
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        c.stats[ST_ACCP] += acc;
        c.stats[ST_PROPP] += lq;
        c.stats[ST_NEAR_TIE] += nties;
    }
}

// One bond family's updates of one slice on the equal-time G, one CTA per
// chain (the t-V bond field, src/dqmc_config_v/dqmc_update.f90:34-105): the
// bonds in nnlf_list order, each a rank-2 change on its sites P = (i1, i2) with
// Delta = diag(delta_bmat_p, delta_bmat_m) of its field value, vukmat =
// I + (1 - G)(P,P) Delta, ratiotot = det vukmat and, on acceptance,
// G <- G - G(:,P) Delta vukmat^-1 (delta(P,:) - G(P,:)).  The field has two
// values, so iflip = ceil(r (lcomp - 1)) is 1 for every draw r in (0, 1).  The
// k-th bond uses the words 2k (iflip) and 2k + 1 (the accept test) of the
// family's 2 nn_lf words: families ascend in the 0b slice layout (dir = 0) and
// descend in the b0 one (dir = 1).
__global__ void __launch_bounds__(PLQ_NT) k_vbond_slice(const ChainDev* __restrict__ chains, int nt, int nf, int visit,
                                                      int dir) {
    extern __shared__ double2 wsm[];           // S V, 2 x N
    __shared__ double2 s_mat[4];
    __shared__ int s_pc[2];
    __shared__ int s_acc;
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    if (!md.lwrapv || !c.vconf) return;
    const int N = c.N, lf = md.nn_lf, nnf = md.nn_nf, tid = threadIdx.x;
    double2* G = c.G;
    int32_t* cf = c.vconf + ((size_t)(nt - 1) * nnf + (nf - 1)) * N;
    const int* rows = md.vrows + (size_t)(nf - 1) * 2 * lf;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_v[dir] + (size_t)(dir ? nnf - nf : nf - 1) * 2 * lf;
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, nties = 0.0;
    for (int b = 0; b < lf; ++b) {
        // every thread has read the previous bond's s_acc (a rejected bond has
        // no barrier of its own) before thread 0 overwrites it
        __syncthreads();
        if (tid == 0) {
            const int i1 = rows[2 * b], i2 = rows[2 * b + 1];
            s_pc[0] = i1; s_pc[1] = i2;
            const int is = cf[b];
            const double2 d0 = md.vdp[is - 1], d1 = md.vdm[is - 1];
            const double2 g11 = G[MIDX(i1, i1, N)], g12 = G[MIDX(i1, i2, N)];
            const double2 g21 = G[MIDX(i2, i1, N)], g22 = G[MIDX(i2, i2, N)];
            // vukmat, column-major
            const double2 v00 = cadd(cmk(1, 0), cmul(cmk(1.0 - g11.x, -g11.y), d0));
            const double2 v10 = cmul(cmk(-g21.x, -g21.y), d0);
            const double2 v01 = cmul(cmk(-g12.x, -g12.y), d1);
            const double2 v11 = cadd(cmk(1, 0), cmul(cmk(1.0 - g22.x, -g22.y), d1));
            const double2 det = csub(cmul(v00, v11), cmul(v01, v10));
            const double2 id = cdiv(cmk(1, 0), det);
            s_mat[0] = cmul(d0, cmul(v11, id));                      // smat = Delta vukmat^-1
            s_mat[1] = cmul(d1, cmul(cmk(-v10.x, -v10.y), id));
            s_mat[2] = cmul(d0, cmul(cmk(-v01.x, -v01.y), id));
            s_mat[3] = cmul(d1, cmul(v00, id));
            const double ra = fabs(cmul(det, ph).x / ph.x), r = plq_stream(rw[2 * b + 1]);
            if (fabs(ra - r) < DQ_NEAR_TIE) nties += 1.0;
            s_acc = ra > r;
            if (s_acc) {
                acc += 1.0;
                ph = cscale(cmul(ph, det), 1.0 / sqrt(cmulc(det, det).x));
                cf[b] = is % 2 + 1;
            }
        }
        __syncthreads();
        if (s_acc) rankz_green(G, N, s_pc, 2, s_mat, wsm);
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        c.stats[ST_ACCV] += acc;
        c.stats[ST_PROPV] += lf;
        c.stats[ST_NEAR_TIE] += nties;
    }
}

// One slice of plaquette props and updates on the projective path (one CTA
// per walker): UR (N x ne), UL stored as UL^T (N x ne) and ULRINV (ne x ne).
// dir = 0 (dqmc_proj_sweep_0b.f90:61-68): ascending, UR(P,:) <- bmat UR(P,:),
// UL(:,P) <- UL(:,P) bmat_inv, then the update; dir = 1
// (dqmc_proj_sweep_b0.f90:91-99): descending, the update, then
// UL(:,P) <- UL(:,P) bmat and UR(P,:) <- bmat_inv UR(P,:).  The update
// (dqmc_proj_update_plqu.f90): vkt = delta UR(P,:), vk = vkt ULRINV, ratio
// det(I + vk UL(:,P)); on acceptance UR(P,:) += vkt and
// ULRINV -= ULRINV UL(:,P) (I + vk UL(:,P))^-1 vk.
__global__ void __launch_bounds__(PLQ_NT) k_plq_proj_slice(const ChainDev* __restrict__ chains, int nt, int visit,
                                                          int dir, int lupdate) {
    extern __shared__ double2 psm[];          // vkt [z][ne], vk [z][ne], lru [z][ne]
    __shared__ double2 s_mat[PLQ_ZMAX * PLQ_ZMAX];
    __shared__ int s_acc;
    const ChainDev& c = chains[blockIdx.x];
    const ModelDev& md = *c.md;
    if (!md.plq) return;
    const int N = c.N, ne = md.ne, z = md.plq_z, lq = md.lq, lc = md.plq_lcomp, tid = threadIdx.x;
    double2 *UR = c.UR, *ULT = c.ULT, *R = c.ULRINV;
    double2 *vkt = psm, *vk = psm + (size_t)z * ne, *lru = psm + (size_t)2 * z * ne;
    int32_t* cf = c.conf_plq + (size_t)(nt - 1) * lq;
    const uint32_t* rw = c.rnd + (size_t)visit * md.rps + md.rw_plq[dir];
    double2 ph = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    double acc = 0.0, nties = 0.0;
    for (int k = 0; k < lq; ++k) {
        const int p = dir ? lq - 1 - k : k;
        const int* pc = md.plq_cord + p * z;
        if (!dir) {
            plq_rows(UR, N, ne, pc, z, md.plq_bmat + (size_t)(cf[p] - 1) * z * z);
            plq_rows(ULT, N, ne, pc, z, md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z, true);
        }
        if (lupdate) {
            const int is = cf[p];
            const int iflip = (int)ceil(plq_stream(rw[2 * k]) * (lc - 1));
            const int k2 = (is - 1) * (lc - 1) + (iflip - 1);
            const double2* dl = md.plq_delta + (size_t)k2 * z * z;
            for (int l = tid; l < ne; l += blockDim.x) {          // vkt = delta UR(P,:)
                double2 u[PLQ_ZMAX];
#pragma unroll
                for (int q = 0; q < PLQ_ZMAX; ++q) if (q < z) u[q] = UR[(size_t)pc[q] + (size_t)N * l];
                for (int a = 0; a < z; ++a) {
                    double2 s = cmk(0, 0);
#pragma unroll
                    for (int q = 0; q < PLQ_ZMAX; ++q) if (q < z) s = cfma(dl[a + z * q], u[q], s);
                    vkt[(size_t)a * ne + l] = s;
                }
            }
            __syncthreads();
            for (int l = tid; l < ne; l += blockDim.x) {          // vk = vkt ULRINV
                double2 s[PLQ_ZMAX];
#pragma unroll
                for (int a = 0; a < PLQ_ZMAX; ++a) s[a] = cmk(0, 0);
                for (int q = 0; q < ne; ++q) {
                    const double2 r = R[(size_t)q + (size_t)ne * l];
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) s[a] = cfma(vkt[(size_t)a * ne + q], r, s[a]);
                }
#pragma unroll
                for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) vk[(size_t)a * ne + l] = s[a];
            }
            __syncthreads();
            if (tid == 0) {
                const int isp = (is + iflip - 1) % lc + 1;
                double2 vu[PLQ_ZMAX * PLQ_ZMAX];
                for (int a = 0; a < z; ++a)                       // I + vk UL(:,P), UL(l, P_b) = ULT(P_b, l)
                    for (int b = 0; b < z; ++b) {
                        double2 s = cmk(a == b ? 1.0 : 0.0, 0.0);
                        for (int l = 0; l < ne; ++l) s = cfma(vk[(size_t)a * ne + l], ULT[(size_t)pc[b] + (size_t)N * l], s);
                        vu[a + z * b] = s;
                    }
                const double2 ratio1 = small_inv_det(vu, z);
                for (int e = 0; e < z * z; ++e) s_mat[e] = vu[e];
                double2 rt = ratio1;
                for (int f = 1; f < md.nflr; ++f) rt = cmul(rt, ratio1);
                rt = cmul(cscale(rt, md.plq_gam_ratio[k2]), md.plq_phase_ratio[k2]);
                const double ra = fabs(cmul(rt, ph).x / ph.x), r = plq_stream(rw[2 * k + 1]);
                if (fabs(ra - r) < DQ_NEAR_TIE) nties += 1.0;
                s_acc = ra > r;
                if (s_acc) {
                    acc += 1.0;
                    ph = cscale(cmul(ph, rt), 1.0 / sqrt(cmulc(rt, rt).x));
                    cf[p] = isp;
                }
            }
            __syncthreads();
            if (s_acc) {
                for (int l = tid; l < ne; l += blockDim.x) {
                    // UR(P,:) += vkt; vk(:,l) <- (I + vk UL(:,P))^-1 vk(:,l)
                    double2 w[PLQ_ZMAX], v[PLQ_ZMAX];
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) v[a] = vk[(size_t)a * ne + l];
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a) {
                        if (a >= z) break;
                        UR[(size_t)pc[a] + (size_t)N * l] = cadd(UR[(size_t)pc[a] + (size_t)N * l], vkt[(size_t)a * ne + l]);
                        double2 s = cmk(0, 0);
#pragma unroll
                        for (int b = 0; b < PLQ_ZMAX; ++b) if (b < z) s = cfma(s_mat[a + z * b], v[b], s);
                        w[a] = s;
                    }
#pragma unroll
                    for (int a = 0; a < PLQ_ZMAX; ++a) if (a < z) vk[(size_t)a * ne + l] = w[a];
                }
                for (int q = tid; q < ne; q += blockDim.x) {      // lru(q, b) = sum_l ULRINV(q,l) UL(l,P_b)
                    double2 s[PLQ_ZMAX];
#pragma unroll
                    for (int b = 0; b < PLQ_ZMAX; ++b) s[b] = cmk(0, 0);
                    for (int l = 0; l < ne; ++l) {
                        const double2 r = R[(size_t)q + (size_t)ne * l];
#pragma unroll
                        for (int b = 0; b < PLQ_ZMAX; ++b) if (b < z) s[b] = cfma(r, ULT[(size_t)pc[b] + (size_t)N * l], s[b]);
                    }
#pragma unroll
                    for (int b = 0; b < PLQ_ZMAX; ++b) if (b < z) lru[(size_t)b * ne + q] = s[b];
                }
                __syncthreads();
                for (int q = tid; q < ne; q += blockDim.x) {      // ULRINV -= lru W
                    double2 lr[PLQ_ZMAX];
#pragma unroll
                    for (int b = 0; b < PLQ_ZMAX; ++b) if (b < z) lr[b] = lru[(size_t)b * ne + q];
                    for (int l = 0; l < ne; ++l) {
                        double2 s = cmk(0, 0);
#pragma unroll
                        for (int b = 0; b < PLQ_ZMAX; ++b) if (b < z) s = cfma(lr[b], vk[(size_t)b * ne + l], s);
                        R[(size_t)q + (size_t)ne * l] = csub(R[(size_t)q + (size_t)ne * l], s);
                    }
                }
                __syncthreads();
            }
        }
        if (dir) {
            plq_rows(ULT, N, ne, pc, z, md.plq_bmat + (size_t)(cf[p] - 1) * z * z, true);
            plq_rows(UR, N, ne, pc, z, md.plq_bmat_inv + (size_t)(cf[p] - 1) * z * z);
        }
    }
    if (tid == 0) {
        c.stats[ST_PHASE_RE] = ph.x;
        c.stats[ST_PHASE_IM] = ph.y;
        if (lupdate) {
            c.stats[ST_ACCP] += acc;
            c.stats[ST_PROPP] += lq;
            c.stats[ST_NEAR_TIE] += nties;
        }
    }
}

static int g_plqp_attr = 0;

void launch_plq_proj_slice(const ChainDev* chains, int nchains, int maxNe, int nt, int visit, int dir, int lupdate,
                           cudaStream_t st) {
    const size_t smem = (size_t)3 * PLQ_ZMAX * maxNe * sizeof(double2);
    if (!g_plqp_attr) {
        cudaFuncSetAttribute(k_plq_proj_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * PLQ_ZMAX * 512 * (int)sizeof(double2));
        g_plqp_attr = 1;
    }
    k_plq_proj_slice<<<nchains, PLQ_NT, smem, st>>>(chains, nt, visit, dir, lupdate);
}

static int g_plq_attr = 0;

static int g_plqd_attr = 0;

// the delayed plaquette updates when every model's flush depth holds one
// plaquette's z columns; returns 0 without launching otherwise
int launch_plq_delay(const ChainDev* chains, int nchains, int nublock, int z, int nt, int visit, int dir,
                     cudaStream_t st) {
    if (min(nublock, 64) < z) return 0;
    const size_t smem = UpdGemm::SMEM_ELEMS * sizeof(double2);
    if (!g_plqd_attr) {
        cudaFuncSetAttribute(k_plq_delay, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        g_plqd_attr = 1;
    }
    k_plq_delay<<<nchains, PLQ_NT, smem, st>>>(chains, nt, visit, dir);
    return 1;
}

void launch_plq_slice(const ChainDev* chains, int nchains, int maxN, int nt, int visit, int dir, int lupdate,
                      cudaStream_t st) {
    const size_t smem = (size_t)PLQ_ZMAX * maxN * sizeof(double2);
    if (!g_plq_attr) {
        cudaFuncSetAttribute(k_plq_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, PLQ_ZMAX * 512 * (int)sizeof(double2));
        g_plq_attr = 1;
    }
    k_plq_slice<<<nchains, PLQ_NT, smem, st>>>(chains, nt, visit, dir, lupdate);
}

static int g_vb_attr = 0;

void launch_vbond_slice(const ChainDev* chains, int nchains, int maxN, int nt, int nf, int visit, int dir,
                        cudaStream_t st) {
    const size_t smem = (size_t)2 * maxN * sizeof(double2);
    if (!g_vb_attr) {
        cudaFuncSetAttribute(k_vbond_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 512 * (int)sizeof(double2));
        g_vb_attr = 1;
    }
    k_vbond_slice<<<nchains, PLQ_NT, smem, st>>>(chains, nt, nf, visit, dir);
}
