// CTA-level dense complex linear algebra for the UDV stabilisation:
// blocked Householder QR (LAPACK zgeqrf/zlarft conventions: beta real,
// H = I - tau v v^H, v(1) = 1), explicit Q (zungqr), Q^H applied to a matrix,
// and an upper-triangular solve.  The trailing updates and the triangular
// solve's off-diagonal blocks run through the DMMA GEMM of zgemm.cuh; the
// panel factorisation runs in shared memory.  One CTA of 256 threads owns
// one chain's matrices (leading dimension N, N <= 512).
#pragma once
#include "zgemm.cuh"

#define QR_NB 16
// shared memory of a panel: m x 16 with an odd leading dimension (m or m + 1),
// so that the 16 columns fall in different banks
#define QR_PANEL_ELEMS(N) ((size_t)((N) + 1) * QR_NB)

struct LinalgScratch {
    double2* Vs;      // N x 64 explicit reflector block (ld N)
    double2* Ws;      // 64 x N (ld 16 for 16-wide blocks, 64 for 64-wide ones)
    double2* Ws2;     // 64 x N
    double2* T;       // (N/16 + 1) x 16 x 16 block-reflector triangles of the panels
    double2* tau;     // N
    double2* T64 = nullptr;   // (N/64 + 1) x 64 x 64 triangles of the 64-wide blocks (two-level QR)
};

struct LinalgSmem {
    double red[64];
    double2 tau_j, scal;
    double2 Tl[QR_NB * QR_NB];
    double2 S[QR_NB * QR_NB];
    double2 w[QR_NB];
    int flag;
};

// ---- panel factorisation (zgeqr2 on an m x jb panel in shared memory) ----
// Reflector of column j from alpha = P(j, j) and xnorm = ||P(j+1:m, j)|| (zlarfg),
// computed by thread 0: tau, the scale 1 / (alpha - beta) of the vector, and
// P(j, j) = beta.
static __device__ void panel_reflector(double2* col, int j, double xnorm, double2* taus, LinalgSmem* L) {
    double2 alpha = col[j];
    if (xnorm == 0.0 && alpha.y == 0.0) {
        L->tau_j = cmk(0, 0);
        L->scal = cmk(1, 0);
    } else {
        double ax = fabs(alpha.x), ay = fabs(alpha.y);
        double w = fmax(ax, fmax(ay, xnorm));
        double nrm = w * sqrt((ax / w) * (ax / w) + (ay / w) * (ay / w) + (xnorm / w) * (xnorm / w));
        double beta = -copysign(nrm, alpha.x);
        L->tau_j = cmk((beta - alpha.x) / beta, -alpha.y / beta);
        L->scal = cdiv(cmk(1, 0), csub(alpha, cmk(beta, 0)));
        col[j] = cmk(beta, 0.0);
    }
    taus[j] = L->tau_j;
}

// Column j of the panel when the plain sum of squares under/overflows: the
// norm is taken with rescaling and the vector is scaled before the products.
static __device__ void panel_column_careful(double2* P, int m, int ldp, int jb, int j, double2* taus, LinalgSmem* L) {
    const int tid = threadIdx.x, nth = blockDim.x;
    double2* col = P + (size_t)j * ldp;
    double mx = 0.0;
    for (int r = j + 1 + tid; r < m; r += nth) mx = fmax(mx, fmax(fabs(col[r].x), fabs(col[r].y)));
    mx = block_max(mx, L->red);
    double s2 = 0.0;
    if (mx > 0.0)
        for (int r = j + 1 + tid; r < m; r += nth) s2 += cabs2(cscale(col[r], 1.0 / mx));
    s2 = block_sum(s2, L->red);
    if (tid == 0) panel_reflector(col, j, mx * sqrt(s2), taus, L);
    __syncthreads();
    const double2 tau = L->tau_j, scal = L->scal;
    if (tau.x == 0.0 && tau.y == 0.0) { __syncthreads(); return; }
    for (int r = j + 1 + tid; r < m; r += nth) col[r] = cmul(col[r], scal);
    __syncthreads();
    // w_c = v^H P[:, c], c > j ; groups of 16 threads
    const int grp = tid >> 4, gl = tid & 15;
    for (int base = j + 1; base < jb; base += nth / 16) {     // uniform trip count
        const int cc = base + grp;
        const bool ok = cc < jb;
        double2 acc = cmk(0, 0);
        if (ok) {
            const double2* pc = P + (size_t)cc * ldp;
            if (gl == 0) acc = pc[j];
            for (int r = j + 1 + gl; r < m; r += 16) acc = cfma(cconj(col[r]), pc[r], acc);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o, 16);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o, 16);
        }
        if (ok && gl == 0) L->w[cc] = acc;
    }
    __syncthreads();
    // P[r, c] -= conj(tau) v_r w_c
    const double2 ctau = cconj(tau);
    const int nc = jb - j - 1, nr = m - j;
    for (int e = tid; e < nc * nr; e += nth) {
        int cc = j + 1 + e / nr, r = j + e % nr;
        double2 v = (r == j) ? cmk(1, 0) : col[r];
        double2 f = cmul(ctau, L->w[cc]);
        P[(size_t)cc * ldp + r] = csub(P[(size_t)cc * ldp + r], cmul(v, f));
    }
    __syncthreads();
}

// Householder QR of the m x jb panel, three barriers per column: one pass
// forms ||P(j+1:m, j)||^2 and the raw products d_c = P(j+1:m, j)^H P(j+1:m, c)
// together (16-thread groups, one per column), thread 0 forms the reflector
// and w_c = v^H P(:, c) = P(j, c) + conj(scal) d_c, and one row-owned pass
// scales the vector and applies P(r, c) -= conj(tau) v_r w_c.
static __device__ void panel_qr(double2* P, int m, int ldp, int jb, double2* taus, LinalgSmem* L) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const int grp = tid >> 4, gl = tid & 15;
    for (int j = 0; j < jb; ++j) {
        double2* col = P + (size_t)j * ldp;
        for (int base = 0; base < jb - j; base += nth / 16) {    // uniform trip count
            const int g = base + grp;
            const bool ok = g < jb - j;
            double2 acc = cmk(0, 0);
            if (ok) {
                if (g == 0) {
                    for (int r = j + 1 + gl; r < m; r += 16) acc.x += cabs2(col[r]);
                } else {
                    const double2* pc = P + (size_t)(j + g) * ldp;
                    for (int r = j + 1 + gl; r < m; r += 16) acc = cfma(cconj(col[r]), pc[r], acc);
                }
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o, 16);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o, 16);
            }
            if (ok && gl == 0) L->w[j + g] = acc;
        }
        __syncthreads();
        if (tid == 0) {
            const double ss = L->w[j].x;
            const int careful = !(ss < 1e300) || (ss > 0.0 && ss < 1e-280);
            L->flag = careful;
            if (!careful) {
                panel_reflector(col, j, sqrt(ss), taus, L);
                const double2 cs = cconj(L->scal);
                for (int cc = j + 1; cc < jb; ++cc) L->w[cc] = cfma(cs, L->w[cc], P[(size_t)cc * ldp + j]);
            }
        }
        __syncthreads();
        if (L->flag) {
            panel_column_careful(P, m, ldp, jb, j, taus, L);
            continue;
        }
        const double2 tau = L->tau_j, scal = L->scal;
        if (tau.x == 0.0 && tau.y == 0.0) continue;
        const double2 ctau = cconj(tau);
        for (int r = j + tid; r < m; r += nth) {
            const double2 v = (r == j) ? cmk(1, 0) : cmul(col[r], scal);
            const double2 cv = cmul(ctau, v);
            for (int cc = j + 1; cc < jb; ++cc)
                P[(size_t)cc * ldp + r] = csub(P[(size_t)cc * ldp + r], cmul(cv, L->w[cc]));
            if (r > j) col[r] = v;
        }
        __syncthreads();
    }
}

// T (jb x jb upper) of the block reflector H_1..H_jb = I - V T V^H (zlarft 'F','C').
// V is the unit-lower panel in shared memory (m x jb).
static __device__ void panel_larft(const double2* P, int m, int ldp, int jb, const double2* taus, double2* Tout, LinalgSmem* L) {
    const int tid = threadIdx.x;
    // Gram S(a,b) = V(:,a)^H V(:,b) for a < b
    for (int e = tid; e < jb * jb; e += blockDim.x) {
        int a = e % jb, b = e / jb;
        if (a < b) {
            double2 s = P[(size_t)a * ldp + b];          // V(b,a)^* * V(b,b)=1, rows r >= b
            s = cconj(s);
            for (int r = b + 1; r < m; ++r) s = cfma(cconj(P[(size_t)a * ldp + r]), P[(size_t)b * ldp + r], s);
            L->S[a + b * QR_NB] = s;
        }
    }
    __syncthreads();
    if (tid < 32) {
        for (int i = 0; i < jb; ++i) {
            double2 ti = taus[i];
            // t_a = -tau_i S(a, i), a < i ;  T(0:i, i) = T(0:i,0:i) t
            if (tid < i) {
                double2 acc = cmk(0, 0);
                for (int b = tid; b < i; ++b) {
                    double2 tb = cmul(cmk(-ti.x, -ti.y), L->S[b + i * QR_NB]);
                    acc = cfma(L->Tl[tid + b * QR_NB], tb, acc);
                }
                L->Tl[tid + i * QR_NB] = acc;
            }
            if (tid == 0) L->Tl[i + i * QR_NB] = ti;
            for (int a = i + 1 + tid; a < QR_NB; a += 32) L->Tl[a + i * QR_NB] = cmk(0, 0);
            __syncwarp();
        }
    }
    __syncthreads();
    for (int e = tid; e < QR_NB * QR_NB; e += blockDim.x) {
        int a = e % QR_NB, b = e / QR_NB;
        Tout[e] = (a < jb && b < jb && a <= b) ? L->Tl[e] : cmk(0, 0);
    }
    __syncthreads();
}

// Explicit reflector block of panel p into Vs (rows p..N-1 stored at Vs[r - p], ld N)
static __device__ void build_vblock(const double2* A, int N, int p, int jb, double2* Vs) {
    int m = N - p;
    for (int e = threadIdx.x; e < m * jb; e += blockDim.x) {
        int r = e % m, cc = e / m;
        double2 v = (r < cc) ? cmk(0, 0) : (r == cc) ? cmk(1, 0) : A[MIDX(p + r, p + cc, N)];
        Vs[MIDX(r, cc, N)] = v;
    }
    __syncthreads();
}

// X[p:N, c0:c0+nc] <- (I - V T V^H)^op X,  op = H (apply Q^H) or none (apply Q)
static __device__ void apply_block(const double2* Vs, const double2* Tp, int N, int p, int jb,
                            double2* X, int c0, int nc, int use_th, LinalgScratch& sc, cplx* gsm) {
    if (nc <= 0) return;
    int m = N - p;
    ZGemmArgs g;
    // W = V^H X
    g.M = jb; g.N = nc; g.K = m; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = Vs; g.lda = N; g.opA = OP_C;
    g.B = X + MIDX(p, c0, N); g.ldb = N; g.opB = OP_N;
    g.C = sc.Ws; g.ldc = QR_NB;
    zgemm_cta<GemmWide>(g, 0, 1, gsm);
    // W2 = T^H W  or  T W, with T^H or T (16 x 16) in shared memory (the
    // staging buffer is free between the GEMMs); stored as the operator
    // itself, so that threads of consecutive rows a read consecutive elements
    double2* Ts = gsm;
    for (int e = threadIdx.x; e < QR_NB * QR_NB; e += blockDim.x) {
        const int r = e % QR_NB, q = e / QR_NB;
        Ts[e] = use_th ? cconj(Tp[q + r * QR_NB]) : Tp[e];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < jb * nc; e += blockDim.x) {
        int a = e % jb, cc = e / jb;
        const double2* w = sc.Ws + (size_t)cc * QR_NB;
        double2 acc = cmk(0, 0);
        if (use_th) {
            for (int b = 0; b <= a; ++b) acc = cfma(Ts[a + b * QR_NB], w[b], acc);
        } else {
            for (int b = a; b < jb; ++b) acc = cfma(Ts[a + b * QR_NB], w[b], acc);
        }
        sc.Ws2[a + cc * QR_NB] = acc;
    }
    __syncthreads();
    // X -= V W2
    g.M = m; g.N = nc; g.K = jb; g.alpha = cmk(-1, 0); g.beta = cmk(1, 0);
    g.A = Vs; g.lda = N; g.opA = OP_N;
    g.B = sc.Ws2; g.ldb = QR_NB; g.opB = OP_N;
    g.C = X + MIDX(p, c0, N); g.ldc = N;
    zgemm_cta<GemmBig>(g, 0, 1, gsm);
}

// In-place QR of the first ncol columns of A (N rows, ld N; ncol <= N, default
// all N): R in the upper triangle, reflectors below, tau and the per-panel T
// factors in the scratch.  smem_panel holds >= QR_PANEL_ELEMS(N) double2.
static __device__ void cta_qr(double2* A, int N, LinalgScratch& sc, double2* smem_panel, cplx* gsm, LinalgSmem* L,
                              int ncol = -1) {
    if (ncol < 0) ncol = N;
    for (int p = 0; p < ncol; p += QR_NB) {
        const int jb = min(QR_NB, ncol - p), m = N - p, ldp = m + ((m & 1) ^ 1);
        double2* P = smem_panel;
        for (int e = threadIdx.x; e < m * jb; e += blockDim.x) {
            int r = e % m, cc = e / m;
            P[(size_t)cc * ldp + r] = A[MIDX(p + r, p + cc, N)];
        }
        __syncthreads();
        panel_qr(P, m, ldp, jb, sc.tau + p, L);
        double2* Tp = sc.T + (size_t)(p / QR_NB) * QR_NB * QR_NB;
        panel_larft(P, m, ldp, jb, sc.tau + p, Tp, L);
        for (int e = threadIdx.x; e < m * jb; e += blockDim.x) {
            int r = e % m, cc = e / m;
            A[MIDX(p + r, p + cc, N)] = P[(size_t)cc * ldp + r];
            sc.Vs[MIDX(r, cc, N)] = (r < cc) ? cmk(0, 0) : (r == cc) ? cmk(1, 0) : P[(size_t)cc * ldp + r];
        }
        __syncthreads();
        if (p + jb < ncol) apply_block(sc.Vs, Tp, N, p, jb, A, p + jb, ncol - p - jb, 1, sc, gsm);
    }
}

// log det Q = sum_i log(1 - tau_i 2 Re(tau_i) / |tau_i|^2)  (s_matrix.f90:1290-1298)
static __device__ double2 cta_logdet_q(const double2* tau, int N, double* red) {
    double2 acc = cmk(0, 0);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double2 t = tau[i];
        double a2 = cabs2(t);
        if (a2 != 0.0) {
            double2 z = csub(cmk(1, 0), cscale(t, 2.0 * t.x / a2));
            acc = cadd(acc, clog_(z));
        }
    }
    return block_csum(acc, red);
}

// The first ncol columns of Q (N x ncol, ld N) from the factored A into Qout
// (zungqr, blocked backward; ncol defaults to N).
static __device__ void cta_form_q(const double2* A, int N, double2* Qout, LinalgScratch& sc, cplx* gsm, int ncol = -1) {
    if (ncol < 0) ncol = N;
    for (int e = threadIdx.x; e < N * ncol; e += blockDim.x) {
        int r = e % N, cc = e / N;
        Qout[e] = cmk(r == cc ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    int last = ((ncol - 1) / QR_NB) * QR_NB;
    for (int p = last; p >= 0; p -= QR_NB) {
        const int jb = min(QR_NB, ncol - p);
        build_vblock(A, N, p, jb, sc.Vs);
        const double2* Tp = sc.T + (size_t)(p / QR_NB) * QR_NB * QR_NB;
        apply_block(sc.Vs, Tp, N, p, jb, Qout, p, ncol - p, 0, sc, gsm);
    }
}

// X <- Q^H X for all N columns of X (Q from the factored A).
static __device__ void cta_apply_qh(const double2* A, int N, double2* X, LinalgScratch& sc, cplx* gsm) {
    for (int p = 0; p < N; p += QR_NB) {
        const int jb = min(QR_NB, N - p);
        build_vblock(A, N, p, jb, sc.Vs);
        const double2* Tp = sc.T + (size_t)(p / QR_NB) * QR_NB * QR_NB;
        apply_block(sc.Vs, Tp, N, p, jb, X, 0, N, 1, sc, gsm);
    }
}

// X <- R^{-1} X with R the upper triangle of A (blocked back substitution).
static __device__ void trsm_rows16(const double2* A, int N, double2* X, int p0, int p1, cplx* gsm, LinalgSmem* L) {
    const int last = p0 + ((p1 - p0 - 1) / QR_NB) * QR_NB;
    for (int p = last; p >= p0; p -= QR_NB) {
        const int jb = min(QR_NB, p1 - p);
        if (p + jb < p1) {
            ZGemmArgs g;
            g.M = jb; g.N = N; g.K = p1 - p - jb; g.alpha = cmk(-1, 0); g.beta = cmk(1, 0);
            g.A = A + MIDX(p, p + jb, N); g.lda = N; g.opA = OP_N;
            g.B = X + (p + jb); g.ldb = N; g.opB = OP_N;
            g.C = X + p; g.ldc = N;
            zgemm_cta<GemmWide>(g, 0, 1, gsm);
        }
        // The diagonal is stored as its reciprocal so the solve multiplies.
        for (int e = threadIdx.x; e < jb * jb; e += blockDim.x) {
            int a = e % jb, b = e / jb;
            double2 v = A[MIDX(p + a, p + b, N)];
            L->S[a + b * QR_NB] = (a == b) ? cdiv(cmk(1, 0), v) : v;
        }
        __syncthreads();
        for (int cc = threadIdx.x; cc < N; cc += blockDim.x) {
            double2 x[QR_NB];
#pragma unroll
            for (int a = 0; a < QR_NB; ++a) x[a] = (a < jb) ? X[MIDX(p + a, cc, N)] : cmk(0, 0);
#pragma unroll
            for (int a = QR_NB - 1; a >= 0; --a) {
                if (a < jb) {
                    double2 sm = x[a];
#pragma unroll
                    for (int b = a + 1; b < QR_NB; ++b)
                        if (b < jb) sm = csub(sm, cmul(L->S[a + b * QR_NB], x[b]));
                    x[a] = cmul(sm, L->S[a + a * QR_NB]);
                }
            }
#pragma unroll
            for (int a = 0; a < QR_NB; ++a)
                if (a < jb) X[MIDX(p + a, cc, N)] = x[a];
        }
        __syncthreads();
    }
}

static __device__ void cta_trsm_upper(const double2* A, int N, double2* X, cplx* gsm, LinalgSmem* L) {
    trsm_rows16(A, N, X, 0, N, gsm, L);
}

// ---------------------------------------------------------------------------
// Two-level blocked QR: 16-wide panels inside 64-wide blocks.  The panels of a
// block update only the block's own columns; the trailing matrix and the later
// applications of Q use the block's 64-wide reflector (I - V T V^H), whose
// GEMMs have an inner dimension of 64 instead of 16.  T of a block is built
// from its panels' triangles: for H = H_a H_b,
//   T = [[T_a, -T_a (V_a^H V_b) T_b], [0, T_b]].
// ---------------------------------------------------------------------------
#define QR_NB2 64

// X <- R^{-1} X, two-level: block rows of 64 are first updated with the solved
// rows below them by one 64-row GEMM (GemmBig), then solved with the 16-row
// scheme of trsm_rows16 restricted to the block, so most of the work runs
// in 64-row DMMA tiles instead of 16-row ones.
static __device__ void cta_trsm_upper64(const double2* A, int N, double2* X, cplx* gsm, LinalgSmem* L) {
    const int last64 = ((N - 1) / QR_NB2) * QR_NB2;
    for (int P = last64; P >= 0; P -= QR_NB2) {
        const int jb2 = min(QR_NB2, N - P);
        if (P + jb2 < N) {
            ZGemmArgs g;
            g.M = jb2; g.N = N; g.K = N - P - jb2; g.alpha = cmk(-1, 0); g.beta = cmk(1, 0);
            g.A = A + MIDX(P, P + jb2, N); g.lda = N; g.opA = OP_N;
            g.B = X + (P + jb2); g.ldb = N; g.opB = OP_N;
            g.C = X + P; g.ldc = N;
            zgemm_cta<GemmBig>(g, 0, 1, gsm);
        }
        trsm_rows16(A, N, X, P, P + jb2, gsm, L);
    }
}

// X[p:N, c0:c0+nc] <- (I - V T V^H)^op X for a jb-wide block (jb <= 64; T ld 64)
static __device__ void apply_block64(const double2* Vs, const double2* Tp, int N, int p, int jb,
                                     double2* X, int c0, int nc, int use_th, LinalgScratch& sc, cplx* gsm) {
    if (nc <= 0) return;
    const int m = N - p;
    ZGemmArgs g;
    g.M = jb; g.N = nc; g.K = m; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
    g.A = Vs; g.lda = N; g.opA = OP_C;
    g.B = X + MIDX(p, c0, N); g.ldb = N; g.opB = OP_N;
    g.C = sc.Ws; g.ldc = QR_NB2;
    zgemm_cta<GemmBig>(g, 0, 1, gsm);
    g.M = jb; g.N = nc; g.K = jb;
    g.A = Tp; g.lda = QR_NB2; g.opA = use_th ? OP_C : OP_N;
    g.B = sc.Ws; g.ldb = QR_NB2; g.opB = OP_N;
    g.C = sc.Ws2; g.ldc = QR_NB2;
    zgemm_cta<GemmBig>(g, 0, 1, gsm);
    g.M = m; g.N = nc; g.K = jb; g.alpha = cmk(-1, 0); g.beta = cmk(1, 0);
    g.A = Vs; g.lda = N; g.opA = OP_N;
    g.B = sc.Ws2; g.ldb = QR_NB2; g.opB = OP_N;
    g.C = X + MIDX(p, c0, N); g.ldc = N;
    zgemm_cta<GemmBig>(g, 0, 1, gsm);
}

// T (64 x 64, ld 64, zero outside the upper triangle) of the block whose explicit
// V (jb2 columns, rows from the block's first row, ld N) is in sc.Vs, from the
// 16 x 16 triangles of its panels (Tp16, consecutive)
static __device__ void build_t64(int N, int P, int jb2, const double2* Tp16, double2* T64, LinalgScratch& sc,
                                 cplx* gsm) {
    const int tid = threadIdx.x, nth = blockDim.x, m = N - P;
    for (int e = tid; e < QR_NB2 * QR_NB2; e += nth) {
        const int a = e % QR_NB2, b = e / QR_NB2;
        T64[e] = (a < QR_NB && b < QR_NB && b < jb2) ? Tp16[a + b * QR_NB] : cmk(0, 0);
    }
    __syncthreads();
    for (int k = QR_NB; k < jb2; k += QR_NB) {
        const int jb = min(QR_NB, jb2 - k);
        const double2* Tb = Tp16 + (size_t)(k / QR_NB) * QR_NB * QR_NB;
        ZGemmArgs g;   // X = V_a^H V_b  (k x jb)
        g.M = k; g.N = jb; g.K = m; g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
        g.A = sc.Vs; g.lda = N; g.opA = OP_C;
        g.B = sc.Vs + (size_t)k * N; g.ldb = N; g.opB = OP_N;
        g.C = sc.Ws; g.ldc = QR_NB2;
        zgemm_cta<GemmBig>(g, 0, 1, gsm);
        // Y = T_a X (T_a upper triangular), then T(0:k, k:k+jb) = -Y T_b, with
        // T_a (k x k, ld k), X and Y (k x jb, ld k) and T_b staged in shared
        // memory (the GEMM staging buffer: k^2 + 2 k QR_NB + QR_NB^2 <= 4096
        // elements for k <= 48)
        double2* Tas = gsm;
        double2* Xs = Tas + k * k;
        double2* Ys = Xs + k * QR_NB;
        double2* Tbs = Ys + k * QR_NB;
        for (int e = tid; e < k * k; e += nth) Tas[e] = T64[(e % k) + (e / k) * QR_NB2];
        for (int e = tid; e < k * jb; e += nth) Xs[e] = sc.Ws[(e % k) + (e / k) * QR_NB2];
        for (int e = tid; e < QR_NB * QR_NB; e += nth) Tbs[e] = Tb[e];
        __syncthreads();
        for (int e = tid; e < k * jb; e += nth) {
            const int a = e % k, b = e / k;
            double2 acc = cmk(0, 0);
            for (int c = a; c < k; ++c) acc = cfma(Tas[a + c * k], Xs[c + b * k], acc);
            Ys[a + b * k] = acc;
        }
        __syncthreads();
        for (int e = tid; e < k * jb; e += nth) {
            const int a = e % k, b = e / k;
            double2 acc = cmk(0, 0);
            for (int c = 0; c <= b; ++c) acc = cfma(Ys[a + c * k], Tbs[c + b * QR_NB], acc);
            T64[a + (k + b) * QR_NB2] = cmk(-acc.x, -acc.y);
        }
        for (int e = tid; e < jb * jb; e += nth) {
            const int a = e % jb, b = e / jb;
            T64[(k + a) + (k + b) * QR_NB2] = Tb[a + b * QR_NB];
        }
        __syncthreads();
    }
}

// In-place QR of the first ncol columns of A (ld N), two-level blocked; R above
// the diagonal, reflectors below, tau, panel triangles in sc.T and block
// triangles in sc.T64.  smem_panel holds >= QR_PANEL_ELEMS(N) double2.
static __device__ void cta_qr64(double2* A, int N, LinalgScratch& sc, double2* smem_panel, cplx* gsm, LinalgSmem* L,
                                int ncol = -1) {
    if (ncol < 0) ncol = N;
    for (int P = 0; P < ncol; P += QR_NB2) {
        const int jb2 = min(QR_NB2, ncol - P);
        for (int p = P; p < P + jb2; p += QR_NB) {
            const int jb = min(QR_NB, P + jb2 - p), m = N - p, ldp = m + ((m & 1) ^ 1);
            double2* Pn = smem_panel;
            for (int e = threadIdx.x; e < m * jb; e += blockDim.x) {
                int r = e % m, cc = e / m;
                Pn[(size_t)cc * ldp + r] = A[MIDX(p + r, p + cc, N)];
            }
            __syncthreads();
            panel_qr(Pn, m, ldp, jb, sc.tau + p, L);
            double2* Tp = sc.T + (size_t)(p / QR_NB) * QR_NB * QR_NB;
            panel_larft(Pn, m, ldp, jb, sc.tau + p, Tp, L);
            for (int e = threadIdx.x; e < m * jb; e += blockDim.x) {
                int r = e % m, cc = e / m;
                A[MIDX(p + r, p + cc, N)] = Pn[(size_t)cc * ldp + r];
                sc.Vs[MIDX(r, cc, N)] = (r < cc) ? cmk(0, 0) : (r == cc) ? cmk(1, 0) : Pn[(size_t)cc * ldp + r];
            }
            __syncthreads();
            if (p + jb < P + jb2) apply_block(sc.Vs, Tp, N, p, jb, A, p + jb, P + jb2 - p - jb, 1, sc, gsm);
        }
        build_vblock(A, N, P, jb2, sc.Vs);
        double2* T64 = sc.T64 + (size_t)(P / QR_NB2) * QR_NB2 * QR_NB2;
        build_t64(N, P, jb2, sc.T + (size_t)(P / QR_NB) * QR_NB * QR_NB, T64, sc, gsm);
        if (P + jb2 < ncol) apply_block64(sc.Vs, T64, N, P, jb2, A, P + jb2, ncol - P - jb2, 1, sc, gsm);
    }
}

// The first ncol columns of Q (ld N) from cta_qr64's factors into Qout.
static __device__ void cta_form_q64(const double2* A, int N, double2* Qout, LinalgScratch& sc, cplx* gsm, int ncol = -1) {
    if (ncol < 0) ncol = N;
    for (int e = threadIdx.x; e < N * ncol; e += blockDim.x) {
        int r = e % N, cc = e / N;
        Qout[e] = cmk(r == cc ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    const int last = ((ncol - 1) / QR_NB2) * QR_NB2;
    for (int P = last; P >= 0; P -= QR_NB2) {
        const int jb2 = min(QR_NB2, ncol - P);
        build_vblock(A, N, P, jb2, sc.Vs);
        apply_block64(sc.Vs, sc.T64 + (size_t)(P / QR_NB2) * QR_NB2 * QR_NB2, N, P, jb2, Qout, P, ncol - P, 0, sc, gsm);
    }
}

// X <- Q^H X for all N columns of X (Q from cta_qr64 of an N x N matrix).
static __device__ void cta_apply_qh64(const double2* A, int N, double2* X, LinalgScratch& sc, cplx* gsm) {
    for (int P = 0; P < N; P += QR_NB2) {
        const int jb2 = min(QR_NB2, N - P);
        build_vblock(A, N, P, jb2, sc.Vs);
        apply_block64(sc.Vs, sc.T64 + (size_t)(P / QR_NB2) * QR_NB2 * QR_NB2, N, P, jb2, X, 0, N, 1, sc, gsm);
    }
}
