/* Dense complex linear algebra for the oracle.  Test infrastructure only.
 *
 * The reference calls Intel MKL (version not pinned: README.md:17-18 links
 * the oneAPI download; src/make.sys.square:31-35).  MKL is not vendored in
 * the reference, so the LAPACK routines are restated here from the published
 * LAPACK algorithms (zlarfg, zgeqr2, zlaqp2, zung2r, zgetf2, ztrti2), and the
 * s_matrix wrappers around them follow lib/s_matrix.f90.  Optional function
 * pointers (orc_set_lapack) route the same calls to an external BLAS/LAPACK,
 * which the CPU baseline uses for speed. */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

static orc_zgemm_fn  p_zgemm;
static orc_zgeqrf_fn p_zgeqrf;
static orc_zgeqp3_fn p_zgeqp3;
static orc_zungqr_fn p_zungqr;
static orc_zgetrf_fn p_zgetrf;
static orc_ztrtri_fn p_ztrtri;

void orc_set_lapack(orc_zgemm_fn a, orc_zgeqrf_fn b, orc_zgeqp3_fn c, orc_zungqr_fn d,
                    orc_zgetrf_fn e, orc_ztrtri_fn f) {
    p_zgemm = a; p_zgeqrf = b; p_zgeqp3 = c; p_zungqr = d; p_zgetrf = e; p_ztrtri = f;
}

/* C = alpha op(A) op(B) + beta C, op in {N, T, C} */
void orc_zgemm(char ta, char tb, int m, int n, int k, zc alpha, const zc *a, int lda,
               const zc *b, int ldb, zc beta, zc *c, int ldc) {
    if (p_zgemm) {
        p_zgemm(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
        return;
    }
    zc *col = malloc(sizeof(zc) * (size_t)(m > 0 ? m : 1));
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) col[i] = 0;
        for (int l = 0; l < k; ++l) {
            zc bl = (tb == 'N') ? b[ZIDX(l, j, ldb)] : (tb == 'T') ? b[ZIDX(j, l, ldb)] : conj(b[ZIDX(j, l, ldb)]);
            if (bl == 0) continue;
            if (ta == 'N') {
                const zc *ac = a + ZIDX(0, l, lda);
                for (int i = 0; i < m; ++i) col[i] += ac[i] * bl;
            } else if (ta == 'T') {
                for (int i = 0; i < m; ++i) col[i] += a[ZIDX(l, i, lda)] * bl;
            } else {
                for (int i = 0; i < m; ++i) col[i] += conj(a[ZIDX(l, i, lda)]) * bl;
            }
        }
        zc *cc = c + ZIDX(0, j, ldc);
        if (beta == 0) for (int i = 0; i < m; ++i) cc[i] = alpha * col[i];
        else for (int i = 0; i < m; ++i) cc[i] = alpha * col[i] + beta * cc[i];
    }
    free(col);
}

/* scaled 2-norm (dznrm2) */
double orc_dznrm2(int n, const zc *x, int incx) {
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        double v[2] = {creal(x[(size_t)i * incx]), cimag(x[(size_t)i * incx])};
        for (int t = 0; t < 2; ++t) {
            if (v[t] != 0.0) {
                double a = fabs(v[t]);
                if (scale < a) { ssq = 1.0 + ssq * (scale / a) * (scale / a); scale = a; }
                else ssq += (a / scale) * (a / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

static double dlapy3(double x, double y, double z) {
    double xa = fabs(x), ya = fabs(y), za = fabs(z);
    double w = fmax(xa, fmax(ya, za));
    if (w == 0.0) return xa + ya + za;
    return w * sqrt((xa / w) * (xa / w) + (ya / w) * (ya / w) + (za / w) * (za / w));
}

/* zlarfg: H^H (alpha; x) = (beta; 0), H = I - tau v v^H, v(1)=1, beta real */
static void zlarfg(int n, zc *alpha, zc *x, int incx, zc *tau) {
    if (n <= 0) { *tau = 0; return; }
    double xnorm = orc_dznrm2(n - 1, x, incx);
    double alphr = creal(*alpha), alphi = cimag(*alpha);
    if (xnorm == 0.0 && alphi == 0.0) { *tau = 0; return; }
    double beta = -copysign(dlapy3(alphr, alphi, xnorm), alphr);
    double safmin = DBL_MIN / (DBL_EPSILON * 0.5), rsafmn = 1.0 / safmin;
    int knt = 0;
    if (fabs(beta) < safmin) {
        do {
            ++knt;
            for (int i = 0; i < n - 1; ++i) x[(size_t)i * incx] *= rsafmn;
            beta *= rsafmn; alphi *= rsafmn; alphr *= rsafmn;
        } while (fabs(beta) < safmin && knt < 20);
        xnorm = orc_dznrm2(n - 1, x, incx);
        *alpha = alphr + I * alphi;
        beta = -copysign(dlapy3(alphr, alphi, xnorm), alphr);
    }
    *tau = (beta - alphr) / beta + I * (-alphi / beta);
    zc scal = 1.0 / (*alpha - beta);
    for (int i = 0; i < n - 1; ++i) x[(size_t)i * incx] *= scal;
    for (int j = 0; j < knt; ++j) beta *= safmin;
    *alpha = beta;
}

/* zlarf('L'): C = (I - tau v v^H) C, C is m x n */
static void zlarf_left(int m, int n, const zc *v, zc tau, zc *c, int ldc) {
    if (tau == 0) return;
    for (int j = 0; j < n; ++j) {
        zc w = 0;
        zc *cj = c + ZIDX(0, j, ldc);
        for (int i = 0; i < m; ++i) w += conj(v[i]) * cj[i];
        w *= tau;
        for (int i = 0; i < m; ++i) cj[i] -= v[i] * w;
    }
}

void orc_zgeqr2(int m, int n, double *ad, int lda, double *taud) {
    zc *a = (zc *)ad, *tau = (zc *)taud;
    int k = m < n ? m : n;
    for (int i = 0; i < k; ++i) {
        zlarfg(m - i, &a[ZIDX(i, i, lda)], &a[ZIDX(i + 1 < m ? i + 1 : i, i, lda)], 1, &tau[i]);
        if (i < n - 1) {
            zc aii = a[ZIDX(i, i, lda)];
            a[ZIDX(i, i, lda)] = 1;
            zlarf_left(m - i, n - i - 1, &a[ZIDX(i, i, lda)], conj(tau[i]), &a[ZIDX(i, i + 1, lda)], lda);
            a[ZIDX(i, i, lda)] = aii;
        }
    }
}

/* zlaqp2 with all columns free (jpvt = 0 on entry, as s_zgeQRPT_logdetQ
 * passes): QR with column pivoting and partial-norm downdating.
 * jpvt returns 1-based original column indices. */
void orc_zgeqp2(int m, int n, double *ad, int lda, int32_t *jpvt, double *taud) {
    zc *a = (zc *)ad, *tau = (zc *)taud;
    double *vn1 = malloc(sizeof(double) * n), *vn2 = malloc(sizeof(double) * n);
    double tol3z = sqrt(DBL_EPSILON * 0.5);
    for (int j = 0; j < n; ++j) {
        jpvt[j] = j + 1;
        vn1[j] = orc_dznrm2(m, &a[ZIDX(0, j, lda)], 1);
        vn2[j] = vn1[j];
    }
    int mn = m < n ? m : n;
    for (int i = 0; i < mn; ++i) {
        int pvt = i;
        double best = fabs(vn1[i]);
        for (int j = i + 1; j < n; ++j) if (fabs(vn1[j]) > best) { best = fabs(vn1[j]); pvt = j; }
        if (pvt != i) {
            for (int r = 0; r < m; ++r) {
                zc t = a[ZIDX(r, pvt, lda)]; a[ZIDX(r, pvt, lda)] = a[ZIDX(r, i, lda)]; a[ZIDX(r, i, lda)] = t;
            }
            int it = jpvt[pvt]; jpvt[pvt] = jpvt[i]; jpvt[i] = it;
            vn1[pvt] = vn1[i]; vn2[pvt] = vn2[i];
        }
        zlarfg(m - i, &a[ZIDX(i, i, lda)], &a[ZIDX(i + 1 < m ? i + 1 : i, i, lda)], 1, &tau[i]);
        if (i < n - 1) {
            zc aii = a[ZIDX(i, i, lda)];
            a[ZIDX(i, i, lda)] = 1;
            zlarf_left(m - i, n - i - 1, &a[ZIDX(i, i, lda)], conj(tau[i]), &a[ZIDX(i, i + 1, lda)], lda);
            a[ZIDX(i, i, lda)] = aii;
        }
        for (int j = i + 1; j < n; ++j) {
            if (vn1[j] != 0.0) {
                double t = cabs(a[ZIDX(i, j, lda)]) / vn1[j];
                t = 1.0 - t * t;
                if (t < 0.0) t = 0.0;
                double t2 = t * (vn1[j] / vn2[j]) * (vn1[j] / vn2[j]);
                if (t2 <= tol3z) {
                    if (i < m - 1) {
                        vn1[j] = orc_dznrm2(m - i - 1, &a[ZIDX(i + 1, j, lda)], 1);
                        vn2[j] = vn1[j];
                    } else { vn1[j] = 0.0; vn2[j] = 0.0; }
                } else {
                    vn1[j] *= sqrt(t);
                }
            }
        }
    }
    free(vn1); free(vn2);
}

/* zung2r: form the m x n matrix Q with orthonormal columns from k reflectors */
void orc_zung2r(int m, int n, int k, double *ad, int lda, const double *taud) {
    zc *a = (zc *)ad;
    const zc *tau = (const zc *)taud;
    for (int j = k; j < n; ++j) {
        for (int l = 0; l < m; ++l) a[ZIDX(l, j, lda)] = 0;
        a[ZIDX(j, j, lda)] = 1;
    }
    for (int i = k - 1; i >= 0; --i) {
        if (i < n - 1) {
            a[ZIDX(i, i, lda)] = 1;
            zlarf_left(m - i, n - i - 1, &a[ZIDX(i, i, lda)], tau[i], &a[ZIDX(i, i + 1, lda)], lda);
        }
        for (int l = i + 1; l < m; ++l) a[ZIDX(l, i, lda)] *= -tau[i];
        a[ZIDX(i, i, lda)] = 1.0 - tau[i];
        for (int l = 0; l < i; ++l) a[ZIDX(l, i, lda)] = 0;
    }
}

static double cabs1(zc z) { return fabs(creal(z)) + fabs(cimag(z)); }

/* zgetf2: LU with partial pivoting; pivot = first max |re|+|im| (izamax).
 * ipiv is 1-based; returns info. */
int orc_zgetf2(int m, int n, double *ad, int lda, int32_t *ipiv) {
    zc *a = (zc *)ad;
    int info = 0, mn = m < n ? m : n;
    double sfmin = DBL_MIN;
    for (int j = 0; j < mn; ++j) {
        int jp = j;
        double best = cabs1(a[ZIDX(j, j, lda)]);
        for (int i = j + 1; i < m; ++i) if (cabs1(a[ZIDX(i, j, lda)]) > best) { best = cabs1(a[ZIDX(i, j, lda)]); jp = i; }
        ipiv[j] = jp + 1;
        if (a[ZIDX(jp, j, lda)] != 0) {
            if (jp != j)
                for (int c = 0; c < n; ++c) {
                    zc t = a[ZIDX(j, c, lda)]; a[ZIDX(j, c, lda)] = a[ZIDX(jp, c, lda)]; a[ZIDX(jp, c, lda)] = t;
                }
            if (j < m - 1) {
                zc piv = a[ZIDX(j, j, lda)];
                if (cabs(piv) >= sfmin) {
                    zc r = 1.0 / piv;
                    for (int i = j + 1; i < m; ++i) a[ZIDX(i, j, lda)] *= r;
                } else {
                    for (int i = j + 1; i < m; ++i) a[ZIDX(i, j, lda)] /= piv;
                }
            }
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; ++c) {
            zc u = a[ZIDX(j, c, lda)];
            if (u == 0) continue;
            for (int i = j + 1; i < m; ++i) a[ZIDX(i, c, lda)] -= a[ZIDX(i, j, lda)] * u;
        }
    }
    return info;
}

/* ztrti2: in-place inverse of the upper (non-unit) or lower (unit) triangle */
static void ztrti2_upper(int n, zc *a, int lda) {
    for (int j = 0; j < n; ++j) {
        a[ZIDX(j, j, lda)] = 1.0 / a[ZIDX(j, j, lda)];
        zc ajj = -a[ZIDX(j, j, lda)];
        /* x = T(0:j,0:j) * a(0:j, j), T upper already inverted */
        for (int i = 0; i < j; ++i) {
            zc s = 0;
            for (int l = i; l < j; ++l) s += a[ZIDX(i, l, lda)] * a[ZIDX(l, j, lda)];
            a[ZIDX(i, j, lda)] = s;
        }
        for (int i = 0; i < j; ++i) a[ZIDX(i, j, lda)] *= ajj;
    }
}

static void ztrti2_lower_unit(int n, zc *a, int lda) {
    for (int j = n - 1; j >= 0; --j) {
        /* x = T(j+1:n, j+1:n) * a(j+1:n, j), T unit lower already inverted */
        for (int i = n - 1; i > j; --i) {
            zc s = a[ZIDX(i, j, lda)];
            for (int l = j + 1; l < i; ++l) s += a[ZIDX(i, l, lda)] * a[ZIDX(l, j, lda)];
            a[ZIDX(i, j, lda)] = s;
        }
        for (int i = j + 1; i < n; ++i) a[ZIDX(i, j, lda)] = -a[ZIDX(i, j, lda)];
    }
}

/* s_zmcpt (lib/s_matrix.f90:785-823): selection sort of columns by 2-norm,
 * decreasing; jpvt(k) = original column now at k (1-based). */
void orc_zmcpt(int rdim, int cdim, double *ad, int32_t *jpvt) {
    zc *a = (zc *)ad;
    double *vn1 = malloc(sizeof(double) * cdim);
    for (int k = 0; k < cdim; ++k) { vn1[k] = orc_dznrm2(rdim, &a[ZIDX(0, k, rdim)], 1); jpvt[k] = k + 1; }
    for (int k = 0; k < cdim; ++k) {
        int pvt = k;
        double best = fabs(vn1[k]);
        for (int j = k + 1; j < cdim; ++j) if (fabs(vn1[j]) > best) { best = fabs(vn1[j]); pvt = j; }
        if (pvt != k) {
            for (int r = 0; r < rdim; ++r) {
                zc t = a[ZIDX(r, pvt, rdim)]; a[ZIDX(r, pvt, rdim)] = a[ZIDX(r, k, rdim)]; a[ZIDX(r, k, rdim)] = t;
            }
            int it = jpvt[pvt]; jpvt[pvt] = jpvt[k]; jpvt[k] = it;
            vn1[pvt] = vn1[k];
        }
    }
    free(vn1);
}

static zc logdet_q(int n, const zc *tau) {   /* s_matrix.f90:1290-1298 */
    zc z = 0;
    for (int i = 0; i < n; ++i)
        if (cabs(tau[i]) != 0.0)
            z += clog(1.0 - tau[i] * (2.0 * creal(tau[i])) / (tau[i] * conj(tau[i])));
    return z;
}

static void split_qr(int n, const zc *a, const zc *tau, zc *q, zc *r) {
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            r[ZIDX(i, j, n)] = (i > j) ? 0 : a[ZIDX(i, j, n)];
            q[ZIDX(i, j, n)] = (i > j) ? a[ZIDX(i, j, n)] : (i == j ? 1 : 0);
        }
    if (p_zungqr) {
        int lwork = 64 * n, info;
        zc *work = malloc(sizeof(zc) * lwork);
        p_zungqr(&n, &n, &n, q, &n, tau, work, &lwork, &info);
        free(work);
    } else {
        orc_zung2r(n, n, n, (double *)q, n, (const double *)tau);
    }
}

/* s_zgeQR_logdetQ (lib/s_matrix.f90:1998-2109), square case */
void orc_qr_logdet(int n, zc *a, zc *q, zc *r, zc *logdet) {
    zc *tau = malloc(sizeof(zc) * n);
    if (p_zgeqrf) {
        int lwork = 64 * n, info;
        zc *work = malloc(sizeof(zc) * lwork);
        p_zgeqrf(&n, &n, a, &n, tau, work, &lwork, &info);
        free(work);
    } else {
        orc_zgeqr2(n, n, (double *)a, n, (double *)tau);
    }
    *logdet = logdet_q(n, tau);
    split_qr(n, a, tau, q, r);
    free(tau);
}

/* s_zgeQRPT_logdetQ (lib/s_matrix.f90:1222-1341), square case */
void orc_qrpt_logdet(int n, zc *a, zc *q, zc *r, int32_t *jpvt, zc *logdet) {
    zc *tau = malloc(sizeof(zc) * n);
    if (p_zgeqp3) {
        int lwork = 64 * n, info;
        zc *work = malloc(sizeof(zc) * lwork);
        double *rwork = malloc(sizeof(double) * 2 * n);
        int *jp = malloc(sizeof(int) * n);
        for (int i = 0; i < n; ++i) jp[i] = 0;
        p_zgeqp3(&n, &n, a, &n, jp, tau, work, &lwork, rwork, &info);
        for (int i = 0; i < n; ++i) jpvt[i] = jp[i];
        free(work); free(rwork); free(jp);
    } else {
        orc_zgeqp2(n, n, (double *)a, n, jpvt, (double *)tau);
    }
    *logdet = logdet_q(n, tau);
    split_qr(n, a, tau, q, r);
    free(tau);
}

/* shared tail of s_invlu_z / s_inv_logdet_lu_z (lib/s_matrix.f90:2586-2820) */
static void lu_inverse(int n, zc *a, const int32_t *ipiv) {
    zc *umat = malloc(sizeof(zc) * n * n), *lmat = malloc(sizeof(zc) * n * n);
    int info;
    if (p_ztrtri) { char u = 'U', d = 'N'; p_ztrtri(&u, &d, &n, a, &n, &info); }
    else ztrti2_upper(n, a, n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) umat[ZIDX(i, j, n)] = (i > j) ? 0 : a[ZIDX(i, j, n)];
    if (p_ztrtri) { char l = 'L', d = 'U'; p_ztrtri(&l, &d, &n, a, &n, &info); }
    else ztrti2_lower_unit(n, a, n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            lmat[ZIDX(i, j, n)] = (i > j) ? a[ZIDX(i, j, n)] : (i == j ? 1 : 0);
    for (int k = n - 2; k >= 0; --k) {
        int pv = ipiv[k] - 1;
        if (pv != k)
            for (int r = 0; r < n; ++r) {
                zc t = lmat[ZIDX(r, k, n)]; lmat[ZIDX(r, k, n)] = lmat[ZIDX(r, pv, n)]; lmat[ZIDX(r, pv, n)] = t;
            }
    }
    orc_zgemm('N', 'N', n, n, n, 1.0, umat, n, lmat, n, 0.0, a, n);
    free(umat); free(lmat);
}

static int lu_factor(int n, zc *a, int32_t *ipiv) {
    if (p_zgetrf) {
        int info, *ip = malloc(sizeof(int) * n);
        p_zgetrf(&n, &n, a, &n, ip, &info);
        for (int i = 0; i < n; ++i) ipiv[i] = ip[i];
        free(ip);
        return info;
    }
    return orc_zgetf2(n, n, (double *)a, n, ipiv);
}

void orc_zinv_logdet(int n, zc *a, zc *logdet) {
    int32_t *ipiv = malloc(sizeof(int32_t) * n);
    lu_factor(n, a, ipiv);
    zc z = 0;
    for (int i = 0; i < n; ++i)
        z += (ipiv[i] == i + 1) ? clog(a[ZIDX(i, i, n)]) : clog(-a[ZIDX(i, i, n)]);
    double im = cimag(z);
    int k = (int)lround(im / 2.0 / M_PI);
    im -= 2.0 * M_PI * k;
    *logdet = creal(z) + I * im;
    lu_inverse(n, a, ipiv);
    free(ipiv);
}

void orc_zinv(int n, zc *a) {
    int32_t *ipiv = malloc(sizeof(int32_t) * n);
    lu_factor(n, a, ipiv);
    lu_inverse(n, a, ipiv);
    free(ipiv);
}

void orc_inv_logdet_lu(int n, double *a, double *logdet) {
    zc z;
    orc_zinv_logdet(n, (zc *)a, &z);
    logdet[0] = creal(z); logdet[1] = cimag(z);
}

/* ------------------------------------------------------------------ */
/* projective-path helpers                                             */
/* ------------------------------------------------------------------ */
static orc_zheev_fn p_zheev;
void orc_set_zheev(orc_zheev_fn f) { p_zheev = f; }

/* s_zgeQR_pqmc (lib/s_matrix.f90:1822-1996): Q of amat (rdim x cdim) with
 * det R > 0, returns log |det R|.  A wide amat is factored through its plain
 * transpose and Q is returned transposed (rdim x cdim). */
double orc_qr_pqmc(int rdim, int cdim, const zc *amat, zc *qmat) {
    int tall = rdim >= cdim;
    int n1 = tall ? rdim : cdim, n2 = tall ? cdim : rdim, mn = n2;
    zc *a = malloc(sizeof(zc) * (size_t)n1 * n2), *tau = malloc(sizeof(zc) * mn);
    zc *q = malloc(sizeof(zc) * (size_t)n1 * n2);
    for (int j = 0; j < n2; ++j)
        for (int i = 0; i < n1; ++i)
            a[ZIDX(i, j, n1)] = tall ? amat[ZIDX(i, j, rdim)] : amat[ZIDX(j, i, rdim)];
    if (p_zgeqrf) {
        int lwork = 64 * n1, info;
        zc *work = malloc(sizeof(zc) * lwork);
        p_zgeqrf(&n1, &n2, a, &n1, tau, work, &lwork, &info);
        free(work);
    } else {
        orc_zgeqr2(n1, n2, (double *)a, n1, (double *)tau);
    }
    int isgn = 0;
    double rlogdet = 0.0;
    for (int i = 0; i < mn; ++i) {
        double r = creal(a[ZIDX(i, i, n1)]);
        if (r < 0.0) { ++isgn; rlogdet += log(-r); } else rlogdet += log(r);
    }
    for (int j = 0; j < mn; ++j)
        for (int i = 0; i < n1; ++i)
            q[ZIDX(i, j, n1)] = (i > j) ? a[ZIDX(i, j, n1)] : (i == j ? 1.0 : 0.0);
    if (p_zungqr) {
        int lwork = 64 * n1, info;
        zc *work = malloc(sizeof(zc) * lwork);
        p_zungqr(&n1, &mn, &mn, q, &n1, tau, work, &lwork, &info);
        free(work);
    } else {
        orc_zung2r(n1, mn, mn, (double *)q, n1, (const double *)tau);
    }
    if (isgn % 2 == 1)
        for (int i = 0; i < n1; ++i) q[ZIDX(i, 0, n1)] = -q[ZIDX(i, 0, n1)];
    for (int j = 0; j < n2; ++j)
        for (int i = 0; i < n1; ++i) {
            if (tall) qmat[ZIDX(i, j, rdim)] = q[ZIDX(i, j, n1)];
            else qmat[ZIDX(j, i, rdim)] = q[ZIDX(i, j, n1)];
        }
    free(a); free(tau); free(q);
    return rlogdet;
}

/* cyclic complex Jacobi for a Hermitian matrix (used when no LAPACK zheev is
 * hooked); eigenvalues ascending, eigenvectors in the columns of v */
static void jacobi_he(int n, const zc *h, double *w, zc *v) {
    zc *a = malloc(sizeof(zc) * (size_t)n * n);
    memcpy(a, h, sizeof(zc) * (size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) v[ZIDX(i, j, n)] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, dia = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double t = cabs(a[ZIDX(i, j, n)]);
                if (i != j) off += t * t; else dia += t * t;
            }
        if (off <= 1e-30 * (dia > 1e-300 ? dia : 1e-300)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                zc apq = a[ZIDX(p, q, n)];
                double ab = cabs(apq);
                if (ab < 1e-300) continue;
                double app = creal(a[ZIDX(p, p, n)]), aqq = creal(a[ZIDX(q, q, n)]);
                zc ph = apq / ab;                     /* apq = |apq| e^{i phi} */
                double theta = 0.5 * atan2(2.0 * ab, aqq - app);
                double cs = cos(theta), sn = sin(theta);
                /* rotation J: columns p,q -> p' = c p - s conj(ph) q ... written as
                 * J = [[c, s ph], [-s conj(ph), c]] acting on the (p,q) plane */
                zc jpp = cs, jpq = sn * ph, jqp = -sn * conj(ph), jqq = cs;
                for (int k = 0; k < n; ++k) {         /* A <- A J */
                    zc x = a[ZIDX(k, p, n)], y = a[ZIDX(k, q, n)];
                    a[ZIDX(k, p, n)] = x * jpp + y * jqp;
                    a[ZIDX(k, q, n)] = x * jpq + y * jqq;
                }
                for (int k = 0; k < n; ++k) {         /* A <- J^H A */
                    zc x = a[ZIDX(p, k, n)], y = a[ZIDX(q, k, n)];
                    a[ZIDX(p, k, n)] = conj(jpp) * x + conj(jqp) * y;
                    a[ZIDX(q, k, n)] = conj(jpq) * x + conj(jqq) * y;
                }
                for (int k = 0; k < n; ++k) {         /* V <- V J */
                    zc x = v[ZIDX(k, p, n)], y = v[ZIDX(k, q, n)];
                    v[ZIDX(k, p, n)] = x * jpp + y * jqp;
                    v[ZIDX(k, q, n)] = x * jpq + y * jqq;
                }
                a[ZIDX(p, q, n)] = 0; a[ZIDX(q, p, n)] = 0;
            }
    }
    /* ascending selection sort of eigenpairs */
    for (int i = 0; i < n; ++i) w[i] = creal(a[ZIDX(i, i, n)]);
    for (int i = 0; i < n; ++i) {
        int k = i;
        for (int j = i + 1; j < n; ++j) if (w[j] < w[k]) k = j;
        if (k != i) {
            double t = w[i]; w[i] = w[k]; w[k] = t;
            for (int r = 0; r < n; ++r) { zc x = v[ZIDX(r, i, n)]; v[ZIDX(r, i, n)] = v[ZIDX(r, k, n)]; v[ZIDX(r, k, n)] = x; }
        }
    }
    free(a);
}

/* s_eig_he (lib/s_matrix.f90:202-253): zheev('V','U') */
void orc_eig_he(int n, const zc *h, double *w, zc *v) {
    if (p_zheev) {
        memcpy(v, h, sizeof(zc) * (size_t)n * n);
        int lwork = 2 * n - 1 > 64 * n ? 2 * n - 1 : 64 * n, info;
        zc *work = malloc(sizeof(zc) * lwork);
        double *rwork = malloc(sizeof(double) * (3 * n > 1 ? 3 * n : 1));
        char jv = 'V', up = 'U';
        p_zheev(&jv, &up, &n, v, &n, w, work, &lwork, rwork, &info);
        free(work); free(rwork);
    } else {
        jacobi_he(n, h, w, v);
    }
}
