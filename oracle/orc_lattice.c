/* Square, honeycomb, chain and cubic lattice tables, restated from
 * src/lattice.f90 (setup_latt2d_sub 386-491, setup_honeycomb_sub 611-776,
 * setup_square_sub 792-961, setup_latt1d_sub 67-135, setup_chain_sub 240-316,
 * setup_latt3d_sub 1033-1157, setup_cubic_sub 1280-1472) and the hopping
 * phase expar (src/dqmc_config_h0/expar.f90, expar1d.f90, expar3d.f90).
 * Test infrastructure only.
 * Stored values are 1-based as in the reference. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

static int npbc(int nr, int l) {   /* lattice.f90:493-500 */
    if (nr > l) return nr - l;
    if (nr < 1) return nr + l;
    return nr;
}

void orc_latt_free(orc_latt *L) {
    free(L->ulist); free(L->list); free(L->cord); free(L->rcord); free(L->nnlist);
    free(L->snlist); free(L->nnlf_list); free(L->nnveci); free(L->nnvecr); free(L->imj);
    free(L->plq_cord); free(L->listk); free(L->zexpiqr); free(L->ulist3);
    memset(L, 0, sizeof(*L));
}

static void setup_2d(orc_latt *L, int l1, int l2, const double a1[2], const double a2[2]) {
    L->l1 = l1; L->l2 = l2; L->ncell = l1 * l2;
    L->a1[0] = a1[0]; L->a1[1] = a1[1]; L->a2[0] = a2[0]; L->a2[1] = a2[1];
    int nc = L->ncell;
    L->ulist = malloc(sizeof(int) * 2 * nc);
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int c = i2 + (i1 - 1) * l2 - 1;
            L->ulist[c * 2 + 0] = i1;
            L->ulist[c * 2 + 1] = i2;
        }
    /* lattice reciprocal vectors b = 2 pi [l1 a1, l2 a2]^{-1} */
    double m11 = l1 * a1[0], m12 = l1 * a1[1], m21 = l2 * a2[0], m22 = l2 * a2[1];
    double x = m11 * m22 - m21 * m12;
    double i11 = m22 / x, i22 = m11 / x, i12 = -m12 / x, i21 = -m21 / x;
    L->b1[0] = 2 * M_PI * i11; L->b1[1] = 2 * M_PI * i21;
    L->b2[0] = 2 * M_PI * i12; L->b2[1] = 2 * M_PI * i22;
    L->listk = malloc(sizeof(int) * 2 * nc);
    int k = 0;
    for (int m = -(l1 + 1) / 2 + 1; m <= l1 / 2; ++m)
        for (int n = -(l2 + 1) / 2 + 1; n <= l2 / 2; ++n) {
            L->listk[k * 2 + 0] = m; L->listk[k * 2 + 1] = n; ++k;
        }
    L->imj = malloc(sizeof(int) * nc * nc);
    for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nc; ++i) {
            int nx = npbc(L->ulist[i * 2] - L->ulist[j * 2], l1);
            int ny = npbc(L->ulist[i * 2 + 1] - L->ulist[j * 2 + 1], l2);
            L->imj[i * nc + j] = ny + (nx - 1) * l2;
        }
    L->zexpiqr = malloc(sizeof(zc) * nc * nc);
    for (int i = 0; i < nc; ++i) {
        double ax = L->ulist[i * 2] * a1[0] + L->ulist[i * 2 + 1] * a2[0];
        double ay = L->ulist[i * 2] * a1[1] + L->ulist[i * 2 + 1] * a2[1];
        for (int nk = 0; nk < nc; ++nk) {
            double kx = L->listk[nk * 2] * L->b1[0] + L->listk[nk * 2 + 1] * L->b2[0];
            double ky = L->listk[nk * 2] * L->b1[1] + L->listk[nk * 2 + 1] * L->b2[1];
            L->zexpiqr[i * nc + nk] = cexp(I * (kx * ax + ky * ay));
        }
    }
}

static void setup_square(orc_latt *L, int l1, int l2) {
    const double a1[2] = {1.0, 0.0}, a2[2] = {0.0, 1.0};
    setup_2d(L, l1, l2, a1, a2);
    L->kind = ORC_SQUARE; L->nsub = 1; L->nsites = l1 * l2; L->z_plq = 4;
    L->nn_nf = 4; L->nn_lf = l1 * l2 / 2; L->nsn = 4;
    int ns = L->nsites;
    L->cord = malloc(sizeof(int) * 2 * ns);
    L->rcord = malloc(sizeof(double) * 2 * ns);
    L->nnlf_list = malloc(sizeof(int) * L->nn_lf);
    L->list = malloc(sizeof(int) * 2 * ns);
    int ind = 0;
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int s = i2 + (i1 - 1) * l2 - 1;
            L->list[s * 2] = s + 1; L->list[s * 2 + 1] = 1;
            L->rcord[s * 2] = i1; L->rcord[s * 2 + 1] = i2;
            if ((i1 + i2) % 2 == 0) L->nnlf_list[ind++] = s + 1;
        }
    memcpy(L->cord, L->ulist, sizeof(int) * 2 * ns);
    L->nnvecr = malloc(sizeof(double) * ns * 4 * 2);
    L->nnveci = malloc(sizeof(int) * ns * 4 * 2);
    static const int v[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    for (int i = 0; i < ns; ++i)
        for (int nf = 0; nf < 4; ++nf) {
            L->nnvecr[(i * 4 + nf) * 2] = v[nf][0]; L->nnvecr[(i * 4 + nf) * 2 + 1] = v[nf][1];
            L->nnveci[(i * 4 + nf) * 2] = v[nf][0]; L->nnveci[(i * 4 + nf) * 2 + 1] = v[nf][1];
        }
    L->nnlist = malloc(sizeof(int) * ns * 4);
    L->snlist = malloc(sizeof(int) * ns * 4);
    for (int i = 0; i < L->ncell; ++i) {
        int u1 = L->ulist[i * 2], u2 = L->ulist[i * 2 + 1];
#define SQ(d1, d2) ((npbc(u1 + (d1), l1) - 1) * l2 + npbc(u2 + (d2), l2))
        L->nnlist[i * 4 + 0] = SQ(1, 0);
        L->nnlist[i * 4 + 1] = SQ(0, 1);
        L->nnlist[i * 4 + 2] = SQ(-1, 0);
        L->nnlist[i * 4 + 3] = SQ(0, -1);
        L->snlist[i * 4 + 0] = SQ(1, 1);
        L->snlist[i * 4 + 1] = SQ(-1, 1);
        L->snlist[i * 4 + 2] = SQ(-1, -1);
        L->snlist[i * 4 + 3] = SQ(1, -1);
#undef SQ
    }
    /* plaquettes: A (odd,odd), B (even,odd), C (even,even), D (odd,even) */
    L->plq_cord = malloc(sizeof(int) * 4 * L->ncell);
    int nd[4] = {0, 0, 0, 0};
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int t = (i1 % 2 == 1 && i2 % 2 == 1) ? 0 : (i1 % 2 == 0 && i2 % 2 == 1) ? 1
                  : (i1 % 2 == 0 && i2 % 2 == 0) ? 2 : 3;
            nd[t]++;
        }
    int id[4] = {0, 0, 0, 0};
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int t = (i1 % 2 == 1 && i2 % 2 == 1) ? 0 : (i1 % 2 == 0 && i2 % 2 == 1) ? 1
                  : (i1 % 2 == 0 && i2 % 2 == 0) ? 2 : 3;
            int off = 0;
            for (int q = 0; q < t; ++q) off += nd[q];
            int pid = ++id[t] + off - 1;
#define INV(a, b) ((b) + ((a) - 1) * l2)
            L->plq_cord[pid * 4 + 0] = INV(i1, i2);
            L->plq_cord[pid * 4 + 1] = INV(npbc(i1 + 1, l1), i2);
            L->plq_cord[pid * 4 + 2] = INV(npbc(i1 + 1, l1), npbc(i2 + 1, l2));
            L->plq_cord[pid * 4 + 3] = INV(i1, npbc(i2 + 1, l2));
#undef INV
        }
}

static void setup_honeycomb(orc_latt *L, int l1, int l2) {
    const double a1[2] = {0.5, -0.5 * sqrt(3.0)}, a2[2] = {0.5, 0.5 * sqrt(3.0)};
    setup_2d(L, l1, l2, a1, a2);
    L->kind = ORC_HONEYCOMB; L->nsub = 2; L->nsites = l1 * l2 * 2; L->z_plq = 6;
    L->nn_nf = 3; L->nn_lf = l1 * l2; L->nsn = 6;
    int ns = L->nsites;
    L->cord = malloc(sizeof(int) * 2 * ns);
    L->rcord = malloc(sizeof(double) * 2 * ns);
    L->nnlf_list = malloc(sizeof(int) * L->nn_lf);
    L->list = malloc(sizeof(int) * 2 * ns);
    for (int i = 0; i < L->nn_lf; ++i) L->nnlf_list[i] = 2 * (i + 1) - 1;
    int ind = 0;
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int o = 1; o <= 2; ++o) {
                int s = ind++;
                L->list[s * 2] = i2 + (i1 - 1) * l2; L->list[s * 2 + 1] = o;
                L->cord[s * 2] = i1; L->cord[s * 2 + 1] = i2;
                if (o == 1) { L->rcord[s * 2] = i1; L->rcord[s * 2 + 1] = i2; }
                else { L->rcord[s * 2] = i1 - 1.0 / 3.0; L->rcord[s * 2 + 1] = i2 + 1.0 / 3.0; }
            }
    L->nnvecr = malloc(sizeof(double) * ns * 3 * 2);
    L->nnveci = malloc(sizeof(int) * ns * 3 * 2);
    static const double vrA[3][2] = {{-1.0 / 3, 1.0 / 3}, {2.0 / 3, 1.0 / 3}, {-1.0 / 3, -2.0 / 3}};
    static const int viA[3][2] = {{0, 0}, {1, 0}, {0, -1}};
    static const double vrB[3][2] = {{1.0 / 3, -1.0 / 3}, {-2.0 / 3, -1.0 / 3}, {1.0 / 3, 2.0 / 3}};
    static const int viB[3][2] = {{0, 0}, {-1, 0}, {0, 1}};
    for (int i = 0; i < ns; ++i)
        for (int nf = 0; nf < 3; ++nf) {
            int isA = (i % 2 == 0);
            L->nnvecr[(i * 3 + nf) * 2] = isA ? vrA[nf][0] : vrB[nf][0];
            L->nnvecr[(i * 3 + nf) * 2 + 1] = isA ? vrA[nf][1] : vrB[nf][1];
            L->nnveci[(i * 3 + nf) * 2] = isA ? viA[nf][0] : viB[nf][0];
            L->nnveci[(i * 3 + nf) * 2 + 1] = isA ? viA[nf][1] : viB[nf][1];
        }
    L->nnlist = malloc(sizeof(int) * ns * 3);
    L->snlist = malloc(sizeof(int) * ns * 6);
    for (int i = 0; i < ns; ++i) {
        int c1 = L->cord[i * 2], c2 = L->cord[i * 2 + 1], i1 = i + 1;
#define HC(d1, d2) (((npbc(c1 + (d1), l1) - 1) * l2 + npbc(c2 + (d2), l2)) * 2)
        if (i1 % 2 == 1) {
            L->nnlist[i * 3 + 0] = i1 + 1;
            L->nnlist[i * 3 + 1] = HC(1, 0);
            L->nnlist[i * 3 + 2] = HC(0, -1);
            L->snlist[i * 6 + 0] = HC(1, 1) - 1;
            L->snlist[i * 6 + 1] = HC(1, 0) - 1;
            L->snlist[i * 6 + 2] = HC(0, -1) - 1;
            L->snlist[i * 6 + 3] = HC(-1, -1) - 1;
            L->snlist[i * 6 + 4] = HC(-1, 0) - 1;
            L->snlist[i * 6 + 5] = HC(0, 1) - 1;
        } else {
            L->nnlist[i * 3 + 0] = i1 - 1;
            L->nnlist[i * 3 + 1] = HC(-1, 0) - 1;
            L->nnlist[i * 3 + 2] = HC(0, 1) - 1;
            L->snlist[i * 6 + 0] = HC(1, 1);
            L->snlist[i * 6 + 1] = HC(1, 0);
            L->snlist[i * 6 + 2] = HC(0, -1);
            L->snlist[i * 6 + 3] = HC(-1, -1);
            L->snlist[i * 6 + 4] = HC(-1, 0);
            L->snlist[i * 6 + 5] = HC(0, 1);
        }
#undef HC
    }
    /* plaquettes: A (i1+i2 mod 3 == 2), B (else), C (== 0) */
    L->plq_cord = malloc(sizeof(int) * 6 * L->ncell);
    int nd[3] = {0, 0, 0};
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int r = (i1 + i2) % 3;
            nd[r == 2 ? 0 : (r == 0 ? 2 : 1)]++;
        }
    int id[3] = {0, 0, 0};
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2) {
            int r = (i1 + i2) % 3;
            int t = r == 2 ? 0 : (r == 0 ? 2 : 1);
            int off = 0;
            for (int q = 0; q < t; ++q) off += nd[q];
            int pid = ++id[t] + off - 1;
#define INV(a, b, o) ((((b) + ((a) - 1) * l2) - 1) * 2 + (o))
            L->plq_cord[pid * 6 + 0] = INV(i1, i2, 2);
            L->plq_cord[pid * 6 + 1] = INV(i1, i2, 1);
            L->plq_cord[pid * 6 + 2] = INV(i1, npbc(i2 - 1, l2), 2);
            L->plq_cord[pid * 6 + 3] = INV(npbc(i1 - 1, l1), npbc(i2 - 1, l2), 1);
            L->plq_cord[pid * 6 + 4] = INV(npbc(i1 - 1, l1), npbc(i2 - 1, l2), 2);
            L->plq_cord[pid * 6 + 5] = INV(npbc(i1 - 1, l1), i2, 1);
#undef INV
        }
}

/* setup_chain_sub: l1 sites, one orbital, bond families +a1 and -a1 from the
 * A sites (even, 1-based), second neighbours at +-2 a1.  The distance table
 * imj(i, j) = npbc(i - j, l1) and zexpiqr are the 2D ones with l2 = 1. */
static void setup_chain(orc_latt *L, int l1) {
    const double a1[2] = {1.0, 0.0}, a2[2] = {0.0, 1.0};
    setup_2d(L, l1, 1, a1, a2);
    L->kind = ORC_CHAIN; L->nsub = 1; L->nsites = l1; L->z_plq = 1;
    L->nn_nf = 2; L->nn_lf = l1 / 2; L->nsn = 2;
    int ns = L->nsites;
    L->cord = malloc(sizeof(int) * 2 * ns);
    L->rcord = malloc(sizeof(double) * 2 * ns);
    L->nnlf_list = malloc(sizeof(int) * (L->nn_lf > 0 ? L->nn_lf : 1));
    L->list = malloc(sizeof(int) * 2 * ns);
    int ind = 0;
    for (int i1 = 1; i1 <= l1; ++i1) {
        L->list[(i1 - 1) * 2] = i1; L->list[(i1 - 1) * 2 + 1] = 1;
        L->rcord[(i1 - 1) * 2] = i1; L->rcord[(i1 - 1) * 2 + 1] = 1;
        if (i1 % 2 == 0 && ind < L->nn_lf) L->nnlf_list[ind++] = i1;
    }
    memcpy(L->cord, L->ulist, sizeof(int) * 2 * ns);
    L->nnvecr = malloc(sizeof(double) * ns * 2 * 2);
    L->nnveci = malloc(sizeof(int) * ns * 2 * 2);
    for (int i = 0; i < ns; ++i)
        for (int nf = 0; nf < 2; ++nf) {
            L->nnvecr[(i * 2 + nf) * 2] = nf == 0 ? 1.0 : -1.0; L->nnvecr[(i * 2 + nf) * 2 + 1] = 0.0;
            L->nnveci[(i * 2 + nf) * 2] = nf == 0 ? 1 : -1; L->nnveci[(i * 2 + nf) * 2 + 1] = 0;
        }
    L->nnlist = malloc(sizeof(int) * ns * 2);
    L->snlist = malloc(sizeof(int) * ns * 2);
    for (int i = 0; i < ns; ++i) {
        int u1 = L->ulist[i * 2];
        L->nnlist[i * 2 + 0] = npbc(u1 + 1, l1);
        L->nnlist[i * 2 + 1] = npbc(u1 - 1, l1);
        L->snlist[i * 2 + 0] = npbc(u1 + 2, l1);
        L->snlist[i * 2 + 1] = npbc(u1 - 2, l1);
    }
    L->plq_cord = malloc(sizeof(int) * ns);
    for (int i = 0; i < ns; ++i) L->plq_cord[i] = i + 1;
}

/* setup_latt3d_sub + setup_cubic_sub.  Cell (= site) index
 * (i3-1) l1 l2 + (i1-1) l2 + i2; listk with l (a3) outermost, then m (a1),
 * then n (a2); zexpiqr(nk, i) = exp(i k.R_i) with k = 2 pi (m/l1, n/l2, l/l3);
 * nnlist directions +a3, +a1, +a2, -a3, -a1, -a2; nnlf_list the sites with
 * i1 + i2 + i3 even in loop order (i1 outer, i3 inner); twelve second
 * neighbours; plq_cord the eight corners of the cube at each cell, the cells
 * grouped by the parities of (i1, i2, i3). */
static void setup_cubic(orc_latt *L, int l1, int l2, int l3) {
    L->kind = ORC_CUBIC; L->l1 = l1; L->l2 = l2; L->l3 = l3;
    const int nc = l1 * l2 * l3;
    L->ncell = nc; L->nsub = 1; L->nsites = nc; L->z_plq = 8; L->nn_nf = 6; L->nn_lf = nc / 2; L->nsn = 12;
#define CELL(a, b, c) ((npbc((c), l3) - 1) * l1 * l2 + (npbc((a), l1) - 1) * l2 + npbc((b), l2))
    L->ulist3 = malloc(sizeof(int) * 3 * nc);
    L->list = malloc(sizeof(int) * 2 * nc);
    L->nnlf_list = malloc(sizeof(int) * (L->nn_lf > 0 ? L->nn_lf : 1));
    int ind = 0;
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) {
                const int c = CELL(i1, i2, i3) - 1;
                L->ulist3[c * 3] = i1; L->ulist3[c * 3 + 1] = i2; L->ulist3[c * 3 + 2] = i3;
                L->list[c * 2] = c + 1; L->list[c * 2 + 1] = 1;
                if ((i1 + i2 + i3) % 2 == 0 && ind < L->nn_lf) L->nnlf_list[ind++] = c + 1;
            }
    L->listk = malloc(sizeof(int) * 3 * nc);
    int k = 0;
    for (int l = -(l3 + 1) / 2 + 1; l <= l3 / 2; ++l)
        for (int mm = -(l1 + 1) / 2 + 1; mm <= l1 / 2; ++mm)
            for (int n = -(l2 + 1) / 2 + 1; n <= l2 / 2; ++n) {
                L->listk[k * 3] = mm; L->listk[k * 3 + 1] = n; L->listk[k * 3 + 2] = l; ++k;
            }
    L->imj = malloc(sizeof(int) * nc * nc);
    for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nc; ++i) {
            int nx = npbc(L->ulist3[i * 3] - L->ulist3[j * 3], l1);
            int ny = npbc(L->ulist3[i * 3 + 1] - L->ulist3[j * 3 + 1], l2);
            int nz = npbc(L->ulist3[i * 3 + 2] - L->ulist3[j * 3 + 2], l3);
            L->imj[i * nc + j] = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2;
        }
    L->zexpiqr = malloc(sizeof(zc) * nc * nc);
    for (int i = 0; i < nc; ++i)
        for (int nk = 0; nk < nc; ++nk) {
            double ph = 2.0 * M_PI * ((double)L->listk[nk * 3] * L->ulist3[i * 3] / l1 +
                                      (double)L->listk[nk * 3 + 1] * L->ulist3[i * 3 + 1] / l2 +
                                      (double)L->listk[nk * 3 + 2] * L->ulist3[i * 3 + 2] / l3);
            L->zexpiqr[i * nc + nk] = cexp(I * ph);
        }
    static const int dnn[6][3] = {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, -1}, {-1, 0, 0}, {0, -1, 0}};
    static const int dsn[12][3] = {{1, 1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {0, 1, 1}, {0, 1, -1},
                                   {0, -1, -1}, {0, -1, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}, {-1, 0, 1}};
    L->nnlist = malloc(sizeof(int) * nc * 6);
    L->snlist = malloc(sizeof(int) * nc * 12);
    for (int i = 0; i < nc; ++i) {
        const int u1 = L->ulist3[i * 3], u2 = L->ulist3[i * 3 + 1], u3 = L->ulist3[i * 3 + 2];
        for (int f = 0; f < 6; ++f) L->nnlist[i * 6 + f] = CELL(u1 + dnn[f][0], u2 + dnn[f][1], u3 + dnn[f][2]);
        for (int f = 0; f < 12; ++f) L->snlist[i * 12 + f] = CELL(u1 + dsn[f][0], u2 + dsn[f][1], u3 + dsn[f][2]);
    }
    /* the bonds of expar3d carry no phase: zero vectors */
    L->nnveci = calloc((size_t)nc * 6 * 2, sizeof(int));
    L->nnvecr = calloc((size_t)nc * 6 * 2, sizeof(double));
    L->cord = malloc(sizeof(int) * 2 * nc);
    L->rcord = malloc(sizeof(double) * 2 * nc);
    for (int i = 0; i < nc; ++i) {
        L->cord[i * 2] = L->ulist3[i * 3]; L->cord[i * 2 + 1] = L->ulist3[i * 3 + 1];
        L->rcord[i * 2] = L->ulist3[i * 3]; L->rcord[i * 2 + 1] = L->ulist3[i * 3 + 1];
    }
    int nd[8] = {0}, id[8] = {0};
#define PTYPE(a, b, c) (((a) % 2 == 0) * 4 + ((b) % 2 == 0) * 2 + ((c) % 2 == 0))
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) nd[PTYPE(i1, i2, i3)]++;
    L->plq_cord = malloc(sizeof(int) * 8 * nc);
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) {
                const int t = PTYPE(i1, i2, i3);
                int q = id[t]++;
                for (int u = 0; u < t; ++u) q += nd[u];
                int *pc = &L->plq_cord[q * 8];
                pc[0] = CELL(i1, i2, i3);         pc[1] = CELL(i1 + 1, i2, i3);
                pc[2] = CELL(i1 + 1, i2 + 1, i3); pc[3] = CELL(i1, i2 + 1, i3);
                pc[4] = CELL(i1, i2, i3 + 1);     pc[5] = CELL(i1 + 1, i2, i3 + 1);
                pc[6] = CELL(i1 + 1, i2 + 1, i3 + 1); pc[7] = CELL(i1, i2 + 1, i3 + 1);
            }
#undef PTYPE
#undef CELL
}

/* setup_latt3d_sub + setup_r_cubic_sub (src/lattice.f90:1486-1605): six
 * sites per cell, (cell-1)*6 + isub with the cells in the order i3, i1, i2;
 * nnlf_list(i) = 2i - 1 for i = 1..3 lq; nnlist as the reference writes it per
 * residue of the site index mod 6; snlist and plq_cord zero. */
static void setup_r_cubic(orc_latt *L, int l1, int l2, int l3) {
    L->kind = ORC_R_CUBIC; L->l1 = l1; L->l2 = l2; L->l3 = l3;
    const int nc = l1 * l2 * l3, ns = 6 * nc;
    L->ncell = nc; L->nsub = 6; L->nsites = ns; L->z_plq = 8; L->nn_nf = 4; L->nn_lf = 3 * nc; L->nsn = 12;
#define CELL(a, b, c) ((npbc((c), l3) - 1) * l1 * l2 + (npbc((a), l1) - 1) * l2 + npbc((b), l2))
    L->ulist3 = malloc(sizeof(int) * 3 * nc);
    L->list = malloc(sizeof(int) * 2 * ns);
    int *cd = malloc(sizeof(int) * 3 * ns);
    int ind = 0;
    for (int i3 = 1; i3 <= l3; ++i3)
        for (int i1 = 1; i1 <= l1; ++i1)
            for (int i2 = 1; i2 <= l2; ++i2) {
                const int c = CELL(i1, i2, i3);
                L->ulist3[(c - 1) * 3] = i1; L->ulist3[(c - 1) * 3 + 1] = i2; L->ulist3[(c - 1) * 3 + 2] = i3;
                for (int isub = 1; isub <= 6; ++isub) {
                    L->list[ind * 2] = c; L->list[ind * 2 + 1] = isub;
                    cd[ind * 3] = i1; cd[ind * 3 + 1] = i2; cd[ind * 3 + 2] = i3;
                    ++ind;
                }
            }
    L->nnlf_list = malloc(sizeof(int) * L->nn_lf);
    for (int i = 1; i <= L->nn_lf; ++i) L->nnlf_list[i - 1] = 2 * i - 1;
    L->listk = malloc(sizeof(int) * 3 * nc);
    int k = 0;
    for (int l = -(l3 + 1) / 2 + 1; l <= l3 / 2; ++l)
        for (int mm = -(l1 + 1) / 2 + 1; mm <= l1 / 2; ++mm)
            for (int n = -(l2 + 1) / 2 + 1; n <= l2 / 2; ++n) {
                L->listk[k * 3] = mm; L->listk[k * 3 + 1] = n; L->listk[k * 3 + 2] = l; ++k;
            }
    L->imj = malloc(sizeof(int) * nc * nc);
    for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nc; ++i) {
            int nx = npbc(L->ulist3[i * 3] - L->ulist3[j * 3], l1);
            int ny = npbc(L->ulist3[i * 3 + 1] - L->ulist3[j * 3 + 1], l2);
            int nz = npbc(L->ulist3[i * 3 + 2] - L->ulist3[j * 3 + 2], l3);
            L->imj[i * nc + j] = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2;
        }
    L->zexpiqr = malloc(sizeof(zc) * nc * nc);
    for (int i = 0; i < nc; ++i)
        for (int nk = 0; nk < nc; ++nk) {
            double ph = 2.0 * M_PI * ((double)L->listk[nk * 3] * L->ulist3[i * 3] / l1 +
                                      (double)L->listk[nk * 3 + 1] * L->ulist3[i * 3 + 1] / l2 +
                                      (double)L->listk[nk * 3 + 2] * L->ulist3[i * 3 + 2] / l3);
            L->zexpiqr[i * nc + nk] = cexp(I * ph);
        }
    L->nnlist = malloc(sizeof(int) * ns * 4);
    for (int i = 1; i <= ns; ++i) {
        const int c1 = cd[(i - 1) * 3], c2 = cd[(i - 1) * 3 + 1], c3 = cd[(i - 1) * 3 + 2], r = i % 6;
        int *nl = &L->nnlist[(i - 1) * 4];
        if (r == 3 || r == 5) {           /* A2, A3 */
            nl[0] = i + 1;
            nl[1] = (CELL(c1 - 1, c2, c3) - 1) * 6 + r + 1;
            nl[2] = (CELL(c1, c2 - 1, c3) - 1) * 6 + r + 1;
            nl[3] = i - 1;
        } else if (r == 1) {              /* A1 */
            nl[0] = i + 1;
            nl[1] = (CELL(c1 - 1, c2, c3) - 1) * 6 + r + 1;
            nl[2] = (CELL(c1, c2 - 1, c3) - 1) * 6 + r + 1;
            nl[3] = (CELL(c1 - 1, c2 - 1, c3 - 1) - 1) * 6 + r + 1;
        } else if (r == 2 || r == 4) {    /* B1, B2 */
            nl[0] = i - 1;
            nl[1] = (CELL(c1 + 1, c2, c3) - 1) * 6 + r - 1;
            nl[2] = (CELL(c1, c2 + 1, c3) - 1) * 6 + r - 1;
            nl[3] = i + 1;
        } else {                           /* B3 */
            nl[0] = i - 1;
            nl[1] = (CELL(c1 + 1, c2, c3) - 1) * 6 + 5;
            nl[2] = (CELL(c1, c2 + 1, c3) - 1) * 6 + 5;
            nl[3] = (CELL(c1 + 1, c2 + 1, c3 + 1) - 1) * 6 + 1;
        }
    }
    L->snlist = calloc((size_t)ns * 12, sizeof(int));
    L->plq_cord = calloc((size_t)nc * 8, sizeof(int));
    L->nnveci = calloc((size_t)ns * 4 * 2, sizeof(int));
    L->nnvecr = calloc((size_t)ns * 4 * 2, sizeof(double));
    L->cord = malloc(sizeof(int) * 2 * ns);
    L->rcord = malloc(sizeof(double) * 2 * ns);
    for (int i = 0; i < ns; ++i) {
        L->cord[i * 2] = cd[i * 3]; L->cord[i * 2 + 1] = cd[i * 3 + 1];
        L->rcord[i * 2] = cd[i * 3]; L->rcord[i * 2 + 1] = cd[i * 3 + 1];
    }
    free(cd);
#undef CELL
}

int orc_latt_build(orc_latt *L, int kind, int l1, int l2, int l3) {
    memset(L, 0, sizeof(*L));
    if (kind == ORC_SQUARE) setup_square(L, l1, l2);
    else if (kind == ORC_HONEYCOMB) setup_honeycomb(L, l1, l2);
    else if (kind == ORC_CHAIN) setup_chain(L, l1);
    else if (kind == ORC_CUBIC) setup_cubic(L, l1, l2, l3);
    else if (kind == ORC_R_CUBIC) setup_r_cubic(L, l1, l2, l3);
    else return -1;
    return 0;
}

/* expar.f90: Landau-gauge Peierls phase for bond (i, nf), twist flux and
 * dimerisation.  i is 0-based, nf is 1-based as in the reference. */
zc orc_expar(const orc_latt *L, int i, int nf, double xmag, double fx, double fy, double dimer) {
    if (L->kind == ORC_CUBIC || L->kind == ORC_R_CUBIC) return 1.0;      /* expar3d.f90 */
    int k = (i * L->nn_nf + (nf - 1)) * 2;
    int nax = L->nnveci[k], nay = L->nnveci[k + 1];
    double vr1 = L->nnvecr[k], vr2 = L->nnvecr[k + 1];
    double rc1 = L->rcord[i * 2], rc2 = L->rcord[i * 2 + 1];
    int c1 = L->cord[i * 2], c2 = L->cord[i * 2 + 1];
    /* the chain has no Peierls phase (expar1d.f90: x = x1 = 0) */
    double xmag1 = (L->kind == ORC_CHAIN) ? 0.0 : xmag / L->ncell * (L->a1[0] * L->a2[1] - L->a1[1] * L->a2[0]);
    double x = -xmag1 * vr1 * (2.0 * rc2 + vr2) * M_PI;
    double x1 = 0.0;
    int edge2 = ((c2 == L->l2 && nay > 0) || (c2 == 1 && nay < 0));
    int edge1 = ((c1 == L->l1 && nax > 0) || (c1 == 1 && nax < 0));
    double proj = (rc2 + vr2) * L->a2[0] + (rc1 + vr1) * L->a1[0];
    int sx = nax > 0 ? 1 : -1, sy = nay > 0 ? 1 : -1;
    if (edge2 && nax == 0) {
        x1 = 2.0 * M_PI * xmag1 * (double)(sy * L->l2) * L->a2[1] * proj;
    } else if (edge1 && nay == 0) {
        x1 = 2.0 * M_PI * xmag1 * (double)(sx * L->l1) * L->a1[1] * proj;
    } else if (edge1 && edge2) {
        x1 = 2.0 * M_PI * xmag1 * ((double)(sx * L->l1) * L->a1[1] + (double)(sy * L->l2) * L->a2[1]) * proj;
    }
    zc e = cexp(I * (x + x1));
    double av0 = fx * L->a1[0] / L->l1 + fy * L->a2[0] / L->l2;
    double av1 = fx * L->a1[1] / L->l1 + fy * L->a2[1] / L->l2;
    double rv0 = nax * L->a1[0] + nay * L->a2[0];
    double rv1 = nax * L->a1[1] + nay * L->a2[1];
    e *= cexp(I * 2.0 * M_PI * (av0 * rv0 + av1 * rv1));
    if (nf == 1) e *= (1.0 + dimer);
    return e;
}
