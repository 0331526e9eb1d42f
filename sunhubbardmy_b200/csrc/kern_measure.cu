// Equal-time measurement of one time slice.
//
// Reference: src/dqmc_measure/equaltime_measure.f90 (equaltime_measure 1-69,
// zkint, zint_u, zint_v, zqsq, ztsq, ztq, measure_cpcm/spsm/nn/jj/bondcorr/
// paircorr) and, for the chain, equaltime_measure1d.f90 (the same bins with
// one cell row; energy_bin 3 scaled by nflr rt, energy_bin 5 = zint_v).
// Observables use Gc(i,j) = delta_ij - G(j,i) and are weighted with
// zphi = sgn/Re(phase) * phase.  G^T is written first (a tiled transpose), so
// that every correlation term reads a column of G or of G^T.  Per chain, one
// CTA sums the single-number energy terms, and CTAs of site bins (cpcm, spsm,
// nn, pair_onsite) and of bond bins (jj, bb, pair_nn, pair_sn) follow.  Two
// threads own a bin (distance d, orbitals a, b); they walk the even and the
// odd unit cells j in order, pairing j with cell i = j + d (imj(i, j) = d, in
// closed form), and their sums are added in a fixed order, so no atomics are
// needed and the result does not depend on scheduling.  Threads of
// consecutive d read consecutive rows of the same columns (coalesced).
//
// Bin layout per chain (complex): energy[10], cpcm, spsm, nn, pair_onsite
// [lq*4 each, index (d) + lq*(no_i + 2 no_j)], jj, bb, pair_nn, pair_sn [lq
// each], zn[2], zj, zb.
#include "chain_access.cuh"
#include "kernels.h"

#define MEAS_NT 256
#define MEAS_SPLIT 2                       // threads per bin
#define MEAS_BH (MEAS_NT / MEAS_SPLIT)    // bins per CTA

DQ_DEV double2 gcf(const double2* G, int N, int i, int j) {   // Gc(i,j)
    double2 g = G[MIDX(j, i, N)];
    return cmk((i == j ? 1.0 : 0.0) - g.x, -g.y);
}
DQ_DEV double2 gf(const double2* G, int N, int i, int j) { return G[MIDX(i, j, N)]; }
DQ_DEV double2 rfma(double a, double2 b, double2 c) { return cmk(fma(a, b.x, c.x), fma(a, b.y, c.y)); }   // a b + c, a real

// cell i = j + d of the distance table imj(i, j) = d (setup_latt2d_sub): with
// cells c = c1 l2 + c2 and d = dy + l2 dx, i1 = (j1 + dx + 1) mod l1 and
// i2 = (j2 + dy + 1) mod l2; dxp = dx + 1, dyp = dy + 1
DQ_DEV int cell_shift(int cj, int dxp, int dyp, int l1, int l2) {
    int i1 = cj / l2 + dxp, i2 = cj % l2 + dyp;
    if (i1 >= l1) i1 -= l1;
    if (i2 >= l2) i2 -= l2;
    return i1 * l2 + i2;
}
// The same for the cubic lattice (setup_latt3d_sub): cells c = (c3 l1 + c1) l2
// + c2 and d = dz l1 l2 + dx l2 + dy; dzp = dz + 1.  With l3 = 1 (dzp = 1) it
// is the 2D shift.
DQ_DEV int cell_shift3(int cj, int dxp, int dyp, int dzp, int l1, int l2, int l3) {
    const int l12 = l1 * l2;
    int i3 = cj / l12 + dzp, i1 = (cj / l2) % l1 + dxp, i2 = cj % l2 + dyp;
    if (i3 >= l3) i3 -= l3;
    if (i1 >= l1) i1 -= l1;
    if (i2 >= l2) i2 -= l2;
    return (i3 * l1 + i1) * l2 + i2;
}
// cell i = j + d on either lattice kind (D3: cubic)
template <bool D3>
struct CellShift {
    int dxp, dyp, dzp, l1, l2, l3;
    DQ_DEV CellShift(int d, const ModelDev& md) : l1(md.l1), l2(md.l2), l3(md.l3) {
        dxp = (D3 ? (d / l2) % l1 : d / l2) + 1;
        dyp = d % l2 + 1;
        dzp = D3 ? d / (l1 * l2) + 1 : 1;
    }
    DQ_DEV int operator()(int cj) const {
        return D3 ? cell_shift3(cj, dxp, dyp, dzp, l1, l2, l3) : cell_shift(cj, dxp, dyp, l1, l2);
    }
};

// The cells cj = c0, c0 + st, c0 + 2 st, ... with their shifts ci = shift(cj),
// walked with carries instead of a division per cell: the coordinates of cj
// advance with carry (j2, then j1, then j3), and each coordinate of ci is the
// matching one of cj plus the shift, less the length once (the shift is at
// most the length).
template <bool D3>
struct CellWalk {
    int j1, j2, j3, l1, l2, l3, dxp, dyp, dzp;
    DQ_DEV CellWalk(const CellShift<D3>& s, int c0)
        : l1(s.l1), l2(s.l2), l3(s.l3), dxp(s.dxp), dyp(s.dyp), dzp(s.dzp) {
        j2 = c0 % l2;
        j1 = D3 ? (c0 / l2) % l1 : c0 / l2;
        j3 = D3 ? c0 / (l1 * l2) : 0;
    }
    DQ_DEV int ci() const {
        int i1 = j1 + dxp, i2 = j2 + dyp;
        if (i1 >= l1) i1 -= l1;
        if (i2 >= l2) i2 -= l2;
        if (!D3) return i1 * l2 + i2;
        int i3 = j3 + dzp;
        if (i3 >= l3) i3 -= l3;
        return (i3 * l1 + i1) * l2 + i2;
    }
    DQ_DEV void step(int st) {
        j2 += st;
        while (j2 >= l2) {
            j2 -= l2;
            if (++j1 == l1) { j1 = 0; if (D3) ++j3; }
        }
    }
};

// Energy terms and the background sums zn, zj, zb (single numbers per chain),
// computed by the chain's second CTA while the first one sums the bins.
DQ_DEV void meas_energy(const ChainDev& c, double2 zphi, double sgn) {
    __shared__ double red[64];
    const ModelDev& md = *c.md;
    const int N = c.N, lq = md.lq, tid = threadIdx.x, nth = blockDim.x;
    const int nnf = md.nn_nf, zp = md.z_plq, nflr = md.nflr;
    const double2* G = c.G;
    double2* bins = c.bins;
    const bool hc = (md.nsub == 2);
    // ---- energy terms ----
    double2 zne = cmk(0, 0), zu = cmk(0, 0), zk = cmk(0, 0), zv = cmk(0, 0);
    // the chain's kinetic energy (equaltime_measure1d.f90) carries nflr rt on the
    // bonds and 2 t2 on its two second neighbours
    const bool chain = md.chain != 0, cubic = md.cubic != 0;
    const double kb = chain ? -2.0 * nflr * md.rt : -2.0, k2 = chain ? -2.0 * md.t2 : -md.t2;
    for (int i = tid; i < N; i += nth) {
        double2 d = gcf(G, N, i, i);
        zne = cadd(zne, d);
        zu = cadd(zu, cmul(d, d));
        if (md.t2 != 0.0 && !cubic) {      // zkint of equaltime_measure3d.f90 has no t2 term
            int ns = chain ? 2 : hc ? 6 : 4;
            for (int f = 0; f < ns; ++f) zk.x += k2 * gcf(G, N, i, md.snlist[i * md.nsn + f]).x;
        }
    }
    for (int b = tid; b < md.nn_lf * nnf; b += nth) {
        int i1 = md.bond_i1[b], i2 = md.bond_i2[b], nf = b / md.nn_lf;
        double2 g = gcf(G, N, i1, i2);
        zk.x += kb * cmul(g, md.expar_nn[i1 * nnf + nf]).x;
        zv.x += g.x;
    }
    // plaquette terms
    double2 zq = cmk(0, 0), zt = cmk(0, 0), ztq = cmk(0, 0);
    const double2 em = cexpi(-md.theta), ep = cexpi(md.theta);
    for (int q = tid; q < (chain || cubic ? 0 : lq); q += nth) {      // plaquette terms: 2D only
        const int* pc = md.plq_cord + q * zp;
        double2 tmp = cmk(0, 0);
        for (int a = 0; a < zp; ++a) tmp = cadd(tmp, gcf(G, N, pc[a], pc[a]));
        zq = cadd(zq, cscale(cmul(tmp, tmp), (double)nflr));
        for (int a = 0; a < zp; ++a)
            for (int b = 0; b < zp; ++b) zq = cfma(gcf(G, N, pc[a], pc[b]), gf(G, N, pc[a], pc[b]), zq);
        double tt = 0.0, t1 = 0.0;
        double2 t2 = cmk(0, 0);
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1], i1a = pc[(a % zp)];
            double2 z1 = (a % 2 == 0) ? cmk(-ep.x, -ep.y) : em;
            double v = 2.0 * cmul(z1, gcf(G, N, i1, i1a)).x;
            tt += v; t1 += v;
            t2 = cadd(t2, cscale(gcf(G, N, i1, i1), 1.0 / 3.0));
        }
        zt.x += tt * tt * nflr;
        ztq = cadd(ztq, cscale(t2, t1 * nflr));
        for (int a = 1; a <= zp; ++a) {
            int i1 = pc[a - 1], i1a = pc[(a % zp)];
            double2 z1 = (a % 2 == 0) ? cmk(-ep.x, -ep.y) : em, z2 = cconj(z1);
            double2 y1 = cscale(z1, 1.0 / 3.0), y2 = cconj(y1);
            for (int b = 1; b <= zp; ++b) {
                int i2 = pc[b - 1], i2a = pc[(b % zp)];
                double2 z3 = (b % 2 == 0) ? cmk(-ep.x, -ep.y) : em, z4 = cconj(z3);
                zt = cadd(zt, cmul(cmul(z1, z3), cmul(gcf(G, N, i1, i2a), gf(G, N, i1a, i2))));
                zt = cadd(zt, cmul(cmul(z1, z4), cmul(gcf(G, N, i1, i2), gf(G, N, i1a, i2a))));
                zt = cadd(zt, cmul(cmul(z2, z3), cmul(gcf(G, N, i1a, i2a), gf(G, N, i1, i2))));
                zt = cadd(zt, cmul(cmul(z2, z4), cmul(gcf(G, N, i1a, i2), gf(G, N, i1, i2a))));
                ztq = cadd(ztq, cmul(y1, cmul(gcf(G, N, i1, i2), gf(G, N, i1a, i2))));
                ztq = cadd(ztq, cmul(y2, cmul(gcf(G, N, i1a, i2), gf(G, N, i1, i2))));
            }
        }
    }
    zne = block_csum(zne, red);
    zu = block_csum(zu, red);
    zk = block_csum(zk, red);
    zv = block_csum(zv, red);
    zq = block_csum(zq, red);
    zt = block_csum(zt, red);
    ztq = block_csum(ztq, red);
    // background terms zn, zj, zb
    double2 zn0 = cmk(0, 0), zn1 = cmk(0, 0), zj = cmk(0, 0), zb = cmk(0, 0);
    for (int j = tid; j < N; j += nth) {
        double2 d = gcf(G, N, j, j);
        if (hc && (j & 1)) zn1 = cadd(zn1, d); else zn0 = cadd(zn0, d);
    }
    for (int cj = tid; cj < lq; cj += nth) {
        int j0 = hc ? 2 * cj : cj;
        int jnj = hc ? md.snlist[j0 * md.nsn] : md.nnlist[j0 * nnf];
        int jnb = md.nnlist[j0 * nnf];
        double2 e = md.expar_nn[j0 * nnf];
        double2 dj = csub(gcf(G, N, j0, jnj), gcf(G, N, jnj, j0));
        if (!cubic) zj = cadd(zj, cmk(-dj.y, dj.x));
        zb = cadd(zb, cadd(cmul(e, gcf(G, N, j0, jnb)), cmul(cconj(e), gcf(G, N, jnb, j0))));
    }
    zn0 = block_csum(zn0, red);
    zn1 = block_csum(zn1, red);
    zj = block_csum(zj, red);
    zb = block_csum(zb, red);
    if (tid == 0) {
        bins[0] = cadd(bins[0], cmk(sgn, 0));
        bins[1] = cadd(bins[1], cscale(cmul(zne, zphi), 1.0 / lq));
        bins[2] = cadd(bins[2], cmul(zk, zphi));
        bins[3] = cadd(bins[3], cmul(zu, zphi));
        if (chain) {
            bins[4] = cadd(bins[4], cmul(zv, zphi));     // energy_bin(5) of the chain, without rv
        } else if (!cubic) {                             // the cubic lattice fills energy_bin(1:4) only
            bins[4] = cadd(bins[4], cscale(cmul(zq, zphi), 1.0 / 9.0));
            bins[5] = cadd(bins[5], cmul(zt, zphi));
            bins[6] = cadd(bins[6], cmul(ztq, zphi));
            bins[7] = cadd(bins[7], cscale(cmul(zv, zphi), md.rv));
        }
        size_t tail = 10 + 20 * (size_t)lq;
        bins[tail + 0] = cadd(bins[tail + 0], cmul(zn0, zphi));
        bins[tail + 1] = cadd(bins[tail + 1], cmul(zn1, zphi));
        bins[tail + 2] = cadd(bins[tail + 2], cmul(zj, zphi));
        bins[tail + 3] = cadd(bins[tail + 3], cmul(zb, zphi));
        c.stats[ST_NOBS] += 1.0;
    }
}

// The cells of a bin are split by residue mod MEAS_SPLIT between threads
// t + k MEAS_BH of the CTA; the partial sums are added to thread t's in the
// order k = 1, 2, ..., so the result does not depend on scheduling.
DQ_DEV void meas_combine(double2& a0, double2& a1, double2& a2, double2& a3, int h) {
    __shared__ double2 part[4][MEAS_BH];
    const int t = threadIdx.x % MEAS_BH;
#pragma unroll
    for (int k = 1; k < MEAS_SPLIT; ++k) {
        if (h == k) { part[0][t] = a0; part[1][t] = a1; part[2][t] = a2; part[3][t] = a3; }
        __syncthreads();
        if (h == 0) { a0 = cadd(a0, part[0][t]); a1 = cadd(a1, part[1][t]); a2 = cadd(a2, part[2][t]); a3 = cadd(a3, part[3][t]); }
        __syncthreads();
    }
}

// Site-correlation bins (cpcm, spsm, nn, pair_onsite): MEAS_SPLIT threads per
// bin (distance d, orbitals a, b) walk interleaved cells j in order.  Accumulates
// S1 = sum GTc, B = sum GTc G, A = sum gcd_i gcd_j, S4 = sum G G with
// GTc(i, j) = GT(i, j) - delta_ij = -Gc(i, j); whether site i of cell j + d
// is site j is the same for every cell j (a translation), so it is taken
// from cell 0.
template <bool HC, bool D3, bool RC>
DQ_DEV void meas_site(const ChainDev& c, int bin, double2 zphi) {   // bin of thread t % MEAS_BH
    constexpr int NS = HC ? 2 : 1;        // orbital pairs binned separately
    constexpr int NO = RC ? 6 : 1;        // orbitals summed into one bin (r_cubic)
    __shared__ double2 gcd[512];     // Gc(i,i)
    const ModelDev& md = *c.md;
    const int N = c.N, lq = md.lq, nflr = md.nflr;
    const double2 *G = c.G, *GT = c.GT;
    for (int i = threadIdx.x; i < N; i += MEAS_NT) gcd[i] = gcf(G, N, i, i);
    __syncthreads();
    const bool valid = bin < lq * NS * NS;
    const int h = threadIdx.x / MEAS_BH;      // cells j = h (mod MEAS_SPLIT)
    if (!valid) bin = 0;
    const double fsp = 1.0 - 1.0 / (double)(nflr * nflr), fn = 1.0 / (double)nflr;
    const int d = bin % lq, ab = bin / lq, a = ab % NS, b = ab / NS;
    const CellShift<D3> shift(d, md);
    const double fd = (shift(0) == 0 && a == b) ? 1.0 : 0.0;
    double2 s1 = cmk(0, 0), sB = cmk(0, 0), sA = cmk(0, 0), s4 = cmk(0, 0);
    if (NO == 1) {
        CellWalk<D3> w(shift, h);
#pragma unroll 4
        for (int cj = valid ? h : lq; cj < lq; cj += MEAS_SPLIT, w.step(MEAS_SPLIT)) {
            const int i = w.ci() * NS + a, j = cj * NS + b;
            const size_t o = (size_t)i + (size_t)N * j;
            double2 gtc = GT[o];
            const double2 g = G[o];
            gtc.x -= fd;
            s1 = cadd(s1, gtc);
            sB = cfma(gtc, g, sB);
            sA = cfma(gcd[i], gcd[j], sA);
            s4 = cfma(g, g, s4);
        }
    } else {
        // every orbital pair (oa, ob) of the cell pair (j + d, j); i == j only
        // for d = 0 and oa == ob
        const bool d0 = shift(0) == 0;
        CellWalk<D3> w(shift, h);
        for (int cj = valid ? h : lq; cj < lq; cj += MEAS_SPLIT, w.step(MEAS_SPLIT)) {
            const int ci = w.ci();
            for (int ob = 0; ob < NO; ++ob) {
                const int j = cj * NO + ob;
#pragma unroll
                for (int oa = 0; oa < NO; ++oa) {
                    const int i = ci * NO + oa;
                    const size_t o = (size_t)i + (size_t)N * j;
                    double2 gtc = GT[o];
                    const double2 g = G[o];
                    if (d0 && oa == ob) gtc.x -= 1.0;
                    s1 = cadd(s1, gtc);
                    sB = cfma(gtc, g, sB);
                    sA = cfma(gcd[i], gcd[j], sA);
                }
            }
        }
    }
    meas_combine(s1, sB, sA, s4, h);
    if (!valid || h) return;
    double2* bins = c.bins;
    double2* cpcm = bins + 10;
    double2* spsm = cpcm + 4 * lq;
    double2* znn = spsm + 4 * lq;
    double2* pons = znn + 4 * lq;
    const int k = d + lq * (a + 2 * b);
    cpcm[k] = cfma(cmk(-s1.x, -s1.y), zphi, cpcm[k]);
    spsm[k] = cfma(cscale(cmk(-sB.x, -sB.y), fsp), zphi, spsm[k]);
    znn[k] = cfma(rfma(-fn, sB, sA), zphi, znn[k]);
    if (!D3) pons[k] = cfma(s4, zphi, pons[k]);     // no pair_onsite on the cubic lattice
}

// Bond-correlation bins (jj, bb, pair_nn, pair_sn): MEAS_SPLIT threads per
// distance d walk interleaved cells j in order, pairing site i0 of cell i = j + d and its
// partners with site j0 and its partners.  The partners are translations
// (current partner pj: nearest neighbour on the square lattice, second
// neighbour on the honeycomb; bond partner pb: nearest neighbour; pair
// partner ps: second neighbour), so on the square lattice the Kronecker
// deltas of Gc = delta - GT depend on d only and are taken from cell 0.
template <bool HC, bool D3, bool RC>
DQ_DEV void meas_bond(const ChainDev& c, int d, double2 zphi) {   // distance of thread t % MEAS_BH
    constexpr int NS = HC ? 2 : 1;
    __shared__ double2 jcell[512];   // Gc(i0,in) - Gc(in,i0), current partner
    __shared__ double2 bcell[512];   // e Gc(i0,ib) + conj(e) Gc(ib,i0), bond partner
    __shared__ double2 pe[512];      // e = expar_nn(i0, first direction)
    __shared__ int pj[512], pb[512], ps[512];
    const ModelDev& md = *c.md;
    const int N = c.N, lq = md.lq, nnf = md.nn_nf;
    const double2 *G = c.G, *GT = c.GT;
    for (int cc = threadIdx.x; cc < lq; cc += MEAS_NT) {
        const int i0 = cc * NS;
        const int inj = HC ? md.snlist[i0 * md.nsn] : md.nnlist[i0 * nnf];
        const int inb = md.nnlist[i0 * nnf];
        const double2 e = md.expar_nn[i0 * nnf];
        pj[cc] = inj; pb[cc] = inb; ps[cc] = D3 ? 0 : md.snlist[i0 * md.nsn]; pe[cc] = e;
        jcell[cc] = csub(gcf(G, N, i0, inj), gcf(G, N, inj, i0));
        bcell[cc] = cadd(cmul(e, gcf(G, N, i0, inb)), cmul(cconj(e), gcf(G, N, inb, i0)));
    }
    __syncthreads();
    const bool valid = d < lq;
    const int h = threadIdx.x / MEAS_BH;      // cells j = h (mod MEAS_SPLIT)
    if (!valid) d = 0;
    const double fn = 1.0 / (double)md.nflr;
    const CellShift<D3> shift(d, md);
    auto gg = [&](int r, int s_) { return G[(size_t)r + (size_t)N * s_]; };
    auto gt = [&](int r, int s_) { return GT[(size_t)r + (size_t)N * s_]; };
    // deltas of the square lattice, from cell 0: [i0 == j0], [in == j0], [i0 == jn], [in == jn]
    double f00 = 0, fn0 = 0, f0n = 0, fnn = 0;
    if (!HC && !RC) {
        const int ci = shift(0), in = pj[ci], jn = pj[0];
        f00 = ci == 0; fn0 = in == 0; f0n = ci == jn; fnn = in == jn;
    }
    double2 sj = cmk(0, 0), sb = cmk(0, 0), sn = cmk(0, 0), ss = cmk(0, 0);
    CellWalk<D3> w(shift, h);
#pragma unroll 4
    for (int cj = valid ? h : lq; cj < lq; cj += MEAS_SPLIT, w.step(MEAS_SPLIT)) {
        const int ci = w.ci();
        const int j0 = cj * NS, i0 = ci * NS, jnj = pj[cj], inj = pj[ci];
        const double2 ei = pe[ci], ej = pe[cj];
        // G and GTc = GT - delta (= -Gc) at rows i0, in of columns j0, jn
        const double2 g00 = gg(i0, j0), an = gg(inj, j0), b0v = gg(i0, jnj), gnn_j = gg(inj, jnj);
        double2 t0 = gt(i0, j0), tn = gt(inj, j0), u0 = gt(i0, jnj), un = gt(inj, jnj);
        if (HC || RC) {
            // the r_cubic bond pairs (site nu, nnlist(nu, 1)) with nu a cell
            // index used as a site index (measure_bondcorr of
            // equaltime_measure3d.f90) are not translates of each other
            t0.x -= i0 == j0; tn.x -= inj == j0; u0.x -= i0 == jnj; un.x -= inj == jnj;
        } else {
            t0.x -= f00; tn.x -= fn0; u0.x -= f0n; un.x -= fnn;
        }
        // connected current-current part (measure_jj), Gc = -GTc:
        // z3 = Gc(i0,jn) G(in,j0) + Gc(in,j0) G(i0,jn) - Gc(i0,j0) G(in,jn) - Gc(in,jn) G(i0,j0)
        const double2 q1 = cmul(u0, an), q2 = cmul(tn, b0v);
        const double2 q3 = cmul(t0, gnn_j), q4 = cmul(un, g00);
        const double2 z3 = csub(cadd(q3, q4), cadd(q1, q2));
        sj = csub(sj, rfma(fn, z3, cmul(jcell[ci], jcell[cj])));
        // bond-bond (measure_bondcorr): x = ei ej Gc(i0,jb) G(ib,j0)
        //   + conj(ei ej) Gc(ib,j0) G(i0,jb) + ei conj(ej) Gc(i0,j0) G(ib,jb)
        //   + conj(ei) ej Gc(ib,jb) G(i0,j0), accumulated here negated
        const double2 ee = cmul(ei, ej), ef = cmul(ei, cconj(ej));
        double2 x, gnn_b;
        if (!HC) {
            // square lattice: the bond partner is the current partner (pb == pj)
            gnn_b = gnn_j;
            x = cmul(ee, q1);
            x = cfma(cconj(ee), q2, x);
            x = cfma(ef, q3, x);
            x = cfma(cconj(ef), q4, x);
        } else {
            const int jnb = pb[cj], inb = pb[ci];
            const bool same = (jnb == jnj && inb == inj);
            gnn_b = same ? gnn_j : gg(inb, jnb);
            double2 tnb = un;                                    // GTc(ib, jb)
            if (!same) { tnb = gt(inb, jnb); tnb.x -= inb == jnb; }
            double2 v1 = gt(i0, jnb), v2 = gt(inb, j0);
            v1.x -= i0 == jnb; v2.x -= inb == j0;
            const double2 r1 = cmul(v1, gg(inb, j0)), r2 = cmul(v2, gg(i0, jnb));
            const double2 r3 = cmul(t0, gnn_b), r4 = cmul(tnb, g00);
            x = cmul(ee, r1);
            x = cfma(cconj(ee), r2, x);
            x = cfma(ef, r3, x);
            x = cfma(cconj(ef), r4, x);
        }
        sb = cadd(sb, rfma(-fn, x, cmul(bcell[cj], bcell[ci])));
        // pair correlations (measure_paircorr; 2D and chain only)
        if (!D3) {
            sn = cfma(g00, gnn_b, sn);
            ss = cfma(g00, gg(ps[ci], ps[cj]), ss);
        }
    }
    meas_combine(sj, sb, sn, ss, h);
    if (!valid || h) return;
    double2* zjj = c.bins + 10 + 16 * (size_t)lq;
    double2* zbb = zjj + lq;
    double2* pnn = zbb + lq;
    double2* psn = pnn + lq;
    zbb[d] = cfma(sb, zphi, zbb[d]);
    if (D3) return;                  // the cubic lattice has bb only (measure_bondcorr of equaltime_measure3d.f90)
    zjj[d] = cfma(sj, zphi, zjj[d]);
    pnn[d] = cfma(sn, zphi, pnn[d]);
    psn[d] = cfma(ss, zphi, psn[d]);
}

// grid (1 + na + nb, chains): x = 0 the energy terms, then na CTAs of site
// bins and nb CTAs of bond bins (sized for the largest lattice of the handle)
template <bool HC, bool D3, bool RC>
__global__ void __launch_bounds__(MEAS_NT, 2) k_measure(const ChainDev* __restrict__ chains, int na) {
    const ChainDev& c = chains[blockIdx.y];
    const double2 phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    const double sgn = phase.x < 0.0 ? -1.0 : 1.0;
    const double2 zphi = cscale(phase, sgn / phase.x);
    const int x = blockIdx.x;
    if (x == 0) meas_energy(c, zphi, sgn);
    else if (x <= na) meas_site<HC, D3, RC>(c, (x - 1) * MEAS_BH + threadIdx.x % MEAS_BH, zphi);
    else meas_bond<HC, D3, RC>(c, (x - 1 - na) * MEAS_BH + threadIdx.x % MEAS_BH, zphi);
}

__global__ void k_bins_clear(const ChainDev* __restrict__ chains, int nbins) {
    const ChainDev c = chains[blockIdx.x];
    (void)nbins;
    const int nb = 10 + 20 * c.md->lq + 4;     // this chain's own bin count
    for (int e = threadIdx.x; e < nb; e += blockDim.x) c.bins[e] = cmk(0, 0);
    if (c.dynbins) {
        const int nd = 4 * c.md->lq * (c.md->ntdm + 1);
        for (int e = threadIdx.x; e < nd; e += blockDim.x) c.dynbins[e] = cmk(0, 0);
    }
    if (threadIdx.x == 0) c.stats[ST_NOBS] = 0.0;
}

// GT = (matrix src_id)^T per chain, 32 x 32 tiles through shared memory (odd pitch)
__global__ void __launch_bounds__(256) k_transpose_g(const ChainDev* __restrict__ chains, int src_id) {
    __shared__ double2 t[32][33];
    const ChainDev& c = chains[blockIdx.z];
    const double2* Src = chain_mat(c, src_id);
    const int N = c.N;
    const int r0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    if (r0 >= N || s0 >= N) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + tx, s_ = s0 + k;
        if (r < N && s_ < N) t[k][tx] = Src[(size_t)r + (size_t)N * s_];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int r = s0 + tx, s_ = r0 + k;       // GT(r, s) = G(s, r)
        if (r < N && s_ < N) c.GT[(size_t)r + (size_t)N * s_] = t[tx][k];
    }
}

// kind: MEAS_ONE_ORBITAL (square, chain), MEAS_HONEYCOMB, MEAS_CUBIC or MEAS_R_CUBIC
void launch_measure(const ChainDev* chains, int nchains, int maxN, int kind, int maxlq, cudaStream_t st) {
    const int nt = (maxN + 31) / 32;
    k_transpose_g<<<dim3(nt, nt, nchains), 256, 0, st>>>(chains, MAT_G);
    const int ns = kind == MEAS_HONEYCOMB ? 2 : 1;
    const int na = (maxlq * ns * ns + MEAS_BH - 1) / MEAS_BH, nb = (maxlq + MEAS_BH - 1) / MEAS_BH;
    const dim3 grid(1 + na + nb, nchains);
    if (kind == MEAS_HONEYCOMB) k_measure<true, false, false><<<grid, MEAS_NT, 0, st>>>(chains, na);
    else if (kind == MEAS_CUBIC) k_measure<false, true, false><<<grid, MEAS_NT, 0, st>>>(chains, na);
    else if (kind == MEAS_R_CUBIC) k_measure<false, true, true><<<grid, MEAS_NT, 0, st>>>(chains, na);
    else k_measure<false, false, false><<<grid, MEAS_NT, 0, st>>>(chains, na);
}

// dyn_measure (src/dqmc_measure/dyn_measure.f90:1-101) at time index nt: the
// density correlation znn_tau(imj, no_i, no_j, nt) +=
//   (1/2 - Re G(t,t)_ii)(1/2 - Re G(0,0)_jj) - G(0,t)_ji G(t,0)_ij / nflr,
// weighted with zphi; G(0,t)^T is in GT.  One thread per bin, cells j in
// order (the reference's summation order for a bin).  On the cubic lattice
// (dyn_measure3d.f90:44-66) the same znn_tau goes to slot 0 of the time
// index's 4 lq bins, zspsm_tau(imj) += -G(0,t)_ji G(t,0)_ij (1 - 1/nflr^2) to
// slot lq and gtau0(imj) += G(t,0)_ij to slot 2 lq.
__global__ void __launch_bounds__(256) k_dyn_measure(const ChainDev* __restrict__ chains, int nt) {
    const ChainDev& c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    if (nt > md.ntdm + 1) return;
    const int N = c.N, lq = md.lq, nsub = md.nsub;
    const double2 phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    const double sgn = phase.x < 0.0 ? -1.0 : 1.0;
    const double2 zphi = cscale(phase, sgn / phase.x);
    const double fn = 1.0 / (double)md.nflr, fsp = 1.0 - fn * fn;
    const double2 *G = c.G, *GT = c.GT, *gt0 = c.gt0, *g00 = c.g00;
    double2* bin = c.dynbins + (size_t)4 * lq * (nt - 1);
    // the 3D lattices sum every orbital pair of a cell pair into one bin
    const int nbin = md.cubic ? lq : lq * nsub * nsub, no = md.cubic ? nsub : 1;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbin; b += gridDim.x * blockDim.x) {
        const int d = b % lq, ab = b / lq, a = ab % nsub, bb = ab / nsub;
        const CellShift<true> shift(d, md);     // l3 = 1 off the 3D lattices
        double2 z = cmk(0, 0), zs = cmk(0, 0), zg = cmk(0, 0);
        for (int cj = 0; cj < lq; ++cj) {
            const int ci = shift(cj);
            for (int ob = 0; ob < no; ++ob)
                for (int oa = 0; oa < no; ++oa) {
                    const int i = md.cubic ? ci * nsub + oa : ci * nsub + a, j = md.cubic ? cj * nsub + ob : cj * nsub + bb;
                    const size_t o = (size_t)i + (size_t)N * j;
                    const double v = (0.5 - G[(size_t)i * (N + 1)].x) * (0.5 - g00[(size_t)j * (N + 1)].x);
                    z = csub(cadd(z, cmk(v, 0.0)), cmul(cscale(GT[o], fn), gt0[o]));
                    if (md.cubic) { zs = csub(zs, cmul(cscale(GT[o], fsp), gt0[o])); zg = cadd(zg, gt0[o]); }
                }
        }
        const size_t k = (size_t)d + (size_t)lq * a + (size_t)2 * lq * bb;
        bin[k] = cfma(z, zphi, bin[k]);
        if (md.cubic) {
            bin[lq + d] = cfma(zs, zphi, bin[lq + d]);
            bin[2 * lq + d] = cfma(zg, zphi, bin[2 * lq + d]);
        }
    }
}

void launch_dyn_measure(const ChainDev* chains, int nchains, int maxN, int nt, cudaStream_t st) {
    const int ntl = (maxN + 31) / 32;
    k_transpose_g<<<dim3(ntl, ntl, nchains), 256, 0, st>>>(chains, MAT_G0T);
    k_dyn_measure<<<dim3(2, nchains), 256, 0, st>>>(chains, nt);
}

void launch_bins_clear(const ChainDev* chains, int nchains, int nbins, cudaStream_t st) {
    k_bins_clear<<<nchains, 256, 0, st>>>(chains, nbins);
}
