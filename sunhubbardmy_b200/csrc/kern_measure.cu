// Equal-time measurement of one time slice; a few CTAs per chain.
//
// Reference: src/dqmc_measure/equaltime_measure.f90 (equaltime_measure 1-69,
// zkint, zint_u, zint_v, zqsq, ztsq, ztq, measure_cpcm/spsm/nn/jj/bondcorr/
// paircorr).  Observables use Gc(i,j) = delta_ij - G(j,i) and are weighted
// with zphi = sgn/Re(phase) * phase.  G^T is written first (a tiled
// transpose), so that every correlation term reads a column of G or of G^T.
// The distance-binned correlations are accumulated without atomics: one
// thread owns one bin (distance d, orbitals a, b) and walks the unit cells j,
// pairing each with cell i = j + d (imj(i, j) = d, in closed form);
// the threads of consecutive d read consecutive rows of the same columns.
// The single-number energy terms run on the chain's first CTA.
//
// Bin layout per chain (complex): energy[10], cpcm, spsm, nn, pair_onsite
// [lq*4 each, index (d) + lq*(no_i + 2 no_j)], jj, bb, pair_nn, pair_sn [lq
// each], zn[2], zj, zb.
#include "chain_access.cuh"
#include "kernels.h"

DQ_DEV double2 gcf(const double2* G, int N, int i, int j) {   // Gc(i,j)
    double2 g = G[MIDX(j, i, N)];
    return cmk((i == j ? 1.0 : 0.0) - g.x, -g.y);
}
DQ_DEV double2 gf(const double2* G, int N, int i, int j) { return G[MIDX(i, j, N)]; }

// cell i = j + d of the distance table imj(i, j) = d (setup_latt2d_sub): with
// cells c = c1 l2 + c2 and d = dy + l2 dx, i1 = (j1 + dx + 1) mod l1 and
// i2 = (j2 + dy + 1) mod l2; dxp = dx + 1, dyp = dy + 1
DQ_DEV int cell_shift(int cj, int dxp, int dyp, int l1, int l2) {
    int i1 = cj / l2 + dxp, i2 = cj % l2 + dyp;
    if (i1 >= l1) i1 -= l1;
    if (i2 >= l2) i2 -= l2;
    return i1 * l2 + i2;
}

__global__ void __launch_bounds__(256) k_measure(const ChainDev* __restrict__ chains) {
    __shared__ double red[64];
    const ChainDev& c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    const int N = c.N, lq = md.lq, tid = threadIdx.x, nth = blockDim.x;
    const int nnf = md.nn_nf, zp = md.z_plq, nflr = md.nflr;
    const double2* G = c.G;
    double2* bins = c.bins;
    const double2 phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    const double sgn = phase.x < 0.0 ? -1.0 : 1.0;
    const double2 zphi = cscale(phase, sgn / phase.x);
    const double fsp = 1.0 - 1.0 / (double)(nflr * nflr), fn = 1.0 / (double)nflr;
    const bool hc = (md.nsub == 2);

    // ---- per-site and per-cell quantities shared by all bins (shared memory) ----
    __shared__ double2 gcd[512];     // Gc(i,i)
    __shared__ double2 jcell[512];   // Gc(i0,in) - Gc(in,i0), current partner
    __shared__ double2 bcell[512];   // e Gc(i0,ib) + conj(e) Gc(ib,i0), bond partner
    __shared__ int pj[512], pb[512], ps[512];
    for (int i = tid; i < N; i += nth) gcd[i] = gcf(G, N, i, i);
    for (int cc = tid; cc < lq; cc += nth) {
        int i0 = hc ? 2 * cc : cc;
        int inj = hc ? md.snlist[i0 * md.nsn] : md.nnlist[i0 * nnf];
        int inb = md.nnlist[i0 * nnf];
        double2 e = md.expar_nn[i0 * nnf];
        pj[cc] = inj; pb[cc] = inb; ps[cc] = md.snlist[i0 * md.nsn];
        jcell[cc] = csub(gcf(G, N, i0, inj), gcf(G, N, inj, i0));
        bcell[cc] = cadd(cmul(e, gcf(G, N, i0, inb)), cmul(cconj(e), gcf(G, N, inb, i0)));
    }
    __syncthreads();
    // ---- distance-binned correlations: one thread per bin, looping over the
    // cells j; for fixed j the threads of consecutive distances read G and G^T
    // down a column, so every access is coalesced and each bin is summed in a
    // fixed order without atomics ----
    double2* cpcm = bins + 10;
    double2* spsm = cpcm + 4 * lq;
    double2* znn = spsm + 4 * lq;
    double2* pons = znn + 4 * lq;
    double2* zjj = pons + 4 * lq;
    double2* zbb = zjj + lq;
    double2* pnn = zbb + lq;
    double2* psn = pnn + lq;
    const double2* GT = c.GT;
    const int nsub = md.nsub, l1 = md.l1, l2 = md.l2;
    const int nbin_a = lq * nsub * nsub, nbin = nbin_a + lq;
    for (int bin = blockIdx.x * nth + tid; bin < nbin; bin += gridDim.x * nth) {
        if (bin < nbin_a) {
            const int d = bin % lq, ab = bin / lq, a = ab % nsub, b = ab / nsub;
            const int dxp = d / l2 + 1, dyp = d % l2 + 1;
            double2 s1 = cmk(0, 0), s2 = cmk(0, 0), s3 = cmk(0, 0), s4 = cmk(0, 0);
#pragma unroll 4
            for (int cj = 0; cj < lq; ++cj) {
                const int i = cell_shift(cj, dxp, dyp, l1, l2) * nsub + a, j = cj * nsub + b;
                const size_t o = (size_t)i + (size_t)N * j;
                const double2 gt = GT[o], g = G[o];          // G(j,i), G(i,j)
                const double2 gc = cmk((i == j ? 1.0 : 0.0) - gt.x, -gt.y);
                const double2 gcg = cmul(gc, g);
                s1 = cadd(s1, gc);
                s2 = cadd(s2, gcg);
                s3 = cadd(s3, cadd(cmul(gcd[i], gcd[j]), cscale(gcg, fn)));
                s4 = cfma(g, g, s4);
            }
            const int k = d + lq * (a + 2 * b);
            cpcm[k] = cfma(s1, zphi, cpcm[k]);
            spsm[k] = cfma(cscale(s2, fsp), zphi, spsm[k]);
            znn[k] = cfma(s3, zphi, znn[k]);
            pons[k] = cfma(s4, zphi, pons[k]);
        } else {
            const int d = bin - nbin_a;
            const int dxp = d / l2 + 1, dyp = d % l2 + 1;
            // element (r, s) of G is G[r + N s], of G^T (= G(s, r)) GT[r + N s]
            auto gg = [&](int r, int s_) { return G[(size_t)r + (size_t)N * s_]; };
            auto gtt = [&](int r, int s_) { return GT[(size_t)r + (size_t)N * s_]; };
            auto cc = [&](int r, int s_) {            // Gc(r, s) = delta_rs - G(s, r)
                double2 t = gtt(r, s_);
                return cmk((r == s_ ? 1.0 : 0.0) - t.x, -t.y);
            };
            double2 sj = cmk(0, 0), sb = cmk(0, 0), sn = cmk(0, 0), ss = cmk(0, 0);
#pragma unroll 4
            for (int cj = 0; cj < lq; ++cj) {
                const int ci = cell_shift(cj, dxp, dyp, l1, l2);
                const int j0 = hc ? 2 * cj : cj, i0 = hc ? 2 * ci : ci;
                const int jnj = pj[cj], inj = pj[ci], jnb = pb[cj], inb = pb[ci];
                const double2 g00 = gg(i0, j0), gc00 = cc(i0, j0);
                // current-current, connected part (measure_jj)
                double2 z3 = cadd(cmul(cc(i0, jnj), gg(inj, j0)), cmul(cc(inj, j0), gg(i0, jnj)));
                const double2 gnn_j = gg(inj, jnj), gcnn_j = cc(inj, jnj);
                z3 = csub(z3, cadd(cmul(gc00, gnn_j), cmul(gcnn_j, g00)));
                sj = csub(sj, cadd(cmul(jcell[ci], jcell[cj]), cscale(z3, fn)));
                // bond-bond (measure_bondcorr)
                const double2 ej = md.expar_nn[j0 * nnf], ei = md.expar_nn[i0 * nnf];
                const bool same = (jnb == jnj && inb == inj);
                const double2 gnn_b = same ? gnn_j : gg(inb, jnb);
                const double2 gcnn_b = same ? gcnn_j : cc(inb, jnb);
                double2 x = cmul(cmul(ei, ej), cmul(cc(i0, jnb), gg(inb, j0)));
                x = cadd(x, cmul(cmul(cconj(ei), cconj(ej)), cmul(cc(inb, j0), gg(i0, jnb))));
                x = cadd(x, cmul(cmul(ei, cconj(ej)), cmul(gc00, gnn_b)));
                x = cadd(x, cmul(cmul(cconj(ei), ej), cmul(gcnn_b, g00)));
                sb = cadd(sb, cadd(cmul(bcell[cj], bcell[ci]), cscale(x, fn)));
                // pair correlations (measure_paircorr)
                sn = cfma(g00, gnn_b, sn);
                ss = cfma(g00, gg(ps[ci], ps[cj]), ss);
            }
            zjj[d] = cfma(sj, zphi, zjj[d]);
            zbb[d] = cfma(sb, zphi, zbb[d]);
            pnn[d] = cfma(sn, zphi, pnn[d]);
            psn[d] = cfma(ss, zphi, psn[d]);
        }
    }
    if (blockIdx.x != 0) return;
    // ---- energy terms ----
    double2 zne = cmk(0, 0), zu = cmk(0, 0), zk = cmk(0, 0), zv = cmk(0, 0);
    for (int i = tid; i < N; i += nth) {
        double2 d = gcf(G, N, i, i);
        zne = cadd(zne, d);
        zu = cadd(zu, cmul(d, d));
        if (md.t2 != 0.0) {
            int ns = hc ? 6 : 4;
            for (int f = 0; f < ns; ++f) zk.x += -md.t2 * gcf(G, N, i, md.snlist[i * md.nsn + f]).x;
        }
    }
    for (int b = tid; b < md.nn_lf * nnf; b += nth) {
        int i1 = md.bond_i1[b], i2 = md.bond_i2[b], nf = b / md.nn_lf;
        double2 g = gcf(G, N, i1, i2);
        zk.x += -2.0 * cmul(g, md.expar_nn[i1 * nnf + nf]).x;
        zv.x += g.x;
    }
    // plaquette terms
    double2 zq = cmk(0, 0), zt = cmk(0, 0), ztq = cmk(0, 0);
    const double2 em = cexpi(-md.theta), ep = cexpi(md.theta);
    for (int q = tid; q < lq; q += nth) {
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
        zj = cadd(zj, cmk(-dj.y, dj.x));
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
        bins[4] = cadd(bins[4], cscale(cmul(zq, zphi), 1.0 / 9.0));
        bins[5] = cadd(bins[5], cmul(zt, zphi));
        bins[6] = cadd(bins[6], cmul(ztq, zphi));
        bins[7] = cadd(bins[7], cscale(cmul(zv, zphi), md.rv));
        size_t tail = 10 + 20 * (size_t)lq;
        bins[tail + 0] = cadd(bins[tail + 0], cmul(zn0, zphi));
        bins[tail + 1] = cadd(bins[tail + 1], cmul(zn1, zphi));
        bins[tail + 2] = cadd(bins[tail + 2], cmul(zj, zphi));
        bins[tail + 3] = cadd(bins[tail + 3], cmul(zb, zphi));
        c.stats[ST_NOBS] += 1.0;
    }
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

void launch_measure(const ChainDev* chains, int nchains, int maxN, int ctas_per_chain, cudaStream_t st) {
    const int nt = (maxN + 31) / 32;
    k_transpose_g<<<dim3(nt, nt, nchains), 256, 0, st>>>(chains, MAT_G);
    dim3 grid(ctas_per_chain, nchains);
    k_measure<<<grid, 256, 0, st>>>(chains);
}

// dyn_measure (src/dqmc_measure/dyn_measure.f90:1-101) at time index nt: the
// density correlation znn_tau(imj, no_i, no_j, nt) +=
//   (1/2 - Re G(t,t)_ii)(1/2 - Re G(0,0)_jj) - G(0,t)_ji G(t,0)_ij / nflr,
// weighted with zphi; G(0,t)^T is in GT.  One thread per bin, cells j in
// order (the reference's summation order for a bin).
__global__ void __launch_bounds__(256) k_dyn_measure(const ChainDev* __restrict__ chains, int nt) {
    const ChainDev& c = chains[blockIdx.y];
    const ModelDev& md = *c.md;
    if (nt > md.ntdm + 1) return;
    const int N = c.N, lq = md.lq, nsub = md.nsub, l1 = md.l1, l2 = md.l2;
    const double2 phase = cmk(c.stats[ST_PHASE_RE], c.stats[ST_PHASE_IM]);
    const double sgn = phase.x < 0.0 ? -1.0 : 1.0;
    const double2 zphi = cscale(phase, sgn / phase.x);
    const double fn = 1.0 / (double)md.nflr;
    const double2 *G = c.G, *GT = c.GT, *gt0 = c.gt0, *g00 = c.g00;
    double2* bin = c.dynbins + (size_t)4 * lq * (nt - 1);
    const int nbin = lq * nsub * nsub;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbin; b += gridDim.x * blockDim.x) {
        const int d = b % lq, ab = b / lq, a = ab % nsub, bb = ab / nsub;
        const int dxp = d / l2 + 1, dyp = d % l2 + 1;
        double2 z = cmk(0, 0);
#pragma unroll 4
        for (int cj = 0; cj < lq; ++cj) {
            const int i = cell_shift(cj, dxp, dyp, l1, l2) * nsub + a, j = cj * nsub + bb;
            const size_t o = (size_t)i + (size_t)N * j;
            const double v = (0.5 - G[(size_t)i * (N + 1)].x) * (0.5 - g00[(size_t)j * (N + 1)].x);
            z = csub(cadd(z, cmk(v, 0.0)), cmul(cscale(GT[o], fn), gt0[o]));
        }
        const size_t k = (size_t)d + (size_t)lq * a + (size_t)2 * lq * bb;
        bin[k] = cfma(z, zphi, bin[k]);
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
