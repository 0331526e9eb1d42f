// Host side of the C ABI in include/dqmc_gpu.h: parameter derivation, model
// tables (lattice, HS constants, kinetic propagators), device allocation and
// the slice-by-slice orchestration of the finite-temperature sweep.
//
// The sweep follows the reference's control flow exactly
// (src/dqmc_ft_core/dqmc_ft_sweep_b0.f90, dqmc_ft_sweep_0b.f90,
// dqmc_ft_sweep_start_0b.f90); every chain of a handle is advanced by the same
// kernel launches (one CTA, or a few, per chain), and a full sweep is captured
// once into a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <thread>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dqmc_gpu.h"
#include "dqmc_types.h"
#include "kernels.h"
#include "nn.h"
#include "zgemm.cuh"

typedef std::complex<double> zc;

static thread_local std::string g_err = "";
static int fail(int code, const std::string& msg) { g_err = msg; return code; }
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(DQMC_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)

extern "C" const char* dqmc_gpu_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// parameters (src/model_para.f90:334-453)
// ---------------------------------------------------------------------------
extern "C" int dqmc_params_derive(dqmc_params* p) {
    if (!p) return fail(DQMC_EINVAL, "null params");
    if (p->lattice < DQMC_LATT_SQUARE || p->lattice > DQMC_LATT_R_CUBIC)
        return fail(DQMC_EINVAL, "lattice must be square, honeycomb, chain, cubic or r_cubic");
    const bool d3 = p->lattice == DQMC_LATT_CUBIC || p->lattice == DQMC_LATT_R_CUBIC;
    if (!d3) p->l3 = 1;
    if (p->lattice == DQMC_LATT_CHAIN) {
        if (p->l2 != 1 || p->l1 < 4 || p->l1 % 2) return fail(DQMC_EINVAL, "the chain needs l2 = 1 and an even l1 >= 4");
    } else if (p->lattice == DQMC_LATT_CUBIC) {
        // the A sublattice (i1 + i2 + i3 even) and its six bond families cover
        // every bond once only for even lengths (setup_cubic_sub, lattice.f90:1300-1312)
        if (p->l1 < 2 || p->l2 < 2 || p->l3 < 2 || p->l1 % 2 || p->l2 % 2 || p->l3 % 2)
            return fail(DQMC_EINVAL, "the cubic lattice needs even l1, l2, l3 >= 2");
    } else if (p->lattice == DQMC_LATT_R_CUBIC) {
        if (p->l1 < 2 || p->l2 < 2 || p->l3 < 2) return fail(DQMC_EINVAL, "the r_cubic lattice needs l1, l2, l3 >= 2");
        // the bond field's props and updates index the bonds in the reference order,
        // which the two-phase device order of the r_cubic family 4 differs from
        if (p->rv != 0.0) return fail(DQMC_EINVAL, "the t-V bond field is not supported on the r_cubic lattice");
    } else if (p->l1 < 2 || p->l2 < 2) {
        return fail(DQMC_EINVAL, "l1, l2 must be >= 2");
    }
    if (p->dtau <= 0 || p->beta <= 0) return fail(DQMC_EINVAL, "beta, dtau must be > 0");
    p->lq = p->l1 * p->l2 * p->l3;
    p->ndim = (p->lattice == DQMC_LATT_HONEYCOMB) ? 2 * p->lq : (p->lattice == DQMC_LATT_R_CUBIC) ? 6 * p->lq : p->lq;
    p->ne = p->ndim / 2 + (int)(p->nu * p->ndim / 8.0);
    p->ltrot = (int)std::lround(p->beta / p->dtau);
    if (p->nublock == 0) {
        if (p->update == DQMC_UPD_DELAY) {
            int q = p->ndim / 5;
            p->nublock = q < 16 ? 4 : q < 32 ? 8 : q < 64 ? 16 : q < 256 ? 32 : 64;
        } else if (p->update == DQMC_UPD_SUBMATRIX) {
            int q = p->ndim / 20;
            p->nublock = q < 32 ? 32 : q < 64 ? 64 : q < 128 ? 16 : q < 256 ? 256 : q < 512 ? 512 : 1024;
        }
    }
    if (p->ltrot < p->nwrap) p->nwrap = p->ltrot;
    if (p->ltrot < p->nwrap || !p->lstabilize) p->nst = 0;
    else p->nst = (p->ltrot % p->nwrap == 0) ? p->ltrot / p->nwrap : p->ltrot / p->nwrap + 1;
    if (p->lproju) p->lcomp = p->nflr / 2 + 1 + (int)(0.5 * std::fabs(p->nu));
    else if (p->hs == DQMC_HS_EXACT && p->nflr == 2) p->lcomp = 2;
    else p->lcomp = 4;
    if (p->obs_mid_len <= 0) p->obs_mid_len = 1;
    p->ntdm = p->ltau ? (int)std::lround(p->dyntau / p->dtau) : 0;
    if (p->ntdm < 0) p->ntdm = 0;
    if (p->ltau && p->proj && std::fabs(p->dyntau - p->beta) <= 1e-12 * std::fabs(p->beta))
        return fail(DQMC_EINVAL, "dyntau = beta is not allowed on the projective path (dqmc_proj_ctrl.f90:13)");
    if (p->ltau && p->nst < 1) return fail(DQMC_EINVAL, "unequal-time measurement (ltau) needs lstabilize and ltrot >= nwrap");
    if (p->proj && p->nst < 1) return fail(DQMC_EINVAL, "the projective sweep needs lstabilize and ltrot >= nwrap");
    if (p->rv < 0.0) return fail(DQMC_EINVAL, "rv must be >= 0 (acosh(exp(dtau rv / 2)))");
    if (p->proj && (p->ne < 1 || p->ne > p->ndim)) return fail(DQMC_EINVAL, "ne out of range 1..ndim");
    if (p->rhub_plq != 0.0) {
        if (p->lattice != DQMC_LATT_SQUARE && p->lattice != DQMC_LATT_HONEYCOMB)
            return fail(DQMC_EINVAL, "the plaquette field needs the square or honeycomb lattice");
        if (p->rhub_plq < 0.0) return fail(DQMC_EINVAL, "rhub_plq must be >= 0 (sqrt(dtau rhub_plq))");
    }
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// host model: lattice tables (src/lattice.f90) and model constants
// ---------------------------------------------------------------------------
static int npbc(int nr, int l) { return nr > l ? nr - l : (nr < 1 ? nr + l : nr); }

struct HostModel {
    dqmc_params p;
    int N, lq, nsub, nn_nf, nn_lf, z_plq, nsn, lcomp, nublock_dev;
    double a1[2], a2[2];
    std::vector<int> cell1, cell2, cell3; // unit-cell coordinates of site (1-based; cell3 cubic only)
    std::vector<double> rc1, rc2;         // real-space coordinates of site
    std::vector<int> nnlist, snlist;      // [site][nf] 0-based
    std::vector<int> nnveci;              // [site][nf][2]
    std::vector<double> nnvecr;           // [site][nf][2]
    std::vector<int> nnlf;                // A sites, 0-based
    std::vector<int> imj;                 // [i][j] 0-based distance index
    std::vector<int> plq;                 // [lq][z_plq] 0-based
    std::vector<zc> expar;                // [site][nf]
    std::vector<zc> urt, urtm1;           // [bond][4]
    std::vector<zc> exph0k, exph0kinv;    // divided by lq
    std::vector<zc> urtd, urtm1d;         // dense kinetic exp(-+dtau H0 / 2), N x N
    bool dense_on_device = false;         // dense kinetic: keep seth0 and build urtd on the device
    std::vector<zc> seth0;                // the hopping matrix of the dense kinetic term (device build)
    std::vector<int> bond_i1, bond_i2;
    std::vector<int> cell_plus;           // [d][j]
    // plaquette field (dqmc_set_plqconf.f90): z x z blocks per field value
    bool plq_on = false;
    int plq_lcomp = 0;
    std::vector<zc> plq_bmat, plq_bmat_inv, plq_delta, plq_phase, plq_phase_ratio;
    std::vector<double> plq_gam_ratio;
    ModelDev dev;                         // host copy with device pointers
    ModelDev* d_dev = nullptr;
    std::vector<void*> allocs;
    int iwrap_first_nonzero;
    std::vector<int> iwrap_nt;            // [0..ltrot]
    std::vector<int> wrap_step;           // [n][2] 1-based
};

// setup_latt3d_sub / setup_cubic_sub (src/lattice.f90:1033-1157, 1280-1472).
// Site s = (i3-1) l1 l2 + (i1-1) l2 + i2 (1-based, i2 fastest) is also the
// cell.  Bond families from the A sites (i1 + i2 + i3 even, in the order of the
// loops i1, i2, i3): +a3, +a1, +a2, -a3, -a1, -a2; twelve second neighbours;
// eight-site cubes in eight parity classes; imj(i, j) = (nz-1) l1 l2 + ny +
// (nx-1) l2 with n = npbc(u_i - u_j).
static void build_cubic(HostModel& m) {
    const dqmc_params& p = m.p;
    const int l1 = p.l1, l2 = p.l2, l3 = p.l3;
    m.a1[0] = 1; m.a1[1] = 0; m.a2[0] = 0; m.a2[1] = 1;
    m.lq = l1 * l2 * l3;
    m.nsub = 1; m.N = m.lq; m.nn_nf = 6; m.nn_lf = m.lq / 2; m.z_plq = 8; m.nsn = 12;
    const int N = m.N;
    auto site = [&](int i1, int i2, int i3) { return (npbc(i3, l3) - 1) * l1 * l2 + (npbc(i1, l1) - 1) * l2 + npbc(i2, l2) - 1; };
    m.cell1.resize(N); m.cell2.resize(N); m.cell3.resize(N); m.rc1.resize(N); m.rc2.resize(N);
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) {
                const int s = site(i1, i2, i3);
                m.cell1[s] = i1; m.cell2[s] = i2; m.cell3[s] = i3; m.rc1[s] = i1; m.rc2[s] = i2;
                if ((i1 + i2 + i3) % 2 == 0) m.nnlf.push_back(s);
            }
    const int nn[6][3] = {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, -1}, {-1, 0, 0}, {0, -1, 0}};
    const int sn[12][3] = {{1, 1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {0, 1, 1}, {0, 1, -1},
                           {0, -1, -1}, {0, -1, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}, {-1, 0, 1}};
    m.nnlist.assign(N * 6, 0); m.snlist.assign(N * 12, 0);
    m.nnveci.assign(N * 6 * 2, 0); m.nnvecr.assign(N * 6 * 2, 0.0);    // unused: the 3D bonds carry no phase
    for (int s = 0; s < N; ++s) {
        const int c1 = m.cell1[s], c2 = m.cell2[s], c3 = m.cell3[s];
        for (int f = 0; f < 6; ++f) m.nnlist[s * 6 + f] = site(c1 + nn[f][0], c2 + nn[f][1], c3 + nn[f][2]);
        for (int f = 0; f < 12; ++f) m.snlist[s * 12 + f] = site(c1 + sn[f][0], c2 + sn[f][1], c3 + sn[f][2]);
    }
    m.imj.assign(m.lq * m.lq, 0);
    m.cell_plus.assign(m.lq * m.lq, 0);
    for (int j = 0; j < m.lq; ++j)
        for (int i = 0; i < m.lq; ++i) {
            const int nx = npbc(m.cell1[i] - m.cell1[j], l1), ny = npbc(m.cell2[i] - m.cell2[j], l2);
            const int nz = npbc(m.cell3[i] - m.cell3[j], l3);
            const int d = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2 - 1;
            m.imj[i * m.lq + j] = d;
            m.cell_plus[d * m.lq + j] = i;
        }
    int nd[8] = {0}, id[8] = {0};
    auto typ = [](int i1, int i2, int i3) { return (i1 % 2 == 0) * 4 + (i2 % 2 == 0) * 2 + (i3 % 2 == 0); };
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) nd[typ(i1, i2, i3)]++;
    m.plq.assign(m.lq * 8, 0);
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int i3 = 1; i3 <= l3; ++i3) {
                const int t = typ(i1, i2, i3);
                int off = 0;
                for (int q = 0; q < t; ++q) off += nd[q];
                int* pc = &m.plq[(id[t]++ + off) * 8];
                pc[0] = site(i1, i2, i3);         pc[1] = site(i1 + 1, i2, i3);
                pc[2] = site(i1 + 1, i2 + 1, i3); pc[3] = site(i1, i2 + 1, i3);
                pc[4] = site(i1, i2, i3 + 1);     pc[5] = site(i1 + 1, i2, i3 + 1);
                pc[6] = site(i1 + 1, i2 + 1, i3 + 1); pc[7] = site(i1, i2 + 1, i3 + 1);
            }
}

// setup_latt3d_sub / setup_r_cubic_sub (src/lattice.f90:1033-1157, 1486-1605):
// three honeycomb layers per cell, sites (cell - 1) 6 + isub with isub = A1,
// B1, A2, B2, A3, B3 and cells numbered as on the cubic lattice; the A sites
// (odd, 1-based) own the nn_lf = 3 lq bonds of the four families.  nnlist is
// the reference's table as written (family 4 of A1 reaches sub-site 2 of the
// cell at (-1, -1, -1), so two family-4 bonds share that B1 site); snlist,
// tnlist and plq_cord are left empty (0 in the reference, -1 here).
static void build_rcubic(HostModel& m) {
    const dqmc_params& p = m.p;
    const int l1 = p.l1, l2 = p.l2, l3 = p.l3;
    m.a1[0] = 1; m.a1[1] = 0; m.a2[0] = 0; m.a2[1] = 1;
    m.lq = l1 * l2 * l3;
    m.nsub = 6; m.N = 6 * m.lq; m.nn_nf = 4; m.nn_lf = 3 * m.lq; m.z_plq = 8; m.nsn = 12;
    const int N = m.N;
    auto cell = [&](int i1, int i2, int i3) { return (npbc(i3, l3) - 1) * l1 * l2 + (npbc(i1, l1) - 1) * l2 + npbc(i2, l2) - 1; };
    m.cell1.resize(N); m.cell2.resize(N); m.cell3.resize(N); m.rc1.resize(N); m.rc2.resize(N);
    for (int i3 = 1; i3 <= l3; ++i3)
        for (int i1 = 1; i1 <= l1; ++i1)
            for (int i2 = 1; i2 <= l2; ++i2)
                for (int o = 0; o < 6; ++o) {
                    const int s = cell(i1, i2, i3) * 6 + o;
                    m.cell1[s] = i1; m.cell2[s] = i2; m.cell3[s] = i3; m.rc1[s] = i1; m.rc2[s] = i2;
                }
    for (int b = 0; b < m.nn_lf; ++b) m.nnlf.push_back(2 * b);
    m.nnlist.assign(N * 4, 0); m.snlist.assign(N * 12, -1);
    m.nnveci.assign(N * 4 * 2, 0); m.nnvecr.assign(N * 4 * 2, 0.0);
    for (int s = 0; s < N; ++s) {
        const int i = s + 1, r = i % 6, c1 = m.cell1[s], c2 = m.cell2[s], c3 = m.cell3[s];
        int* nl = &m.nnlist[s * 4];
        if (r == 3 || r == 5 || r == 1) {          // A2, A3, A1
            nl[0] = s + 1;
            nl[1] = cell(c1 - 1, c2, c3) * 6 + r;     // 0-based sub-site r = 1-based r + 1
            nl[2] = cell(c1, c2 - 1, c3) * 6 + r;
            nl[3] = (r == 1) ? cell(c1 - 1, c2 - 1, c3 - 1) * 6 + r : s - 1;
        } else if (r == 2 || r == 4) {              // B1, B2
            nl[0] = s - 1;
            nl[1] = cell(c1 + 1, c2, c3) * 6 + r - 2;
            nl[2] = cell(c1, c2 + 1, c3) * 6 + r - 2;
            nl[3] = s + 1;
        } else {                                     // B3
            nl[0] = s - 1;
            nl[1] = cell(c1 + 1, c2, c3) * 6 + 4;
            nl[2] = cell(c1, c2 + 1, c3) * 6 + 4;
            nl[3] = cell(c1 + 1, c2 + 1, c3 + 1) * 6;
        }
    }
    m.imj.assign(m.lq * m.lq, 0);
    m.cell_plus.assign(m.lq * m.lq, 0);
    for (int j = 0; j < m.lq; ++j)
        for (int i = 0; i < m.lq; ++i) {
            const int si = i * 6, sj = j * 6;
            const int nx = npbc(m.cell1[si] - m.cell1[sj], l1), ny = npbc(m.cell2[si] - m.cell2[sj], l2);
            const int nz = npbc(m.cell3[si] - m.cell3[sj], l3);
            const int d = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2 - 1;
            m.imj[i * m.lq + j] = d;
            m.cell_plus[d * m.lq + j] = i;
        }
    m.plq.assign(m.lq * 8, -1);
}

static void build_lattice(HostModel& m) {
    const dqmc_params& p = m.p;
    int l1 = p.l1, l2 = p.l2;
    if (p.lattice == DQMC_LATT_CUBIC) { build_cubic(m); return; }
    if (p.lattice == DQMC_LATT_R_CUBIC) { build_rcubic(m); return; }
    m.lq = l1 * l2;
    if (p.lattice == DQMC_LATT_CHAIN) {
        // setup_latt1d_sub / setup_chain_sub (src/lattice.f90:67-135, 240-316): bond
        // families +a1 and -a1 from the A sites (even, 1-based), second neighbours
        // at +-2 a1; imj(i, j) = npbc(i - j, l1) is the 2D table with l2 = 1
        m.a1[0] = 1; m.a1[1] = 0; m.a2[0] = 0; m.a2[1] = 1;
        m.nsub = 1; m.N = l1; m.nn_nf = 2; m.nn_lf = l1 / 2; m.z_plq = 1; m.nsn = 2;
        const int N = m.N;
        m.cell1.resize(N); m.cell2.assign(N, 1); m.rc1.resize(N); m.rc2.assign(N, 1.0);
        m.nnlist.assign(N * 2, 0); m.snlist.assign(N * 2, 0);
        m.nnveci.assign(N * 2 * 2, 0); m.nnvecr.assign(N * 2 * 2, 0.0);
        for (int i = 0; i < N; ++i) {
            const int i1 = i + 1;
            m.cell1[i] = i1; m.rc1[i] = i1;
            m.nnlist[i * 2 + 0] = npbc(i1 + 1, l1) - 1;
            m.nnlist[i * 2 + 1] = npbc(i1 - 1, l1) - 1;
            m.snlist[i * 2 + 0] = npbc(i1 + 2, l1) - 1;
            m.snlist[i * 2 + 1] = npbc(i1 - 2, l1) - 1;
            m.nnveci[(i * 2 + 0) * 2] = 1; m.nnvecr[(i * 2 + 0) * 2] = 1.0;
            m.nnveci[(i * 2 + 1) * 2] = -1; m.nnvecr[(i * 2 + 1) * 2] = -1.0;
            if (i1 % 2 == 0) m.nnlf.push_back(i);
        }
        m.imj.assign(m.lq * m.lq, 0);
        m.cell_plus.assign(m.lq * m.lq, 0);
        for (int j = 0; j < m.lq; ++j)
            for (int i = 0; i < m.lq; ++i) {
                const int d = npbc(i - j, l1) - 1;
                m.imj[i * m.lq + j] = d;
                m.cell_plus[d * m.lq + j] = i;
            }
        m.plq.resize(m.lq);
        for (int c = 0; c < m.lq; ++c) m.plq[c] = c;
        return;
    }
    bool sq = (p.lattice == DQMC_LATT_SQUARE);
    if (sq) { m.a1[0] = 1; m.a1[1] = 0; m.a2[0] = 0; m.a2[1] = 1; }
    else { m.a1[0] = 0.5; m.a1[1] = -0.5 * std::sqrt(3.0); m.a2[0] = 0.5; m.a2[1] = 0.5 * std::sqrt(3.0); }
    m.nsub = sq ? 1 : 2;
    m.N = m.lq * m.nsub;
    m.nn_nf = sq ? 4 : 3;
    m.nn_lf = sq ? m.lq / 2 : m.lq;
    m.z_plq = sq ? 4 : 6;
    m.nsn = sq ? 4 : 6;
    int N = m.N;
    m.cell1.resize(N); m.cell2.resize(N); m.rc1.resize(N); m.rc2.resize(N);
    // unit cell index c = i2 + (i1-1) l2 (1-based); site = c (square) or 2(c-1)+orb
    for (int i1 = 1; i1 <= l1; ++i1)
        for (int i2 = 1; i2 <= l2; ++i2)
            for (int o = 1; o <= m.nsub; ++o) {
                int cidx = i2 + (i1 - 1) * l2;
                int s = (cidx - 1) * m.nsub + (o - 1);
                m.cell1[s] = i1; m.cell2[s] = i2;
                if (sq || o == 1) { m.rc1[s] = i1; m.rc2[s] = i2; }
                else { m.rc1[s] = i1 - 1.0 / 3.0; m.rc2[s] = i2 + 1.0 / 3.0; }
            }
    auto cellsite = [&](int i1, int i2, int o) { return ((npbc(i1, l1) - 1) * l2 + npbc(i2, l2) - 1) * m.nsub + o; };
    m.nnlist.assign(N * m.nn_nf, 0);
    m.snlist.assign(N * m.nsn, 0);
    m.nnveci.assign(N * m.nn_nf * 2, 0);
    m.nnvecr.assign(N * m.nn_nf * 2, 0.0);
    if (sq) {
        const int v[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
        const int s[4][2] = {{1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
        for (int i = 0; i < N; ++i) {
            for (int f = 0; f < 4; ++f) {
                m.nnlist[i * 4 + f] = cellsite(m.cell1[i] + v[f][0], m.cell2[i] + v[f][1], 0);
                m.snlist[i * 4 + f] = cellsite(m.cell1[i] + s[f][0], m.cell2[i] + s[f][1], 0);
                m.nnveci[(i * 4 + f) * 2] = v[f][0]; m.nnveci[(i * 4 + f) * 2 + 1] = v[f][1];
                m.nnvecr[(i * 4 + f) * 2] = v[f][0]; m.nnvecr[(i * 4 + f) * 2 + 1] = v[f][1];
            }
        }
        for (int i1 = 1; i1 <= l1; ++i1)
            for (int i2 = 1; i2 <= l2; ++i2)
                if ((i1 + i2) % 2 == 0) m.nnlf.push_back(i2 + (i1 - 1) * l2 - 1);
    } else {
        // A (orb 0) -> B neighbours: same cell, cell + a1, cell - a2 (lattice.f90:713-742)
        const int vA[3][2] = {{0, 0}, {1, 0}, {0, -1}}, vB[3][2] = {{0, 0}, {-1, 0}, {0, 1}};
        const double rA[3][2] = {{-1.0 / 3, 1.0 / 3}, {2.0 / 3, 1.0 / 3}, {-1.0 / 3, -2.0 / 3}};
        const double rB[3][2] = {{1.0 / 3, -1.0 / 3}, {-2.0 / 3, -1.0 / 3}, {1.0 / 3, 2.0 / 3}};
        const int sn[6][2] = {{1, 1}, {1, 0}, {0, -1}, {-1, -1}, {-1, 0}, {0, 1}};
        for (int i = 0; i < N; ++i) {
            bool A = (i % 2 == 0);
            int c1 = m.cell1[i], c2 = m.cell2[i];
            for (int f = 0; f < 3; ++f) {
                const int* v = A ? vA[f] : vB[f];
                m.nnlist[i * 3 + f] = cellsite(c1 + v[0], c2 + v[1], A ? 1 : 0);
                m.nnveci[(i * 3 + f) * 2] = v[0]; m.nnveci[(i * 3 + f) * 2 + 1] = v[1];
                m.nnvecr[(i * 3 + f) * 2] = A ? rA[f][0] : rB[f][0];
                m.nnvecr[(i * 3 + f) * 2 + 1] = A ? rA[f][1] : rB[f][1];
            }
            for (int f = 0; f < 6; ++f) m.snlist[i * 6 + f] = cellsite(c1 + sn[f][0], c2 + sn[f][1], A ? 0 : 1);
        }
        for (int c = 0; c < m.lq; ++c) m.nnlf.push_back(2 * c);
    }
    // imj (setup_latt2d_sub) and the cell table cell_plus[d][j]
    m.imj.assign(m.lq * m.lq, 0);
    m.cell_plus.assign(m.lq * m.lq, 0);
    for (int j = 0; j < m.lq; ++j)
        for (int i = 0; i < m.lq; ++i) {
            int ui1 = i / l2 + 1, ui2 = i % l2 + 1, uj1 = j / l2 + 1, uj2 = j % l2 + 1;
            int nx = npbc(ui1 - uj1, l1), ny = npbc(ui2 - uj2, l2);
            int d = ny + (nx - 1) * l2 - 1;
            m.imj[i * m.lq + j] = d;
            m.cell_plus[d * m.lq + j] = i;
        }
    // plaquettes
    m.plq.assign(m.lq * m.z_plq, 0);
    if (sq) {
        int nd[4] = {0, 0, 0, 0}, id[4] = {0, 0, 0, 0};
        auto typ = [](int i1, int i2) {
            return (i1 % 2 == 1 && i2 % 2 == 1) ? 0 : (i1 % 2 == 0 && i2 % 2 == 1) ? 1 : (i1 % 2 == 0 && i2 % 2 == 0) ? 2 : 3;
        };
        for (int i1 = 1; i1 <= l1; ++i1) for (int i2 = 1; i2 <= l2; ++i2) nd[typ(i1, i2)]++;
        for (int i1 = 1; i1 <= l1; ++i1)
            for (int i2 = 1; i2 <= l2; ++i2) {
                int t = typ(i1, i2), off = 0;
                for (int q = 0; q < t; ++q) off += nd[q];
                int pid = id[t]++ + off;
                m.plq[pid * 4 + 0] = cellsite(i1, i2, 0);
                m.plq[pid * 4 + 1] = cellsite(i1 + 1, i2, 0);
                m.plq[pid * 4 + 2] = cellsite(i1 + 1, i2 + 1, 0);
                m.plq[pid * 4 + 3] = cellsite(i1, i2 + 1, 0);
            }
    } else {
        int nd[3] = {0, 0, 0}, id[3] = {0, 0, 0};
        auto typ = [](int i1, int i2) { int r = (i1 + i2) % 3; return r == 2 ? 0 : (r == 0 ? 2 : 1); };
        for (int i1 = 1; i1 <= l1; ++i1) for (int i2 = 1; i2 <= l2; ++i2) nd[typ(i1, i2)]++;
        for (int i1 = 1; i1 <= l1; ++i1)
            for (int i2 = 1; i2 <= l2; ++i2) {
                int t = typ(i1, i2), off = 0;
                for (int q = 0; q < t; ++q) off += nd[q];
                int pid = id[t]++ + off;
                m.plq[pid * 6 + 0] = cellsite(i1, i2, 1);
                m.plq[pid * 6 + 1] = cellsite(i1, i2, 0);
                m.plq[pid * 6 + 2] = cellsite(i1, i2 - 1, 1);
                m.plq[pid * 6 + 3] = cellsite(i1 - 1, i2 - 1, 0);
                m.plq[pid * 6 + 4] = cellsite(i1 - 1, i2 - 1, 1);
                m.plq[pid * 6 + 5] = cellsite(i1 - 1, i2, 0);
            }
    }
}

// Peierls / twist / dimerisation phase of bond (site i, family nf 1-based): expar.f90
static zc expar(const HostModel& m, int i, int nf) {
    const dqmc_params& p = m.p;
    if (p.lattice == DQMC_LATT_CUBIC || p.lattice == DQMC_LATT_R_CUBIC) return zc(1.0, 0.0);    // expar3d.f90: no phase
    int k = (i * m.nn_nf + nf - 1) * 2;
    int nax = m.nnveci[k], nay = m.nnveci[k + 1];
    double vr1 = m.nnvecr[k], vr2 = m.nnvecr[k + 1];
    double rc1 = m.rc1[i], rc2 = m.rc2[i];
    int c1 = m.cell1[i], c2 = m.cell2[i];
    // the chain has no Peierls phase (expar1d.f90: x = x1 = 0)
    double xmag1 = (p.lattice == DQMC_LATT_CHAIN) ? 0.0 : p.xmag / m.lq * (m.a1[0] * m.a2[1] - m.a1[1] * m.a2[0]);
    double x = -xmag1 * vr1 * (2.0 * rc2 + vr2) * M_PI, x1 = 0.0;
    bool e2 = (c2 == p.l2 && nay > 0) || (c2 == 1 && nay < 0);
    bool e1 = (c1 == p.l1 && nax > 0) || (c1 == 1 && nax < 0);
    double proj = (rc2 + vr2) * m.a2[0] + (rc1 + vr1) * m.a1[0];
    int sx = nax > 0 ? 1 : -1, sy = nay > 0 ? 1 : -1;
    if (e2 && nax == 0) x1 = 2.0 * M_PI * xmag1 * (double)(sy * p.l2) * m.a2[1] * proj;
    else if (e1 && nay == 0) x1 = 2.0 * M_PI * xmag1 * (double)(sx * p.l1) * m.a1[1] * proj;
    else if (e1 && e2) x1 = 2.0 * M_PI * xmag1 * ((double)(sx * p.l1) * m.a1[1] + (double)(sy * p.l2) * m.a2[1]) * proj;
    zc e = std::exp(zc(0.0, x + x1));
    double av0 = p.flux_x * m.a1[0] / p.l1 + p.flux_y * m.a2[0] / p.l2;
    double av1 = p.flux_x * m.a1[1] / p.l1 + p.flux_y * m.a2[1] / p.l2;
    double rv0 = nax * m.a1[0] + nay * m.a2[0], rv1 = nax * m.a1[1] + nay * m.a2[1];
    e *= std::exp(zc(0.0, 2.0 * M_PI * (av0 * rv0 + av1 * rv1)));
    if (nf == 1) e *= (1.0 + p.dimer);
    return e;
}

// exp(-s h) of h = [[d, z],[conj z, d]] in closed form
static void exp2x2(double d, zc z, double s, zc* out) {
    double az = std::abs(z), e = std::exp(-s * d);
    double ch = std::cosh(s * az), sh = az > 0 ? std::sinh(s * az) / az : 0.0;
    out[0] = e * ch; out[1] = -e * sh * z; out[2] = -e * sh * std::conj(z); out[3] = e * ch;
}

static void eig_herm(int n, std::vector<zc>& a, std::vector<double>& w);
static void set_plq(HostModel& m);

static int build_model(HostModel& m) {
    dqmc_params& p = m.p;
    if (p.t3 != 0.0) return fail(DQMC_EINVAL, "t3 != 0 is not supported");
    if (p.kinetic < DQMC_KIN_CHECKERBOARD || p.kinetic > DQMC_KIN_DENSE) return fail(DQMC_EINVAL, "kinetic must be 0, 1 or 2");
    if (p.lattice < DQMC_LATT_SQUARE || p.lattice > DQMC_LATT_R_CUBIC) return fail(DQMC_EINVAL, "lattice must be 1 to 5");
    if (p.lattice == DQMC_LATT_CUBIC && (p.l1 < 2 || p.l2 < 2 || p.l3 < 2 || p.l1 % 2 || p.l2 % 2 || p.l3 % 2))
        return fail(DQMC_EINVAL, "the cubic lattice needs even l1, l2, l3 >= 2");
    if (p.lattice == DQMC_LATT_CHAIN && (p.l2 != 1 || p.l1 < 4 || p.l1 % 2))
        return fail(DQMC_EINVAL, "the chain needs l2 = 1 and an even l1 >= 4");
    if (p.kinetic == DQMC_KIN_FFT && (p.lattice != DQMC_LATT_SQUARE || p.l1 != p.l2))
        return fail(DQMC_EINVAL, "FFT kinetic term needs a square lattice with l1 == l2");
    if (p.lattice == DQMC_LATT_SQUARE && ((p.l1 * p.l2) % 2 != 0 || p.l1 % 2 || p.l2 % 2) && p.kinetic == DQMC_KIN_CHECKERBOARD)
        return fail(DQMC_EINVAL, "checkerboard square lattice needs even l1, l2");
    build_lattice(m);
    if (m.N > 512) return fail(DQMC_EINVAL, "ndim > 512 is not supported");
    if (p.nst < 1) return fail(DQMC_EINVAL, "the sweep needs stabilisation (nst >= 1)");
    int N = m.N;
    m.lcomp = p.lcomp;
    m.nublock_dev = (p.update == DQMC_UPD_FAST) ? 32 : p.nublock;
    if (m.nublock_dev > 64) m.nublock_dev = 64;
    if (m.nublock_dev < 1) m.nublock_dev = 1;
    m.expar.resize(N * m.nn_nf);
    for (int i = 0; i < N; ++i)
        for (int f = 1; f <= m.nn_nf; ++f) m.expar[i * m.nn_nf + f - 1] = expar(m, i, f);
    // bonds (dqmc_set_h0conf.f90:76-123)
    int nb = m.nn_nf * m.nn_lf;
    m.bond_i1.resize(nb); m.bond_i2.resize(nb); m.urt.resize(nb * 4); m.urtm1.resize(nb * 4);
    for (int f = 1; f <= m.nn_nf; ++f)
        for (int b = 0; b < m.nn_lf; ++b) {
            int ist = b + (f - 1) * m.nn_lf;
            int i0 = m.nnlf[b], i1 = m.nnlist[i0 * m.nn_nf + f - 1];
            m.bond_i1[ist] = i0; m.bond_i2[ist] = i1;
            // the r_cubic build hops rtd on family 4 (dqmc_set_h0conf.f90:22-73)
            const double t = (p.lattice == DQMC_LATT_R_CUBIC && f == 4) ? p.rtd : p.rt;
            zc z = -t * m.expar[i0 * m.nn_nf + f - 1];
            double d = -p.mu / m.nn_nf;
            exp2x2(d, z, 0.5 * p.dtau, &m.urt[ist * 4]);
            exp2x2(d, z, -0.5 * p.dtau, &m.urtm1[ist * 4]);
        }
    if (p.kinetic == DQMC_KIN_DENSE) {
        // urt = U exp(-dtau e / 2) U^H and urtm1 = U exp(+dtau e / 2) U^H from the
        // eigen-decomposition of the seth0 matrix (dqmc_set_h0conf.f90:484-509,
        // seth0.f90): nearest-neighbour bonds -rt expar, diagonal -mu
        std::vector<zc> H((size_t)N * N, 0.0);
        for (int b = 0; b < m.nn_lf; ++b) {
            int i0 = m.nnlf[b];
            for (int f = 1; f <= m.nn_nf; ++f) {
                int in = m.nnlist[i0 * m.nn_nf + f - 1];
                zc z1 = -p.rt * m.expar[i0 * m.nn_nf + f - 1];
                H[i0 + (size_t)in * N] += z1;
                H[in + (size_t)i0 * N] += std::conj(z1);
            }
        }
        for (int i = 0; i < N; ++i) H[i + (size_t)i * N] -= p.mu;
        if (m.dense_on_device) {
            m.seth0 = std::move(H);       // upload_model diagonalises it on the device
        } else {
            std::vector<double> w;
            eig_herm(N, H, w);
            m.urtd.assign((size_t)N * N, 0.0);
            m.urtm1d.assign((size_t)N * N, 0.0);
            std::vector<double> em(N), ep(N);
            for (int k = 0; k < N; ++k) { em[k] = std::exp(-0.5 * p.dtau * w[k]); ep[k] = std::exp(0.5 * p.dtau * w[k]); }
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) {
                    zc z0 = 0, z1 = 0;
                    for (int k = 0; k < N; ++k) {
                        zc t = H[i + (size_t)k * N] * std::conj(H[j + (size_t)k * N]);
                        z0 += t * em[k];
                        z1 += t * ep[k];
                    }
                    m.urtd[i + (size_t)j * N] = z0;
                    m.urtm1d[i + (size_t)j * N] = z1;
                }
        }
    }
    if (p.kinetic == DQMC_KIN_FFT) {
        // eigenvalues h0k = diag(F H F^-1), F the unitary forward DFT over (l1, l2)
        // with column index j1 + l1 j2 (dqmc_set_h0conf.f90:225-291); H from seth0.f90
        int l1 = p.l1, l2 = p.l2, lq = m.lq;
        std::vector<std::pair<std::pair<int, int>, zc>> H;
        for (int b = 0; b < nb; ++b) {
            int f = b / m.nn_lf + 1;
            zc z = -p.rt * m.expar[m.bond_i1[b] * m.nn_nf + f - 1];
            H.push_back({{m.bond_i1[b], m.bond_i2[b]}, z});
            H.push_back({{m.bond_i2[b], m.bond_i1[b]}, std::conj(z)});
        }
        for (int i = 0; i < N; ++i) H.push_back({{i, i}, zc(-p.mu, 0.0)});
        m.exph0k.resize(lq); m.exph0kinv.resize(lq);
        for (int k = 0; k < lq; ++k) {
            int k1 = k % l1, k2 = k / l1;
            zc h = 0;
            for (auto& e : H) {
                int j = e.first.first, jp = e.first.second;
                double ph = -2 * M_PI * ((double)(j % l1) * k1 / l1 + (double)(j / l1) * k2 / l2)
                            + 2 * M_PI * ((double)(jp % l1) * k1 / l1 + (double)(jp / l1) * k2 / l2);
                h += e.second * std::exp(zc(0.0, ph));
            }
            h /= (double)lq;
            m.exph0k[k] = std::exp(-0.5 * p.dtau * h) / (double)lq;
            m.exph0kinv[k] = std::exp(0.5 * p.dtau * h) / (double)lq;
        }
    }
    set_plq(m);
    // stabilisation schedule
    m.iwrap_nt.assign(p.ltrot + 1, 0);
    m.wrap_step.assign(2 * p.nst, 0);
    for (int i = 1; i <= p.nst; ++i) {
        int hi = (i == p.nst) ? p.ltrot : i * p.nwrap;
        m.iwrap_nt[hi] = i;
        m.wrap_step[(i - 1) * 2] = (i - 1) * p.nwrap + 1;
        m.wrap_step[(i - 1) * 2 + 1] = hi;
    }
    return DQMC_OK;
}

// Plaquette-field constants (src/dqmc_config_plqu/dqmc_set_plqconf.f90:1-200):
// vstmat has 1/nn_nf on the diagonal and alpha e^{-+i theta} around the
// plaquette (the reference's column-major listing); bmat(is) =
// U exp(i a_is e) U^H with a_is = sqrt(dtau rhub_plq) eta(is), or
// pi 2 nn_nf is / lcomp under lprojplqu (nu integer); the field values follow
// the 4-component eta/gamma of dqmc_config_plqu.f90:44-52.
static void set_plq(HostModel& m) {
    const dqmc_params& p = m.p;
    m.plq_on = p.rhub_plq != 0.0;
    if (!m.plq_on) return;
    const int z = m.z_plq, nnf = m.nn_nf;
    const bool hc = p.lattice == DQMC_LATT_HONEYCOMB;
    const bool lproj = p.lprojplqu && (double)(int)p.nu == p.nu;
    m.plq_lcomp = lproj ? (hc ? nnf * (int)(p.nflr + std::fabs(p.nu)) + 1 : (int)(nnf * (0.5 * p.nflr + std::fabs(p.nu))) + 1) : 4;
    const int lc = m.plq_lcomp;
    const double ap = std::sqrt(p.dtau * p.rhub_plq), th = p.theta * M_PI;
    const zc z0 = 1.0 / nnf, z1 = p.alpha * std::exp(zc(0, -th)), z1h = p.alpha * std::exp(zc(0, th)), o = 0.0;
    std::vector<zc> v;
    if (z == 6) v = {z0, z1, o, o, o, -z1,  z1h, z0, -z1h, o, o, o,  o, -z1, z0, z1, o, o,
                     o, o, z1h, z0, -z1h, o,  o, o, o, -z1, z0, z1,  -z1h, o, o, o, z1h, z0};
    else v = {z0, z1, o, -z1,  z1h, z0, -z1h, o,  o, -z1, z0, z1,  -z1h, o, z1h, z0};
    std::vector<double> e;
    eig_herm(z, v, e);                                  // v <- eigenvectors (columns)
    auto eta = [](int is) {
        const double a = std::sqrt(2.0 * (3.0 + std::sqrt(6.0))), b = std::sqrt(2.0 * (3.0 - std::sqrt(6.0)));
        return is == 1 ? -a : is == 2 ? -b : is == 3 ? b : a;
    };
    auto gam = [](int is) { return (is == 1 || is == 4) ? 1.0 - std::sqrt(6.0) / 3.0 : 1.0 + std::sqrt(6.0) / 3.0; };
    auto block = [&](double a, zc* out, double shift) {
        for (int j = 0; j < z; ++j)
            for (int i = 0; i < z; ++i) {
                zc s0 = 0;
                for (int k = 0; k < z; ++k) s0 += v[i + z * k] * std::exp(zc(0, e[k] * a)) * std::conj(v[j + z * k]);
                out[i + z * j] = (i == j) ? s0 - shift : s0;
            }
    };
    const double fac = hc ? 1.0 : 0.5;
    m.plq_bmat.assign((size_t)lc * z * z, 0.0); m.plq_bmat_inv.assign((size_t)lc * z * z, 0.0);
    m.plq_delta.assign((size_t)lc * (lc - 1) * z * z, 0.0); m.plq_phase.assign(lc, 0.0);
    m.plq_phase_ratio.assign((size_t)lc * (lc - 1), 0.0); m.plq_gam_ratio.assign((size_t)lc * (lc - 1), 1.0);
    for (int is = 1; is <= lc; ++is) {
        const double a = lproj ? M_PI * 2.0 * nnf * is / lc : ap * eta(is);
        block(a, &m.plq_bmat[(size_t)(is - 1) * z * z], 0.0);
        block(-a, &m.plq_bmat_inv[(size_t)(is - 1) * z * z], 0.0);
        m.plq_phase[is - 1] = lproj ? std::exp(zc(0, M_PI * (-2.0 * nnf * is) * fac * (p.nflr + p.nu) / lc))
                                    : std::exp(zc(0, ap * (-eta(is)) * fac * (p.nflr + p.nu)));
        for (int iflip = 1; iflip <= lc - 1; ++iflip) {
            const int isp = (is + iflip - 1) % lc + 1;
            const size_t k2 = (size_t)(is - 1) * (lc - 1) + (iflip - 1);
            const double ad = lproj ? M_PI * (2.0 * nnf * isp - 2.0 * nnf * is) / lc : ap * (eta(isp) - eta(is));
            block(ad, &m.plq_delta[k2 * z * z], 1.0);
            m.plq_phase_ratio[k2] = lproj ? std::exp(zc(0, M_PI * (2.0 * nnf * is - 2.0 * nnf * isp) * fac * (p.nflr + p.nu) / lc))
                                          : std::exp(zc(0, ap * (eta(is) - eta(isp)) * fac * (p.nflr + p.nu)));
            m.plq_gam_ratio[k2] = lproj ? 1.0 : gam(isp) / gam(is);
        }
    }
}

// HS constants (src/dqmc_config_u/dqmc_set_conf.f90:1-176)
static void set_hs(const HostModel& m, ModelDev& d) {
    const dqmc_params& p = m.p;
    int nflr = p.nflr, lc = m.lcomp;
    double u = p.rhub, dtau = p.dtau, nu = p.nu, al;
    double eta[4], gam[4];
    bool exact = (p.hs == DQMC_HS_EXACT);
    bool general = !exact || (nflr != 2 && nflr != 4 && nflr != 6);
    if (!general && nflr == 2) {
        eta[0] = -1; eta[1] = 1;
        al = (u >= 0) ? std::acos(std::exp(-dtau * std::fabs(u) * 0.5)) : std::acosh(std::exp(dtau * std::fabs(u) * 0.5));
        gam[0] = gam[1] = 1.0;
    } else if (!general) {
        double a = std::exp(-0.5 * dtau * u);
        double dd = std::sqrt(8.0 + a * a * (3.0 + a * a) * (3.0 + a * a));
        double xp = (a + 2 * a * a * a + std::pow(a, 5) + (a * a - 1.0) * dd) / 4.0;
        double xm = (a + 2 * a * a * a + std::pow(a, 5) - (a * a - 1.0) * dd) / 4.0;
        if (u >= 0) { eta[0] = -std::acos(xm); eta[1] = -std::acos(xp); eta[2] = std::acos(xp); eta[3] = std::acos(xm); }
        else { eta[0] = -std::acosh(xm); eta[1] = -std::acosh(xp); eta[2] = std::acosh(xp); eta[3] = std::acosh(xm); }
        al = 1.0;
        double t = a * (3.0 + a * a);
        gam[0] = (t + dd) / dd; gam[1] = (-t + dd) / dd; gam[2] = (-t + dd) / dd; gam[3] = (t + dd) / dd;
    } else {
        double s6 = std::sqrt(6.0);
        eta[0] = -std::sqrt(2.0 * (3.0 + s6)); eta[1] = -std::sqrt(2.0 * (3.0 - s6));
        eta[2] = std::sqrt(2.0 * (3.0 - s6)); eta[3] = std::sqrt(2.0 * (3.0 + s6));
        al = std::sqrt(dtau * std::fabs(u) * 0.5);
        gam[0] = 1.0 - s6 / 3.0; gam[1] = 1.0 + s6 / 3.0; gam[2] = 1.0 + s6 / 3.0; gam[3] = 1.0 - s6 / 3.0;
    }
    auto put = [](double2& o, zc z) { o.x = z.real(); o.y = z.imag(); };
    for (int is = 1; is <= lc; ++is) {
        zc ph, b, bi;
        double ang;
        if (p.lproju) {
            ang = M_PI * (-2.0 * is) * 0.5 * (nflr + nu) / lc;
            ph = std::exp(zc(0, ang));
            b = std::exp(zc(0, M_PI * 2.0 * is / lc));
            bi = std::exp(zc(0, -M_PI * 2.0 * is / lc));
        } else if (u >= 0) {
            ang = al * (-eta[is - 1]) * 0.5 * (nflr + nu);
            ph = std::exp(zc(0, ang));
            b = std::exp(zc(0, al * eta[is - 1]));
            bi = std::exp(zc(0, -al * eta[is - 1]));
        } else {
            ang = 0.0;
            ph = std::exp(al * (-eta[is - 1]) * 0.5 * (nflr + nu));
            b = std::exp(al * eta[is - 1]);
            bi = std::exp(-al * eta[is - 1]);
        }
        put(d.phase[is - 1], ph); put(d.bmat[is - 1], b); put(d.bmat_inv[is - 1], bi);
        d.phase_angle[is - 1] = ang;
    }
    for (int is = 1; is <= lc; ++is)
        for (int iflip = 1; iflip <= lc - 1; ++iflip) {
            int isp = (is + iflip - 1) % lc + 1, k = (is - 1) * (lc - 1) + iflip - 1;
            zc pr, dl;
            if (p.lproju) {
                pr = std::exp(zc(0, M_PI * (2.0 * is - 2.0 * isp) * 0.5 * (nflr + nu) / lc));
                dl = std::exp(zc(0, M_PI * (2.0 * isp - 2.0 * is) / lc)) - 1.0;
            } else if (u >= 0) {
                pr = std::exp(zc(0, al * (eta[is - 1] - eta[isp - 1]) * 0.5 * (nflr + nu)));
                dl = std::exp(zc(0, al * (eta[isp - 1] - eta[is - 1]))) - 1.0;
            } else {
                pr = std::exp(al * (eta[is - 1] - eta[isp - 1]) * 0.5 * (nflr + nu));
                dl = std::exp(al * (eta[isp - 1] - eta[is - 1])) - 1.0;
            }
            put(d.phase_ratio[k], pr); put(d.delta[k], dl);
            d.gam_ratio[k] = p.lproju ? 1.0 : gam[isp - 1] / gam[is - 1];
        }
}

template <class T>
static int upload(HostModel& m, const std::vector<T>& v, const T** out) {
    void* p = nullptr;
    size_t bytes = v.size() * sizeof(T);
    if (bytes == 0) { *out = nullptr; return DQMC_OK; }
    if (cudaMalloc(&p, bytes) != cudaSuccess) return fail(DQMC_ENOMEM, "cudaMalloc model table");
    if (cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return fail(DQMC_ECUDA, "model upload");
    m.allocs.push_back(p);
    *out = (const T*)p;
    return DQMC_OK;
}

static std::vector<double2> to_d2(const std::vector<zc>& v) {
    std::vector<double2> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) { o[i].x = v[i].real(); o[i].y = v[i].imag(); }
    return o;
}

static int upload_model(HostModel& m) {
    ModelDev& d = m.dev;
    memset(&d, 0, sizeof(d));
    const dqmc_params& p = m.p;
    d.N = m.N; d.lq = m.lq; d.nsub = m.nsub; d.l1 = p.l1; d.l2 = p.l2; d.nn_nf = m.nn_nf; d.nn_lf = m.nn_lf;
    d.z_plq = m.z_plq; d.nsn = m.nsn; d.lcomp = m.lcomp; d.nflr = p.nflr; d.lproju = p.lproju;
    d.kinetic = p.kinetic; d.update = p.update; d.nublock = m.nublock_dev; d.ltrot = p.ltrot; d.nst = p.nst;
    d.ntdm = p.ltau ? p.ntdm : -1;
    d.nwrap = p.nwrap; d.lwrapT = (p.rt != 0.0); d.lwrapu = (p.rhub != 0.0);
    d.phase_on = (p.rhub > 0.0) ? 1 : 0;
    d.rt = p.rt; d.rv = p.rv; d.t2 = p.t2; d.theta = p.theta * M_PI;
    d.chain = p.lattice == DQMC_LATT_CHAIN;
    d.cubic = p.lattice == DQMC_LATT_CUBIC || p.lattice == DQMC_LATT_R_CUBIC;
    d.l3 = p.l3;
    set_hs(m, d);
    // projective path and vconf constants (src/dqmc_config_v/dqmc_set_conf.f90:1-79)
    d.proj = p.proj ? 1 : 0;
    d.ne = p.ne;
    d.lwrapv = (p.rv != 0.0);
    d.rps = d.proj ? ((d.lwrapu ? 2 * m.N : 0) + (d.lwrapv ? 2 * m.nn_lf * m.nn_nf : 0)) : 2 * m.N;
    if (m.plq_on || d.lwrapv) {
        // a slice's draws in the reference's order: 0b visits the plaquettes,
        // then the bond families 1..nn_nf, then the U field
        // (dqmc_ft_sweep_0b.f90:82-119, dqmc_proj_sweep_0b.f90:61-90); b0 the U
        // field, the families nn_nf..1, then the plaquettes
        // (dqmc_ft_sweep_b0.f90:70-101, dqmc_proj_sweep_b0.f90:70-99)
        const int wu = d.lwrapu ? 2 * m.N : 0, wp = m.plq_on ? 2 * m.lq : 0;
        const int wv = d.lwrapv ? 2 * m.nn_lf * m.nn_nf : 0;
        d.rps = wu + wv + wp;
        d.rw_plq[0] = 0; d.rw_v[0] = wp; d.rw_u[0] = wp + wv;
        d.rw_u[1] = 0; d.rw_v[1] = wu; d.rw_plq[1] = wu + wv;
        d.rw_pre0 = wp;
    }
    if (m.plq_on) {
        d.plq = 1; d.plq_z = m.z_plq; d.plq_lcomp = m.plq_lcomp;
        if (m.plq_lcomp > DQ_MAX_PLQ_LCOMP) return fail(DQMC_EINVAL, "too many plaquette field values");
        for (int is = 0; is < m.plq_lcomp; ++is) d.plq_phase_angle[is] = std::arg(m.plq_phase[is]);
    }
    if (d.lwrapv) {
        const double etal[2] = {-1.0, 1.0};
        double al = std::acosh(std::exp(p.dtau * p.rv * 0.5));
        auto put = [](double2& o, zc z) { o.x = z.real(); o.y = z.imag(); };
        for (int is = 1; is <= 2; ++is) {
            int isp = is % 2 + 1;
            if (p.lprojv) {
                zc z = std::exp(zc(0, M_PI * 2.0 * is / 2.0));
                put(d.vbp[is - 1], z); put(d.vbm[is - 1], z);
                put(d.vbpi[is - 1], std::conj(z)); put(d.vbmi[is - 1], std::conj(z));
                put(d.vdp[is - 1], std::exp(zc(0, M_PI * (2.0 * isp - 2.0 * is) / 2.0)) - 1.0);
                put(d.vdm[is - 1], zc(std::exp(al * (etal[isp - 1] - etal[is - 1])) - 1.0, 0.0));
            } else {
                put(d.vbp[is - 1], zc(std::exp(al * etal[is - 1]), 0.0));
                put(d.vbpi[is - 1], zc(std::exp(-al * etal[is - 1]), 0.0));
                put(d.vbm[is - 1], zc(std::exp(-al * etal[is - 1]), 0.0));
                put(d.vbmi[is - 1], zc(std::exp(al * etal[is - 1]), 0.0));
                put(d.vdp[is - 1], zc(std::exp(al * (etal[isp - 1] - etal[is - 1])) - 1.0, 0.0));
                put(d.vdm[is - 1], zc(std::exp(-al * (etal[isp - 1] - etal[is - 1])) - 1.0, 0.0));
            }
        }
    }
    int rc;
    {
        // The reference applies the bonds of a family one after the other
        // (dqmc_left_forward_prop.f90:27-38); the device applies a family's
        // bonds in parallel, which is the same product only for bonds without
        // a common site.  Each family is stored as two such phases: the bonds
        // none of whose sites occurred earlier in the family, then the rest
        // (the r_cubic family 4 shares its B1 sites); phase 2 runs after phase 1.
        const int lf = m.nn_lf, nnf = m.nn_nf;
        if (nnf > DQ_MAX_NNF) return fail(DQMC_EINVAL, "too many bond families");
        std::vector<int> b1(m.bond_i1.size()), b2(m.bond_i2.size());
        std::vector<zc> u(m.urt.size()), um(m.urtm1.size());
        for (int f = 0; f < nnf; ++f) {
            std::vector<int> seen(m.N, 0), order, late;
            for (int b = 0; b < lf; ++b) {
                const int ist = f * lf + b, x = m.bond_i1[ist], y = m.bond_i2[ist];
                (seen[x] || seen[y] ? late : order).push_back(ist);
                seen[x]++; seen[y]++;
            }
            std::vector<int> seen2(m.N, 0);
            for (int ist : late)
                if (seen2[m.bond_i1[ist]]++ || seen2[m.bond_i2[ist]]++)
                    return fail(DQMC_EINVAL, "a bond family needs more than two disjoint phases");
            d.cb_split[f] = (int)order.size();
            order.insert(order.end(), late.begin(), late.end());
            for (int b = 0; b < lf; ++b) {
                const int src = order[b], dst = f * lf + b;
                b1[dst] = m.bond_i1[src]; b2[dst] = m.bond_i2[src];
                for (int e = 0; e < 4; ++e) { u[dst * 4 + e] = m.urt[src * 4 + e]; um[dst * 4 + e] = m.urtm1[src * 4 + e]; }
            }
        }
        if ((rc = upload(m, b1, &d.bond_i1))) return rc;
        if ((rc = upload(m, b2, &d.bond_i2))) return rc;
        std::vector<double2> tb;
        tb = to_d2(u); if ((rc = upload(m, tb, &d.urt))) return rc;
        tb = to_d2(um); if ((rc = upload(m, tb, &d.urtm1))) return rc;
    }
    std::vector<double2> t;
    if (p.kinetic == DQMC_KIN_DENSE && m.dense_on_device) {
        // urt / urtm1 from the device eigen-decomposition of seth0
        std::vector<double2> z((size_t)m.N * m.N, make_double2(0.0, 0.0));
        if ((rc = upload(m, z, &d.urtd))) return rc;
        if ((rc = upload(m, z, &d.urtm1d))) return rc;
        std::vector<double2> H = to_d2(m.seth0);
        const int sw = dense_kinetic_device(H.data(), m.N, p.dtau, (double2*)d.urtd, (double2*)d.urtm1d, nullptr);
        if (sw == -2) return fail(DQMC_ENUMERIC, "the seth0 eigensolver did not converge");
        if (sw < 0) return fail(DQMC_ECUDA, "device eigensolver of seth0 failed");
    } else if (p.kinetic == DQMC_KIN_DENSE) {
        t = to_d2(m.urtd); if ((rc = upload(m, t, &d.urtd))) return rc;
        t = to_d2(m.urtm1d); if ((rc = upload(m, t, &d.urtm1d))) return rc;
    }
    if (p.kinetic == DQMC_KIN_FFT) {
        t = to_d2(m.exph0k); if ((rc = upload(m, t, &d.exph0k))) return rc;
        t = to_d2(m.exph0kinv); if ((rc = upload(m, t, &d.exph0kinv))) return rc;
        if (p.l1 == p.l2) {
            const int l = p.l1;
            std::vector<zc> tk(m.exph0k.size()), tki(m.exph0k.size());
            for (int k1 = 0; k1 < l; ++k1)
                for (int k2 = 0; k2 < l; ++k2) {
                    tk[k2 + l * k1] = m.exph0k[k1 + l * k2];
                    tki[k2 + l * k1] = m.exph0kinv[k1 + l * k2];
                }
            t = to_d2(tk); if ((rc = upload(m, t, &d.exph0kT))) return rc;
            t = to_d2(tki); if ((rc = upload(m, t, &d.exph0kinvT))) return rc;
        }
        std::vector<zc> w1(p.l1), w2(p.l2);
        for (int k = 0; k < p.l1; ++k) w1[k] = std::exp(zc(0, -2 * M_PI * k / p.l1));
        for (int k = 0; k < p.l2; ++k) w2[k] = std::exp(zc(0, -2 * M_PI * k / p.l2));
        t = to_d2(w1); if ((rc = upload(m, t, &d.tw1))) return rc;
        t = to_d2(w2); if ((rc = upload(m, t, &d.tw2))) return rc;
    }
    if (m.plq_on) {
        t = to_d2(m.plq_bmat); if ((rc = upload(m, t, &d.plq_bmat))) return rc;
        t = to_d2(m.plq_bmat_inv); if ((rc = upload(m, t, &d.plq_bmat_inv))) return rc;
        t = to_d2(m.plq_delta); if ((rc = upload(m, t, &d.plq_delta))) return rc;
        t = to_d2(m.plq_phase_ratio); if ((rc = upload(m, t, &d.plq_phase_ratio))) return rc;
        if ((rc = upload(m, m.plq_gam_ratio, &d.plq_gam_ratio))) return rc;
    }
    if ((rc = upload(m, m.cell_plus, &d.cell_plus))) return rc;
    if ((rc = upload(m, m.nnlist, &d.nnlist))) return rc;
    if ((rc = upload(m, m.snlist, &d.snlist))) return rc;
    if ((rc = upload(m, m.plq, &d.plq_cord))) return rc;
    t = to_d2(m.expar); if ((rc = upload(m, t, &d.expar_nn))) return rc;
    {
        std::vector<int> vr(2 * m.nn_lf * m.nn_nf);
        for (int f = 0; f < m.nn_nf; ++f)
            for (int b = 0; b < m.nn_lf; ++b) {
                vr[f * 2 * m.nn_lf + 2 * b] = m.bond_i1[f * m.nn_lf + b];
                vr[f * 2 * m.nn_lf + 2 * b + 1] = m.bond_i2[f * m.nn_lf + b];
            }
        if ((rc = upload(m, vr, &d.vrows))) return rc;
    }
    void* pd = nullptr;
    if (cudaMalloc(&pd, sizeof(ModelDev)) != cudaSuccess) return fail(DQMC_ENOMEM, "cudaMalloc model");
    m.allocs.push_back(pd);
    m.d_dev = (ModelDev*)pd;
    if (cudaMemcpy(pd, &d, sizeof(ModelDev), cudaMemcpyHostToDevice) != cudaSuccess) return fail(DQMC_ECUDA, "model upload");
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// SFMT seeding (lib/m_spring.f90:187-243), on the host
// ---------------------------------------------------------------------------
static void sfmt_seed(uint32_t* st, int32_t seed) {
    static const uint32_t parity[4] = {1u, 0u, 0u, 0x13c9e684u};
    st[0] = (uint32_t)seed;
    for (int i = 1; i < 624; ++i) st[i] = 1812433253u * (st[i - 1] ^ (st[i - 1] >> 30)) + (uint32_t)i;
    uint32_t inner = 0;
    for (int i = 0; i < 4; ++i) inner ^= st[i] & parity[i];
    for (int i = 16; i > 0; i >>= 1) inner ^= inner >> i;
    if ((inner & 1) != 1) {
        bool done = false;
        for (int i = 0; i < 4 && !done; ++i) {
            uint32_t work = 1;
            for (int j = 0; j < 32; ++j) {
                if (work & parity[i]) { st[i] ^= work; done = true; break; }
                work <<= 1;
            }
        }
    }
    st[624] = 624;   // read index: the first draw regenerates the block
}

// host restatement of spring_sfmt_source for the fresh-start conf draw
struct HostSfmt {
    uint32_t st[625];
    void gen() {
        static const uint32_t msk[4] = {0xdfffffefU, 0xddfecb7fU, 0xbffaffffU, 0xbffffff6U};
        auto rec = [&](uint32_t* r, const uint32_t* a, const uint32_t* b, const uint32_t* c, const uint32_t* d) {
            uint64_t ah = ((uint64_t)a[3] << 32) | a[2], al = ((uint64_t)a[1] << 32) | a[0];
            uint64_t ch = ((uint64_t)c[3] << 32) | c[2], cl = ((uint64_t)c[1] << 32) | c[0];
            uint64_t xh = (ah << 8) | (al >> 56), xl = al << 8, yh = ch >> 8, yl = (cl >> 8) | (ch << 56);
            uint32_t x[4] = {(uint32_t)xl, (uint32_t)(xl >> 32), (uint32_t)xh, (uint32_t)(xh >> 32)};
            uint32_t y[4] = {(uint32_t)yl, (uint32_t)(yl >> 32), (uint32_t)yh, (uint32_t)(yh >> 32)};
            uint32_t o[4];
            for (int k = 0; k < 4; ++k) o[k] = a[k] ^ x[k] ^ ((b[k] >> 11) & msk[k]) ^ y[k] ^ (d[k] << 18);
            for (int k = 0; k < 4; ++k) r[k] = o[k];
        };
        uint32_t *r1 = st + 4 * 154, *r2 = st + 4 * 155;
        for (int i = 0; i < 156; ++i) {
            int bi = i < 34 ? i + 122 : i + 122 - 156;
            rec(st + 4 * i, st + 4 * i, st + 4 * bi, r1, r2);
            r1 = r2; r2 = st + 4 * i;
        }
    }
    uint32_t next() { if (st[624] >= 624) { gen(); st[624] = 0; } return st[st[624]++]; }
    double stream() { return ((double)next() + 0.5) * (1.0 / 4294967296.0); }
};

// ---------------------------------------------------------------------------
// trial state of the projective path (dqmc_set_proj, src/dqmc_proj_core/
// dqmc_set_proj.f90:1-78, with set_trial_h0, src/dqmc_config_h0/
// set_trial_h0.f90:1-29).  The Hermitian eigenproblem (s_eig_he / zheev in
// the reference) is solved on the host: Householder reduction to a real
// symmetric tridiagonal matrix (reflectors with a real beta, as in LAPACK's
// zhetrd), then the implicit QL iteration with Wilkinson-type shifts of the
// EISPACK tql2 procedure, accumulated into the complex eigenvectors.
// ---------------------------------------------------------------------------
static void eig_herm(int n, std::vector<zc>& a, std::vector<double>& w) {
    // a: n x n Hermitian (column-major) in, eigenvectors (columns) out
    std::vector<zc> q(n * n, 0.0), v(n), pv(n), row(n);
    for (int i = 0; i < n; ++i) q[i + i * n] = 1.0;
    std::vector<double> d(n), e(n, 0.0);
    auto A = [&](int i, int j) -> zc& { return a[i + (size_t)j * n]; };
    for (int k = 0; k + 2 < n; ++k) {
        int m = n - k - 1;                     // reflector acts on rows/cols k+1..n-1
        zc alpha = A(k + 1, k);
        double xn2 = 0.0;
        for (int i = k + 2; i < n; ++i) xn2 += std::norm(A(i, k));
        double xnorm = std::sqrt(xn2);
        zc tau = 0.0;
        if (!(xnorm == 0.0 && alpha.imag() == 0.0)) {
            double beta = -std::copysign(std::sqrt(std::norm(alpha) + xn2), alpha.real());
            tau = zc((beta - alpha.real()) / beta, -alpha.imag() / beta);
            zc scal = 1.0 / (alpha - beta);
            v[0] = 1.0;
            for (int i = 1; i < m; ++i) v[i] = A(k + 1 + i, k) * scal;
            // B <- B H (B = trailing block), H = I - tau v v^H
            for (int i = 0; i < m; ++i) pv[i] = 0.0;
            for (int j = 0; j < m; ++j) {
                zc vj = v[j];
                const zc* col = &A(k + 1, k + 1 + j);
                for (int i = 0; i < m; ++i) pv[i] += col[i] * vj;
            }
            for (int j = 0; j < m; ++j) {
                zc f = tau * std::conj(v[j]);
                for (int i = 0; i < m; ++i) A(k + 1 + i, k + 1 + j) -= pv[i] * f;
            }
            // B <- H^H B
            for (int j = 0; j < m; ++j) {
                zc s = 0.0;
                for (int i = 0; i < m; ++i) s += std::conj(v[i]) * A(k + 1 + i, k + 1 + j);
                row[j] = s;
            }
            for (int j = 0; j < m; ++j) {
                zc f = std::conj(tau) * row[j];
                for (int i = 0; i < m; ++i) A(k + 1 + i, k + 1 + j) -= v[i] * f;
            }
            // Q <- Q H
            std::vector<zc>& qs = row;
            for (int i = 0; i < n; ++i) qs[i] = 0.0;
            for (int j = 0; j < m; ++j) {
                zc vj = v[j];
                const zc* col = &q[(size_t)(k + 1 + j) * n];
                for (int i = 0; i < n; ++i) qs[i] += col[i] * vj;
            }
            for (int j = 0; j < m; ++j) {
                zc f = tau * std::conj(v[j]);
                zc* col = &q[(size_t)(k + 1 + j) * n];
                for (int i = 0; i < n; ++i) col[i] -= qs[i] * f;
            }
            alpha = beta;
        }
        e[k] = alpha.real();                 // real after the reflection (or already real)
        // a complex subdiagonal left by a zero reflector is made real by a phase
        if (alpha.imag() != 0.0) e[k] = std::abs(alpha);
        if (alpha.imag() != 0.0) {
            zc ph = alpha / std::abs(alpha);  // scale basis vector k+1 by ph
            for (int j = 0; j < n; ++j) A(k + 1, j) *= std::conj(ph);
            for (int i = 0; i < n; ++i) A(i, k + 1) *= ph;
            for (int i = 0; i < n; ++i) q[i + (size_t)(k + 1) * n] *= ph;
        }
    }
    if (n >= 2) {
        zc last = A(n - 1, n - 2);
        if (last.imag() != 0.0) {
            zc ph = last / std::abs(last);
            for (int j = 0; j < n; ++j) A(n - 1, j) *= std::conj(ph);
            for (int i = 0; i < n; ++i) A(i, n - 1) *= ph;
            for (int i = 0; i < n; ++i) q[i + (size_t)(n - 1) * n] *= ph;
        }
        e[n - 2] = A(n - 1, n - 2).real();
    }
    for (int i = 0; i < n; ++i) d[i] = A(i, i).real();
    // implicit QL on (d, e), e[i] couples i and i+1
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < n; ++l) {
        for (int iter = 0; iter < 60; ++iter) {
            int mm = l;
            for (; mm < n - 1; ++mm) {
                double dd = std::fabs(d[mm]) + std::fabs(d[mm + 1]);
                if (std::fabs(e[mm]) <= eps * dd) break;
            }
            if (mm == l) break;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + std::copysign(r, g));
            double sn = 1.0, cs = 1.0, pp = 0.0;
            int i = mm - 1;
            bool underflow = false;
            for (; i >= l; --i) {
                double f = sn * e[i], b = cs * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) { d[i + 1] -= pp; e[mm] = 0.0; underflow = true; break; }
                sn = f / r; cs = g / r;
                g = d[i + 1] - pp;
                r = (d[i] - g) * sn + 2.0 * cs * b;
                pp = sn * r;
                d[i + 1] = g + pp;
                g = cs * r - b;
                for (int k = 0; k < n; ++k) {
                    zc fz = q[k + (size_t)(i + 1) * n];
                    q[k + (size_t)(i + 1) * n] = sn * q[k + (size_t)i * n] + cs * fz;
                    q[k + (size_t)i * n] = cs * q[k + (size_t)i * n] - sn * fz;
                }
            }
            if (underflow) continue;
            d[l] -= pp; e[l] = g; e[mm] = 0.0;
        }
    }
    // ascending order
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return d[x] < d[y]; });
    w.resize(n);
    for (int j = 0; j < n; ++j) {
        w[j] = d[idx[j]];
        for (int i = 0; i < n; ++i) a[i + (size_t)j * n] = q[i + (size_t)idx[j] * n];
    }
}

// set_trial_h0: nn_lf * nn_nf draws in (bond, family) order, then -mu
static void trial_hamiltonian(const HostModel& m, HostSfmt& rng, std::vector<zc>& H) {
    const dqmc_params& p = m.p;
    int N = m.N;
    H.assign((size_t)N * N, 0.0);
    for (int b = 0; b < m.nn_lf; ++b) {
        int i0 = m.nnlf[b];
        for (int f = 1; f <= m.nn_nf; ++f) {
            int in = m.nnlist[i0 * m.nn_nf + f - 1];
            double r = rng.stream();
            zc z1 = (-p.rt + p.rndness * (r - 1.0)) * m.expar[i0 * m.nn_nf + f - 1];
            H[i0 + (size_t)in * N] += z1;
            H[in + (size_t)i0 * N] += std::conj(z1);
        }
    }
    for (int i = 0; i < N; ++i) H[i + (size_t)i * N] -= p.mu;
}

// the fresh-start draws of one chain, in the reference's order (dqmc_start,
// src/dqmc_ft_ctrl.f90:9-45): plaquette field (hconf%input_plqconf), U field
// (uconf%input_conf), bond field (vconf%input_conf), then the trial hopping
static void draw_fields(const HostModel& m, HostSfmt& rng, int draw_conf, std::vector<int32_t>& conf,
                        std::vector<int32_t>& vconf, std::vector<int32_t>* conf_plq = nullptr) {
    int N = m.N, lt = m.p.ltrot, nnf = m.nn_nf;
    if (m.plq_on) {          // dqmc_input_plqconf.f90:53-60: nt outer, plaquette inner
        std::vector<int32_t> cp((size_t)lt * m.lq, 1);
        if (draw_conf)
            for (size_t e = 0; e < cp.size(); ++e) cp[e] = (int32_t)std::ceil(rng.stream() * m.plq_lcomp);
        if (conf_plq) *conf_plq = std::move(cp);
    }
    conf.assign((size_t)lt * N, 1);
    if (draw_conf && m.p.rhub != 0.0)
        for (size_t e = 0; e < conf.size(); ++e) conf[e] = (int32_t)std::ceil(rng.stream() * m.lcomp);
    vconf.clear();
    if (m.p.rv != 0.0) {
        vconf.assign((size_t)lt * nnf * N, 1);
        if (draw_conf)
            for (int nt = 0; nt < lt; ++nt)
                for (int i = 0; i < N; ++i)
                    for (int f = 0; f < nnf; ++f)
                        vconf[((size_t)nt * nnf + f) * N + i] = (int32_t)std::ceil(rng.stream() * 2);
    }
}

extern "C" int dqmc_trial_state(const dqmc_params* pin, int32_t seed, int draw_conf, double* proj, double* w) {
    if (!pin || !proj) return fail(DQMC_EINVAL, "null argument");
    HostModel m;
    m.p = *pin;
    int rc = dqmc_params_derive(&m.p);
    if (rc) return rc;
    if ((rc = build_model(m))) return rc;
    HostSfmt rng;
    sfmt_seed(rng.st, seed);
    std::vector<int32_t> conf, vconf;
    draw_fields(m, rng, draw_conf, conf, vconf);
    std::vector<zc> H;
    trial_hamiltonian(m, rng, H);
    std::vector<double> ww;
    eig_herm(m.N, H, ww);
    memcpy(proj, H.data(), H.size() * sizeof(zc));
    if (w) memcpy(w, ww.data(), ww.size() * sizeof(double));
    return DQMC_OK;
}

// host-only view of the model tables (no device needed)
extern "C" int dqmc_model_tables(const dqmc_params* pin, int32_t* nnlist, int32_t* nnlf_list, int32_t* list,
                                 int32_t* imj, int32_t* plq_cord, int32_t* snlist, double* urt, double* exph0k) {
    if (!pin) return fail(DQMC_EINVAL, "null params");
    HostModel m;
    m.p = *pin;
    int rc = dqmc_params_derive(&m.p);
    if (rc) return rc;
    if ((rc = build_model(m))) return rc;
    int N = m.N, lq = m.lq;
    if (nnlist) for (int i = 0; i < N * m.nn_nf; ++i) nnlist[i] = m.nnlist[i] + 1;
    if (nnlf_list) for (int i = 0; i < m.nn_lf; ++i) nnlf_list[i] = m.nnlf[i] + 1;
    if (list) for (int i = 0; i < N; ++i) { list[2 * i] = i / m.nsub + 1; list[2 * i + 1] = i % m.nsub + 1; }
    if (imj) for (int i = 0; i < lq * lq; ++i) imj[i] = m.imj[i] + 1;
    if (plq_cord) for (int i = 0; i < lq * m.z_plq; ++i) plq_cord[i] = m.plq[i] + 1;
    if (snlist) for (int i = 0; i < N * m.nsn; ++i) snlist[i] = m.snlist[i] + 1;
    if (urt) memcpy(urt, m.urt.data(), m.urt.size() * sizeof(zc));
    if (exph0k && !m.exph0k.empty())
        for (int k = 0; k < lq; ++k) { exph0k[2 * k] = m.exph0k[k].real() * lq; exph0k[2 * k + 1] = m.exph0k[k].imag() * lq; }
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
struct ChainHost {
    int model;
    ChainDev dev;
    std::vector<zc> trial;           // projective path: trial eigenvectors (N x N)
    std::vector<double> trial_w;     // and eigenvalues
};

struct dqmc_handle {
    std::vector<HostModel*> models;
    std::vector<ChainHost> chains;
    ChainDev* d_chains = nullptr;
    int* d_slotmap = nullptr;
    int* d_slotmap_b = nullptr;      // push_stage copy of the slot map (ltau)
    int after_b0 = 0;                // the stack holds the left factors of a b0 sweep
    std::vector<void*> allocs;
    cudaStream_t st = nullptr;
    int nch = 0, maxN = 0, ltrot = 0, nst = 0, nwrap = 0, nnf_max = 0;
    int started = 0;
    cudaGraphExec_t sweep_graph = nullptr;
    int graph_meas = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int ctas_per_chain = 1;
    int max_lq = 0;           // largest number of unit cells over the models
    size_t graph_nodes = 0;
    int proj = 0;
    // recording of (HS field, nflr Re log weight) pairs at every stabilisation
    int rec_on = 0, rec_cap = 0, rec_V = 0;
    int8_t* rec_f = nullptr;
    double* rec_v = nullptr;
    int* rec_count = nullptr;
    // global block moves
    int blocks = 0;
    // register-resident FFT propagation (square l x l lattice, one site per
    // cell, l = 4, 8, 16, the same size in every parameter set), else 0
    int fft_L = 0, maxNe = 0;
    // per-launch timing of a sweep (dqmc_gpu_sweep_profile): an event after
    // every launch group, tagged with its kind
    int tm_on = 0, tm_n = 0;
    std::vector<cudaEvent_t> tm_ev;
    std::vector<int> tm_kind;
    int* d_org = nullptr;        // [nch][3]
    double* d_u = nullptr;       // [nch][2]
    double* d_S = nullptr;       // [nch][2]
    uint64_t blk_rng = 0x9e3779b97f4a7c15ULL;
    // numerical-failure reporting: the device word the kernels raise DQ_FAIL_*
    // codes into, the control words they read (wrap-error tolerance), and the
    // host-side re-stabilisation policy and count
    int* d_fail = nullptr;
    double* d_ctl = nullptr;
    int restab = 0;
    double n_restab = 0.0;
};

// Host <-> device copies of the entry points, ordered on the library's stream:
// the stream is non-blocking, so a plain cudaMemcpy on the legacy stream is not
// ordered with its kernels (a pageable host-to-device copy may still be in
// flight when the next kernel on the stream starts).
static cudaError_t copy_sync(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    return e != cudaSuccess ? e : e2;
}

static void* dalloc(dqmc_handle* h, size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
    if (h->st) {           // ordered with the library's (non-blocking) stream
        cudaMemsetAsync(p, 0, bytes ? bytes : 16, h->st);
        cudaStreamSynchronize(h->st);
    } else {
        cudaMemset(p, 0, bytes ? bytes : 16);   // creation ends with a device synchronisation
    }
    h->allocs.push_back(p);
    return p;
}

// frees one allocation made by dalloc (and forgets it)
static void dfree(dqmc_handle* h, void* p) {
    if (!p) return;
    for (size_t k = 0; k < h->allocs.size(); ++k)
        if (h->allocs[k] == p) { h->allocs.erase(h->allocs.begin() + k); break; }
    cudaFree(p);
}

// the captured sweep holds device pointers and sizes as kernel arguments: any
// change of them (record buffers) must drop it
static void drop_sweep_graph(dqmc_handle* h) {
    if (h->sweep_graph) { cudaGraphExecDestroy(h->sweep_graph); h->sweep_graph = nullptr; }
    h->graph_meas = -1;
}

extern "C" int dqmc_gpu_destroy(dqmc_handle* h) {
    if (!h) return DQMC_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->sweep_graph) cudaGraphExecDestroy(h->sweep_graph);
    for (void* p : h->allocs) cudaFree(p);
    for (HostModel* m : h->models) { for (void* p : m->allocs) cudaFree(p); delete m; }
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (cudaEvent_t e : h->tm_ev) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return DQMC_OK;
}

// projR = first ne trial vectors, projLc = their complex conjugate (UL^T of P^H)
static int upload_trial(dqmc_handle* h, int c) {
    ChainHost& ch = h->chains[c];
    const HostModel& m = *h->models[ch.model];
    int N = m.N, ne = m.p.ne;
    std::vector<zc> pr((size_t)N * ne), pl((size_t)N * ne);
    for (size_t e = 0; e < pr.size(); ++e) { pr[e] = ch.trial[e]; pl[e] = std::conj(ch.trial[e]); }
    CK(cudaMemcpy(ch.dev.projR, pr.data(), pr.size() * sizeof(zc), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ch.dev.projLc, pl.data(), pl.size() * sizeof(zc), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_create(const dqmc_params* params, int n_params, int n_chains, const int32_t* seeds,
                               int draw_conf, dqmc_handle** out) {
    if (!params || n_params < 1 || n_chains < 1 || !out) return fail(DQMC_EINVAL, "invalid arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(DQMC_ECUDA, "no CUDA device");
    dqmc_handle* h = new dqmc_handle();
    *out = nullptr;
    int rc;
    std::vector<int> model_of(n_params);
    for (int k = 0; k < n_params; ++k) {
        // identical parameter sets share one model (tables uploaded once)
        int same = -1;
        for (int q = 0; q < k && same < 0; ++q)
            if (memcmp(&params[q], &params[k], sizeof(dqmc_params)) == 0) same = model_of[q];
        if (same >= 0) { model_of[k] = same; continue; }
        model_of[k] = (int)h->models.size();
        HostModel* m = new HostModel();
        m->p = params[k];
        m->dense_on_device = true;
        if ((rc = dqmc_params_derive(&m->p))) { delete m; dqmc_gpu_destroy(h); return rc; }
        if ((rc = build_model(*m))) { delete m; dqmc_gpu_destroy(h); return rc; }
        h->models.push_back(m);
        if (h->models.size() == 1) { h->ltrot = m->p.ltrot; h->nst = m->p.nst; h->nwrap = m->p.nwrap; }
        else if (m->p.ltrot != h->ltrot || m->p.nst != h->nst || m->p.nwrap != h->nwrap) {
            dqmc_gpu_destroy(h);
            return fail(DQMC_EINVAL, "all parameter sets of a handle must share ltrot and nwrap");
        } else if (m->p.lattice != h->models[0]->p.lattice || m->p.kinetic != h->models[0]->p.kinetic ||
                   (m->p.rt == 0.0) != (h->models[0]->p.rt == 0.0) || (m->p.rhub == 0.0) != (h->models[0]->p.rhub == 0.0) ||
                   (m->p.rv == 0.0) != (h->models[0]->p.rv == 0.0) || (m->p.proj != 0) != (h->models[0]->p.proj != 0) ||
                   (m->p.ltau != 0) != (h->models[0]->p.ltau != 0)) {
            dqmc_gpu_destroy(h);
            return fail(DQMC_EINVAL, "all parameter sets of a handle must share lattice kind, kinetic propagator, "
                                     "the presence of the U / V / hopping terms, the projective flag and ltau");
        }
        if ((rc = upload_model(*m))) { dqmc_gpu_destroy(h); return rc; }
        h->maxN = std::max(h->maxN, m->N);
        h->nnf_max = std::max(h->nnf_max, m->nn_nf);
        h->maxNe = std::max(h->maxNe, m->p.ne);
        h->max_lq = std::max(h->max_lq, m->lq);
    }
    {
        const dqmc_params& p0 = h->models[0]->p;
        int L = p0.l1;
        bool ok = p0.kinetic == DQMC_KIN_FFT && p0.l1 == p0.l2 && (L == 4 || L == 8 || L == 16);
        for (HostModel* m : h->models) ok = ok && m->N == L * L && m->p.l1 == L && m->p.l2 == L;
        h->fft_L = ok ? L : 0;
    }
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { dqmc_gpu_destroy(h); return fail(DQMC_ECUDA, "stream"); }
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    h->nch = n_chains;
    h->d_fail = (int*)dalloc(h, 16);
    h->d_ctl = (double*)dalloc(h, 4 * sizeof(double));
    if (!h->d_fail || !h->d_ctl) { dqmc_gpu_destroy(h); return fail(DQMC_ENOMEM, "device allocation failed"); }
    int nst = h->nst, lt = h->ltrot;
    h->d_slotmap = (int*)dalloc(h, sizeof(int) * (nst + 2));
    if (h->models[0]->p.ltau) h->d_slotmap_b = (int*)dalloc(h, sizeof(int) * (nst + 2));
    {
        std::vector<int> sm(nst + 2);
        for (int i = 0; i < nst + 2; ++i) sm[i] = i;
        cudaMemcpy(h->d_slotmap, sm.data(), sizeof(int) * (nst + 2), cudaMemcpyHostToDevice);
    }
    h->chains.resize(n_chains);
    h->proj = h->models[0]->p.proj != 0;
    std::vector<std::vector<zc>> trial_H(n_chains);
    for (int c = 0; c < n_chains; ++c) {
        HostModel* m = h->models[model_of[c % n_params]];
        ChainHost& ch = h->chains[c];
        ch.model = model_of[c % n_params];
        ChainDev& d = ch.dev;
        memset(&d, 0, sizeof(d));
        int N = m->N;
        size_t NN = (size_t)N * N, z = sizeof(double2);
        d.md = m->d_dev;
        d.N = N;
        const bool proj = m->p.proj != 0;
        const int ne = m->p.ne, nnf = m->nn_nf;
        d.G = (double2*)dalloc(h, NN * z);
        d.Gnew = (double2*)dalloc(h, NN * z);
        d.GT = (double2*)dalloc(h, NN * z);
        for (int k = 0; k < 6; ++k) d.W[k] = (double2*)dalloc(h, NN * z);
        if (!proj) {
            d.U = (double2*)dalloc(h, (size_t)(nst + 2) * NN * z);
            d.V = (double2*)dalloc(h, (size_t)(nst + 2) * NN * z);
            d.D = (double*)dalloc(h, (size_t)(nst + 2) * N * sizeof(double));
            d.logdetQ = (double2*)dalloc(h, (size_t)(nst + 2) * z);
            d.A = (double2*)dalloc(h, (size_t)N * m->nublock_dev * z);
            d.B = (double2*)dalloc(h, (size_t)N * m->nublock_dev * z);
            if (m->p.ltau) {
                d.gt0 = (double2*)dalloc(h, NN * z);
                d.g0t = (double2*)dalloc(h, NN * z);
                d.g00 = (double2*)dalloc(h, NN * z);
                d.dynbins = (double2*)dalloc(h, (size_t)m->lq * 4 * (m->p.ntdm + 1) * z);
                d.Ub = (double2*)dalloc(h, (size_t)(nst + 2) * NN * z);
                d.Vb = (double2*)dalloc(h, (size_t)(nst + 2) * NN * z);
                d.Db = (double*)dalloc(h, (size_t)(nst + 2) * N * sizeof(double));
                d.ldqb = (double2*)dalloc(h, (size_t)(nst + 2) * z);
                d.Gb = (double2*)dalloc(h, NN * z);
            }
        } else {
            size_t Nne = (size_t)N * ne;
            d.UR = (double2*)dalloc(h, Nne * z);
            d.ULT = (double2*)dalloc(h, Nne * z);
            d.ULRINV = (double2*)dalloc(h, (size_t)ne * ne * z);
            d.Pst = (double2*)dalloc(h, (size_t)(nst + 1) * Nne * z);
            d.projR = (double2*)dalloc(h, Nne * z);
            d.projLc = (double2*)dalloc(h, Nne * z);
            d.logwDV = (double*)dalloc(h, (size_t)(nst + 2) * sizeof(double));
            if (m->p.ltau) {
                d.gt0 = (double2*)dalloc(h, NN * z);
                d.g0t = (double2*)dalloc(h, NN * z);
                d.g00 = (double2*)dalloc(h, NN * z);
                d.dynbins = (double2*)dalloc(h, (size_t)m->lq * 4 * (m->p.ntdm + 1) * z);
                d.URs = (double2*)dalloc(h, Nne * z);
                d.ULTs = (double2*)dalloc(h, Nne * z);
            }
            d.pw = (double2*)dalloc(h, ((size_t)5 * 32 * ne + 2 * 32 * 32) * z);
            d.pw_flag = (int*)dalloc(h, 16 * sizeof(int));
            if (!d.UR || !d.ULT || !d.ULRINV || !d.Pst || !d.projR || !d.projLc || !d.logwDV || !d.pw) {
                dqmc_gpu_destroy(h);
                return fail(DQMC_ENOMEM, "device allocation failed");
            }
        }
        if (m->p.rv != 0.0) d.vconf = (int32_t*)dalloc(h, (size_t)lt * nnf * N * sizeof(int32_t));
        d.tau = (double2*)dalloc(h, (size_t)N * z);
        d.T = (double2*)dalloc(h, (size_t)(N / 16 + 1) * 256 * z);
        d.T64 = (double2*)dalloc(h, (size_t)(N / 64 + 1) * 4096 * z);
        d.smallw = (double2*)dalloc(h, (size_t)128 * N * z);
        d.vecs = (double*)dalloc(h, (size_t)8 * N * sizeof(double));
        d.perm = (int*)dalloc(h, (size_t)N * sizeof(int));
        d.conf = (int32_t*)dalloc(h, (size_t)lt * N * sizeof(int32_t));
        if (m->plq_on) d.conf_plq = (int32_t*)dalloc(h, (size_t)lt * m->lq * sizeof(int32_t));
        d.sfmt = (uint32_t*)dalloc(h, 625 * sizeof(uint32_t));
        d.rnd = (uint32_t*)dalloc(h, (size_t)lt * std::max(2 * N, m->dev.rps) * sizeof(uint32_t));
        d.bins = (double2*)dalloc(h, (size_t)(10 + 20 * m->lq + 4) * z);
        d.stats = (double*)dalloc(h, ST_COUNT * sizeof(double));
        d.slotmap = h->d_slotmap;
        d.fail = h->d_fail;
        d.ctl = h->d_ctl;
        if (!d.G || !d.Gnew || !d.W[5] || (!proj && (!d.U || !d.V || !d.D)) || !d.rnd || !d.stats || !d.bins ||
            (m->p.rv != 0.0 && !d.vconf)) {
            dqmc_gpu_destroy(h);
            return fail(DQMC_ENOMEM, "device allocation failed");
        }
        // generator state and fresh-start fields, drawn in the reference's order
        HostSfmt rng;
        sfmt_seed(rng.st, seeds ? seeds[c] : 0);
        std::vector<int32_t> conf, vconf, conf_plq;
        draw_fields(*m, rng, draw_conf, conf, vconf, &conf_plq);
        if (proj) {
            trial_hamiltonian(*m, rng, trial_H[c]);
        }
        cudaMemcpy(d.sfmt, rng.st, 625 * sizeof(uint32_t), cudaMemcpyHostToDevice);
        cudaMemcpy(d.conf, conf.data(), conf.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (!vconf.empty()) cudaMemcpy(d.vconf, vconf.data(), vconf.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (m->plq_on) {
            if (!d.conf_plq) { dqmc_gpu_destroy(h); return fail(DQMC_ENOMEM, "device allocation failed"); }
            cudaMemcpy(d.conf_plq, conf_plq.data(), conf_plq.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        }
        double stats[ST_COUNT] = {0};
        stats[ST_PHASE_RE] = 1.0;
        cudaMemcpy(d.stats, stats, sizeof(stats), cudaMemcpyHostToDevice);
    }
    if (h->proj) {
        // eigenvectors of every walker's trial Hamiltonian (set_trial_h0): one
        // batched device eigensolve per lattice size
        std::vector<std::vector<double>> ws(n_chains);
        std::vector<int> sizes;
        for (int c = 0; c < n_chains; ++c)
            if (std::find(sizes.begin(), sizes.end(), h->chains[c].dev.N) == sizes.end()) sizes.push_back(h->chains[c].dev.N);
        for (int Nb : sizes) {
            std::vector<int> cs;
            for (int c = 0; c < n_chains; ++c) if (h->chains[c].dev.N == Nb) cs.push_back(c);
            const size_t nn = (size_t)Nb * Nb;
            std::vector<double2> Hb(nn * cs.size()), Vb(nn * cs.size());
            std::vector<double> wb((size_t)Nb * cs.size());
            for (size_t q = 0; q < cs.size(); ++q)
                memcpy(&Hb[q * nn], trial_H[cs[q]].data(), nn * sizeof(double2));
            const int sw = eig_herm_device(Hb.data(), Nb, (int)cs.size(), Vb.data(), wb.data(), h->st);
            if (sw < 0) {
                dqmc_gpu_destroy(h);
                return sw == -2 ? fail(DQMC_ENUMERIC, "the trial-state eigensolver did not converge")
                                : fail(DQMC_ECUDA, "device eigensolver of the trial states failed");
            }
            for (size_t q = 0; q < cs.size(); ++q) {
                memcpy(trial_H[cs[q]].data(), &Vb[q * nn], nn * sizeof(double2));
                ws[cs[q]].assign(wb.begin() + q * Nb, wb.begin() + (q + 1) * Nb);
            }
        }
        for (int c = 0; c < n_chains; ++c) {
            h->chains[c].trial = std::move(trial_H[c]);
            h->chains[c].trial_w = std::move(ws[c]);
            int rc2 = upload_trial(h, c);
            if (rc2) { dqmc_gpu_destroy(h); return rc2; }
        }
    }
    h->d_chains = (ChainDev*)dalloc(h, sizeof(ChainDev) * n_chains);
    {
        std::vector<ChainDev> v(n_chains);
        for (int c = 0; c < n_chains; ++c) v[c] = h->chains[c].dev;
        cudaMemcpy(h->d_chains, v.data(), sizeof(ChainDev) * n_chains, cudaMemcpyHostToDevice);
    }
    set_stab_maxN(h->maxN);
    if (h->proj) set_proj_maxN(h->maxN);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    h->ctas_per_chain = std::max(1, std::min(h->maxN / 16, (2 * sms + n_chains - 1) / n_chains));
    CK(cudaDeviceSynchronize());
    CK(cudaGetLastError());
    *out = h;
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// sweep profiling: an event after each launch group while tm_on is set (never
// during graph capture); the interval since the previous event is charged to
// the group's kind (DQMC_PROF_*)
// ---------------------------------------------------------------------------
static void tmark(dqmc_handle* h, int kind) {
    if (!h->tm_on) return;
    if (h->tm_n >= (int)h->tm_ev.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) { h->tm_on = 0; return; }
        h->tm_ev.push_back(e);
        h->tm_kind.push_back(0);
    }
    cudaEventRecord(h->tm_ev[h->tm_n], h->st);
    h->tm_kind[h->tm_n] = kind;
    ++h->tm_n;
}

// ---------------------------------------------------------------------------
// propagation programs
// ---------------------------------------------------------------------------
static void prog_add(PropProg& p, int kind, int which, int nf, int nt) {
    if (p.n < DQ_MAX_PROG) p.op[p.n++] = kind | (which << 4) | (nf << 8) | (nt << 16);
}

// kinetic half step, families 1..nnf (reversed = nnf..1); `which` urt/urtm1
static void prog_k(const HostModel& m, PropProg& p, int which, int reversed) {
    if (m.p.rt == 0.0) return;
    if (m.p.kinetic == DQMC_KIN_FFT) { prog_add(p, PK_FFT, which, 0, 0); return; }
    if (m.p.kinetic == DQMC_KIN_DENSE) { prog_add(p, PK_DENSE, which, 0, 0); return; }
    for (int k = 1; k <= m.nn_nf; ++k) prog_add(p, PK_CB, which == PW_CONJ ? PW_FWD : which, reversed ? m.nn_nf + 1 - k : k, 0);
}
static void prog_v(const HostModel& m, PropProg& p, int which, int nt) {
    if (m.p.rhub == 0.0) return;
    prog_add(p, PK_DIAG, which, 0, nt);
}
// the bond field of slice nt in a B product (left_forward, which = PW_FWD) or
// B^-1 from the right (right_backward, PW_INV): per family the nflag = 2 step
// (mix, scale) then nflag = 1 (mix); families 1..nn_nf, or nn_nf..1 when desc
// (src/dqmc_ft_core.f90:98-104, 150-156, 264-270)
static void prog_bond(const HostModel& m, PropProg& p, int which, int nt, int desc) {
    if (m.p.rv == 0.0) return;
    for (int k = 1; k <= m.nn_nf; ++k) {
        const int nf = desc ? m.nn_nf + 1 - k : k;
        prog_add(p, PK_VMIX, 0, nf, nt);
        prog_add(p, PK_VSCALE, which, nf, nt);
        prog_add(p, PK_VMIX, 0, nf, nt);
    }
}

// all chains share structure; programs are built from model 0 (same nn_nf
// per handle for a given lattice kind)
static int launch_prog(dqmc_handle* h, int mat_id, const PropProg& prog, int right) {
    if (prog.n == 0) return DQMC_OK;
    if (h->fft_L && prop_fft_eligible(prog)) {
        launch_prop_fft(h->d_chains, h->nch, h->fft_L, h->maxN, mat_id, prog, right, right, 0, h->st);
        return DQMC_OK;
    }
    // dense kinetic steps are GEMMs of their own; the element-wise ops between
    // them run as one propagation kernel per stretch
    PropProg seg; seg.n = 0;
    for (int k = 0; k <= prog.n; ++k) {
        const bool dense = k < prog.n && (prog.op[k] & 15) == PK_DENSE;
        if (k == prog.n || dense) {
            if (seg.n) launch_prop(h->d_chains, h->nch, h->maxN, mat_id, seg, right, h->ctas_per_chain, h->st);
            seg.n = 0;
            if (dense) launch_kin_dense(h->d_chains, h->nch, h->maxN, mat_id, (prog.op[k] >> 4) & 15, right, 0, h->st);
        } else {
            seg.op[seg.n++] = prog.op[k];
        }
    }
    return DQMC_OK;
}

// B(nt1, nt2) from the left (Bmat_left_forward, src/dqmc_ft_core.f90:70-121) or
// B(nt1, nt2)^H (Bmat_left_forward_hc, 123-175) applied to matrix mat_id.  The
// slices are collected into programs of at most DQ_MAX_PROG ops, each launched
// when the next slice would not fit, so any nwrap is applied in full (a
// checkerboard slice is 2 nn_nf + 1 ops).  Splitting a program only stores and
// reloads the vectors between two ops, so the result does not depend on it.
static int launch_bmat(dqmc_handle* h, int mat_id, int nt1, int nt2, int hc) {
    const HostModel& m = *h->models[0];
    PropProg p; p.n = 0;
    for (int s = 0; s <= nt1 - nt2; ++s) {
        const int nt = hc ? nt1 - s : nt2 + s;
        const int which = hc ? PW_CONJ : PW_FWD;
        PropProg sl; sl.n = 0;
        prog_k(m, sl, which, 0);
        // plaquettes ascending before the U field (Bmat_left_forward), descending
        // after it with bmat^H = bmat_inv (Bmat_left_forward_hc)
        if (m.plq_on && !hc) prog_add(sl, PK_PLQ, PW_FWD, 0, nt);
        if (!hc) prog_bond(m, sl, PW_FWD, nt, 0);
        prog_v(m, sl, which, nt);
        // the bond field in B^H: families nn_nf..1 with the same steps and
        // values as in B (dqmc_left_forward_prop_hc.f90 equals
        // dqmc_left_forward_prop.f90)
        if (hc) prog_bond(m, sl, PW_FWD, nt, 1);
        if (m.plq_on && hc) prog_add(sl, PK_PLQ, PW_INV, 1, nt);
        prog_k(m, sl, which, 1);
        if (p.n + sl.n > DQ_MAX_PROG) {
            int rc = launch_prog(h, mat_id, p, 0); if (rc) return rc;
            p.n = 0;
        }
        for (int k = 0; k < sl.n; ++k) p.op[p.n++] = sl.op[k];
    }
    return launch_prog(h, mat_id, p, 0);
}

enum { MAT_G = 0, MAT_GT0 = 15, MAT_G0T = 16, MAT_U = 100, MAT_V = 400 };   // ids of chain_access.cuh

// one projective update call (a bond family, or the site field when nf = 0):
// window count and per-walker CTA counts of the window GEMMs, maximised over
// the handle's models
static void proj_update(dqmc_handle* h, int nt, int nf, int visit, int dir, int rnd_off) {
    int nwin = 0, grg = 1, gfl = 1;
    for (const HostModel* m : h->models) {
        int b = nf > 0 ? 2 : 1;
        int units = nf > 0 ? m->nn_lf : m->N;
        int R = std::min(m->nublock_dev, 32);
        R -= R % b;
        if (R < b) R = b;
        int upw = R / b, ne = m->p.ne;
        nwin = std::max(nwin, (units + upw - 1) / upw);
        int nr = std::min(R, units * b);
        int t1 = zt_tiles(zt_pick(nr, ne), nr, ne) + zt_tiles(zt_pick(ne, nr), ne, nr);
        int t3 = zt_tiles(zt_pick(ne, ne), ne, ne);
        grg = std::max(grg, std::min(t1, 16));
        gfl = std::max(gfl, std::min(t3, 16));
    }
    launch_proj_update(h->d_chains, h->nch, nt, nf, visit, dir, rnd_off, nwin, grg, gfl, h->st);
}

// one stabilisation of the 0b sweep at stack index n: new factor into the spare
// slot, Green's function from (new R, old L), wrap check, then swap slots.
static void maybe_record(dqmc_handle* h) {
    if (h->rec_on) launch_record(h->d_chains, h->nch, h->rec_f, h->rec_v, h->rec_count, h->rec_cap, h->rec_V, h->st);
}

static void stab_0b(dqmc_handle* h, int n, int record) {
    const HostModel& m = *h->models[0];
    int spare = h->nst + 1;
    launch_copy_mat(h->d_chains, h->nch, 2 /*W0*/, MAT_U + (n - 1), 0, h->st);
    tmark(h, DQMC_PROF_OTHER);
    launch_bmat(h, 2, m.wrap_step[(n - 1) * 2 + 1], m.wrap_step[(n - 1) * 2], 0);
    tmark(h, DQMC_PROF_BPROD);
    launch_stab_slots(h->d_chains, h->nch, n - 1, spare, h->st);
    tmark(h, DQMC_PROF_STAB);
    launch_green(h->d_chains, h->nch, spare, n, 0, 0, 0, 0, 0, h->st);
    tmark(h, DQMC_PROF_GREEN);
    launch_wrap_check(h->d_chains, h->nch, record, h->st);
    launch_swap_slots(h->d_slotmap, n, spare, h->st);
    maybe_record(h);
    tmark(h, DQMC_PROF_OTHER);
}

// one stabilisation of the b0 sweep at stack index n (stablize_b0(n+1))
static void stab_b0(dqmc_handle* h, int n) {
    const HostModel& m = *h->models[0];
    int spare = h->nst + 1;
    launch_copy_mat(h->d_chains, h->nch, 2, MAT_U + (n + 1), 0, h->st);
    tmark(h, DQMC_PROF_OTHER);
    launch_bmat(h, 2, m.wrap_step[n * 2 + 1], m.wrap_step[n * 2], 1);
    tmark(h, DQMC_PROF_BPROD);
    launch_stab_slots(h->d_chains, h->nch, n + 1, spare, h->st);
    tmark(h, DQMC_PROF_STAB);
    launch_green(h->d_chains, h->nch, n, spare, 0, 0, 0, 0, 0, h->st);
    tmark(h, DQMC_PROF_GREEN);
    launch_wrap_check(h->d_chains, h->nch, 1, h->st);
    launch_swap_slots(h->d_slotmap, n, spare, h->st);
    maybe_record(h);
    tmark(h, DQMC_PROF_OTHER);
}

// ---------------------------------------------------------------------------
// projective path (src/dqmc_proj_core/): pending propagation ops of UR (left
// multiplications) and UL^T (right multiplications) are collected and run as
// one pass each whenever an update, a measurement or a stabilisation needs
// the current matrices.
// ---------------------------------------------------------------------------
enum { PMAT_W3 = 5, PMAT_UR = 10, PMAT_ULT = 11, PMAT_PROJR = 12, PMAT_PROJLC = 13, PMAT_ULRINV = 14,
       PMAT_URS = 18, PMAT_ULTS = 19, PMAT_PST0 = 1000, PMAT_G = 0, PMAT_GNEW = 1 };

struct ProjPass {
    PropProg r, l;   // r: ops on UR (left), l: ops on UL^T (right)
    ProjPass() { r.n = 0; l.n = 0; }
};

static void pflush(dqmc_handle* h, ProjPass& pp) {
    for (int side = 0; side < 2; ++side) {
        const PropProg& pr = side ? pp.l : pp.r;
        const int mat = side ? PMAT_ULT : PMAT_UR;
        if (!pr.n) continue;
        if (h->fft_L && prop_fft_eligible(pr)) {
            launch_prop_fft(h->d_chains, h->nch, h->fft_L, h->maxNe, mat, pr, 0, side, 1, h->st);
        } else {
            PropProg seg; seg.n = 0;
            for (int k = 0; k <= pr.n; ++k) {
                const bool dense = k < pr.n && (pr.op[k] & 15) == PK_DENSE;
                if (k == pr.n || dense) {
                    if (seg.n) launch_prop_tall(h->d_chains, h->nch, h->maxN, mat, seg, side, h->ctas_per_chain, h->st);
                    seg.n = 0;
                    if (dense) launch_kin_dense(h->d_chains, h->nch, h->maxN, mat, (pr.op[k] >> 4) & 15, side, 1, h->st);
                } else {
                    seg.op[seg.n++] = pr.op[k];
                }
            }
        }
        tmark(h, side ? DQMC_PROF_PROP_R : DQMC_PROF_PROP_L);
    }
    pp.r.n = 0; pp.l.n = 0;
}
static void padd(dqmc_handle* h, ProjPass& pp, PropProg& p, int kind, int which, int nf, int nt) {
    if (p.n >= DQ_MAX_PROG) pflush(h, pp);
    prog_add(p, kind, which, nf, nt);
}
// kinetic half step: families 1..nnf (or reversed) with urt (which = PW_FWD) or urtm1
static void pk(dqmc_handle* h, ProjPass& pp, PropProg& p, int which, int reversed) {
    const HostModel& m = *h->models[0];
    if (m.p.rt == 0.0) return;
    if (m.p.kinetic == DQMC_KIN_FFT) { padd(h, pp, p, PK_FFT, which, 0, 0); return; }
    if (m.p.kinetic == DQMC_KIN_DENSE) { padd(h, pp, p, PK_DENSE, which, 0, 0); return; }
    for (int k = 1; k <= m.nn_nf; ++k) padd(h, pp, p, PK_CB, which, reversed ? m.nn_nf + 1 - k : k, 0);
}

static bool proj_mid(const HostModel& m, int nt) {
    int lt = m.p.ltrot, len = m.p.obs_mid_len;
    return nt > (lt / 2 - (len + 1) / 2) && nt <= (lt / 2 + len / 2);
}

// equal-time measurement of the current G (equaltime_measure)
static void launch_measure_h(dqmc_handle* h) {
    const int lat = h->models[0]->p.lattice;
    const int kind = lat == DQMC_LATT_CUBIC ? MEAS_CUBIC : lat == DQMC_LATT_R_CUBIC ? MEAS_R_CUBIC
                   : h->models[0]->nsub == 2 ? MEAS_HONEYCOMB : MEAS_ONE_ORBITAL;
    launch_measure(h->d_chains, h->nch, h->maxN, kind, h->max_lq, h->st);
}

// ULRINV = (UL UR)^-1 fresh, G = I - UR ULRINV UL, equaltime_measure
static void proj_measure(dqmc_handle* h) {
    launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 0, 0, -1, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_G, h->ctas_per_chain, h->st);
    tmark(h, DQMC_PROF_GREEN);
    launch_measure_h(h);
    tmark(h, DQMC_PROF_MEASURE);
}

// G of the current (UL, UR) into G, before a stabilisation replaces them
static void proj_old_green(dqmc_handle* h) {
    launch_proj_ulr(h->d_chains, h->nch, PMAT_W3, 0, 0, -1, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_W3, PMAT_G, h->ctas_per_chain, h->st);
    tmark(h, DQMC_PROF_GREEN);
}

// dqmc_proj_sweep_0b.f90:133-190 at wrap point n
static void stab_proj_0b(dqmc_handle* h, int n) {
    int nst = h->nst;
    proj_old_green(h);
    launch_tall_copy(h->d_chains, h->nch, PMAT_ULT, PMAT_PST0 + n, h->st);
    tmark(h, DQMC_PROF_OTHER);
    launch_proj_qr(h->d_chains, h->nch, PMAT_UR, n, n - 1, h->st);
    tmark(h, DQMC_PROF_STAB);
    launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 1, n, n == nst ? -1 : n + 1, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_GNEW, h->ctas_per_chain, h->st);
    tmark(h, DQMC_PROF_GREEN);
    launch_wrap_check(h->d_chains, h->nch, 1, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + n, PMAT_UR, h->st);
    tmark(h, DQMC_PROF_OTHER);
}

// dqmc_proj_sweep_b0.f90:128-190 at wrap point n
static void stab_proj_b0(dqmc_handle* h, int n) {
    int nst = h->nst;
    proj_old_green(h);
    launch_tall_copy(h->d_chains, h->nch, PMAT_UR, PMAT_PST0 + n, h->st);
    tmark(h, DQMC_PROF_OTHER);
    launch_proj_qr(h->d_chains, h->nch, PMAT_ULT, n + 1, (n + 1 == nst) ? -1 : n + 2, h->st);
    tmark(h, DQMC_PROF_STAB);
    launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 1, n + 1, n == 0 ? -1 : n, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_GNEW, h->ctas_per_chain, h->st);
    tmark(h, DQMC_PROF_GREEN);
    launch_wrap_check(h->d_chains, h->nch, 1, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + n, PMAT_ULT, h->st);
    tmark(h, DQMC_PROF_OTHER);
}

// Bmat_left_forward on UR over slices nt2..nt1 (src/dqmc_proj_core.f90:61-104)
static void proj_bmat(dqmc_handle* h, ProjPass& pp, int nt1, int nt2) {
    const HostModel& m = *h->models[0];
    for (int nt = nt2; nt <= nt1; ++nt) {
        pk(h, pp, pp.r, PW_FWD, 0);
        if (m.plq_on) padd(h, pp, pp.r, PK_PLQ, PW_FWD, 0, nt);     // dqmc_proj_core.f90:89-94
        if (m.p.rv != 0.0)
            for (int nf = 1; nf <= m.nn_nf; ++nf) {
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);
                padd(h, pp, pp.r, PK_VSCALE, PW_FWD, nf, nt);
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);
            }
        if (m.p.rhub != 0.0) padd(h, pp, pp.r, PK_DIAG, PW_FWD, 0, nt);
        pk(h, pp, pp.r, PW_FWD, 1);
    }
}

// dqmc_proj_sweep_start_0b (src/dqmc_proj_core/dqmc_proj_sweep_start_0b.f90:1-48)
static int proj_sweep_start(dqmc_handle* h, int sync) {
    const HostModel& m = *h->models[0];
    int nst = h->nst;
    launch_tall_copy(h->d_chains, h->nch, PMAT_UR, PMAT_PROJR, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + nst, PMAT_PROJLC, h->st);
    for (int n = 1; n <= nst; ++n) {
        ProjPass pp;
        proj_bmat(h, pp, m.wrap_step[(n - 1) * 2 + 1], m.wrap_step[(n - 1) * 2]);
        pflush(h, pp);
        launch_proj_qr(h->d_chains, h->nch, PMAT_UR, n, n - 1, h->st);
        launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + n, PMAT_UR, h->st);
    }
    launch_tall_copy(h->d_chains, h->nch, PMAT_ULT, PMAT_PROJLC, h->st);
    launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 1, nst, -1, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_GNEW, h->ctas_per_chain, h->st);
    launch_wrap_check(h->d_chains, h->nch, 0, h->st);
    if (sync) {
        CK(cudaStreamSynchronize(h->st));
        CK(cudaGetLastError());
    }
    h->started = 1;
    return DQMC_OK;
}

// dqmc_proj_sweep_b0 (src/dqmc_proj_core/dqmc_proj_sweep_b0.f90:1-220)
static void enqueue_proj_b0(dqmc_handle* h, int lupdate, int lmeasure) {
    const HostModel& m = *h->models[0];
    int lt = h->ltrot, nnf = m.nn_nf;
    bool lu = m.p.rhub != 0.0, lv = m.p.rv != 0.0;
    launch_tall_copy(h->d_chains, h->nch, PMAT_ULT, PMAT_PROJLC, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + 0, PMAT_PROJR, h->st);
    if (lupdate && (lu || lv || m.plq_on)) launch_sfmt(h->d_chains, h->nch, lt, h->st);
    tmark(h, DQMC_PROF_OTHER);
    ProjPass pp;
    for (int nt = lt; nt >= 1; --nt) {
        int visit = lt - nt;
        if (lmeasure && proj_mid(m, nt)) { pflush(h, pp); proj_measure(h); }
        pk(h, pp, pp.r, PW_INV, 0);     // h0 left_backward on UR
        pk(h, pp, pp.l, PW_FWD, 0);     // h0 right_forward on UL
        if (lu) {
            if (lupdate) { pflush(h, pp); proj_update(h, nt, 0, visit, 1, -1); tmark(h, DQMC_PROF_UPDATE); }
            padd(h, pp, pp.l, PK_DIAG, PW_FWD, 0, nt);
            padd(h, pp, pp.r, PK_DIAG, PW_INV, 0, nt);
        }
        if (lv)
            for (int nf = nnf; nf >= 1; --nf) {
                padd(h, pp, pp.l, PK_VMIX, 0, nf, nt);           // right_forward, nflag 2
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);           // left_backward, nflag 2
                if (lupdate) { pflush(h, pp); proj_update(h, nt, nf, visit, 1, -1); tmark(h, DQMC_PROF_UPDATE); }
                padd(h, pp, pp.l, PK_VSCALE, PW_FWD, nf, nt);    // right_forward, nflag 1
                padd(h, pp, pp.l, PK_VMIX, 0, nf, nt);
                padd(h, pp, pp.r, PK_VSCALE, PW_INV, nf, nt);    // left_backward, nflag 1
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);
            }
        if (m.plq_on) {                 // plaquettes: update, then props, descending
            pflush(h, pp);
            launch_plq_proj_slice(h->d_chains, h->nch, h->maxNe, nt, visit, 1, lupdate, h->st);
            tmark(h, DQMC_PROF_UPDATE);
        }
        pk(h, pp, pp.r, PW_INV, 1);
        pk(h, pp, pp.l, PW_FWD, 1);
        if ((m.iwrap_nt[nt - 1] > 0 || m.p.nwrap == 1) || nt == 1) { pflush(h, pp); stab_proj_b0(h, m.iwrap_nt[nt - 1]); }
    }
    pflush(h, pp);
}

// Bmat_left_forward (left = 1) or Bmat_right_backward (left = 0) over slice nt on
// an N x N matrix (src/dqmc_ft_core.f90:70-121, 234-288), with the projective
// runs' bond field: per family nflag 2 (mix, scale) then nflag 1 (mix)
static PropProg prog_bslice_proj(const HostModel& m, int nt, int left) {
    PropProg p; p.n = 0;
    const int which = left ? PW_FWD : PW_INV;
    prog_k(m, p, which, 0);
    if (m.plq_on) prog_add(p, PK_PLQ, which, 0, nt);      // plaquettes ascending (dqmc_proj_core.f90:89-94, 255-260)
    if (m.p.rv != 0.0)
        for (int nf = 1; nf <= m.nn_nf; ++nf) {
            prog_add(p, PK_VMIX, 0, nf, nt);
            prog_add(p, PK_VSCALE, which, nf, nt);
            prog_add(p, PK_VMIX, 0, nf, nt);
        }
    prog_v(m, p, which, nt);
    prog_k(m, p, which, 1);
    return p;
}

// dqmc_proj_dyn (src/dqmc_proj_core/dqmc_proj_dyn.f90:1-128), run by the measured
// 0b sweep at nt = ntauin (dqmc_proj_sweep_0b.f90:206-211) on copies of UL and
// UR: the sweep's UR and UL^T are set aside and restored afterwards, the
// stack slots beyond ntauin still hold the b0 sweep's UL^T.  G(t,t) is
// propagated in G and recomputed from (UL, UR) at the stabilisation points
// (max deviation into xmax_dyn), G(t,0) = G gt0 and G(0,t) = g0t (1 - G) there,
// and dyn_measure runs at every time index.  The reference assumes that ntauin
// is a stabilisation point; G is computed fresh at ntauin in either case.
static void proj_dyn(dqmc_handle* h) {
    const HostModel& m = *h->models[0];
    const int ntdm = m.p.ntdm, t0 = (m.p.ltrot - ntdm) / 2;
    launch_tall_copy(h->d_chains, h->nch, PMAT_URS, PMAT_UR, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_ULTS, PMAT_ULT, h->st);
    for (int nt = t0; nt <= t0 + ntdm - 1; ++nt) {
        const int ntau = nt - t0;
        if (m.iwrap_nt[nt] > 0 || ntau == 0) {
            if (ntau > 0) launch_tall_copy(h->d_chains, h->nch, PMAT_ULT, PMAT_PST0 + m.iwrap_nt[nt], h->st);
            launch_proj_ulr(h->d_chains, h->nch, PMAT_W3, 0, 0, -1, h->st);
            if (ntau == 0) {
                launch_proj_green(h->d_chains, h->nch, PMAT_W3, PMAT_G, h->ctas_per_chain, h->st);
                launch_dyn_init(h->d_chains, h->nch, h->st);
                launch_dyn_measure(h->d_chains, h->nch, h->maxN, 1, h->st);
            } else {
                launch_proj_green(h->d_chains, h->nch, PMAT_W3, PMAT_GNEW, h->ctas_per_chain, h->st);
                launch_chain_gemm(h->d_chains, h->nch, h->maxN, MAT_GT0, PMAT_GNEW, MAT_GT0, 0, h->st);
                launch_chain_gemm(h->d_chains, h->nch, h->maxN, MAT_G0T, MAT_G0T, PMAT_GNEW, 1, h->st);
                launch_dyn_err(h->d_chains, h->nch, h->st);
            }
        }
        const int nt1 = nt + 1;
        const PropProg pl = prog_bslice_proj(m, nt1, 1), pr = prog_bslice_proj(m, nt1, 0);
        launch_prog(h, MAT_GT0, pl, 0);
        launch_prog(h, MAT_G0T, pr, 1);
        launch_prog(h, MAT_G, pr, 1);
        launch_prog(h, MAT_G, pl, 0);
        launch_dyn_measure(h->d_chains, h->nch, h->maxN, nt1 - t0 + 1, h->st);
        ProjPass pp;
        proj_bmat(h, pp, nt1, nt1);
        pflush(h, pp);
        if (m.iwrap_nt[nt] > 0 && nt1 != t0 + ntdm) launch_proj_qr(h->d_chains, h->nch, PMAT_UR, -1, -1, h->st);
    }
    launch_tall_copy(h->d_chains, h->nch, PMAT_UR, PMAT_URS, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_ULT, PMAT_ULTS, h->st);
    tmark(h, DQMC_PROF_MEASURE);
}

// dqmc_proj_sweep_0b (src/dqmc_proj_core/dqmc_proj_sweep_0b.f90:1-235); with
// ltau the measured sweep runs the unequal-time pass at nt = ntauin (206-211)
static void enqueue_proj_0b(dqmc_handle* h, int lupdate, int lmeasure) {
    const HostModel& m = *h->models[0];
    int lt = h->ltrot, nnf = m.nn_nf, nst = h->nst;
    bool lu = m.p.rhub != 0.0, lv = m.p.rv != 0.0;
    launch_tall_copy(h->d_chains, h->nch, PMAT_UR, PMAT_PROJR, h->st);
    launch_tall_copy(h->d_chains, h->nch, PMAT_PST0 + nst, PMAT_PROJLC, h->st);
    if (lupdate && (lu || lv || m.plq_on)) launch_sfmt(h->d_chains, h->nch, lt, h->st);
    tmark(h, DQMC_PROF_OTHER);
    ProjPass pp;
    for (int nt = 1; nt <= lt; ++nt) {
        int visit = nt - 1;
        pk(h, pp, pp.r, PW_FWD, 0);     // h0 left_forward on UR
        pk(h, pp, pp.l, PW_INV, 0);     // h0 right_backward on UL
        if (m.plq_on) {                 // plaquettes: props, then update, ascending
            pflush(h, pp);
            launch_plq_proj_slice(h->d_chains, h->nch, h->maxNe, nt, visit, 0, lupdate, h->st);
            tmark(h, DQMC_PROF_UPDATE);
        }
        if (lv)
            for (int nf = 1; nf <= nnf; ++nf) {
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);           // left_forward, nflag 2
                padd(h, pp, pp.r, PK_VSCALE, PW_FWD, nf, nt);
                padd(h, pp, pp.l, PK_VMIX, 0, nf, nt);           // right_backward, nflag 2
                padd(h, pp, pp.l, PK_VSCALE, PW_INV, nf, nt);
                if (lupdate) { pflush(h, pp); proj_update(h, nt, nf, visit, 0, -1); tmark(h, DQMC_PROF_UPDATE); }
                padd(h, pp, pp.r, PK_VMIX, 0, nf, nt);           // nflag 1
                padd(h, pp, pp.l, PK_VMIX, 0, nf, nt);
            }
        if (lu) {
            padd(h, pp, pp.r, PK_DIAG, PW_FWD, 0, nt);
            padd(h, pp, pp.l, PK_DIAG, PW_INV, 0, nt);
            if (lupdate) { pflush(h, pp); proj_update(h, nt, 0, visit, 0, -1); tmark(h, DQMC_PROF_UPDATE); }
        }
        pk(h, pp, pp.r, PW_FWD, 1);
        pk(h, pp, pp.l, PW_INV, 1);
        if (lmeasure && proj_mid(m, nt)) { pflush(h, pp); proj_measure(h); }
        if (m.iwrap_nt[nt] > 0) { pflush(h, pp); stab_proj_0b(h, m.iwrap_nt[nt]); }
        if (lmeasure && m.p.ltau && nt == (lt - m.p.ntdm) / 2) { pflush(h, pp); proj_dyn(h); }
    }
    pflush(h, pp);
}

// sync = 0: enqueue only (the caller synchronises the handle's stream)
static int sweep_start_impl(dqmc_handle* h, int sync = 1) {
    h->after_b0 = 0;
    if (h->proj) return proj_sweep_start(h, sync);
    const HostModel& m = *h->models[0];
    {
        std::vector<int> sm(h->nst + 2);
        for (int i = 0; i < h->nst + 2; ++i) sm[i] = i;
        CK(cudaMemcpyAsync(h->d_slotmap, sm.data(), sizeof(int) * sm.size(), cudaMemcpyHostToDevice, h->st));
    }
    launch_stack_identity(h->d_chains, h->nch, 0, h->st);
    for (int n = 1; n <= h->nst; ++n) {
        launch_copy_mat(h->d_chains, h->nch, 2, MAT_U + (n - 1), 0, h->st);
        launch_bmat(h, 2, m.wrap_step[(n - 1) * 2 + 1], m.wrap_step[(n - 1) * 2], 0);
        launch_stab_slots(h->d_chains, h->nch, n - 1, n, h->st);
    }
    launch_green(h->d_chains, h->nch, h->nst, 0, 0, 0, 0, 0, 1, h->st);
    launch_wrap_check(h->d_chains, h->nch, 0, h->st);
    if (sync) {
        CK(cudaStreamSynchronize(h->st));
        CK(cudaGetLastError());
    }
    h->started = 1;
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// numerical-failure status.  The kernels raise DQ_FAIL_* codes into the
// handle's fail word (and each chain's stats[ST_INFO]); every sweep entry point
// clears the word before its launches and reads it after them.  The reference
// stops the run at these points (lib/s_matrix.f90:1264-1267,
// src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:188-194); the library returns
// DQMC_ENUMERIC (singular or non-finite Green's function) or DQMC_EWRAP (wrap
// error above the caller's tolerance) instead, or, with re-stabilisation on,
// rebuilds the UDV stack and G of every chain from its HS field
// (dqmc_ft_sweep_start_0b / dqmc_proj_sweep_start_0b) and goes on.
// ---------------------------------------------------------------------------
static void clear_fail(dqmc_handle* h) { cudaMemsetAsync(h->d_fail, 0, sizeof(int), h->st); }

static int report_fail(dqmc_handle* h, int f) {
    std::string msg = (f & (DQ_FAIL_SINGULAR | DQ_FAIL_NONFINITE))
                          ? "numerical failure (singular or non-finite Green's function)"
                          : "wrap error above the tolerance";
    msg += ", code " + std::to_string(f) + "; chains:";
    int listed = 0;
    for (int c = 0; c < h->nch && listed < 16; ++c) {
        double info = 0.0;
        if (copy_sync(h->st, &info, h->chains[c].dev.stats + ST_INFO, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            break;
        if (info != 0.0) { msg += " " + std::to_string(c) + " (" + std::to_string((int)info) + ")"; ++listed; }
    }
    return fail((f & (DQ_FAIL_SINGULAR | DQ_FAIL_NONFINITE)) ? DQMC_ENUMERIC : DQMC_EWRAP, msg);
}

// end of a sweep entry point: wait, then read the fail word.  at_beta: the
// call left the chains at tau = beta with the stack of a 0b sweep, the state
// sweep_start rebuilds, so re-stabilisation applies.
static int finish_checked(dqmc_handle* h, int at_beta) {
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    int f = 0;
    CK(copy_sync(h->st, &f, h->d_fail, sizeof(int), cudaMemcpyDeviceToHost));
    if (!f) return DQMC_OK;
    if (h->restab && at_beta) {
        clear_fail(h);
        int rc = sweep_start_impl(h); if (rc) return rc;
        h->n_restab += 1.0;
        CK(copy_sync(h->st, &f, h->d_fail, sizeof(int), cudaMemcpyDeviceToHost));
        if (!f) return DQMC_OK;
    }
    return report_fail(h, f);
}

extern "C" int dqmc_gpu_sweep_start(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    clear_fail(h);
    int rc = sweep_start_impl(h); if (rc) return rc;
    return finish_checked(h, 0);
}

// dqmc_gpu_sweep_start of several handles at once: every handle's work is
// enqueued on its own stream before any of them is waited for, so the
// handles' start-ups run concurrently.
extern "C" int dqmc_gpu_sweep_start_multi(dqmc_handle* const* hs, int n) {
    if (!hs || n < 1 || n > 16) return fail(DQMC_EINVAL, "1..16 handles");
    for (int k = 0; k < n; ++k)
        if (!hs[k]) return fail(DQMC_EINVAL, "null handle");
    int rc0 = DQMC_OK;
    for (int k = 0; k < n && !rc0; ++k) {
        clear_fail(hs[k]);
        rc0 = sweep_start_impl(hs[k], 0);
    }
    // every stream is waited for, also after an enqueue error
    for (int k = 0; k < n; ++k) {
        const cudaError_t e = cudaStreamSynchronize(hs[k]->st);
        if (e != cudaSuccess && !rc0) rc0 = fail(DQMC_ECUDA, cudaGetErrorString(e));
    }
    if (rc0) return rc0;
    CK(cudaGetLastError());
    for (int k = 0; k < n; ++k) {
        const int rc = finish_checked(hs[k], 0);
        if (rc) return rc;
    }
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_checks(dqmc_handle* h, double wrap_tol, int restabilize) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!(wrap_tol >= 0.0)) return fail(DQMC_EINVAL, "wrap_tol must be >= 0");
    double ctl[4] = {wrap_tol, 0.0, 0.0, 0.0};
    CK(copy_sync(h->st, h->d_ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice));
    h->restab = restabilize != 0;
    return DQMC_OK;
}

// one slice of the plaquette field in the finite-temperature sweep: delayed
// updates when every model's flush depth holds a plaquette's z columns, else
// rank-z changes straight on G (and the props alone without updates)
static void launch_plq(dqmc_handle* h, int nt, int visit, int dir, int lupdate) {
    int nbmin = 64;
    for (const HostModel* m : h->models) nbmin = std::min(nbmin, m->nublock_dev);
    if (!lupdate || !launch_plq_delay(h->d_chains, h->nch, nbmin, h->models[0]->z_plq, nt, visit, dir, h->st))
        launch_plq_slice(h->d_chains, h->nch, h->maxN, nt, visit, dir, lupdate, h->st);
}

// one bond family's finite-temperature updates: delayed when every model's
// flush depth holds two columns (dqmc_update_delay.f90), else rank-2 changes
// straight on G (dqmc_update.f90)
static void launch_vbond(dqmc_handle* h, int nt, int nf, int visit, int dir) {
    int nbmin = 64;
    for (const HostModel* m : h->models) nbmin = std::min(nbmin, m->nublock_dev);
    if (!launch_vbond_delay(h->d_chains, h->nch, nbmin, nt, nf, visit, dir, h->st))
        launch_vbond_slice(h->d_chains, h->nch, h->maxN, nt, nf, visit, dir, h->st);
}

static void enqueue_b0(dqmc_handle* h, int lupdate, int lmeasure) {
    const HostModel& m = *h->models[0];
    int lt = h->ltrot;
    launch_stack_identity(h->d_chains, h->nch, h->nst, h->st);
    const bool plq = m.plq_on, lv = m.p.rv != 0.0;
    if (lupdate && (m.p.rhub != 0.0 || plq || lv)) launch_sfmt(h->d_chains, h->nch, lt, h->st);
    tmark(h, DQMC_PROF_OTHER);
    for (int nt = lt; nt >= 1; --nt) {
        int visit = lt - nt;
        if (lmeasure) { launch_measure_h(h); tmark(h, DQMC_PROF_MEASURE); }
        PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
        prog_k(m, pl, PW_INV, 0);          // left_backward, nf = 1..nnf
        prog_k(m, pr, PW_FWD, 0);          // right_forward, nf = 1..nnf
        launch_prog(h, MAT_G, pl, 0);
        tmark(h, DQMC_PROF_PROP_L);
        launch_prog(h, MAT_G, pr, 1);
        tmark(h, DQMC_PROF_PROP_R);
        if (lupdate && m.p.rhub != 0.0) { launch_update(h->d_chains, h->nch, nt, visit, h->st, 0, 1); tmark(h, DQMC_PROF_UPDATE); }
        pl.n = 0; pr.n = 0;
        prog_v(m, pl, PW_INV, nt);         // u left_backward
        prog_v(m, pr, PW_FWD, nt);         // u right_forward
        if (lv)
            // the bond field, families nn_nf..1: nflag 2 (mix), the update,
            // nflag 1 (scale, mix) (dqmc_ft_sweep_b0.f90:79-90)
            for (int nf = m.nn_nf; nf >= 1; --nf) {
                prog_add(pr, PK_VMIX, 0, nf, nt);            // right_forward
                prog_add(pl, PK_VMIX, 0, nf, nt);            // left_backward
                if (lupdate) {
                    launch_prog(h, MAT_G, pl, 0);
                    launch_prog(h, MAT_G, pr, 1);
                    tmark(h, DQMC_PROF_PROP_L);
                    launch_vbond(h, nt, nf, visit, 1);
                    tmark(h, DQMC_PROF_UPDATE);
                    pl.n = 0; pr.n = 0;
                }
                prog_add(pr, PK_VSCALE, PW_FWD, nf, nt);
                prog_add(pr, PK_VMIX, 0, nf, nt);
                prog_add(pl, PK_VSCALE, PW_INV, nf, nt);
                prog_add(pl, PK_VMIX, 0, nf, nt);
            }
        if (plq) {
            // the plaquettes (update, then props, descending) between the U field
            // and the kinetic half step (dqmc_ft_sweep_b0.f90:91-101)
            launch_prog(h, MAT_G, pl, 0);
            launch_prog(h, MAT_G, pr, 1);
            tmark(h, DQMC_PROF_PROP_L);
            launch_plq(h, nt, visit, 1, lupdate);
            tmark(h, DQMC_PROF_UPDATE);
            pl.n = 0; pr.n = 0;
        }
        prog_k(m, pl, PW_INV, 1);          // h0 left_backward, nf = nnf..1
        prog_k(m, pr, PW_FWD, 1);
        launch_prog(h, MAT_G, pl, 0);
        tmark(h, DQMC_PROF_PROP_L);
        launch_prog(h, MAT_G, pr, 1);
        tmark(h, DQMC_PROF_PROP_R);
        if ((m.iwrap_nt[nt - 1] > 0 || m.p.nwrap == 1) || nt == 1) stab_b0(h, m.iwrap_nt[nt - 1]);
    }
}

static void enqueue_0b(dqmc_handle* h, int lupdate, int lmeasure) {
    const HostModel& m = *h->models[0];
    int lt = h->ltrot;
    launch_stack_identity(h->d_chains, h->nch, 0, h->st);
    const bool plq = m.plq_on, lv = m.p.rv != 0.0;
    if (lupdate && (m.p.rhub != 0.0 || plq || lv)) launch_sfmt(h->d_chains, h->nch, lt, h->st);
    tmark(h, DQMC_PROF_OTHER);
    for (int nt = 1; nt <= lt; ++nt) {
        int visit = nt - 1;
        PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
        prog_k(m, pl, PW_FWD, 0);          // left_forward, nf = 1..nnf
        prog_k(m, pr, PW_INV, 0);          // right_backward
        if (plq) {
            // the plaquettes (props, then update, ascending) between the kinetic
            // half step and the U field (dqmc_ft_sweep_0b.f90:82-93)
            launch_prog(h, MAT_G, pl, 0);
            launch_prog(h, MAT_G, pr, 1);
            tmark(h, DQMC_PROF_PROP_L);
            launch_plq(h, nt, visit, 0, lupdate);
            tmark(h, DQMC_PROF_UPDATE);
            pl.n = 0; pr.n = 0;
        }
        if (lv)
            // the bond field, families 1..nn_nf: nflag 2 (mix, scale), the
            // update, nflag 1 (mix) (dqmc_ft_sweep_0b.f90:96-106)
            for (int nf = 1; nf <= m.nn_nf; ++nf) {
                prog_add(pl, PK_VMIX, 0, nf, nt);            // left_forward
                prog_add(pl, PK_VSCALE, PW_FWD, nf, nt);
                prog_add(pr, PK_VMIX, 0, nf, nt);            // right_backward
                prog_add(pr, PK_VSCALE, PW_INV, nf, nt);
                if (lupdate) {
                    launch_prog(h, MAT_G, pl, 0);
                    launch_prog(h, MAT_G, pr, 1);
                    tmark(h, DQMC_PROF_PROP_L);
                    launch_vbond(h, nt, nf, visit, 0);
                    tmark(h, DQMC_PROF_UPDATE);
                    pl.n = 0; pr.n = 0;
                }
                prog_add(pl, PK_VMIX, 0, nf, nt);
                prog_add(pr, PK_VMIX, 0, nf, nt);
            }
        prog_v(m, pl, PW_FWD, nt);         // u left_forward
        prog_v(m, pr, PW_INV, nt);         // u right_backward
        launch_prog(h, MAT_G, pl, 0);
        tmark(h, DQMC_PROF_PROP_L);
        launch_prog(h, MAT_G, pr, 1);
        tmark(h, DQMC_PROF_PROP_R);
        if (lupdate && m.p.rhub != 0.0) { launch_update(h->d_chains, h->nch, nt, visit, h->st); tmark(h, DQMC_PROF_UPDATE); }
        pl.n = 0; pr.n = 0;
        prog_k(m, pl, PW_FWD, 1);
        prog_k(m, pr, PW_INV, 1);
        launch_prog(h, MAT_G, pl, 0);
        tmark(h, DQMC_PROF_PROP_L);
        launch_prog(h, MAT_G, pr, 1);
        tmark(h, DQMC_PROF_PROP_R);
        if (lmeasure) { launch_measure_h(h); tmark(h, DQMC_PROF_MEASURE); }
        if (m.iwrap_nt[nt] > 0) stab_0b(h, m.iwrap_nt[nt], 1);
    }
}

static int chk_chain(dqmc_handle* h, int c);

// one stabilisation of the unequal-time pass (dqmc_ft_sweep_0b.f90:145-230 with
// lmeasure_dyn): new right factor into the spare slot, green_tau from (new R,
// old L), wrap check, swap
static void stab_dyn(dqmc_handle* h, int n) {
    const HostModel& m = *h->models[0];
    int spare = h->nst + 1;
    launch_copy_mat(h->d_chains, h->nch, 2 /*W0*/, MAT_U + (n - 1), 0, h->st);
    launch_bmat(h, 2, m.wrap_step[(n - 1) * 2 + 1], m.wrap_step[(n - 1) * 2], 0);
    launch_stab_slots(h->d_chains, h->nch, n - 1, spare, h->st);
    launch_green_tau(h->d_chains, h->nch, spare, n, h->st);
    launch_wrap_check(h->d_chains, h->nch, 1, h->st);
    launch_swap_slots(h->d_slotmap, n, spare, h->st);
}

// The unequal-time pass of dqmc_sweep (src/dqmc_ft_ctrl.f90:97-101): push_stage,
// dqmc_ft_sweep_0b(lupdate = F, lmeasure_equaltime = F, lmeasure_dyn = T) with
// dyn.f90 (G(t',0) = B(t',t) G(t,0), G(0,t') = G(0,t) B(t',t)^-1 between
// stabilisations, green_tau at them) and dyn_measure at every time index, then
// pop_stage (src/dqmc_ft_core.f90:290-312).
static void enqueue_dyn(dqmc_handle* h) {
    const HostModel& m = *h->models[0];
    const int lt = h->ltrot, nslots = h->nst + 2;
    launch_stage(h->d_chains, h->nch, nslots, 0, h->st);
    cudaMemcpyAsync(h->d_slotmap_b, h->d_slotmap, sizeof(int) * nslots, cudaMemcpyDeviceToDevice, h->st);
    launch_stack_identity(h->d_chains, h->nch, 0, h->st);
    launch_dyn_init(h->d_chains, h->nch, h->st);
    launch_dyn_measure(h->d_chains, h->nch, h->maxN, 1, h->st);
    for (int nt = 1; nt <= lt; ++nt) {
        PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
        // Bmat_left_forward / Bmat_right_backward of one slice: kinetic, the
        // plaquettes ascending, the bond field, the U field, kinetic
        // (src/dqmc_ft_core.f90:80-117, 234-288)
        prog_k(m, pl, PW_FWD, 0);
        if (m.plq_on) prog_add(pl, PK_PLQ, PW_FWD, 0, nt);
        prog_bond(m, pl, PW_FWD, nt, 0);
        prog_v(m, pl, PW_FWD, nt);
        prog_k(m, pl, PW_FWD, 1);
        prog_k(m, pr, PW_INV, 0);
        if (m.plq_on) prog_add(pr, PK_PLQ, PW_INV, 0, nt);
        prog_bond(m, pr, PW_INV, nt, 0);
        prog_v(m, pr, PW_INV, nt);
        prog_k(m, pr, PW_INV, 1);
        launch_prog(h, MAT_G, pl, 0);
        launch_prog(h, MAT_G, pr, 1);
        if (m.iwrap_nt[nt] > 0) {
            stab_dyn(h, m.iwrap_nt[nt]);
        } else {
            launch_prog(h, MAT_GT0, pl, 0);     // Bmat_left_forward(nt, nt, gt0)
            launch_prog(h, MAT_G0T, pr, 1);     // Bmat_right_backward(nt, nt, g0t)
        }
        launch_dyn_measure(h->d_chains, h->nch, h->maxN, nt + 1, h->st);
    }
    launch_stage(h->d_chains, h->nch, nslots, 1, h->st);
    cudaMemcpyAsync(h->d_slotmap, h->d_slotmap_b, sizeof(int) * nslots, cudaMemcpyDeviceToDevice, h->st);
}

extern "C" int dqmc_gpu_sweep_dyn(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
    if (h->proj) return fail(DQMC_ESTATE, "on the projective path the unequal-time pass runs inside the measured 0b sweep");
    if (!h->models[0]->p.ltau) return fail(DQMC_ESTATE, "the unequal-time pass needs ltau = 1");
    if (!h->after_b0) return fail(DQMC_ESTATE, "the unequal-time pass follows a b0 sweep (it needs the b0 sweep's left factors)");
    clear_fail(h);
    enqueue_dyn(h);
    return finish_checked(h, 0);
}

extern "C" int dqmc_gpu_get_dyn_bins(dqmc_handle* h, int chain, double* out) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (!out) return fail(DQMC_EINVAL, "null output");
    const HostModel& m = *h->models[h->chains[chain].model];
    if (!m.p.ltau) return fail(DQMC_ESTATE, "ltau = 0: no unequal-time bins");
    CK(copy_sync(h->st, out, h->chains[chain].dev.dynbins, (size_t)m.lq * 4 * (m.p.ntdm + 1) * sizeof(double2),
                 cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_dyn_mats(dqmc_handle* h, int chain, double* g00, double* gt0, double* g0t) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    if (!d.gt0) return fail(DQMC_ESTATE, "ltau = 0: no unequal-time Green's functions");
    const size_t b = (size_t)d.N * d.N * sizeof(double2);
    if (g00) CK(copy_sync(h->st, g00, d.g00, b, cudaMemcpyDeviceToHost));
    if (gt0) CK(copy_sync(h->st, gt0, d.gt0, b, cudaMemcpyDeviceToHost));
    if (g0t) CK(copy_sync(h->st, g0t, d.g0t, b, cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_sweep_b0(dqmc_handle* h, int lupdate, int lmeasure) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
    clear_fail(h);
    if (h->proj) enqueue_proj_b0(h, lupdate, lmeasure);
    else enqueue_b0(h, lupdate, lmeasure);
    h->after_b0 = 1;
    return finish_checked(h, 0);
}

extern "C" int dqmc_gpu_sweep_0b(dqmc_handle* h, int lupdate, int lmeasure) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
    clear_fail(h);
    if (h->proj) enqueue_proj_0b(h, lupdate, lmeasure);
    else enqueue_0b(h, lupdate, lmeasure);
    h->after_b0 = 0;
    return finish_checked(h, 1);
}

// the captured sweep (b0 + 0b) of dqmc_gpu_sweeps, rebuilt when lmeasure or
// recording changed
static int ensure_sweep_graph(dqmc_handle* h, int lmeasure) {
    if (!h->sweep_graph || h->graph_meas != lmeasure + 2 * h->rec_on) {
        drop_sweep_graph(h);
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        if (h->proj) {
            enqueue_proj_b0(h, 1, lmeasure);
            enqueue_proj_0b(h, 1, lmeasure);
        } else {
            enqueue_b0(h, 1, lmeasure);
            if (lmeasure && h->models[0]->p.ltau) enqueue_dyn(h);   // dqmc_sweep (src/dqmc_ft_ctrl.f90:97-101)
            enqueue_0b(h, 1, lmeasure);
        }
        // the capture always ends here, so the stream leaves capture mode on
        // every path; a failed capture's partial graph is discarded
        cudaError_t e = cudaStreamEndCapture(h->st, &g);
        if (e != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return fail(DQMC_ECUDA, std::string("sweep capture: ") + cudaGetErrorString(e));
        }
        e = cudaGraphInstantiate(&h->sweep_graph, g, 0);
        size_t nn = 0;
        if (e == cudaSuccess) cudaGraphGetNodes(g, nullptr, &nn);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            h->sweep_graph = nullptr;
            return fail(DQMC_ECUDA, std::string("sweep graph instantiation: ") + cudaGetErrorString(e));
        }
        h->graph_nodes = nn;
        h->graph_meas = lmeasure + 2 * h->rec_on;
    }
    return DQMC_OK;
}

extern "C" int dqmc_gpu_sweeps(dqmc_handle* h, int n, int lmeasure) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
    if (n <= 0) return DQMC_OK;
    int rc = ensure_sweep_graph(h, lmeasure); if (rc) return rc;
    h->after_b0 = 0;
    clear_fail(h);
    CK(cudaEventRecord(h->ev0, h->st));
    for (int i = 0; i < n; ++i) CK(cudaGraphLaunch(h->sweep_graph, h->st));
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_ms = ms / n;
    return finish_checked(h, 1);
}

// n sweeps of several handles at once: each handle's sweep graph on its own
// stream, forked from and joined to the first handle's stream, so that the
// kernels of different handles (different phases of their sweeps) share the
// SMs.  The device time between fork and join goes to every handle's last_ms
// and to *ms_out.
extern "C" int dqmc_gpu_sweeps_multi(dqmc_handle* const* hs, int nh, int n, int lmeasure, double* ms_out) {
    if (!hs || nh < 1 || nh > 16) return fail(DQMC_EINVAL, "1..16 handles");
    for (int k = 0; k < nh; ++k) {
        if (!hs[k]) return fail(DQMC_EINVAL, "null handle");
        if (!hs[k]->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
        for (int q = 0; q < k; ++q)
            if (hs[q] == hs[k]) return fail(DQMC_EINVAL, "a handle appears twice");
    }
    if (n <= 0) return DQMC_OK;
    for (int k = 0; k < nh; ++k) {
        int rc = ensure_sweep_graph(hs[k], lmeasure); if (rc) return rc;
        hs[k]->after_b0 = 0;
        clear_fail(hs[k]);
    }
    dqmc_handle* h0 = hs[0];
    cudaEvent_t fork = nullptr, join[16] = {};
    // the first error is kept; every stream is still joined and every event
    // destroyed before returning
    cudaError_t err = cudaSuccess;
    auto keep = [&](cudaError_t e) { if (err == cudaSuccess && e != cudaSuccess) err = e; };
    keep(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int k = 1; k < nh; ++k) keep(cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming));
    if (err == cudaSuccess) {
        keep(cudaEventRecord(h0->ev0, h0->st));
        keep(cudaEventRecord(fork, h0->st));
        for (int k = 1; k < nh; ++k) keep(cudaStreamWaitEvent(hs[k]->st, fork, 0));
        for (int i = 0; i < n && err == cudaSuccess; ++i)
            for (int k = 0; k < nh; ++k) keep(cudaGraphLaunch(hs[k]->sweep_graph, hs[k]->st));
        for (int k = 1; k < nh; ++k) {
            keep(cudaEventRecord(join[k], hs[k]->st));
            keep(cudaStreamWaitEvent(h0->st, join[k], 0));
        }
        keep(cudaEventRecord(h0->ev1, h0->st));
    }
    for (int k = 0; k < nh; ++k) keep(cudaStreamSynchronize(hs[k]->st));
    keep(cudaGetLastError());
    float ms = 0;
    if (err == cudaSuccess) keep(cudaEventElapsedTime(&ms, h0->ev0, h0->ev1));
    if (fork) cudaEventDestroy(fork);
    for (int k = 1; k < nh; ++k) if (join[k]) cudaEventDestroy(join[k]);
    if (err != cudaSuccess) return fail(DQMC_ECUDA, std::string("sweeps_multi: ") + cudaGetErrorString(err));
    for (int k = 0; k < nh; ++k) hs[k]->last_ms = ms / n;
    if (ms_out) *ms_out = ms / n;
    for (int k = 0; k < nh; ++k) {
        int rc = finish_checked(hs[k], 1); if (rc) return rc;
    }
    return DQMC_OK;
}

extern "C" double dqmc_gpu_last_sweeps_ms(dqmc_handle* h) { return h ? h->last_ms : 0.0; }

extern "C" int dqmc_gpu_sweep_kernels(dqmc_handle* h) { return h ? (int)h->graph_nodes : 0; }

// ---------------------------------------------------------------------------
// data access
// ---------------------------------------------------------------------------
static int chk_chain(dqmc_handle* h, int c) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (c < 0 || c >= h->nch) return fail(DQMC_EINVAL, "chain index out of range");
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_conf(dqmc_handle* h, int chain, const int32_t* conf) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    int lcomp = h->models[h->chains[chain].model]->lcomp;
    size_t n = (size_t)h->ltrot * d.N;
    for (size_t e = 0; e < n; ++e)
        if (conf[e] < 1 || conf[e] > lcomp) return fail(DQMC_EINVAL, "HS field value out of range 1..lcomp");
    CK(copy_sync(h->st, d.conf, conf, n * sizeof(int32_t), cudaMemcpyHostToDevice));
    h->started = 0;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_conf(dqmc_handle* h, int chain, int32_t* conf) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    CK(copy_sync(h->st, conf, d.conf, (size_t)h->ltrot * d.N * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_conf_all(dqmc_handle* h, const int32_t* conf) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    size_t off = 0;
    for (int c = 0; c < h->nch; ++c) {
        const ChainDev& d = h->chains[c].dev;
        size_t n = (size_t)h->ltrot * d.N;
        int lcomp = h->models[h->chains[c].model]->lcomp;
        for (size_t e = 0; e < n; ++e)
            if (conf[off + e] < 1 || conf[off + e] > lcomp) return fail(DQMC_EINVAL, "HS field value out of range 1..lcomp");
        CK(cudaMemcpyAsync(d.conf, conf + off, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->st));
        off += n;
    }
    CK(cudaStreamSynchronize(h->st));
    h->started = 0;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_conf_all(dqmc_handle* h, int32_t* conf) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    size_t off = 0;
    for (int c = 0; c < h->nch; ++c) {
        const ChainDev& d = h->chains[c].dev;
        size_t n = (size_t)h->ltrot * d.N;
        CK(cudaMemcpyAsync(conf + off, d.conf, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
        off += n;
    }
    CK(cudaStreamSynchronize(h->st));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_green(dqmc_handle* h, int chain, double* g) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    CK(copy_sync(h->st, g, d.G, (size_t)d.N * d.N * sizeof(double2), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_green(dqmc_handle* h, int chain, const double* g) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    CK(copy_sync(h->st, d.G, g, (size_t)d.N * d.N * sizeof(double2), cudaMemcpyHostToDevice));
    h->started = 1;
    return DQMC_OK;
}

// wrap trace of one chain: the fresh G and the wrap error at each of the next
// `capacity` recorded wrap checks (capacity 0 stops it and frees the buffers);
// the counterpart of the reference's -DTEST_LEVEL3 print of gf_tmp at every
// stabilisation (src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:160-179)
extern "C" int dqmc_gpu_trace_wraps(dqmc_handle* h, int chain, int capacity) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (capacity < 0) return fail(DQMC_EINVAL, "capacity >= 0");
    ChainDev& d = h->chains[chain].dev;
    CK(cudaStreamSynchronize(h->st));
    dfree(h, d.trace_g); dfree(h, d.trace_err); dfree(h, d.trace_n);
    d.trace_g = nullptr; d.trace_err = nullptr; d.trace_n = nullptr; d.trace_cap = 0;
    if (capacity > 0) {
        d.trace_g = (double2*)dalloc(h, (size_t)capacity * d.N * d.N * sizeof(double2));
        d.trace_err = (double*)dalloc(h, (size_t)capacity * sizeof(double));
        d.trace_n = (int*)dalloc(h, sizeof(int));
        if (!d.trace_g || !d.trace_err || !d.trace_n) {
            dfree(h, d.trace_g); dfree(h, d.trace_err); dfree(h, d.trace_n);
            d.trace_g = nullptr; d.trace_err = nullptr; d.trace_n = nullptr;
            CK(copy_sync(h->st, h->d_chains + chain, &d, sizeof(ChainDev), cudaMemcpyHostToDevice));
            return fail(DQMC_ENOMEM, "trace buffers");
        }
        d.trace_cap = capacity;
    }
    CK(copy_sync(h->st, h->d_chains + chain, &d, sizeof(ChainDev), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_trace_count(dqmc_handle* h, int chain) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    if (!d.trace_n) return 0;
    int n = 0;
    CK(copy_sync(h->st, &n, d.trace_n, sizeof(int), cudaMemcpyDeviceToHost));
    return n;
}

extern "C" int dqmc_gpu_trace_get(dqmc_handle* h, int chain, int i, double* g, double* err) {
    int n = dqmc_gpu_trace_count(h, chain); if (n < 0) return n;
    if (i < 0 || i >= n) return fail(DQMC_EINVAL, "trace index out of range");
    const ChainDev& d = h->chains[chain].dev;
    const size_t NN = (size_t)d.N * d.N;
    if (g) CK(copy_sync(h->st, g, d.trace_g + (size_t)i * NN, NN * sizeof(double2), cudaMemcpyDeviceToHost));
    if (err) CK(copy_sync(h->st, err, d.trace_err + i, sizeof(double), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

// Ust(n), Dst(n), Vst(n), logdetQst(n) of the finite-temperature UDV stack
// (src/dqmc_ft_core.f90:11-19), logical index n = 0..nst, through the slot map
static int stack_slot(dqmc_handle* h, int chain, int n, int* slot) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (h->proj) return fail(DQMC_ESTATE, "the projective path has no UDV stack");
    if (n < 0 || n > h->nst) return fail(DQMC_EINVAL, "stack index 0..nst");
    CK(copy_sync(h->st, slot, h->d_slotmap + n, sizeof(int), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_stack(dqmc_handle* h, int chain, int n, double* u, double* d, double* v, double* logdetq) {
    int slot = 0;
    int rc = stack_slot(h, chain, n, &slot); if (rc) return rc;
    const ChainDev& c = h->chains[chain].dev;
    const size_t NN = (size_t)c.N * c.N;
    if (u) CK(copy_sync(h->st, u, c.U + slot * NN, NN * sizeof(double2), cudaMemcpyDeviceToHost));
    if (v) CK(copy_sync(h->st, v, c.V + slot * NN, NN * sizeof(double2), cudaMemcpyDeviceToHost));
    if (d) CK(copy_sync(h->st, d, c.D + (size_t)slot * c.N, c.N * sizeof(double), cudaMemcpyDeviceToHost));
    if (logdetq) CK(copy_sync(h->st, logdetq, c.logdetQ + slot, sizeof(double2), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_stack(dqmc_handle* h, int chain, int n, const double* u, const double* d, const double* v,
                                  const double* logdetq) {
    int slot = 0;
    int rc = stack_slot(h, chain, n, &slot); if (rc) return rc;
    const ChainDev& c = h->chains[chain].dev;
    const size_t NN = (size_t)c.N * c.N;
    if (u) CK(copy_sync(h->st, c.U + slot * NN, u, NN * sizeof(double2), cudaMemcpyHostToDevice));
    if (v) CK(copy_sync(h->st, c.V + slot * NN, v, NN * sizeof(double2), cudaMemcpyHostToDevice));
    if (d) CK(copy_sync(h->st, c.D + (size_t)slot * c.N, d, c.N * sizeof(double), cudaMemcpyHostToDevice));
    if (logdetq) CK(copy_sync(h->st, c.logdetQ + slot, logdetq, sizeof(double2), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_work(dqmc_handle* h, int chain, int which, const double* mtx) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (which < 0 || which > 5) return fail(DQMC_EINVAL, "work index 0..5");
    const ChainDev& d = h->chains[chain].dev;
    CK(copy_sync(h->st, d.W[which], mtx, (size_t)d.N * d.N * sizeof(double2), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_work(dqmc_handle* h, int chain, int which, double* mtx) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (which < 0 || which > 5) return fail(DQMC_EINVAL, "work index 0..5");
    const ChainDev& d = h->chains[chain].dev;
    CK(copy_sync(h->st, mtx, d.W[which], (size_t)d.N * d.N * sizeof(double2), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_test_zgemm(dqmc_handle* h, int m, int n, int k, int opa, int opb, int a, int b, int c, double beta) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (m < 0 || n < 0 || k < 0 || m > h->maxN || n > h->maxN || k > h->maxN) return fail(DQMC_EINVAL, "gemm size");
    if (a < 0 || a > 5 || b < 0 || b > 5 || c < 0 || c > 5) return fail(DQMC_EINVAL, "work index 0..5");
    launch_zgemm_test(h->d_chains, h->nch, m, n, k, opa, opb, 2 + a, 2 + b, 2 + c, beta, h->st);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

extern "C" int dqmc_gpu_test_qr(dqmc_handle* h, int a, int q, double* logdetq) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (a < 0 || a > 4 || q < 0 || q > 4 || a == q) return fail(DQMC_EINVAL, "work index 0..4, a != q");
    launch_qr_test(h->d_chains, h->nch, 2 + a, 2 + q, h->st);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    for (int c = 0; c < h->nch; ++c) {
        double st[ST_COUNT];
        CK(copy_sync(h->st, st, h->chains[c].dev.stats, sizeof(st), cudaMemcpyDeviceToHost));
        logdetq[2 * c] = st[ST_LOGDETM_RE];
        logdetq[2 * c + 1] = st[ST_LOGDETM_IM];
    }
    return DQMC_OK;
}

extern "C" int dqmc_gpu_obser_init(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    int maxb = 0;
    for (auto* m : h->models) maxb = std::max(maxb, 10 + 20 * m->lq + 4);
    launch_bins_clear(h->d_chains, h->nch, maxb, h->st);
    CK(cudaStreamSynchronize(h->st));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_nbins(dqmc_handle* h, int chain) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    return 10 + 20 * h->models[h->chains[chain].model]->lq + 4;
}

extern "C" int dqmc_gpu_get_bins(dqmc_handle* h, int chain, double* out) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    int nb = dqmc_gpu_nbins(h, chain);
    CK(copy_sync(h->st, out, h->chains[chain].dev.bins, (size_t)nb * sizeof(double2), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_energy_all(dqmc_handle* h, double* out) {
    if (!h || !out) return fail(DQMC_EINVAL, "invalid arguments");
    for (int c = 0; c < h->nch; ++c)
        CK(cudaMemcpyAsync(out + 20 * (size_t)c, h->chains[c].dev.bins, 10 * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_diag(dqmc_handle* h, int chain, dqmc_diag* out) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    double st[ST_COUNT];
    CK(copy_sync(h->st, st, h->chains[chain].dev.stats, sizeof(st), cudaMemcpyDeviceToHost));
    out->phase_re = st[ST_PHASE_RE]; out->phase_im = st[ST_PHASE_IM];
    out->logweight_re = st[ST_LOGW_RE]; out->logweight_im = st[ST_LOGW_IM];
    out->max_wrap_error = st[ST_MAX_WRAP]; out->max_phasediff = st[ST_MAX_PHASEDIFF];
    out->avglog10error_sum = st[ST_AVGLOG10]; out->logcount = st[ST_LOGCOUNT];
    out->avgexpphasediff_sum = st[ST_AVGEXPPD];
    out->accepted = st[ST_ACC]; out->proposed = st[ST_PROP]; out->nobs = st[ST_NOBS];
    out->accepted_v = st[ST_ACCV]; out->proposed_v = st[ST_PROPV];
    out->blk_proposed = st[ST_BLK_PROP]; out->blk_stage1 = st[ST_BLK_S1]; out->blk_accepted = st[ST_BLK_ACC];
    out->blk_sum_logratio = st[ST_BLK_SUMLR];
    out->blk_err_learned = st[ST_BLK_ERR1]; out->blk_err_zero = st[ST_BLK_ERR0];
    out->max_dyn_error = st[ST_MAX_DYN];
    out->dyn_log10_sum = st[ST_DYN_LOG10]; out->dyn_count = st[ST_DYN_COUNT];
    out->info = st[ST_INFO];
    out->restabilized = h->n_restab;
    out->near_ties = st[ST_NEAR_TIE];
    out->accepted_plq = st[ST_ACCP]; out->proposed_plq = st[ST_PROPP];
    return DQMC_OK;
}

extern "C" int dqmc_gpu_reset_diag(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    for (int c = 0; c < h->nch; ++c) {
        double st[ST_COUNT];
        CK(copy_sync(h->st, st, h->chains[c].dev.stats, sizeof(st), cudaMemcpyDeviceToHost));
        st[ST_MAX_WRAP] = st[ST_MAX_PHASEDIFF] = st[ST_AVGLOG10] = st[ST_LOGCOUNT] = st[ST_AVGEXPPD] = 0.0;
        st[ST_ACC] = st[ST_PROP] = st[ST_ACCV] = st[ST_PROPV] = st[ST_ACCP] = st[ST_PROPP] = 0.0;
        st[ST_BLK_PROP] = st[ST_BLK_S1] = st[ST_BLK_ACC] = st[ST_BLK_SUMLR] = 0.0;
        st[ST_BLK_ERR1] = st[ST_BLK_ERR0] = 0.0;
        st[ST_MAX_DYN] = st[ST_DYN_LOG10] = st[ST_DYN_COUNT] = 0.0;
        st[ST_INFO] = 0.0;
        st[ST_NEAR_TIE] = 0.0;
        CK(copy_sync(h->st, h->chains[c].dev.stats, st, sizeof(st), cudaMemcpyHostToDevice));
    }
    h->n_restab = 0.0;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_phase(dqmc_handle* h, int chain, double re, double im) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    double v[2] = {re, im};
    CK(copy_sync(h->st, h->chains[chain].dev.stats + ST_PHASE_RE, v, sizeof(v), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

// SFMT-19937 state of one chain in the reference's representation
// (lib/m_spring.f90:66-71): pt32(0:623), the 32-bit view of the 128-bit state
// array, then the read index idx (624 = the next draw regenerates the block).
// The device generator keeps exactly these 625 words, so a mid-run state
// handed over by a Fortran caller continues its stream.
extern "C" int dqmc_gpu_get_rng(dqmc_handle* h, int chain, int32_t* state) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (!state) return fail(DQMC_EINVAL, "null state");
    CK(copy_sync(h->st, state, h->chains[chain].dev.sfmt, 625 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_rng(dqmc_handle* h, int chain, const int32_t* state) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (!state) return fail(DQMC_EINVAL, "null state");
    if (state[624] < 0 || state[624] > 624) return fail(DQMC_EINVAL, "SFMT read index outside 0..624");
    CK(copy_sync(h->st, h->chains[chain].dev.sfmt, state, 625 * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_draw_u32(dqmc_handle* h, int chain, int count, uint32_t* out) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    if (count < 0 || count > h->ltrot * 2 * d.N) return fail(DQMC_EINVAL, "count out of range");
    launch_sfmt_raw(h->d_chains, chain, count, h->st);
    CK(cudaStreamSynchronize(h->st));
    CK(copy_sync(h->st, out, d.rnd, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// operator-level entry points
// ---------------------------------------------------------------------------
extern "C" int dqmc_gpu_h0_prop(dqmc_handle* h, int op, int nf) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    const HostModel& m = *h->models[0];
    if (op < 0 || op > 4) return fail(DQMC_EINVAL, "op 0..4");
    if (m.p.kinetic == DQMC_KIN_CHECKERBOARD && (nf < 1 || nf > m.nn_nf)) return fail(DQMC_EINVAL, "nf out of range");
    PropProg p; p.n = 0;
    int which = (op == 1 || op == 3) ? PW_INV : (op == 4 ? PW_CONJ : PW_FWD);
    if (m.p.kinetic == DQMC_KIN_FFT) prog_add(p, PK_FFT, which, 0, 0);
    else if (m.p.kinetic == DQMC_KIN_DENSE) prog_add(p, PK_DENSE, which, 0, 0);
    else prog_add(p, PK_CB, which == PW_CONJ ? PW_FWD : which, nf, 0);
    launch_prog(h, MAT_G, p, (op == 2 || op == 3) ? 1 : 0);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

extern "C" int dqmc_gpu_u_prop(dqmc_handle* h, int op, int nt) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (op < 0 || op > 4) return fail(DQMC_EINVAL, "op 0..4");
    if (nt < 1 || nt > h->ltrot) return fail(DQMC_EINVAL, "nt out of range");
    PropProg p; p.n = 0;
    int which = (op == 1 || op == 3) ? PW_INV : (op == 4 ? PW_CONJ : PW_FWD);
    prog_add(p, PK_DIAG, which, 0, nt);
    launch_prog(h, MAT_G, p, (op == 2 || op == 3) ? 1 : 0);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

extern "C" int dqmc_gpu_update(dqmc_handle* h, int nt) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (h->proj) return fail(DQMC_ESTATE, "projective handle: use dqmc_gpu_proj_update");
    if (nt < 1 || nt > h->ltrot) return fail(DQMC_EINVAL, "nt out of range");
    const HostModel& m0 = *h->models[0];
    if (m0.plq_on || m0.p.rv != 0.0) {
        // exactly the 2 N draws of uconf%update (the slice layout of a sweep also
        // holds the plaquette and bond words); the U words start the b0 layout
        launch_sfmt(h->d_chains, h->nch, -2 * m0.N, h->st);
        launch_update(h->d_chains, h->nch, nt, 0, h->st, 0, 1);
    } else {
        launch_sfmt(h->d_chains, h->nch, 1, h->st);
        launch_update(h->d_chains, h->nch, nt, 0, h->st);
    }
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

extern "C" int dqmc_gpu_measure(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    launch_measure_h(h);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// per-kernel timing on the library stream (CUDA events), used by bench.py for
// the roofline of the dominant kernel.  op: 0 update (slice 1), 1 UDV step
// (stabilisation kernel, into the spare stack slot), 2 Green's function
// (equal-time, stack slots 1 and 0, into Gnew), 3 kinetic+HS column pass on
// G, 4 measurement, 5 kinetic+HS row pass on G, 6 the delayed update's flush
// GEMM alone (G += A B^T over nublock columns).  The chains' state is modified
// (update, measurement, flush): call it after the timed region.
// ---------------------------------------------------------------------------
extern "C" int dqmc_gpu_time_op(dqmc_handle* h, int op, int reps, double* ms_out) {
    if (!h || reps < 1 || !ms_out) return fail(DQMC_EINVAL, "invalid arguments");
    const HostModel& m = *h->models[0];
    int spare = h->nst + 1;
    auto enqueue = [&]() {
        switch (op) {
        case 0: launch_update(h->d_chains, h->nch, 1, 0, h->st); break;
        case 1: launch_stab_slots(h->d_chains, h->nch, 0, spare, h->st); break;
        case 2: launch_green(h->d_chains, h->nch, 1, 0, 0, 0, 0, 0, 0, h->st); break;
        case 3: { PropProg p; p.n = 0; prog_k(m, p, PW_INV, 0); prog_v(m, p, PW_INV, 1); prog_k(m, p, PW_INV, 1);
                  launch_prog(h, MAT_G, p, 0); break; }
        case 4: launch_measure_h(h); break;
        case 5: { PropProg p; p.n = 0; prog_k(m, p, PW_FWD, 0); prog_v(m, p, PW_FWD, 1); prog_k(m, p, PW_FWD, 1);
                  launch_prog(h, MAT_G, p, 1); break; }
        case 6: launch_update_flush(h->d_chains, h->nch, h->st); break;
        default: break;
        }
    };
    // projective handles: 0 bond-family (or site) update, 1 tall QR, 2 (UL UR)^-1
    // with log det and G, 3 / 5 one slice of propagation over UR / UL^T, 4 measurement
    int pnf = (m.p.rv != 0.0) ? 1 : 0;
    auto enqueue_proj = [&]() {
        switch (op) {
        case 0: proj_update(h, 1, pnf, 0, 0, -1); break;
        case 1: launch_proj_qr(h->d_chains, h->nch, PMAT_UR, 1, 0, h->st); break;
        case 2: launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 1, 1, -1, h->st);
                launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_GNEW, h->ctas_per_chain, h->st); break;
        case 3: case 5: {
            ProjPass pp;
            PropProg& pr = (op == 3) ? pp.r : pp.l;
            pk(h, pp, pr, PW_FWD, 0);
            if (m.p.rv != 0.0)
                for (int nf = 1; nf <= m.nn_nf; ++nf) {
                    padd(h, pp, pr, PK_VMIX, 0, nf, 1);
                    padd(h, pp, pr, PK_VSCALE, PW_FWD, nf, 1);
                    padd(h, pp, pr, PK_VMIX, 0, nf, 1);
                }
            if (m.p.rhub != 0.0) padd(h, pp, pr, PK_DIAG, PW_FWD, 0, 1);
            pk(h, pp, pr, PW_FWD, 1);
            pflush(h, pp);
            break;
        }
        case 4: launch_measure_h(h); break;
        default: break;
        }
    };
    if (op < 0 || op > 6 || (op == 6 && h->proj)) return fail(DQMC_EINVAL, "op 0..5 (0..6 at finite temperature)");
    if (h->proj) {
        if (!h->started) return fail(DQMC_ESTATE, "time_op before sweep_start");
        if (op == 0) launch_sfmt(h->d_chains, h->nch, 1, h->st);
        enqueue_proj();
        CK(cudaStreamSynchronize(h->st));
        CK(cudaEventRecord(h->ev0, h->st));
        for (int r = 0; r < reps; ++r) enqueue_proj();
        CK(cudaEventRecord(h->ev1, h->st));
        CK(cudaStreamSynchronize(h->st));
        CK(cudaGetLastError());
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        *ms_out = ms / reps;
        return DQMC_OK;
    }
    if (op == 0) launch_sfmt(h->d_chains, h->nch, 1, h->st);
    enqueue();   // warm-up
    CK(cudaStreamSynchronize(h->st));
    CK(cudaEventRecord(h->ev0, h->st));
    for (int r = 0; r < reps; ++r) enqueue();
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    *ms_out = ms / reps;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_sweep_profile(dqmc_handle* h, int nsweeps, int lmeasure, double* ms, int* groups) {
    if (!h || nsweeps < 1 || !ms || !groups) return fail(DQMC_EINVAL, "invalid arguments");
    if (!h->started) return fail(DQMC_ESTATE, "sweep_profile before sweep_start");
    CK(cudaStreamSynchronize(h->st));
    h->tm_on = 1;
    h->tm_n = 0;
    tmark(h, -1);
    for (int s = 0; s < nsweeps; ++s) {
        if (h->proj) { enqueue_proj_b0(h, 1, lmeasure); enqueue_proj_0b(h, 1, lmeasure); }
        else { enqueue_b0(h, 1, lmeasure); enqueue_0b(h, 1, lmeasure); }
        h->after_b0 = 0;
    }
    const int ok = h->tm_on;
    h->tm_on = 0;
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    if (!ok) return fail(DQMC_ECUDA, "could not create the profiling events");
    for (int k = 0; k < DQMC_PROF_KINDS; ++k) { ms[k] = 0.0; groups[k] = 0; }
    for (int i = 1; i < h->tm_n; ++i) {
        float dt = 0.f;
        CK(cudaEventElapsedTime(&dt, h->tm_ev[i - 1], h->tm_ev[i]));
        const int k = h->tm_kind[i];
        if (k >= 0 && k < DQMC_PROF_KINDS) { ms[k] += dt; groups[k] += 1; }
    }
    return DQMC_OK;
}

// ---------------------------------------------------------------------------
// projective path: data access and operator-level entry points
// ---------------------------------------------------------------------------
static int chk_proj(dqmc_handle* h, int c) {
    int rc = chk_chain(h, c); if (rc) return rc;
    if (!h->proj) return fail(DQMC_ESTATE, "not a projective handle (params.proj = 0)");
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_vconf(dqmc_handle* h, int chain, const int32_t* v) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    if (!d.vconf) return fail(DQMC_ESTATE, "no bond field (rv == 0)");
    size_t n = (size_t)h->ltrot * h->models[h->chains[chain].model]->nn_nf * d.N;
    for (size_t e = 0; e < n; ++e)
        if (v[e] < 1 || v[e] > 2) return fail(DQMC_EINVAL, "bond field value out of range 1..2");
    CK(copy_sync(h->st, d.vconf, v, n * sizeof(int32_t), cudaMemcpyHostToDevice));
    h->started = 0;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_vconf(dqmc_handle* h, int chain, int32_t* v) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    if (!d.vconf) return fail(DQMC_ESTATE, "no bond field (rv == 0)");
    size_t n = (size_t)h->ltrot * h->models[h->chains[chain].model]->nn_nf * d.N;
    CK(copy_sync(h->st, v, d.vconf, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

// plaquette field conf_plqu of one chain (dqmc_input_plqconf / dqmc_output_plqconf)
extern "C" int dqmc_gpu_set_conf_plq(dqmc_handle* h, int chain, const int32_t* v) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (!v) return fail(DQMC_EINVAL, "null field");
    const ChainDev& d = h->chains[chain].dev;
    const HostModel& m = *h->models[h->chains[chain].model];
    if (!d.conf_plq) return fail(DQMC_ESTATE, "no plaquette field (rhub_plq == 0)");
    const size_t n = (size_t)h->ltrot * m.lq;
    for (size_t e = 0; e < n; ++e)
        if (v[e] < 1 || v[e] > m.plq_lcomp) return fail(DQMC_EINVAL, "plaquette field value out of range 1..lcomp");
    CK(copy_sync(h->st, d.conf_plq, v, n * sizeof(int32_t), cudaMemcpyHostToDevice));
    h->started = 0;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_conf_plq(dqmc_handle* h, int chain, int32_t* v) {
    int rc = chk_chain(h, chain); if (rc) return rc;
    if (!v) return fail(DQMC_EINVAL, "null field");
    const ChainDev& d = h->chains[chain].dev;
    if (!d.conf_plq) return fail(DQMC_ESTATE, "no plaquette field (rhub_plq == 0)");
    const size_t n = (size_t)h->ltrot * h->models[h->chains[chain].model]->lq;
    CK(copy_sync(h->st, v, d.conf_plq, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_get_trial(dqmc_handle* h, int chain, double* proj, double* w) {
    int rc = chk_proj(h, chain); if (rc) return rc;
    const ChainHost& ch = h->chains[chain];
    if (proj) memcpy(proj, ch.trial.data(), ch.trial.size() * sizeof(zc));
    if (w) memcpy(w, ch.trial_w.data(), ch.trial_w.size() * sizeof(double));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_trial(dqmc_handle* h, int chain, const double* proj) {
    int rc = chk_proj(h, chain); if (rc) return rc;
    ChainHost& ch = h->chains[chain];
    memcpy(ch.trial.data(), proj, ch.trial.size() * sizeof(zc));
    h->started = 0;
    return upload_trial(h, chain);
}

extern "C" int dqmc_gpu_get_proj(dqmc_handle* h, int chain, double* ur, double* ul, double* ulrinv) {
    int rc = chk_proj(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    int N = d.N, ne = h->models[h->chains[chain].model]->p.ne;
    size_t Nne = (size_t)N * ne;
    if (ur) CK(copy_sync(h->st, ur, d.UR, Nne * sizeof(zc), cudaMemcpyDeviceToHost));
    if (ul) {
        std::vector<zc> t(Nne);
        CK(copy_sync(h->st, t.data(), d.ULT, Nne * sizeof(zc), cudaMemcpyDeviceToHost));
        zc* o = (zc*)ul;
        for (int l = 0; l < ne; ++l)
            for (int i = 0; i < N; ++i) o[l + (size_t)i * ne] = t[i + (size_t)l * N];
    }
    if (ulrinv) CK(copy_sync(h->st, ulrinv, d.ULRINV, (size_t)ne * ne * sizeof(zc), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_set_proj(dqmc_handle* h, int chain, const double* ur, const double* ul, const double* ulrinv) {
    int rc = chk_proj(h, chain); if (rc) return rc;
    const ChainDev& d = h->chains[chain].dev;
    int N = d.N, ne = h->models[h->chains[chain].model]->p.ne;
    size_t Nne = (size_t)N * ne;
    if (ur) CK(copy_sync(h->st, d.UR, ur, Nne * sizeof(zc), cudaMemcpyHostToDevice));
    if (ul) {
        std::vector<zc> t(Nne);
        const zc* in = (const zc*)ul;
        for (int l = 0; l < ne; ++l)
            for (int i = 0; i < N; ++i) t[i + (size_t)l * N] = in[l + (size_t)i * ne];
        CK(copy_sync(h->st, d.ULT, t.data(), Nne * sizeof(zc), cudaMemcpyHostToDevice));
    }
    if (ulrinv) CK(copy_sync(h->st, d.ULRINV, ulrinv, (size_t)ne * ne * sizeof(zc), cudaMemcpyHostToDevice));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_proj_update(dqmc_handle* h, int nt, int nf) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->proj) return fail(DQMC_ESTATE, "not a projective handle (params.proj = 0)");
    const HostModel& m = *h->models[0];
    if (nt < 1 || nt > h->ltrot || nf < 0 || nf > m.nn_nf) return fail(DQMC_EINVAL, "nt or nf out of range");
    if (nf == 0 && m.p.rhub == 0.0) return fail(DQMC_EINVAL, "no U field (rhub == 0)");
    if (nf > 0 && m.p.rv == 0.0) return fail(DQMC_EINVAL, "no bond field (rv == 0)");
    for (int c = 0; c < h->nch; ++c) {
        const HostModel& mc = *h->models[h->chains[c].model];
        launch_sfmt_raw(h->d_chains, c, 2 * (nf > 0 ? mc.nn_lf : mc.N), h->st);
    }
    proj_update(h, nt, nf, 0, 0, 0);
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DQMC_OK;
}

extern "C" int dqmc_gpu_proj_green(dqmc_handle* h) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (!h->proj) return fail(DQMC_ESTATE, "not a projective handle (params.proj = 0)");
    clear_fail(h);
    launch_proj_ulr(h->d_chains, h->nch, PMAT_ULRINV, 0, 0, -1, h->st);
    launch_proj_green(h->d_chains, h->nch, PMAT_ULRINV, PMAT_G, h->ctas_per_chain, h->st);
    return finish_checked(h, 0);
}

// ---------------------------------------------------------------------------
// learned effective action (kern_nn.cu) and global block moves (kern_block.cu)
// ---------------------------------------------------------------------------
struct dqmc_nn {
    int Lt = 0, L = 0, V = 0, maxB = 0, step = 0, nsm = 148;
    float b3 = 0.f;
    float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *W2T = nullptr, *W2R = nullptr, *h1 = nullptr, *h2 = nullptr, *dp2 = nullptr;
    int8_t* fbuf = nullptr;
    double *S = nullptr, *r = nullptr;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
};

static NNW nn_w(const dqmc_nn* nn) {
    NNW w;
    w.W1 = nn->theta; w.b1 = nn->theta + NN_GB1; w.W2T = nn->W2T; w.W2R = nn->W2R;
    w.b2 = nn->theta + NN_GB2; w.w3 = nn->theta + NN_GW3; w.b3 = nn->b3;
    return w;
}
static NNIn nn_in_fields(const dqmc_nn* nn) {
    NNIn in;
    in.mode = 0; in.f8 = nn->fbuf; in.chains = nullptr;
    in.Lt = nn->Lt; in.L = nn->L; in.V = nn->V; in.t_lo = 0; in.nT = nn->Lt;
    return in;
}

extern "C" int dqmc_nn_nparams(void) { return NN_NPARAM; }

extern "C" int dqmc_nn_destroy(dqmc_nn* nn) {
    if (!nn) return DQMC_OK;
    if (nn->st) cudaStreamSynchronize(nn->st);
    for (void* p : nn->allocs) cudaFree(p);
    if (nn->st) cudaStreamDestroy(nn->st);
    delete nn;
    return DQMC_OK;
}

extern "C" int dqmc_nn_create(int ltrot, int l, int max_batch, uint64_t seed, dqmc_nn** out) {
    if (!out || ltrot < 1 || l < 2 || max_batch < 1) return fail(DQMC_EINVAL, "invalid arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(DQMC_ECUDA, "no CUDA device");
    dqmc_nn* nn = new dqmc_nn();
    nn->Lt = ltrot; nn->L = l; nn->V = ltrot * l * l; nn->maxB = max_batch;
    cudaDeviceGetAttribute(&nn->nsm, cudaDevAttrMultiProcessorCount, 0);
    auto al = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, bytes ? bytes : 16);
        nn->allocs.push_back(p);
        return p;
    };
    size_t act = (size_t)max_batch * nn->V * 32 * sizeof(__nv_bfloat16);
    nn->theta = (float*)al(NN_NPARAM * sizeof(float));
    nn->grad = (float*)al(NN_NPARAM * sizeof(float));
    nn->m1 = (float*)al(NN_NPARAM * sizeof(float));
    nn->m2 = (float*)al(NN_NPARAM * sizeof(float));
    nn->W2T = (__nv_bfloat16*)al(32 * 872 * sizeof(__nv_bfloat16));
    nn->W2R = (__nv_bfloat16*)al(32 * 872 * sizeof(__nv_bfloat16));
    nn->h1 = (__nv_bfloat16*)al(act);
    nn->h2 = (__nv_bfloat16*)al(act);
    nn->dp2 = (__nv_bfloat16*)al(act);
    nn->fbuf = (int8_t*)al((size_t)max_batch * nn->V);
    nn->S = (double*)al((size_t)max_batch * sizeof(double));
    nn->r = (double*)al((size_t)max_batch * sizeof(double));
    if (!nn->theta || !nn->h1 || !nn->h2 || !nn->dp2 || !nn->fbuf || !nn->S || !nn->r) {
        dqmc_nn_destroy(nn);
        return fail(DQMC_ENOMEM, "device allocation failed (effective action)");
    }
    if (cudaStreamCreateWithFlags(&nn->st, cudaStreamNonBlocking) != cudaSuccess) {
        dqmc_nn_destroy(nn);
        return fail(DQMC_ECUDA, "stream");
    }
    cudaDeviceSynchronize();   // the allocations were cleared on the legacy stream
    // initial weights: uniform in +-sqrt(3/fan_in) (unit-variance pre-activations);
    // the readout w3 is scaled by 0.01 so that S starts close to a constant
    // (a sum over all sites of an O(1) readout would start with fluctuations far
    // larger than those of -log|W|)
    std::vector<float> th(NN_NPARAM, 0.f);
    uint64_t z = seed ? seed : 1;
    auto uni = [&]() {
        z += 0x9e3779b97f4a7c15ULL;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
        x ^= x >> 31;
        return ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    for (int i = 0; i < 27 * 32; ++i) th[i] = (float)(uni() * std::sqrt(3.0 / 27.0));
    for (int i = 0; i < 27 * 32 * 32; ++i) th[NN_GW2 + i] = (float)(uni() * std::sqrt(3.0 / 864.0));
    for (int i = 0; i < 32; ++i) th[NN_GW3 + i] = (float)(0.01 * uni() * std::sqrt(3.0 / 32.0));
    copy_sync(nn->st, nn->theta, th.data(), th.size() * sizeof(float), cudaMemcpyHostToDevice);
    launch_nn_pack(nn->theta, nn->W2T, nn->W2R, nn->st);
    if (cudaStreamSynchronize(nn->st) != cudaSuccess) { dqmc_nn_destroy(nn); return fail(DQMC_ECUDA, "init"); }
    *out = nn;
    return DQMC_OK;
}

extern "C" int dqmc_nn_set_params(dqmc_nn* nn, const float* theta) {
    if (!nn || !theta) return fail(DQMC_EINVAL, "invalid arguments");
    CK(copy_sync(nn->st, nn->theta, theta, NN_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    nn->b3 = theta[NN_GB3];
    CK(cudaMemsetAsync(nn->m1, 0, NN_NPARAM * sizeof(float), nn->st));
    CK(cudaMemsetAsync(nn->m2, 0, NN_NPARAM * sizeof(float), nn->st));
    nn->step = 0;
    launch_nn_pack(nn->theta, nn->W2T, nn->W2R, nn->st);
    CK(cudaStreamSynchronize(nn->st));
    return DQMC_OK;
}

extern "C" int dqmc_nn_get_params(dqmc_nn* nn, float* theta) {
    if (!nn || !theta) return fail(DQMC_EINVAL, "invalid arguments");
    CK(copy_sync(nn->st, theta, nn->theta, NN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    theta[NN_GB3] = nn->b3;
    return DQMC_OK;
}

static int nn_load_fields(dqmc_nn* nn, const int8_t* fields, int B) {
    if (B < 1 || B > nn->maxB) return fail(DQMC_EINVAL, "batch size out of range 1..max_batch");
    CK(cudaMemcpyAsync(nn->fbuf, fields, (size_t)B * nn->V, cudaMemcpyHostToDevice, nn->st));
    return DQMC_OK;
}

extern "C" int dqmc_nn_forward(dqmc_nn* nn, const int8_t* fields, int B, double* S) {
    if (!nn || !fields || !S) return fail(DQMC_EINVAL, "invalid arguments");
    int rc = nn_load_fields(nn, fields, B); if (rc) return rc;
    CK(cudaMemsetAsync(nn->S, 0, B * sizeof(double), nn->st));
    launch_nn_forward(nn_w(nn), nn_in_fields(nn), B, nn->S, nullptr, nullptr, nn->st);
    CK(cudaMemcpyAsync(S, nn->S, B * sizeof(double), cudaMemcpyDeviceToHost, nn->st));
    CK(cudaStreamSynchronize(nn->st));
    CK(cudaGetLastError());
    if (nn_timed_out()) return fail(DQMC_ECUDA, "a tensor-core wait of the network kernels ran out");
    return DQMC_OK;
}

// forward with stored activations (S to the host), then, if r_host is given, the
// gradient of sum_b r_b S_b into grad
static int nn_fwd(dqmc_nn* nn, int B, double* S_host) {
    CK(cudaMemsetAsync(nn->S, 0, B * sizeof(double), nn->st));
    launch_nn_forward(nn_w(nn), nn_in_fields(nn), B, nn->S, nn->h1, nn->h2, nn->st);
    CK(cudaMemcpyAsync(S_host, nn->S, B * sizeof(double), cudaMemcpyDeviceToHost, nn->st));
    CK(cudaStreamSynchronize(nn->st));
    if (nn_timed_out()) return fail(DQMC_ECUDA, "a tensor-core wait of the network kernels ran out");
    return DQMC_OK;
}
static int nn_bwd(dqmc_nn* nn, int B, const double* r_host) {
    CK(cudaMemcpyAsync(nn->r, r_host, B * sizeof(double), cudaMemcpyHostToDevice, nn->st));
    CK(cudaMemsetAsync(nn->grad, 0, NN_NPARAM * sizeof(float), nn->st));
    launch_nn_backward(nn_w(nn), nn_in_fields(nn), B, nn->r, nn->h1, nn->h2, nn->dp2, nn->grad, 2 * nn->nsm, nn->st);
    return DQMC_OK;
}
static int nn_fwd_bwd(dqmc_nn* nn, int B, const double* r_host, double* S_host) {
    int rc = nn_fwd(nn, B, S_host); if (rc) return rc;
    return r_host ? nn_bwd(nn, B, r_host) : DQMC_OK;
}

extern "C" int dqmc_nn_gradient(dqmc_nn* nn, const int8_t* fields, int B, const double* r, double* S, float* grad) {
    if (!nn || !fields || !r || !S || !grad) return fail(DQMC_EINVAL, "invalid arguments");
    int rc = nn_load_fields(nn, fields, B); if (rc) return rc;
    if ((rc = nn_fwd_bwd(nn, B, r, S))) return rc;
    CK(cudaMemcpyAsync(grad, nn->grad, NN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, nn->st));
    CK(cudaStreamSynchronize(nn->st));
    CK(cudaGetLastError());
    if (nn_timed_out()) return fail(DQMC_ECUDA, "a tensor-core wait of the network kernels ran out");
    return DQMC_OK;
}

// one Adam step on the centred squared error of S against the targets y
static int nn_train_loaded(dqmc_nn* nn, const double* y, int B, double lr, double* loss) {
    std::vector<double> S(B), r(B);
    int rc = nn_fwd(nn, B, S.data()); if (rc) return rc;
    double mean = 0.0;
    for (int b = 0; b < B; ++b) mean += (S[b] - y[b]) / B;
    double l = 0.0;
    for (int b = 0; b < B; ++b) {
        double d = S[b] - y[b] - mean;
        l += d * d / B;
        r[b] = 2.0 * d / B;
    }
    if ((rc = nn_bwd(nn, B, r.data()))) return rc;   // the activations of the forward above
    nn->step += 1;
    const float b1c = 1.f - (float)std::pow(0.9, nn->step), b2c = 1.f - (float)std::pow(0.999, nn->step);
    launch_nn_adam(nn->theta, nn->grad, nn->m1, nn->m2, NN_NPARAM, (float)lr, b1c, b2c, nn->W2T, nn->W2R, nn->st);
    CK(cudaStreamSynchronize(nn->st));
    CK(cudaGetLastError());
    if (loss) *loss = l;
    return DQMC_OK;
}

extern "C" int dqmc_nn_train_step(dqmc_nn* nn, const int8_t* fields, const double* y, int B, double lr, double* loss) {
    if (!nn || !fields || !y) return fail(DQMC_EINVAL, "invalid arguments");
    int rc = nn_load_fields(nn, fields, B); if (rc) return rc;
    return nn_train_loaded(nn, y, B, lr, loss);
}

// ---- recording of training pairs during the sweeps ----
extern "C" int dqmc_gpu_record(dqmc_handle* h, int capacity) {
    if (!h) return fail(DQMC_EINVAL, "null handle");
    if (h->proj) return fail(DQMC_ESTATE, "recording is for the finite-temperature sweep");
    if (capacity <= 0) { h->rec_on = 0; return DQMC_OK; }
    int V = h->ltrot * h->chains[0].dev.N;
    for (auto& ch : h->chains)
        if (ch.dev.N * h->ltrot != V) return fail(DQMC_EINVAL, "recording needs chains of one size");
    if (capacity != h->rec_cap) {
        // a captured sweep that records still points at the old buffers
        CK(cudaStreamSynchronize(h->st));
        drop_sweep_graph(h);
        dfree(h, h->rec_f);
        dfree(h, h->rec_v);
        dfree(h, h->rec_count);
        h->rec_f = nullptr; h->rec_v = nullptr; h->rec_count = nullptr; h->rec_cap = 0;
        h->rec_f = (int8_t*)dalloc(h, (size_t)capacity * V);
        h->rec_v = (double*)dalloc(h, (size_t)capacity * sizeof(double));
        h->rec_count = (int*)dalloc(h, sizeof(int));
        if (!h->rec_f || !h->rec_v || !h->rec_count) return fail(DQMC_ENOMEM, "record buffers");
        h->rec_cap = capacity;
    }
    h->rec_V = V;
    CK(cudaMemsetAsync(h->rec_count, 0, sizeof(int), h->st));
    CK(cudaStreamSynchronize(h->st));
    h->rec_on = 1;
    return DQMC_OK;
}

extern "C" int dqmc_gpu_record_count(dqmc_handle* h) {
    if (!h || !h->rec_count) return 0;
    int n = 0;
    copy_sync(h->st, &n, h->rec_count, sizeof(int), cudaMemcpyDeviceToHost);
    long long tot = (long long)n * h->nch;
    return (int)std::min<long long>(tot, h->rec_cap);
}

extern "C" int dqmc_gpu_record_get(dqmc_handle* h, int i, int8_t* field, double* value) {
    if (!h || !h->rec_f || i < 0 || i >= h->rec_cap) return fail(DQMC_EINVAL, "record index out of range");
    if (field) CK(copy_sync(h->st, field, h->rec_f + (size_t)i * h->rec_V, h->rec_V, cudaMemcpyDeviceToHost));
    if (value) CK(copy_sync(h->st, value, h->rec_v + i, sizeof(double), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

extern "C" int dqmc_gpu_record_values(dqmc_handle* h, double* values) {
    if (!h || !h->rec_v || !values) return fail(DQMC_EINVAL, "no record buffer");
    CK(copy_sync(h->st, values, h->rec_v, (size_t)h->rec_cap * sizeof(double), cudaMemcpyDeviceToHost));
    return DQMC_OK;
}

// one Adam step on recorded pairs idx[0..B) of the handle (targets -values, i.e.
// the effective action is fitted to -log|W| up to a constant)
extern "C" int dqmc_nn_train_recorded(dqmc_nn* nn, dqmc_handle* h, const int32_t* idx, const double* y, int B,
                                      double lr, double* loss) {
    if (!nn || !h || !idx || !y || !h->rec_f) return fail(DQMC_EINVAL, "invalid arguments");
    if (B < 1 || B > nn->maxB) return fail(DQMC_EINVAL, "batch size out of range 1..max_batch");
    if (h->rec_V != nn->V) return fail(DQMC_EINVAL, "field size differs from the effective action's");
    CK(cudaStreamSynchronize(h->st));
    for (int b = 0; b < B; ++b) {
        if (idx[b] < 0 || idx[b] >= h->rec_cap) return fail(DQMC_EINVAL, "record index out of range");
        CK(cudaMemcpyAsync(nn->fbuf + (size_t)b * nn->V, h->rec_f + (size_t)idx[b] * nn->V, nn->V,
                           cudaMemcpyDeviceToDevice, nn->st));
    }
    return nn_train_loaded(nn, y, B, lr, loss);
}

// One Adam step on differences of recorded pairs: loss = mean over b of
// ((S(field idx_b[b]) - S(field idx_a[b])) - dy[b])^2, so that the network
// learns how log|W| changes between nearby fields (the pairs of one chain one
// stabilisation apart differ by one interval of local updates).
extern "C" int dqmc_nn_train_recorded_pairs(dqmc_nn* nn, dqmc_handle* h, const int32_t* idx_a, const int32_t* idx_b,
                                            const double* dy, int B, double lr, double* loss) {
    if (!nn || !h || !idx_a || !idx_b || !dy || !h->rec_f) return fail(DQMC_EINVAL, "invalid arguments");
    if (B < 1 || 2 * B > nn->maxB) return fail(DQMC_EINVAL, "2 B must be within 1..max_batch");
    if (h->rec_V != nn->V) return fail(DQMC_EINVAL, "field size differs from the effective action's");
    CK(cudaStreamSynchronize(h->st));
    for (int b = 0; b < 2 * B; ++b) {
        const int i = b < B ? idx_a[b] : idx_b[b - B];
        if (i < 0 || i >= h->rec_cap) return fail(DQMC_EINVAL, "record index out of range");
        CK(cudaMemcpyAsync(nn->fbuf + (size_t)b * nn->V, h->rec_f + (size_t)i * nn->V, nn->V,
                           cudaMemcpyDeviceToDevice, nn->st));
    }
    std::vector<double> S(2 * B), r(2 * B);
    int rc = nn_fwd(nn, 2 * B, S.data()); if (rc) return rc;
    double l = 0.0;
    for (int b = 0; b < B; ++b) {
        const double d = (S[B + b] - S[b]) - dy[b];
        l += d * d / B;
        r[b] = -2.0 * d / B;
        r[B + b] = 2.0 * d / B;
    }
    if ((rc = nn_bwd(nn, 2 * B, r.data()))) return rc;
    nn->step += 1;
    const float b1c = 1.f - (float)std::pow(0.9, nn->step), b2c = 1.f - (float)std::pow(0.999, nn->step);
    launch_nn_adam(nn->theta, nn->grad, nn->m1, nn->m2, NN_NPARAM, (float)lr, b1c, b2c, nn->W2T, nn->W2R, nn->st);
    CK(cudaStreamSynchronize(nn->st));
    CK(cudaGetLastError());
    if (loss) *loss = l;
    return DQMC_OK;
}

// ---- global block moves inside the 0b sweep ----
static int enable_blocks(dqmc_handle* h) {
    if (h->blocks) return DQMC_OK;
    for (auto& ch : h->chains) {
        ChainDev& d = ch.dev;
        int N = d.N;
        d.blk = (int*)dalloc(h, (size_t)(N + 8) * sizeof(int));
        d.Gsave = (double2*)dalloc(h, (size_t)N * N * sizeof(double2));
        d.confsave = (int32_t*)dalloc(h, (size_t)NN_BLK_T * N * sizeof(int32_t));
        if (!d.blk || !d.Gsave || !d.confsave) return fail(DQMC_ENOMEM, "block buffers");
    }
    h->d_org = (int*)dalloc(h, (size_t)h->nch * 3 * sizeof(int));
    h->d_u = (double*)dalloc(h, (size_t)h->nch * 2 * sizeof(double));
    h->d_S = (double*)dalloc(h, (size_t)h->nch * 2 * sizeof(double));
    std::vector<ChainDev> v(h->nch);
    for (int c = 0; c < h->nch; ++c) v[c] = h->chains[c].dev;
    CK(copy_sync(h->st, h->d_chains, v.data(), sizeof(ChainDev) * h->nch, cudaMemcpyHostToDevice));
    h->blocks = 1;
    if (h->sweep_graph) { cudaGraphExecDestroy(h->sweep_graph); h->sweep_graph = nullptr; }
    return DQMC_OK;
}

static uint64_t blk_next(uint64_t& z) {
    z += 0x9e3779b97f4a7c15ULL;
    uint64_t x = z;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// one block proposal with its first slice at nt = t0 (G at the update point of t0)
static void block_move(dqmc_handle* h, dqmc_nn* nn, int t0) {
    const HostModel& m = *h->models[0];
    const int L = m.p.l1, nch = h->nch;
    std::vector<int> org(3 * nch);
    std::vector<double> u(2 * nch);
    for (int c = 0; c < nch; ++c) {
        org[3 * c] = t0 - 1;
        org[3 * c + 1] = (int)(blk_next(h->blk_rng) % (uint64_t)L);
        org[3 * c + 2] = (int)(blk_next(h->blk_rng) % (uint64_t)L);
        u[2 * c] = ((double)(blk_next(h->blk_rng) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        u[2 * c + 1] = ((double)(blk_next(h->blk_rng) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    cudaMemcpyAsync(h->d_org, org.data(), org.size() * sizeof(int), cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->d_u, u.data(), u.size() * sizeof(double), cudaMemcpyHostToDevice, h->st);
    launch_blk_setup(h->d_chains, nch, h->d_org, L, h->st);
    cudaMemsetAsync(h->d_S, 0, 2 * nch * sizeof(double), h->st);
    NNIn in;
    in.mode = 1; in.f8 = nullptr; in.chains = h->d_chains;
    in.Lt = nn->Lt; in.L = nn->L; in.V = nn->V;
    in.t_lo = t0 - 1 - 2; in.nT = NN_BLK_T + 4;
    launch_nn_forward(nn_w(nn), in, 2 * nch, h->d_S, nullptr, nullptr, h->st);
    launch_blk_begin(h->d_chains, nch, h->d_S, h->d_u, t0, NN_BLK_T, h->st);
    for (int j = 0; j < NN_BLK_T; ++j) {
        launch_update(h->d_chains, nch, t0 + j, 0, h->st, 1);
        if (j + 1 < NN_BLK_T) {
            PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
            prog_k(m, pl, PW_FWD, 1); prog_k(m, pl, PW_FWD, 0); prog_v(m, pl, PW_FWD, t0 + j + 1);
            prog_k(m, pr, PW_INV, 1); prog_k(m, pr, PW_INV, 0); prog_v(m, pr, PW_INV, t0 + j + 1);
            launch_prog(h, MAT_G, pl, 0);
            launch_prog(h, MAT_G, pr, 1);
        }
    }
    launch_blk_decide(h->d_chains, nch, h->st);
    // back to the update point of t0 through the (possibly flipped) slices
    for (int j = NN_BLK_T - 1; j >= 1; --j) {
        PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
        prog_v(m, pl, PW_INV, t0 + j); prog_k(m, pl, PW_INV, 1); prog_k(m, pl, PW_INV, 0);
        prog_v(m, pr, PW_FWD, t0 + j); prog_k(m, pr, PW_FWD, 1); prog_k(m, pr, PW_FWD, 0);
        launch_prog(h, MAT_G, pl, 0);
        launch_prog(h, MAT_G, pr, 1);
    }
    launch_blk_end(h->d_chains, nch, t0, NN_BLK_T, h->st);
}

// dqmc_ft_sweep_0b with a block proposal at the first slice of the chosen
// stabilisation intervals (intervals n with n % 2 == parity; the slice offset
// inside the interval is drawn so the block stays inside it)
static void enqueue_0b_blocks(dqmc_handle* h, dqmc_nn* nn, int lupdate, int lmeasure, int parity) {
    const HostModel& m = *h->models[0];
    int lt = h->ltrot;
    std::vector<int> start(lt + 2, 0);
    for (int n = 1; n <= h->nst; ++n) {
        if (n % 2 != parity) continue;
        int a = m.wrap_step[(n - 1) * 2], b = m.wrap_step[(n - 1) * 2 + 1];
        int len = b - a + 1;
        if (len < NN_BLK_T) continue;
        int off = (int)(blk_next(h->blk_rng) % (uint64_t)(len - NN_BLK_T + 1));
        start[a + off] = 1;
    }
    launch_stack_identity(h->d_chains, h->nch, 0, h->st);
    if (lupdate) launch_sfmt(h->d_chains, h->nch, lt, h->st);
    for (int nt = 1; nt <= lt; ++nt) {
        int visit = nt - 1;
        PropProg pl; pl.n = 0; PropProg pr; pr.n = 0;
        prog_k(m, pl, PW_FWD, 0);
        prog_v(m, pl, PW_FWD, nt);
        prog_k(m, pr, PW_INV, 0);
        prog_v(m, pr, PW_INV, nt);
        launch_prog(h, MAT_G, pl, 0);
        launch_prog(h, MAT_G, pr, 1);
        if (start[nt]) block_move(h, nn, nt);
        if (lupdate) launch_update(h->d_chains, h->nch, nt, visit, h->st);
        pl.n = 0; pr.n = 0;
        prog_k(m, pl, PW_FWD, 1);
        prog_k(m, pr, PW_INV, 1);
        launch_prog(h, MAT_G, pl, 0);
        launch_prog(h, MAT_G, pr, 1);
        if (lmeasure) launch_measure_h(h);
        if (m.iwrap_nt[nt] > 0) stab_0b(h, m.iwrap_nt[nt], 1);
    }
}

extern "C" int dqmc_gpu_sweep_learned(dqmc_handle* h, dqmc_nn* nn, int n, int lupdate, int lmeasure, uint64_t seed) {
    if (!h || !nn) return fail(DQMC_EINVAL, "null argument");
    if (!h->started) return fail(DQMC_ESTATE, "sweep before sweep_start");
    if (h->proj) return fail(DQMC_ESTATE, "block moves are for the finite-temperature sweep");
    const HostModel& m = *h->models[0];
    if (h->models.size() != 1 || m.p.lattice != DQMC_LATT_SQUARE || m.p.l1 != nn->L || m.p.l2 != nn->L ||
        m.p.ltrot != nn->Lt)
        return fail(DQMC_EINVAL, "the effective action's lattice differs from the handle's (square L x L, ltrot)");
    if (m.lcomp != 2) return fail(DQMC_EINVAL, "block flips need a two-valued HS field (lcomp = 2)");
    if (m.p.rhub == 0.0) return fail(DQMC_EINVAL, "no HS field (rhub == 0)");
    if (m.plq_on || m.p.rv != 0.0) return fail(DQMC_EINVAL, "block moves need the U field alone (rhub_plq = rv = 0)");
    int rc = enable_blocks(h); if (rc) return rc;
    if (seed) h->blk_rng = seed;
    clear_fail(h);
    cudaEvent_t e0 = h->ev0, e1 = h->ev1;
    CK(cudaEventRecord(e0, h->st));
    for (int i = 0; i < n; ++i) {
        enqueue_b0(h, lupdate, lmeasure);
        enqueue_0b_blocks(h, nn, lupdate, lmeasure, (int)(blk_next(h->blk_rng) & 1));
        h->after_b0 = 0;
    }
    CK(cudaEventRecord(e1, h->st));
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    h->last_ms = n > 0 ? ms / n : 0.0;
    return finish_checked(h, 1);
}
