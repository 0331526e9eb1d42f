// Matrix selection and small device helpers shared by the kernels.
#pragma once
#include "common.cuh"
#include "dqmc_types.h"

// matrix ids used by the host to address per-chain matrices
enum { MAT_G = 0, MAT_GNEW = 1, MAT_W0 = 2, MAT_UR = 10, MAT_ULT = 11, MAT_PROJR = 12, MAT_PROJLC = 13,
       MAT_ULRINV = 14, MAT_GT0 = 15, MAT_G0T = 16, MAT_G00 = 17, MAT_URS = 18, MAT_ULTS = 19, MAT_U0 = 100, MAT_V0 = 400, MAT_PST0 = 1000 };

DQ_DEV double2* chain_mat(const ChainDev& c, int id) {
    size_t nn = (size_t)c.N * c.N;
    if (id == MAT_G) return c.G;
    if (id == MAT_GNEW) return c.Gnew;
    if (id >= MAT_PST0) return c.Pst + (size_t)(id - MAT_PST0) * c.N * c.md->ne;
    if (id == MAT_UR) return c.UR;
    if (id == MAT_ULT) return c.ULT;
    if (id == MAT_PROJR) return c.projR;
    if (id == MAT_PROJLC) return c.projLc;
    if (id == MAT_ULRINV) return c.ULRINV;
    if (id == MAT_GT0) return c.gt0;
    if (id == MAT_G0T) return c.g0t;
    if (id == MAT_G00) return c.g00;
    if (id == MAT_URS) return c.URs;
    if (id == MAT_ULTS) return c.ULTs;
    if (id >= MAT_V0) return c.V + (size_t)c.slotmap[id - MAT_V0] * nn;
    if (id >= MAT_U0) return c.U + (size_t)c.slotmap[id - MAT_U0] * nn;
    return c.W[id - MAT_W0];
}

// Record a numerical failure of chain c (one thread calls it): the chain's
// sticky stats[ST_INFO] and the handle's fail word.  The reference stops the
// run at these points (lib/s_matrix.f90:1264-1267, dqmc_ft_sweep_b0.f90:188-194);
// the library reports them to the host instead.
DQ_DEV void chain_raise(const ChainDev& c, int code) {
    c.stats[ST_INFO] = (double)((int)c.stats[ST_INFO] | code);
    if (c.fail) atomicOr(c.fail, code);
}

// Radix-2 DFT of a length-n line held in registers (n a power of two, fully
// unrolled).  tw[k] = exp(-2 pi i k / n); sign -1 forward, +1 backward.
template <int n>
DQ_DEV void line_fft_reg(double2* x, int st, const double2* __restrict__ tw, int sign) {
    double2 r[n];
#pragma unroll
    for (int i = 0; i < n; ++i) {
        int j = 0;
#pragma unroll
        for (int b = 1, t = i; b < n; b <<= 1, t >>= 1) j = (j << 1) | (t & 1);
        r[j] = x[i * st];
    }
#pragma unroll
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = n / len;
#pragma unroll
        for (int s0 = 0; s0 < n; s0 += len)
#pragma unroll
            for (int k = 0; k < half; ++k) {
                double2 w = __ldg(&tw[k * step]);
                if (sign > 0) w.y = -w.y;
                double2 u = r[s0 + k], v = cmul(w, r[s0 + k + half]);
                r[s0 + k] = cadd(u, v);
                r[s0 + k + half] = csub(u, v);
            }
    }
#pragma unroll
    for (int i = 0; i < n; ++i) x[i * st] = r[i];
}

// In-place DFT of a length-n line (element stride `st`) in shared memory.
// sign = -1: forward exp(-2 pi i j k / n); sign = +1: backward.  tw[k] =
// exp(-2 pi i k / n).  Unnormalised.  Power-of-two lengths use an iterative
// radix-2 transform; other lengths a direct O(n^2) sum (n <= 64).
DQ_DEV void line_dft(double2* x, int n, int st, const double2* tw, int sign) {
    switch (n) {
    case 4: line_fft_reg<4>(x, st, tw, sign); return;
    case 8: line_fft_reg<8>(x, st, tw, sign); return;
    case 16: line_fft_reg<16>(x, st, tw, sign); return;
    default: break;
    }
    if ((n & (n - 1)) == 0) {
        // bit reversal
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { double2 t = x[i * st]; x[i * st] = x[j * st]; x[j * st] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int s = 0; s < n; s += len)
                for (int k = 0; k < half; ++k) {
                    double2 w = tw[k * step];
                    if (sign > 0) w.y = -w.y;
                    double2 u = x[(s + k) * st], v = cmul(w, x[(s + k + half) * st]);
                    x[(s + k) * st] = cadd(u, v);
                    x[(s + k + half) * st] = csub(u, v);
                }
        }
    } else {
        double2 tmp[64];
        for (int k = 0; k < n; ++k) {
            double2 s = cmk(0, 0);
            for (int j = 0; j < n; ++j) {
                double2 w = tw[(j * k) % n];
                if (sign > 0) w.y = -w.y;
                s = cfma(w, x[j * st], s);
            }
            tmp[k] = s;
        }
        for (int k = 0; k < n; ++k) x[k * st] = tmp[k];
    }
}
