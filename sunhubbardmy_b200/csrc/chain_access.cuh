// Matrix selection and small device helpers shared by the kernels.
#pragma once
#include "common.cuh"
#include "dqmc_types.h"

// matrix ids used by the host to address per-chain matrices
enum { MAT_G = 0, MAT_GNEW = 1, MAT_W0 = 2, MAT_U0 = 100, MAT_V0 = 400 };

DQ_DEV double2* chain_mat(const ChainDev& c, int id) {
    size_t nn = (size_t)c.N * c.N;
    if (id == MAT_G) return c.G;
    if (id == MAT_GNEW) return c.Gnew;
    if (id >= MAT_V0) return c.V + (size_t)c.slotmap[id - MAT_V0] * nn;
    if (id >= MAT_U0) return c.U + (size_t)c.slotmap[id - MAT_U0] * nn;
    return c.W[id - MAT_W0];
}

// In-place DFT of a length-n line (element stride `st`) in shared memory.
// sign = -1: forward exp(-2 pi i j k / n); sign = +1: backward.  tw[k] =
// exp(-2 pi i k / n).  Unnormalised.  Power-of-two lengths use an iterative
// radix-2 transform; other lengths a direct O(n^2) sum (n <= 64).
DQ_DEV void line_dft(double2* x, int n, int st, const double2* tw, int sign) {
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
