// Shared device-side definitions for the B200 DQMC sweep.
//
// Complex FP64 is stored as double2 (x = real, y = imag), matrices are
// column-major with leading dimension N, exactly the Fortran layout of the
// reference's gfunc containers (src/dqmc_basic_data.f90:8-19).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DQ_DEV __device__ __forceinline__

typedef double2 cplx;

DQ_DEV cplx cmk(double r, double i) { return make_double2(r, i); }
DQ_DEV cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
DQ_DEV cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
DQ_DEV cplx cmul(cplx a, cplx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DQ_DEV cplx cconj(cplx a) { return cmk(a.x, -a.y); }
DQ_DEV cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
DQ_DEV double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
DQ_DEV double cabsd(cplx a) { return hypot(a.x, a.y); }
// a * conj(b)
DQ_DEV cplx cmulc(cplx a, cplx b) { return cmk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
// conj(a) * b
DQ_DEV cplx ccmul(cplx a, cplx b) { return cmk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
// a * b + c (complex fma)
DQ_DEV cplx cfma(cplx a, cplx b, cplx c) {
    return cmk(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
DQ_DEV cplx cdiv(cplx a, cplx b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return cmk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.y + b.x * r;
        return cmk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
DQ_DEV cplx cexpi(double t) { double s, c; sincos(t, &s, &c); return cmk(c, s); }
DQ_DEV cplx clog_(cplx z) { return cmk(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

// column-major element access
#define MIDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

// ---- block reductions (blockDim.x multiple of 32, <= 1024) ----
template <typename T>
DQ_DEV T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
DQ_DEV double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over the block; every thread gets the result.  red must hold 32 doubles.
DQ_DEV double block_sum(double v, double* red) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = (lane < nw) ? red[lane] : 0.0;
    t = warp_sum(t);
    return t;
}
DQ_DEV double block_max(double v, double* red) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = (lane < nw) ? red[lane] : 0.0;
    return warp_max(t);
}
DQ_DEV cplx block_csum(cplx v, double* red) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v.x = warp_sum(v.x);
    v.y = warp_sum(v.y);
    __syncthreads();
    if (lane == 0) { red[2 * w] = v.x; red[2 * w + 1] = v.y; }
    __syncthreads();
    cplx t = (lane < nw) ? cmk(red[2 * lane], red[2 * lane + 1]) : cmk(0, 0);
    t.x = warp_sum(t.x);
    t.y = warp_sum(t.y);
    return t;
}
