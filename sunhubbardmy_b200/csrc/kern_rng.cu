// SFMT-19937 on the device, one warp per chain.
//
// Reference: lib/m_spring.f90:187-379 (spring_sfmt_init/_source/_kernel/_core);
// spring_sfmt_stream maps the 32-bit output u to (u + 0.5) / 2^32.  The
// generator state (624 words + read index) lives in the chain's device memory
// and advances exactly as the reference's does, so the draws of a chain are
// the reference's draws for the same seed.  The draws of a whole half sweep
// (two per site and slice) are produced ahead of the update kernels, which read
// them in visiting order.
#include "chain_access.cuh"
#include "kernels.h"

#define SFMT_N 156
#define SFMT_N32 624
#define SFMT_POS1 122

__device__ __forceinline__ void sfmt_recursion(uint32_t* r, const uint32_t* a, const uint32_t* b,
                                               const uint32_t* cc, const uint32_t* d) {
    const uint32_t msk[4] = {0xdfffffefU, 0xddfecb7fU, 0xbffaffffU, 0xbffffff6U};
    // x = a << 8 (128-bit), y = c >> 8 (128-bit)
    uint64_t ah = ((uint64_t)a[3] << 32) | a[2], al = ((uint64_t)a[1] << 32) | a[0];
    uint64_t ch = ((uint64_t)cc[3] << 32) | cc[2], cl = ((uint64_t)cc[1] << 32) | cc[0];
    uint64_t xh = (ah << 8) | (al >> 56), xl = al << 8;
    uint64_t yh = ch >> 8, yl = (cl >> 8) | (ch << 56);
    uint32_t x[4] = {(uint32_t)xl, (uint32_t)(xl >> 32), (uint32_t)xh, (uint32_t)(xh >> 32)};
    uint32_t y[4] = {(uint32_t)yl, (uint32_t)(yl >> 32), (uint32_t)yh, (uint32_t)(yh >> 32)};
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = a[k] ^ x[k] ^ ((b[k] >> 11) & msk[k]) ^ y[k] ^ (d[k] << 18);
}

__device__ void sfmt_gen_all(uint32_t* st) {
    uint32_t* r1 = st + 4 * (SFMT_N - 2);
    uint32_t* r2 = st + 4 * (SFMT_N - 1);
    int i;
    for (i = 0; i < SFMT_N - SFMT_POS1; ++i) {
        uint32_t out[4];
        sfmt_recursion(out, st + 4 * i, st + 4 * (i + SFMT_POS1), r1, r2);
        for (int k = 0; k < 4; ++k) st[4 * i + k] = out[k];
        r1 = r2; r2 = st + 4 * i;
    }
    for (; i < SFMT_N; ++i) {
        uint32_t out[4];
        sfmt_recursion(out, st + 4 * i, st + 4 * (i + SFMT_POS1 - SFMT_N), r1, r2);
        for (int k = 0; k < 4; ++k) st[4 * i + k] = out[k];
        r1 = r2; r2 = st + 4 * i;
    }
}

// count = slices * rps draws per chain (slices > 0; rps = words per time slice
// of the chain's model), or exactly -slices draws.  One warp per chain: the
// state is held in shared memory while lane 0 runs the recursion (the serial
// part), and the warp copies each block of 624 outputs to the chain's draw
// buffer with coalesced stores.
#define SFMT_WARPS 4
__global__ void __launch_bounds__(32 * SFMT_WARPS) k_sfmt_fill(const ChainDev* __restrict__ chains, int ch0,
                                                               int nchains, int slices) {
    __shared__ uint32_t sst[SFMT_WARPS][SFMT_N32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ch = ch0 + blockIdx.x * SFMT_WARPS + w;
    if (ch >= ch0 + nchains) return;      // whole warps; no block barrier below
    const int count = slices > 0 ? slices * chains[ch].md->rps : -slices;
    uint32_t* gst = chains[ch].sfmt;
    uint32_t* out = chains[ch].rnd;
    uint32_t* s = sst[w];
    for (int e = lane; e < SFMT_N32; e += 32) s[e] = gst[e];
    int idx = (int)gst[SFMT_N32];
    __syncwarp();
    for (int k = 0; k < count;) {
        if (idx >= SFMT_N32) {
            if (lane == 0) sfmt_gen_all(s);
            __syncwarp();
            idx = 0;
        }
        const int n = min(SFMT_N32 - idx, count - k);
        for (int e = lane; e < n; e += 32) out[k + e] = s[idx + e];
        k += n;
        idx += n;
        __syncwarp();                     // the block is read before it is regenerated
    }
    for (int e = lane; e < SFMT_N32; e += 32) gst[e] = s[e];
    if (lane == 0) gst[SFMT_N32] = (uint32_t)idx;
}

void launch_sfmt(const ChainDev* chains, int nchains, int slices, cudaStream_t st) {
    k_sfmt_fill<<<(nchains + SFMT_WARPS - 1) / SFMT_WARPS, 32 * SFMT_WARPS, 0, st>>>(chains, 0, nchains, slices);
}

void launch_sfmt_raw(const ChainDev* chains, int chain, int count, cudaStream_t st) {
    k_sfmt_fill<<<1, 32 * SFMT_WARPS, 0, st>>>(chains, chain, 1, -count);
}
