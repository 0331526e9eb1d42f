// Global block moves with delayed acceptance, and the recording of
// (HS field, log weight) pairs for training the effective action.
//
// A block is NN_BLK_T slices x NN_BLK_Y x NN_BLK_X sites of the HS field
// (lcomp = 2), all flipped.  Stage 1 accepts with min(1, exp(-dS)), dS the
// change of the learned effective action; stage 2 with
// min(1, |Re(R phase)/Re(phase)| exp(dS)), R = W(s')/W(s) the exact weight
// ratio, obtained as the product of the forced flips' sequential ratios while
// G is wrapped through the block's slices (k_update_delay, forced mode).  The
// two stages together satisfy detailed balance for the weight |Re W| that the
// local updates sample (delayed-acceptance Metropolis-Hastings; the block flip
// is its own inverse and the block origin is uniform).
#include "chain_access.cuh"
#include "kernels.h"
#include "nn.h"

// block origin and spatial mask; org[3c..3c+2] = (t0 - 1, y0, x0)
__global__ void k_blk_setup(const ChainDev* __restrict__ chains, const int* __restrict__ org, int L) {
    const ChainDev& c = chains[blockIdx.x];
    const int N = c.N;
    const int t0 = org[3 * blockIdx.x], y0 = org[3 * blockIdx.x + 1], x0 = org[3 * blockIdx.x + 2];
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int y = i / L, x = i % L;
        const int dy = (y - y0 + L) % L, dx = (x - x0 + L) % L;
        c.blk[i] = (dy < NN_BLK_Y && dx < NN_BLK_X) ? 1 : 0;
    }
    if (threadIdx.x == 0) {
        c.blk[N] = 0; c.blk[N + 1] = 0;
        c.blk[N + 4] = t0; c.blk[N + 5] = y0; c.blk[N + 6] = x0;
    }
}

// stage 1 and the checkpoint: S[2c], S[2c+1] = effective action (slab) of the
// current and of the proposed field; u[2c], u[2c+1] = the two uniforms
__global__ void k_blk_begin(const ChainDev* __restrict__ chains, const double* __restrict__ S, const double* __restrict__ u,
                            int t0, int nsl) {
    const ChainDev& c = chains[blockIdx.y];
    const int N = c.N, ch = blockIdx.y;
    const size_t NN = (size_t)N * N;
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < NN; e += (size_t)gridDim.x * blockDim.x) c.Gsave[e] = c.G[e];
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)nsl * N; e += (size_t)gridDim.x * blockDim.x)
        c.confsave[e] = c.conf[(size_t)(t0 - 1) * N + e];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double dS = S[2 * ch + 1] - S[2 * ch];
        const int active = log(u[2 * ch]) < -dS;
        c.blk[N] = active;
        c.stats[ST_BLK_DS] = dS;
        c.stats[ST_BLK_U2] = u[2 * ch + 1];
        c.stats[ST_BLK_PH_RE] = c.stats[ST_PHASE_RE];
        c.stats[ST_BLK_PH_IM] = c.stats[ST_PHASE_IM];
        c.stats[ST_BLK_LR_RE] = 0.0;
        c.stats[ST_BLK_LR_IM] = 0.0;
        c.stats[ST_BLK_PROP] += 1.0;
        c.stats[ST_BLK_S1] += active;
    }
}

// stage 2 with the exact ratio accumulated by the forced flips
__global__ void k_blk_decide(const ChainDev* __restrict__ chains, int nchains) {
    const int ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch >= nchains) return;
    const ChainDev& c = chains[ch];
    const int N = c.N;
    int acc = 0;
    if (c.blk[N]) {
        const double2 lr = cmk(c.stats[ST_BLK_LR_RE], c.stats[ST_BLK_LR_IM]);
        const double2 ph0 = cmk(c.stats[ST_BLK_PH_RE], c.stats[ST_BLK_PH_IM]);
        // log |Re(R ph0) / Re(ph0)| with R = exp(lr)
        const double2 rp = cmul(cexpi(lr.y), ph0);
        const double rre = rp.x / ph0.x;
        if (rre != 0.0) {
            const double logr = lr.x + log(fabs(rre));
            acc = log(c.stats[ST_BLK_U2]) < logr + c.stats[ST_BLK_DS];
            // how well -dS predicts the exact log ratio, against predicting 0
            const double e1 = logr + c.stats[ST_BLK_DS];
            c.stats[ST_BLK_ERR1] += e1 * e1;
            c.stats[ST_BLK_ERR0] += logr * logr;
        }
    }
    c.blk[N + 1] = acc;
    if (acc) {
        c.stats[ST_BLK_ACC] += 1.0;
        c.stats[ST_BLK_SUMLR] += c.stats[ST_BLK_LR_RE];
    }
}

// rejected (or never proposed) blocks: G, field and phase back to the checkpoint
__global__ void k_blk_end(const ChainDev* __restrict__ chains, int t0, int nsl) {
    const ChainDev& c = chains[blockIdx.y];
    const int N = c.N;
    if (c.blk[N + 1]) return;
    const size_t NN = (size_t)N * N;
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < NN; e += (size_t)gridDim.x * blockDim.x) c.G[e] = c.Gsave[e];
    for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)nsl * N; e += (size_t)gridDim.x * blockDim.x)
        c.conf[(size_t)(t0 - 1) * N + e] = c.confsave[e];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.stats[ST_PHASE_RE] = c.stats[ST_BLK_PH_RE];
        c.stats[ST_PHASE_IM] = c.stats[ST_BLK_PH_IM];
    }
}

// append (field as +-1 int8, nflr Re log weight) of every chain; slot
// (count * nchains + chain) mod capacity; the count advances in k_record_bump
__global__ void k_record(const ChainDev* __restrict__ chains, int8_t* fields, double* vals, const int* count,
                         int capacity, int nchains, int V) {
    const ChainDev& c = chains[blockIdx.y];
    const long long slot = ((long long)count[0] * nchains + blockIdx.y) % capacity;
    int8_t* f = fields + (size_t)slot * V;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < V; e += gridDim.x * blockDim.x)
        f[e] = (int8_t)(2 * c.conf[e] - 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) vals[slot] = c.md->nflr * c.stats[ST_LOGW_RE];
}
__global__ void k_record_bump(int* count) { count[0] += 1; }

void launch_blk_setup(const ChainDev* chains, int nchains, const int* org, int L, cudaStream_t st) {
    k_blk_setup<<<nchains, 256, 0, st>>>(chains, org, L);
}
void launch_blk_begin(const ChainDev* chains, int nchains, const double* S, const double* u, int t0, int nsl, cudaStream_t st) {
    k_blk_begin<<<dim3(16, nchains), 256, 0, st>>>(chains, S, u, t0, nsl);
}
void launch_blk_decide(const ChainDev* chains, int nchains, cudaStream_t st) {
    k_blk_decide<<<(nchains + 63) / 64, 64, 0, st>>>(chains, nchains);
}
void launch_blk_end(const ChainDev* chains, int nchains, int t0, int nsl, cudaStream_t st) {
    k_blk_end<<<dim3(16, nchains), 256, 0, st>>>(chains, t0, nsl);
}
void launch_record(const ChainDev* chains, int nchains, int8_t* fields, double* vals, int* count, int capacity, int V,
                   cudaStream_t st) {
    k_record<<<dim3(8, nchains), 256, 0, st>>>(chains, fields, vals, count, capacity, nchains, V);
    k_record_bump<<<1, 1, 0, st>>>(count);
}
