// Descriptors shared by the effective-action kernels (kern_nn.cu) and the host.
#pragma once
#include <cuda_bf16.h>
#include "dqmc_types.h"

// proposed block of the global update: NN_BLK_T slices x NN_BLK_Y x NN_BLK_X sites
#define NN_BLK_T 8
#define NN_BLK_Y 4
#define NN_BLK_X 4

// flat FP32 parameter vector: W1 [27][32], b1 [32], W2 [27][32 ci][32 co], b2 [32], w3 [32], b3
#define NN_GB1 (27 * 32)
#define NN_GW2 (NN_GB1 + 32)
#define NN_GB2 (NN_GW2 + 27 * 32 * 32)
#define NN_GW3 (NN_GB2 + 32)
#define NN_GB3 (NN_GW3 + 32)
#define NN_NPARAM (NN_GB3 + 1)

struct NNW {
    const float* W1;
    const float* b1;
    const __nv_bfloat16* W2T;   // [32 co][872], k = tap*32 + ci        (forward)
    const __nv_bfloat16* W2R;   // [32 ci][872], k = (26-tap)*32 + co   (transposed convolution)
    const float* b2;
    const float* w3;
    float b3;
};

// where the fields come from: mode 0 = int8 +-1 fields [B][V]; mode 1 = the
// chains' HS fields (field b = chain b >> 1, odd b with the chain's proposed
// block flipped).  Outputs cover time slices t_lo .. t_lo + nT - 1 (periodic).
struct NNIn {
    int mode;
    const int8_t* f8;
    const ChainDev* chains;
    int Lt, L, V;
    int t_lo, nT;
};

int nn_nbricks(const NNIn& in);
void launch_nn_forward(const NNW& w, const NNIn& in, int B, double* S, __nv_bfloat16* h1g, __nv_bfloat16* h2g,
                       cudaStream_t st);
void launch_nn_backward(const NNW& w, const NNIn& in, int B, const double* r, const __nv_bfloat16* h1g,
                        const __nv_bfloat16* h2g, __nv_bfloat16* dp2g, float* grad, int nsm, cudaStream_t st);
void launch_nn_adam(float* theta, const float* grad, float* m1, float* m2, int n, float lr, float b1c, float b2c,
                    __nv_bfloat16* W2T, __nv_bfloat16* W2R, cudaStream_t st);
void launch_nn_pack(const float* theta, __nv_bfloat16* W2T, __nv_bfloat16* W2R, cudaStream_t st);
// 1 when a tensor-core wait of the network kernels ran out since the last call (then cleared)
int nn_timed_out();
