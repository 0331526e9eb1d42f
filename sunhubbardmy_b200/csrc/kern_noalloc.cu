// Allocation-free QR with log det Q: dqmc_gpu_qr_logdet_noalloc.
//
// Some host codes cannot allocate device memory themselves -- for example a
// simulation whose device memory is handed out by a pool it does not
// control, or a long production run that must not allocate once it has
// started.  This entry point serves them: it factors a caller-owned N x N
// complex matrix (blocked Householder QR, explicit Q, log det Q, the same
// device code as the stabilisation kernel) using only the buffers the caller
// passes plus a fixed scratch area that is part of the library image.
//
// The scratch is a file-scope __device__ array sized for N <= DQMC_NOALLOC_MAX_N
// (about 0.55 MB); every GPU that loads the library holds it until the process
// exits.  In host code the array's name is only a host-side stand-in, so its
// device address is looked up once per device with cudaGetSymbolAddress (on
// the first call made while that device is current) and then passed to the
// kernel.  All calls share the array: no part of it is read before the same
// call has written it, so nothing has to be cleared between calls, but two
// calls whose kernels overlap on the GPU race on it.
#include <atomic>
#include <cstdio>
#include <mutex>

#include "../../include/dqmc_gpu.h"
#include "linalg.cuh"

#define DQMC_NOALLOC_MAX_N 512

// scratch layout (double2 units): Vs [N*16], Ws [16*N], Ws2 [16*N],
// T [(N/16+1)*256], tau [N]
#define NOALLOC_ELEMS (3 * DQMC_NOALLOC_MAX_N * QR_NB + (DQMC_NOALLOC_MAX_N / QR_NB + 1) * QR_NB * QR_NB + DQMC_NOALLOC_MAX_N)

static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_ELEMS];

struct NoallocSmem {
    LinalgSmem L;
    double red[64];
};

static size_t noalloc_smem_bytes(int n) {
    size_t a = QR_PANEL_ELEMS(n), b = GemmBig::SMEM_ELEMS;
    if ((size_t)GemmWide::SMEM_ELEMS > b) b = GemmWide::SMEM_ELEMS;
    return (a > b ? a : b) * sizeof(double2) + sizeof(NoallocSmem) + 64;
}

__global__ void __launch_bounds__(256) k_qr_noalloc(int n, double2* A, double2* Q, double2* logdet, double2* scratch) {
    extern __shared__ double2 nsm[];
    size_t off = (QR_PANEL_ELEMS(n) > (size_t)GemmBig::SMEM_ELEMS) ? QR_PANEL_ELEMS(n) : (size_t)GemmBig::SMEM_ELEMS;
    NoallocSmem* S = (NoallocSmem*)(nsm + off);
    LinalgScratch sc;
    sc.Vs = scratch;
    sc.Ws = scratch + (size_t)n * QR_NB;
    sc.Ws2 = sc.Ws + (size_t)QR_NB * n;
    sc.T = sc.Ws2 + (size_t)QR_NB * n;
    sc.tau = sc.T + (size_t)(n / QR_NB + 1) * QR_NB * QR_NB;
    cta_qr(A, n, sc, nsm, nsm, &S->L);
    double2 ld = cta_logdet_q(sc.tau, n, S->red);
    if (threadIdx.x == 0) *logdet = ld;
    __syncthreads();
    cta_form_q(A, n, Q, sc, nsm);
}

#define NOALLOC_MAX_DEVICES 64
// per-device set-up (scratch address, shared-memory attribute), done once per
// device under a lock so that host threads making their first call on a
// device at the same time do not race on it; later calls only read the
// published address.  The address belongs to the device's current context: a
// cudaDeviceReset invalidates it, and calls after such a reset are not
// supported.
static std::atomic<void*> g_noalloc_ptr[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_lock;

static thread_local char g_noalloc_err[256] = "";

extern "C" const char* dqmc_gpu_noalloc_error(void) { return g_noalloc_err; }

extern "C" int dqmc_gpu_qr_logdet_noalloc(int n, double* a, double* q, double* logdetq, void* stream) {
    if (n < 1 || n > DQMC_NOALLOC_MAX_N) {
        snprintf(g_noalloc_err, sizeof(g_noalloc_err),
                 "dqmc_gpu_qr_logdet_noalloc: n = %d outside 1..%d (the fixed scratch size)", n, DQMC_NOALLOC_MAX_N);
        return DQMC_EINVAL;
    }
    if (!a || !q || !logdetq) {
        snprintf(g_noalloc_err, sizeof(g_noalloc_err), "dqmc_gpu_qr_logdet_noalloc: null pointer argument");
        return DQMC_EINVAL;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        snprintf(g_noalloc_err, sizeof(g_noalloc_err), "dqmc_gpu_qr_logdet_noalloc: no usable current device");
        return DQMC_ECUDA;
    }
    void* scratch = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        // first call on this device: device address of the static scratch and
        // the kernel's shared-memory limit, published only once both are set
        std::lock_guard<std::mutex> lock(g_noalloc_lock);
        scratch = g_noalloc_ptr[dev].load(std::memory_order_acquire);
        if (!scratch) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                snprintf(g_noalloc_err, sizeof(g_noalloc_err), "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
                return DQMC_ECUDA;
            }
            e = cudaFuncSetAttribute(k_qr_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) {
                snprintf(g_noalloc_err, sizeof(g_noalloc_err), "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
                return DQMC_ECUDA;
            }
            g_noalloc_ptr[dev].store(p, std::memory_order_release);
            scratch = p;
        }
    }
    k_qr_noalloc<<<1, 256, noalloc_smem_bytes(n), (cudaStream_t)stream>>>(
        n, (double2*)a, (double2*)q, (double2*)logdetq, (double2*)scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_noalloc_err, sizeof(g_noalloc_err), "k_qr_noalloc launch: %s", cudaGetErrorString(e));
        return DQMC_ECUDA;
    }
    return DQMC_OK;
}
