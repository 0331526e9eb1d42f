// Batched Hermitian eigensolver on the device: cyclic two-sided Jacobi in the
// parallel (round-robin) ordering, for the set-up eigenproblems of the sweep.
//
// Reference: s_eig_he (lib/s_matrix.f90:202-253, LAPACK zheev) as called by
// dqmc_set_h0conf.f90:484-509 (the dense kinetic exponentials from the seth0
// matrix) and by dqmc_set_proj.f90:1-78 / set_trial_h0.f90:1-29 (the trial
// wave function: the ne lowest eigenvectors of the trial Hamiltonian, one per
// walker).  zheev reduces to tridiagonal form, a sequential O(N^3) sweep that
// suits one CPU core; Jacobi instead applies N/2 independent plane rotations
// per round, all matrices and all pairs of a round in one launch, and reaches
// the same eigenpairs (eigenvalues ascending; eigenvectors up to a phase, and
// up to a unitary rotation inside a degenerate level).
//
// A round r (0 <= r < Np - 1, Np = N rounded up to even) pairs position k
// with position Np - 1 - k of the list (0, 1 + (r mod (Np-1)), ...); every
// pair of indices meets once per sweep.  Pair (p, q) rotates with
//   J = [[c, s e^{i phi}], [-s e^{-i phi}, c]],   A(p,q) = |A(p,q)| e^{i phi},
//   t = tan theta = sgn(zeta) / (|zeta| + sqrt(1 + zeta^2)),  zeta = (A(q,q) - A(p,p)) / (2 |A(p,q)|),
// the smaller annihilating angle (|theta| <= pi/4, which the cyclic method needs to
// converge), so that (J^H A J)(p,q) = 0: first A <- A J and V <- V J (columns; disjoint
// columns per pair, so the pairs of a round run concurrently), then A <- J^H A
// (rows) with the rotations of the whole round, which together is
// A <- J_r^H A J_r for the round's block-diagonal J_r.
#include "common.cuh"
#include "kernels.h"

DQ_DEV int jac_slot(int r, int j, int np) { return j == 0 ? 0 : 1 + (j - 1 + r) % (np - 1); }

// rotation of every pair of round r (from the current A), then the column
// rotation of A and V; grid (np / 2, nmat), rot[m][k] = (c, s cos phi, s sin phi, on)
__global__ void __launch_bounds__(128) k_jac_cols(double2* A, double2* V, double4* rot, int N, int np, int r) {
    const int k = blockIdx.x, m = blockIdx.y;
    const int p0 = jac_slot(r, k, np), q0 = jac_slot(r, np - 1 - k, np);
    const int p = min(p0, q0), q = max(p0, q0);
    double2* a = A + (size_t)m * N * N;
    double2* v = V + (size_t)m * N * N;
    __shared__ double4 R;
    if (threadIdx.x == 0) {
        double4 t = make_double4(1.0, 0.0, 0.0, 0.0);
        if (q < N) {
            const double2 apq = a[MIDX(p, q, N)];
            const double ab = hypot(apq.x, apq.y);
            if (ab > 1e-300) {
                // the smaller of the two annihilating angles, |theta| <= pi/4:
                // t = tan theta solves t^2 + 2 zeta t - 1 = 0, zeta = (A(q,q) - A(p,p)) / (2 |A(p,q)|)
                const double app = a[MIDX(p, p, N)].x, aqq = a[MIDX(q, q, N)].x;
                const double zeta = (aqq - app) / (2.0 * ab);
                const double tn = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / sqrt(1.0 + tn * tn), sn = tn * cs;
                t = make_double4(cs, sn * apq.x / ab, sn * apq.y / ab, 1.0);
            }
        }
        R = t;
        rot[(size_t)m * (np / 2) + k] = t;
    }
    __syncthreads();
    const double4 t = R;
    if (t.w == 0.0) return;
    const double2 jpq = cmk(t.y, t.z), jqp = cmk(-t.y, t.z);    // s e^{i phi}, -s e^{-i phi}
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double2 x = a[MIDX(i, p, N)], y = a[MIDX(i, q, N)];
        a[MIDX(i, p, N)] = cfma(y, jqp, cscale(x, t.x));
        a[MIDX(i, q, N)] = cfma(x, jpq, cscale(y, t.x));
        x = v[MIDX(i, p, N)]; y = v[MIDX(i, q, N)];
        v[MIDX(i, p, N)] = cfma(y, jqp, cscale(x, t.x));
        v[MIDX(i, q, N)] = cfma(x, jpq, cscale(y, t.x));
    }
}

// A <- J^H A for the rotations of the round (rows p, q of each pair); the
// rotated element A(p,q) (and A(q,p)) is set to zero
__global__ void __launch_bounds__(128) k_jac_rows(double2* A, const double4* rot, int N, int np, int r) {
    const int k = blockIdx.x, m = blockIdx.y;
    const double4 t = rot[(size_t)m * (np / 2) + k];
    if (t.w == 0.0) return;
    const int p0 = jac_slot(r, k, np), q0 = jac_slot(r, np - 1 - k, np);
    const int p = min(p0, q0), q = max(p0, q0);
    double2* a = A + (size_t)m * N * N;
    // J^H = [[c, -s e^{i phi}], [s e^{-i phi}, c]]
    const double2 hpq = cmk(-t.y, -t.z), hqp = cmk(t.y, -t.z);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const double2 x = a[MIDX(p, j, N)], y = a[MIDX(q, j, N)];
        a[MIDX(p, j, N)] = cfma(hpq, y, cscale(x, t.x));
        a[MIDX(q, j, N)] = cfma(hqp, x, cscale(y, t.x));
    }
    __syncthreads();
    if (threadIdx.x == 0) { a[MIDX(p, q, N)] = cmk(0, 0); a[MIDX(q, p, N)] = cmk(0, 0); }
}

// off-diagonal and diagonal sums of squares per matrix: done[m] = 1 when
// off <= tol2 dia
__global__ void __launch_bounds__(256) k_jac_off(const double2* A, int N, double tol2, int* done) {
    __shared__ double red[64];
    const double2* a = A + (size_t)blockIdx.x * N * N;
    double off = 0.0, dia = 0.0;
    for (size_t e = threadIdx.x; e < (size_t)N * N; e += blockDim.x) {
        const double t = cabs2(a[e]);
        if ((int)(e % N) == (int)(e / N)) dia += t; else off += t;
    }
    off = block_sum(off, red);
    __syncthreads();
    dia = block_sum(dia, red);
    if (threadIdx.x == 0) done[blockIdx.x] = off <= tol2 * fmax(dia, 1e-300);
}

// eigenvalues ascending (stable rank of the diagonal) into w, the eigenvector
// columns in the same order into Vout
__global__ void __launch_bounds__(256) k_jac_sort(const double2* A, const double2* V, double2* Vout, double* w, int N) {
    extern __shared__ int jrank[];
    const size_t off = (size_t)blockIdx.x * N * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double x = A[off + MIDX(i, i, N)].x;
        int rk = 0;
        for (int j = 0; j < N; ++j) {
            const double y = A[off + MIDX(j, j, N)].x;
            rk += (y < x) || (y == x && j < i);
        }
        jrank[i] = rk;
        w[(size_t)blockIdx.x * N + rk] = x;
    }
    __syncthreads();
    for (size_t e = threadIdx.x; e < (size_t)N * N; e += blockDim.x) {
        const int i = (int)(e % N), j = (int)(e / N);
        Vout[off + MIDX(i, jrank[j], N)] = V[off + e];
    }
}

__global__ void k_jac_init(double2* V, int N, int nmat) {
    const size_t n = (size_t)nmat * N * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e % ((size_t)N * N);
        V[e] = cmk((int)(r % N) == (int)(r / N) ? 1.0 : 0.0, 0.0);
    }
}

// Eigen-decomposition of nmat Hermitian N x N matrices (column-major, ld N,
// consecutive) in A (destroyed): ascending eigenvalues into w (nmat x N) and
// eigenvectors into Vout (nmat x N x N).  Scratch: V (nmat N N), rot (nmat
// np/2 double4), done (nmat ints, device), done_h (nmat ints, host).  Sweeps
// until every matrix meets off <= (4 N eps)^2 dia (sums of squares; the
// off-diagonal part cannot fall much below N rounding errors of the
// rotations), at most max_sweeps; returns the number of sweeps, or -1 on a
// CUDA error.
int eig_herm_batched(double2* A, double2* V, double2* Vout, double* w, double4* rot, int* done, int* done_h,
                     int N, int nmat, int max_sweeps, cudaStream_t st) {
    const int np = N + (N & 1);
    k_jac_init<<<256, 256, 0, st>>>(V, N, nmat);
    int sweeps = 0;
    for (; sweeps < max_sweeps; ++sweeps) {
        const double tol = 4.0 * N * 2.220446049250313e-16;
        k_jac_off<<<nmat, 256, 0, st>>>(A, N, tol * tol, done);
        if (cudaMemcpyAsync(done_h, done, sizeof(int) * nmat, cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
        if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
        int all = 1;
        for (int m = 0; m < nmat; ++m) all &= done_h[m];
        if (all) break;
        for (int r = 0; r < np - 1; ++r) {
            k_jac_cols<<<dim3(np / 2, nmat), 128, 0, st>>>(A, V, rot, N, np, r);
            k_jac_rows<<<dim3(np / 2, nmat), 128, 0, st>>>(A, rot, N, np, r);
        }
    }
    k_jac_sort<<<nmat, 256, N * sizeof(int), st>>>(A, V, Vout, w, N);
    if (cudaGetLastError() != cudaSuccess) return -1;
    return sweeps;
}

// urt = V exp(-hdt w) V^H and urtm1 = V exp(+hdt w) V^H (hdt = dtau / 2), one
// thread per element (i, j), summed over the eigenvalues in order
__global__ void __launch_bounds__(256) k_eig_expm(const double2* V, const double* w, double hdt, double2* Um,
                                                  double2* Up, int N) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)N * N) return;
    const int i = (int)(e % N), j = (int)(e / N);
    double2 z0 = cmk(0, 0), z1 = cmk(0, 0);
    for (int k = 0; k < N; ++k) {
        const double2 t = cmulc(V[MIDX(i, k, N)], V[MIDX(j, k, N)]);
        z0 = cadd(z0, cscale(t, exp(-hdt * w[k])));
        z1 = cadd(z1, cscale(t, exp(hdt * w[k])));
    }
    Um[e] = z0;
    Up[e] = z1;
}

// scratch of eig_herm_batched for nmat matrices of order N (device and pinned host)
struct EigScratch {
    double2 *A = nullptr, *V = nullptr, *Vout = nullptr;
    double* w = nullptr;
    double4* rot = nullptr;
    int *done = nullptr, *done_h = nullptr;
    void release() {
        cudaFree(A); cudaFree(V); cudaFree(Vout); cudaFree(w); cudaFree(rot); cudaFree(done); cudaFreeHost(done_h);
        A = V = Vout = nullptr; w = nullptr; rot = nullptr; done = done_h = nullptr;
    }
    bool alloc(int N, int nmat) {
        const size_t nn = (size_t)N * N * nmat;
        const int np = N + (N & 1);
        bool ok = cudaMalloc(&A, nn * sizeof(double2)) == cudaSuccess;
        ok = ok && cudaMalloc(&V, nn * sizeof(double2)) == cudaSuccess;
        ok = ok && cudaMalloc(&Vout, nn * sizeof(double2)) == cudaSuccess;
        ok = ok && cudaMalloc(&w, (size_t)N * nmat * sizeof(double)) == cudaSuccess;
        ok = ok && cudaMalloc(&rot, (size_t)(np / 2) * nmat * sizeof(double4)) == cudaSuccess;
        ok = ok && cudaMalloc(&done, nmat * sizeof(int)) == cudaSuccess;
        ok = ok && cudaMallocHost(&done_h, nmat * sizeof(int)) == cudaSuccess;
        if (!ok) release();
        return ok;
    }
};

// Eigenpairs of nmat host matrices (consecutive, N x N, column-major) on the
// device: eigenvectors into Vh (same layout), ascending eigenvalues into wh
// (nmat x N).  Returns the sweep count, -1 on a CUDA error, -2 without
// convergence in 40 sweeps.
int eig_herm_device(const double2* Hh, int N, int nmat, double2* Vh, double* wh, cudaStream_t st) {
    EigScratch s;
    if (!s.alloc(N, nmat)) return -1;
    const size_t nn = (size_t)N * N * nmat;
    int rc = -1;
    if (cudaMemcpyAsync(s.A, Hh, nn * sizeof(double2), cudaMemcpyHostToDevice, st) == cudaSuccess) {
        rc = eig_herm_batched(s.A, s.V, s.Vout, s.w, s.rot, s.done, s.done_h, N, nmat, 40, st);
        if (rc >= 40) rc = -2;
        if (rc >= 0 &&
            (cudaMemcpyAsync(Vh, s.Vout, nn * sizeof(double2), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaMemcpyAsync(wh, s.w, (size_t)N * nmat * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaStreamSynchronize(st) != cudaSuccess))
            rc = -1;
    }
    s.release();
    return rc;
}

// The dense kinetic exponentials of one Hermitian hopping matrix Hh (host),
// urt = U exp(-dtau e / 2) U^H and urtm1 = U exp(+dtau e / 2) U^H, written to
// the device arrays d_urt, d_urtm1 (N x N).  Returns as eig_herm_device.
int dense_kinetic_device(const double2* Hh, int N, double dtau, double2* d_urt, double2* d_urtm1, cudaStream_t st) {
    EigScratch s;
    if (!s.alloc(N, 1)) return -1;
    int rc = -1;
    if (cudaMemcpyAsync(s.A, Hh, (size_t)N * N * sizeof(double2), cudaMemcpyHostToDevice, st) == cudaSuccess) {
        rc = eig_herm_batched(s.A, s.V, s.Vout, s.w, s.rot, s.done, s.done_h, N, 1, 40, st);
        if (rc >= 40) rc = -2;
        if (rc >= 0) {
            k_eig_expm<<<(N * N + 255) / 256, 256, 0, st>>>(s.Vout, s.w, 0.5 * dtau, d_urt, d_urtm1, N);
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
        }
    }
    s.release();
    return rc;
}
