// Eigenvalues of the last extrapolated Fock matrix (the reference's mo_energies are the
// eigenvalues of the F* of its last iteration, src/scf.rs:654-689), without eigenvectors:
//   k_tridiag : Householder reduction A = Q T Q^T (Golub & Van Loan, Alg. 8.3.1), one CTA per
//               matrix, the trailing block streamed from global memory (L2) by one warp per row;
//   k_bisect  : every eigenvalue of T by bisection on the Sturm sequence count (Barth, Martin &
//               Wilkinson), one thread per eigenvalue index, ascending by construction.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

constexpr int TRI_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

__global__ void __launch_bounds__(TRI_THREADS) k_tridiag(const TriJob* __restrict__ jobs, const int* __restrict__ mask) {
    const TriJob jb = jobs[blockIdx.x];
    if (mask && !mask[jb.mol]) return;
    const int n = jb.n;
    double* W = jb.W;
    extern __shared__ double sh[];
    double* v = sh;        // Householder vector
    double* p = sh + n;    // p, then w
    __shared__ double red[TRI_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = TRI_THREADS / 32;
    for (long long i = tid; i < (long long)n * n; i += TRI_THREADS) W[i] = jb.A[i];
    __syncthreads();
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        const double* rowk = W + (long long)k * n + k + 1;
        double nrm = 0.0;
        for (int i = tid; i < m; i += TRI_THREADS) {
            const double x = rowk[i];
            v[i] = x;
            nrm += x * x;
        }
        nrm = block_sum(nrm, red);
        const double alpha = sqrt(nrm);
        if (tid == 0) jb.d[k] = W[(long long)k * n + k];
        if (alpha == 0.0) {
            if (tid == 0) jb.e[k] = 0.0;
            __syncthreads();
            continue;
        }
        const double x0 = v[0];
        const double sg = x0 >= 0.0 ? 1.0 : -1.0;
        const double beta = 1.0 / (alpha * (alpha + fabs(x0)));
        __syncthreads();
        if (tid == 0) {
            v[0] = x0 + sg * alpha;
            jb.e[k] = -sg * alpha;
        }
        __syncthreads();
        // p = beta * W_sub v (one warp per row of the trailing block)
        for (int r = warp; r < m; r += nw) {
            const double* row = W + (long long)(k + 1 + r) * n + k + 1;
            double acc = 0.0;
            for (int c = lane; c < m; c += 32) acc = fma(row[c], v[c], acc);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) p[r] = beta * acc;
        }
        __syncthreads();
        double pv = 0.0;
        for (int i = tid; i < m; i += TRI_THREADS) pv += p[i] * v[i];
        pv = block_sum(pv, red);
        const double kk = 0.5 * beta * pv;
        for (int i = tid; i < m; i += TRI_THREADS) p[i] = p[i] - kk * v[i];  // p <- w
        __syncthreads();
        // W_sub -= v w^T + w v^T
        for (int r = warp; r < m; r += nw) {
            double* row = W + (long long)(k + 1 + r) * n + k + 1;
            const double vr = v[r], wr = p[r];
            for (int c = lane; c < m; c += 32) row[c] -= vr * p[c] + wr * v[c];
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            jb.d[n - 2] = W[(long long)(n - 2) * n + n - 2];
            jb.e[n - 2] = W[(long long)(n - 1) * n + n - 2];
        }
        jb.d[n - 1] = W[(long long)(n - 1) * n + n - 1];
    }
}

// number of eigenvalues of T below x
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x) {
    int c = 0;
    double q = d[0] - x;
    if (q < 0.0) ++c;
    for (int i = 1; i < n; ++i) {
        const double qq = q == 0.0 ? 1e-300 : q;
        q = d[i] - x - e2[i - 1] / qq;
        if (q < 0.0) ++c;
    }
    return c;
}

__global__ void k_bisect(const TriJob* __restrict__ jobs, const int* __restrict__ mask) {
    const TriJob jb = jobs[blockIdx.x];
    if (mask && !mask[jb.mol]) return;
    const int n = jb.n;
    extern __shared__ double sh[];
    double* d = sh;
    double* e2 = sh + n;
    __shared__ double bounds[2];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = jb.d[i];
        e2[i] = i + 1 < n ? jb.e[i] * jb.e[i] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < n; ++i) {
            const double r = (i > 0 ? fabs(jb.e[i - 1]) : 0.0) + (i + 1 < n ? fabs(jb.e[i]) : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
        }
        const double pad = 1e-12 * fmax(fabs(lo), fabs(hi)) + 1e-300;
        bounds[0] = lo - pad;
        bounds[1] = hi + pad;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double lo = bounds[0], hi = bounds[1];
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (!(mid > lo && mid < hi)) break;
            if (hi - lo <= 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi))) break;
            if (sturm_count(d, e2, n, mid) <= k) lo = mid;
            else hi = mid;
        }
        jb.eps[k] = 0.5 * (lo + hi);
    }
}

}  // namespace am1
