// Eigenvalues of the last extrapolated Fock matrix (the reference's mo_energies are the
// eigenvalues of the F* of its last iteration, src/scf.rs:654-689), without eigenvectors:
//   k_tridiag : Householder reduction A = Q T Q^T (Golub & Van Loan, Alg. 8.3.1), the matrix held
//               in the shared memory of a thread-block cluster (rows spread over its CTAs);
//   k_bisect  : every eigenvalue of T by bisection on the Sturm sequence count (Barth, Martin &
//               Wilkinson), one thread per eigenvalue index, ascending by construction.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

namespace cg = cooperative_groups;

// Householder reduction of one symmetric matrix held on chip.  The n x n matrix is distributed by
// rows over a thread-block cluster of C CTAs (row r lives in CTA r % C, at local row r / C, full
// length n), so the whole reduction runs out of shared memory; C is the smallest cluster whose
// share fits one CTA.  Step k (GVL Alg. 8.3.1: the reflector I - beta v v^T zeroes row/column k
// below the subdiagonal):
//   sync #1   the owner of row k has v_k, beta_k ready; every other CTA copies them (distributed
//             shared memory)
//   p_r = beta A[r, k+1:] . v for the CTA's rows r > k, sent to every CTA with the warp's share of p.v
//   sync #2   A[r, k+1:] -= v_r w + w_r v with w = p - (beta/2)(p.v) v, formed on the fly
// Look-ahead: the warp that updates row k+1 (warp 0 of its owner) derives v_{k+1}, beta_{k+1}, d, e
// from it at once, into the other half of the double-buffered v, so a step costs two cluster
// barriers and one CTA barrier.  All control flow is uniform over the cluster (alpha = 0 gives
// beta = 0 and a no-op update), so every CTA takes the same barriers.
constexpr int TRI_THREADS = 512;
constexpr int TRI_WARPS = TRI_THREADS / 32;

// Dynamic shared memory of one CTA: local rows, v (two buffers), p, the per-warp shares of p.v
// from every CTA, beta (two buffers).
size_t tridiag_smem_bytes(int n, int C) {
    const size_t rows = (size_t)(n + C - 1) / C;
    return sizeof(double) * (rows * n + 3 * (size_t)n + (size_t)C * TRI_WARPS + 2);
}

// Householder vector of row `row` (the trailing part from column c0 = k + 1), computed by one
// warp: v = x + sign(x0) |x| e1 into vbuf, beta into *beta, and d[k], e[k].
__device__ __forceinline__ void tri_reflector(const double* row, int k, int n, double* vbuf, double* beta, double* d, double* e) {
    const int lane = threadIdx.x & 31, c0 = k + 1;
    double nrm = 0.0;
    for (int c = c0 + lane; c < n; c += 32) {
        const double x = row[c];
        vbuf[c] = x;
        nrm += x * x;
    }
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    const double alpha = sqrt(nrm);
    const double x0 = row[c0];
    const double sg = x0 >= 0.0 ? 1.0 : -1.0;
    __syncwarp();
    if (lane == 0) {
        d[k] = row[k];
        e[k] = alpha == 0.0 ? 0.0 : -sg * alpha;
        *beta = alpha == 0.0 ? 0.0 : 1.0 / (alpha * (alpha + fabs(x0)));
        if (alpha != 0.0) vbuf[c0] = x0 + sg * alpha;
    }
}

__global__ void __launch_bounds__(TRI_THREADS) k_tridiag(const TriJob* __restrict__ jobs, const int* __restrict__ mask) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const TriJob jb = jobs[blockIdx.x / C];
    if (mask && !mask[jb.mol]) return;  // uniform over the cluster
    const int n = jb.n;
    const int R = (n + C - 1) / C;
    extern __shared__ double sh[];
    double* A = sh;                     // R x n: global row lr * C + crank at local row lr
    double* vb = A + (size_t)R * n;     // v, two buffers of n (global column index)
    double* p = vb + 2 * (size_t)n;     // p (global index)
    double* part = p + n;               // [C * TRI_WARPS] shares of p.v
    double* bb = part + C * TRI_WARPS;  // beta, two buffers
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto csync = [&]() {
        if (C > 1) cluster.sync();
        else __syncthreads();
    };
    for (int lr = warp; lr < R; lr += TRI_WARPS) {
        const int r = lr * C + crank;
        if (r >= n) break;
        for (int c = lane; c < n; c += 32) A[(size_t)lr * n + c] = jb.A[(size_t)r * n + c];
    }
    __syncthreads();
    if (n >= 3 && crank == 0 && warp == 0) tri_reflector(A, 0, n, vb, bb, jb.d, jb.e);
    for (int k = 0; k + 2 < n; ++k) {
        const int par = k & 1, owner = k % C, c0 = k + 1;
        double* v = vb + (size_t)par * n;
        csync();  // #1: v_k and beta_k are ready in the owner
        if (crank != owner) {
            const double* rv = cluster.map_shared_rank(v, owner);
            for (int c = c0 + tid; c < n; c += TRI_THREADS) v[c] = rv[c];
            if (tid == 0) bb[par] = *cluster.map_shared_rank(bb + par, owner);
            __syncthreads();
        }
        const double beta = bb[par];
        const int lr0 = (c0 - crank + C - 1) / C;  // first local row with global index >= c0
        double wpart = 0.0;
        for (int lr = lr0 + warp; lr < R; lr += TRI_WARPS) {
            const int r = lr * C + crank;
            if (r >= n) break;
            const double* row = A + (size_t)lr * n;
            double acc = 0.0;
            for (int c = c0 + lane; c < n; c += 32) acc = fma(row[c], v[c], acc);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            const double pr = beta * acc;
            if (lane < C) *cluster.map_shared_rank(&p[r], lane) = pr;  // to every CTA, itself included
            wpart += pr * v[r];
        }
        if (lane < C) *cluster.map_shared_rank(&part[crank * TRI_WARPS + warp], lane) = wpart;
        csync();  // #2: p and every share of p.v are complete everywhere
        double pv = 0.0;
        for (int q = lane; q < C * TRI_WARPS; q += 32) pv += part[q];
        for (int o = 16; o > 0; o >>= 1) pv += __shfl_xor_sync(0xffffffffu, pv, o);
        const double kk = 0.5 * beta * pv;
        for (int lr = lr0 + warp; lr < R; lr += TRI_WARPS) {
            const int r = lr * C + crank;
            if (r >= n) break;
            double* row = A + (size_t)lr * n;
            const double vr = v[r], wr = p[r] - kk * vr;
            for (int c = c0 + lane; c < n; c += 32) row[c] -= vr * (p[c] - kk * v[c]) + wr * v[c];
            // look-ahead: row k+1 is final now; its reflector is the next step's
            if (r == c0 && c0 + 2 < n) {
                __syncwarp();
                tri_reflector(row, c0, n, vb + (size_t)(par ^ 1) * n, bb + (par ^ 1), jb.d, jb.e);
            }
        }
    }
    __syncthreads();
    // the last 2 x 2 block (or the 1 x 1 matrix)
    if (tid == 0) {
        if (n >= 2) {
            if ((n - 2) % C == crank) jb.d[n - 2] = A[(size_t)((n - 2) / C) * n + n - 2];
            if ((n - 1) % C == crank) {
                jb.e[n - 2] = A[(size_t)((n - 1) / C) * n + n - 2];
                jb.d[n - 1] = A[(size_t)((n - 1) / C) * n + n - 1];
            }
        } else if (crank == 0) {
            jb.d[0] = A[0];
        }
    }
    csync();  // no CTA leaves while another may still address its shared memory
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
