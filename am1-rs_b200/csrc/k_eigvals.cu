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
// share fits one CTA.  Step k (GVL Alg. 8.3.1; the reflector zeroes row/column k below the
// subdiagonal):
//   owner of row k:  x = A[k, k+1:], alpha = |x|, v = x + sign(x0) alpha e1, beta = 1/(alpha(alpha+|x0|))
//   cluster sync #1; every CTA copies v and beta from the owner (distributed shared memory)
//   every CTA:       p_r = beta A[r, k+1:] . v for its rows, sent to every CTA; its share of p.v
//   cluster sync #2; w = p - (beta/2)(p.v) v;  A[r, k+1:] -= v_r w + w_r v for its rows
// All control flow is uniform over the cluster (alpha = 0 gives beta = 0 and a no-op update),
// so every CTA takes the same cluster barriers.
constexpr int TRI_THREADS = 512;
constexpr int TRI_WARPS = TRI_THREADS / 32;

// Dynamic shared memory of one CTA: local rows, v, p/w and the C partial sums of p.v.
size_t tridiag_smem_bytes(int n, int C) {
    const size_t rows = (size_t)(n + C - 1) / C;
    return sizeof(double) * (rows * n + 2 * (size_t)n + 1 + 16);
}

__device__ __forceinline__ double tri_block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < TRI_WARPS; ++w) s += red[w];
    return s;
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
    double* A = sh;            // R x n: global row lr * C + crank at local row lr
    double* v = A + (size_t)R * n;
    double* pw = v + n;        // p, then w (global column index)
    double* sc = pw + n;       // sc[0] = beta, sc[1 + q] = CTA q's share of p.v
    __shared__ double red[TRI_WARPS];
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
    for (int k = 0; k + 2 < n; ++k) {
        const int owner = k % C;
        const int c0 = k + 1;  // trailing block: rows and columns c0 .. n-1
        if (crank == owner) {
            const double* rowk = A + (size_t)(k / C) * n;
            double nrm = 0.0;
            for (int c = c0 + tid; c < n; c += TRI_THREADS) {
                const double x = rowk[c];
                v[c] = x;
                nrm += x * x;
            }
            nrm = tri_block_sum(nrm, red);
            const double alpha = sqrt(nrm);
            const double x0 = rowk[c0];
            const double sg = x0 >= 0.0 ? 1.0 : -1.0;
            if (tid == 0) {
                jb.d[k] = rowk[k];
                jb.e[k] = alpha == 0.0 ? 0.0 : -sg * alpha;
                sc[0] = alpha == 0.0 ? 0.0 : 1.0 / (alpha * (alpha + fabs(x0)));
                if (alpha != 0.0) v[c0] = x0 + sg * alpha;
            }
        }
        csync();  // #1: v and beta are ready in the owner
        if (crank != owner) {
            const double* rv = cluster.map_shared_rank(v, owner);
            for (int c = c0 + tid; c < n; c += TRI_THREADS) v[c] = rv[c];
            if (tid == 0) sc[0] = *cluster.map_shared_rank(sc, owner);
        }
        __syncthreads();
        const double beta = sc[0];
        // p_r = beta * A[r, c0:] . v for this CTA's rows r >= c0, one warp per row
        const int lr0 = (c0 - crank + C - 1) / C;  // first local row with global index >= c0
        double part = 0.0;
        for (int lr = lr0 + warp; lr < R; lr += TRI_WARPS) {
            const int r = lr * C + crank;
            if (r >= n) break;
            const double* row = A + (size_t)lr * n;
            double acc = 0.0;
            for (int c = c0 + lane; c < n; c += 32) acc = fma(row[c], v[c], acc);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            const double p = beta * acc;
            if (lane < C) *cluster.map_shared_rank(&pw[r], lane) = p;  // to every CTA, itself included
            part += p * v[r];
        }
        part = tri_block_sum(lane == 0 ? part : 0.0, red);
        if (tid < C) *cluster.map_shared_rank(&sc[1 + crank], tid) = part;
        csync();  // #2: p and the shares of p.v are complete everywhere
        double pv = 0.0;
        for (int q = 0; q < C; ++q) pv += sc[1 + q];
        const double kk = 0.5 * beta * pv;
        for (int c = c0 + tid; c < n; c += TRI_THREADS) pw[c] -= kk * v[c];  // pw <- w
        __syncthreads();
        for (int lr = lr0 + warp; lr < R; lr += TRI_WARPS) {
            const int r = lr * C + crank;
            if (r >= n) break;
            double* row = A + (size_t)lr * n;
            const double vr = v[r], wr = pw[r];
            for (int c = c0 + lane; c < n; c += 32) row[c] -= vr * pw[c] + wr * v[c];
        }
        __syncthreads();
    }
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
