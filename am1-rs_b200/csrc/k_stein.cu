// Eigenvectors of matrices too large for the cluster Jacobi (the reference's symmetric_eigen,
// src/linalg.rs:276-331, at every size): A = Q T Q^T by the Householder reduction of k_eigvals.cu
// (which leaves reflector s in row s of its working copy W, columns s+1..n-1, and e[s]),
// eigenvalues of T by bisection, then
//   inverse iteration on T (Wilkinson; the cluster handling of LAPACK's dstein):
//     every eigenvector solves (T - sigma_k I) x = y by Gaussian elimination with partial pivoting,
//     one thread per eigenvector, four times; eigenvalues closer than kSteinOrtol ||T|| form a
//     cluster, whose shifts are pulled at least 10 eps ||T|| apart and whose vectors are
//     re-orthogonalised after every solve (two passes of classical Gram-Schmidt per vector, one
//     CTA per cluster); a zero pivot becomes eps ||T||; the last solve's growth is tested as
//     dstein tests its iterates, and a vector below the threshold fails the call (LINALG).
//   back-transformation X = Q Z = H_0 (H_1 (... H_{n-3} Z)), H_s = I - beta_s v_s v_s^T, in
//     blocks of kWyNb reflectors in the compact WY form H_k ... H_{k+nb-1} = I - V T V^T
//     (Schreiber & Van Loan 1989): T from the Gram matrix V^T V, then per block
//     Y = (T V^T) Z and Z -= V Y on the FP64 tensor cores (dmma_gemm.cuh).
// Layout: Z[i * n + k] is component i of eigenvector k (row-major, eigenvectors as columns, the
// reference's layout), so thread k of the solve reads and writes consecutive words with its
// neighbours.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {

constexpr double kEps = 2.220446049250313e-16;

// Deterministic start vector in [-1, 1): a 64-bit mix of (i, k) (the splitmix64 finaliser).
__device__ __forceinline__ double stein_start(int i, int k) {
    unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + (unsigned long long)k * 0xBF58476D1CE4E5B9ull + 1ull;
    h ^= h >> 31;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 29;
    return (double)(h >> 11) * 0x1p-53 * 2.0 - 1.0;
}

// ||T||_inf, the shifts and the clusters.  One block; the scan over the eigenvalues is serial.
__global__ void k_stein_prep(SteinJob sj) {
    const int n = sj.n;
    __shared__ double red[32];
    double mx = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double r = fabs(sj.d[i]) + (i > 0 ? fabs(sj.e[i - 1]) : 0.0) + (i + 1 < n ? fabs(sj.e[i]) : 0.0);
        mx = fmax(mx, r);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double tn = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) tn = fmax(tn, red[w]);
    if (!(tn > 0.0)) tn = 1.0;  // the zero matrix: any orthonormal basis
    sj.tn[0] = tn;
    sj.tn[1] = kEps * tn;  // pivot floor
    const double ortol = kSteinOrtol * tn, pert = 10.0 * kEps * tn;
    int count = 0;
    double prev = sj.eps[0];
    sj.shift[0] = prev;
    sj.cl[0] = 0;
    sj.scale[0] = 1.0;
    for (int k = 1; k < n; ++k) {
        const double lam = sj.eps[k];
        double sh = lam;
        if (lam - sj.eps[k - 1] <= ortol) {
            const int c0 = sj.cl[k - 1];
            sj.cl[k] = c0;
            if (c0 == k - 1) sj.cl_list[count++] = c0;  // a cluster of two or more starts at c0
            sh = fmax(lam, prev + pert);
        } else {
            sj.cl[k] = k;
        }
        sj.shift[k] = sh;
        sj.scale[k] = 1.0;
        prev = sh;
    }
    sj.counts[0] = count;
}

// One inverse-iteration solve per eigenvector: y = scale[k] * Z[:, k] (or the start vector),
// x = (T - shift[k] I)^-1 y into Z[:, k], and scale[k] = 1 / ||x||.  Elimination with partial
// pivoting: the current row keeps (diagonal, first superdiagonal) in registers; U row i (up to two
// superdiagonals) goes to U0/U1/U2[i][k], the eliminated right-hand side to Z[i][k].
// On the last solve (`last`), y has unit 2-norm, so ||x|| is the growth of the solve.  A shift
// within rounding of an eigenvalue grows y by about 1 / (eps ||T||); the vector is accepted when
// the growth reaches sqrt(0.1 / n) / (n eps ||T||): dstein's acceptance threshold sqrt(0.1 / n)
// for an iterate whose right-hand side it scaled to n ||T|| eps.  Below it, bit 4 of counts[1]
// marks the solve as not converged (dstein reports such vectors in INFO).
__global__ void __launch_bounds__(64) k_stein_solve(SteinJob sj, int first, int last) {
    const int n = sj.n;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t nn = (size_t)n * n;
    double* Z = sj.Z;
    double* U0 = sj.U;
    double* U1 = sj.U + nn;
    double* U2 = sj.U + 2 * nn;
    const double lam = sj.shift[k];
    const double sc = first ? 1.0 : sj.scale[k];
    const double floor_ = sj.tn[1];
    auto rhs = [&](int i) { return first ? stein_start(i, k) : Z[(size_t)i * n + k] * sc; };
    double cd = sj.d[0] - lam;
    double cs = n > 1 ? sj.e[0] : 0.0;
    double y = rhs(0);
#pragma unroll 4
    for (int i = 0; i < n - 1; ++i) {
        const double c = sj.e[i];
        const double a1 = sj.d[i + 1] - lam;
        const double b1 = i + 2 < n ? sj.e[i + 1] : 0.0;
        const double yn = rhs(i + 1);
        const size_t o = (size_t)i * n + k;
        if (fabs(cd) >= fabs(c)) {
            if (cd == 0.0) cd = floor_;
            const double m = c / cd;
            U0[o] = cd;
            U1[o] = cs;
            U2[o] = 0.0;
            Z[o] = y;
            y = yn - m * y;
            cd = a1 - m * cs;
            cs = b1;
        } else {
            const double m = cd / c;
            U0[o] = c;
            U1[o] = a1;
            U2[o] = b1;
            Z[o] = yn;
            y = y - m * yn;
            cd = cs - m * a1;
            cs = -m * b1;
        }
    }
    if (cd == 0.0) cd = floor_;
    // back substitution, with the 2-norm accumulated as scale * sqrt(ssq) (no overflow)
    double x1 = y / cd, x2 = 0.0;
    Z[(size_t)(n - 1) * n + k] = x1;
    double smax = fabs(x1), ssq = x1 != 0.0 ? 1.0 : 0.0;
#pragma unroll 4
    for (int i = n - 2; i >= 0; --i) {
        const size_t o = (size_t)i * n + k;
        const double x = (Z[o] - U1[o] * x1 - U2[o] * x2) / U0[o];
        Z[o] = x;
        x2 = x1;
        x1 = x;
        const double ax = fabs(x);
        if (ax > smax) {
            const double r = smax / ax;
            ssq = 1.0 + ssq * r * r;
            smax = ax;
        } else if (ax > 0.0) {
            const double r = ax / smax;
            ssq += r * r;
        }
    }
    const double nrm = smax * sqrt(ssq);
    if (!(nrm > 0.0) || !isfinite(nrm)) {
        atomicOr(sj.counts + 1, 1);
        sj.scale[k] = 1.0;
        return;
    }
    if (last && nrm * ((double)n * kEps * sj.tn[0]) < sqrt(0.1 / (double)n)) atomicOr(sj.counts + 1, 4);
    sj.scale[k] = 1.0 / nrm;
}

// Block-wide sum or max (fixed order), every thread gets the result.
template <bool MAX>
__device__ __forceinline__ double stein_block_reduce(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = MAX ? fmax(v, u) : v + u;
    }
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = red[0];
    for (int w = 1; w < nw; ++w) t = MAX ? fmax(t, red[w]) : t + red[w];
    return t;
}

// Orthonormalise the vectors of every cluster (one CTA per cluster, in ascending order inside it):
// copy them (times their scale) to Zt, vector-major; for each vector two passes of
// x -= sum_{l<j} (q_l . x) q_l (a warp per dot product, then a thread per component), then
// x /= ||x||; copy back with scale 1.  Dynamic shared memory: n doubles for the dot products.
__global__ void __launch_bounds__(256) k_stein_orth(SteinJob sj) {
    const int b = blockIdx.x;
    if (b >= sj.counts[0]) return;
    const int n = sj.n;
    const int k0 = sj.cl_list[b];
    int m = 1;
    while (k0 + m < n && sj.cl[k0 + m] == k0) ++m;
    extern __shared__ double dl[];
    __shared__ double red[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    double* Zt = sj.Zt + (size_t)k0 * n;
    for (long long idx = tid; idx < (long long)m * n; idx += blockDim.x) {
        const int i = (int)(idx / m), l = (int)(idx % m);
        Zt[(size_t)l * n + i] = sj.Z[(size_t)i * n + k0 + l] * sj.scale[k0 + l];
    }
    __syncthreads();
    for (int j = 0; j < m; ++j) {
        double* x = Zt + (size_t)j * n;
        for (int pass = 0; pass < 2 && j > 0; ++pass) {
            for (int l = warp; l < j; l += nw) {
                const double* q = Zt + (size_t)l * n;
                double s = 0.0;
                for (int i = lane; i < n; i += 32) s = fma(q[i], x[i], s);
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) dl[l] = s;
            }
            __syncthreads();
            for (int i = tid; i < n; i += blockDim.x) {
                double t = x[i];
                for (int l = 0; l < j; ++l) t = fma(-dl[l], Zt[(size_t)l * n + i], t);
                x[i] = t;
            }
            __syncthreads();
        }
        double mx = 0.0;
        for (int i = tid; i < n; i += blockDim.x) mx = fmax(mx, fabs(x[i]));
        mx = stein_block_reduce<true>(mx, red);
        double inv = 0.0;
        if (mx > 0.0 && isfinite(mx)) {
            const double rs = 1.0 / mx;
            double s = 0.0;
            for (int i = tid; i < n; i += blockDim.x) {
                const double u = x[i] * rs;
                s = fma(u, u, s);
            }
            s = stein_block_reduce<false>(s, red);
            inv = rs / sqrt(s);
        } else if (tid == 0) {
            atomicOr(sj.counts + 1, 2);
        }
        for (int i = tid; i < n; i += blockDim.x) x[i] *= inv;
        __syncthreads();
    }
    for (long long idx = tid; idx < (long long)m * n; idx += blockDim.x) {
        const int i = (int)(idx / m), l = (int)(idx % m);
        sj.Z[(size_t)i * n + k0 + l] = Zt[(size_t)l * n + i];
    }
    for (int l = tid; l < m; l += blockDim.x) sj.scale[k0 + l] = 1.0;
}

// Z[:, k] *= scale[k]: the pending normalisation of every vector.
__global__ void k_stein_scale(SteinJob sj) {
    const int n = sj.n;
    const long long nn = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nn; idx += (long long)gridDim.x * blockDim.x)
        sj.Z[idx] *= sj.scale[idx % n];
}

// A[r][c] = A[c][r] for r < c: the lower triangle mirrored into the upper one (the reference reads
// the lower triangle, Side::Lower).  Block (32, 8) per 32 x 32 tile pair (tile row tr <= tile column
// tc): the lower tile (tc, tr) goes through shared memory into the upper tile (tr, tc); a diagonal
// tile is read whole before any of it is written.  Grid (ceil(n / 32), ceil(n / 32)).
__global__ void k_mirror_lower(double* A, int n) {
    __shared__ double tile[32][33];
    const int tr = blockIdx.y, tc = blockIdx.x;
    if (tr > tc) return;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = tc * 32 + y, c = tr * 32 + threadIdx.x;  // lower source rows / columns
        tile[y][threadIdx.x] = (r < n && c < n) ? A[(size_t)r * n + c] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = tr * 32 + y, c = tc * 32 + threadIdx.x;  // upper destination
        if (r < n && c < n && r < c) A[(size_t)r * n + c] = tile[threadIdx.x][y];
    }
}

// Zt[k][i] = Z[i][k] for the first m columns, through a 32 x 32 shared-memory tile.
__global__ void k_transpose_cols(const double* __restrict__ Z, int n, int m, double* __restrict__ Zt) {
    __shared__ double tile[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int i = i0 + y, k = k0 + threadIdx.x;
        tile[y][threadIdx.x] = (i < n && k < m) ? Z[(size_t)i * n + k] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int k = k0 + y, i = i0 + threadIdx.x;
        if (k < m && i < n) Zt[(size_t)k * n + i] = tile[threadIdx.x][y];
    }
}

// P = w (P + P^T) / 2: tile pair (tr <= tc) read whole into shared memory, then both written.
__global__ void k_sym_scale(double* P, int n, double w) {
    __shared__ double up[32][33], lo[32][33];
    const int tr = blockIdx.y, tc = blockIdx.x;
    if (tr > tc) return;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = tr * 32 + y, c = tc * 32 + threadIdx.x;
        up[y][threadIdx.x] = (r < n && c < n) ? P[(size_t)r * n + c] : 0.0;
        const int r2 = tc * 32 + y, c2 = tr * 32 + threadIdx.x;
        lo[y][threadIdx.x] = (r2 < n && c2 < n) ? P[(size_t)r2 * n + c2] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = tr * 32 + y, c = tc * 32 + threadIdx.x;
        const double v = 0.5 * w * (up[y][threadIdx.x] + lo[threadIdx.x][y]);
        if (r < n && c < n) P[(size_t)r * n + c] = v;
        const int r2 = tc * 32 + y, c2 = tr * 32 + threadIdx.x;
        if (r2 < n && c2 < n) P[(size_t)r2 * n + c2] = 0.5 * w * (lo[y][threadIdx.x] + up[threadIdx.x][y]);
    }
}

// ---------------------------------------------------------------------------------------------
// Back-transformation
// ---------------------------------------------------------------------------------------------

// Vt[s][c] = v_s[c] = W[s][c] for c > s (else 0), rows s < P (P = padded reflector count; rows
// s >= nref are zero), and V = Vt^T (n x P, row-major), through a 32 x 32 shared-memory tile.
// Block (32, 8); grid (ceil(n / 32), P / 32).
__global__ void k_wy_split(const double* __restrict__ W, int n, int nref, int P, double* __restrict__ Vt, double* __restrict__ V) {
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int s = s0 + r, c = c0 + threadIdx.x;
        double x = 0.0;
        if (s < nref && c < n && c > s) x = W[(size_t)s * n + c];
        if (c < n) Vt[(size_t)s * n + c] = x;
        tile[r][threadIdx.x] = x;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int c = c0 + r, s = s0 + threadIdx.x;
        if (c < n) V[(size_t)c * P + s] = tile[threadIdx.x][r];
    }
}

// The triangular factor of each block b of kWyNb reflectors (one CTA per block, a thread per row):
// T[j][j] = beta_j, T[0:j, j] = -beta_j T[0:j, 0:j] S[0:j, j] with S = Vt_b Vt_b^T (from Sg), and
// beta_s = 1 / (|e_s| |v_s[s+1]|) (= 1 / (alpha (alpha + |x_{s+1}|)) of the reduction; 0 when e_s = 0).
__global__ void __launch_bounds__(kWyNb) k_wy_tfactor(const double* __restrict__ Sg, const double* __restrict__ W, const double* __restrict__ e,
                                                      int n, int nref, double* __restrict__ Tg) {
    __shared__ double T[kWyNb][kWyNb + 1];
    const int b = blockIdx.x, r = threadIdx.x;
    const int k = b * kWyNb;
    const int m = min(kWyNb, nref - k);
    const double* S = Sg + (size_t)b * kWyNb * kWyNb;
    for (int c = 0; c < kWyNb; ++c) T[r][c] = 0.0;
    __syncthreads();
    for (int j = 0; j < m; ++j) {
        const int s = k + j;
        const double es = fabs(e[s]);
        const double v1 = fabs(W[(size_t)s * n + s + 1]);
        const double beta = es == 0.0 || v1 == 0.0 ? 0.0 : 1.0 / (es * v1);
        if (r < j) {
            double t = 0.0;
            for (int l = r; l < j; ++l) t = fma(T[r][l], S[(size_t)l * kWyNb + j], t);
            T[r][j] = -beta * t;
        } else if (r == j) {
            T[j][j] = beta;
        }
        __syncthreads();
    }
    double* To = Tg + (size_t)b * kWyNb * kWyNb;
    for (int c = 0; c < kWyNb; ++c) To[(size_t)r * kWyNb + c] = T[r][c];
}

// C_z (=, or -=) A_z B_z for z = blockIdx.z (pointers advanced by the strides), 64 x 64 tiles:
// grid (ceil(N / 64), ceil(M / 64), batch).
template <bool PAIRS>
__device__ __forceinline__ void dgemm_body(const double* A, int lda, long long sA, const double* B, int ldb, long long sB, double* C, int ldc,
                                           long long sC, int M, int N, int K, int sub) {
    extern __shared__ __align__(16) double dsm[];
    const long long z = blockIdx.z;
    A += z * sA;
    B += z * sB;
    C += z * sC;
    const int m0 = blockIdx.y * DG_TILE, n0 = blockIdx.x * DG_TILE;
    const bool compute = dg_quarter_on(m0, n0, M, N, false);
    double acc[2][4][4];
    dg_mainloop<PAIRS>(dsm, A, lda, B, ldb, M, N, K, m0, n0, acc, compute);
    if (!compute) return;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = m0 + dg_row(i, q), c = n0 + dg_col(j, q);
                if (r < M && c < N) {
                    double* p = C + (size_t)r * ldc + c;
                    *p = sub ? *p - acc[i][j][q] : acc[i][j][q];
                }
            }
}

__global__ void __launch_bounds__(DG_THREADS, 4) k_dgemm16(const double* A, int lda, long long sA, const double* B, int ldb, long long sB,
                                                          double* C, int ldc, long long sC, int M, int N, int K, int sub) {
    dgemm_body<true>(A, lda, sA, B, ldb, sB, C, ldc, sC, M, N, K, sub);
}
__global__ void __launch_bounds__(DG_THREADS, 4) k_dgemm8(const double* A, int lda, long long sA, const double* B, int ldb, long long sB,
                                                         double* C, int ldc, long long sC, int M, int N, int K, int sub) {
    dgemm_body<false>(A, lda, sA, B, ldb, sB, C, ldc, sC, M, N, K, sub);
}

}  // namespace am1
