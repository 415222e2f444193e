// Density matrix of the SCF step by trace-correcting purification (SP2), batched.
//
// The SCF needs only P = w * (projector onto the n_occ lowest eigenvectors of F*), which is what
// am1-rs builds from the eigenvectors (src/scf.rs:654-661: symmetric_eigen then
// density_from_coeff).  SP2 (Niklasson, Phys. Rev. B 66, 155115 (2002)) reaches the same
// projector with matrix products only:
//     X0 = (e_max I - F*) / (e_max - e_min)         (Gershgorin bounds, spectrum mapped into [0,1])
//     X <- X^2  or  X <- 2X - X^2                   (whichever brings tr X closer to n_occ)
// until X is idempotent to rounding.  Each step is one symmetric FP64 product X.X on the tensor
// cores (mma.sync m16n8k8 f64), upper-triangle tiles only, mirrored in the epilogue, which also
// folds in the choice of branch and the tile's share of tr X and ||X||_F^2 (= tr X^2 for the
// next step's decision).  No eigenvectors, no fine-grained synchronisation: every step is one
// launch over all (molecule, channel) tiles of the batch.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {


// X0 = (e_max I - F*) / (e_max - e_min); per-block partial sums of tr X0 and ||X0||_F^2.
__global__ void k_sp2_init(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, const MolState* __restrict__ st, int nblk) {
    const Sp2Job jb = jobs[blockIdx.y];
    if (!st[jb.mol].active) return;
    const int n = jb.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    __shared__ double red[2][32];
    // spectral bounds (every block reduces the row bounds itself)
    double lo = 1e300, hi = -1e300;
    for (int i = tid; i < n; i += blockDim.x) {
        lo = fmin(lo, jb.rowmin[i]);
        hi = fmax(hi, jb.rowmax[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
        red[0][warp] = lo;
        red[1][warp] = hi;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < nw; ++w) {
            red[0][0] = fmin(red[0][0], red[0][w]);
            red[1][0] = fmax(red[1][0], red[1][w]);
        }
    }
    __syncthreads();
    const double emin = red[0][0], emax = red[1][0];
    const double inv = 1.0 / fmax(emax - emin, 1e-300);
    __syncthreads();
    double tr = 0.0, fr = 0.0;
    for (int r = blockIdx.x * nw + warp; r < n; r += nblk * nw) {
        const double* Fr = jb.F + (long long)r * n;
        double* Xr = jb.X0 + (long long)r * n;
        for (int c = lane; c < n; c += 32) {
            const double x = ((c == r ? emax : 0.0) - Fr[c]) * inv;
            Xr[c] = x;
            fr += x * x;
            if (c == r) tr += x;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        tr += __shfl_xor_sync(0xffffffffu, tr, o);
        fr += __shfl_xor_sync(0xffffffffu, fr, o);
    }
    if (lane == 0) {
        red[0][warp] = tr;
        red[1][warp] = fr;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < nw; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        jb.part[2 * blockIdx.x] = a;
        jb.part[2 * blockIdx.x + 1] = b;
        if (blockIdx.x == 0) {
            Sp2State& s = sst[blockIdx.y];
            s.emin = emin;
            s.emax = emax;
        }
    }
}

// Reduce the init partials: state of step 0.
__global__ void k_sp2_start(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, const MolState* __restrict__ st, int njobs,
                            int nblk) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const Sp2Job jb = jobs[j];
    Sp2State& s = sst[j];
    s.active = st[jb.mol].active;
    s.steps = 0;
    s.cur = 0;
    s.converged = 0;
    double tr = 0.0, fr = 0.0;
    for (int b = 0; b < nblk; ++b) {
        tr += jb.part[2 * b];
        fr += jb.part[2 * b + 1];
    }
    s.trX = tr;
    s.trX2 = fr;
    s.idem[0] = s.idem[1] = 1e300;
    s.square = fabs(fr - jb.nocc) < fabs(2.0 * tr - fr - jb.nocc) ? 1 : 0;
}

// One SP2 step over all upper-triangle 64x64 tiles of every active channel.
__global__ void __launch_bounds__(DG_THREADS, 4) k_sp2_step(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                            int ntiles, const Sp2State* __restrict__ sst) {
    extern __shared__ double dsm[];
    __shared__ double red[2][4];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State s = sst[tl.job];
    if (!s.active) return;
    const Sp2Job jb = jobs[tl.job];
    const int n = jb.n;
    const double* X = s.cur ? jb.X1 : jb.X0;
    double* Y = s.cur ? jb.X0 : jb.X1;
    const int m0 = tl.tm * DG_TILE, n0 = tl.tn * DG_TILE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool diag_tile = tl.tm == tl.tn;
    // this warp's 32x32 quarter: skip it when it is padding, or the lower-left quarter of a
    // diagonal tile (the upper-right quarter computes and mirrors it)
    const int qr = (warp >> 1) * 32, qc = (warp & 1) * 32;
    const bool lower_quarter = diag_tile && qr > qc;
    const bool compute = m0 + qr < n && n0 + qc < n && !lower_quarter;
    double acc[2][4][4];
    dg_mainloop(dsm, X, n, X, n, n, n, n, m0, n0, acc, compute);  // X symmetric: X[rows m0..] . X[:, n0..]
    // epilogue: Y = X^2 or 2X - X^2, mirrored; partial trace / Frobenius sums
    const bool mirror = !diag_tile || qr < qc;  // off-diagonal content: write the transpose too
    double tr = 0.0, fr = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = m0 + dg_row(i, e);
                const int c = n0 + dg_col(j, e);
                if (compute && r < n && c < n) {
                    const double x2 = acc[i][j][e];
                    const double y = s.square ? x2 : 2.0 * X[(long long)r * n + c] - x2;
                    Y[(long long)r * n + c] = y;
                    if (mirror) Y[(long long)c * n + r] = y;
                    fr += (mirror ? 2.0 : 1.0) * y * y;
                    if (r == c) tr += y;
                }
            }
    for (int o = 16; o > 0; o >>= 1) {
        tr += __shfl_xor_sync(0xffffffffu, tr, o);
        fr += __shfl_xor_sync(0xffffffffu, fr, o);
    }
    if (lane == 0) {
        red[0][warp] = tr;
        red[1][warp] = fr;
    }
    __syncthreads();
    if (tid == 0) {
        double* p = jb.part + 2 * (t - jb.tile0);
        p[0] = red[0][0] + red[0][1] + red[0][2] + red[0][3];
        p[1] = red[1][0] + red[1][1] + red[1][2] + red[1][3];
    }
}

// C = alpha A.B for every (molecule, channel) job of a tile list, on the FP64 tensor cores
// (the commutator product F.P, src/scf.rs:531-544).
__global__ void __launch_bounds__(DG_THREADS, 4) k_dgemm_nn(const GemmJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                            int ntiles, const MolState* __restrict__ st, int force,
                                                            const int* __restrict__ mask) {
    extern __shared__ double dsm[];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const GemmJob jb = jobs[tl.job];
    if (!force && !st[jb.mol].active) return;
    if (mask && !mask[jb.mol]) return;
    const int m0 = tl.tm * DG_TILE, n0 = tl.tn * DG_TILE;
    const int warp = threadIdx.x >> 5;
    const bool compute = m0 + (warp >> 1) * 32 < jb.M && n0 + (warp & 1) * 32 < jb.N;  // skip pure padding
    double acc[2][4][4];
    dg_mainloop(dsm, jb.A, jb.lda, jb.B, jb.ldb, jb.M, jb.N, jb.K, m0, n0, acc, compute);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = m0 + dg_row(i, e);
                const int c = n0 + dg_col(j, e);
                if (r < jb.M && c < jb.N) jb.C[(long long)r * jb.ldc + c] = jb.alpha * acc[i][j][e];
            }
}

// After a step: reduce the tile partials (in tile order), test idempotency, choose the next branch.
__global__ void k_sp2_update(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, int njobs, int max_steps,
                             int* __restrict__ active_count, double* __restrict__ work) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    Sp2State& s = sst[j];
    if (!s.active) return;
    const Sp2Job jb = jobs[j];
    // algorithmic work of the product just taken: a symmetric X.X, n^3 flops
    atomicAdd(&work[0], 1.0);
    atomicAdd(&work[1], (double)jb.n * jb.n * jb.n);
    double tr = 0.0, fr = 0.0;
    for (int t = 0; t < jb.ntiles; ++t) {
        tr += jb.part[2 * t];
        fr += jb.part[2 * t + 1];
    }
    s.cur ^= 1;
    s.steps += 1;
    s.trX = tr;
    s.trX2 = fr;
    // idempotency error tr X - tr X^2 (sum of x(1-x) over the spectrum, >= 0)
    const double idem = fabs(tr - fr);
    const bool floor_reached = idem < 1.0e-6 && idem >= s.idem[0];  // stagnation at the rounding floor
    s.idem[0] = s.idem[1];
    s.idem[1] = idem;
    if (floor_reached || idem < 1.0e-15 * fmax(1.0, (double)jb.n)) {
        s.active = 0;
        s.converged = 1;
        return;
    }
    if (s.steps >= max_steps) {
        s.active = 0;
        s.converged = 0;
        return;
    }
    s.square = fabs(fr - jb.nocc) < fabs(2.0 * tr - fr - jb.nocc) ? 1 : 0;
    atomicAdd(active_count, 1);
}

// P_new = w X (the converged X); molecules whose purification stalled are flagged for the
// eigensolver path.
__global__ void k_sp2_finish(const Sp2Job* __restrict__ jobs, const Sp2State* __restrict__ sst, const MolState* __restrict__ st,
                             int* __restrict__ need_eigen, double* __restrict__ work) {
    const Sp2Job jb = jobs[blockIdx.y];
    if (!st[jb.mol].active) return;
    const Sp2State& s = sst[blockIdx.y];
    if (!s.converged) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            need_eigen[jb.mol] = 1;
            atomicAdd(&work[2], 1.0);
        }
        return;
    }
    const double* X = s.cur ? jb.X1 : jb.X0;
    const long long nn = (long long)jb.n * jb.n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (long long)gridDim.x * blockDim.x)
        jb.P[i] = jb.weight * X[i];
}

size_t dgemm_smem_bytes() { return DG_SMEM; }

}  // namespace am1
