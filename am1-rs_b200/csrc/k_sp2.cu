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
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {

namespace cg = cooperative_groups;


// Spectral bounds [e_min, e_max] of F* for the SP2 mapping.  The number of purification steps
// grows with the width of the interval, and the Gershgorin interval of an NDDO Fock matrix is
// about twice the true spectral width (the row sums over the many small long-range elements), so
// the bounds come from a short Lanczos run (SP2_LANCZOS steps from a fixed start vector, no
// reorthogonalisation: only the extreme Ritz values are used):
//     e_max = min(Gershgorin max, theta_max + r_max + 0.005 w)
//     e_min = max(Gershgorin min, theta_min - r_min - 0.005 w)
// with r = |beta_m s_m| the residual of the extreme Ritz pair (s from inverse iteration on the
// Lanczos tridiagonal T) and w = theta_max - theta_min.  An eigenvalue left slightly outside
// the interval maps just outside [0, 1], where the trace-correcting steps pull it back; a run
// that still fails to converge falls back to the eigensolver.  One CTA per channel.
constexpr int SP2_LANCZOS = 12;
// largest widening of a reused spectral interval, as a fraction of the width of the last Lanczos run's
constexpr double SP2_REUSE_FRAC = 0.01;
constexpr int SP2_BOUND_THREADS = 512;

__device__ double bounds_block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < SP2_BOUND_THREADS / 32; ++w) t += red[w];
    return t;
}

// Eigenvalues of T (m x m, diagonal a, off-diagonal b) below x.
__device__ int lz_count(const double* a, const double* b, int m, double x) {
    int c = 0;
    double q = a[0] - x;
    if (q < 0.0) ++c;
    for (int i = 1; i < m; ++i) {
        q = a[i] - x - b[i - 1] * b[i - 1] / (q == 0.0 ? 1e-300 : q);
        if (q < 0.0) ++c;
    }
    return c;
}

// k-th smallest eigenvalue of T by bisection inside [lo, hi].
__device__ double lz_eig(const double* a, const double* b, int m, int k, double lo, double hi) {
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (!(mid > lo && mid < hi)) break;
        if (lz_count(a, b, m, mid) <= k) lo = mid;
        else hi = mid;
    }
    return 0.5 * (lo + hi);
}

// The same eigenvalue by one warp: 32-way multisection, each round 31 Sturm counts at interior
// points of [lo, hi] on the lanes and the interval narrowed to the gap where the count passes k (a
// factor 32 per round; 11 rounds reach the rounding level of the bisection).  Every lane of the warp
// calls it and gets the same value.
__device__ double lz_eig_warp(const double* a, const double* b, int m, int k, double lo, double hi) {
    const int lane = threadIdx.x & 31;
    for (int round = 0; round < 11; ++round) {
        const double h = (hi - lo) * (1.0 / 32.0);
        if (!(h > 0.0)) break;
        const double x = lo + h * (lane + 1);
        const bool below = lane < 31 && lz_count(a, b, m, x) <= k;  // x <= the k-th eigenvalue
        const unsigned ball = __ballot_sync(0xffffffffu, below);
        const int j = ball ? 31 - __clz(ball) : -1;  // the last interior point still below it
        const double nlo = j >= 0 ? lo + h * (j + 1) : lo;
        const double nhi = j + 2 <= 31 ? lo + h * (j + 2) : hi;
        lo = nlo;
        hi = nhi;
    }
    return 0.5 * (lo + hi);
}

// |last component| of the unit eigenvector of T for an exterior eigenvalue: inverse iteration
// with the shift sigma just outside the spectrum, so T - sigma I is definite and the
// tridiagonal solve needs no pivoting.
__device__ double lz_last_component(const double* a, const double* b, int m, double sigma) {
    double x[SP2_LANCZOS], cp[SP2_LANCZOS], rp[SP2_LANCZOS];
    for (int i = 0; i < m; ++i) x[i] = 1.0;
    for (int it = 0; it < 3; ++it) {
        double den = a[0] - sigma;
        cp[0] = m > 1 ? b[0] / den : 0.0;
        rp[0] = x[0] / den;
        for (int i = 1; i < m; ++i) {
            den = a[i] - sigma - b[i - 1] * cp[i - 1];
            cp[i] = i + 1 < m ? b[i] / den : 0.0;
            rp[i] = (x[i] - b[i - 1] * rp[i - 1]) / den;
        }
        x[m - 1] = rp[m - 1];
        for (int i = m - 2; i >= 0; --i) x[i] = rp[i] - cp[i] * x[i + 1];
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += x[i] * x[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0.0) || !isfinite(nrm)) return 1.0;
        for (int i = 0; i < m; ++i) x[i] /= nrm;
    }
    return fabs(x[m - 1]);
}

__global__ void __launch_bounds__(SP2_BOUND_THREADS) k_sp2_bounds(const Sp2Job* __restrict__ jobs, const MolState* __restrict__ st) {
    const Sp2Job jb = jobs[blockIdx.x];
    if (!st[jb.mol].active || !jb.fallback) return;  // large matrices: k_sp2_bounds_big
    const int n = jb.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = SP2_BOUND_THREADS / 32;
    extern __shared__ double lz[];
    double* q = lz;        // current Lanczos vector
    double* qp = lz + n;   // previous one
    double* w = lz + 2 * n;
    __shared__ double red[NW];
    __shared__ double alpha[SP2_LANCZOS], beta[SP2_LANCZOS];
    // Gershgorin interval (rows of F*)
    __shared__ double gred[2][NW];
    double glo = 1e300, ghi = -1e300;
    for (int i = tid; i < n; i += SP2_BOUND_THREADS) {
        glo = fmin(glo, jb.rowmin[i]);
        ghi = fmax(ghi, jb.rowmax[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
        ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
    }
    if (lane == 0) {
        gred[0][warp] = glo;
        gred[1][warp] = ghi;
    }
    // From the second SCF iteration on, F* has moved by delta = ||F* - F*_previous||_F from the matrix
    // of the previous interval, and no eigenvalue moves further than that (Weyl's inequality,
    // |lambda_i(A + E) - lambda_i(A)| <= ||E||_2 <= ||E||_F).  While the widening added since the last
    // Lanczos run stays below SP2_REUSE_FRAC of that run's width, the previous interval widened by
    // delta on both sides (and capped by the Gershgorin interval of F*) is taken instead of a new run.
    const bool may_reuse = jb.rowdf != nullptr && st[jb.mol].iter > 0;
    const double b_lo = jb.bounds[0], b_hi = jb.bounds[1], b_slack = jb.bounds[2], b_width = jb.bounds[3];
    double dsum = 0.0;
    if (may_reuse)
        for (int i = tid; i < n; i += SP2_BOUND_THREADS) dsum += jb.rowdf[i];
    dsum = bounds_block_sum(dsum, red);  // its barriers also publish gred
    if (may_reuse) {
        double rlo = gred[0][0], rhi = gred[1][0];
        for (int v = 1; v < NW; ++v) {
            rlo = fmin(rlo, gred[0][v]);
            rhi = fmax(rhi, gred[1][v]);
        }
        const double delta = sqrt(dsum) * (1.0 + 1e-12);
        const double slack = b_slack + delta;
        const double lo = fmax(b_lo - delta, rlo), hi = fmin(b_hi + delta, rhi);
        if (isfinite(slack) && b_width > 0.0 && slack <= SP2_REUSE_FRAC * b_width && hi > lo) {
            __syncthreads();  // every thread has read the previous interval
            if (tid == 0) {
                jb.bounds[0] = lo;
                jb.bounds[1] = hi;
                jb.bounds[2] = slack;
            }
            return;
        }
    }
    // fixed start vector, normalised
    double nq = 0.0;
    for (int i = tid; i < n; i += SP2_BOUND_THREADS) {
        const double x = cos(0.7 * i + 0.3) + 0.5;
        q[i] = x;
        qp[i] = 0.0;
        nq += x * x;
    }
    nq = bounds_block_sum(nq, red);  // its barriers also publish gred
    glo = gred[0][0];
    ghi = gred[1][0];
    for (int v = 1; v < NW; ++v) {
        glo = fmin(glo, gred[0][v]);
        ghi = fmax(ghi, gred[1][v]);
    }
    const double inq = 1.0 / sqrt(nq);
    for (int i = tid; i < n; i += SP2_BOUND_THREADS) q[i] *= inq;
    __syncthreads();
    const int K = min(SP2_LANCZOS, n);
    const bool pairs = (n & 1) == 0 && (reinterpret_cast<uintptr_t>(jb.F) & 15) == 0;
    int m = 0;
    double bprev = 0.0;
    for (int j = 0; j < K; ++j) {
        // w = F q: eight lanes per row, so every warp has four rows' loads in flight; rows of even
        // length on 16-byte boundaries are read as pairs (16-byte loads, two partial sums per lane)
        const int sub = lane >> 3, sl = lane & 7;
        for (int r0 = 4 * warp; r0 < n; r0 += 4 * NW) {
            const int r = r0 + sub;
            double acc = 0.0;
            if (r < n) {
                const double* Fr = jb.F + (long long)r * n;
                if (pairs) {
                    const double2* F2 = reinterpret_cast<const double2*>(Fr);
                    const double2* q2 = reinterpret_cast<const double2*>(q);
                    double acc1 = 0.0;
#pragma unroll 4
                    for (int c = sl; c < n / 2; c += 8) {
                        const double2 f = F2[c], x = q2[c];
                        acc = fma(f.x, x.x, acc);
                        acc1 = fma(f.y, x.y, acc1);
                    }
                    acc += acc1;
                } else {
                    for (int c = sl; c < n; c += 8) acc = fma(Fr[c], q[c], acc);
                }
            }
            for (int o = 4; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (sl == 0 && r < n) w[r] = acc;
        }
        __syncthreads();
        double part = 0.0;
        for (int i = tid; i < n; i += SP2_BOUND_THREADS) part += q[i] * w[i];
        const double a = bounds_block_sum(part, red);
        part = 0.0;
        for (int i = tid; i < n; i += SP2_BOUND_THREADS) {
            const double x = w[i] - a * q[i] - bprev * qp[i];
            w[i] = x;
            part += x * x;
        }
        const double bnorm = sqrt(bounds_block_sum(part, red));
        if (tid == 0) {
            alpha[j] = a;
            beta[j] = bnorm;
        }
        m = j + 1;
        if (!(bnorm > 1e-12 * fmax(fabs(a), 1.0))) break;  // invariant subspace: T is exact
        const double ib = 1.0 / bnorm;
        for (int i = tid; i < n; i += SP2_BOUND_THREADS) {
            qp[i] = q[i];
            q[i] = w[i] * ib;
        }
        bprev = bnorm;
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) {
        // Gershgorin interval of T contains its spectrum
        double tlo = 1e300, thi = -1e300;
        for (int i = 0; i < m; ++i) {
            const double rad = (i > 0 ? fabs(beta[i - 1]) : 0.0) + (i + 1 < m ? fabs(beta[i]) : 0.0);
            tlo = fmin(tlo, alpha[i] - rad);
            thi = fmax(thi, alpha[i] + rad);
        }
        const double pad = 1e-12 * (fabs(tlo) + fabs(thi)) + 1e-300;
        tlo -= pad;
        thi += pad;
        const double th_min = lz_eig_warp(alpha, beta, m, 0, tlo, thi);
        const double th_max = lz_eig_warp(alpha, beta, m, m - 1, tlo, thi);
        if (lane != 0) return;
        const double width = fmax(th_max - th_min, 1e-6);
        const double eps = 1e-8 * (fabs(th_min) + fabs(th_max) + 1.0);
        const double bm = beta[m - 1];
        const double r_min = fabs(bm) * lz_last_component(alpha, beta, m, th_min - eps);
        const double r_max = fabs(bm) * lz_last_component(alpha, beta, m, th_max + eps);
        double lo = th_min - r_min - 0.005 * width;
        double hi = th_max + r_max + 0.005 * width;
        if (!isfinite(lo) || !isfinite(hi) || !(hi > lo)) {
            lo = glo;
            hi = ghi;
        }
        jb.bounds[0] = fmax(lo, glo);
        jb.bounds[1] = fmin(hi, ghi);
        jb.bounds[2] = 0.0;
        jb.bounds[3] = jb.bounds[1] - jb.bounds[0];
    }
}

// The interval from the Lanczos tridiagonal (alpha, beta of m steps) and the Gershgorin bounds.
__device__ void lz_interval(const double* alpha, const double* beta, int m, double glo, double ghi, double* out) {
    double tlo = 1e300, thi = -1e300;
    for (int i = 0; i < m; ++i) {
        const double rad = (i > 0 ? fabs(beta[i - 1]) : 0.0) + (i + 1 < m ? fabs(beta[i]) : 0.0);
        tlo = fmin(tlo, alpha[i] - rad);
        thi = fmax(thi, alpha[i] + rad);
    }
    const double pad = 1e-12 * (fabs(tlo) + fabs(thi)) + 1e-300;
    tlo -= pad;
    thi += pad;
    const double th_min = lz_eig(alpha, beta, m, 0, tlo, thi);
    const double th_max = lz_eig(alpha, beta, m, m - 1, tlo, thi);
    const double width = fmax(th_max - th_min, 1e-6);
    const double eps = 1e-8 * (fabs(th_min) + fabs(th_max) + 1.0);
    const double bm = beta[m - 1];
    const double r_min = fabs(bm) * lz_last_component(alpha, beta, m, th_min - eps);
    const double r_max = fabs(bm) * lz_last_component(alpha, beta, m, th_max + eps);
    double lo = th_min - r_min - 0.005 * width;
    double hi = th_max + r_max + 0.005 * width;
    if (!isfinite(lo) || !isfinite(hi) || !(hi > lo)) {
        lo = glo;
        hi = ghi;
    }
    out[0] = fmax(lo, glo);
    out[1] = fmin(hi, ghi);
}

// k_sp2_bounds for one matrix too large for one CTA (no eigensolver fallback, n > ~448): the same
// Lanczos run by a group of G CTAs, either the whole GPU (one cooperative launch per matrix) or a
// thread-block cluster (one cluster per matrix, all such matrices of a batch in one launch).
// Row r of F* belongs to CTA r % G; the vectors live in global scratch (job.X1, free until
// purification starts) and every CTA keeps the same alpha, beta (sums of the per-CTA shares in one
// fixed order).  Three group barriers per step; cross-CTA data is read through L2 (__ldcg).
// Scratch: q[3][n] | share[2][G].
template <class Sync>
__device__ void sp2_bounds_group(const Sp2Job& jb, int G, int gi, Sync sync) {
    const int n = jb.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = SP2_BOUND_THREADS / 32;
    double* qb = jb.X1;                 // three Lanczos vectors
    double* share = qb + 3 * (size_t)n; // [2][G]
    __shared__ double red[NW + 2];
    __shared__ double alpha[SP2_LANCZOS], beta[SP2_LANCZOS];
    auto bsum = [&](double v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if (lane == 0) red[warp] = v;
        __syncthreads();
        double t = 0.0;
        for (int q = 0; q < NW; ++q) t += red[q];
        __syncthreads();
        return t;
    };
    // Gershgorin interval and the start vector (every CTA computes the norm itself)
    double glo = 1e300, ghi = -1e300, nq = 0.0;
    for (int i = tid; i < n; i += SP2_BOUND_THREADS) {
        glo = fmin(glo, jb.rowmin[i]);
        ghi = fmax(ghi, jb.rowmax[i]);
        const double x = cos(0.7 * i + 0.3) + 0.5;
        nq += x * x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
        ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
    }
    __shared__ double gred[2][NW];
    if (lane == 0) {
        gred[0][warp] = glo;
        gred[1][warp] = ghi;
    }
    nq = bsum(nq);
    glo = gred[0][0];
    ghi = gred[1][0];
    for (int v = 1; v < NW; ++v) {
        glo = fmin(glo, gred[0][v]);
        ghi = fmax(ghi, gred[1][v]);
    }
    const double inq = 1.0 / sqrt(nq);
    for (int i = gi * SP2_BOUND_THREADS + tid; i < n; i += G * SP2_BOUND_THREADS) {
        qb[i] = (cos(0.7 * i + 0.3) + 0.5) * inq;  // q_0
        qb[2 * (size_t)n + i] = 0.0;            // q_{-1}
    }
    sync();
    const int K = min(SP2_LANCZOS, n);
    int m = 0, cur = 0, prv = 2;
    double bprev = 0.0;
    for (int j = 0; j < K; ++j) {
        const int nxt = 3 - cur - prv;  // the third buffer: w, then q_{j+1}
        const double* q = qb + (size_t)cur * n;
        const double* qp = qb + (size_t)prv * n;
        double* wq = qb + (size_t)nxt * n;
        // w_r = F[r, :] . q for own rows (a warp per row) and the CTA's share of q . w
        double part = 0.0;
        for (int r = gi + warp * G; r < n; r += NW * G) {
            const double* Fr = jb.F + (long long)r * n;
            double acc = 0.0;
#pragma unroll 4
            for (int c = lane; c < n; c += 32) acc = fma(Fr[c], __ldcg(q + c), acc);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) wq[r] = acc;
            part += acc * __ldcg(q + r);
        }
        part = bsum(lane == 0 ? part : 0.0);
        if (tid == 0) share[gi] = part;
        sync();
        const double a = group_share_sum(share, G);
        // w <- w - a q - b_prev q_prev on own rows, the CTA's share of |w|^2
        part = 0.0;
        for (int r = gi + warp * G; r < n; r += NW * G) {
            if (lane == 0) {
                const double x = __ldcg(wq + r) - a * __ldcg(q + r) - bprev * __ldcg(qp + r);
                wq[r] = x;
                part += x * x;
            }
        }
        part = bsum(part);
        if (tid == 0) share[G + gi] = part;
        sync();
        const double bnorm = sqrt(group_share_sum(share + G, G));
        if (tid == 0) {
            alpha[j] = a;
            beta[j] = bnorm;
        }
        m = j + 1;
        if (!(bnorm > 1e-12 * fmax(fabs(a), 1.0))) break;  // invariant subspace: T is exact (uniform)
        const double ib = 1.0 / bnorm;
        for (int r = gi + warp * G; r < n; r += NW * G)
            if (lane == 0) wq[r] = __ldcg(wq + r) * ib;
        bprev = bnorm;
        prv = cur;
        cur = nxt;
        sync();
    }
    __syncthreads();
    if (gi == 0 && tid == 0) lz_interval(alpha, beta, m, glo, ghi, jb.bounds);
}

__global__ void __launch_bounds__(SP2_BOUND_THREADS) k_sp2_bounds_big(const Sp2Job* __restrict__ jobs, int job,
                                                                       const MolState* __restrict__ st) {
    cg::grid_group grid = cg::this_grid();
    const Sp2Job jb = jobs[job];
    if (!st[jb.mol].active) return;  // uniform over the grid
    sp2_bounds_group(jb, (int)gridDim.x, (int)blockIdx.x, [&] { grid.sync(); });
}

// One cluster (gridDim.x CTAs) per large matrix; blockIdx.y indexes big[], the purification jobs
// without the eigensolver fallback.
__global__ void __launch_bounds__(SP2_BOUND_THREADS) k_sp2_bounds_cl(const Sp2Job* __restrict__ jobs, const int* __restrict__ big,
                                                                      const MolState* __restrict__ st) {
    cg::cluster_group cl = cg::this_cluster();
    const Sp2Job jb = jobs[big[blockIdx.y]];
    if (!st[jb.mol].active) return;  // uniform over the cluster
    sp2_bounds_group(jb, (int)cl.num_blocks(), (int)cl.block_rank(), [&] { cl.sync(); });
}

// X0 = (e_max I - F*) / (e_max - e_min); per-block partial sums of tr X0 and ||X0||_F^2.
__global__ void k_sp2_init(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, const MolState* __restrict__ st, int nblk) {
    const Sp2Job jb = jobs[blockIdx.y];
    if (!st[jb.mol].active) return;
    const int n = jb.n;
    const int nb = sp2_init_blocks(n);
    if ((int)blockIdx.x >= nb) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    __shared__ double red[2][32];
    const double emin = jb.bounds[0], emax = jb.bounds[1];  // from k_sp2_bounds
    const double inv = 1.0 / fmax(emax - emin, 1e-300);
    const bool lowp = st[jb.mol].lowp;
    double tr = 0.0, fr = 0.0;
    for (int r = blockIdx.x * nw + warp; r < n; r += nb * nw) {
        const double* Fr = jb.F + (long long)r * n;
        if (lowp) {  // FP32 iterate (rows of ldf floats, pad columns zero in both buffers)
            float* Xr = jb.Xf0 + (long long)r * jb.ldf;
            for (int c = lane; c < jb.ldf; c += 32) {
                const float xf = c < n ? (float)(((c == r ? emax : 0.0) - Fr[c]) * inv) : 0.0f;
                const float x = jb.lowp_tc == 1 ? xf : tf32_round(xf);  // 3xTF32 keeps the full FP32 iterate
                Xr[c] = x;
                if (c >= n) jb.Xf1[(long long)r * jb.ldf + c] = 0.0f;
                fr += (double)x * x;
                if (c == r) tr += x;
            }
            continue;
        }
        double* Xr = jb.X0 + (long long)r * n;
        // four columns per lane per trip, their loads before their stores (each lane keeps its order)
        for (int c0 = lane; c0 < n; c0 += 128) {
            double f[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) f[u] = c0 + 32 * u < n ? Fr[c0 + 32 * u] : 0.0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int c = c0 + 32 * u;
                if (c >= n) break;
                const double x = ((c == r ? emax : 0.0) - f[u]) * inv;
                Xr[c] = x;
                fr += x * x;
                if (c == r) tr += x;
            }
        }
        if (jb.oz) {  // the digit planes of X0, and zero pad columns in both digit buffers
            const long long plane = (long long)n * jb.ldq;
            for (int c = lane; c < jb.ldq; c += 32) {
                const long long o = (long long)r * jb.ldq + c;
                if (c < n) {
                    oz_digits_of(Xr[c], jb.Dq0, plane, o);
                } else {
                    for (int i = 0; i < kOzPlanes; ++i) jb.Dq0[i * plane + o] = jb.Dq1[i * plane + o] = 0;
                }
            }
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
    s.lowp = st[jb.mol].lowp;
    s.steps = 0;
    s.cur = 0;
    s.converged = 0;
    double tr = 0.0, fr = 0.0;
    for (int b = 0; b < sp2_init_blocks(jb.n); ++b) {
        tr += jb.part[2 * b];
        fr += jb.part[2 * b + 1];
    }
    s.trX = tr;
    s.trX2 = fr;
    s.idem[0] = s.idem[1] = 1e300;
    s.square = fabs(fr - jb.nocc) < fabs(2.0 * tr - fr - jb.nocc) ? 1 : 0;
}

// Epilogue of one purification-step tile: Y = X^2 or 2X - X^2 for r <= c, mirrored; the tile's
// partial trace and Frobenius sums into the job's partials (the job fields it needs are read only
// now, so they hold no registers during the k-loop).
__device__ __forceinline__ void sp2_step_epilogue(const Sp2Job* __restrict__ jp, const Sp2State* __restrict__ sp, int t, int n,
                                                  int m0, int n0, const double acc[2][4][4], bool compute, double red[2][4]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cur = sp->cur;
    const double* X = cur ? jp->X1 : jp->X0;
    double* Y = cur ? jp->X0 : jp->X1;
    const int square = sp->square;
    double tr = 0.0, fr = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = m0 + dg_row(i, e);
                const int c = n0 + dg_col(j, e);
                if (compute && r <= c && c < n) {
                    const double x2 = acc[i][j][e];
                    const double y = square ? x2 : 2.0 * X[(long long)r * n + c] - x2;
                    Y[(long long)r * n + c] = y;
                    if (r < c) {
                        Y[(long long)c * n + r] = y;
                        fr += 2.0 * y * y;
                    } else {
                        fr += y * y;
                        tr += y;
                    }
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
        double* p = jp->part + 2 * (t - jp->tile0);
        p[0] = red[0][0] + red[0][1] + red[0][2] + red[0][3];
        p[1] = red[1][0] + red[1][1] + red[1][2] + red[1][3];
    }
}

// One SP2 step over all upper-triangle 64x64 tiles of every active channel (operands copied by
// cp.async: k_sp2_step8 for odd n, and k_sp2_step16 where the tensor-map kernel is not used).
template <bool PAIRS>
__device__ __forceinline__ void sp2_step_body(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles, int ntiles,
                                              const Sp2State* __restrict__ sst) {
    extern __shared__ __align__(16) double dsm[];
    __shared__ double red[2][4];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || sp->lowp || jp->oz) return;  // TF32 runs: k_sp2_step_tf32 / _tc; digit products: k_sp2_step_oz
    const int n = jp->n;
    const double* X = sp->cur ? jp->X1 : jp->X0;
    const int m0 = tl.tm * DG_TILE, n0 = tl.tn * DG_TILE;
    // only the upper triangle of X^2 is computed: a warp whose quarter is padding or lies below
    // the diagonal of a diagonal tile issues no MMAs
    const bool compute = dg_quarter_on(m0, n0, n, n, tl.tm == tl.tn);
    double acc[2][4][4];
    dg_mainloop<PAIRS>(dsm, X, n, X, n, n, n, n, m0, n0, acc, compute);  // X symmetric: X[rows m0..] . X[:, n0..]
    sp2_step_epilogue(jp, sp, t, n, m0, n0, acc, compute, red);
}

// The same step for even n with the operands copied by the tensor memory accelerator from the
// job's tensor maps (maps[4 job + cur] describes the current iterate), through the mbarrier
// pipeline of dg_mainloop_tma: bit-identical to k_sp2_step16.  A copy wait that runs out sets bit
// 11 of *err and the tile is left unwritten.
__global__ void __launch_bounds__(DG_THREADS, 4) k_sp2_step_tma(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                               int ntiles, const Sp2State* __restrict__ sst,
                                                               const TmaDesc* __restrict__ maps, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char dtsm[];
    __shared__ DtBars bars;
    __shared__ double red[2][4];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || sp->lowp || jp->oz) return;
    const int n = jp->n;
    const int m0 = tl.tm * DG_TILE, n0 = tl.tn * DG_TILE;
    const int shape = dg_quarter_shape(m0, n0, n, n, tl.tm == tl.tn);
    const bool compute = shape != 0;
    const TmaDesc* map = maps + 4 * tl.job + sp->cur;
    double acc[2][4][4];
    if (!dg_mainloop_tma(dt_stages(dtsm), bars, map, map, nullptr, nullptr, tl.tm == tl.tn, n, m0, n0, acc, shape)) {
        if (threadIdx.x == 0) atomicOr(err, 1 << 11);
        return;
    }
    sp2_step_epilogue(jp, sp, t, n, m0, n0, acc, compute, red);
}

// After a step: reduce the tile partials (in tile order), test idempotency, choose the next branch.
// The update of channel j after its product; true while it still purifies.
__device__ __forceinline__ bool sp2_update_job(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, int j, int max_steps,
                                               double* __restrict__ work) {
    Sp2State& s = sst[j];
    if (!s.active) return false;
    const Sp2Job jb = jobs[j];
    // algorithmic work of the product just taken: a symmetric X.X, n^3 flops
    if (s.lowp) {
        atomicAdd(&work[4], 1.0);
        atomicAdd(&work[5], (double)jb.n * jb.n * jb.n);
    } else {
        atomicAdd(&work[0], 1.0);
        atomicAdd(&work[1], (double)jb.n * jb.n * jb.n);
        atomicAdd(&work[3], 16.0 * jb.n * jb.n);  // read X, write X^2 (both triangles), FP64
    }
    double tr = 0.0, fr = 0.0;
    // the partial sums come from the tiles of the kernel that took the product
    const int nparts = s.lowp ? (jb.lowp_tc ? jb.tc_ntiles : jb.ntiles) : (jb.oz ? jb.oz_ntiles : jb.ntiles);
    for (int t = 0; t < nparts; ++t) {
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
    // TF32 runs stop at their own rounding level (about 1e-6 relative per eigenvalue), and their
    // result is always taken: it only starts the FP64 iterations
    const bool low_done = s.lowp && ((idem < 1.0e-2 * jb.n && idem >= s.idem[0]) || idem < 1.0e-5 * jb.n);
    s.idem[0] = s.idem[1];
    s.idem[1] = idem;
    if (low_done || floor_reached || idem < 1.0e-15 * fmax(1.0, (double)jb.n)) {
        s.active = 0;
        s.converged = 1;
        return false;
    }
    if (s.steps >= max_steps) {
        s.active = 0;
        s.converged = s.lowp;
        return false;
    }
    s.square = fabs(fr - jb.nocc) < fabs(2.0 * tr - fr - jb.nocc) ? 1 : 0;
    return true;
}

__global__ void k_sp2_update(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, int njobs, int max_steps,
                             int* __restrict__ active_count, double* __restrict__ work) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    if (sp2_update_job(jobs, sst, j, max_steps, work)) atomicAdd(active_count, 1);
}

// The update of every channel and the purification loop's decision in one CTA (the captured solve
// of a batch of at most SP2_UPDATE_ONE channels): the same per-channel update, the channels still
// purifying counted by the CTA, then k_sp2_cond's step counters and condition.
__global__ void __launch_bounds__(SP2_UPDATE_ONE) k_sp2_update_cond(const Sp2Job* __restrict__ jobs, Sp2State* __restrict__ sst, int njobs,
                                                                    int max_steps, double* __restrict__ work,
                                                                    cudaGraphConditionalHandle h, GraphLoop* __restrict__ loop) {
    const int j = threadIdx.x;
    const bool more_j = j < njobs && sp2_update_job(jobs, sst, j, max_steps, work);
    const int active = __syncthreads_count(more_j);
    if (threadIdx.x == 0) {
        const int step = loop->sp2_step + 1;
        loop->sp2_step = step;
        loop->sp2_total += 1;
        cudaGraphSetConditional(h, (active > 0 && step < max_steps) ? 1u : 0u);
    }
}

// P_new = w X (the converged X); molecules whose purification stalled are flagged for the
// eigensolver path: need_eigen (cluster Jacobi, up to 448 orbitals) or big_stall per channel job
// and the count in big_count (the large-matrix eigensolver, above 448).
__global__ void k_sp2_finish(const Sp2Job* __restrict__ jobs, const Sp2State* __restrict__ sst, const MolState* __restrict__ st,
                             int* __restrict__ need_eigen, double* __restrict__ work, int* __restrict__ big_stall,
                             int* __restrict__ big_count) {
    const Sp2Job jb = jobs[blockIdx.y];
    if (!st[jb.mol].active) return;
    const Sp2State& s = sst[blockIdx.y];
    if (!s.converged) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            atomicAdd(&work[2], 1.0);
            if (jb.fallback) {
                need_eigen[jb.mol] = 1;
            } else {  // above the cluster Jacobi's size: the host runs the large-matrix eigensolver
                big_stall[blockIdx.y] = 1;
                atomicAdd(big_count, 1);
            }
        }
        return;
    }
    const long long nn = (long long)jb.n * jb.n;
    if (s.lowp) {
        // the TF32 iterate, rescaled to the exact electron count (its trace is off by the rounding)
        const float* Xf = s.cur ? jb.Xf1 : jb.Xf0;
        const double w = jb.weight * (s.trX > 0.0 ? jb.nocc / s.trX : 1.0);
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (long long)gridDim.x * blockDim.x) {
            const long long r = i / jb.n, c = i - r * jb.n;
            jb.P[i] = w * (double)Xf[r * jb.ldf + c];
        }
        return;
    }
    const double* X = s.cur ? jb.X1 : jb.X0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < nn; i0 += 4 * stride) {
        double x[4];  // P may be X0: every load of the trip before its stores
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = i0 + u * stride < nn ? X[i0 + u * stride] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (i0 + u * stride < nn) jb.P[i0 + u * stride] = jb.weight * x[u];
    }
}

size_t dgemm_smem_bytes() { return DG_SMEM; }
size_t dgemm_tma_smem_bytes() { return DT_SMEM; }

__global__ void __launch_bounds__(DG_THREADS, 4) k_sp2_step16(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                              int ntiles, const Sp2State* __restrict__ sst) {
    sp2_step_body<true>(jobs, tiles, ntiles, sst);
}
__global__ void __launch_bounds__(DG_THREADS, 4) k_sp2_step8(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                             int ntiles, const Sp2State* __restrict__ sst) {
    sp2_step_body<false>(jobs, tiles, ntiles, sst);
}

}  // namespace am1
