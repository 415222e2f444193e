// Eigenvalues of the last extrapolated Fock matrix (the reference's mo_energies are the
// eigenvalues of the F* of its last iteration, src/scf.rs:654-689), without eigenvectors:
//   k_tridiag : Householder reduction A = Q T Q^T (Golub & Van Loan, Alg. 8.3.1), the matrix held
//               in the shared memory of a thread-block cluster (rows spread over its CTAs);
//   k_bisect  : every eigenvalue of T by bisection on the Sturm sequence count (Barth, Martin &
//               Wilkinson), one thread per eigenvalue index, ascending by construction.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {

namespace cg = cooperative_groups;

// Householder reduction of one symmetric matrix held on chip.  The n x n matrix is distributed by
// rows over a thread-block cluster of C CTAs (row r lives in CTA r % C, at local row r / C, full
// length n), so the whole reduction runs out of shared memory; C is the smallest cluster whose
// share fits one CTA.  Reflector s (GVL Alg. 8.3.1) zeroes row/column s below the subdiagonal:
// v_s = x + sign(x0)|x| e1 from x = A[s, s+1:], beta_s = 1/(|x|(|x| + |x0|)), and the trailing
// block takes the rank-2 update A -= v w^T + w v^T with p = beta A v, w = p - (beta/2)(p.v) v.
// Iteration s of the loop:
//   (a) one warp of the owner of row s applies update s-1 to row s and derives reflector s
//   cluster barrier: v_s ready; the other CTAs copy it (distributed shared memory)
//   (b) one fused pass over the CTA's rows > s, a thread per column > s: apply update s-1 and
//       accumulate this CTA's share of A v_s (A symmetric: column r of the share is a dot product
//       down the rows, so consecutive threads read consecutive words)
//   cluster barrier: every CTA's share ready; each CTA sums the C shares itself -> p, w_s
// Column s below the diagonal is never updated: row s holds the same numbers and is the one read.
// All control flow is uniform over the cluster, so every CTA takes the same barriers.
// With job.stop > 0 the loop ends after reflector stop - 1: the trailing block (rows and columns
// >= stop) with update stop - 1 applied goes to job.W (row-major, n - stop rows), and a job on fewer
// CTAs reduces it as a matrix of its own, writing d and e from index stop on.  Its tridiagonal
// continues this one's: the block's reflectors act on indices >= stop + 1 and leave e[stop - 1] as is.
constexpr int TRI_THREADS = 512;
constexpr int TRI_WARPS = TRI_THREADS / 32;

// Dynamic shared memory of one CTA: local rows, v and w (two buffers each), the share of A v,
// beta (two buffers) and two reduction scratches.
size_t tridiag_smem_bytes(int n, int C) {
    const size_t rows = (size_t)(n + C - 1) / C;
    return sizeof(double) * (rows * n + 5 * (size_t)n + 2 + TRI_WARPS + TRI_THREADS);
}

// Householder vector of row `row` (the trailing part from column s + 1), computed by one warp:
// v into vbuf, beta into *beta, and d[s], e[s].
__device__ __forceinline__ void tri_reflector(const double* row, int s, int n, double* vbuf, double* beta, double* d, double* e) {
    const int lane = threadIdx.x & 31, c0 = s + 1;
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
        d[s] = row[s];
        e[s] = alpha == 0.0 ? 0.0 : -sg * alpha;
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
    double* A = sh;                    // R x n: global row lr * C + crank at local row lr
    double* vb = A + (size_t)R * n;    // v, two buffers of n (global column index)
    double* wb = vb + 2 * (size_t)n;   // w, two buffers of n
    double* pp = wb + 2 * (size_t)n;   // this CTA's share of A v
    double* bb = pp + n;               // beta, two buffers
    double* red = bb + 2;              // [TRI_WARPS]
    double* red2 = red + TRI_WARPS;    // [TRI_THREADS] partial column sums of the row groups
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
    for (int c = tid; c < n; c += TRI_THREADS) {  // update "-1" is the identity
        vb[n + c] = 0.0;
        wb[n + c] = 0.0;
    }
    __syncthreads();
    for (int s = 0; s + 1 < n; ++s) {
        const int cur = (s + 1) & 1, nxt = s & 1;
        const double* v = vb + (size_t)cur * n;  // reflector s - 1
        const double* w = wb + (size_t)cur * n;
        double* vn = vb + (size_t)nxt * n;       // reflector s
        const bool has_next = s + 2 < n;
        const int owner = s % C;
        if (crank == owner && warp == 0) {  // (a)
            double* row = A + (size_t)(s / C) * n;
            const double vs = v[s], ws = w[s];
            for (int c = s + lane; c < n; c += 32) row[c] -= vs * w[c] + ws * v[c];
            __syncwarp();
            if (has_next) tri_reflector(row, s, n, vn, bb + nxt, jb.d, jb.e);
        }
        csync();  // v_s ready in the owner
        if (has_next && crank != owner) {
            const double* rv = cluster.map_shared_rank(vn, owner);
            for (int c = s + 1 + tid; c < n; c += TRI_THREADS) vn[c] = rv[c];
            if (tid == 0) bb[nxt] = *cluster.map_shared_rank(bb + nxt, owner);
            __syncthreads();
        }
        // (b) columns r > s, rows c > s of this CTA: threads in G groups of cpg; thread (g, j) owns
        // column s + 1 + j and rows lr0 + g, lr0 + g + G, ... (more groups when there are few columns)
        const int lr0 = (s + 1 - crank + C - 1) / C;  // first local row with global index > s
        const int lre = (n - crank + C - 1) / C;      // local rows with global index < n
        const int ncol = n - (s + 1);
        const int G = max(1, min(16, TRI_THREADS / (((ncol + 31) / 32) * 32)));
        const int cpg = TRI_THREADS / G;
        const int g = tid / cpg, j = tid - g * cpg;
        // columns s + 1 + j, j = this thread's index in its group, then strided by the group size
        // (more columns than threads take several trips; more groups only when columns are few)
        for (int jj = j; jj < ncol || (G > 1 && jj == j); jj += cpg) {
            double acc = 0.0;
            if (g < G && jj < ncol) {
                const int r = s + 1 + jj;
                const double vr = v[r], wr = w[r];
                int lr = lr0 + g;
                for (; lr + 3 * G < lre; lr += 4 * G) {  // four independent rows per trip
                    double* a0 = A + (size_t)lr * n + r;
                    double* a1 = a0 + (size_t)G * n;
                    double* a2 = a1 + (size_t)G * n;
                    double* a3 = a2 + (size_t)G * n;
                    const int c0 = lr * C + crank, c1 = c0 + G * C, c2 = c1 + G * C, c3 = c2 + G * C;
                    const double x0 = *a0, x1 = *a1, x2 = *a2, x3 = *a3;
                    const double y0 = x0 - v[c0] * wr - w[c0] * vr, y1 = x1 - v[c1] * wr - w[c1] * vr;
                    const double y2 = x2 - v[c2] * wr - w[c2] * vr, y3 = x3 - v[c3] * wr - w[c3] * vr;
                    *a0 = y0;
                    *a1 = y1;
                    *a2 = y2;
                    *a3 = y3;
                    acc = fma(y0, vn[c0], acc);
                    acc = fma(y1, vn[c1], acc);
                    acc = fma(y2, vn[c2], acc);
                    acc = fma(y3, vn[c3], acc);
                }
                for (; lr < lre; lr += G) {
                    const int c = lr * C + crank;
                    double* ap = A + (size_t)lr * n + r;
                    const double y = *ap - v[c] * wr - w[c] * vr;
                    *ap = y;
                    acc = fma(y, vn[c], acc);
                }
            }
            if (G == 1) {
                if (jj < ncol) pp[s + 1 + jj] = acc;
            } else {  // one trip only (ncol <= cpg), uniform over the CTA
                red2[tid] = acc;
                __syncthreads();
                if (g == 0 && jj < ncol) {
                    double t = 0.0;
                    for (int q = 0; q < G; ++q) t += red2[q * cpg + jj];
                    pp[s + 1 + jj] = t;
                }
                break;
            }
        }
        if (!has_next) break;
        csync();  // every CTA's share of A v_s ready
        const double beta = bb[nxt];
        double part = 0.0;
        for (int r = s + 1 + tid; r < n; r += TRI_THREADS) {
            double sum = 0.0;
            for (int q = 0; q < C; ++q) sum += *cluster.map_shared_rank(pp + r, q);
            const double p = beta * sum;
            wb[(size_t)nxt * n + r] = p;  // p for now, w below
            part += p * vn[r];
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        double pv = 0.0;
        for (int q = 0; q < TRI_WARPS; ++q) pv += red[q];
        const double kk = 0.5 * beta * pv;
        for (int r = s + 1 + tid; r < n; r += TRI_THREADS) wb[(size_t)nxt * n + r] -= kk * vn[r];
        __syncthreads();
        if (s + 1 == jb.stop) {  // uniform over the cluster
            // hand-off: the trailing block with update s applied, to W (m x m, row-major)
            const int s0 = s + 1, m = n - s0;
            const double* wv = wb + (size_t)nxt * n;
            for (int lr = (s0 - crank + C - 1) / C + warp; lr < R; lr += TRI_WARPS) {
                const int c = lr * C + crank;
                if (c >= n) break;
                const double vc = vn[c], wc = wv[c];
                const double* arow = A + (size_t)lr * n;
                double* out = jb.W + (size_t)(c - s0) * m - s0;
                for (int r = s0 + lane; r < n; r += 32) out[r] = arow[r] - vc * wv[r] - wc * vn[r];
            }
            csync();  // no CTA leaves while another may still address its shared memory
            return;
        }
    }
    __syncthreads();
    // the last 2 x 2 block (or the 1 x 1 matrix)
    if (tid == 0) {
        if (n >= 2) {
            if ((n - 2) % C == crank) {
                jb.d[n - 2] = A[(size_t)((n - 2) / C) * n + n - 2];
                jb.e[n - 2] = A[(size_t)((n - 2) / C) * n + n - 1];
            }
            if ((n - 1) % C == crank) jb.d[n - 1] = A[(size_t)((n - 1) / C) * n + n - 1];
        } else if (crank == 0) {
            jb.d[0] = A[0];
        }
    }
    csync();  // no CTA leaves while another may still address its shared memory
}

// Householder reduction of one matrix too large for a cluster's shared memory (n > ~448), by a
// group of G CTAs: the whole GPU (one cooperative launch per matrix) or a thread-block cluster
// (one cluster per matrix, all such matrices of a batch in one launch).  The matrix is copied to
// W (global memory, row-major), row r belongs to CTA r % G, and every step takes two group
// barriers.  Step s, as in k_tridiag:
//   every CTA stages v_{s-1} and w_{s-1} = p_{s-1} - kk_{s-1} v_{s-1} (columns >= s) in shared
//   memory
//   (a) the CTA owning row s applies update s-1 to it (all its threads, a column each) and derives
//       reflector s (a block reduction for the norm): v_s into global scratch, beta_s, d[s], e[s]
//   group barrier; every CTA stages v_s
//   (b) every CTA, a warp per own row r > s: apply update s-1 to row r (columns > s) and form
//       p_r = beta_s W[r, s+1:] . v_s in the same pass; the CTA's share of p.v.  Each lane loads
//       TRIB_BATCH elements of the row before it stores any, so that many loads are in flight.
//   group barrier
//   every warp sums the G shares in the same order, so all hold the same kk_s = beta_s (p.v) / 2.
// Global scratch (job.work): v[2][n] | p[2][n] | share[G] | beta[2]; dynamic shared memory: 3 n
// doubles (tridiag_big_smem_bytes).  Row s of W ends holding reflector v_s in columns s+1..n-1
// (its first entry corrected after the norm), for the eigenvector back-transformation.
constexpr int TRIB_BATCH = 8;

size_t tridiag_big_smem_bytes(int n) { return sizeof(double) * 3 * (size_t)n; }

template <class Sync>
__device__ void tridiag_group(const TriJob& jb, int G, int gi, Sync sync) {
    const int n = jb.n;
    double* W = jb.W;
    double* vb = jb.work;              // v_s, two buffers
    double* pb = vb + 2 * (size_t)n;   // p_s, two buffers
    double* share = pb + 2 * (size_t)n;
    double* bb = share + G;            // beta_s, two buffers
    extern __shared__ double tsh[];
    double* sv = tsh;           // v_{s-1}
    double* sw = tsh + n;       // w_{s-1}
    double* svn = tsh + 2 * n;  // v_s
    constexpr int NW = TRIB_THREADS / 32;
    __shared__ double red[NW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto bsum = [&](double v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if (lane == 0) red[warp] = v;
        __syncthreads();
        double t = 0.0;
        for (int q = 0; q < NW; ++q) t += red[q];
        return t;
    };
    // own rows into W; update "-1" is the identity: v = p = 0, kk = 0
    for (int r = gi + warp * G; r < n; r += NW * G)
        for (int c = lane; c < n; c += 32) W[(size_t)r * n + c] = jb.A[(size_t)r * n + c];
    for (int c = gi * TRIB_THREADS + tid; c < n; c += G * TRIB_THREADS) {
        vb[n + c] = 0.0;
        pb[n + c] = 0.0;
    }
    double kk = 0.0;
    sync();
    for (int s = 0; s + 1 < n; ++s) {
        const int cur = (s + 1) & 1, nxt = s & 1;
        const double* v = vb + (size_t)cur * n;  // reflector s - 1
        const double* p = pb + (size_t)cur * n;
        double* vn = vb + (size_t)nxt * n;       // reflector s
        double* pn = pb + (size_t)nxt * n;
        const bool has_next = s + 2 < n;
        for (int c = s + tid; c < n; c += TRIB_THREADS) {
            const double vc = __ldcg(v + c);
            sv[c] = vc;
            sw[c] = __ldcg(p + c) - kk * vc;
        }
        __syncthreads();
        if (gi == s % G) {  // (a)
            double* row = W + (size_t)s * n;
            const double vs = sv[s], ws = sw[s];
            double nrm = 0.0;
            for (int c = s + tid; c < n; c += TRIB_THREADS) {
                const double vc = sv[c];
                const double y = row[c] - vs * sw[c] - ws * vc;
                row[c] = y;
                if (c > s) {
                    vn[c] = y;
                    nrm += y * y;
                }
            }
            nrm = bsum(nrm);  // its barriers also make row[s], row[s + 1] visible to thread 0
            if (tid == 0) {
                const double alpha = sqrt(nrm), x0 = row[s + 1];
                const double sg = x0 >= 0.0 ? 1.0 : -1.0;
                jb.d[s] = row[s];
                if (has_next) {
                    jb.e[s] = alpha == 0.0 ? 0.0 : -sg * alpha;
                    bb[nxt] = alpha == 0.0 ? 0.0 : 1.0 / (alpha * (alpha + fabs(x0)));
                    if (alpha != 0.0) {
                        vn[s + 1] = x0 + sg * alpha;
                        row[s + 1] = x0 + sg * alpha;  // row s now holds v_s exactly (read by no later step)
                    }
                } else {
                    jb.e[s] = row[s + 1];  // the last 2 x 2 block: e[n-2]
                }
            }
        }
        sync();  // v_s and beta_s ready
        for (int c = s + 1 + tid; c < n; c += TRIB_THREADS) svn[c] = __ldcg(vn + c);
        __syncthreads();
        // (b) own rows r > s, a warp per row
        const double beta = has_next ? __ldcg(bb + nxt) : 0.0;
        double part = 0.0;
        const int r0 = s + 1 + ((gi - (s + 1) % G) % G + G) % G;  // first own row > s
        for (int r = r0 + warp * G; r < n; r += NW * G) {
            double* row = W + (size_t)r * n;
            const double vr = sv[r], wr = sw[r];
            double acc = 0.0;
            for (int c0 = s + 1 + lane; c0 < n; c0 += 32 * TRIB_BATCH) {
                double x[TRIB_BATCH];
#pragma unroll
                for (int u = 0; u < TRIB_BATCH; ++u) {
                    const int c = c0 + 32 * u;
                    x[u] = c < n ? row[c] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < TRIB_BATCH; ++u) {
                    const int c = c0 + 32 * u;
                    if (c < n) {
                        const double y = x[u] - vr * sw[c] - wr * sv[c];
                        row[c] = y;
                        acc = fma(y, svn[c], acc);
                    }
                }
            }
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            const double pr = beta * acc;
            if (lane == 0 && has_next) pn[r] = pr;
            part += pr * svn[r];
        }
        if (!has_next) break;
        part = bsum(lane == 0 ? part : 0.0);
        if (tid == 0) share[gi] = part;
        sync();  // p_s and every share ready
        kk = 0.5 * beta * group_share_sum(share, G);
    }
    __syncthreads();
    if (n == 1 && gi == 0 && tid == 0) jb.d[0] = W[0];
    if (n >= 2 && gi == (n - 1) % G && tid == 0) jb.d[n - 1] = W[(size_t)(n - 1) * n + n - 1];
}

__global__ void __launch_bounds__(TRIB_THREADS) k_tridiag_big(TriJob jb) {
    cg::grid_group grid = cg::this_grid();
    tridiag_group(jb, (int)gridDim.x, (int)blockIdx.x, [&] { grid.sync(); });
}

// One cluster (gridDim.x CTAs) per matrix of jobs[blockIdx.y].
__global__ void __launch_bounds__(TRIB_THREADS) k_tridiag_cl(const TriJob* __restrict__ jobs) {
    cg::cluster_group cl = cg::this_cluster();
    tridiag_group(jobs[blockIdx.y], (int)cl.num_blocks(), (int)cl.block_rank(), [&] { cl.sync(); });
}

// Number of eigenvalues of T below x: the sign changes of the leading principal minors
// p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2} (p_{-1} = 1), the Sturm sequence of the
// tridiagonal.  Same count as the LDL^T pivots q_i = p_i / p_{i-1} < 0, without the division on the
// critical path (one FMA per step).  The pair (p_{i-1}, p_{i-2}) is rescaled by a power of two
// every 8 steps (exact), which keeps it far from overflow and underflow; a zero p_i is replaced by a
// tiny multiple of p_{i-1} (a zero pivot counts as non-negative, as in the division form).
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x) {
    int c = 0;
    double p2 = 1.0;
    double p1 = d[0] - x;
    if (p1 == 0.0) p1 = 0x1p-200;
    bool neg = p1 < 0.0;
    if (neg) ++c;
    for (int i = 1; i < n; ++i) {
        double p = fma(d[i] - x, p1, -e2[i - 1] * p2);
        if (p == 0.0) p = 0x1p-200 * p1;
        const bool ng = p < 0.0;
        c += ng != neg;
        neg = ng;
        p2 = p1;
        p1 = p;
        if ((i & 7) == 0) {
            const double m = fmax(fabs(p1), fabs(p2));
            const int ex = (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1023;
            if (ex > 400 || ex < -400) {
                const double sc = __longlong_as_double((long long)(1023 - ex) << 52);  // 2^-ex
                p1 *= sc;
                p2 *= sc;
            }
        }
    }
    return c;
}

// lanes = 1: a thread per eigenvalue, bisection; lanes = 32: a warp per eigenvalue, 32-way
// multisection (31 Sturm counts per round on the lanes, the interval narrowed to the gap where the
// count passes k: a factor 32 per round, to the bisection's stopping width), for launches with few
// eigenvalues, where the latency of one thread's ~50 dependent counts is the cost.
__global__ void k_bisect(const TriJob* __restrict__ jobs, const int* __restrict__ mask, int lanes) {
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
    if (lanes == 32) {
        const int k = (blockIdx.y * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
        if (k >= n) return;  // whole warps: blockDim is a multiple of 32
        double lo = bounds[0], hi = bounds[1];
        for (int round = 0; round < 16; ++round) {
            const double h = (hi - lo) * (1.0 / 32.0);
            if (!(h > 0.0) || hi - lo <= 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi))) break;
            const double x = lo + h * (lane + 1);
            const bool below = lane < 31 && sturm_count(d, e2, n, x) <= k;
            const unsigned ball = __ballot_sync(0xffffffffu, below);
            const int j = ball ? 31 - __clz(ball) : -1;
            const double nlo = j >= 0 ? lo + h * (j + 1) : lo;
            const double nhi = j + 2 <= 31 ? lo + h * (j + 2) : hi;
            lo = nlo;
            hi = nhi;
        }
        if (lane == 0) jb.eps[k] = 0.5 * (lo + hi);
        return;
    }
    const int k0 = blockIdx.y * blockDim.x;  // this block's share of the eigenvalue indices
    if (k0 >= n) return;
    for (int k = k0 + threadIdx.x; k < min(n, k0 + (int)blockDim.x); k += blockDim.x) {
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

namespace am1 {

// ---------------------------------------------------------------------------------------------
// Blocked Householder reduction for the largest matrices (the whole GPU per matrix): panels of
// TRP_B columns, each reduced by one cooperative launch (k_tridiag_panel, the DLATRD scheme) with
// the trailing matrix left untouched, then the trailing matrix updated once per panel,
// A <- A - V W^T - W V^T, by a rank-2 TRP_B product on the FP64 tensor cores (k_tridiag_syr2k*).
// Per column the panel kernel reads the trailing matrix once (A v) instead of reading and writing
// it (the unblocked k_tridiag_big), and the writes happen once per panel.
//
// Column c = k + j of the panel (V, W: the panel's reflectors and their w vectors so far, rows
// > c; V_c., W_c. row c of them):
//   x_i  = A_ic - sum_{l<j} (V_il W_cl + W_il V_cl)               i >= c   (column c, updated)
//   d_c  = x_c;  alpha = |x_{c+1:}|,  v = x_{c+1:} + sign(x_{c+1}) alpha e_1,
//   beta = 1 / (alpha (alpha + |x_{c+1}|)),  e_c = -sign(x_{c+1}) alpha
//   p    = beta (A v - V (W^T v) - W (V^T v))                      over rows and columns > c
//   w    = p - (beta/2)(p . v) v,  V_.j = v,  W_.j = w
// W^T v and V^T v come from W^T x and V^T x (summed with |x|^2 in the first grid barrier) and
// row c+1 of W and V.  Two grid barriers per column: row c+1's newest entries of V and W, which
// its owner writes after the second barrier, every CTA forms itself (v_{c+1} and p_{c+1} are
// known to all by then) for the next column's first phase.  Rows are cyclic over the CTAs (r % G).
// Scratch (job.work, 16-byte aligned): VW[n][2B] = [V | W] | WVt[2B][n] = [W | V]^T | x[n] |
// p[n] | share[G][2B + 2]; dynamic shared memory: v (n doubles) and W^T v, V^T v.  As in
// tridiag_group, row c of job.W ends holding reflector v_c in columns c+1..n-1.
// ---------------------------------------------------------------------------------------------

size_t tridiag_panel_smem_bytes(int n) { return sizeof(double) * ((size_t)n + 2 * TRP_B); }

__global__ void __launch_bounds__(TRIB_THREADS) k_tridiag_panel(TriJob jb, int k, int bw) {
    cg::grid_group grid = cg::this_grid();
    const int G = (int)gridDim.x, gi = (int)blockIdx.x;
    const int n = jb.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = TRIB_THREADS / 32;
    constexpr int B = TRP_B, SW = 2 * TRP_B + 2;
    double* A = jb.W;
    double* VW = jb.work;
    double* WVt = VW + (size_t)2 * B * n;
    double* xb = WVt + (size_t)2 * B * n;
    double* pb = xb + n;
    double* share = pb + n;
    extern __shared__ double psh[];
    double* sv = psh;      // v, rows c+1..n-1
    double* st = psh + n;  // [0, B): W^T v;  [B, 2B): V^T v
    __shared__ double xr[64];  // this CTA's x_i of the current column (its rows > c, at most 64 of them)
    __shared__ int xi_row[64];
    __shared__ double red[NW];
    // the panel's V and W on this CTA's own rows (row gi + q G in slot q), kept here as they are
    // formed: the per-column corrections read them from shared memory, not global
    __shared__ double svw[64][2 * TRP_B];
    __shared__ double rowc[2];  // V and W of row c in the previous column (formed locally)
    __shared__ double red4[4][NW];
    for (int j = 0; j < bw; ++j) {
        const int c = k + j;
        __syncthreads();  // own rows' V, W of the previous column, and rowc, are written
        // ---- phase 1: column c for own rows i >= c, and this CTA's shares of |x|^2, W^T x, V^T x
        const int first = c + ((gi - c % G) % G + G) % G;  // first own row >= c
        int nr = 0;
        for (int i = first; i < n; i += G) ++nr;  // own rows >= c (<= 64: n <= 8192 and G >= 128)
        const int q0 = (first - gi) / G;  // slot of the first own row >= c
        if (tid < nr) {
            const int i = first + tid * G;
            const double* Vi = svw[q0 + tid];
            const double* Vc = VW + (size_t)c * 2 * B;
            double x = __ldcg(A + (size_t)i * n + c);
            for (int l = 0; l < j; ++l) {
                // row c's entries of the previous column are not yet visible from its owner
                const double vc = l + 1 == j ? rowc[0] : __ldcg(Vc + l), wc = l + 1 == j ? rowc[1] : __ldcg(Vc + B + l);
                x -= Vi[l] * wc + Vi[B + l] * vc;
            }
            xr[tid] = x;
            xi_row[tid] = i;
            xb[i] = x;
            if (i == c) jb.d[c] = x;
        }
        __syncthreads();
        if (tid < 2 * j + 1) {  // share slot 0: |x_{>c}|^2; 1..j: W^T x; j+1..2j: V^T x
            double s = 0.0;
            for (int q = 0; q < nr; ++q) {
                const int i = xi_row[q];
                if (i <= c) continue;
                const double x = xr[q];
                if (tid == 0) s += x * x;
                else if (tid <= j) s += svw[q0 + q][B + (tid - 1)] * x;
                else s += svw[q0 + q][tid - 1 - j] * x;
            }
            share[(size_t)gi * SW + tid] = s;
        }
        grid.sync();
        // ---- the reflector (every CTA forms the same values: fixed-order sums of the shares)
        const bool has_next = c + 2 < n;
        const double x1 = __ldcg(xb + c + 1);
        if (!has_next) {  // the last 2 x 2 block: e[n-2], and d[n-1] with this panel's updates
            if (gi == (n - 1) % G && tid == 0) {
                jb.e[c] = x1;
                double dn = __ldcg(A + (size_t)(n - 1) * n + n - 1);
                const double* Vn = VW + (size_t)(n - 1) * 2 * B;
                for (int l = 0; l < j; ++l) dn -= 2.0 * __ldcg(Vn + l) * __ldcg(Vn + B + l);
                jb.d[n - 1] = dn;
            }
            break;
        }
        double nrm2 = 0.0;
        for (int q = lane; q < G; q += 32) nrm2 += __ldcg(share + (size_t)q * SW);
        for (int o = 16; o > 0; o >>= 1) nrm2 += __shfl_xor_sync(0xffffffffu, nrm2, o);
        const double alpha = sqrt(nrm2);
        const double sg = x1 >= 0.0 ? 1.0 : -1.0;
        const double beta = alpha == 0.0 ? 0.0 : 1.0 / (alpha * (alpha + fabs(x1)));
        const double* V1 = VW + (size_t)(c + 1) * 2 * B;
        // W^T v and V^T v: slot s < 2j summed over the CTAs by one warp, lane-strided in a fixed
        // order (as group_share_sum), plus the e_{c+1} part of v = x + sg alpha e_{c+1}
        for (int sl = warp; sl < 2 * j; sl += NW) {
            double t = 0.0;
            for (int q = lane; q < G; q += 32) t += __ldcg(share + (size_t)q * SW + 1 + sl);
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) {
                const int l = sl < j ? sl : sl - j;
                t += sg * alpha * (sl < j ? __ldcg(V1 + B + l) : __ldcg(V1 + l));
                st[sl < j ? l : B + l] = t;
            }
        }
        for (int i = c + 1 + tid; i < n; i += TRIB_THREADS) sv[i] = __ldcg(xb + i);
        __syncthreads();
        if (tid == 0) sv[c + 1] = x1 + sg * alpha;
        __syncthreads();
        // ---- phase 2a: p_i for own rows i > c, this CTA's share of p . v.  Rows go in groups of
        // four; every thread takes a stride of the columns for all four (many loads in flight),
        // and the partial sums are reduced over the CTA in a fixed order.
        double part = 0.0;
        for (int g0 = first > c ? 0 : 1; g0 < nr; g0 += 4) {
            const int gr = min(4, nr - g0);
            const double* Ar[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) Ar[u] = A + (size_t)(first + (g0 + (u < gr ? u : 0)) * G) * n;
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
            for (int m = c + 1 + tid; m < n; m += TRIB_THREADS) {
                const double vm = sv[m];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(__ldcg(Ar[u] + m), vm, acc[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                for (int o = 16; o > 0; o >>= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
            if (lane == 0)
#pragma unroll
                for (int u = 0; u < 4; ++u) red4[u][warp] = acc[u];
            __syncthreads();
            if (tid < gr) {
                const int q = g0 + tid, i = first + q * G;
                double t = 0.0;
                for (int w = 0; w < NW; ++w) t += red4[tid][w];
                const double* Vi = svw[q0 + q];
                for (int l = 0; l < j; ++l) t -= Vi[l] * st[l] + Vi[B + l] * st[B + l];
                const double pi = beta * t;
                pb[i] = pi;
                part += pi * sv[i];
            }
            __syncthreads();
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int q = 0; q < NW; ++q) t += red[q];
            share[(size_t)gi * SW + SW - 1] = t;
        }
        grid.sync();
        // ---- phase 2b: w = p - kk v for own rows i > c; column j of V and W in both layouts
        double pv = 0.0;
        for (int q = lane; q < G; q += 32) pv += __ldcg(share + (size_t)q * SW + SW - 1);
        for (int o = 16; o > 0; o >>= 1) pv += __shfl_xor_sync(0xffffffffu, pv, o);
        const double kk = 0.5 * beta * pv;
        if (tid < nr) {
            const int i = first + tid * G;
            if (i > c) {
                const double v = sv[i], w = __ldcg(pb + i) - kk * v;
                svw[q0 + tid][j] = v;
                svw[q0 + tid][B + j] = w;
                VW[(size_t)i * 2 * B + j] = v;
                VW[(size_t)i * 2 * B + B + j] = w;
                WVt[(size_t)j * n + i] = w;
                WVt[(size_t)(B + j) * n + i] = v;
                A[(size_t)c * n + i] = v;  // reflector c into row c (columns > c), which nothing reads again
            }
        }
        if (gi == c % G && tid == 0) jb.e[c] = alpha == 0.0 ? 0.0 : -sg * alpha;
        if (tid == 0) {  // row c+1's entries of this column, for the next column's phase 1
            rowc[0] = sv[c + 1];
            rowc[1] = __ldcg(pb + c + 1) - kk * sv[c + 1];
        }
    }
}

// A[t0 + r][t0 + q] -= (V W^T + W V^T)[t0 + r][t0 + q] over the upper-triangle 64 x 64 tiles of the
// trailing block (t0 = k + TRP_B), mirrored: C = [V | W][rows] . [W | V]^T[:, cols], K = 2 TRP_B.
template <bool PAIRS>
__device__ __forceinline__ void syr2k_body(TriJob jb, int t0) {
    extern __shared__ __align__(16) double dsm[];
    const int n = jb.n, T = n - t0;
    const int nt = (T + DG_TILE - 1) / DG_TILE;
    int rem = blockIdx.x, tm = 0;
    while (rem >= nt - tm) {
        rem -= nt - tm;
        ++tm;
    }
    const int tn = tm + rem;
    const int m0 = tm * DG_TILE, n0 = tn * DG_TILE;
    const double* VW = jb.work;
    const double* WVt = VW + (size_t)2 * TRP_B * n;
    const bool compute = dg_quarter_on(m0, n0, T, T, tm == tn);
    double acc[2][4][4];
    dg_mainloop<PAIRS>(dsm, VW + (size_t)t0 * 2 * TRP_B, 2 * TRP_B, WVt + t0, n, T, T, 2 * TRP_B, m0, n0, acc, compute);
    double* A = jb.W + (size_t)t0 * n + t0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = m0 + dg_row(i, e), c = n0 + dg_col(j, e);
                if (compute && r <= c && c < T) {
                    const double y = A[(size_t)r * n + c] - acc[i][j][e];
                    A[(size_t)r * n + c] = y;
                    if (r < c) A[(size_t)c * n + r] = y;
                }
            }
}

__global__ void __launch_bounds__(DG_THREADS, 4) k_tridiag_syr2k16(TriJob jb, int t0) { syr2k_body<true>(jb, t0); }
__global__ void __launch_bounds__(DG_THREADS, 4) k_tridiag_syr2k8(TriJob jb, int t0) { syr2k_body<false>(jb, t0); }

}  // namespace am1
