// Dense FP64 linear algebra of the SCF step, batched over ragged molecules:
//   * k_gemm     : C = alpha op(A) B for every (molecule, channel) job, 64x64 output tiles
//                  drawn from one flat tile list; used for F.P (commutator, src/scf.rs:531-544),
//                  C^T.F (the eigensolver's warm start) and C_occ^T C_occ (density,
//                  src/scf.rs:503-524).
//   * k_jacobi   : symmetric eigensolver (replaces faer's self_adjoint_eigen behind
//                  src/linalg.rs:276-331).  One-sided (Hestenes) Jacobi on G = (F + sigma I) C0:
//                  pairs of columns of G are rotated until mutually orthogonal, the same
//                  rotations applied to V = C0.  Then (F + sigma I) V has orthogonal columns, so V
//                  holds eigenvectors of (F + sigma I)^2, which are those of F because sigma (a
//                  Gershgorin bound) makes F + sigma I positive definite; lambda_k = v_k.g_k - sigma.
//                  C0 is the previous SCF iteration's eigenvectors, so late iterations start
//                  nearly diagonal and need one or two sweeps.  Columns live in shared memory,
//                  spread over a thread-block cluster of 1..16 CTAs; the round-robin ordering
//                  moves one column per neighbour per step through distributed shared memory.
//   * k_eig_sort : ascending eigenvalues (the reference sorts, src/linalg.rs:321-329) and the
//                  matching rows of C^T.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace am1 {

// ---------------------------------------------------------------------------------------
// Batched GEMM
// ---------------------------------------------------------------------------------------
constexpr int GB_M = 64, GB_N = 64, GB_K = 16;

template <bool TA>
__device__ __forceinline__ void gemm_tile(const GemmJob* __restrict__ jobs, const GemmTile* __restrict__ tiles, int ntiles,
                                          const MolState* __restrict__ st, int force, const int* __restrict__ mask) {
    __shared__ double As[GB_K][GB_M + 1];
    __shared__ double Bs[GB_K][GB_N + 1];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const GemmJob jb = jobs[tl.job];
    if (!force && !st[jb.mol].active) return;
    if (mask && !mask[jb.mol]) return;
    const int m0 = tl.tm * GB_M, n0 = tl.tn * GB_N;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
    for (int k0 = 0; k0 < jb.K; k0 += GB_K) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int idx = tid + l * 256;
            if (TA) {  // A is K x M: element (k, i)
                const int i = idx & 63, k = idx >> 6;
                const int gi = m0 + i, gk = k0 + k;
                As[k][i] = (gi < jb.M && gk < jb.K) ? jb.A[(long long)gk * jb.lda + gi] : 0.0;
            } else {  // A is M x K: element (i, k)
                const int k = idx & 15, i = idx >> 4;
                const int gi = m0 + i, gk = k0 + k;
                As[k][i] = (gi < jb.M && gk < jb.K) ? jb.A[(long long)gi * jb.lda + gk] : 0.0;
            }
            const int j = idx & 63, kb = idx >> 6;
            const int gj = n0 + j, gkb = k0 + kb;
            Bs[kb][j] = (gj < jb.N && gkb < jb.K) ? jb.B[(long long)gkb * jb.ldb + gj] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < GB_K; ++k) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[k][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = Bs[k][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int gi = m0 + ty + 16 * r;
        if (gi >= jb.M) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int gj = n0 + tx + 16 * c;
            if (gj < jb.N) jb.C[(long long)gi * jb.ldc + gj] = jb.alpha * acc[r][c];
        }
    }
}

__global__ void __launch_bounds__(256) k_gemm_nn(const GemmJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                 int ntiles, const MolState* __restrict__ st, int force, const int* __restrict__ mask) {
    gemm_tile<false>(jobs, tiles, ntiles, st, force, mask);
}

__global__ void __launch_bounds__(256) k_gemm_tn(const GemmJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                 int ntiles, const MolState* __restrict__ st, int force, const int* __restrict__ mask) {
    gemm_tile<true>(jobs, tiles, ntiles, st, force, mask);
}

// ---------------------------------------------------------------------------------------
// One-sided Jacobi in a cluster
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Rotate the pair of columns (buffers bp, bq) until orthogonal; returns 1 if rotated.
__device__ __forceinline__ int rotate_pair(double* __restrict__ gp, double* __restrict__ gq, int n, double tol, int lane) {
    double* vp = gp + n;
    double* vq = gq + n;
    double al = 0.0, be = 0.0, ga = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double x = gp[i], y = gq[i];
        al = fma(x, x, al);
        be = fma(y, y, be);
        ga = fma(x, y, ga);
    }
    al = warp_sum(al);
    be = warp_sum(be);
    ga = warp_sum(ga);
    if (!(fabs(ga) > tol * sqrt(al * be)) || al == 0.0 || be == 0.0) return 0;
    const double zeta = (be - al) / (2.0 * ga);
    const double tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
    const double c = 1.0 / sqrt(1.0 + tt * tt), s = c * tt;
    for (int i = lane; i < n; i += 32) {
        const double x = gp[i], y = gq[i];
        gp[i] = c * x - s * y;
        gq[i] = s * x + c * y;
        const double u = vp[i], w = vq[i];
        vp[i] = c * u - s * w;
        vq[i] = s * u + c * w;
    }
    return 1;
}

constexpr int JAC_THREADS = 256;
constexpr int JAC_MAX_SWEEPS = 60;

// Shared memory: nbuf = 2q + 2 buffers of 2n doubles ([g | v]), then int metadata.
__global__ void __launch_bounds__(JAC_THREADS) k_jacobi(const EigJob* __restrict__ jobs, const MolState* __restrict__ st,
                                                        int* __restrict__ mol_status, int force, const int* __restrict__ mask) {
    extern __shared__ double smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const EigJob jb = jobs[blockIdx.x / C];
    if (!force && !st[jb.mol].active) return;  // uniform over the cluster
    if (mask && !mask[jb.mol]) return;
    const int n = jb.n, npad = jb.npad, m = npad / 2, q = m / C;
    const int nbuf = 2 * q + 2;
    const int LAND_TOP = 2 * q, LAND_BOT = 2 * q + 1;
    double* buf = smem;
    int* colid = (int*)(smem + (long long)nbuf * 2 * n);
    int* Tring = colid + nbuf;  // top ring (buffer ids)
    int* Bring = Tring + q;     // bottom ring
    int* ctl = Bring + q;       // [0] ht, [1] hb, [2] rot counter, [3] bad input, [4] total
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = JAC_THREADS / 32;
    const double tol = fmax(1.0e-14, 2.0 * n * 2.220446049250313e-16);

    // shift sigma from the Gershgorin lower bound of F (rowmin) so F + sigma I > 0
    double mn = 1e300;
    for (int i = tid; i < n; i += JAC_THREADS) mn = fmin(mn, jb.rowmin[i]);
    __shared__ double red[JAC_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if (lane == 0) red[warp] = mn;
    __syncthreads();
    if (tid == 0) {
        double v = red[0];
        for (int w = 1; w < nwarps; ++w) v = fmin(v, red[w]);
        red[0] = v;
    }
    __syncthreads();
    const double sigma = fmax(0.0, -red[0]) + 1.0;

    // initial assignment: local top k -> global column crank*q + k, bottom k -> m + crank*q + k
    if (tid == 0) {
        ctl[0] = 0;
        ctl[1] = 0;
        ctl[2] = 0;
        ctl[3] = 0;
        ctl[4] = 0;
    }
    for (int b = tid; b < 2 * q; b += JAC_THREADS) {
        colid[b] = b < q ? crank * q + b : m + crank * q + (b - q);
        if (b < q) Tring[b] = b;
        else Bring[b - q] = b;
    }
    __syncthreads();
    for (long long e = tid; e < (long long)2 * q * n; e += JAC_THREADS) {
        const int b = (int)(e / n), i = (int)(e % n);
        const int col = colid[b];
        double g = 0.0, v = 0.0;
        if (col < n) {
            v = jb.Ct[(long long)col * n + i];
            g = jb.Gt[(long long)col * n + i] + sigma * v;
            if (!isfinite(g)) ctl[3] = 1;
        }
        buf[(long long)b * 2 * n + i] = g;
        buf[(long long)b * 2 * n + n + i] = v;
    }
    __syncthreads();
    if (C > 1) cluster.sync();
    int bad = ctl[3];
    if (C > 1) {
        // agree on bad input across the cluster
        if (tid == 0 && bad) atomicOr(cluster.map_shared_rank(&ctl[3], 0), 1);
        cluster.sync();
        bad = *cluster.map_shared_rank(&ctl[3], 0);
        cluster.sync();
    }
    if (bad) {
        if (crank == 0 && tid == 0) atomicExch(&mol_status[jb.mol], 5);  // AM1GPU_LINALG
        return;
    }
    // ring helpers
    const int L1 = 2 * q - 1;                      // single-CTA ring length
    const int qt = (crank == 0) ? q - 1 : q;       // top ring size when C > 1
    auto top_buf = [&](int k, int s) -> int {
        if (C == 1) {
            if (k == 0) return Tring[0];
            const int r = k - 1;                    // ring position
            const int src = ((r - s) % L1 + L1) % L1;
            // ring order: top[1..q-1] then bot[q-1..0]
            return src < q - 1 ? Tring[1 + src] : Bring[q - 1 - (src - (q - 1))];
        }
        if (crank == 0 && k == 0) return Tring[q - 1];  // fixed slot kept at the end of Tring
        const int kk = (crank == 0) ? k - 1 : k;
        return Tring[(ctl[0] + kk) % qt];
    };
    auto bot_buf = [&](int k, int s) -> int {
        if (C == 1) {
            const int r = L1 - 1 - k;
            const int src = ((r - s) % L1 + L1) % L1;
            return src < q - 1 ? Tring[1 + src] : Bring[q - 1 - (src - (q - 1))];
        }
        return Bring[(ctl[1] + k) % q];
    };
    if (C > 1 && crank == 0) {
        // CTA 0 keeps top[0] fixed: store its buffer at Tring[q-1] and use Tring[0..q-2] as the ring
        if (tid == 0) {
            const int fixed = Tring[0];
            for (int k = 0; k < q - 1; ++k) Tring[k] = Tring[k + 1];
            Tring[q - 1] = fixed;
        }
        __syncthreads();
    }

    int sweeps = 0;
    bool done = false;
    while (!done && sweeps < JAC_MAX_SWEEPS) {
        int local_rot = 0;
        for (int s = 0; s < npad - 1; ++s) {
            for (int k = warp; k < q; k += nwarps) {
                const int bp = top_buf(k, s), bq = bot_buf(k, s);
                local_rot += rotate_pair(buf + (long long)bp * 2 * n, buf + (long long)bq * 2 * n, n, tol, lane);
            }
            if (C == 1) {
                __syncthreads();
                continue;
            }
            __syncthreads();
            cluster.sync();
            // send top[q-1] right and bot[0] left (full [g|v] buffers and their column ids)
            const int LT = top_buf(q - 1, s), LB = bot_buf(0, s);
            if (crank < C - 1) {
                double* dst = cluster.map_shared_rank(buf + (long long)LAND_TOP * 2 * n, crank + 1);
                const double* src = buf + (long long)LT * 2 * n;
                for (int i = tid; i < 2 * n; i += JAC_THREADS) dst[i] = src[i];
                if (tid == 0) *cluster.map_shared_rank(&colid[LAND_TOP], crank + 1) = colid[LT];
            }
            if (crank > 0) {
                double* dst = cluster.map_shared_rank(buf + (long long)LAND_BOT * 2 * n, crank - 1);
                const double* src = buf + (long long)LB * 2 * n;
                for (int i = tid; i < 2 * n; i += JAC_THREADS) dst[i] = src[i];
                if (tid == 0) *cluster.map_shared_rank(&colid[LAND_BOT], crank - 1) = colid[LB];
            }
            cluster.sync();
            // re-map: tops shift right, bottoms shift left
            int copy_top_to = -1, copy_bot_to = -1;
            const int ht = ctl[0], hb = ctl[1];
            const int nht = (ht - 1 + qt) % qt, nhb = (hb + 1) % q;
            if (crank == 0) {
                // entering top[1] is the old bot[0] (local); LT's buffer receives the landed bottom
                copy_bot_to = LT;
                __syncthreads();
                if (tid == 0) {
                    Tring[nht] = LB;
                    Bring[hb] = LT;
                }
            } else if (crank == C - 1) {
                // entering top[0] is the landed top, into LB's (sent) buffer; old top[q-1] wraps to bot[q-1]
                copy_top_to = LB;
                __syncthreads();
                if (tid == 0) {
                    Tring[nht] = LB;
                    Bring[hb] = LT;
                }
            } else {
                copy_top_to = LT;
                copy_bot_to = LB;
            }
            if (copy_top_to >= 0) {
                double* d = buf + (long long)copy_top_to * 2 * n;
                const double* sgl = buf + (long long)LAND_TOP * 2 * n;
                for (int i = tid; i < 2 * n; i += JAC_THREADS) d[i] = sgl[i];
                if (tid == 0) colid[copy_top_to] = colid[LAND_TOP];
            }
            if (copy_bot_to >= 0) {
                double* d = buf + (long long)copy_bot_to * 2 * n;
                const double* sgl = buf + (long long)LAND_BOT * 2 * n;
                for (int i = tid; i < 2 * n; i += JAC_THREADS) d[i] = sgl[i];
                if (tid == 0) colid[copy_bot_to] = colid[LAND_BOT];
            }
            __syncthreads();
            if (tid == 0) {
                ctl[0] = nht;
                ctl[1] = nhb;
            }
            __syncthreads();
        }
        // sweep total over the cluster
        if (lane == 0 && local_rot) atomicAdd(&ctl[2], local_rot);
        __syncthreads();
        int total;
        if (C > 1) {
            if (tid == 0 && ctl[2]) atomicAdd(cluster.map_shared_rank(&ctl[4], 0), ctl[2]);
            cluster.sync();
            total = *cluster.map_shared_rank(&ctl[4], 0);
            cluster.sync();
            if (tid == 0) {
                ctl[2] = 0;
                if (crank == 0) ctl[4] = 0;
            }
        } else {
            total = ctl[2];
            __syncthreads();
            if (tid == 0) ctl[2] = 0;
        }
        __syncthreads();
        ++sweeps;
        done = total == 0;
    }
    if (!done && crank == 0 && tid == 0) atomicExch(&mol_status[jb.mol], 5);  // AM1GPU_LINALG
    // write out: eigenvalue lambda = v.g - sigma (Rayleigh quotient), vector, column id
    for (int b = warp; b < 2 * q; b += nwarps) {
        const double* g = buf + (long long)b * 2 * n;
        const double* v = g + n;
        double d = 0.0;
        for (int i = lane; i < n; i += 32) d = fma(v[i], g[i], d);
        d = warp_sum(d);
        const int slot = crank * 2 * q + b;
        const int col = colid[b];
        if (lane == 0) {
            jb.lam[slot] = col < n ? d - sigma : 1e300;
            jb.colid_out[slot] = col;
        }
        double* out = jb.Vs + (long long)slot * n;
        for (int i = lane; i < n; i += 32) out[i] = v[i];
    }
    if (jb.sweeps_out && crank == 0 && tid == 0) *jb.sweeps_out = sweeps;
}

// ---------------------------------------------------------------------------------------
// Sort eigenpairs ascending (bitonic sort of up to 1024 keys per job) and gather rows.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_eig_sort(const EigJob* __restrict__ jobs, const MolState* __restrict__ st, int force,
                                                  const int* __restrict__ mask) {
    const EigJob jb = jobs[blockIdx.x];
    if (!force && !st[jb.mol].active) return;
    if (mask && !mask[jb.mol]) return;
    __shared__ double key[1024];
    __shared__ int val[1024];
    int P2 = 1;
    while (P2 < jb.npad) P2 <<= 1;
    for (int i = threadIdx.x; i < P2; i += blockDim.x) {
        if (i < jb.npad) {
            key[i] = jb.lam[i];
            val[i] = i;
        } else {
            key[i] = 1e308;
            val[i] = -1;
        }
    }
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P2; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const double a = key[i], b = key[ixj];
                    const int va = val[i], vb = val[ixj];
                    // ties broken by slot index so the order is deterministic
                    const bool gt = a > b || (a == b && va > vb);
                    if (gt == up) {
                        key[i] = b;
                        key[ixj] = a;
                        val[i] = vb;
                        val[ixj] = va;
                    }
                }
            }
            __syncthreads();
        }
    const int n = jb.n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) jb.eps[i] = key[i];
    // gather the sorted rows into C^T
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < n; r += nw) {
        const double* src = jb.Vs + (long long)val[r] * n;
        double* dst = jb.Ct_out + (long long)r * n;
        for (int i = lane; i < n; i += 32) dst[i] = src[i];
    }
}

size_t jacobi_smem_bytes(int n, int npad, int C) {
    const int q = npad / 2 / C;
    const int nbuf = 2 * q + 2;
    return (size_t)nbuf * 2 * n * sizeof(double) + (size_t)(nbuf + 2 * q + 8) * sizeof(int);
}

}  // namespace am1
