// SP2 step of the mixed-precision SCF's early iterations: the same step as k_sp2_step16/8
// (X <- X^2 or 2X - X^2 over the upper-triangle 64x64 tiles, mirrored, with the tile's share of
// tr X and ||X||_F^2), with X held in FP32 and the product X.X on the TF32 tensor cores
// (mma.sync m16n8k8 tf32, FP32 accumulation).  Every stored iterate is rounded to the nearest
// TF32 value (tf32_round), so the tensor cores read exact operands and the rounding of each step
// is unbiased (operands truncated by the hardware would shrink every product, and with it the
// trace).  Partial sums are accumulated in FP64.  The FP64 iterations that follow remove the
// rounding of these steps from the converged result.
//
// X rows are ldf floats apart (n rounded up to a multiple of 4, pad columns zero), so every
// row starts on 16 bytes and the tiles are copied in 16-byte chunks: a chunk is valid when its
// row is inside the matrix and it starts inside the padded row (pad columns read as the zeros
// they hold).
//
// Tile layout as in dmma_gemm.cuh (4 warps, each a 32x32 quarter of 2x4 MMA blocks); the
// m16n8k8 tf32 fragments have the same (row, column) map as the f64 ones:
//   A (16x8, row): a0 (g, t)  a1 (g+8, t)  a2 (g, t+4)  a3 (g+8, t+4)
//   B (8x8, col):  b0 (t, g)  b1 (t+4, g)
//   C (16x8):      c0 (g, 2t)  c1 (g, 2t+1)  c2 (g+8, 2t)  c3 (g+8, 2t+1)
// with g = lane / 4, t = lane % 4.  Shared-memory strides of 36 (A) and 72 (B) floats make the
// fragment loads conflict-free and keep every 16-byte chunk aligned.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {

constexpr int TF_TILE = 64;
constexpr int TF_BK = 32;
constexpr int TF_AS = TF_BK + 4;
constexpr int TF_BS = TF_TILE + 8;
constexpr int TF_STAGE = TF_TILE * TF_AS + TF_BK * TF_BS;  // floats per pipeline stage
constexpr int TF_STAGES = 3;
constexpr int TF_THREADS = 128;

size_t tf32_smem_bytes() { return sizeof(float) * TF_STAGE * TF_STAGES; }

__device__ __forceinline__ void tf_mma(float c[4], const float a[4], const float b[2]) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(__float_as_uint(a[0])), "r"(__float_as_uint(a[1])), "r"(__float_as_uint(a[2])), "r"(__float_as_uint(a[3])),
                   "r"(__float_as_uint(b[0])), "r"(__float_as_uint(b[1])));
}

__device__ __forceinline__ void tf_cp16(float* smem_dst, const float* gsrc, const float* base, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    const int bytes = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(valid ? gsrc : base), "r"(bytes));
}

// k-tile kt of A = X[m0:m0+64, :] and B = X[:, n0:n0+64] into stage st
__device__ __forceinline__ void tf_load(float* smem, int st, const float* __restrict__ X, int ldf, int n, int m0, int n0, int kt) {
    float* As = smem + st * TF_STAGE;
    float* Bs = As + TF_TILE * TF_AS;
    const int k0 = kt * TF_BK;
    const int tid = threadIdx.x;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const int idx = tid + l * TF_THREADS;  // 0 .. 511
        const int ar = idx >> 3, ak = (idx & 7) * 4;
        const int gi = m0 + ar, gk = k0 + ak;
        tf_cp16(&As[ar * TF_AS + ak], X + (long long)gi * ldf + gk, X, gi < n && gk < ldf);
        const int bk = idx >> 4, bc = (idx & 15) * 4;
        const int gbk = k0 + bk, gj = n0 + bc;
        tf_cp16(&Bs[bk * TF_BS + bc], X + (long long)gbk * ldf + gj, X, gbk < n && gj < ldf);
    }
}

__global__ void __launch_bounds__(TF_THREADS, 4) k_sp2_step_tf32(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                                 int ntiles, const Sp2State* __restrict__ sst) {
    extern __shared__ __align__(16) float fsm[];
    __shared__ double red[2][4];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || !sp->lowp || jp->lowp_tc) return;  // FP64 runs: k_sp2_step_tma / 16 / 8; tcgen05: k_sp2_step_tc / _tc1
    const int n = jp->n, ldf = jp->ldf;
    const int cur = sp->cur;
    const float* X = cur ? jp->Xf1 : jp->Xf0;
    const int m0 = tl.tm * TF_TILE, n0 = tl.tn * TF_TILE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
    const bool compute = dg_quarter_on(m0, n0, n, n, tl.tm == tl.tn);
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;
    const int KT = (n + TF_BK - 1) / TF_BK;
#pragma unroll
    for (int s = 0; s < TF_STAGES - 1; ++s) {
        if (s < KT) tf_load(fsm, s, X, ldf, n, m0, n0, s);
        dg_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        dg_wait<TF_STAGES - 2>();
        __syncthreads();
        const int nk = kt + TF_STAGES - 1;
        if (nk < KT) tf_load(fsm, nk % TF_STAGES, X, ldf, n, m0, n0, nk);
        dg_commit();
        const float* As = fsm + (kt % TF_STAGES) * TF_STAGE;
        const float* Bs = As + TF_TILE * TF_AS;
        if (!compute) continue;
#pragma unroll
        for (int kk = 0; kk < TF_BK; kk += 8) {
            if (kk > 0 && kt * TF_BK + kk >= n) break;
            float a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const float* ar = As + (wr + i * 16 + g) * TF_AS + kk + tq;
                a[i][0] = ar[0];
                a[i][1] = ar[8 * TF_AS];
                a[i][2] = ar[4];
                a[i][3] = ar[8 * TF_AS + 4];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float* br = Bs + (kk + tq) * TF_BS + wc + j * 8 + g;
                b[j][0] = br[0];
                b[j][1] = br[4 * TF_BS];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) tf_mma(acc[i][j], a[i], b[j]);
        }
    }
    dg_wait<0>();
    __syncthreads();
    // epilogue: Y = X^2 or 2X - X^2 for r <= c, mirrored; FP64 partial sums of the stored values
    float* Y = cur ? jp->Xf0 : jp->Xf1;
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
                    const float x2 = acc[i][j][e];
                    const float y = tf32_round(square ? x2 : 2.0f * X[(long long)r * ldf + c] - x2);
                    Y[(long long)r * ldf + c] = y;
                    if (r < c) {
                        Y[(long long)c * ldf + r] = y;
                        fr += 2.0 * (double)y * y;
                    } else {
                        fr += (double)y * y;
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

}  // namespace am1
