// FP64 tensor-core GEMM main loop for 64x64 output tiles: C_tile = A[m0:m0+64, :K] . B[:K, n0:n0+64]
// with mma.sync.m8n8k4.f64 (4 warps, each a 32x32 sub-tile of 4x4 MMA blocks) and a
// STAGES-deep cp.async pipeline feeding shared memory, so global (L2) latency is overlapped
// with the MMAs.  Row-major operands with arbitrary leading dimensions; out-of-range elements
// are zero-filled by the copy itself (src-size 0).
#pragma once

#include <cuda_runtime.h>

namespace am1 {

constexpr int DG_TILE = 64;
constexpr int DG_BK = 16;
constexpr int DG_AS = DG_BK + 4;    // A tile row stride: conflict-free 8-byte fragment loads
constexpr int DG_BS = DG_TILE + 4;  // B tile row stride
constexpr int DG_STAGE = DG_TILE * DG_AS + DG_BK * DG_BS;  // doubles per pipeline stage
constexpr int DG_STAGES = 3;
constexpr int DG_THREADS = 128;
constexpr size_t DG_SMEM = sizeof(double) * DG_STAGE * DG_STAGES;

__device__ __forceinline__ void dg_mma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// 8-byte asynchronous copy; an invalid element reads nothing (src-size 0) from the operand's
// base address and is zero-filled.
__device__ __forceinline__ void dg_cp8(double* smem_dst, const double* gsrc, const double* base, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(valid ? gsrc : base), "r"(bytes));
}
__device__ __forceinline__ void dg_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void dg_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Issue the copies of k-tile kt into pipeline stage `st`.
__device__ __forceinline__ void dg_load(double* smem, int st, const double* __restrict__ A, int lda, const double* __restrict__ B,
                                        int ldb, int M, int N, int K, int m0, int n0, int kt) {
    double* As = smem + st * DG_STAGE;
    double* Bs = As + DG_TILE * DG_AS;
    const int k0 = kt * DG_BK;
    const int tid = threadIdx.x;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int idx = tid + l * DG_THREADS;
        const int ar = idx >> 4, ak = idx & 15;
        const int gi = m0 + ar, gk = k0 + ak;
        dg_cp8(&As[ar * DG_AS + ak], A + (long long)gi * lda + gk, A, gi < M && gk < K);
        const int bk = idx >> 6, bc = idx & 63;
        const int gbk = k0 + bk, gj = n0 + bc;
        dg_cp8(&Bs[bk * DG_BS + bc], B + (long long)gbk * ldb + gj, B, gbk < K && gj < N);
    }
}

// acc[i][j][e]: row wr + 8i + (lane>>2), column wc + 8j + 2(lane&3) + e of the 64x64 tile.
__device__ __forceinline__ void dg_mainloop(double* smem, const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
                                            int M, int N, int K, int m0, int n0, double acc[4][4][2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int KT = (K + DG_BK - 1) / DG_BK;
#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; ++s) {
        if (s < KT) dg_load(smem, s, A, lda, B, ldb, M, N, K, m0, n0, s);
        dg_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        dg_wait<DG_STAGES - 2>();
        __syncthreads();
        const int nk = kt + DG_STAGES - 1;
        if (nk < KT) dg_load(smem, nk % DG_STAGES, A, lda, B, ldb, M, N, K, m0, n0, nk);
        dg_commit();
        const double* As = smem + (kt % DG_STAGES) * DG_STAGE;
        const double* Bs = As + DG_TILE * DG_AS;
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[(wr + i * 8 + g) * DG_AS + kk + tq];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(kk + tq) * DG_BS + wc + j * 8 + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dg_mma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    dg_wait<0>();
    __syncthreads();
}

}  // namespace am1
