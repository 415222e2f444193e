// FP64 tensor-core GEMM main loop for 64x64 output tiles: C_tile = A[m0:m0+64, :K] . B[:K, n0:n0+64]
// with mma.sync.m16n8k8.f64 (4 warps, each a 32x32 sub-tile of 2x4 MMA blocks) and a
// STAGES-deep cp.async pipeline feeding shared memory, so global (L2) latency is overlapped
// with the MMAs.  Row-major operands with arbitrary leading dimensions; out-of-range elements
// are zero-filled by the copy itself (src-size 0).  Operands with even shapes and 16-byte
// aligned rows are copied in 16-byte pairs (half the copy instructions), others element-wise.
//
// Fragment layout of m16n8k8 f64 (g = lane/4, t = lane%4):
//   A (16x8, row): a0 (g, t)  a1 (g+8, t)  a2 (g, t+4)  a3 (g+8, t+4)
//   B (8x8, col):  b0 (t, g)  b1 (t+4, g)
//   C (16x8):      c0 (g, 2t)  c1 (g, 2t+1)  c2 (g+8, 2t)  c3 (g+8, 2t+1)
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

__device__ __forceinline__ void dg_mma(double c[4], const double a[4], const double b[2]) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Row and column (inside the 64x64 tile) of accumulator element acc[i][j][e].
__device__ __forceinline__ int dg_row(int i, int e) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return (warp >> 1) * 32 + i * 16 + (lane >> 2) + (e >= 2 ? 8 : 0);
}
__device__ __forceinline__ int dg_col(int j, int e) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return (warp & 1) * 32 + j * 8 + (lane & 3) * 2 + (e & 1);
}

// 8- and 16-byte asynchronous copies; an invalid element reads nothing (src-size 0) from the
// operand's base address and is zero-filled.
__device__ __forceinline__ void dg_cp8(double* smem_dst, const double* gsrc, const double* base, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(valid ? gsrc : base), "r"(bytes));
}
__device__ __forceinline__ void dg_cp16(double* smem_dst, const double* gsrc, const double* base, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    const int bytes = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(valid ? gsrc : base), "r"(bytes));
}

__device__ __forceinline__ void dg_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void dg_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Issue the copies of k-tile kt into pipeline stage `st` (16-byte pairs when PAIRS).
template <bool PAIRS>
__device__ __forceinline__ void dg_load(double* smem, int st, const double* __restrict__ A, int lda, const double* __restrict__ B,
                                        int ldb, int M, int N, int K, int m0, int n0, int kt) {
    double* As = smem + st * DG_STAGE;
    double* Bs = As + DG_TILE * DG_AS;
    const int k0 = kt * DG_BK;
    const int tid = threadIdx.x;
    if constexpr (PAIRS) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int idx = tid + l * DG_THREADS;
            const int ar = idx >> 3, ak = (idx & 7) * 2;
            const int gi = m0 + ar, gk = k0 + ak;
            dg_cp16(&As[ar * DG_AS + ak], A + (long long)gi * lda + gk, A, gi < M && gk < K);
            const int bk = idx >> 5, bc = (idx & 31) * 2;
            const int gbk = k0 + bk, gj = n0 + bc;
            dg_cp16(&Bs[bk * DG_BS + bc], B + (long long)gbk * ldb + gj, B, gbk < K && gj < N);
        }
    } else {
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
}

// Whether this warp's 32x32 quarter of the 64x64 tile needs computing: not when it is padding
// or, in a tile on the diagonal of a symmetric result (only its upper triangle is needed), when it
// lies below the diagonal.  (Skipping finer 16x8 blocks inside a quarter costs more in predicated
// issue than it saves.)
__device__ __forceinline__ bool dg_quarter_on(int m0, int n0, int M, int N, bool diag_tile) {
    const int warp = threadIdx.x >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    return m0 + wr < M && n0 + wc < N && !(diag_tile && wr > wc);
}

// acc[i][j][e]: element (dg_row(i, e), dg_col(j, e)) of the 64x64 tile.  A warp with
// compute == false still takes part in the copies and barriers but issues no MMAs; the SM gives
// its issue slots to other CTAs' warps.  PAIRS: both operands can be copied in 16-byte pairs
// (16-byte aligned bases, even leading dimensions, even K and N; the host sorts tiles by it).
// The last k-tile skips its second half when K ends inside the first.
template <bool PAIRS>
__device__ __forceinline__ void dg_mainloop(double* smem, const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
                                            int M, int N, int K, int m0, int n0, double acc[2][4][4], bool compute) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    const int KT = (K + DG_BK - 1) / DG_BK;
#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; ++s) {
        if (s < KT) dg_load<PAIRS>(smem, s, A, lda, B, ldb, M, N, K, m0, n0, s);
        dg_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        dg_wait<DG_STAGES - 2>();
        __syncthreads();
        const int nk = kt + DG_STAGES - 1;
        if (nk < KT) dg_load<PAIRS>(smem, nk % DG_STAGES, A, lda, B, ldb, M, N, K, m0, n0, nk);
        dg_commit();
        const double* As = smem + (kt % DG_STAGES) * DG_STAGE;
        const double* Bs = As + DG_TILE * DG_AS;
        if (!compute) continue;
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 8) {
            if (kk > 0 && kt * DG_BK + kk >= K) break;
            double a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double* ar = As + (wr + i * 16 + g) * DG_AS + kk + tq;
                a[i][0] = ar[0];
                a[i][1] = ar[8 * DG_AS];
                a[i][2] = ar[4];
                a[i][3] = ar[8 * DG_AS + 4];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double* br = Bs + (kk + tq) * DG_BS + wc + j * 8 + g;
                b[j][0] = br[0];
                b[j][1] = br[4 * DG_BS];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dg_mma(acc[i][j], a[i], b[j]);
        }
    }
    dg_wait<0>();
    __syncthreads();
}

// acc = A1[m0:, :K] . B1[:K, n0:] - A2[m0:, :K] . B2[:K, n0:], as one pipelined k-loop over 2K:
// the k-tiles of the second product follow those of the first, and the accumulator is negated
// between the two (so the pipeline never drains in the middle).  All four operands share M = N = K
// and the leading dimension ld.  Same fragment layout and `compute` rule as dg_mainloop.
template <bool PAIRS>
__device__ __forceinline__ void dg_mainloop_diff(double* smem, const double* __restrict__ A1, const double* __restrict__ B1,
                                                 const double* __restrict__ A2, const double* __restrict__ B2, int ld,
                                                 int n, int m0, int n0, double acc[2][4][4], bool compute) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    const int KT = (n + DG_BK - 1) / DG_BK;  // k-tiles per product
    auto load = [&](int st, int kt) {
        if (kt < KT)
            dg_load<PAIRS>(smem, st, A1, ld, B1, ld, n, n, n, m0, n0, kt);
        else
            dg_load<PAIRS>(smem, st, A2, ld, B2, ld, n, n, n, m0, n0, kt - KT);
    };
#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; ++s) {
        if (s < 2 * KT) load(s, s);
        dg_commit();
    }
    for (int kt = 0; kt < 2 * KT; ++kt) {
        dg_wait<DG_STAGES - 2>();
        __syncthreads();
        const int nk = kt + DG_STAGES - 1;
        if (nk < 2 * KT) load(nk % DG_STAGES, nk);
        dg_commit();
        const double* As = smem + (kt % DG_STAGES) * DG_STAGE;
        const double* Bs = As + DG_TILE * DG_AS;
        if (!compute) continue;
        if (kt == KT) {  // first product done: acc = -A1.B1, then accumulate A2.B2
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[i][j][e] = -acc[i][j][e];
        }
        const int kbase = (kt < KT ? kt : kt - KT) * DG_BK;
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 8) {
            if (kk > 0 && kbase + kk >= n) break;
            double a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double* ar = As + (wr + i * 16 + g) * DG_AS + kk + tq;
                a[i][0] = ar[0];
                a[i][1] = ar[8 * DG_AS];
                a[i][2] = ar[4];
                a[i][3] = ar[8 * DG_AS + 4];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double* br = Bs + (kk + tq) * DG_BS + wc + j * 8 + g;
                b[j][0] = br[0];
                b[j][1] = br[4 * DG_BS];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dg_mma(acc[i][j], a[i], b[j]);
        }
    }
    dg_wait<0>();
    __syncthreads();
    // acc = A2.B2 - A1.B1: flip to A1.B1 - A2.B2
    if (compute) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = -acc[i][j][e];
    }
}

}  // namespace am1
