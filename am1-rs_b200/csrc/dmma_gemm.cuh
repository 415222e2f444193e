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

#include <cstdint>

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
// lies below the diagonal.  (In the cp.async loops, skipping finer 16x8 blocks inside a quarter by
// predicates cost more in issue than it saved; the TMA loop dispatches once per k-tile on the
// quarter's shape instead, dg_quarter_shape.)
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

// ---------------------------------------------------------------------------------------------
// TMA-fed main loop for products of symmetric matrices.  Both operands of a 64x64 output tile are
// 64-row blocks read along k: A = Ma[m0:m0+64, :], and B[:, n0:n0+64] = Mb[n0:n0+64, :]^T (Mb
// symmetric).  Each k-tile of an operand is one 2D box of 16 doubles (128 bytes) x 64 rows copied by
// the tensor memory accelerator (cp.async.bulk.tensor) from a tensor map of the n x n row-major
// matrix; rows and columns past n read as zero.  The map uses the 128-byte swizzle: 16-byte chunk c
// of box row r lands at r * 128 + (c ^ (r % 8)) * 16.
//
// Thread 0 issues the copies.  Each stage has a "full" mbarrier (the copies' byte count) and an
// "empty" one (one arrival per warp when it has read the stage).  After its own k-tile g, thread 0
// refills the stage that k-tile g - 1 used with k-tile g - 1 + DT_STAGES, so a warp may run up to two
// k-tiles ahead of the others: no CTA barrier inside the k-loop.  The MMAs, their fragments and
// their order are those of dg_mainloop (acc bit-identical for symmetric operands).
//
// Every wait is bounded (DT_WAIT_LIMIT polls).  A wait that runs out stops the loop in every warp,
// thread 0 waits (bounded) for the copies it issued, and the function returns false on all threads:
// the caller writes nothing for the tile and reports the error.
constexpr int DT_STAGES = 3;
constexpr int DT_OP_BYTES = DG_TILE * DG_BK * 8;  // one operand box: 64 rows x 128 bytes
constexpr int DT_STAGE_BYTES = 2 * DT_OP_BYTES;
constexpr size_t DT_SMEM = DT_STAGES * DT_STAGE_BYTES + 1024;  // + room to align the stages to 1024 bytes
constexpr long long DT_WAIT_LIMIT = 1LL << 22;

struct DtBars {
    unsigned long long full[DT_STAGES], empty[DT_STAGES];
};

__device__ __forceinline__ uint32_t dt_saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// the stages: the dynamic shared memory rounded up to 1024 bytes (the swizzle atom)
__device__ __forceinline__ unsigned char* dt_stages(unsigned char* dyn) {
    const uint32_t a = dt_saddr(dyn);
    return dyn + (((a + 1023u) & ~1023u) - a);
}

// Which 16x8 MMA blocks of this warp's 32x32 quarter the TMA main loop issues, as one code:
// mi row blocks (1-2) and nj column blocks (1-4) that reach inside the M x N result, and, in a
// quarter on the diagonal of a diagonal tile (a symmetric or antisymmetric result, only its upper
// triangle kept), dg = 1: blocks (1, 0) and (1, 1) lie wholly below the diagonal and are skipped.
// 0: the warp issues no MMAs (dg_quarter_on is false).  Skipped blocks keep a zero accumulator,
// and the epilogues read no element of them, so the kept elements are bit-identical to a full
// quarter's.  At the benchmark's sizes this issues 1.10 instead of 1.28 times the algorithmic flops.
__host__ __device__ constexpr int dt_shape(int mi, int nj, int dg) { return mi * 16 + nj * 2 + dg; }
constexpr int DT_FULL = dt_shape(2, 4, 0);

__device__ __forceinline__ int dg_quarter_shape(int m0, int n0, int M, int N, bool diag_tile) {
    if (!dg_quarter_on(m0, n0, M, N, diag_tile)) return 0;
    const int warp = threadIdx.x >> 5;
    const int r0 = m0 + (warp >> 1) * 32, c0 = n0 + (warp & 1) * 32;
    const int mi = min(2, (M - r0 + 15) / 16), nj = min(4, (N - c0 + 7) / 8);
    return dt_shape(mi, nj, (diag_tile && r0 - m0 == c0 - n0 && mi == 2) ? 1 : 0);
}

// one k-tile (two k-steps of 8; the second skipped when K ends inside the first) over the blocks of
// shape (MI, NJ, DG), operands in the 128-byte-swizzled boxes; c0 = (tq >> 1) ^ g of the lane
template <int MI, int NJ, bool DG>
__device__ __forceinline__ void dt_ktile(const unsigned char* As, const unsigned char* Bs, int ra, int rb, int c0, int kbase, int K,
                                         double acc[2][4][4]) {
#pragma unroll
    for (int kk = 0; kk < DG_BK; kk += 8) {
        if (kk > 0 && kbase + kk >= K) break;
        const int x0 = (c0 ^ (kk >> 1)) << 4, x1 = (c0 ^ ((kk >> 1) | 2)) << 4;
        double a[MI][4], b[NJ][2];
#pragma unroll
        for (int i = 0; i < MI; ++i) {
            const unsigned char* p = As + ra + i * 16 * 128;
            a[i][0] = *reinterpret_cast<const double*>(p + x0);
            a[i][1] = *reinterpret_cast<const double*>(p + 8 * 128 + x0);
            a[i][2] = *reinterpret_cast<const double*>(p + x1);
            a[i][3] = *reinterpret_cast<const double*>(p + 8 * 128 + x1);
        }
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const unsigned char* p = Bs + rb + j * 8 * 128;
            b[j][0] = *reinterpret_cast<const double*>(p + x0);
            b[j][1] = *reinterpret_cast<const double*>(p + x1);
        }
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j)
                if (!(DG && i == 1 && j < 2)) dg_mma(acc[i][j], a[i], b[j]);
    }
}

__device__ __forceinline__ void dt_ktile_shape(int shape, const unsigned char* As, const unsigned char* Bs, int ra, int rb, int c0,
                                               int kbase, int K, double acc[2][4][4]) {
    if (shape == DT_FULL) {
        dt_ktile<2, 4, false>(As, Bs, ra, rb, c0, kbase, K, acc);
        return;
    }
    switch (shape) {
        case dt_shape(2, 4, 1): dt_ktile<2, 4, true>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(2, 3, 1): dt_ktile<2, 3, true>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(2, 3, 0): dt_ktile<2, 3, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(2, 2, 0): dt_ktile<2, 2, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(2, 1, 0): dt_ktile<2, 1, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(1, 4, 0): dt_ktile<1, 4, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(1, 3, 0): dt_ktile<1, 3, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(1, 2, 0): dt_ktile<1, 2, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        case dt_shape(1, 1, 0): dt_ktile<1, 1, false>(As, Bs, ra, rb, c0, kbase, K, acc); break;
        default: break;
    }
}

// true once the phase with this parity has completed; false after DT_WAIT_LIMIT polls
__device__ __forceinline__ bool dt_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < DT_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\n"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// one 16 x 64 box (x = first k, y = first row) of the matrix behind `map` into shared memory at
// `dst`, counted on mbarrier `bar`
__device__ __forceinline__ void dt_copy(uint32_t dst, const void* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// acc = Ma1[m0:, :].Mb1[n0:, :]^T (map_a2 == nullptr), or that minus Ma2[m0:, :].Mb2[n0:, :]^T as
// one pipeline over 2K k-tiles (the accumulator is negated between the two products, as in
// dg_mainloop_diff).  same_ab: Ma1 == Mb1 and m0 == n0 (a diagonal tile of X.X): one box per k-tile.
// K: the matrices' order.  Same fragment layout as dg_mainloop; shape (dg_quarter_shape) says which
// MMA blocks the warp issues, none when 0.
__device__ __forceinline__ bool dg_mainloop_tma(unsigned char* stages, DtBars& bars, const void* map_a1, const void* map_b1,
                                                const void* map_a2, const void* map_b2, bool same_ab, int K, int m0, int n0,
                                                double acc[2][4][4], int shape) {
    const bool compute = shape != 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    const int KT = (K + DG_BK - 1) / DG_BK;  // k-tiles per product
    const int NT = map_a2 ? 2 * KT : KT;
    const uint32_t sbase = dt_saddr(stages);
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < DT_STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(dt_saddr(&bars.full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(dt_saddr(&bars.empty[s])), "r"(DG_THREADS / 32));
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    int issued = 0, landed = 0;  // thread 0: k-tiles issued; warp 0: k-tiles seen landed
    auto issue = [&](int kt) {
        const int s = kt % DT_STAGES;
        const uint32_t fb = dt_saddr(&bars.full[s]);
        const uint32_t a = sbase + s * DT_STAGE_BYTES;
        const bool second = kt >= KT;
        const int x = (second ? kt - KT : kt) * DG_BK;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb),
                     "r"(same_ab ? DT_OP_BYTES : DT_STAGE_BYTES)
                     : "memory");
        dt_copy(a, second ? map_a2 : map_a1, x, m0, fb);
        if (!same_ab) dt_copy(a + DT_OP_BYTES, second ? map_b2 : map_b1, x, n0, fb);
    };
    if (tid == 0)
        for (; issued < DT_STAGES && issued < NT; ++issued) issue(issued);
    // lane-constant part of the swizzled fragment addresses: row g of each 8-row group, chunk
    // (k / 2) ^ g with k = kk + tq (a0, a1, b0) or kk + tq + 4 (a2, a3, b1)
    const int lo8 = (tq & 1) * 8;
    const int ra = (wr + g) * 128 + lo8, rb = (wc + g) * 128 + lo8;
    const int c0 = (tq >> 1) ^ g;
    bool ok = true;
    for (int kt = 0; kt < NT; ++kt) {
        const int s = kt % DT_STAGES;
        ok = __all_sync(0xffffffffu, dt_wait(dt_saddr(&bars.full[s]), (kt / DT_STAGES) & 1));
        if (!ok) break;
        if (warp == 0) landed = kt + 1;
        const unsigned char* As = stages + s * DT_STAGE_BYTES;
        const unsigned char* Bs = same_ab ? As : As + DT_OP_BYTES;
        if (compute) {
            if (kt == KT) {  // first product done: acc = -A1.B1, then accumulate A2.B2
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int e = 0; e < 4; ++e) acc[i][j][e] = -acc[i][j][e];
            }
            const int kbase = (kt < KT ? kt : kt - KT) * DG_BK;
            dt_ktile_shape(shape, As, Bs, ra, rb, c0, kbase, K, acc);
        }
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(dt_saddr(&bars.empty[s])) : "memory");
        if (warp == 0) {
            // the stage k-tile kt - 1 used takes k-tile kt - 1 + DT_STAGES
            int pok = 1;
            if (lane == 0 && kt >= 1 && issued < NT) {
                const int kp = kt - 1;
                if (dt_wait(dt_saddr(&bars.empty[kp % DT_STAGES]), (kp / DT_STAGES) & 1))
                    issue(issued++);
                else
                    pok = 0;
            }
            ok = __shfl_sync(0xffffffffu, pok, 0) != 0;
            if (!ok) break;
        }
    }
    if (tid == 0 && !ok)
        for (int k = landed; k < issued; ++k) dt_wait(dt_saddr(&bars.full[k % DT_STAGES]), (k / DT_STAGES) & 1);
    if (!__syncthreads_and(ok)) return false;
    if (map_a2 && compute) {  // acc = A2.B2 - A1.B1: flip to A1.B1 - A2.B2
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = -acc[i][j][e];
    }
    return true;
}

}  // namespace am1
