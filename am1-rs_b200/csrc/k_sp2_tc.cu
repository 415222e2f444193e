// Reduced-precision purification step on the fifth-generation tensor cores (tcgen05): the product
// X.X of the mixed path's early SCF iterations, at FP32 accuracy from TF32 operands (3xTF32), in
// 128 x 128 output tiles accumulated in tensor memory.
//
// The iterate X is held in FP32 (rows of ldf floats, pad columns zero) and is symmetric, so both
// operands of a tile are row blocks of X read along k: A = X[m0:m0+128, :], B = X[n0:n0+128, :]
// (D = A B^T = X^2 on that tile), both K-major.  A k-stage of 32 columns is 128 bytes per row: one
// 128-byte swizzle atom, copied with 16-byte cp.async into the swizzled layout the MMA descriptors
// describe (chunk c of row r at r * 128 + ((c ^ (r % 8)) * 16)).  Each value is split in shared
// memory into hi (its top 19 bits, a TF32 value) and lo = x - hi (exact in FP32, read as TF32 by the
// tensor cores), for both operands, and each k-stage issues hi.hi + hi.lo + lo.hi
// (tcgen05.mma kind::tf32, M = N = 128, K = 8, FP32 accumulation in TMEM): products to about 2^-22
// relative, FP32 accuracy.  One thread issues the MMAs; tcgen05.commit signals an mbarrier per
// stage, which frees the stage for the copies of the stage after next (three stages in flight).
//
// Epilogue: each warp reads its 32 TMEM lanes (tile rows) with tcgen05.ld, the tile goes through
// shared memory, and Y = X^2 or 2X - X^2 is written with coalesced rows, mirrored across the
// diagonal (Y stays exactly symmetric), with the tile's FP64 share of tr Y and ||Y||_F^2.
//
// Every mbarrier wait is bounded; a wait that runs out sets bit 8 of the job's error word, the CTA
// waits (bounded) for its MMAs, frees its TMEM and returns without writing the tile.
//
// k_sp2_step_tc1 is the single-pass form for iterates held as TF32 values (Sp2Job::lowp_tc == 2, the
// precision of the mma.sync TF32 kernel): no lo parts, one MMA per K = 8, every stored iterate rounded
// to the nearest TF32 value, the operands copied by TMA from tensor maps of the FP32 iterates; its
// stages are half the size, so two CTAs fit an SM.
#include <cuda_runtime.h>

#include <cstdint>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

namespace {

constexpr int TC_TILE = 128;                // output tile rows and columns (UMMA M = N)
constexpr int TC_BK = 32;                   // floats per k-stage: one 128-byte swizzle row
constexpr int TC_STAGES = 3;
constexpr int TC_OP_BYTES = TC_TILE * 128;  // one operand of one stage: 128 rows x 128 B
constexpr int TC_STAGE_BYTES = 4 * TC_OP_BYTES;  // A, B, A_lo, B_lo
constexpr int TC1_STAGE_BYTES = 2 * TC_OP_BYTES;  // A, B (single pass)
constexpr int TC_THREADS = 128;
constexpr int TC_OUT_LD = TC_TILE + 1;      // staged output tile row stride (floats)
constexpr uint32_t TC_TMEM_COLS = 128;      // FP32 accumulator: 128 lanes x 128 columns
constexpr long long TC_WAIT_LIMIT = 1LL << 22;

// Instruction descriptor of tcgen05.mma kind::tf32: FP32 accumulator (bits 4-5 = 1), A and B TF32
// (bits 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_TILE >> 3) << 17) |
                              ((uint32_t)(TC_TILE >> 4) << 24);

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzled layout: start
// address >> 4 (bits 0-13), leading-dimension offset 1 (unused by swizzled K-major layouts, bits
// 16-29), 1024 bytes between 8-row groups >> 4 (bits 32-45), descriptor version 1 (bits 46-47),
// swizzle mode 2 = 128-byte (bits 61-63).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_cp16(uint32_t sdst, const float* gsrc, const float* base, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(valid ? gsrc : base), "r"(valid ? 16 : 0));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

// true once the phase with this parity has completed; false after TC_WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < TC_WAIT_LIMIT; ++it) {
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

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

// The copies of k-stage kt (columns 32 kt .. 32 kt + 31) of the A and B row blocks into stage st.
// Thread t takes chunks t, t + 128, ... of the 1024 chunks (128 rows x 8) of each operand.
__device__ __forceinline__ void tc_load(uint32_t stage, const float* __restrict__ X, int ldf, int n, int m0, int n0, int kt) {
    const int k0 = kt * TC_BK;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int idx = threadIdx.x + l * TC_THREADS;
        const int r = idx >> 3, c = idx & 7;
        const uint32_t off = (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
        const int gk = k0 + 4 * c;
        const int ga = m0 + r, gb = n0 + r;
        tc_cp16(stage + off, X + (long long)ga * ldf + gk, X, ga < n && gk < ldf);
        tc_cp16(stage + TC_OP_BYTES + off, X + (long long)gb * ldf + gk, X, gb < n && gk < ldf);
    }
}

// hi = x with its low 13 bits cleared (exactly a TF32 value, whatever the tensor cores do with the
// low bits of an FP32 word) in place, and lo = x - hi (exact in FP32) into the A_lo and B_lo parts
// of the stage, for the chunks this thread copied.
__device__ __forceinline__ void tc_split(unsigned char* stage) {
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int idx = threadIdx.x + l * TC_THREADS;
        const int r = idx >> 3, c = idx & 7;
        const int off = r * 128 + ((c ^ (r & 7)) << 4);
#pragma unroll
        for (int op = 0; op < 2; ++op) {
            float4* hp = reinterpret_cast<float4*>(stage + op * TC_OP_BYTES + off);
            const float4 v = *hp;
            float4 hi, lo;
            hi.x = __uint_as_float(__float_as_uint(v.x) & 0xFFFFE000u);
            hi.y = __uint_as_float(__float_as_uint(v.y) & 0xFFFFE000u);
            hi.z = __uint_as_float(__float_as_uint(v.z) & 0xFFFFE000u);
            hi.w = __uint_as_float(__float_as_uint(v.w) & 0xFFFFE000u);
            lo.x = v.x - hi.x;
            lo.y = v.y - hi.y;
            lo.z = v.z - hi.z;
            lo.w = v.w - hi.w;
            *hp = hi;
            *reinterpret_cast<float4*>(stage + (2 + op) * TC_OP_BYTES + off) = lo;
        }
    }
}

}  // namespace

size_t tc_smem_bytes() { return (size_t)TC_STAGES * TC_STAGE_BYTES + 1024; }
size_t tc1_smem_bytes() { return (size_t)TC_STAGES * TC1_STAGE_BYTES + 1024; }
static_assert(TC_STAGES * TC1_STAGE_BYTES >= TC_TILE * TC_OUT_LD * (int)sizeof(float), "the staged output tile fits the stages");

// The tile after its MMAs (every thread; `good`: the k-loop finished): the accumulator out of TMEM
// into the free stages, TMEM freed, then Y = X^2 or 2X - X^2 written along rows (the direct block)
// and along the mirrored rows, with the tile's share of tr Y and ||Y||_F^2.  ROUND: every stored
// value rounded to the nearest TF32 value.
template <bool ROUND>
__device__ __forceinline__ void tc_epilogue(const Sp2Job* __restrict__ jp, const Sp2State* __restrict__ sp, int t, const float* X, float* Y,
                                            int n, int ldf, int m0, int n0, bool diag, uint32_t tmem, unsigned char* base, bool good,
                                            int* __restrict__ err, double (&red)[2][4]) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* out = reinterpret_cast<float*>(base);  // the stages are free: the tile of X.X, row stride TC_OUT_LD
    if (good) {
        const int r = warp * 32 + lane;  // the tile row this thread reads from TMEM lane r
#pragma unroll 1
        for (int c0 = 0; c0 < TC_TILE; c0 += 32) {
            uint32_t v[32];
            const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
                  "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
                  "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
                  "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; ++j) out[r * TC_OUT_LD + c0 + j] = __uint_as_float(v[j]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_TMEM_COLS));
    if (!good) {
        if (tid == 0) atomicOr(err, 1 << 8);
        return;
    }
    // Y = X^2 or 2X - X^2, written along rows (the direct block) and along the mirrored rows; on a
    // diagonal tile element (i, j) takes the value of (min, max), so Y is exactly symmetric
    const int square = sp->square;
    double tr = 0.0, fr = 0.0;
    for (int idx = tid; idx < TC_TILE * TC_TILE; idx += TC_THREADS) {
        const int i = idx / TC_TILE, j = idx % TC_TILE;  // consecutive threads: consecutive columns
        const int r = m0 + i, c = n0 + j;
        if (r >= n || c >= n) continue;
        int si = i, sj = j;
        if (diag && i > j) {
            si = j;
            sj = i;
        }
        const float x2 = out[si * TC_OUT_LD + sj];
        const float y0 = square ? x2 : 2.0f * X[(long long)(m0 + si) * ldf + (n0 + sj)] - x2;
        const float y = ROUND ? tf32_round(y0) : y0;
        Y[(long long)r * ldf + c] = y;
        if (diag) {
            fr += (double)y * y;
            if (i == j) tr += y;
        } else {
            fr += 2.0 * (double)y * y;
        }
    }
    if (!diag) {
        for (int idx = tid; idx < TC_TILE * TC_TILE; idx += TC_THREADS) {
            const int j = idx / TC_TILE, i = idx % TC_TILE;  // consecutive threads: consecutive tile rows
            const int r = m0 + i, c = n0 + j;
            if (r >= n || c >= n) continue;
            const float x2 = out[i * TC_OUT_LD + j];
            const float y0 = square ? x2 : 2.0f * X[(long long)r * ldf + c] - x2;
            Y[(long long)c * ldf + r] = ROUND ? tf32_round(y0) : y0;
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
        double* p = jp->part + 2 * (t - jp->tc_tile0);
        p[0] = red[0][0] + red[0][1] + red[0][2] + red[0][3];
        p[1] = red[1][0] + red[1][1] + red[1][2] + red[1][3];
    }
}


// The cp.async-fed k-loop: SPLIT, 3xTF32 from unrounded FP32 iterates (k_sp2_step_tc, lowp_tc == 1);
// otherwise one TF32 pass over TF32 iterates (lowp_tc == 2; k_sp2_step_tc1 feeds that one by TMA)
template <bool SPLIT>
__device__ __forceinline__ void sp2_step_tc_body(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles, int ntiles,
                                                 const Sp2State* __restrict__ sst, int* __restrict__ err) {
    constexpr int STAGE_BYTES = SPLIT ? TC_STAGE_BYTES : TC1_STAGE_BYTES;
    extern __shared__ unsigned char tc_raw[];
    __shared__ __align__(8) uint64_t bars[TC_STAGES];
    __shared__ uint32_t tmem_slot;
    __shared__ double red[2][4];
    __shared__ int fail;
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || !sp->lowp || jp->lowp_tc != (SPLIT ? 1 : 2)) return;  // FP64, mma.sync TF32, other tcgen05 form elsewhere
    const int n = jp->n, ldf = jp->ldf;
    const int cur = sp->cur;
    const float* X = cur ? jp->Xf1 : jp->Xf0;
    float* Y = cur ? jp->Xf0 : jp->Xf1;
    const int m0 = tl.tm * TC_TILE, n0 = tl.tn * TC_TILE;
    const bool diag = tl.tm == tl.tn;
    const int tid = threadIdx.x, warp = tid >> 5;
    // 1024-byte aligned stages (the swizzle atom)
    unsigned char* base = tc_raw + ((1024u - (smem_addr(tc_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(base);
    if (tid == 0) {
        fail = 0;
        for (int s = 0; s < TC_STAGES; ++s) mbar_init(smem_addr(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int KT = (n + TC_BK - 1) / TC_BK;
    for (int s = 0; s < TC_STAGES - 1 && s < KT; ++s) {
        tc_load(sbase + s * STAGE_BYTES, X, ldf, n, m0, n0, s);
        asm volatile("cp.async.commit_group;\n");
    }
    uint32_t phase_bits = 0;  // parity of the next completion of each stage's barrier
    bool ok = true;
    for (int kt = 0; kt < KT; ++kt) {
        const int st = kt % TC_STAGES;
        // stage st holds k-stage kt once this thread's copies of it have landed
        if (kt + 1 < KT) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        if constexpr (SPLIT) tc_split(base + st * STAGE_BYTES);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t a = sbase + st * STAGE_BYTES, b = a + TC_OP_BYTES, alo = a + 2 * TC_OP_BYTES, blo = a + 3 * TC_OP_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_BK / 8; ++kk) {  // K = 8 per MMA: 32 bytes along the swizzled row
                const uint32_t o = 32u * kk;
                tc_mma(tmem, tc_desc(a + o), tc_desc(b + o), (kt > 0 || kk > 0) ? 1u : 0u);
                if constexpr (SPLIT) {
                    tc_mma(tmem, tc_desc(a + o), tc_desc(blo + o), 1u);
                    tc_mma(tmem, tc_desc(alo + o), tc_desc(b + o), 1u);
                }
            }
            tc_commit(smem_addr(&bars[st]));
        }
        // the copies of k-stage kt + 2 go into the stage k-stage kt - 1 used, once its MMAs are done
        const int nk = kt + TC_STAGES - 1;
        if (nk < KT) {
            const int ns = nk % TC_STAGES;
            if (kt >= 1) {
                if (!mbar_wait(smem_addr(&bars[ns]), (phase_bits >> ns) & 1u)) ok = false;
                phase_bits ^= 1u << ns;
            }
            tc_load(sbase + ns * STAGE_BYTES, X, ldf, n, m0, n0, nk);
        }
        asm volatile("cp.async.commit_group;\n");
        if (__syncthreads_or(!ok)) {  // every thread leaves together (the barrier at the top of the loop)
            ok = false;
            break;
        }
    }
    // every MMA is done once the barrier of the last k-stage completes (commits are in order)
    if (ok) {
        const int ls = (KT - 1) % TC_STAGES;
        // completions of stage ls so far: the ones already waited for, plus this last one
        if (!mbar_wait(smem_addr(&bars[ls]), (phase_bits >> ls) & 1u)) ok = false;
    }
    if (!ok) atomicOr(&fail, 1);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    tc_epilogue<!SPLIT>(jp, sp, t, X, Y, n, ldf, m0, n0, diag, tmem, base, fail == 0, err, red);
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_sp2_step_tc(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                               int ntiles, const Sp2State* __restrict__ sst, int* __restrict__ err) {
    sp2_step_tc_body<true>(jobs, tiles, ntiles, sst, err);
}

// Single pass with TMA-fed operands.  Thread 0 alone runs the k-loop: each k-stage of A and B is one
// 32-float x 128-row box (cp.async.bulk.tensor, 128-byte swizzle: exactly the layout the UMMA
// descriptors describe) counted on the stage's full mbarrier; after the MMAs of k-stage kt it
// commits them to the stage's empty mbarrier and refills the stage k-stage kt - 1 used once that
// one's MMAs are done, so copies and MMAs overlap with no CTA barrier in the loop.  A diagonal tile
// loads one box per k-stage.  Every wait is bounded; a wait that runs out stops the loop, thread 0
// lets its copies and MMAs still in flight finish (bounded), and the tile is not written.
__global__ void __launch_bounds__(TC_THREADS, 2) k_sp2_step_tc1(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                                int ntiles, const Sp2State* __restrict__ sst,
                                                                const TmaDesc* __restrict__ maps, int* __restrict__ err) {
    extern __shared__ unsigned char tc_raw[];
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES];
    __shared__ uint32_t tmem_slot;
    __shared__ double red[2][4];
    __shared__ int fail;
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || !sp->lowp || jp->lowp_tc != 2) return;
    const int n = jp->n, ldf = jp->ldf;
    const int cur = sp->cur;
    const float* X = cur ? jp->Xf1 : jp->Xf0;
    float* Y = cur ? jp->Xf0 : jp->Xf1;
    const int m0 = tl.tm * TC_TILE, n0 = tl.tn * TC_TILE;
    const bool diag = tl.tm == tl.tn;
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned char* base = tc_raw + ((1024u - (smem_addr(tc_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(base);
    if (tid == 0) {
        fail = 0;
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int KT = (n + TC_BK - 1) / TC_BK;
    if (tid == 0) {
        const void* map = maps + 2 * tl.job + cur;
        const uint32_t tx = diag ? TC_OP_BYTES : 2 * TC_OP_BYTES;
        auto load = [&](int kt) {
            const int s = kt % TC_STAGES;
            const uint32_t fb = smem_addr(&full[s]);
            const uint32_t a = sbase + s * TC1_STAGE_BYTES;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(tx) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(a),
                "l"(map), "r"(kt * TC_BK), "r"(m0), "r"(fb)
                : "memory");
            if (!diag)
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
                        a + TC_OP_BYTES),
                    "l"(map), "r"(kt * TC_BK), "r"(n0), "r"(fb)
                    : "memory");
        };
        int issued = 0, landed = 0, mma_last = -1;
        for (; issued < TC_STAGES && issued < KT; ++issued) load(issued);
        bool ok = true;
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % TC_STAGES;
            if (!mbar_wait(smem_addr(&full[s]), (kt / TC_STAGES) & 1)) {
                ok = false;
                break;
            }
            landed = kt + 1;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a = sbase + s * TC1_STAGE_BYTES, b = diag ? a : a + TC_OP_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_BK / 8; ++kk) {
                const uint32_t o = 32u * kk;
                tc_mma(tmem, tc_desc(a + o), tc_desc(b + o), (kt > 0 || kk > 0) ? 1u : 0u);
            }
            tc_commit(smem_addr(&empty[s]));
            mma_last = kt;
            if (kt >= 1 && issued < KT) {  // issued == kt - 1 + TC_STAGES
                const int kp = kt - 1;
                if (!mbar_wait(smem_addr(&empty[kp % TC_STAGES]), (kp / TC_STAGES) & 1)) {
                    ok = false;
                    break;
                }
                load(issued++);
            }
        }
        // every MMA is done once the commit of the last k-stage has arrived (commits are in order)
        if (mma_last >= 0 && !mbar_wait(smem_addr(&empty[mma_last % TC_STAGES]), (mma_last / TC_STAGES) & 1)) ok = false;
        if (!ok) {
            for (int k = landed; k < issued; ++k) mbar_wait(smem_addr(&full[k % TC_STAGES]), (k / TC_STAGES) & 1);
            fail = 1;
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    tc_epilogue<true>(jp, sp, t, X, Y, n, ldf, m0, n0, diag, tmem, base, fail == 0, err, red);
}

}  // namespace am1
