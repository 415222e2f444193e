// The FP64 purification product X.X on the fifth-generation tensor cores' integer path (tcgen05
// kind::i8), by splitting X into 7-bit digits (the Ozaki scheme with a fixed scale).
//
// Every element of a purification iterate satisfies |x| < 2 (its eigenvalues lie in [0, 1] up to the
// margin of the spectral bounds), so it is written exactly as
//     x = sum_{i=0}^{7} d_i 2^-(5 + 7 i) + r,   d_i = rint(r_i 2^(5 + 7 i)) in [-64, 64],  |r| <= 2^-55
// (each r_{i+1} = r_i - d_i 2^-(5+7i) is exact in FP64).  The digits of X are kept as eight int8 planes
// beside the FP64 iterate.  A product of planes, sum_k d_i[a][k] d_j[b][k], is exact in int32 (|d d| <=
// 2^12, k < 2^13, at most 8 planes per group), and
//     (X X)[a][b] = sum_g 2^-(10 + 7 g) sum_{i + j = g} (D_i D_j^T)[a][b] + O(2^-55 n)
// The groups g = 0..8 are kept (43 plane products; a numpy model of the scheme on SP2 iterates of n = 200
// and 400 gives a largest error of 6e-17 against exact products, below FP64 GEMM's 6e-16).
//
// Tiles of 128 output rows x 48 output columns, upper triangle of the symmetric product (a tile is
// computed when any of its elements has row <= column; it writes those and mirrors them).  Both operands
// are row blocks of the digit planes read along k (X is symmetric: the B operand of column block c is the
// row block c), K-major, 64-byte rows in the 64-byte swizzle (chunk c of row r at r * 64 + ((c ^ ((r >> 1)
// & 3)) * 16)).  A k-stage is 64 columns of all eight planes of both operands (88 KB), two stages; each
// stage issues 43 pairs x 2 MMAs (M = 128, N = 48, K = 32), one accumulator of 48 TMEM columns per group
// (9 x 48 of 512 columns).  The epilogue reads the nine accumulators of its row, forms the FP64 product
// (smallest group first), Y = X^2 or 2X - X^2 in FP64, and writes Y and its digits, both triangles, through
// shared memory, with the tile's FP64 share of tr Y and ||Y||_F^2.
//
// Every mbarrier wait is bounded; a wait that runs out, or an element with |y| >= 2, sets a bit in the error
// word and the tile is not written.
#include <cuda_runtime.h>

#include <cstdint>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

namespace {

constexpr int OZ_M = 128;   // output rows per tile (UMMA M)
constexpr int OZ_N = 48;    // output columns per tile (UMMA N)
constexpr int OZ_BK = 64;   // k per stage: a 64-byte swizzle row of int8
constexpr int OZ_STAGES = 2;
constexpr int OZ_A_PLANE = OZ_M * OZ_BK;   // bytes of one plane of A in a stage
constexpr int OZ_B_PLANE = OZ_N * OZ_BK;
constexpr int OZ_STAGE = kOzPlanes * (OZ_A_PLANE + OZ_B_PLANE);
constexpr int OZ_THREADS = 128;
constexpr int OZ_OUT_LD = OZ_N + 1;  // staged output tile row stride (doubles)
constexpr uint32_t OZ_TMEM_COLS = 512;
constexpr long long OZ_WAIT_LIMIT = 1LL << 22;

// Instruction descriptor of tcgen05.mma kind::i8: S32 accumulator (bits 4-5 = 2), A and B signed 8-bit
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_N >> 3) << 17) | ((uint32_t)(OZ_M >> 4) << 24);

// K-major operand in the 64-byte swizzle: 512 bytes between 8-row groups, swizzle mode 4 (64-byte).
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)4 << 61);
}

__device__ __forceinline__ uint32_t oz_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void oz_cp16(uint32_t sdst, const int8_t* gsrc, const int8_t* base, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(valid ? gsrc : base), "r"(valid ? 16 : 0));
}

__device__ __forceinline__ bool oz_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < OZ_WAIT_LIMIT; ++it) {
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

__device__ __forceinline__ void oz_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(OZ_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// The copies of k-stage kt of every plane of the A rows (m0..m0+127) and B rows (n0..n0+47).
__device__ __forceinline__ void oz_load(uint32_t stage, const int8_t* __restrict__ D, long long plane, int ldq, int n, int m0, int n0,
                                        int kt) {
    const int k0 = kt * OZ_BK;
    // A: 8 planes x 128 rows x 4 chunks = 4096 chunks; B: 8 x 48 x 4 = 1536
    for (int idx = threadIdx.x; idx < kOzPlanes * (OZ_M + OZ_N) * 4; idx += OZ_THREADS) {
        const int c = idx & 3;
        const int rowid = idx >> 2;  // plane-major rows: A planes first, then B planes
        int p, r, base_off, grow;
        if (rowid < kOzPlanes * OZ_M) {
            p = rowid / OZ_M;
            r = rowid % OZ_M;
            base_off = p * OZ_A_PLANE;
            grow = m0 + r;
        } else {
            const int q = rowid - kOzPlanes * OZ_M;
            p = q / OZ_N;
            r = q % OZ_N;
            base_off = kOzPlanes * OZ_A_PLANE + p * OZ_B_PLANE;
            grow = n0 + r;
        }
        const uint32_t off = (uint32_t)(base_off + r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
        const int gk = k0 + 16 * c;
        oz_cp16(stage + off, D + p * plane + (long long)grow * ldq + gk, D, grow < n && gk < ldq);
    }
}

}  // namespace

size_t oz_smem_bytes() { return (size_t)OZ_STAGES * OZ_STAGE + 1024; }

__global__ void __launch_bounds__(OZ_THREADS, 1) k_sp2_step_oz(const Sp2Job* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                               int ntiles, const Sp2State* __restrict__ sst, int* __restrict__ err) {
    extern __shared__ unsigned char oz_raw[];
    __shared__ __align__(8) uint64_t bars[OZ_STAGES];
    __shared__ uint32_t tmem_slot;
    __shared__ double red[2][4];
    __shared__ int fail;
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const Sp2State* sp = sst + tl.job;
    const Sp2Job* jp = jobs + tl.job;
    if (!sp->active || sp->lowp || !jp->oz) return;
    const int n = jp->n, ldq = jp->ldq;
    const long long plane = (long long)n * ldq;
    const int cur = sp->cur;
    const double* X = cur ? jp->X1 : jp->X0;
    double* Y = cur ? jp->X0 : jp->X1;
    const int8_t* Dx = cur ? jp->Dq1 : jp->Dq0;
    int8_t* Dy = cur ? jp->Dq0 : jp->Dq1;
    const int m0 = tl.tm * OZ_M, n0 = tl.tn * OZ_N;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* base = oz_raw + ((1024u - (oz_smem(oz_raw) & 1023u)) & 1023u);
    const uint32_t sbase = oz_smem(base);
    if (tid == 0) {
        fail = 0;
        for (int s = 0; s < OZ_STAGES; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(oz_smem(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(oz_smem(&tmem_slot)), "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int KT = (n + OZ_BK - 1) / OZ_BK;
    oz_load(sbase, Dx, plane, ldq, n, m0, n0, 0);
    asm volatile("cp.async.commit_group;\n");
    uint32_t phase_bits = 0;
    bool ok = true;
    for (int kt = 0; kt < KT; ++kt) {
        const int st = kt & 1;
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // k-stage kt has landed (this thread's copies)
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t a0 = sbase + st * OZ_STAGE, b0 = a0 + kOzPlanes * OZ_A_PLANE;
            // a plane or k offset moves only the start-address field (address >> 4, 14 bits; shared-memory
            // addresses stay below 2^18, so the sum never carries out of the field)
            const uint64_t da0 = oz_desc(a0), db0 = oz_desc(b0);
#pragma unroll
            for (int g = 0; g < kOzGroups; ++g) {
                const uint32_t acc_col = tmem + (uint32_t)(g * OZ_N);
#pragma unroll
                for (int i = 0; i < kOzPlanes; ++i) {
                    const int j = g - i;
                    if (j < 0 || j >= kOzPlanes) continue;
                    const int ilo = g - (kOzPlanes - 1) > 0 ? g - (kOzPlanes - 1) : 0;
#pragma unroll
                    for (int kk = 0; kk < OZ_BK / 32; ++kk) {  // K = 32 per MMA: 32 bytes along the swizzled row
                        const uint64_t da = da0 + (uint64_t)((i * OZ_A_PLANE + 32 * kk) >> 4);
                        const uint64_t db = db0 + (uint64_t)((j * OZ_B_PLANE + 32 * kk) >> 4);
                        oz_mma(acc_col, da, db, (kt > 0 || i > ilo || kk > 0) ? 1u : 0u);
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(oz_smem(&bars[st]))
                         : "memory");
        }
        // while those MMAs run: k-stage kt + 1 into the other stage, once the MMAs of k-stage kt - 1
        // (which read it) are done
        if (kt + 1 < KT) {
            const int ns = st ^ 1;
            if (kt >= 1) {
                if (!oz_wait(oz_smem(&bars[ns]), (phase_bits >> ns) & 1u)) ok = false;
                phase_bits ^= 1u << ns;
            }
            if (ok) oz_load(sbase + ns * OZ_STAGE, Dx, plane, ldq, n, m0, n0, kt + 1);
            asm volatile("cp.async.commit_group;\n");
        }
    }
    if (ok) {  // every MMA is done once the last k-stage's barrier completes
        const int ls = (KT - 1) & 1;
        if (!oz_wait(oz_smem(&bars[ls]), (phase_bits >> ls) & 1u)) ok = false;
    }
    if (!ok) atomicOr(&fail, 1);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    bool good = fail == 0;
    double* out = reinterpret_cast<double*>(base);  // X.X of the tile, row stride OZ_OUT_LD (the stages are free)
    if (good) {
        const int r = warp * 32 + lane;  // tile row = TMEM lane
        double acc[OZ_N];
#pragma unroll
        for (int c = 0; c < OZ_N; ++c) acc[c] = 0.0;
#pragma unroll 1
        for (int g = kOzGroups - 1; g >= 0; --g) {  // smallest contributions first
            const double sc = ldexp(1.0, -(10 + 7 * g));
#pragma unroll
            for (int c0 = 0; c0 < OZ_N; c0 += 16) {
                uint32_t v[16];
                const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * OZ_N + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
                    "[%16];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
                      "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                    : "r"(addr));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[c0 + j] = fma((double)(int)v[j], sc, acc[c0 + j]);
            }
        }
#pragma unroll
        for (int c = 0; c < OZ_N; ++c) out[r * OZ_OUT_LD + c] = acc[c];
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(OZ_TMEM_COLS));
    if (!good) {
        if (tid == 0) atomicOr(err, 1 << 9);
        return;
    }
    // Y = X^2 or 2X - X^2 for the tile's elements with row <= column, mirrored, in FP64, and its digits
    // (computed once per element: the mirrored pass reads them back from shared memory)
    unsigned long long* dig = reinterpret_cast<unsigned long long*>(base + OZ_M * OZ_OUT_LD * sizeof(double));
    const int square = sp->square;
    double tr = 0.0, fr = 0.0;
    int bad = 0;
    for (int idx = tid; idx < OZ_M * OZ_N; idx += OZ_THREADS) {
        const int i = idx / OZ_N, j = idx % OZ_N;  // consecutive threads: consecutive columns
        const int r = m0 + i, c = n0 + j;
        if (r >= n || c >= n || r > c) continue;
        const double x2 = out[i * OZ_OUT_LD + j];
        const double y = square ? x2 : 2.0 * X[(long long)r * n + c] - x2;
        if (!(fabs(y) < 2.0)) bad = 1;
        const unsigned long long dp = oz_digits_packed(y);
        out[i * OZ_OUT_LD + j] = y;
        dig[i * OZ_N + j] = dp;
        Y[(long long)r * n + c] = y;
        oz_store_digits(dp, Dy, plane, (long long)r * ldq + c);
        if (r == c) {
            tr += y;
            fr += y * y;
        } else {
            fr += 2.0 * y * y;
        }
    }
    __syncthreads();
    // the mirrored elements (row > column of the product: element (c, r) for the tile's r < c)
    for (int idx = tid; idx < OZ_M * OZ_N; idx += OZ_THREADS) {
        const int j = idx / OZ_M, i = idx % OZ_M;  // consecutive threads: consecutive tile rows = mirrored columns
        const int r = m0 + i, c = n0 + j;
        if (r >= n || c >= n || r >= c) continue;
        Y[(long long)c * n + r] = out[i * OZ_OUT_LD + j];
        oz_store_digits(dig[i * OZ_N + j], Dy, plane, (long long)c * ldq + r);
    }
    if (bad) atomicOr(err, 1 << 10);
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
        double* p = jp->part + 2 * (t - jp->oz_tile0);
        p[0] = red[0][0] + red[0][1] + red[0][2] + red[0][3];
        p[1] = red[1][0] + red[1][1] + red[1][2] + red[1][3];
    }
}

}  // namespace am1
