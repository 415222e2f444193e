// Fock G(P) build: F^s = H_core + J(P_tot) - K(spin_scale * P^s), am1-rs src/fock.rs:249-511.
//
// One warp per atom A; every off-diagonal block has exactly one writer and every sum is a
// gather in a fixed order, so the result is deterministic and needs no atomics.
//   * the Coulomb term J_A = sum_B (A A | B B) . P_BB (src/fock.rs:427-448) is gathered
//     lane-parallel, a partner per lane, 32 at a time, in registers, and reduced over the warp once
//     per atom;
//   * the exchange blocks K_AB = -s sum P^s_ab (mu nu | lambda sigma) (src/fock.rs:449-466) of a
//     heavy A with heavy B > A: four pairs at a time, their adjacent 100-integral blocks staged
//     through shared memory with coalesced loads, eight lanes per pair and a lane per two outputs,
//     written to F_AB and F_BA;
//   * the exchange of every other pair (a hydrogen on either side: blocks of 10 or 1 integrals)
//     lane-parallel, the lane of the partner writing F_AB and F_BA when A is the pair's first atom.
// The one-centre terms (oc_two_electron, src/fock.rs:27-65 and 321-344) finish the diagonal.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

// packed index of the AO pair (a, b) of one atom (0..9); constexpr, so unrolled loops index
// register arrays with it at compile time
__host__ __device__ constexpr int pack2(int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

// One-centre integral (a b | c d) of one atom (src/fock.rs:27-65).
__device__ __forceinline__ double oc_integral(int a, int b, int c, int d, const DevElem& e) {
    if (a == b && c == d) {
        if (a == 0 && c == 0) return e.g_ss;
        if ((a == 0) != (c == 0)) return e.g_sp;
        return a == c ? e.g_pp : e.g_p2;
    }
    const int ba = min(a, b), bb = max(a, b), kc = min(c, d), kd = max(c, d);
    if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return e.h_sp;
    if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (e.g_pp - e.g_p2);
    return 0.0;
}

constexpr int FOCK_WARPS = 8;
constexpr int FOCK_XX_ROUND = 4;  // heavy-heavy exchange blocks per round of a warp

// the AO pair of packed index q (inverse of pack2)
__host__ __device__ constexpr int pair_hi(int q) { return q < 1 ? 0 : q < 3 ? 1 : q < 6 ? 2 : 3; }
__host__ __device__ constexpr int pair_lo(int q) { return q - pair_hi(q) * (pair_hi(q) + 1) / 2; }

__global__ void __launch_bounds__(32 * FOCK_WARPS, 2) k_fock(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol,
                                                         int natoms_total, const DevElem* __restrict__ params,
                                                         const int* __restrict__ atom_z, const double* __restrict__ wstore,
                                                         double* __restrict__ arena, const MolState* __restrict__ st, int force) {
    __shared__ double s_w[FOCK_WARPS][100 * FOCK_XX_ROUND];
    __shared__ double s_q[FOCK_WARPS][10];
    __shared__ double s_pab[FOCK_WARPS][FOCK_XX_ROUND][2][16];
    __shared__ double s_j[FOCK_WARPS][10];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int a = blockIdx.x * FOCK_WARPS + warp;
    if (a >= natoms_total) return;
    const int m = atom_mol[a];
    if (!force && !st[m].active) return;
    const MolDesc md = mols[m];
    const int n = md.nao, N = md.natoms, h = md.nheavy, Hn = N - h, A = a - md.atom_base;
    const long long nn = (long long)n * n;
    const double* H0 = arena + md.h_base;
    const double* P0 = arena + md.ch_base[0] + SLOT_P * nn;
    const double* P1 = md.nch == 2 ? arena + md.ch_base[1] + SLOT_P * nn : nullptr;
    double* F0 = arena + md.ch_base[0] + SLOT_F * nn;
    double* F1 = md.nch == 2 ? arena + md.ch_base[1] + SLOT_F * nn : nullptr;
    const double sc = md.spin_scale;
    const long long xxsz = 100LL * h * (h - 1) / 2, xhsz = 10LL * h * Hn;
    const double* w = wstore + md.w_base;
    const bool aheavy = A < h;
    const int oA = aheavy ? 4 * A : 4 * h + (A - h);
    const int naA = aheavy ? 4 : 1;
    const int npA = aheavy ? 10 : 1;
    double* wb = s_w[warp];
    auto ptot = [&](long long idx) { return P1 ? P0[idx] + P1[idx] : P0[idx]; };

    // Coulomb gather J_A (per lane over its partners, reduced over the warp once at the end)
    double jl[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) jl[k] = 0.0;
    if (aheavy) {
        // heavy partners, lane-parallel: J_A += (AA|BB) . P_BB over the 10x10 block of the pair
        for (int B = lane; B < h; B += 32) {
            if (B == A) continue;
            const int oB = 4 * B;
            const int i = min(A, B), j = max(A, B);
            const double* blk = w + 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
            double pq[10];  // packed P_BB, off-diagonal pairs counted twice
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                const int hi = pair_hi(q), lo = pair_lo(q);
                const double v = ptot((long long)(oB + hi) * n + oB + lo);
                pq[q] = hi == lo ? v : 2.0 * v;
            }
            if (A == i) {  // A's side of the block is its rows
#pragma unroll
                for (int k = 0; k < 10; ++k) {
                    double acc = 0.0;
#pragma unroll
                    for (int q = 0; q < 10; ++q) acc = fma(blk[k * 10 + q], pq[q], acc);
                    jl[k] += acc;
                }
            } else {  // A is the pair's second atom: its side is the columns
#pragma unroll
                for (int k = 0; k < 10; ++k) {
                    double acc = 0.0;
#pragma unroll
                    for (int q = 0; q < 10; ++q) acc = fma(blk[q * 10 + k], pq[q], acc);
                    jl[k] += acc;
                }
            }
        }
        // exchange blocks with the heavier-indexed heavy partners (A is the pair's first atom), four
        // partners at a time: lanes 8p..8p+7 take B0 + p, a lane per two output elements of the 4 x 4
        // block (each element the same sum, in the same order, as one partner at a time)
        const int slot = lane >> 3, l8 = lane & 7;
        for (int B0 = A + 1; B0 < h; B0 += FOCK_XX_ROUND) {
            const int nb = min(FOCK_XX_ROUND, h - B0);  // partners in this round
            const double* blk0 = w + 100LL * ((long long)A * h - (long long)A * (A + 1) / 2 + (B0 - A - 1));
            for (int l = lane; l < 100 * nb; l += 32) wb[l] = blk0[l];  // the blocks of (A, B0 ..) are adjacent
            const int B = B0 + slot;
            const bool mine = slot < nb;
            const int oB = 4 * B;
            if (mine) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = 2 * l8 + u;
                    const long long idx = (long long)(oA + (e >> 2)) * n + oB + (e & 3);
                    s_pab[warp][slot][0][e] = P0[idx];
                    if (P1) s_pab[warp][slot][1][e] = P1[idx];
                }
            }
            __syncwarp();
            if (mine) {
                const double* wbh = wb + 100 * slot;
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = 2 * l8 + u;
                    const int mu = e >> 2, la = e & 3;
                    const long long ab = (long long)(oA + mu) * n + oB + la;
                    const long long ba = (long long)(oB + la) * n + oA + mu;
                    const double hab = H0[ab];
                    for (int c = 0; c < md.nch; ++c) {
                        double acc = 0.0;
#pragma unroll
                        for (int nu = 0; nu < 4; ++nu) {
                            const double* row = wbh + pack2(mu, nu) * 10;
#pragma unroll
                            for (int sg = 0; sg < 4; ++sg) acc += s_pab[warp][slot][c][nu * 4 + sg] * row[pack2(la, sg)];
                        }
                        const double v = hab - acc * sc;
                        double* F = c == 0 ? F0 : F1;
                        F[ab] = v;
                        F[ba] = v;
                    }
                }
            }
            __syncwarp();
        }
    }
    // every other partner, lane-parallel
    if (aheavy) {
        // hydrogen partners B (XH blocks: A's 10 packed pairs x B's ss); A is the first atom
        for (int B = h + lane; B < N; B += 32) {
            const int oB = 4 * h + (B - h);
            const double* blk = w + xxsz + 10LL * ((long long)A * Hn + (B - h));
            double wv[10];
#pragma unroll
            for (int k = 0; k < 10; ++k) wv[k] = blk[k];
            const double pbb = ptot((long long)oB * n + oB);
#pragma unroll
            for (int k = 0; k < 10; ++k) jl[k] += wv[k] * pbb;
            const double* Hrow = H0 + (long long)oB * n + oA;
            for (int c = 0; c < md.nch; ++c) {
                const double* Pr = (c == 0 ? P0 : P1) + (long long)oB * n + oA;  // P_BA = P_AB (symmetric)
                const double p0 = Pr[0], p1 = Pr[1], p2 = Pr[2], p3 = Pr[3];
                double* F = c == 0 ? F0 : F1;
#pragma unroll
                for (int mu = 0; mu < 4; ++mu) {
                    const double acc = p0 * wv[pack2(mu, 0)] + p1 * wv[pack2(mu, 1)] + p2 * wv[pack2(mu, 2)] + p3 * wv[pack2(mu, 3)];
                    const double v = Hrow[mu] - acc * sc;
                    F[(long long)oB * n + oA + mu] = v;
                    F[(long long)(oA + mu) * n + oB] = v;
                }
            }
        }
    } else {
        const int A2 = A - h;
        // heavy partners B (XH block of (B, A): B's 10 packed pairs x A's ss); B is the first atom
        for (int B = lane; B < h; B += 32) {
            const int oB = 4 * B;
            const double* blk = w + xxsz + 10LL * ((long long)B * Hn + A2);
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                const int hi = pair_hi(q), lo = pair_lo(q);
                const double v = ptot((long long)(oB + hi) * n + oB + lo);
                acc += blk[q] * (hi == lo ? v : 2.0 * v);
            }
            jl[0] += acc;
        }
        // hydrogen partners B (HH blocks); exchange when A is the first atom (B > A).  Two partners per
        // lane per trip, every load of the trip before its stores; each lane keeps its partner order.
        for (int B0 = h + lane; B0 < N; B0 += 64) {
            double wv[2], pbb[2], hab[2], pab[2][2];
            long long ab[2], ba[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int B = B0 + 32 * u;
                const bool valid = B < N && B != A, ex = valid && B > A;
                const int B2 = B - h;
                const int i2 = min(A2, B2), j2 = max(A2, B2);
                const int oB = 4 * h + B2;
                wv[u] = valid ? w[xxsz + xhsz + ((long long)i2 * Hn - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1))] : 0.0;
                pbb[u] = valid ? ptot((long long)oB * n + oB) : 0.0;
                ab[u] = (long long)oA * n + oB;
                ba[u] = (long long)oB * n + oA;
                hab[u] = ex ? H0[ab[u]] : 0.0;
                pab[u][0] = ex ? P0[ab[u]] : 0.0;
                pab[u][1] = ex && P1 ? P1[ab[u]] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int B = B0 + 32 * u;
                if (!(B < N && B != A)) continue;
                jl[0] += wv[u] * pbb[u];
                if (B > A) {
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        if (c >= md.nch) break;
                        const double v = hab[u] - sc * pab[u][c] * wv[u];
                        double* F = c == 0 ? F0 : F1;
                        F[ab[u]] = v;
                        F[ba[u]] = v;
                    }
                }
            }
        }
    }
    // J_A: the lane-parallel sums reduced over the warp
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        double v = jl[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        jl[k] = v;
    }
    if (lane == 0) {  // s_q is free after the heavy-heavy loop
#pragma unroll
        for (int k = 0; k < 10; ++k) s_q[warp][k] = jl[k];
    }
    __syncwarp();
    if (lane < npA) s_j[warp][lane] = s_q[warp][lane];
    __syncwarp();
    // one-centre terms and the diagonal block
    if (lane < 16) {
        const int mu = lane >> 2, nu = lane & 3;
        if (mu < naA && nu < naA) {
            const DevElem& e = params[md.method * (MAX_Z + 1) + atom_z[a]];
            for (int c = 0; c < md.nch; ++c) {
                const double* Pc = c == 0 ? P0 : P1;
                double acc = 0.0;
                for (int la = 0; la < naA; ++la)
                    for (int sg = 0; sg < naA; ++sg) {
                        const long long idx = (long long)(oA + la) * n + oA + sg;
                        acc += ptot(idx) * oc_integral(mu, nu, la, sg, e);
                        acc -= sc * Pc[idx] * oc_integral(mu, la, nu, sg, e);
                    }
                const long long d = (long long)(oA + mu) * n + oA + nu;
                double* F = c == 0 ? F0 : F1;
                F[d] = H0[d] + acc + s_j[warp][pack2(mu, nu)];
            }
        }
    }
}

}  // namespace am1
