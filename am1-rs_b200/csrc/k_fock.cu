// Fock G(P) build: F^s = H_core + J(P_tot) - K(spin_scale * P^s), am1-rs src/fock.rs:249-511.
//
// One warp per atom A.  The warp walks every partner B of its molecule in order and
//   * accumulates the Coulomb term of A's diagonal block, J_A = sum_B (A A | B B) . P_BB
//     (the reference's ja/jb, src/fock.rs:427-448) in registers -- a gather, so the sum is
//     deterministic and needs no atomics;
//   * for B > A (A is then the pair's first, heavier atom) computes the exchange block
//     K_AB = -s sum P^s_ab (mu nu | lambda sigma) (src/fock.rs:449-466) for every spin channel
//     and writes F_AB = H_AB + K_AB into both triangles; each off-diagonal block has exactly one
//     writer.
// Each pair's integral block is staged through shared memory once per visit with coalesced
// loads; lanes 0..15 own the 16 exchange outputs, lanes 16..25 the 10 Coulomb outputs.
// The one-centre terms (oc_two_electron, src/fock.rs:27-65 and 321-344) finish the diagonal.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

__device__ __forceinline__ int pack2(int a, int b) {
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

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

__global__ void __launch_bounds__(32 * FOCK_WARPS) k_fock(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol,
                                                         int natoms_total, const DevElem* __restrict__ params,
                                                         const int* __restrict__ atom_z, const double* __restrict__ wstore,
                                                         double* __restrict__ arena, const MolState* __restrict__ st, int force) {
    __shared__ double s_w[FOCK_WARPS][100];
    __shared__ double s_q[FOCK_WARPS][10];
    __shared__ double s_pab[FOCK_WARPS][2][16];
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
    const double sc = md.spin_scale;
    const long long xxsz = 100LL * h * (h - 1) / 2, xhsz = 10LL * h * Hn;
    const double* w = wstore + md.w_base;
    const bool aheavy = A < h;
    const int oA = aheavy ? 4 * A : 4 * h + (A - h);
    const int naA = aheavy ? 4 : 1;
    const int npA = aheavy ? 10 : 1;
    double* wb = s_w[warp];
    double jacc = 0.0;  // lane 16 + k owns J_A[k]

    auto ptot = [&](long long idx) { return P1 ? P0[idx] + P1[idx] : P0[idx]; };

    for (int B = 0; B < N; ++B) {
        if (B == A) continue;
        const bool bheavy = B < h;
        const int oB = bheavy ? 4 * B : 4 * h + (B - h);
        const int naB = bheavy ? 4 : 1, npB = bheavy ? 10 : 1;
        const int i = min(A, B), j = max(A, B);
        const double* blk;
        int sz;
        if (j < h) {
            blk = w + 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
            sz = 100;
        } else if (i < h) {
            blk = w + xxsz + 10LL * ((long long)i * Hn + (j - h));
            sz = 10;
        } else {
            const int i2 = i - h, j2 = j - h;
            blk = w + xxsz + xhsz + ((long long)i2 * Hn - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1));
            sz = 1;
        }
        for (int l = lane; l < sz; l += 32) wb[l] = blk[l];
        if (lane < npB) {
            // packed P_BB with the off-diagonal pairs counted twice
            int hi = 0;
            while ((hi + 1) * (hi + 2) / 2 <= lane) ++hi;
            const int lo = lane - hi * (hi + 1) / 2;
            const double v = ptot((long long)(oB + hi) * n + oB + lo);
            s_q[warp][lane] = hi == lo ? v : 2.0 * v;
        }
        const bool do_k = B > A;
        if (do_k && lane < 16) {
            const int nu = lane >> 2, sg = lane & 3;
            if (nu < naA && sg < naB) {
                const long long idx = (long long)(oA + nu) * n + oB + sg;
                s_pab[warp][0][lane] = P0[idx];
                if (P1) s_pab[warp][1][lane] = P1[idx];
            }
        }
        __syncwarp();
        // Coulomb: the A-side of the block is its rows when A is the first atom, else its columns
        if (lane >= 16 && lane < 16 + npA) {
            const int k = lane - 16;
            double acc = 0.0;
            if (A == i) {
                for (int q = 0; q < npB; ++q) acc += wb[k * npB + q] * s_q[warp][q];
            } else {
                for (int q = 0; q < npB; ++q) acc += wb[q * npA + k] * s_q[warp][q];
            }
            jacc += acc;
        }
        // Exchange block (A = first atom, B = second)
        if (do_k && lane < 16) {
            const int mu = lane >> 2, la = lane & 3;
            if (mu < naA && la < naB) {
                const int ncol = npB;
                for (int c = 0; c < md.nch; ++c) {
                    double acc = 0.0;
                    for (int nu = 0; nu < naA; ++nu) {
                        const double* row = wb + pack2(mu, nu) * ncol;
                        for (int sg = 0; sg < naB; ++sg) acc += s_pab[warp][c][nu * 4 + sg] * row[pack2(la, sg)];
                    }
                    const double kval = -(acc * sc);
                    double* F = arena + md.ch_base[c] + SLOT_F * nn;
                    const long long ab = (long long)(oA + mu) * n + oB + la;
                    const long long ba = (long long)(oB + la) * n + oA + mu;
                    const double v = H0[ab] + kval;
                    F[ab] = v;
                    F[ba] = v;
                }
            }
        }
        __syncwarp();
    }
    if (lane >= 16 && lane < 16 + npA) s_j[warp][lane - 16] = jacc;
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
                double* F = arena + md.ch_base[c] + SLOT_F * nn;
                F[d] = H0[d] + acc + s_j[warp][pack2(mu, nu)];
            }
        }
    }
}

}  // namespace am1
