// Two-centre integrals, overlap, core Hamiltonian and core-core energy kernels.
//
// One thread per atom pair: each pair's work is a fixed, branch-uniform sequence of FP64
// transcendental evaluations (about 70 reciprocal square roots for a heavy-heavy pair plus the
// Slater overlap's exponentials), so a thread per pair keeps all 32 lanes of a warp on the FP64
// pipe; the warp's pairs are consecutive pairs of one molecule, so their coordinates and
// parameters are read from the same few cache lines.
//
// The formulas (integrals_t.cuh) follow am1-rs; here also:
//   resonance              src/hamiltonian.rs:340-352  H_ab = (beta_a + beta_b)/2 * S_ab
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "integrals_t.cuh"
#include "kernels.h"

namespace am1 {

// Locate the molecule and the (i, j) pair of a flat pair index.
__device__ __forceinline__ int find_mol(const long long* __restrict__ prefix, int nmol, long long g) {
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void pair_ij(long long p, int n, int& i, int& j) {
    // rows i hold n-1-i pairs; S(i) = i*n - i(i+1)/2 pairs precede row i
    const double nn = n - 0.5;
    int ii = (int)floor(nn - sqrt(fmax(nn * nn - 2.0 * (double)p, 0.0)));
    ii = max(0, min(ii, n - 2));
    while (ii > 0 && (long long)ii * n - (long long)ii * (ii + 1) / 2 > p) --ii;
    while ((long long)(ii + 1) * n - (long long)(ii + 1) * (ii + 2) / 2 <= p) ++ii;
    i = ii;
    j = (int)(p - ((long long)ii * n - (long long)ii * (ii + 1) / 2)) + ii + 1;
}

__global__ void k_pair_integrals(const MolDesc* __restrict__ mols, int nmol, const long long* __restrict__ pair_prefix,
                                 long long npairs, const DevElem* __restrict__ params, const int* __restrict__ atom_z,
                                 const double* __restrict__ atom_xyz, double* __restrict__ wstore, double* __restrict__ hmat,
                                 double* __restrict__ ecc, int* __restrict__ mol_status) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npairs) return;
    const int m = find_mol(pair_prefix, nmol, g);
    const MolDesc md = mols[m];
    const long long p = g - pair_prefix[m];
    int i, j;
    pair_ij(p, md.natoms, i, j);
    const int ai = md.atom_base + i, aj = md.atom_base + j;
    const int zi = atom_z[ai], zj = atom_z[aj];
    const DevElem& ei = params[md.method * (MAX_Z + 1) + zi];
    const DevElem& ej = params[md.method * (MAX_Z + 1) + zj];
    const double d0 = atom_xyz[3 * aj] - atom_xyz[3 * ai];
    const double d1 = atom_xyz[3 * aj + 1] - atom_xyz[3 * ai + 1];
    const double d2 = atom_xyz[3 * aj + 2] - atom_xyz[3 * ai + 2];
    const double r0 = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    // core-core uses the plain distance (src/repulsion.rs:38-56)
    ecc[md.pair_base + p] = pair_core_energy(ei, ej, zi, zj, r0);
    // integrals see delta/r * r (src/hamiltonian.rs:296-298 -> src/integrals.rs:196-200)
    const double x0 = d0 / r0, x1 = d1 / r0, x2 = d2 / r0;
    const double dv[3] = {x0 * r0, x1 * r0, x2 * r0};
    const double r = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    const int h = md.nheavy, H = md.natoms - md.nheavy;
    long long off;
    if (j < h) {
        off = 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
    } else if (i < h) {
        off = 100LL * h * (h - 1) / 2 + 10LL * ((long long)i * H + (j - h));
    } else {
        const int i2 = i - h, j2 = j - h;
        off = 100LL * h * (h - 1) / 2 + 10LL * h * H + ((long long)i2 * H - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1));
    }
    pair_integrals(ei, ej, dv, r, wstore + md.w_base + off);
    // resonance block: overlap between the positions pos_i and pos_i + delta
    double S[4][4];
    const double pb0 = atom_xyz[3 * ai] + d0, pb1 = atom_xyz[3 * ai + 1] + d1, pb2 = atom_xyz[3 * ai + 2] + d2;
    const double e0 = pb0 - atom_xyz[3 * ai], e1 = pb1 - atom_xyz[3 * ai + 1], e2 = pb2 - atom_xyz[3 * ai + 2];
    const double rs = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    if (rs < 1.0e-8) {
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) S[a][b] = a == b ? 1.0 : 0.0;
    } else {
        const double dir[3] = {e0 / rs, e1 / rs, e2 / rs};
        if (!overlap_block(ei, ej, rs, dir, S)) {
            atomicExch(&mol_status[m], 6);  // AM1GPU_UNSUPPORTED
            return;
        }
    }
    const int na = ei.norb, nb = ej.norb, n = md.nao;
    const int oa = i < h ? 4 * i : 4 * h + (i - h);
    const int ob = j < h ? 4 * j : 4 * h + (j - h);
    double* H0 = hmat + md.h_base;
    for (int a = 0; a < na; ++a) {
        const double ba = a == 0 ? ei.beta_s : ei.beta_p;
        for (int b = 0; b < nb; ++b) {
            const double bb = b == 0 ? ej.beta_s : ej.beta_p;
            const double v = 0.5 * (ba + bb) * S[a][b];
            H0[(long long)(oa + a) * n + ob + b] = v;
            H0[(long long)(ob + b) * n + oa + a] = v;
        }
    }
}

// H_core diagonal blocks: U_ss/U_pp plus the electron-core attraction of every other atom,
// -Z_B (mu nu | s_B s_B), gathered per atom in partner order (deterministic).
__global__ void k_core_diag(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol, int natoms_total,
                            const DevElem* __restrict__ params, const int* __restrict__ atom_z, const double* __restrict__ wstore,
                            double* __restrict__ hmat) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms_total) return;
    const int m = atom_mol[a];
    const MolDesc md = mols[m];
    const int A = a - md.atom_base, N = md.natoms, h = md.nheavy, H = N - h;
    const DevElem& eA = params[md.method * (MAX_Z + 1) + atom_z[a]];
    const double* w = wstore + md.w_base;
    const long long xxsz = 100LL * h * (h - 1) / 2, xhsz = 10LL * h * H;
    double acc[10];
    for (int k = 0; k < 10; ++k) acc[k] = 0.0;
    const bool heavy = A < h;
    for (int B = 0; B < N; ++B) {
        if (B == A) continue;
        const double zb = -params[md.method * (MAX_Z + 1) + atom_z[md.atom_base + B]].core_charge;
        const bool bheavy = B < h;
        if (heavy && bheavy) {
            const int i = min(A, B), j = max(A, B);
            const double* blk = w + 100LL * ((long long)i * h - (long long)i * (i + 1) / 2 + (j - i - 1));
            if (A == i)
                for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k * 10];  // column 0: (A A| s_B s_B)
            else
                for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k];       // row 0
        } else if (heavy) {  // A heavy, B hydrogen
            const double* blk = w + xxsz + 10LL * ((long long)A * H + (B - h));
            for (int k = 0; k < 10; ++k) acc[k] += zb * blk[k];
        } else if (bheavy) {  // A hydrogen, B heavy
            acc[0] += zb * w[xxsz + 10LL * ((long long)B * H + (A - h))];
        } else {
            const int i2 = min(A, B) - h, j2 = max(A, B) - h;
            acc[0] += zb * w[xxsz + xhsz + ((long long)i2 * H - (long long)i2 * (i2 + 1) / 2 + (j2 - i2 - 1))];
        }
    }
    const int n = md.nao;
    double* H0 = hmat + md.h_base;
    if (heavy) {
        const int o = 4 * A;
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu) {
                const int hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
                double v = acc[hi * (hi + 1) / 2 + lo];
                if (mu == nu) v += mu == 0 ? eA.u_ss : eA.u_pp;
                H0[(long long)(o + mu) * n + o + nu] = v;
            }
    } else {
        const int o = 4 * h + (A - h);
        H0[(long long)o * n + o] = eA.u_ss + acc[0];
    }
}

// Per-molecule sum of the core-core pair energies, in pair order (one block per molecule).
__global__ void k_core_energy(const MolDesc* __restrict__ mols, const double* __restrict__ ecc, MolState* __restrict__ st) {
    const int m = blockIdx.x;
    const MolDesc md = mols[m];
    const long long np = (long long)md.natoms * (md.natoms - 1) / 2;
    __shared__ double part[256];
    double s = 0.0;
    for (long long p = threadIdx.x; p < np; p += blockDim.x) s += ecc[md.pair_base + p];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) st[m].core_ev = part[0];
}

}  // namespace am1
