// Closed-form nuclear gradient of the NDDO energy at a fixed (converged) density: the
// Hellmann-Feynman gradient of am1-rs's closed_form_gradient (src/gradient.rs:173-253), i.e.
// fixed_density_gradient (src/gradient.rs:317-334) = the core-core gradient
// (src/repulsion.rs:81-115) + the electronic pair gradient (src/gradient.rs:366-493).
//
// Every term of the energy is a sum over atom pairs of a function of the pair displacement
// delta = x_b - x_a, so each pair contributes f = dE_pair/d(delta) to atom b and -f to atom a:
//   core-core        dE_cc(r)/d(delta)
//   resonance        sum_{mu in a, la in b} P_{mu la} (beta_mu + beta_la) dS_{mu la}
//   electron-core    sum_{mu nu in a} P_{mu nu} de1b_{mu nu} + sum_{la si in b} P_{la si} de2a_{la si}
//   two-electron     sum_{mu nu in a, la si in b} [P_{mu nu} P_{la si}
//                         - (Pa_{mu la} Pa_{nu si} + Pb_{mu la} Pb_{nu si})] d(mu nu|la si)
// with P the total density and Pa, Pb the spin densities (RHF: Pa = Pb = P/2, which gives the
// reference's -1/2 P_{mu la} P_{nu si}).  The derivatives are exact: the integral, overlap and
// core-core templates of integrals_t.cuh run on D3 dual numbers carrying d/d(delta).
//
// A warp per atom walks its partners, a pair per lane; each pair is evaluated for both of its
// atoms (twice in all) so that every atom's sum is a fixed-order warp reduction: deterministic,
// no atomics and no per-pair scratch.  The two-centre integrals are contracted as they are formed
// (pair_integrals_each), so no block of 100 dual numbers is held per thread.
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "integrals_t.cuh"
#include "kernels.h"

namespace am1 {

// dE_pair/d(delta) of the pair (a, b) at fixed densities; false for an element without the
// closed-form overlap (valence shell n >= 4).  Pa: channel-0 density (RHF: total), Pb: channel 1
// or nullptr (RHF), both n x n in the internal AO order; oa, ob: first AO of a and b.
__device__ bool pair_force(const DevElem& ea, const DevElem& eb, int za, int zb, const double dl[3], const double* __restrict__ Pa,
                           const double* __restrict__ Pb, int n, int oa, int ob, double f[3]) {
    const D3 dv[3] = {D3{dl[0], {1.0, 0.0, 0.0}}, D3{dl[1], {0.0, 1.0, 0.0}}, D3{dl[2], {0.0, 0.0, 1.0}}};
    const D3 r = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    f[0] = f[1] = f[2] = 0.0;
    if (r.v < 1.0e-8) return true;  // coincident atoms: no direction, nothing to differentiate
    auto acc = [&](double c, const D3& x) {
        f[0] += c * x.d[0];
        f[1] += c * x.d[1];
        f[2] += c * x.d[2];
    };
    auto pt = [&](int r0, int c0) { return Pb ? Pa[(long long)r0 * n + c0] + Pb[(long long)r0 * n + c0] : Pa[(long long)r0 * n + c0]; };
    // exchange weight Pa Pa + Pb Pb (RHF: 2 (P/2)(P/2))
    auto px = [&](int r1, int c1, int r2, int c2) {
        const double x = Pa[(long long)r1 * n + c1] * Pa[(long long)r2 * n + c2];
        return Pb ? x + Pb[(long long)r1 * n + c1] * Pb[(long long)r2 * n + c2] : 0.5 * x;
    };
    // core-core (src/repulsion.rs:81-115)
    acc(1.0, pair_core_energy(ea, eb, za, zb, r));
    // resonance: H_{mu la} = (beta_mu + beta_la)/2 S_{mu la} in both triangles (src/gradient.rs:424-433)
    const D3 dir[3] = {dv[0] / r, dv[1] / r, dv[2] / r};
    D3 S[4][4];
    if (!overlap_block(ea, eb, r, dir, S)) return false;
    const int na = ea.norb, nb = eb.norb;
    for (int i = 0; i < na; ++i) {
        const double bi = i == 0 ? ea.beta_s : ea.beta_p;
        for (int j = 0; j < nb; ++j) acc(pt(oa + i, ob + j) * (bi + (j == 0 ? eb.beta_s : eb.beta_p)), S[i][j]);
    }
    // two-centre integrals, contracted as they are formed (no integral block is stored): the
    // element (kk ll | mm nn), kk >= ll on a and mm >= nn on b, stands for every ordering of its
    // index pairs (src/gradient.rs:434-466 sums over all of them):
    //   electron-core  e1b = -Z_b (mu nu | s s) on a's block, e2a = -Z_a (s s | la si) on b's
    //   Coulomb        P_{mu nu} P_{la si}
    //   exchange       -(Pa_{mu la} Pa_{nu si} + Pb_{mu la} Pb_{nu si})
    pair_integrals_each(ea, eb, dv, r, [&](int kk, int ll, int mm, int nn, const D3& v) {
        const int ma = kk == ll ? 1 : 2, mb = mm == nn ? 1 : 2;
        const double pa = pt(oa + kk, oa + ll), pb = pt(ob + mm, ob + nn);
        double c = ma * mb * pa * pb;
        c -= px(oa + kk, ob + mm, oa + ll, ob + nn);
        if (ll != kk) c -= px(oa + ll, ob + mm, oa + kk, ob + nn);
        if (nn != mm) {
            c -= px(oa + kk, ob + nn, oa + ll, ob + mm);
            if (ll != kk) c -= px(oa + ll, ob + nn, oa + kk, ob + mm);
        }
        if (mm == 0) c -= eb.core_charge * ma * pa;  // (kk ll | s s)
        if (kk == 0) c -= ea.core_charge * mb * pb;  // (s s | mm nn)
        acc(c, v);
    });
    return true;
}

constexpr int GRAD_WARPS = 8;

// gradient[3 a + k] = dE/dx_{a,k} (eV/Bohr) for every atom of the batch, internal atom order.
__global__ void __launch_bounds__(32 * GRAD_WARPS) k_gradient(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol,
                                                              int natoms_total, const DevElem* __restrict__ params,
                                                              const int* __restrict__ atom_z, const double* __restrict__ atom_xyz,
                                                              const ChanJob* __restrict__ jobs, const int* __restrict__ mol_job0,
                                                              double* __restrict__ gradient, int* __restrict__ mol_status) {
    const int a = blockIdx.x * GRAD_WARPS + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= natoms_total) return;  // uniform over the warp
    const int m = atom_mol[a];
    const MolDesc md = mols[m];
    const int A = a - md.atom_base, N = md.natoms, h = md.nheavy, n = md.nao;
    const ChanJob& j0 = jobs[mol_job0[m]];
    const double* Pa = j0.P;
    const double* Pb = md.nch == 2 ? jobs[mol_job0[m] + 1].P : nullptr;
    const DevElem* tab = params + md.method * (MAX_Z + 1);
    double g[3] = {0.0, 0.0, 0.0};
    bool ok = true;
    for (int B = lane; B < N; B += 32) {
        if (B == A) continue;
        // the pair (i < j): heavy atoms come first in the internal order, so i is the heavy one
        // whenever the pair mixes a heavy atom and a hydrogen (src/gradient.rs:394-401)
        const int i = min(A, B), j = max(A, B);
        const int ai = md.atom_base + i, aj = md.atom_base + j;
        const int zi = atom_z[ai], zj = atom_z[aj];
        const double dl[3] = {atom_xyz[3 * aj] - atom_xyz[3 * ai], atom_xyz[3 * aj + 1] - atom_xyz[3 * ai + 1],
                              atom_xyz[3 * aj + 2] - atom_xyz[3 * ai + 2]};
        const int oi = i < h ? 4 * i : 4 * h + (i - h), oj = j < h ? 4 * j : 4 * h + (j - h);
        double f[3];
        ok &= pair_force(tab[zi], tab[zj], zi, zj, dl, Pa, Pb, n, oi, oj, f);
        const double sg = A == j ? 1.0 : -1.0;  // +f on the second atom of the pair, -f on the first
        g[0] += sg * f[0];
        g[1] += sg * f[1];
        g[2] += sg * f[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        g[0] += __shfl_xor_sync(0xffffffffu, g[0], o);
        g[1] += __shfl_xor_sync(0xffffffffu, g[1], o);
        g[2] += __shfl_xor_sync(0xffffffffu, g[2], o);
    }
    if (!ok) atomicExch(&mol_status[m], 6);  // AM1GPU_UNSUPPORTED (also refused by the SCF itself)
    if (lane == 0) {
        gradient[3LL * a] = g[0];
        gradient[3LL * a + 1] = g[1];
        gradient[3LL * a + 2] = g[2];
    }
}

}  // namespace am1
