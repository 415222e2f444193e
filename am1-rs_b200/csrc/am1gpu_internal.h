// Internal declarations shared by the host driver and the CUDA kernels of libam1gpu.
//
// Device data layout (one "batch" = any number of molecules solved together):
//   * atoms of every molecule are stored in an internal order, heavy (s,p) atoms first and
//     hydrogens after, each group in input order.  The pair (i, j), i < j, then always has its
//     heavy atom first, which is the orientation the reference uses (src/hamiltonian.rs:289-294),
//     and a molecule's pairs fall into three contiguous classes:
//       XX (both heavy) -> 100 two-electron integrals, 10x10 packed bra x ket
//       XH              -> 10 integrals (heavy bra pair x (ss| of the hydrogen)
//       HH              -> 1 integral
//     so the integral store of a molecule is [XX | XH | HH] with closed-form offsets.
//   * AOs follow the internal atom order: heavy atom i owns AOs 4i..4i+3 (s, px, py, pz),
//     hydrogen j >= h owns AO 4h + (j - h).  Results are permuted back to the caller's order.
//   * every n x n matrix is dense row-major with leading dimension n, FP64.
#pragma once

#include <cstdint>
#include <string>

#ifdef __CUDACC__
#define AM1_HD __host__ __device__
#else
#define AM1_HD
#endif

namespace am1 {

constexpr double AM1_EV = 27.21;          // src/constants.rs:13
constexpr double AM1_A0 = 0.529167;       // src/constants.rs:15
constexpr double EV_TO_KCAL = 23.061;     // src/constants.rs:24
constexpr double AU_DIPOLE_TO_DEBYE = 2.541746473;  // src/constants.rs:32
constexpr int MAX_DIIS = 8;               // src/scf.rs:579
constexpr int MAX_Z = 86;

// Derived per-element parameters (Am1Element, src/params.rs:24-55), as the kernels read them.
struct DevElem {
    int present, n, norb, ngauss;
    double u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p;
    double g_ss, g_sp, g_pp, g_p2, h_sp, alpha;
    double gk[4], gl[4], gm[4];
    double core_charge, eheat_ev, e_isol, dd, qq, rho0, rho1, rho2;
};

// One molecule of a batch.
struct MolDesc {
    int natoms, nheavy, nao, nch;   // nch: 1 = RHF, 2 = UHF (alpha, beta)
    int n_occ[2];                   // occupied orbitals per channel
    int method;                     // 0 AM1, 1 RM1
    int atom_base;                  // first atom in the batch atom arrays
    long long pair_base;            // first pair in the batch pair arrays (i<j, internal order)
    long long w_base;               // first double of the molecule's integral store
    long long h_base;               // H_core matrix (n*n)
    long long ch_base[2];           // per channel: base of its matrix slots (see ChSlot)
    long long pk_base[2];           // per channel: base of its packed DIIS history
    double spin_scale;              // exchange weight of the channel density: 0.5 RHF, 1 UHF
    double occ_weight;              // density weight: 2 RHF, 1 UHF
};

// Matrix slots of one channel, each n*n doubles, at ch_base + slot*n*n (VS holds npad*n).
enum ChSlot { SLOT_F = 0, SLOT_FX = 1, SLOT_P = 2, SLOT_CT = 3, SLOT_GT = 4, SLOT_VS = 5, NUM_SLOTS = 6 };

// Packed history of one channel: MAX_DIIS entries each of F (n(n+1)/2), E (n(n-1)/2) and,
// for A-DIIS, D (n(n+1)/2); laid out [F x8][E x8][D x8].
AM1_HD inline long long packed_sym_len(int n) { return (long long)n * (n + 1) / 2; }
AM1_HD inline long long packed_anti_len(int n) { return (long long)n * (n - 1) / 2; }

// Per-molecule SCF state kept on the device across iterations.
struct MolState {
    int active;        // 1 while iterating
    int iter;          // iterations done
    int converged;
    int status;        // am1gpu_status code
    int hist_count;    // entries in the DIIS history (<= MAX_DIIS)
    int hist_head;     // physical slot of the oldest entry
    int mode;          // extrapolation of this iteration: 0 plain F, 1 combine history
    int accel_used;    // 0 none, 1 CDIIS, 2 ADIIS (diagnostic)
    int lowp;          // mixed precision: 1 while this molecule's purification runs in TF32
    int lowp_end;      // iteration at which the TF32 phase ended (convergence is tested only after it)
    int lowp_flush;    // 1 in the first FP64 iteration: its history entry still holds the TF32 density
    double e_old, e_elec, err_norm, dp, residual;
    double coeff[MAX_DIIS];            // combination coefficients in logical order
    double bmat[MAX_DIIS * MAX_DIIS];  // CDIIS Gram <e_i, e_j>, logical order
    double gmat[MAX_DIIS * MAX_DIIS];  // A-DIIS Gram <D_i, F_j>, logical order
    double e_final, core_ev;
};

// Reduction outputs of the post-Fock pass: per channel and per block.
constexpr int RED_E_H = 0;            // sum P.H
constexpr int RED_E_F = 1;            // sum P.F
constexpr int RED_ERR2 = 2;           // sum e^2 (full matrix)
constexpr int RED_B = 3;              // 8 entries: <e_new, e_j> (packed, x2 applied later)
constexpr int RED_GROW = 11;          // 8 entries: <D_new, F_j>
constexpr int RED_GCOL = 19;          // 8 entries: <D_i, F_new>
constexpr int RED_N = 27;

// Message returned by am1gpu_last_error for the calling host thread.
void set_last_error(const std::string& msg);

}  // namespace am1
