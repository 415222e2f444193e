// Kernel interfaces of libam1gpu (device side), shared with the host driver.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "am1gpu_internal.h"

namespace am1 {

struct GemmJob {
    const double* A;
    const double* B;
    double* C;
    int M, N, K, lda, ldb, ldc;
    double alpha;
    int mol;
};

struct GemmTile {
    int job;
    int tm, tn;
};

// A tensor map (the driver's opaque 128-byte CUtensorMap, 64-byte aligned) as the kernels receive
// it: the device only passes its address to cp.async.bulk.tensor.
struct __align__(64) TmaDesc {
    unsigned long long w[16];
};

// One eigenproblem (a channel of a molecule).
struct EigJob {
    const double* Gt;      // C0^T F (rows = columns of F C0), n x n
    const double* Ct;      // warm start C0^T (rows = vectors), n x n
    double* Vs;            // npad x n: eigenvector rows in slot order (scratch)
    double* lam;           // npad: eigenvalues in slot order (scratch)
    int* colid_out;        // npad: column id per slot (scratch)
    double* eps;           // n: sorted eigenvalues (output)
    double* Ct_out;        // n x n: sorted eigenvector rows (output)
    const double* rowmin;  // n: Gershgorin row lower bounds of F
    int* sweeps_out;       // optional
    int n, npad, mol;
};

// One (molecule, channel) job of the element-wise SCF passes.
struct ChanJob {
    int mol, ch, n;
    double* F;
    double* Fx;       // the extrapolated Fock matrix F* (DIIS combination)
    double* P;
    double* Pnew;
    double* Ct;       // eigenvector rows (C^T), n x n
    double* eps;      // sorted eigenvalues, n
    const double* H;
    double* hF;       // packed history of F  [8][n(n+1)/2]
    double* hE;       // packed history of [F,P] [8][n(n-1)/2]
    double* hD;       // packed history of P  [8][n(n+1)/2] (A-DIIS) or nullptr
    double* rowmin;   // n: Gershgorin lower bound of each row of F*
    double* rowmax;   // n: Gershgorin upper bound
    double* rowdf;    // n: sum over the row of (F* - F* of the previous iteration)^2 (from the second iteration on)
    double* red;      // per-block partial sums [nblk][RED_N]
    double* red2;     // per-block partial sums of (P_new - P)^2 [nblk]
    double* cpart;    // per-tile partial sums of the commutator pass [ntiles][CP_N]
    int ntiles;       // upper-triangle 64x64 tiles of the channel
};

// Partial sums of k_commutator per tile: CP_ERR2 = sum of e^2 over the full matrix,
// CP_B + slot = <e_new, e_slot> over the strict upper triangle (slot = physical history slot).
constexpr int CP_ERR2 = 0, CP_B = 1, CP_N = 1 + MAX_DIIS;

// One purification problem (a channel of a molecule).
struct Sp2Job {
    const double* F;        // the extrapolated Fock matrix F*
    const double* rowmin;   // Gershgorin bounds of F*
    const double* rowmax;
    const double* rowdf;    // row sums of (F* - F*_previous)^2, or nullptr (always run the Lanczos bounds)
    double* X0;             // ping-pong iterates, n x n each
    double* X1;
    double* P;              // output density (w X), n x n (may alias X0)
    double* part;           // partial sums [max(nblk, ntiles)][2]
    double* bounds;         // [4] spectral interval of F* used for the mapping (k_sp2_bounds), the widening
                            // added since the last Lanczos run, the width of that run's interval
    double nocc, weight;
    int n, mol, tile0, ntiles;
    int fallback;           // 1: a stalled purification falls back to the eigensolver; 0: LINALG
    // mixed precision: the FP32 ping-pong iterates of the TF32 iterations, rows of ldf floats
    // (n rounded up to a multiple of 4; the pad columns hold zeros), 16-byte aligned
    float* Xf0;
    float* Xf1;
    int ldf;
    // the reduced-precision products: 1 on tcgen05 at FP32 accuracy (k_sp2_step_tc, 3xTF32, FP32
    // iterates), 2 on tcgen05 in one TF32 pass (k_sp2_step_tc1, TF32-rounded iterates), both on the
    // 128 x 128 tiles tc_tile0 .. tc_tile0 + tc_ntiles - 1 of their launch; 0 mma.sync TF32
    // (k_sp2_step_tf32, TF32-rounded iterates, the 64 x 64 tiles)
    int lowp_tc, tc_tile0, tc_ntiles;
    // 1: the FP64 products run on tcgen05's integer path from the iterate's 7-bit digit planes
    // (k_sp2_step_oz, 128 x 48 tiles oz_tile0 .. oz_tile0 + oz_ntiles - 1 of their launch); the digits of
    // X0 / X1 are kOzPlanes int8 planes of n rows of ldq bytes each (pad columns zero)
    int oz, oz_tile0, oz_ntiles, ldq;
    int8_t* Dq0;
    int8_t* Dq1;
};
constexpr int kOzPlanes = 8;  // 7-bit digits of an iterate: 2^-5 .. 2^-54
constexpr int kOzGroups = 9;  // digit-plane products kept: i + j <= 8

struct Sp2State {
    int active, steps, cur, square, converged;
    int lowp;  // this run's products are TF32 (the molecule's MolState::lowp when it started)
    double trX, trX2, emin, emax;
    double idem[2];
};

// One tridiagonalisation + bisection problem.
struct TriJob {
    const double* A;   // symmetric input, n x n
    double* W;         // large matrices only: working copy, n x n (global memory)
    double* work;      // large matrices only: scratch vectors, 4 n + grid + 4 doubles
    double* d;         // diagonal, n
    double* e;         // off-diagonal, n
    double* eps;       // ascending eigenvalues, n
    int n, mol;
    // k_tridiag on a cluster: 0 runs the reduction to the end; stop > 0 ends it after `stop`
    // reflectors and writes the trailing block (rows and columns >= stop, its last update applied)
    // row-major to W, n - stop rows of n - stop, which a one-CTA job (A = W, d and e from index
    // stop on) then reduces
    int stop;
};

// Loop counters of the captured solve (k_graph.cu), in device memory.
struct GraphLoop {
    int scf_iter;   // SCF iterations done in this launch
    int sp2_step;   // purification steps of the current iteration
    int sp2_total;  // purification steps of this launch
    int eig_runs;   // iterations of this launch in which the stalled-purification eigensolver ran
};
__global__ void k_scf_arm(cudaGraphConditionalHandle h, GraphLoop* loop, int max_scf);
__global__ void k_sp2_arm(cudaGraphConditionalHandle h, GraphLoop* loop, int* active_count);
__global__ void k_sp2_cond(cudaGraphConditionalHandle h, GraphLoop* loop, int* active_count, int max_steps);
__global__ void k_stall_arm(cudaGraphConditionalHandle h, GraphLoop* loop, const int* need_eigen, int nmol);
__global__ void k_scf_cond(cudaGraphConditionalHandle h, GraphLoop* loop, const int* active, int max_scf);

struct ScfParams {
    int max_scf, use_diis, accelerator;
    double e_tol, p_tol, adiis_switch;
    // mixed precision: a molecule leaves its TF32 phase once the RMS density change falls below
    // lowp_switch, or after lowp_max_iter iterations
    double lowp_switch;
    int lowp_max_iter;
};

__global__ void k_pair_integrals(const MolDesc* mols, int nmol, const long long* pair_prefix, long long npairs,
                                 const DevElem* params, const int* atom_z, const double* atom_xyz, double* wstore,
                                 double* hmat, double* ecc, int* mol_status);
__global__ void k_core_diag(const MolDesc* mols, const int* atom_mol, int natoms_total, const DevElem* params,
                            const int* atom_z, const double* wstore, double* hmat);
__global__ void k_core_energy(const MolDesc* mols, const double* ecc, MolState* st);
// nuclear gradient at the current densities (jobs[].P), a warp per atom (8 per block); gradient:
// 3 doubles per atom, internal atom order
__global__ void k_gradient(const MolDesc* mols, const int* atom_mol, int natoms_total, const DevElem* params, const int* atom_z,
                           const double* atom_xyz, const ChanJob* jobs, const int* mol_job0, double* gradient, int* mol_status);
__global__ void k_fock(const MolDesc* mols, const int* atom_mol, int natoms_total, const DevElem* params,
                       const int* atom_z, const double* wstore, double* arena, const MolState* st, int force);
// C = alpha A B (A row-major M x K) and C = alpha A^T B (A stored K x M)
// mask (optional): only molecules with mask[mol] != 0 take part
__global__ void k_gemm_nn(const GemmJob* jobs, const GemmTile* tiles, int ntiles, const MolState* st, int force, const int* mask);
__global__ void k_gemm_tn(const GemmJob* jobs, const GemmTile* tiles, int ntiles, const MolState* st, int force, const int* mask);
__global__ void k_jacobi(const EigJob* jobs, const MolState* st, int* mol_status, int force, const int* mask);
__global__ void k_eig_sort(const EigJob* jobs, const MolState* st, int force, const int* mask);
// one CTA of 512 threads per job, 3 n doubles of dynamic shared memory; jobs without an eigensolver
// fallback (large matrices) are left to k_sp2_bounds_big (one cooperative launch per matrix) or
// k_sp2_bounds_cl (a cluster per matrix, grid (C, count of big), blockIdx.y indexes big[])
__global__ void k_sp2_bounds(const Sp2Job* jobs, const MolState* st);
__global__ void k_sp2_bounds_big(const Sp2Job* jobs, int job, const MolState* st);
__global__ void k_sp2_bounds_cl(const Sp2Job* jobs, const int* big, const MolState* st);
// Blocks of a channel's row reductions (post-Fock pass and density difference: red_blocks; the
// purification start: sp2_init_blocks).  They depend on the channel's own n only, so a molecule's
// sums are the same whatever else is in its batch; a launch's x extent is the batch's largest
// count, and the blocks past a channel's own count leave at once.
__host__ __device__ __forceinline__ int red_blocks(int n) { return n >= 497 ? 32 : (n + 15) / 16 < 1 ? 1 : (n + 15) / 16; }
__host__ __device__ __forceinline__ int sp2_init_blocks(int n) { return n >= 249 ? 32 : (n + 7) / 8 < 1 ? 1 : (n + 7) / 8; }
__global__ void k_sp2_init(const Sp2Job* jobs, Sp2State* sst, const MolState* st, int nblk);
__global__ void k_sp2_start(const Sp2Job* jobs, Sp2State* sst, const MolState* st, int njobs, int nblk);
// *16: every matrix of the tile list has even n and 16-byte aligned rows (16-byte copies);
// *8: any matrix (8-byte copies)
__global__ void k_sp2_step16(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst);
__global__ void k_sp2_step8(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst);
// the *16 tiles with the operands copied by the tensor memory accelerator: maps[4 job + i] is the
// tensor map of job's X_i, maps[4 job + 2] and [4 job + 3] those of the channel's F and P (n x n
// FP64, box 16 x 64, 128-byte swizzle); dgemm_tma_smem_bytes() of dynamic shared memory; a copy
// wait that runs out sets bit 11 of *err
__global__ void k_sp2_step_tma(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst, const TmaDesc* maps,
                               int* err);
size_t dgemm_tma_smem_bytes();
// the TF32 step of the mixed path's reduced-precision iterations (jobs with Sp2State::lowp);
// tf32_smem_bytes() of dynamic shared memory, same tile lists
__global__ void k_sp2_step_tf32(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst);
size_t tf32_smem_bytes();
// E = F.P - P.F over the upper-triangle tiles: history push of E and its CDIIS Gram row
__global__ void k_commutator16(const ChanJob* jobs, const GemmTile* tiles, int ntiles, const MolState* st);
__global__ void k_commutator8(const ChanJob* jobs, const GemmTile* tiles, int ntiles, const MolState* st);
// the *16 tiles from the tensor maps of F and P (maps[4 job + 2], [4 job + 3]); dgemm_tma_smem_bytes()
__global__ void k_commutator_tma(const ChanJob* jobs, const GemmTile* tiles, int ntiles, const MolState* st, const TmaDesc* maps,
                                 int* err);
size_t dgemm_smem_bytes();
__global__ void k_sp2_update(const Sp2Job* jobs, Sp2State* sst, int njobs, int max_steps, int* active_count, double* work);
constexpr int SP2_UPDATE_ONE = 1024;  // channels k_sp2_update_cond takes in its one CTA
__global__ void k_sp2_update_cond(const Sp2Job* jobs, Sp2State* sst, int njobs, int max_steps, double* work, cudaGraphConditionalHandle h,
                                  GraphLoop* loop);
size_t tc_smem_bytes();
size_t tc1_smem_bytes();
size_t oz_smem_bytes();
__global__ void k_sp2_step_oz(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst, int* err);
// The eight 7-bit digits of y (|y| < 2) packed one per byte, digit i in byte i: d_i = rint(r_i 2^(5+7i)),
// r_{i+1} = r_i - d_i 2^-(5+7i), every step exact (powers of two, no division).
__device__ __forceinline__ unsigned long long oz_digits_packed(double y) {
    double r = y;
    unsigned long long packed = 0;
#pragma unroll
    for (int i = 0; i < kOzPlanes; ++i) {
        const double sc = __longlong_as_double((long long)(1023 + 5 + 7 * i) << 52);    // 2^(5+7i)
        const double isc = __longlong_as_double((long long)(1023 - 5 - 7 * i) << 52);   // 2^-(5+7i)
        const double d = rint(r * sc);
        r = fma(-d, isc, r);
        packed |= (unsigned long long)(unsigned char)(signed char)(int)d << (8 * i);
    }
    return packed;
}
__device__ __forceinline__ void oz_store_digits(unsigned long long packed, int8_t* __restrict__ D, long long plane, long long o) {
#pragma unroll
    for (int i = 0; i < kOzPlanes; ++i) D[i * plane + o] = (int8_t)(packed >> (8 * i));
}
__device__ __forceinline__ void oz_digits_of(double y, int8_t* __restrict__ D, long long plane, long long o) {
    oz_store_digits(oz_digits_packed(y), D, plane, o);
}
__global__ void k_sp2_step_tc(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst, int* err);
// maps[2 job + i]: the tensor map of job's Xf_i (ldf x n FP32, box 32 x 128, 128-byte swizzle)
__global__ void k_sp2_step_tc1(const Sp2Job* jobs, const GemmTile* tiles, int ntiles, const Sp2State* sst, const TmaDesc* maps,
                               int* err);
__global__ void k_sp2_finish(const Sp2Job* jobs, const Sp2State* sst, const MolState* st, int* need_eigen, double* work,
                             int* big_stall, int* big_count);
// launched in clusters of C CTAs (one cluster per job), tridiag_smem_bytes(n, C) each
__global__ void k_tridiag(const TriJob* jobs, const int* mask);
size_t tridiag_smem_bytes(int n, int C);
// lanes = 1: a thread per eigenvalue, blockIdx.y the block of blockDim eigenvalue indices; lanes =
// 32: a warp per eigenvalue, blockIdx.y the block of blockDim / 32 indices (bisect_launch sizes both)
__global__ void k_bisect(const TriJob* jobs, const int* mask, int lanes);
// matrices too large for a cluster's shared memory, the matrix in global memory: one cooperative
// launch over the whole GPU (grid <= co-resident CTAs of TRIB_THREADS threads), or a cluster of
// C CTAs per matrix (grid (C, count), blockIdx.y indexes jobs); tridiag_big_smem_bytes(largest n)
// of dynamic shared memory
constexpr int TRIB_THREADS = 512;
__global__ void k_tridiag_big(TriJob job);
__global__ void k_tridiag_cl(const TriJob* jobs);
size_t tridiag_big_smem_bytes(int n);
// blocked reduction of one large matrix (job.W, a copy of job.A): for each panel of TRP_B columns
// starting at k (bw columns; the last panel ends at column n - 2), one cooperative launch of
// k_tridiag_panel (tridiag_panel_smem_bytes(n); grid <= co-resident CTAs and >= n / 64), then,
// unless it was the last panel, the trailing update over the upper tiles of [k + TRP_B, n)
// (k_tridiag_syr2k16 when n is even, else ...8; dgemm_smem_bytes()).  job.work: 16-byte aligned,
// 4 TRP_B n + 2 n + grid (2 TRP_B + 2) doubles.
constexpr int TRP_B = 32;
__global__ void k_tridiag_panel(TriJob job, int k, int bw);
__global__ void k_tridiag_syr2k16(TriJob job, int t0);
__global__ void k_tridiag_syr2k8(TriJob job, int t0);
size_t tridiag_panel_smem_bytes(int n);
size_t jacobi_smem_bytes(int n, int npad, int C);

// Eigenvectors of one large matrix (k_stein.cu): after the global-memory reduction (reflector s
// in row s of W, columns > s) and k_bisect.  Inverse iteration on T: k_stein_prep (one block of
// 1024), then four times k_stein_solve (grid ceil(n / 64) x 64, first = 1 the first time, last = 1
// the fourth, which tests each vector's growth: bit 4 of counts[1] if it falls short) and
// k_stein_orth (grid max(1, n / 2) x 256, n doubles of dynamic shared memory), then k_stein_scale.
// Z[i * n + k] = component i of eigenvector k.
constexpr double kSteinOrtol = 1e-4;  // eigenvalues closer than this times ||T|| share a cluster
struct SteinJob {
    const double* d;    // tridiagonal: diagonal (n), off-diagonal (n - 1)
    const double* e;
    const double* eps;  // its eigenvalues, ascending
    double* shift;      // n: the solve's shift of each vector
    int* cl;            // n: first vector of each vector's cluster
    int* cl_list;       // n / 2: first vector of every cluster of two or more
    int* counts;        // [0]: clusters of two or more; [1]: error bits (a vector of zero or non-finite norm)
    double* scale;      // n: pending 1 / norm of each vector
    double* tn;         // [2]: ||T||_inf and the pivot floor eps ||T||
    double* Z;          // n x n
    double* U;          // 3 n x n: the three diagonals of the pivoted factor (same layout as Z)
    double* Zt;         // n x n scratch: the vectors of the clusters, vector-major
    int n;
};
__global__ void k_stein_prep(SteinJob sj);
__global__ void k_stein_solve(SteinJob sj, int first, int last);
__global__ void k_stein_orth(SteinJob sj);
__global__ void k_stein_scale(SteinJob sj);
// A[r][c] = A[c][r] for r < c; block (32, 8), grid (ceil(n / 32), ceil(n / 32))
__global__ void k_mirror_lower(double* A, int n);
// Zt[k][i] = Z[i][k] for k < m (Z n x n row-major, Zt m x n); block (32, 8), grid (ceil(n/32), ceil(m/32)).
__global__ void k_transpose_cols(const double* Z, int n, int m, double* Zt);
// P = w (P + P^T) / 2 in place (n x n); block (32, 8), grid (ceil(n/32), ceil(n/32)).
__global__ void k_sym_scale(double* P, int n, double w);
// Back-transformation in compact WY blocks of kWyNb reflectors (nref = n - 2 reflectors, P =
// nref rounded up to kWyNb): k_wy_split (block (32, 8), grid (ceil(n / 32), P / 32)) gives Vt
// (P x n) and V = Vt^T (n x P); S_b = Vt_b V_b by k_dgemm; k_wy_tfactor (grid P / kWyNb, kWyNb
// threads) gives T_b; U_b = T_b Vt_b by k_dgemm; then per block, last first, Y = U_b Z and Z -= V_b Y.
constexpr int kWyNb = 64;
__global__ void k_wy_split(const double* W, int n, int nref, int P, double* Vt, double* V);
__global__ void k_wy_tfactor(const double* Sg, const double* W, const double* e, int n, int nref, double* Tg);
// C_z = A_z B_z (sub = 0) or C_z -= A_z B_z (sub = 1), z = blockIdx.z, operands advanced by the
// strides; grid (ceil(N / 64), ceil(M / 64), batch), 128 threads, dgemm_smem_bytes().  k_dgemm16:
// 16-byte aligned A and B, even lda, ldb, K and N.
__global__ void k_dgemm16(const double* A, int lda, long long sA, const double* B, int ldb, long long sB, double* C, int ldc,
                          long long sC, int M, int N, int K, int sub);
__global__ void k_dgemm8(const double* A, int lda, long long sA, const double* B, int ldb, long long sB, double* C, int ldc,
                         long long sC, int M, int N, int K, int sub);

#ifdef __CUDACC__
// FP32 -> nearest TF32 value (ties away from zero), kept in an FP32 register
__device__ __forceinline__ float tf32_round(float x) {
    unsigned u;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(u) : "f"(x));
    return __uint_as_float(u);
}

// Sum of the G per-CTA shares of a multi-CTA reduction, the same in every warp of every CTA: lane
// l adds shares l, l+32, ... in that order, then a butterfly over the lanes (every lane ends with
// the same sum: each level adds the same two partial sums, and addition commutes exactly).  All
// loads are in flight at once, so the cost is one L2 round trip whatever G is.
__device__ __forceinline__ double group_share_sum(const double* share, int G) {
    const int lane = threadIdx.x & 31;
    double t = 0.0;
    for (int g = lane; g < G; g += 32) t += __ldcg(share + g);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}
#endif

__global__ void k_sad_init(const MolDesc* mols, const int* atom_mol, int natoms_total, const DevElem* params,
                           const int* atom_z, double* arena);
__global__ void k_identity(const ChanJob* jobs);
// largest open-shell molecule (orbitals) that takes the mixed path's TF32 phase
constexpr int kLowpMaxOpenShellAo = 448;
__global__ void k_state_init(MolState* st, const MolDesc* mols, int nmol, int lowp);
__global__ void k_post_fock(const ChanJob* jobs, const MolDesc* mols, const MolState* st, int nblk, int energy_only,
                            int force);
__global__ void k_diis_solve(const MolDesc* mols, const ChanJob* jobs, const int* mol_job0, int nmol, MolState* st,
                             int* mol_status, int nblk, ScfParams prm);
__global__ void k_combine(const ChanJob* jobs, const MolState* st, int force);
__global__ void k_density_post(const ChanJob* jobs, const MolState* st, int nblk);
__global__ void k_converge(const MolDesc* mols, const ChanJob* jobs, const int* mol_job0, int nmol, MolState* st,
                           int* mol_status, int nblk, ScfParams prm, int* active_count);
__global__ void k_final_energy(const MolDesc* mols, const ChanJob* jobs, const int* mol_job0, int nmol, MolState* st,
                               int nblk);
// Per-molecule result record (doubles), see RES_* below; charges in internal atom order.
__global__ void k_results(const MolDesc* mols, const ChanJob* jobs, const int* mol_job0, int nmol, const MolState* st,
                          const int* mol_status, const DevElem* params, const int* atom_z, const double* atom_xyz,
                          double* res, double* charges);
constexpr int RES_ELEC = 0, RES_CORE = 1, RES_TOTAL = 2, RES_HOF = 3, RES_DIP = 4, RES_DIPMAG = 7, RES_HOMO = 8,
              RES_LUMO = 9, RES_HOMO_B = 10, RES_LUMO_B = 11, RES_RESID = 12, RES_ITER = 13, RES_CONV = 14,
              RES_STATUS = 15, RES_N = 16;

}  // namespace am1
