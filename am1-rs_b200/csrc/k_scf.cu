// The per-iteration SCF bookkeeping kernels (am1-rs src/scf.rs:475-1204), batched over
// molecules and spin channels:
//   k_sad_init     superposition-of-atomic-densities guess            scf.rs:475-494, 730-740
//   k_commutator   the commutator e = FP - (FP)^T = F.P - P.F (scf.rs:531-544) straight from F and
//                  P on the FP64 tensor cores, upper-triangle tiles only; its epilogue pushes e
//                  into the packed history and forms |e|^2 (scf.rs:600) and the new row of the
//                  CDIIS Gram matrix, so F.P is never stored
//   k_post_fock    one pass over the upper triangle of F, P, H: energy traces (scf.rs:595, 767),
//                  the packed history push of F and P (scf.rs:603-614, 877-952) and the new
//                  row/column of the A-DIIS Gram matrix (only those change)
//   k_diis_solve   one thread per molecule: history bookkeeping, divergence guard
//                  (scf.rs:621-625), CDIIS bordered solve with the 1e-12 pivot guard
//                  (scf.rs:966-988, 1095-1141), A-DIIS simplex (scf.rs:1061-1091, 1144-1204)
//   k_combine      F* = sum c_i F_i from the packed history (scf.rs:955-963), Gershgorin bounds
//   k_density_post rms(P_new - P) and P <- P_new                      scf.rs:546-555
//   k_converge     de / dp test and iteration count                   scf.rs:663-696, 810-823
#include <cuda_runtime.h>

#include "am1gpu_internal.h"
#include "dmma_gemm.cuh"
#include "kernels.h"

namespace am1 {

__device__ __forceinline__ long long sym_row(int r, int n) { return (long long)r * n - (long long)r * (r - 1) / 2; }
__device__ __forceinline__ long long anti_row(int r, int n) { return (long long)r * n - (long long)r * (r + 1) / 2; }

__global__ void k_sad_init(const MolDesc* __restrict__ mols, const int* __restrict__ atom_mol, int natoms_total,
                           const DevElem* __restrict__ params, const int* __restrict__ atom_z, double* __restrict__ arena) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms_total) return;
    const MolDesc md = mols[atom_mol[a]];
    const int A = a - md.atom_base, h = md.nheavy, n = md.nao;
    const DevElem& e = params[md.method * (MAX_Z + 1) + atom_z[a]];
    const double zv = e.core_charge;
    const double ns = fmin(zv, 2.0), np = fmax(zv - ns, 0.0);
    double scale[2] = {1.0, 1.0};
    if (md.nch == 2) {
        const double tot = (double)max(md.n_occ[0] + md.n_occ[1], 1);
        scale[0] = (double)md.n_occ[0] / tot;
        scale[1] = (double)md.n_occ[1] / tot;
    }
    for (int c = 0; c < md.nch; ++c) {
        double* P = arena + md.ch_base[c] + SLOT_P * (long long)n * n;
        if (A < h) {
            const int o = 4 * A;
            P[(long long)o * n + o] = ns * scale[c];
            for (int k = 1; k < 4; ++k) P[(long long)(o + k) * n + o + k] = np / 3.0 * scale[c];
        } else {
            const int o = 4 * h + (A - h);
            P[(long long)o * n + o] = ns * scale[c];
        }
    }
}

// Fresh SCF state for every molecule of a batch (each run starts from the SAD guess).
__global__ void k_state_init(MolState* __restrict__ st, const MolDesc* __restrict__ mols, int nmol, int lowp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmol) return;
    MolState s{};
    s.active = 1;
    // mixed precision: every closed shell, and the open shells that keep the eigensolver fallback
    // (at most kLowpMaxOpenShellAo orbitals).  Large radicals start FP64: a TF32 start left a few
    // of them (3 of about 1900 in a 100 000-request stream) in a UHF basin that CDIIS did not leave.
    s.lowp = lowp && (mols[i].nch == 1 || mols[i].nao <= kLowpMaxOpenShellAo);
    s.residual = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    st[i] = s;
}

// Identity warm start for the eigensolver (C^T = I; the slot is zero-filled beforehand).
__global__ void k_identity(const ChanJob* __restrict__ jobs) {
    const ChanJob jb = jobs[blockIdx.y];
    double* Ct = jb.Ct;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < jb.n; i += gridDim.x * blockDim.x) Ct[(long long)i * jb.n + i] = 1.0;
}

__device__ __forceinline__ void live_slots(const MolState& s, int& newslot, unsigned& live_mask) {
    const int c = s.hist_count, head = s.hist_head;
    live_mask = 0;
    if (c < MAX_DIIS) {
        newslot = (head + c) % MAX_DIIS;
        for (int i = 0; i < c; ++i) live_mask |= 1u << ((head + i) % MAX_DIIS);
    } else {
        newslot = head;
        for (int i = 1; i < MAX_DIIS; ++i) live_mask |= 1u << ((head + i) % MAX_DIIS);
    }
}

constexpr int POST_WARPS = 8;

__global__ void __launch_bounds__(32 * POST_WARPS) k_post_fock(const ChanJob* __restrict__ jobs, const MolDesc* __restrict__ mols,
                                                               const MolState* __restrict__ st, int nblk, int energy_only, int force) {
    const ChanJob jb = jobs[blockIdx.y];
    const MolState& s = st[jb.mol];
    if (!force && !s.active) return;
    const int n = jb.n;
    const int nb = red_blocks(n);
    if ((int)blockIdx.x >= nb) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int newslot = 0;
    unsigned live = 0;
    live_slots(s, newslot, live);
    const long long ls = packed_sym_len(n);
    double acc[RED_N];
#pragma unroll
    for (int k = 0; k < RED_N; ++k) acc[k] = 0.0;
    const bool adiis = jb.hD != nullptr;
    for (int r = blockIdx.x * POST_WARPS + warp; r < n; r += nb * POST_WARPS) {
        const double* Fr = jb.F + (long long)r * n;
        const double* Pr = jb.P + (long long)r * n;
        const double* Hr = jb.H + (long long)r * n;
        const long long rs = sym_row(r, n);
        for (int c = r + lane; c < n; c += 32) {
            const long long si = rs + (c - r);
            // the live history entries are loaded with F, P and H, before this element's stores, so
            // an element costs one round trip to memory
            double hf[MAX_DIIS], hd[MAX_DIIS];
#pragma unroll
            for (int j = 0; j < MAX_DIIS; ++j) {
                const bool ld = !energy_only && adiis && j != newslot && (live >> j & 1u);
                hf[j] = ld ? jb.hF[j * ls + si] : 0.0;
                hd[j] = ld ? jb.hD[j * ls + si] : 0.0;
            }
            const double f = Fr[c], p = Pr[c], hh = Hr[c];
            const double wgt = c == r ? 1.0 : 2.0;
            acc[RED_E_H] += wgt * p * hh;
            acc[RED_E_F] += wgt * p * f;
            if (energy_only) continue;
            jb.hF[newslot * ls + si] = f;
            if (adiis) {
                jb.hD[newslot * ls + si] = p;
#pragma unroll
                for (int j = 0; j < MAX_DIIS; ++j)  // unrolled: no dynamic index into acc
                    if (j == newslot) {
                        acc[RED_GROW + j] += wgt * p * f;
                    } else if (live >> j & 1u) {
                        acc[RED_GROW + j] += wgt * p * hf[j];
                        acc[RED_GCOL + j] += wgt * hd[j] * f;
                    }
            }
        }
    }
    __shared__ double part[POST_WARPS][RED_N];
#pragma unroll
    for (int k = 0; k < RED_N; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) part[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < RED_N) {
        double v = 0.0;
        for (int w = 0; w < POST_WARPS; ++w) v += part[w][threadIdx.x];
        jb.red[(long long)blockIdx.x * RED_N + threadIdx.x] = v;
    }
}

// The DIIS error e = FP - (FP)^T of the new Fock matrix (scf.rs:531-544).  F and P are symmetric,
// so (FP)^T = P.F and e = F.P - P.F: tile (I, J) of e is F[I,:].P[:,J] - P[I,:].F[:,J], one
// pipelined FP64 tensor-core k-loop over both products, and e is antisymmetric, so only the
// upper-triangle tiles are computed.  The epilogue takes the strict upper triangle: it stores e in
// the packed history slot of this iteration and forms this tile's share of |e|_F^2 and of
// <e, e_slot> for every live slot (the new CDIIS Gram row).
//
// COPY: how the operands reach shared memory: 0 8-byte cp.async, 1 16-byte cp.async (even n, 16-byte
// aligned rows), 2 tensor-memory-accelerator boxes from the job's tensor maps of F and P
// (maps[4 job + 2], maps[4 job + 3]; a copy wait that runs out sets bit 11 of *err).
constexpr int CT_LD = DG_TILE + 1;  // row stride of the staged commutator tile (doubles)

template <int COPY>
__device__ __forceinline__ void commutator_body(const ChanJob* __restrict__ jobs, const GemmTile* __restrict__ tiles, int ntiles,
                                                const MolState* __restrict__ st, const TmaDesc* __restrict__ maps, int* __restrict__ err) {
    __shared__ double red[CP_N][4];
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const GemmTile tl = tiles[t];
    const ChanJob jb = jobs[tl.job];
    const MolState& s = st[jb.mol];
    if (!s.active) return;
    const int n = jb.n;
    int newslot = 0;
    unsigned live = 0;
    live_slots(s, newslot, live);
    const long long la = packed_anti_len(n);
    const int m0 = tl.tm * DG_TILE, n0 = tl.tn * DG_TILE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // e is antisymmetric: a warp whose quarter is padding or lies below the diagonal issues no MMAs
    const bool compute = dg_quarter_on(m0, n0, n, n, tl.tm == tl.tn);
    double acc[2][4][4];
    double* T;  // the tile staged for the epilogue, in the pipeline's shared memory (free after the k-loop)
    if constexpr (COPY == 2) {
        extern __shared__ __align__(1024) unsigned char ctsm[];
        __shared__ DtBars bars;
        const TmaDesc* mp = maps + 4 * tl.job;  // F and P are symmetric: B = F or P read by rows
        const int shape = dg_quarter_shape(m0, n0, n, n, tl.tm == tl.tn);
        if (!dg_mainloop_tma(dt_stages(ctsm), bars, mp + 2, mp + 3, mp + 3, mp + 2, false, n, m0, n0, acc, shape)) {
            if (threadIdx.x == 0) atomicOr(err, 1 << 11);
            return;
        }
        T = reinterpret_cast<double*>(dt_stages(ctsm));
    } else {
        extern __shared__ __align__(16) double dsm[];
        dg_mainloop_diff<COPY == 1>(dsm, jb.F, jb.P, jb.P, jb.F, n, n, m0, n0, acc, compute);
        T = dsm;
    }
    // e by tile rows: the strict upper triangle of a row is contiguous in the packed history, so each
    // warp's stores of e and loads of the live slots' error vectors are runs of consecutive words
    if (compute) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) T[dg_row(i, e) * CT_LD + dg_col(j, e)] = acc[i][j][e];
    }
    __syncthreads();
    double v[CP_N];
#pragma unroll
    for (int k = 0; k < CP_N; ++k) v[k] = 0.0;
    for (int rl = warp; rl < DG_TILE; rl += DG_THREADS / 32) {
        const int r = m0 + rl;
        if (r >= n) break;
        const long long arow = anti_row(r, n) - r - 1;  // packed index of (r, c) is arow + c
        // both columns' loads of the live slots before the row's stores: one round trip per row
        double eq[2][MAX_DIIS];
#pragma unroll
        for (int hlf = 0; hlf < 2; ++hlf) {
            const int c = n0 + lane + 32 * hlf;
            const bool in = r < c && c < n;
#pragma unroll
            for (int q = 0; q < MAX_DIIS; ++q)
                eq[hlf][q] = in && q != newslot && (live >> q & 1u) ? jb.hE[q * la + arow + c] : 0.0;
        }
#pragma unroll
        for (int hlf = 0; hlf < 2; ++hlf) {
            const int cl = lane + 32 * hlf, c = n0 + cl;
            if (r < c && c < n) {
                const double ev = T[rl * CT_LD + cl];
                const long long ai = arow + c;
                jb.hE[newslot * la + ai] = ev;
                v[CP_ERR2] += 2.0 * ev * ev;
#pragma unroll
                for (int q = 0; q < MAX_DIIS; ++q)
                    if (q == newslot)
                        v[CP_B + q] += ev * ev;
                    else if (live >> q & 1u)
                        v[CP_B + q] += ev * eq[hlf][q];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < CP_N; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][warp] = x;
    }
    __syncthreads();
    if (tid < CP_N) {
        // index of tile (tm, tn), tm <= tn, in the channel's row-major upper-triangle tile list
        const int nt = (n + DG_TILE - 1) / DG_TILE;
        const int local = tl.tm * nt - tl.tm * (tl.tm - 1) / 2 + (tl.tn - tl.tm);
        jb.cpart[(long long)local * CP_N + tid] = red[tid][0] + red[tid][1] + red[tid][2] + red[tid][3];
    }
}

__global__ void __launch_bounds__(DG_THREADS, 4) k_commutator16(const ChanJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                                int ntiles, const MolState* __restrict__ st) {
    commutator_body<1>(jobs, tiles, ntiles, st, nullptr, nullptr);
}
__global__ void __launch_bounds__(DG_THREADS, 4) k_commutator8(const ChanJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                               int ntiles, const MolState* __restrict__ st) {
    commutator_body<0>(jobs, tiles, ntiles, st, nullptr, nullptr);
}
__global__ void __launch_bounds__(DG_THREADS, 4) k_commutator_tma(const ChanJob* __restrict__ jobs, const GemmTile* __restrict__ tiles,
                                                                  int ntiles, const MolState* __restrict__ st,
                                                                  const TmaDesc* __restrict__ maps, int* __restrict__ err) {
    commutator_body<2>(jobs, tiles, ntiles, st, maps, err);
}

// Gaussian elimination with partial pivoting; false when a pivot is below 1e-12.
__device__ bool solve_small(int n, double* m, double* rhs, double* x) {
    for (int col = 0; col < n; ++col) {
        int piv = col;
        double best = fabs(m[col * n + col]);
        for (int row = col + 1; row < n; ++row) {
            const double v = fabs(m[row * n + col]);
            if (v > best) {
                best = v;
                piv = row;
            }
        }
        if (best < 1.0e-12) return false;
        if (piv != col) {
            for (int j = 0; j < n; ++j) {
                const double t = m[col * n + j];
                m[col * n + j] = m[piv * n + j];
                m[piv * n + j] = t;
            }
            const double t = rhs[col];
            rhs[col] = rhs[piv];
            rhs[piv] = t;
        }
        for (int row = col + 1; row < n; ++row) {
            const double factor = m[row * n + col] / m[col * n + col];
            if (factor == 0.0) continue;
            for (int j = col; j < n; ++j) m[row * n + j] -= factor * m[col * n + j];
            rhs[row] -= factor * rhs[col];
        }
    }
    for (int col = n - 1; col >= 0; --col) {
        double sum = rhs[col];
        for (int j = col + 1; j < n; ++j) sum -= m[col * n + j] * x[j];
        x[col] = sum / m[col * n + col];
    }
    return true;
}

// Euclidean projection onto the probability simplex (sort descending, running threshold).
__device__ void simplex_project(int n, const double* v, double* out) {
    double u[MAX_DIIS];
    for (int i = 0; i < n; ++i) u[i] = v[i];
    for (int i = 1; i < n; ++i) {  // insertion sort, descending
        const double x = u[i];
        int j = i - 1;
        while (j >= 0 && u[j] < x) {
            u[j + 1] = u[j];
            --j;
        }
        u[j + 1] = x;
    }
    double css = 0.0, theta = 0.0;
    for (int j = 0; j < n; ++j) {
        css += u[j];
        const double t = (css - 1.0) / ((double)j + 1.0);
        if (u[j] - t > 0.0) theta = t;
    }
    for (int i = 0; i < n; ++i) out[i] = fmax(v[i] - theta, 0.0);
}

__device__ void adiis_simplex(int m, const double* d, const double* S, double* c) {
    double L = 1.0e-12;
    for (int i = 0; i < m; ++i) {
        double row = 0.0;
        for (int j = 0; j < m; ++j) row += fabs(S[i * MAX_DIIS + j] + S[j * MAX_DIIS + i]);
        L = fmax(L, row);
    }
    const double lr = 1.0 / L;
    for (int i = 0; i < m; ++i) c[i] = 0.0;
    c[m - 1] = 1.0;
    for (int it = 0; it < 400; ++it) {
        double trial[MAX_DIIS], proj[MAX_DIIS];
        for (int k = 0; k < m; ++k) {
            double acc = 2.0 * d[k];
            for (int j = 0; j < m; ++j) acc += (S[k * MAX_DIIS + j] + S[j * MAX_DIIS + k]) * c[j];
            trial[k] = c[k] - lr * acc;
        }
        simplex_project(m, trial, proj);
        double delta = 0.0;
        for (int i = 0; i < m; ++i) {
            delta += fabs(proj[i] - c[i]);
            c[i] = proj[i];
        }
        if (delta < 1.0e-12) break;
    }
}

__global__ void k_diis_solve(const MolDesc* __restrict__ mols, const ChanJob* __restrict__ jobs, const int* __restrict__ mol_job0,
                             int nmol, MolState* __restrict__ st, int* __restrict__ mol_status, int nblk, ScfParams prm) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= nmol) return;
    MolState& s = st[mi];
    if (!s.active) return;
    const MolDesc md = mols[mi];
    double tot[RED_N];
    for (int k = 0; k < RED_N; ++k) tot[k] = 0.0;
    for (int c = 0; c < md.nch; ++c) {
        const ChanJob& jb = jobs[mol_job0[mi] + c];
        for (int b = 0; b < red_blocks(jb.n); ++b)
            for (int k = 0; k < RED_N; ++k) tot[k] += jb.red[(long long)b * RED_N + k];
        for (int t = 0; t < jb.ntiles; ++t) {  // the commutator pass, in tile order
            tot[RED_ERR2] += jb.cpart[(long long)t * CP_N + CP_ERR2];
            for (int k = 0; k < MAX_DIIS; ++k) tot[RED_B + k] += jb.cpart[(long long)t * CP_N + CP_B + k];
        }
    }
    const double e_elec = 0.5 * (tot[RED_E_H] + tot[RED_E_F]);
    const double err = sqrt(tot[RED_ERR2]);
    // history bookkeeping: physical slot of logical index i is (head + i) % 8
    const int cnt = s.hist_count;
    int newslot;
    unsigned live;
    live_slots(s, newslot, live);
    if (cnt == MAX_DIIS) {  // drop the oldest: shift the Gram matrices up-left
        for (int i = 0; i < MAX_DIIS - 1; ++i)
            for (int j = 0; j < MAX_DIIS - 1; ++j) {
                s.bmat[i * MAX_DIIS + j] = s.bmat[(i + 1) * MAX_DIIS + j + 1];
                s.gmat[i * MAX_DIIS + j] = s.gmat[(i + 1) * MAX_DIIS + j + 1];
            }
        s.hist_head = (s.hist_head + 1) % MAX_DIIS;
        s.hist_count = MAX_DIIS;
    } else {
        s.hist_count = cnt + 1;
    }
    const int m = s.hist_count, last = m - 1;
    for (int i = 0; i < m; ++i) {
        const int phys = (s.hist_head + i) % MAX_DIIS;
        const double b = 2.0 * tot[RED_B + phys];
        s.bmat[last * MAX_DIIS + i] = b;
        s.bmat[i * MAX_DIIS + last] = b;
        s.gmat[last * MAX_DIIS + i] = tot[RED_GROW + phys];  // <D_last, F_i>
        s.gmat[i * MAX_DIIS + last] = tot[RED_GCOL + phys];  // <D_i, F_last>
    }
    s.gmat[last * MAX_DIIS + last] = tot[RED_GROW + newslot];
    s.e_elec = e_elec;
    s.err_norm = err;
    s.mode = 0;
    s.accel_used = 0;
    if (!isfinite(e_elec) || !isfinite(err)) {
        s.status = 4;  // AM1GPU_SCF_DIVERGED
        mol_status[mi] = 4;
        s.active = 0;
        s.iter += 1;
        return;
    }
    int accel = prm.use_diis ? prm.accelerator : 0;
    if (md.nch == 2) accel = prm.use_diis ? 1 : 0;  // UHF: CDIIS only (scf.rs:770-803)
    bool use_adiis = accel == 2 && err > prm.adiis_switch;
    if (accel == 1 || (accel == 2 && !use_adiis)) {
        if (m >= 2) {
            const int dim = m + 1;
            double B[(MAX_DIIS + 1) * (MAX_DIIS + 1)], rhs[MAX_DIIS + 1], x[MAX_DIIS + 1];
            for (int i = 0; i < dim * dim; ++i) B[i] = 0.0;
            for (int i = 0; i < m; ++i) {
                for (int j = 0; j < m; ++j) B[i * dim + j] = s.bmat[i * MAX_DIIS + j];
                B[i * dim + m] = -1.0;
                B[m * dim + i] = -1.0;
            }
            for (int i = 0; i < dim; ++i) rhs[i] = 0.0;
            rhs[m] = -1.0;
            if (solve_small(dim, B, rhs, x)) {
                double wsum = 0.0;
                bool fin = true;
                for (int i = 0; i < m; ++i) {
                    wsum += fabs(x[i]);
                    fin = fin && isfinite(x[i]);
                }
                if (isfinite(wsum) && fin) {
                    for (int i = 0; i < m; ++i) s.coeff[i] = x[i];
                    s.mode = 1;
                    s.accel_used = 1;
                }
            }
        }
    } else if (use_adiis && m >= 2) {
        double d[MAX_DIIS], S[MAX_DIIS * MAX_DIIS], c[MAX_DIIS];
        const double gll = s.gmat[last * MAX_DIIS + last];
        for (int i = 0; i < m; ++i) d[i] = s.gmat[i * MAX_DIIS + last] - gll;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                S[i * MAX_DIIS + j] = s.gmat[i * MAX_DIIS + j] - s.gmat[i * MAX_DIIS + last] - s.gmat[last * MAX_DIIS + j] + gll;
        adiis_simplex(m, d, S, c);
        bool fin = true;
        for (int i = 0; i < m; ++i) fin = fin && isfinite(c[i]);
        if (fin) {
            for (int i = 0; i < m; ++i) s.coeff[i] = c[i];
            s.mode = 1;
            s.accel_used = 2;
        }
    }
}

constexpr int COMBINE_CHUNK = 8;
constexpr double COMBINE_DIFF_GATE = 0.5;

__global__ void k_combine(const ChanJob* __restrict__ jobs, const MolState* __restrict__ st, int force) {
    const ChanJob jb = jobs[blockIdx.y];
    const MolState& s = st[jb.mol];
    if (!force && !s.active) return;
    const int n = jb.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const long long ls = packed_sym_len(n);
    const int m = s.hist_count;
    // from the second iteration on, F* still holds the previous iteration's: the distance between the
    // two (row sums of squares) lets k_sp2_bounds widen the previous spectral interval instead of
    // running the Lanczos bounds again.  It is only worth its extra read of F* once the density has
    // nearly settled (||P - P_previous||_F < COMBINE_DIFF_GATE); before that the rows report NaN and
    // the bounds run Lanczos.
    const bool diff = s.iter > 0 && s.dp * n < COMBINE_DIFF_GATE;
    const int mode = s.mode;
    const double* hrow[MAX_DIIS];  // history entries in logical order, and their coefficients
    double cf[MAX_DIIS];
#pragma unroll
    for (int i = 0; i < MAX_DIIS; ++i) {
        hrow[i] = jb.hF + ((s.hist_head + i) % MAX_DIIS) * ls;
        cf[i] = i < m ? s.coeff[i] : 0.0;
    }
    for (int r = blockIdx.x * nw + warp; r < n; r += gridDim.x * nw) {
        double* out = jb.Fx + (long long)r * n;
        double bound = 0.0, diag = 0.0, dd = 0.0;
        // chunks of COMBINE_CHUNK columns per lane: every load of a chunk (history entries, the previous
        // F*) is issued before any of its stores; each lane still visits its columns in ascending order
        for (int c0 = 0; c0 < n; c0 += 32 * COMBINE_CHUNK) {
            double val[COMBINE_CHUNK];
#pragma unroll
            for (int u = 0; u < COMBINE_CHUNK; ++u) {
                const int c = c0 + 32 * u + lane;
                double v = 0.0;
                if (c < n) {
                    if (mode == 0) {
                        v = jb.F[(long long)r * n + c];
                    } else {
                        const int lo = min(r, c), hi = max(r, c);
                        const long long si = sym_row(lo, n) + (hi - lo);
#pragma unroll
                        for (int i = 0; i < MAX_DIIS; ++i)
                            if (i < m) v += cf[i] * hrow[i][si];
                    }
                    if (diff) {
                        const double d = v - out[c];
                        dd = fma(d, d, dd);
                    }
                }
                val[u] = v;
            }
#pragma unroll
            for (int u = 0; u < COMBINE_CHUNK; ++u) {
                const int c = c0 + 32 * u + lane;
                if (c < n) {
                    out[c] = val[u];
                    if (c == r) diag = val[u];
                    else bound += fabs(val[u]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bound += __shfl_xor_sync(0xffffffffu, bound, o);
            diag += __shfl_xor_sync(0xffffffffu, diag, o);
            dd += __shfl_xor_sync(0xffffffffu, dd, o);
        }
        if (lane == 0) {
            jb.rowmin[r] = diag - bound;
            jb.rowmax[r] = diag + bound;
            jb.rowdf[r] = diff ? dd : __longlong_as_double(0x7ff8000000000000LL);
        }
    }
}

__global__ void k_density_post(const ChanJob* __restrict__ jobs, const MolState* __restrict__ st, int nblk) {
    const ChanJob jb = jobs[blockIdx.y];
    if (!st[jb.mol].active) return;
    const int nb = red_blocks(jb.n);
    if ((int)blockIdx.x >= nb) return;
    const long long nn = (long long)jb.n * jb.n;
    double acc = 0.0;
    const long long stride = (long long)nb * blockDim.x;
    // four elements per trip, their loads before their stores; each thread keeps its order of the sum
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < nn; i0 += 4 * stride) {
        double pn[4], po[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long i = i0 + u * stride;
            pn[u] = i < nn ? jb.Pnew[i] : 0.0;
            po[u] = i < nn ? jb.P[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long i = i0 + u * stride;
            if (i >= nn) break;
            const double d = pn[u] - po[u];
            acc += d * d;
            jb.P[i] = pn[u];
        }
    }
    __shared__ double part[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += part[w];
        jb.red2[blockIdx.x] = v;
    }
}

__global__ void k_converge(const MolDesc* __restrict__ mols, const ChanJob* __restrict__ jobs, const int* __restrict__ mol_job0,
                           int nmol, MolState* __restrict__ st, int* __restrict__ mol_status, int nblk, ScfParams prm,
                           int* __restrict__ active_count) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= nmol) return;
    MolState& s = st[mi];
    if (!s.active) return;
    if (mol_status[mi] != 0) {  // the eigensolver refused its input
        s.active = 0;
        s.status = mol_status[mi];
        s.iter += 1;
        return;
    }
    const MolDesc md = mols[mi];
    double dp = 0.0;
    for (int c = 0; c < md.nch; ++c) {
        const ChanJob& jb = jobs[mol_job0[mi] + c];
        double ss = 0.0;
        for (int b = 0; b < red_blocks(jb.n); ++b) ss += jb.red2[b];
        dp += sqrt(ss / fmax((double)jb.n * jb.n, 1.0));
    }
    const double de = fabs(s.e_elec - s.e_old);
    s.dp = dp;
    s.e_old = s.e_elec;
    s.residual = s.err_norm;
    const int it = s.iter;
    s.iter = it + 1;
    if (s.lowp) {
        // mixed precision: this iteration's density came from TF32 purification, so no
        // convergence is declared on it; the TF32 phase ends once the density has settled near its
        // rounding level, and the FP64 iterations that follow take the SCF to convergence
        if ((it > 0 && dp < prm.lowp_switch) || s.iter >= prm.lowp_max_iter) {
            s.lowp = 0;
            s.lowp_end = it;
            s.lowp_flush = 1;
        }
        if (s.iter >= prm.max_scf) s.active = 0;
    } else if (s.lowp_flush) {
        // first FP64 iteration: its Fock matrix was built from the last TF32 density.  The
        // history restarts after it, so the extrapolation (A-DIIS in particular, whose energy
        // model would favour that slightly non-idempotent density) sees FP64 iterations only.
        s.lowp_flush = 0;
        s.hist_count = 0;
        if (s.iter >= prm.max_scf) s.active = 0;
    } else if (it > s.lowp_end && it > 0 && de < prm.e_tol && (dp < prm.p_tol || s.err_norm < 1.0e-7)) {
        s.converged = 1;
        s.active = 0;
    } else if (s.iter >= prm.max_scf) {
        s.active = 0;
    }
    if (s.active) {
        atomicAdd(active_count, 1);
        if (s.lowp) atomicAdd(active_count + 1, 1);
    }
}

__global__ void k_final_energy(const MolDesc* __restrict__ mols, const ChanJob* __restrict__ jobs, const int* __restrict__ mol_job0,
                               int nmol, MolState* __restrict__ st, int nblk) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= nmol) return;
    const MolDesc md = mols[mi];
    double eh = 0.0, ef = 0.0;
    for (int c = 0; c < md.nch; ++c) {
        const ChanJob& jb = jobs[mol_job0[mi] + c];
        for (int b = 0; b < red_blocks(jb.n); ++b) {
            eh += jb.red[(long long)b * RED_N + RED_E_H];
            ef += jb.red[(long long)b * RED_N + RED_E_F];
        }
    }
    st[mi].e_final = 0.5 * (eh + ef);
}

// Result record of one molecule (src/scf.rs:370-438): energies, heat of formation, Mulliken
// charges, dipole (point charges + s-p hybrid term), frontier orbitals.
__global__ void k_results(const MolDesc* __restrict__ mols, const ChanJob* __restrict__ jobs, const int* __restrict__ mol_job0,
                          int nmol, const MolState* __restrict__ st, const int* __restrict__ mol_status,
                          const DevElem* __restrict__ params, const int* __restrict__ atom_z, const double* __restrict__ atom_xyz,
                          double* __restrict__ res, double* __restrict__ charges) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= nmol) return;
    const MolDesc md = mols[mi];
    const MolState& s = st[mi];
    const int n = md.nao, h = md.nheavy;
    const long long nn = (long long)n * n;
    const double* P0 = jobs[mol_job0[mi]].P;
    const double* P1 = md.nch == 2 ? jobs[mol_job0[mi] + 1].P : nullptr;
    double e_isol = 0.0, eheat = 0.0, dip[3] = {0.0, 0.0, 0.0};
    for (int A = 0; A < md.natoms; ++A) {
        const int a = md.atom_base + A;
        const DevElem& e = params[md.method * (MAX_Z + 1) + atom_z[a]];
        e_isol += e.e_isol;
        eheat += e.eheat_ev;
        const int o = A < h ? 4 * A : 4 * h + (A - h), no = A < h ? 4 : 1;
        double pop = 0.0;
        for (int k = 0; k < no; ++k) {
            const long long d = (long long)(o + k) * n + o + k;
            pop += P1 ? P0[d] + P1[d] : P0[d];
        }
        const double q = e.core_charge - pop;
        charges[a] = q;
        for (int k = 0; k < 3; ++k) dip[k] += atom_xyz[3 * a + k] * q;
        if (e.norb == 4) {
            const double hyb = -2.0 * e.dd;
            for (int k = 0; k < 3; ++k) {
                const long long idx = (long long)o * n + o + 1 + k;
                dip[k] += hyb * (P1 ? P0[idx] + P1[idx] : P0[idx]);
            }
        }
    }
    (void)nn;
    double* r = res + (long long)mi * RES_N;
    const double total = s.e_final + s.core_ev;
    r[RES_ELEC] = s.e_final;
    r[RES_CORE] = s.core_ev;
    r[RES_TOTAL] = total;
    r[RES_HOF] = (total - e_isol + eheat) * EV_TO_KCAL;
    double mag = 0.0;
    for (int k = 0; k < 3; ++k) {
        r[RES_DIP + k] = dip[k] * AU_DIPOLE_TO_DEBYE;
        mag += r[RES_DIP + k] * r[RES_DIP + k];
    }
    r[RES_DIPMAG] = sqrt(mag);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const double* ea = jobs[mol_job0[mi]].eps;
    const int na = md.n_occ[0], nb = md.n_occ[1];
    r[RES_HOMO] = na >= 1 ? ea[na - 1] : nan;
    r[RES_LUMO] = na < n ? ea[na] : nan;
    r[RES_HOMO_B] = nan;
    r[RES_LUMO_B] = nan;
    if (md.nch == 2) {
        const double* eb = jobs[mol_job0[mi] + 1].eps;
        r[RES_HOMO_B] = nb >= 1 ? eb[nb - 1] : nan;
        r[RES_LUMO_B] = nb < n ? eb[nb] : nan;
    }
    r[RES_RESID] = s.residual;
    r[RES_ITER] = (double)s.iter;
    r[RES_CONV] = (double)s.converged;
    r[RES_STATUS] = (double)(mol_status[mi] ? mol_status[mi] : s.status);
}

}  // namespace am1
