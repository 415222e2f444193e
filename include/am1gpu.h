/*
 * am1gpu.h -- C ABI of the B200 NDDO (AM1/RM1) SCF library, libam1gpu.so.
 *
 * This is the drop-in boundary for am1-rs's molecular single point.  Every entry point takes
 * plain pointers and sizes; all buffers are caller-owned host memory.  Units follow am1-rs:
 * positions in Bohr in, energies in eV and kcal/mol out, with MOPAC7's constants
 * (27.21 eV/Hartree, 0.529167 Angstrom/Bohr, 23.061 kcal/mol per eV; src/constants.rs:13-25).
 *
 * Thread safety: every entry point may be called from several host threads at once (the
 * reference's Python binding releases the GIL around run_am1, src/python.rs:162-164).  Each
 * host thread gets its own CUDA stream and device workspace; the only shared state is the
 * once-initialised device context and the per-method parameter upload.
 *
 * There is no CPU fallback behind these functions: without a usable CUDA device every compute
 * entry point returns AM1GPU_DEVICE_ERROR.
 */
#ifndef AM1GPU_H
#define AM1GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes.  They mirror am1-rs's Am1Error variants (src/error.rs:13-93). */
enum am1gpu_status {
    AM1GPU_OK = 0,
    AM1GPU_INVALID_INPUT = 1,              /* Am1Error::InvalidInput            (error.rs:18) */
    AM1GPU_ELEMENT_NOT_PARAMETERIZED = 2,  /* Am1Error::ElementNotParameterized (error.rs:28-32) */
    AM1GPU_SCF_NOT_CONVERGED = 3,          /* Am1Error::ScfNotConverged          (error.rs:35-38) */
    AM1GPU_SCF_DIVERGED = 4,               /* Am1Error::ScfDiverged              (error.rs:45-47) */
    AM1GPU_LINALG = 5,                     /* Am1Error::LinearAlgebra            (error.rs:33) */
    AM1GPU_UNSUPPORTED = 6,                /* more than 8192 orbitals */
    AM1GPU_DEVICE_ERROR = 7                /* CUDA failure or no device */
};

/* ScfReference (src/scf.rs:28-38). */
enum { AM1GPU_REF_AUTO = 0, AM1GPU_REF_RHF = 1, AM1GPU_REF_UHF = 2 };
/* ScfAccelerator (src/scf.rs:42-52). */
enum { AM1GPU_ACCEL_NONE = 0, AM1GPU_ACCEL_CDIIS = 1, AM1GPU_ACCEL_ADIIS_CDIIS = 2 };
/* NddoMethod (src/method.rs). */
enum { AM1GPU_METHOD_AM1 = 0, AM1GPU_METHOD_RM1 = 1 };
/* Arithmetic of the batched path (the plain path is always FP64). */
enum { AM1GPU_PRECISION_FP64 = 0, AM1GPU_PRECISION_MIXED = 1 };

/*
 * The molecular subset of Am1Options (src/scf.rs:54-154, defaults :174-197).  Fields that do
 * nothing for a molecule with default options (realspace_cutoff, ewald, klopman_ohno_tail,
 * exchange_cutoff, multipole_cutoff, electric_field, cphf_*) are not carried.
 */
typedef struct {
    int32_t reference;     /* AM1GPU_REF_*, default AUTO */
    int32_t method;        /* AM1GPU_METHOD_*, default AM1 (selects the parameter table) */
    int32_t max_scf;       /* default 200 */
    int32_t use_diis;      /* default 1; 0 forces plain iteration */
    int32_t accelerator;   /* AM1GPU_ACCEL_*, default ADIIS_CDIIS */
    int32_t precision;     /* AM1GPU_PRECISION_*, default FP64; only am1gpu_scf_batch reads it */
    double e_tol;          /* eV, default 1e-8 */
    double p_tol;          /* default 1e-7 */
    double adiis_switch;   /* default 0.1 */
} am1gpu_options;

/* One molecule: Molecule (src/system.rs:27-39) plus Am1Options::charge / multiplicity. */
typedef struct {
    int32_t natoms;
    int32_t multiplicity;      /* 2S+1, >= 1 */
    double charge;             /* total charge, e */
    const int32_t* z;          /* natoms atomic numbers */
    const double* xyz_bohr;    /* natoms*3 positions, Bohr */
} am1gpu_molecule;

/*
 * Am1Result (src/scf.rs:200-240).  Scalars are always written when the SCF ran (also when it
 * returns AM1GPU_SCF_NOT_CONVERGED, so the caller can see the residual it reached); the
 * array pointers are caller-owned outputs and any of them may be NULL to skip it.
 */
typedef struct {
    double electronic_ev;
    double core_ev;
    double total_ev;
    double heat_of_formation_kcal;
    double dipole_debye[3];
    double dipole_magnitude;
    double homo_ev, lumo_ev;             /* NaN when absent */
    double homo_beta_ev, lumo_beta_ev;   /* UHF only, NaN otherwise */
    double residual;                     /* ||[F,P]|| of the last iteration */
    int32_t nao;
    int32_t n_occ;                       /* doubly occupied (RHF) or alpha occupied (UHF) */
    int32_t n_occ_beta;
    int32_t iterations;
    int32_t converged;
    int32_t unrestricted;
    double* charges;        /* [natoms]   Mulliken net charges */
    double* density;        /* [nao*nao]  total density, row-major */
    double* spin_density;   /* [nao*nao]  P_alpha - P_beta (UHF only) */
    double* mo_energies;    /* [nao]      ascending, eV (alpha for UHF) */
    double* mo_coeff;       /* [nao*nao]  row-major, columns are MOs (alpha for UHF) */
    double* beta_energies;  /* [nao]      UHF only */
    double* beta_coeff;     /* [nao*nao]  UHF only */
} am1gpu_result;

/*
 * One element's parameters: Am1Element (src/params.rs:24-55), the published numbers and the
 * quantities derived from them, field for field.  gauss_k/l/m hold the n_gauss nonzero core-core
 * Gaussian triples (K, L, M) of Am1Element::gauss, in order.
 */
typedef struct {
    int32_t z;
    int32_t n;              /* valence principal quantum number */
    int32_t n_orb;          /* valence AOs: 1 (s) or 4 (s, p) */
    int32_t n_gauss;        /* 0..4 */
    double u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p;
    double g_ss, g_sp, g_pp, g_p2, h_sp, alpha;
    double gauss_k[4], gauss_l[4], gauss_m[4];
    double core_charge;     /* valence electrons */
    double eheat_ev;        /* experimental atomic heat of formation, eV */
    double e_isol;          /* isolated-atom electronic energy, eV */
    double dd, qq;          /* dipole / quadrupole charge separations, Bohr */
    double rho0, rho1, rho2;  /* Klopman-Ohno additive terms, Bohr */
} am1gpu_element;

/*
 * A parameter set: Am1Parameters (src/params.rs:61-70).  elements[0..count) (distinct z) are
 * every element a calculation may use; method names the parameterization the numbers belong
 * to (AM1GPU_METHOD_*), which -- as in the reference, where the method travels with the
 * parameters -- is the method of the calculation.
 */
typedef struct {
    int32_t method;
    int32_t count;
    const am1gpu_element* elements;
} am1gpu_param_table;

/* Fill *opts with Am1Options::default() (src/scf.rs:174-197). */
void am1gpu_default_options(am1gpu_options* opts);

/*
 * The built-in parameters of element z for a method: Am1Parameters::shared(method).element(z)
 * (src/params.rs:100-130).  Returns AM1GPU_ELEMENT_NOT_PARAMETERIZED when the method does not
 * cover z.  A caller starts a modified set from these records.
 */
int am1gpu_element_params(int32_t method, int32_t z, am1gpu_element* out);

/*
 * One row of a parameter table to an element: the per-row derivation of Am1Parameters::from_csv
 * (src/params.rs:139-263; dd, qq, rho0..rho2 by MOPAC's closed forms and secant solves, e_isol,
 * core charge and eheat from the element's tabulated facts).  raw: U_ss U_pp zeta_s zeta_p beta_s
 * beta_p g_ss g_sp g_pp g_p2 h_sp alpha; gauss: K1 L1 M1 .. K4 L4 M4 (triples with K = L = 0 are
 * dropped, as from_csv drops them).  Returns AM1GPU_INVALID_INPUT for z outside 1..86.
 */
int am1gpu_derive_element(int32_t z, const double raw[12], const double gauss[12], am1gpu_element* out);

/* Number of valence AOs of a molecule: Basis::build (src/basis.rs:37-60).  Returns
 * AM1GPU_ELEMENT_NOT_PARAMETERIZED for an element the method does not cover. */
int am1gpu_basis_size(int32_t natoms, const int32_t* z, int32_t method, int32_t* nao);

/*
 * Plain FP64 single point of one molecule: replaces run_am1 (src/scf.rs:294-468) for a
 * molecule.  Returns AM1GPU_OK, or the error run_am1 would raise; AM1GPU_SCF_NOT_CONVERGED
 * still fills *res.
 */
int am1gpu_scf(const am1gpu_molecule* mol, const am1gpu_options* opts, am1gpu_result* res);

/*
 * Batched single points: nmol independent molecules solved together on the device, each with
 * its own SCF trajectory and convergence test (same per-molecule semantics as am1gpu_scf).
 * status[i] receives molecule i's return code.  The return value is AM1GPU_OK when every
 * molecule succeeded, otherwise the first failing code.  opts->precision selects FP64 or
 * the mixed path (FP32 eigensolve and density with FP64 refinement).
 */
int am1gpu_scf_batch(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts,
                     am1gpu_result* results, int32_t* status);

/*
 * The same single points with the caller's parameter set: run_am1(molecule, params, options)
 * (src/scf.rs:294) with any &Am1Parameters, e.g. one built by Am1Parameters::from_csv or with
 * modified entries in its public elements map.  params == NULL uses the built-in set of
 * opts->method; otherwise params->method is the method and opts->method is not read.  An
 * element of the molecule that the set lacks returns AM1GPU_ELEMENT_NOT_PARAMETERIZED; a set
 * with a repeated z, z outside 1..86, n_orb other than 1 or 4, n_gauss outside 0..4 or a
 * non-finite number returns AM1GPU_INVALID_INPUT.  The set travels with the call's inputs
 * (about 50 KB): nothing is cached between calls.
 */
int am1gpu_scf_params(const am1gpu_molecule* mol, const am1gpu_param_table* params, const am1gpu_options* opts,
                      am1gpu_result* res);
int am1gpu_scf_batch_params(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_param_table* params,
                            const am1gpu_options* opts, am1gpu_result* results, int32_t* status);

/*
 * SCF single point plus the closed-form nuclear gradient at its converged density: replaces
 * closed_form_gradient (src/gradient.rs:173-253) for a molecule (RHF and, through the same
 * spin-resolved pair formula, UHF: fixed_density_gradient_uhf, src/gradient.rs:495-544).
 * gradient receives dE/dx (eV/Bohr) as natoms * 3 doubles in the caller's atom order; the
 * forces are its negation.  The result and return code are those of am1gpu_scf (FP64); a
 * molecule that did not converge still gets the gradient at its last density, with
 * AM1GPU_SCF_NOT_CONVERGED returned, as the reference's run_am1 error would stop it there.
 */
int am1gpu_gradient(const am1gpu_molecule* mol, const am1gpu_options* opts, am1gpu_result* res, double* gradient);

/* The batched form: gradients[i] (natoms_i * 3 doubles, or NULL to skip) per molecule. */
int am1gpu_gradient_batch(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts,
                          am1gpu_result* results, double* const* gradients, int32_t* status);

/* The gradient with the caller's parameter set (closed_form_gradient takes &Am1Parameters too);
 * params as in am1gpu_scf_batch_params. */
int am1gpu_gradient_batch_params(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_param_table* params,
                                 const am1gpu_options* opts, am1gpu_result* results, double* const* gradients,
                                 int32_t* status);

/*
 * Core Hamiltonian and core-core energy of one molecule: replaces build_core_with_neighbors
 * (src/hamiltonian.rs:211-366) and core_core_energy_with_neighbors (src/repulsion.rs:38-56)
 * for a molecule.  h_core is nao*nao row-major (eV); *core_ev in eV.
 */
int am1gpu_build_core(const am1gpu_molecule* mol, int32_t method, double* h_core, double* core_ev);

/*
 * Two-electron matrices G(P_r) = J(P_r) - K(P_r / 2), no H_core, for nrhs densities of one
 * molecule: replaces build_g_matrix (src/fock.rs:556-575, FockBase::Zero), which the CPHF
 * response calls 3N times per iteration (src/hessian.rs:1401, 1567).  densities and g are
 * nrhs consecutive nao x nao row-major matrices in the caller's AO order.
 */
int am1gpu_g_matrix_batch(const am1gpu_molecule* mol, int32_t method, int32_t nrhs, const double* densities,
                          double* g);

/*
 * Spin Fock matrix F = H_core + J(p_tot) - K(spin_scale * p_spin): replaces
 * build_fock_spin_with (src/fock.rs:249-511) with FockBase::CoreHamiltonian.  RHF is
 * p_spin = p_tot with spin_scale 0.5 (build_fock, src/fock.rs:526-546).
 */
int am1gpu_build_fock(const am1gpu_molecule* mol, int32_t method, const double* p_tot,
                      const double* p_spin, double spin_scale, double* fock);

/*
 * Symmetric eigendecomposition: replaces symmetric_eigen (src/linalg.rs:276-331).
 * a is n*n row-major (its lower triangle is read); w receives ascending eigenvalues; v
 * (row-major) the eigenvectors as columns.  Up to 448 rows a cluster Jacobi on chip; up to 8192
 * the Householder reduction, bisection, inverse iteration on the tridiagonal and a blocked
 * back-transformation.  Non-finite input returns AM1GPU_LINALG, as the reference refuses it.
 */
int am1gpu_symmetric_eigen(int32_t n, const double* a, double* w, double* v);

/*
 * Eigenvalues only (ascending), for a symmetric matrix of up to 8192 rows: the first half of
 * symmetric_eigen (src/linalg.rs:276-331), by the SCF's final-spectrum path (Householder
 * tridiagonalisation, blocked with FP64 tensor-core trailing updates from 2048 rows, then Sturm
 * bisection).  a is n*n row-major (its lower triangle is read); non-finite input returns AM1GPU_LINALG.
 */
int am1gpu_symmetric_eigenvalues(int32_t n, const double* a, double* w);

/*
 * Density of one symmetric matrix f (n <= 448 rows, its lower triangle read):
 * p = weight * (projector onto its n_occ lowest eigenvectors), by trace-correcting purification
 * -- the step an SCF iteration takes after the extrapolation, symmetric_eigen + density_from_coeff
 * (src/scf.rs:654-661, 503-524), alone.  precision: 0 FP64 tensor cores (the products of the FP64
 * SCF), 1 FP32-accurate products on the fifth-generation tensor cores (tcgen05, TF32 operands split
 * in two, as the mixed path's early iterations use), 2 TF32 products on mma.sync, 3 FP64 products on
 * tcgen05's integer path from 7-bit digit planes of the iterate (AM1GPU_FP64_DIGITS), 4 TF32 products
 * on tcgen05 in one pass over TF32-rounded iterates.  The reduced-
 * precision runs stop at their own rounding floor and are rescaled to trace n_occ.  *steps (may be
 * NULL) receives the number of products.  A matrix whose gap is too small to purify in 100 steps
 * returns AM1GPU_LINALG.
 */
int am1gpu_density_purify(int32_t n, const double* f, double n_occ, double weight, int32_t precision, double* p,
                          int32_t* steps);

/*
 * The autotuner's table for the current device: which kernel the mixed path's reduced-precision
 * purification products use per size class (n <= 128, <= 256, <= 384, larger): choice[c] = 0
 * mma.sync TF32, 1 tcgen05 at FP32 accuracy (3xTF32), 2 tcgen05 in one TF32 pass, -1 not tuned
 * yet; ms[3c + k] (12 floats) the time of one purification of the class's test matrix with kernel
 * k.  Either pointer may be NULL.  No counterpart in the reference.
 */
int am1gpu_lowp_tuning(int32_t* choice, float* ms);

/*
 * count independent symmetric eigendecompositions in one call (each as am1gpu_symmetric_eigen:
 * those of n[i] <= 448 in one set of launches, larger ones after them, one at a time): replaces the per-subsystem symmetric_eigen calls of the divide-and-conquer SCF
 * (solve_subsystems, src/divide_conquer.rs:587-617).  a[i], w[i], v[i] as above for matrix i;
 * status[i] (may be NULL) receives its code, and the first nonzero one is returned.
 */
int am1gpu_symmetric_eigen_batch(int32_t count, const int32_t* n, const double* const* a, double* const* w,
                                 double* const* v, int32_t* status);

/* Message of the last failing call on this host thread ("" if none). */
const char* am1gpu_last_error(void);

/*
 * Allocation-free symmetric eigensolver, for callers that may not allocate device memory
 * (code running beside a framework that owns the whole device memory pool, real-time loops
 * where an allocation is an unbounded stall, hosts that only hand out device buffers).  No
 * counterpart in the reference: am1-rs has no device memory to allocate.
 * a (n*n), w (n) and v (n*n) are DEVICE pointers owned by the caller; a is read (lower
 * triangle, as symmetric_eigen does), w receives ascending eigenvalues, v (row-major) the
 * eigenvectors as columns.  stream is a cudaStream_t (NULL: the default stream); the call
 * returns when the results are in w and v.  Scratch is a fixed 512 KiB device array inside
 * the library, so n <= 128 (larger n returns AM1GPU_INVALID_INPUT) and no cudaMalloc/cudaFree
 * is ever called.  The first call on a device sets up (fetches the array's address) and must
 * come before any stream capture on that device; a set-up that fails is tried again by the next
 * call.  Calls share the array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller.  Non-finite input returns
 * AM1GPU_LINALG (w and v are then unspecified).
 */
int am1gpu_symmetric_eigen_noalloc(int32_t n, const double* a, double* w, double* v, void* stream);

/*
 * Resident batch: the molecules are uploaded once and stay in device memory, so the SCF can be
 * re-run (and its results fetched) without moving inputs again -- the form a serving loop or a
 * benchmark of the device path uses.  The handle owns its device memory and CUDA stream; it is
 * not thread-safe (one handle per host thread at a time).  Inputs are copied at creation.
 * No counterpart in the reference: am1-rs keeps all state in host memory.
 */
typedef struct am1gpu_batch am1gpu_batch;
int am1gpu_batch_create(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts,
                        am1gpu_batch** out);
/* Runs integrals + SCF + result records on the device; no host<->device copy of inputs or
 * results (only the 4-byte count of molecules still iterating is read back). */
int am1gpu_batch_run(am1gpu_batch* batch);
/* Copies the results of the last run into caller-owned records (same semantics as
 * am1gpu_scf_batch's results/status). */
int am1gpu_batch_results(am1gpu_batch* batch, am1gpu_result* results, int32_t* status);
void am1gpu_batch_destroy(am1gpu_batch* batch);

/* Phases of a call, named after the reference's AM1_TIMING scopes (src/scf.rs:315-659). */
enum {
    AM1GPU_PHASE_CORE = 0,        /* "basis+core": integrals, overlap, H_core, core-core, guess */
    AM1GPU_PHASE_FOCK = 1,        /* "scf:fock" */
    AM1GPU_PHASE_COMMUTATOR = 2,  /* "scf:commutator": F.P, [F,P], energy, DIIS history */
    AM1GPU_PHASE_ACCEL = 3,       /* "scf:accel": CDIIS / A-DIIS solve and extrapolation */
    AM1GPU_PHASE_EIGEN = 4,       /* "scf:eigen": P from F* (purification, or eigensolver) */
    AM1GPU_PHASE_DENSITY_CORE = 5,/* the inner kernel of scf:eigen alone: the purification
                                     steps, or the Jacobi kernel on the eigensolver path */
    AM1GPU_PHASE_DENSITY = 6,     /* "scf:density": C_occ C_occ^T, dP, convergence */
    AM1GPU_PHASE_FINAL = 7        /* final Fock, energy and result records */
};

/* Statistics of the last call on this host thread (or of a batch handle's last run). */
typedef struct {
    double device_ms;            /* the call's device time (CUDA events on the library's stream) */
    double phase_ms[8];          /* per phase, when timing is on (else 0) */
    int64_t phase_launches[8];   /* kernel launches per phase */
    int64_t kernel_launches;     /* all kernels the call launched */
    int64_t h2d_bytes;           /* host->device bytes the call copied */
    int64_t d2h_bytes;           /* device->host bytes the call copied */
    int32_t scf_cycles;          /* batched SCF iterations run (the slowest molecule's count) */
    int32_t eigen_fallbacks;     /* molecule-iterations whose purification stalled (eigensolver used) */
    double purification_steps;   /* purification steps summed over molecules, channels, iterations */
    double purification_flops;   /* their algorithmic work: n^3 per symmetric product X.X */
    double purification_bytes;   /* their algorithmic HBM traffic: 16 n^2 per product (read X, write X^2) */
    double lowp_purification_steps;  /* products X.X of the mixed path's reduced-precision (TF32) iterations */
    double lowp_purification_flops;  /* their algorithmic work, n^3 each (not in purification_flops) */
    int64_t graph_launches;      /* 1 when the SCF loop ran as one CUDA graph launch with device-side loops, 0 when the host drove it */
} am1gpu_call_stats;

/* Per-phase CUDA-event timing on (1) or off (0); the default follows AM1_TIMING. */
void am1gpu_set_timing(int32_t enable);

/*
 * CUDA priority of the calling host thread's stream, on which its calls run (0 the default,
 * negative higher; clamped to the device's range).  A serving loop gives its small-request workers
 * a higher priority, so their kernels go before long batches' on the SMs.  No counterpart in the
 * reference (which has no device stream).
 */
int am1gpu_set_stream_priority(int32_t priority);
int am1gpu_last_call_stats(am1gpu_call_stats* out);
int am1gpu_batch_stats(const am1gpu_batch* batch, am1gpu_call_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* AM1GPU_H */
