// Host driver of libam1gpu: input validation (src/scf.rs:294-366), batch planning, the device
// memory pool, the SCF iteration loop and the C ABI of include/am1gpu.h.
//
// A call solves any number of molecules at once.  All per-molecule work runs in batched kernels
// (one launch per SCF phase for the whole batch); each molecule keeps its own trajectory and
// convergence test and retires in place (MolState::active), so a molecule's result does not
// depend on what else is in the batch.  The host only reads one integer (molecules still
// active) every few iterations.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/am1gpu.h"
#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

const DevElem* host_param_table();
DevElem derive_from_raw(int z, const double raw[12], const double gauss[12]);

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(AM1GPU_DEVICE_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

const char* kSymbols[] = {"X",  "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si",
                          "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu",
                          "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru",
                          "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr",
                          "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",
                          "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn"};

inline const DevElem& helem(int method, int z) { return host_param_table()[method * (MAX_Z + 1) + z]; }

// ---------------------------------------------------------------------------------------
// Caller parameter sets (am1gpu_param_table, the reference's Am1Parameters) <-> device records
// ---------------------------------------------------------------------------------------
void element_to_abi(const DevElem& e, int z, am1gpu_element* o) {
    *o = am1gpu_element{};
    o->z = z;
    o->n = e.n;
    o->n_orb = e.norb;
    o->n_gauss = e.ngauss;
    o->u_ss = e.u_ss; o->u_pp = e.u_pp; o->zeta_s = e.zeta_s; o->zeta_p = e.zeta_p; o->beta_s = e.beta_s; o->beta_p = e.beta_p;
    o->g_ss = e.g_ss; o->g_sp = e.g_sp; o->g_pp = e.g_pp; o->g_p2 = e.g_p2; o->h_sp = e.h_sp; o->alpha = e.alpha;
    for (int k = 0; k < 4; ++k) {
        o->gauss_k[k] = k < e.ngauss ? e.gk[k] : 0.0;
        o->gauss_l[k] = k < e.ngauss ? e.gl[k] : 0.0;
        o->gauss_m[k] = k < e.ngauss ? e.gm[k] : 0.0;
    }
    o->core_charge = e.core_charge; o->eheat_ev = e.eheat_ev; o->e_isol = e.e_isol;
    o->dd = e.dd; o->qq = e.qq; o->rho0 = e.rho0; o->rho1 = e.rho1; o->rho2 = e.rho2;
}

// A caller's element record to the device record; false (with the reason) when it cannot be used.
bool element_from_abi(const am1gpu_element& a, DevElem& e, std::string& why) {
    if (a.z < 1 || a.z > MAX_Z) { why = "atomic number " + std::to_string(a.z) + " outside 1.." + std::to_string(MAX_Z); return false; }
    const std::string who = std::string("element ") + kSymbols[a.z];
    if (a.n_orb != 1 && a.n_orb != 4) { why = who + ": n_orb must be 1 or 4"; return false; }
    if (a.n_gauss < 0 || a.n_gauss > 4) { why = who + ": n_gauss must be 0..4"; return false; }
    if (a.n < 1 || a.n > 6) { why = who + ": principal quantum number must be 1..6"; return false; }
    const double v[] = {a.u_ss, a.u_pp, a.zeta_s, a.zeta_p, a.beta_s, a.beta_p, a.g_ss, a.g_sp, a.g_pp, a.g_p2, a.h_sp, a.alpha,
                        a.core_charge, a.eheat_ev, a.e_isol, a.dd, a.qq, a.rho0, a.rho1, a.rho2};
    for (double x : v)
        if (!std::isfinite(x)) { why = who + ": a parameter is not finite"; return false; }
    for (int k = 0; k < a.n_gauss; ++k)
        if (!std::isfinite(a.gauss_k[k]) || !std::isfinite(a.gauss_l[k]) || !std::isfinite(a.gauss_m[k])) {
            why = who + ": a core-core Gaussian is not finite";
            return false;
        }
    e = DevElem{};
    e.present = 1;
    e.n = a.n;
    e.norb = a.n_orb;
    e.ngauss = a.n_gauss;
    e.u_ss = a.u_ss; e.u_pp = a.u_pp; e.zeta_s = a.zeta_s; e.zeta_p = a.zeta_p; e.beta_s = a.beta_s; e.beta_p = a.beta_p;
    e.g_ss = a.g_ss; e.g_sp = a.g_sp; e.g_pp = a.g_pp; e.g_p2 = a.g_p2; e.h_sp = a.h_sp; e.alpha = a.alpha;
    for (int k = 0; k < a.n_gauss; ++k) {
        e.gk[k] = a.gauss_k[k];
        e.gl[k] = a.gauss_l[k];
        e.gm[k] = a.gauss_m[k];
    }
    e.core_charge = a.core_charge; e.eheat_ev = a.eheat_ev; e.e_isol = a.e_isol;
    e.dd = a.dd; e.qq = a.qq; e.rho0 = a.rho0; e.rho1 = a.rho1; e.rho2 = a.rho2;
    return true;
}

// The device table of a call with the caller's set: [method][Z] like the built-in upload, the
// set's method slot holding exactly its elements (the other slot keeps the built-in numbers,
// which nothing in the call reads).
int custom_param_table(const am1gpu_param_table* t, std::vector<DevElem>& tab, int* method) {
    if (t->method != AM1GPU_METHOD_AM1 && t->method != AM1GPU_METHOD_RM1)
        return fail(AM1GPU_INVALID_INPUT, "unknown method " + std::to_string(t->method) + " in the parameter set");
    if (t->count < 0 || (t->count > 0 && !t->elements)) return fail(AM1GPU_INVALID_INPUT, "null parameter set elements");
    *method = t->method == AM1GPU_METHOD_RM1 ? 1 : 0;
    tab.assign(host_param_table(), host_param_table() + 2 * (MAX_Z + 1));
    DevElem* slot = tab.data() + *method * (MAX_Z + 1);
    for (int z = 0; z <= MAX_Z; ++z) slot[z] = DevElem{};
    for (int i = 0; i < t->count; ++i) {
        DevElem e;
        std::string why;
        if (!element_from_abi(t->elements[i], e, why)) return fail(AM1GPU_INVALID_INPUT, "parameter set: " + why);
        if (slot[t->elements[i].z].present)
            return fail(AM1GPU_INVALID_INPUT, std::string("parameter set: element ") + kSymbols[t->elements[i].z] + " appears twice");
        slot[t->elements[i].z] = e;
    }
    return AM1GPU_OK;
}

// ---------------------------------------------------------------------------------------
// Device context: parameter table uploaded once per device
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ---------------------------------------------------------------------------------------
struct DeviceCtx {
    std::once_flag once;
    int rc = AM1GPU_OK;
    std::string err;
    DevElem* d_params = nullptr;
    int sms = 0;
    int jacobi_smem = 0;  // dynamic shared memory available to one eigensolver CTA
    int tridiag_smem = 0;  // ... and to one tridiagonalisation CTA
    int sp2b_grid = 0;     // CTAs of the grid-wide Lanczos bounds (all co-resident)
};

// Shared-memory budgets the planner sizes eigensolver and tridiagonalisation clusters for (set
// when a device is opened).
int g_jacobi_budget = 232448 - 1024;
int g_tridiag_budget = 232448 - 1024;
int g_sp2b_grid = 148;  // CTAs of the grid-wide Lanczos bounds (set when a device is opened)
int g_sms = 148;        // SMs of the current device

// Smallest cluster (1, 2, 4, 8, 16 CTAs) whose row share of an n x n matrix fits one CTA's
// shared memory; 0 when none does.
// Largest matrix a tridiagonalisation cluster of C CTAs holds (the order a reduction on 2 C CTAs
// hands over at).
int tridiag_cluster_max(int C) {
    static thread_local int cached_budget = -1, cached[5] = {};
    if (cached_budget != g_tridiag_budget) {
        for (int k = 0; k < 5; ++k) {
            int m = 2;
            while (tridiag_smem_bytes(m + 1, 1 << k) <= (size_t)g_tridiag_budget) ++m;
            cached[k] = m;
        }
        cached_budget = g_tridiag_budget;
    }
    return cached[C == 1 ? 0 : C == 2 ? 1 : C == 4 ? 2 : C == 8 ? 3 : 4];
}

int tridiag_cluster(int n) {
    for (int C = 1; C <= 16; C *= 2)
        if (tridiag_smem_bytes(n, C) <= (size_t)g_tridiag_budget) return C;
    return 0;
}

DeviceCtx g_dev[64];

int device_ctx(DeviceCtx** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(AM1GPU_DEVICE_ERROR, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(AM1GPU_DEVICE_ERROR, "device index out of range");
    DeviceCtx& c = g_dev[dev];
    std::call_once(c.once, [&c, dev] {
        auto bad = [&c](const char* what, cudaError_t err) {
            c.rc = AM1GPU_DEVICE_ERROR;
            c.err = std::string(what) + ": " + cudaGetErrorString(err);
        };
        cudaError_t err;
        if ((err = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return bad("attr", err);
        const size_t bytes = sizeof(DevElem) * 2 * (MAX_Z + 1);
        if ((err = cudaMalloc(&c.d_params, bytes)) != cudaSuccess) return bad("cudaMalloc params", err);
        if ((err = cudaMemcpy(c.d_params, host_param_table(), bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
            return bad("upload params", err);
        // dynamic shared memory of the eigensolver: the opt-in limit minus its static shared memory
        int optin = 0;
        if ((err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
            return bad("smem attr", err);
        cudaFuncAttributes fa{};
        if ((err = cudaFuncGetAttributes(&fa, k_jacobi)) != cudaSuccess) return bad("jacobi attributes", err);
        c.jacobi_smem = optin - (int)fa.sharedSizeBytes;
        if ((err = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, c.jacobi_smem)) != cudaSuccess)
            return bad("jacobi smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
            return bad("jacobi cluster attribute", err);
        {
            int per_sm = 0;
            if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sp2_bounds_big, 512, 0)) != cudaSuccess)
                return bad("grid bounds occupancy", err);
            c.sp2b_grid = std::max(1, std::min(per_sm, 2)) * c.sms;
        }
        for (const void* f : {(const void*)k_bisect, (const void*)k_sp2_bounds}) {  // 2 n and 3 n doubles
            cudaFuncAttributes fb{};
            if ((err = cudaFuncGetAttributes(&fb, f)) != cudaSuccess) return bad("bisection / bounds attributes", err);
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fb.sharedSizeBytes)) !=
                cudaSuccess)
                return bad("bisection / bounds smem attribute", err);
        }
        if ((err = cudaFuncGetAttributes(&fa, k_tridiag)) != cudaSuccess) return bad("tridiag attributes", err);
        c.tridiag_smem = optin - (int)fa.sharedSizeBytes;
        if ((err = cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, c.tridiag_smem)) != cudaSuccess)
            return bad("tridiag smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
            return bad("tridiag cluster attribute", err);
        for (const void* f : {(const void*)k_tridiag_cl, (const void*)k_sp2_bounds_cl})
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
                return bad("large-matrix cluster attribute", err);
        for (const void* f : {(const void*)k_tridiag_cl, (const void*)k_tridiag_big, (const void*)k_tridiag_panel}) {
            cudaFuncAttributes fb{};
            if ((err = cudaFuncGetAttributes(&fb, f)) != cudaSuccess) return bad("large tridiagonalisation attributes", err);
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fb.sharedSizeBytes)) !=
                cudaSuccess)
                return bad("large tridiagonalisation smem attribute", err);
        }
        for (const void* f : {(const void*)k_sp2_step16, (const void*)k_sp2_step8, (const void*)k_commutator16,
                              (const void*)k_commutator8})
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dgemm_smem_bytes())) != cudaSuccess)
                return bad("tile kernel smem attribute", err);
        for (const void* f : {(const void*)k_sp2_step_tma, (const void*)k_commutator_tma})
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dgemm_tma_smem_bytes())) != cudaSuccess)
                return bad("tensor-map tile kernel smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_sp2_step_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tf32_smem_bytes())) !=
            cudaSuccess)
            return bad("tf32 tile kernel smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_sp2_step_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes())) != cudaSuccess)
            return bad("tcgen05 tile kernel smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_sp2_step_tc1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc1_smem_bytes())) !=
            cudaSuccess)
            return bad("single-pass tcgen05 tile kernel smem attribute", err);
        if ((err = cudaFuncSetAttribute(k_sp2_step_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz_smem_bytes())) != cudaSuccess)
            return bad("digit-plane tile kernel smem attribute", err);
        for (const void* f : {(const void*)k_tridiag_syr2k16, (const void*)k_tridiag_syr2k8, (const void*)k_dgemm16,
                              (const void*)k_dgemm8})
            if ((err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dgemm_smem_bytes())) != cudaSuccess)
                return bad("trailing-update / back-transformation smem attribute", err);
        {
            cudaFuncAttributes fo{};
            if ((err = cudaFuncGetAttributes(&fo, k_stein_orth)) != cudaSuccess) return bad("cluster orthogonalisation attributes", err);
            if ((err = cudaFuncSetAttribute(k_stein_orth, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fo.sharedSizeBytes)) !=
                cudaSuccess)
                return bad("cluster orthogonalisation smem attribute", err);
        }
    });
    if (c.rc != AM1GPU_OK) return fail(c.rc, c.err);
    g_jacobi_budget = c.jacobi_smem;
    g_tridiag_budget = c.tridiag_smem;
    g_sms = c.sms;
    g_sp2b_grid = c.sp2b_grid;
    *out = &c;
    return AM1GPU_OK;
}

// ---------------------------------------------------------------------------------------
// Device memory: a grow-only device pool + pinned host staging + a stream.  One per host
// thread (the ABI calls) and one per resident batch handle.
// ---------------------------------------------------------------------------------------
struct Mem {
    int dev = -1;
    int priority = 0;  // the stream's CUDA priority (0 default, negative higher)
    cudaStream_t stream = nullptr;
    char* dpool = nullptr;
    size_t dcap = 0;
    char* hpin = nullptr;
    size_t hcap = 0;
    std::vector<cudaEvent_t> events;  // timing events, reused across calls
    cudaStream_t cap_stream = nullptr;  // stream the SCF graph is captured on
};

// Stream priority asked for by the calling host thread (am1gpu_set_stream_priority).
thread_local int tl_priority = 0;

int mem_ensure(Mem& w, size_t dbytes, size_t hbytes) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (w.dev != dev) {  // first use on this device
        w = Mem();
        w.dev = dev;
        w.priority = tl_priority;
        CK(cudaStreamCreateWithPriority(&w.stream, cudaStreamNonBlocking, w.priority));
    }
    if (dbytes > w.dcap) {
        if (w.dpool) CK(cudaFree(w.dpool));
        w.dpool = nullptr;
        w.dcap = 0;
        CK(cudaMalloc(&w.dpool, dbytes));
        w.dcap = dbytes;
    }
    if (hbytes > w.hcap) {
        if (w.hpin) CK(cudaFreeHost(w.hpin));
        w.hpin = nullptr;
        w.hcap = 0;
        CK(cudaMallocHost(&w.hpin, hbytes));
        w.hcap = hbytes;
    }
    return AM1GPU_OK;
}

void mem_release(Mem& w) {
    if (w.dpool) cudaFree(w.dpool);
    if (w.hpin) cudaFreeHost(w.hpin);
    for (auto e : w.events) cudaEventDestroy(e);
    if (w.stream) cudaStreamDestroy(w.stream);
    if (w.cap_stream) cudaStreamDestroy(w.cap_stream);
    w = Mem();
}

thread_local Mem tl_mem;
using Workspace = Mem;

int workspace(Workspace** out, size_t dbytes, size_t hbytes) {
    int rc = mem_ensure(tl_mem, dbytes, hbytes);
    if (rc) return rc;
    *out = &tl_mem;
    return AM1GPU_OK;
}

// ---------------------------------------------------------------------------------------
// Call statistics and phase timing (the reference's AM1_TIMING phases, src/timing.rs)
// ---------------------------------------------------------------------------------------
std::atomic<int> g_timing{-1};  // -1: read AM1_TIMING on first use

bool timing_on() {
    int t = g_timing.load();
    if (t < 0) {
        const char* e = std::getenv("AM1_TIMING");
        t = (e && *e && std::strcmp(e, "0") != 0) ? 1 : 0;
        g_timing.store(t);
    }
    return t == 1;
}

thread_local am1gpu_call_stats tl_stats;

constexpr int kSp2MaxSteps = 100;
constexpr int kWorkN = 8;  // device counters of a run (Batch::d_work)

// Mixed precision: a molecule's TF32 phase ends when its RMS density change falls below
// kLowpSwitch (about where TF32 purification stops improving the density), or after
// kLowpMaxIter iterations.
// AM1GPU_LOWP_SWITCH / AM1GPU_LOWP_MAXIT override them (for tuning).
constexpr double kLowpSwitch = 1e-3;
constexpr int kLowpMaxIter = 12;

double lowp_switch() {
    static const double v = [] {
        const char* e = std::getenv("AM1GPU_LOWP_SWITCH");
        return e && *e ? std::atof(e) : kLowpSwitch;
    }();
    return v;
}

int lowp_max_iter() {
    static const int v = [] {
        const char* e = std::getenv("AM1GPU_LOWP_MAXIT");
        return e && *e ? std::atoi(e) : kLowpMaxIter;
    }();
    return v;
}

// How the SCF step forms P from F*: 0 purification (default), 1 eigenvectors every iteration.
// AM1GPU_DENSITY=jacobi selects the eigensolver path (kept for comparison and testing).
// Purification steps before a molecule counts as stalled (AM1GPU_SP2_MAX_STEPS, 1..kSp2MaxSteps;
// default kSp2MaxSteps).  A stalled molecule takes the eigensolver for that iteration; a small
// cap exercises that path on every iteration.
int sp2_max_steps() {
    static const int v = [] {
        const char* e = std::getenv("AM1GPU_SP2_MAX_STEPS");
        const int k = e ? std::atoi(e) : kSp2MaxSteps;
        return k < 1 ? kSp2MaxSteps : std::min(k, kSp2MaxSteps);
    }();
    return v;
}

// Which kernel takes a molecule's reduced-precision purification products: 0 mma.sync TF32
// (k_sp2_step_tf32), 1 tcgen05 at FP32 accuracy from 3xTF32 (k_sp2_step_tc), 2 tcgen05 in one TF32
// pass (k_sp2_step_tc1).  AM1GPU_LOWP_TC=0, 1 or 2 forces one kernel; otherwise the autotuner's
// choice for the molecule's size class (tune_lowp_kernels, run once per device and class before the
// first mixed batch that holds such a molecule).
constexpr int kTuneClasses = 4;
inline int tune_class(int n) { return n <= 128 ? 0 : n <= 256 ? 1 : n <= 384 ? 2 : 3; }
constexpr int kTuneSize[kTuneClasses] = {96, 192, 320, 448};  // the matrix each class is timed on
struct LowpTune {
    std::mutex mu;
    int choice[kTuneClasses] = {-1, -1, -1, -1};  // -1 untuned, else the lowp_tc_for kind
    float ms[kTuneClasses][3] = {};                // time of one purification with kind 0, 1, 2
};
LowpTune g_lowp_tune[64];

// Which molecules' FP64 purification products run on tcgen05's integer path from digit planes
// (k_sp2_step_oz) rather than on the FP64 tensor cores (k_sp2_step16/8): AM1GPU_FP64_DIGITS=1 all,
// 0 none (the default).
bool fp64_oz_for(int n) {
    static const int v = [] {
        const char* e = std::getenv("AM1GPU_FP64_DIGITS");
        return e ? std::atoi(e) : 0;
    }();
    (void)n;
    return v != 0;
}
// The FP64 purification products of even-order matrices copy their operands with the tensor memory
// accelerator (k_sp2_step_tma) unless AM1GPU_SP2_TMA=0 (k_sp2_step16, cp.async) or the driver has no
// tensor-map encoder.  cuTensorMapEncodeTiled is looked up once through the runtime, so the library
// does not link the driver library itself.
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        const char* e = std::getenv("AM1GPU_SP2_TMA");
        if (e && std::atoi(e) == 0) return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        return (PFN_cuTensorMapEncodeTiled_v12000)f;
    }();
    return fn;
}
static_assert(sizeof(CUtensorMap) == sizeof(TmaDesc), "TmaDesc mirrors CUtensorMap");

// The tensor map k_sp2_step_tma reads an n x n row-major FP64 matrix through: boxes of 16 columns
// (128 bytes) x 64 rows, 128-byte swizzle, zero fill past the edges.  Needs n even and a 16-byte
// aligned base (row pitch a multiple of 16 bytes); false otherwise or when encoding fails.
bool encode_square_map(TmaDesc* out, const double* base, int n) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
    if (!enc || n < 1 || n % 2 != 0 || !aligned16(base)) return false;
    const cuuint64_t dim[2] = {(cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t pitch[1] = {(cuuint64_t)n * sizeof(double)};
    const cuuint32_t box[2] = {16, 64}, es[2] = {1, 1};
    return enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dim, pitch, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The tensor map k_sp2_step_tc1 reads an FP32 iterate through: n rows of ldf floats (ldf a multiple
// of 4, so the row pitch is a multiple of 16 bytes), boxes of 32 floats (128 bytes) x 128 rows,
// 128-byte swizzle, zero fill past the edges.
bool encode_rows_map_f32(TmaDesc* out, const float* base, int ldf, int n) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
    if (!enc || n < 1 || ldf % 4 != 0 || !aligned16(base)) return false;
    const cuuint64_t dim[2] = {(cuuint64_t)ldf, (cuuint64_t)n};
    const cuuint64_t pitch[1] = {(cuuint64_t)ldf * sizeof(float)};
    const cuuint32_t box[2] = {32, 128}, es[2] = {1, 1};
    return enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dim, pitch, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// k_bisect for njobs matrices of at most maxn rows: a warp per eigenvalue while the whole launch stays
// within about two waves of resident threads (one molecule, small batches), a thread per eigenvalue
// otherwise (the warp form does about seven times the work, so it only pays when the GPU is idle).
// warp_ok = false keeps the thread-per-eigenvalue bisection: the eigenvalues that seed inverse
// iteration (whose cluster treatment was tuned on them).
void bisect_launch(const TriJob* jobs, int njobs, int maxn, cudaStream_t s, bool warp_ok) {
    constexpr long long kTwoWaves = 2LL * 148 * 2048;  // resident threads of two waves on a B200
    const int lanes = warp_ok && (long long)njobs * maxn * 32 <= kTwoWaves ? 32 : 1;
    const int per_block = 512 / lanes;
    k_bisect<<<dim3(njobs, (maxn + per_block - 1) / per_block), 512, 2 * sizeof(double) * maxn, s>>>(jobs, nullptr, lanes);
}

inline int oz_ldq(int n) { return (n + 15) & ~15; }
inline int oz_tiles_of(int n) {  // 128 x 48 tiles with an element on or above the diagonal
    int k = 0;
    for (int tm = 0; tm < (n + 127) / 128; ++tm)
        for (int tn = 0; tn < (n + 47) / 48; ++tn)
            if (48 * tn + 47 >= 128 * tm) ++k;
    return k;
}

int lowp_tc_env() {
    static const int v = [] {
        const char* e = std::getenv("AM1GPU_LOWP_TC");
        return e ? std::atoi(e) : -1;
    }();
    return v;
}

int lowp_tc_for(int n) {
    const int env = lowp_tc_env();
    if (env >= 0) return env == 0 ? 0 : (env == 2 && tma_encoder()) ? 2 : 1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    const int c = g_lowp_tune[dev].choice[tune_class(n)];
    return c >= 0 ? c : 1;  // untuned classes (the tuner could not run) take the FP32-accurate tcgen05 kernel
}

int density_mode() {
    static const int mode = [] {
        const char* e = std::getenv("AM1GPU_DENSITY");
        return (e && std::strcmp(e, "jacobi") == 0) ? 1 : 0;
    }();
    return mode;
}

// Matrices too large for a cluster's shared memory (tridiagonalisation, Lanczos bounds): one of
// at least kBigGridN orbitals takes the whole GPU (a cooperative launch each); all the others of
// the batch get a cluster of big_cluster(count) CTAs each, in one launch.
// AM1GPU_BIG=grid / cluster forces one form (for measurements).
constexpr int kBigGridN = 2048;

bool big_on_grid(int n) {
    static const int force = [] {
        const char* e = std::getenv("AM1GPU_BIG");
        if (e && std::strcmp(e, "grid") == 0) return 1;
        if (e && std::strcmp(e, "cluster") == 0) return 2;
        return 0;
    }();
    if (force) return force == 1;
    return n >= kBigGridN;
}

// Cluster size for `count` matrices: about two CTAs of 512 threads per SM in all.
int big_cluster(int count, int sms) {
    int C = 16;
    while (C > 4 && (long long)C * count > 2LL * sms) C /= 2;
    return C;
}

struct Run {
    Mem* mem;
    am1gpu_call_stats* stats;
    bool timed;
    size_t next_ev = 0;
    std::vector<std::pair<int, std::pair<size_t, size_t>>> spans;  // phase, (start, stop) event slots
    size_t t0 = 0, t1 = 0;

    int event(size_t* slot) {
        if (next_ev == mem->events.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            mem->events.push_back(e);
        }
        *slot = next_ev++;
        CK(cudaEventRecord(mem->events[*slot], mem->stream));
        return AM1GPU_OK;
    }
    int begin(size_t* slot) { return timed ? event(slot) : AM1GPU_OK; }
    int end(int phase, size_t start) {
        if (!timed) return AM1GPU_OK;
        size_t stop;
        int rc = event(&stop);
        if (rc) return rc;
        spans.push_back({phase, {start, stop}});
        return AM1GPU_OK;
    }
    void launched(int phase, int k = 1) {
        stats->kernel_launches += k;
        stats->phase_launches[phase] += k;
    }
    // after the stream has been synchronized
    int collect() {
        for (auto& sp : spans) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, mem->events[sp.second.first], mem->events[sp.second.second]));
            stats->phase_ms[sp.first] += ms;
        }
        return AM1GPU_OK;
    }
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------------------
// Batch planning
// ---------------------------------------------------------------------------------------
struct MolPlan {
    int user;          // index in the caller's array
    int natoms, nheavy, nao, nch, n_occ[2], npad, cluster;
    std::vector<int> order;  // internal atom -> caller atom
    std::vector<int> ao_map; // internal AO -> caller AO
};

// Rows of a channel's VS slot (n doubles each): the eigensolver's npad vectors, and room for the
// mixed path's two FP32 iterates of n rows of (n rounded up to 4) floats plus 16-byte alignment.
long long vs_rows(const MolPlan& p) { return std::max<long long>(p.npad, ((p.nao + 3) & ~3) + 2); }

// Largest molecule (orbitals) the purification path takes: the Lanczos bounds and the bisection hold
// 3 n and 2 n doubles in one CTA's shared memory.
constexpr int kMaxAo = 8192;
int density_mode();

int choose_cluster(int n, int* npad_out, int* c_out) {
    static const int cs[5] = {1, 2, 4, 8, 16};
    for (int k = 0; k < 5; ++k) {
        const int C = cs[k];
        const int npad = ((std::max(n, 2) + 2 * C - 1) / (2 * C)) * (2 * C);
        const int q = npad / 2 / C;
        if (C > 1 && q < 2) continue;
        if ((long long)jacobi_smem_bytes(n, npad, C) <= g_jacobi_budget) {
            *npad_out = npad;
            *c_out = C;
            return 1;
        }
    }
    return 0;
}

// Validates one molecule exactly as run_am1's head does (src/scf.rs:294-366) and plans it.
// tab_all: the call's [method][Z] host table (NULL: the built-in one).
int plan_molecule(const am1gpu_molecule& m, const am1gpu_options& o, int user, MolPlan& p, const DevElem* tab_all = nullptr) {
    if (m.natoms < 0 || (m.natoms > 0 && (!m.z || !m.xyz_bohr))) return fail(AM1GPU_INVALID_INPUT, "null molecule arrays");
    if (m.multiplicity < 1) return fail(AM1GPU_INVALID_INPUT, "multiplicity must be >= 1");
    const int method = o.method == AM1GPU_METHOD_RM1 ? 1 : 0;
    const DevElem* tab = (tab_all ? tab_all : host_param_table()) + method * (MAX_Z + 1);  // once, not per atom
    for (int i = 0; i < m.natoms; ++i) {
        const int z = m.z[i];
        if (z < 0 || z > MAX_Z || !tab[z].present) {
            std::string sup;
            for (int k = 1; k <= MAX_Z; ++k)
                if (tab[k].present) sup += (sup.empty() ? "" : ", ") + std::string(kSymbols[k]);
            const char* name = method ? "RM1" : "AM1";
            return fail(AM1GPU_ELEMENT_NOT_PARAMETERIZED, std::string(name) + " has no parameters for element Z=" +
                                                              std::to_string(z) + "; " + name + " covers " + sup);
        }
        if (!std::isfinite(m.xyz_bohr[3 * i]) || !std::isfinite(m.xyz_bohr[3 * i + 1]) || !std::isfinite(m.xyz_bohr[3 * i + 2]))
            return fail(AM1GPU_INVALID_INPUT, "non-finite coordinate for atom " + std::to_string(i));
    }
    double n_elec = 0.0;
    for (int i = 0; i < m.natoms; ++i) n_elec += tab[m.z[i]].core_charge;
    n_elec -= m.charge;
    const long long ne = (long long)std::llround(n_elec);
    if (std::fabs(n_elec - (double)ne) > 1.0e-6 || ne < 0)
        return fail(AM1GPU_INVALID_INPUT, "invalid electron count " + std::to_string(n_elec));
    const long long unp = m.multiplicity - 1;
    if ((ne - unp) < 0 || (ne - unp) % 2 != 0)
        return fail(AM1GPU_INVALID_INPUT, "electron count " + std::to_string(ne) + " is incompatible with multiplicity " +
                                              std::to_string(m.multiplicity) + " (need same parity)");
    const int n_alpha = (int)((ne + unp) / 2), n_beta = (int)((ne - unp) / 2);
    const bool closed = n_alpha == n_beta;
    bool uhf;
    if (o.reference == AM1GPU_REF_AUTO) uhf = !closed;
    else if (o.reference == AM1GPU_REF_UHF) uhf = true;
    else {
        if (!closed)
            return fail(AM1GPU_INVALID_INPUT, "restricted (RHF) reference requires a closed shell, but multiplicity " +
                                                  std::to_string(m.multiplicity) + " gives " + std::to_string(n_alpha) +
                                                  " alpha and " + std::to_string(n_beta) +
                                                  " beta electrons; use the unrestricted (UHF) reference for open-shell systems");
        uhf = false;
    }
    p.user = user;
    p.natoms = m.natoms;
    p.nch = uhf ? 2 : 1;
    p.n_occ[0] = n_alpha;
    p.n_occ[1] = uhf ? n_beta : n_alpha;
    p.order.clear();
    for (int i = 0; i < m.natoms; ++i)
        if (tab[m.z[i]].norb == 4) p.order.push_back(i);
    p.nheavy = (int)p.order.size();
    for (int i = 0; i < m.natoms; ++i)
        if (tab[m.z[i]].norb != 4) p.order.push_back(i);
    p.nao = 4 * p.nheavy + (m.natoms - p.nheavy);
    // caller AO offsets
    std::vector<int> uoff(m.natoms);
    int acc = 0;
    for (int i = 0; i < m.natoms; ++i) {
        uoff[i] = acc;
        acc += tab[m.z[i]].norb;
    }
    p.ao_map.assign(p.nao, 0);
    int k = 0;
    for (int ia = 0; ia < m.natoms; ++ia) {
        const int u = p.order[ia];
        const int no = tab[m.z[u]].norb;
        for (int t = 0; t < no; ++t) p.ao_map[k++] = uoff[u] + t;
    }
    if (!choose_cluster(p.nao, &p.npad, &p.cluster)) {
        // larger than the cluster eigensolver holds: the purification SCF and the final spectrum
        // (grid-wide tridiagonalisation) still run, and eigenvectors on request come from the
        // large-matrix path; the per-iteration eigensolver density path does not run
        if (p.nao > kMaxAo)
            return fail(AM1GPU_UNSUPPORTED, "molecule with " + std::to_string(p.nao) + " orbitals exceeds the limit of " +
                                                std::to_string(kMaxAo));
        if (density_mode() != 0)
            return fail(AM1GPU_UNSUPPORTED, "the eigensolver density path holds at most 448 orbitals; this molecule has " +
                                                std::to_string(p.nao));
        p.cluster = 0;
        p.npad = p.nao;
    }
    return AM1GPU_OK;
}

struct Batch {
    int nmol = 0, natoms = 0, nblk = 1, maxn = 0;
    long long npairs = 0;
    std::vector<MolPlan> plans;
    // device pointers (into the pool)
    MolDesc* d_mols;
    int *d_atom_z, *d_atom_mol;
    double* d_atom_xyz;
    long long* d_pair_prefix;
    ChanJob* d_jobs;
    int* d_job0;
    GemmJob *d_gj_gt, *d_gj_dn;
    GemmTile *d_gt_gt, *d_gt_dn;
    int nt_gt = 0, nt_dn = 0;
    EigJob* d_eig;
    int neig = 0;
    struct Bucket { int off, count, C; size_t smem; };
    std::vector<Bucket> buckets;      // eigensolver jobs by cluster size
    std::vector<Bucket> tri_buckets;  // tridiagonalisation jobs by cluster size
    std::vector<TriJob> tri_big;      // matrices too large for a cluster's shared memory (d_tri[0 .. count))
    std::vector<int> sp2_big;         // purification jobs of those matrices (d_sp2_big), largest first
    int* d_sp2_big;
    Sp2Job* d_sp2;
    GemmTile* d_sp2_tiles;  // upper-triangle tiles: the pair-copy jobs' first, then the others
    TmaDesc* d_sp2_maps;    // tensor maps of every pair-copy job's X0, X1, F, P (4 per job)
    TmaDesc* d_xf_maps;     // tensor maps of the FP32 iterates Xf0, Xf1 of every single-pass tcgen05 job (2 per job)
    bool sp2_tma = false;   // the pair-copy tiles run k_sp2_step_tma and k_commutator_tma (every map encoded)
    bool has_tc3 = false, has_tc1 = false;  // some job's reduced-precision products run k_sp2_step_tc / _tc1
    int nt_sp2 = 0, nt_sp2_pairs = 0, sp2_nblk = 1;
    GemmTile* d_tc_tiles = nullptr;  // 128 x 128 upper-triangle tiles of the tcgen05 reduced-precision step
    int nt_tc = 0;
    GemmTile* d_oz_tiles = nullptr;  // 128 x 48 tiles of the digit-plane FP64 step
    int nt_oz = 0;
    Sp2State* d_sp2_state;
    TriJob* d_tri;
    int* d_need_eigen;
    int* d_sp2_active;
    double* d_work;  // [0] purification steps, [1] their flops, [2] eigensolver fallbacks, [3] their bytes,
                     // [4] TF32 purification steps, [5] their flops
    MolState* d_st;
    int* d_status;
    double *d_wstore, *d_ecc, *d_arena, *d_res, *d_charges;
    int* d_active;
    // host mirrors needed for output
    std::vector<MolDesc> mols;
    std::vector<ChanJob> jobs;
    std::vector<int> job0;
    int* h_active;
    double* h_work;
    double* h_res;
    double* h_charges;
    double* d_eps;  // every channel's orbital energies, contiguous (job order)
    double* h_eps;  // their pinned host copy
    double* d_grad;  // nuclear gradient, 3 per atom (internal atom order), when asked for
    double* h_grad;
    long long eps_total = 0;
    long long arena_doubles = 0;
    const DevElem* d_params = nullptr;  // the call's own parameter table (staged with the inputs), or NULL: the built-in upload
    int* d_big_stall = nullptr;  // per channel job: 1 when a large molecule's purification stalled this iteration
    GraphLoop* d_loop = nullptr;  // loop counters of the captured solve
    GraphLoop* h_loop = nullptr;  // their pinned host copy
    // kernels per captured head (+ arm), step (+ condition), tail (+ its two control kernels), and
    // stalled-purification eigensolver (run in GraphLoop::eig_runs iterations)
    int64_t graph_counts[4] = {0, 0, 0, 0};
    bool graph_cacheable = false;  // a resident batch keeps its instantiated graph across runs
    cudaGraphExec_t graph_exec = nullptr;
};

// Lays out the batch in one device pool and one pinned staging area, copies inputs.
int build_batch(const am1gpu_molecule* in, const am1gpu_options& o, std::vector<MolPlan>&& plans, Batch& b, Mem& mem,
                am1gpu_call_stats* stats, double spin_scale_override = -1.0, const DevElem* host_tab = nullptr) {
    b.plans = std::move(plans);
    b.nmol = (int)b.plans.size();
    const int method = o.method == AM1GPU_METHOD_RM1 ? 1 : 0;
    const bool adiis = o.use_diis && o.accelerator == AM1GPU_ACCEL_ADIIS_CDIIS;
    // sizes
    long long natoms = 0, npairs = 0, wsize = 0, arena = 0, hist = 0, nch_total = 0;
    int maxn = 0;
    for (auto& p : b.plans) {
        natoms += p.natoms;
        npairs += (long long)p.natoms * (p.natoms - 1) / 2;
        const long long h = p.nheavy, H = p.natoms - p.nheavy;
        wsize += 100 * h * (h - 1) / 2 + 10 * h * H + H * (H - 1) / 2;
        const long long nn = (long long)p.nao * p.nao;
        arena += nn + p.nch * (5 * nn + (long long)vs_rows(p) * p.nao) + 64;
        const long long ls = packed_sym_len(p.nao), la = packed_anti_len(p.nao);
        hist += p.nch * MAX_DIIS * (ls + la + ((adiis && p.nch == 1) ? ls : 0)) + 64;
        nch_total += p.nch;
        maxn = std::max(maxn, p.nao);
    }
    b.natoms = (int)natoms;
    b.npairs = npairs;
    b.maxn = maxn;
    b.nblk = std::max(1, std::min(32, (maxn + 15) / 16));
    const int nblk = b.nblk;
    // GEMM tile counts
    int tiles_nn = 0, tiles_up = 0, tiles_tc = 0, tiles_oz = 0;
    long long dq_bytes = 0;
    const bool mixed = o.precision == AM1GPU_PRECISION_MIXED;
    for (auto& p : b.plans) {
        const int tn = (p.nao + 63) / 64;
        tiles_nn += p.nch * tn * tn;
        tiles_up += p.nch * tn * (tn + 1) / 2;
        const int tc = (p.nao + 127) / 128;
        if (mixed && lowp_tc_for(p.nao) != 0) tiles_tc += p.nch * tc * (tc + 1) / 2;
        if (fp64_oz_for(p.nao)) {
            tiles_oz += p.nch * oz_tiles_of(p.nao);
            dq_bytes += p.nch * (2LL * kOzPlanes * p.nao * oz_ldq(p.nao) + 256);
        }
    }
    const int sp2_nblk = std::max(1, std::min(32, (maxn + 7) / 8));
    // ---- staged (host -> device) region layout
    size_t st = 0;
    auto take = [](size_t& cur, size_t bytes) {
        cur = align256(cur);
        const size_t o2 = cur;
        cur += bytes;
        return o2;
    };
    const size_t o_mols = take(st, sizeof(MolDesc) * b.nmol);
    const size_t o_z = take(st, sizeof(int) * natoms);
    const size_t o_am = take(st, sizeof(int) * natoms);
    const size_t o_xyz = take(st, sizeof(double) * 3 * natoms);
    const size_t o_pp = take(st, sizeof(long long) * (b.nmol + 1));
    const size_t o_jobs = take(st, sizeof(ChanJob) * nch_total);
    const size_t o_job0 = take(st, sizeof(int) * b.nmol);
    const size_t o_ggt = take(st, sizeof(GemmJob) * nch_total);
    const size_t o_gdn = take(st, sizeof(GemmJob) * nch_total);
    const size_t o_tgt = take(st, sizeof(GemmTile) * tiles_nn);
    const size_t o_tdn = take(st, sizeof(GemmTile) * tiles_nn);
    const size_t o_eig = take(st, sizeof(EigJob) * nch_total);
    const size_t o_sp2 = take(st, sizeof(Sp2Job) * nch_total);
    const size_t o_sp2t = take(st, sizeof(GemmTile) * std::max(tiles_up, 1));
    const size_t o_maps = take(st, sizeof(TmaDesc) * 4 * std::max<long long>(nch_total, 1));
    const size_t o_xfmaps = take(st, mixed ? sizeof(TmaDesc) * 2 * std::max<long long>(nch_total, 1) : sizeof(TmaDesc) * 2);
    const size_t o_tct = take(st, sizeof(GemmTile) * std::max(tiles_tc, 1));
    const size_t o_ozt = take(st, sizeof(GemmTile) * std::max(tiles_oz, 1));
    const size_t o_tri = take(st, sizeof(TriJob) * 5 * nch_total);  // the jobs, then up to 4 continuations each
    const size_t o_sp2big = take(st, sizeof(int) * nch_total);
    const size_t o_st = take(st, sizeof(MolState) * b.nmol);
    const size_t par_bytes = host_tab ? sizeof(DevElem) * 2 * (MAX_Z + 1) : 0;
    const size_t o_par = take(st, par_bytes);
    const size_t staged = align256(st);
    // ---- device-only region
    size_t dv = staged;
    const size_t o_status = take(dv, sizeof(int) * b.nmol);
    const size_t o_need = take(dv, sizeof(int) * b.nmol);
    const size_t o_sp2a = take(dv, sizeof(int) * 4);
    const size_t o_work = take(dv, sizeof(double) * kWorkN);
    const size_t o_sp2s = take(dv, sizeof(Sp2State) * nch_total);
    const size_t o_active = take(dv, sizeof(int) * 4);
    const size_t o_w = take(dv, sizeof(double) * std::max<long long>(wsize, 1));
    const size_t o_ecc = take(dv, sizeof(double) * std::max<long long>(npairs, 1));
    const size_t o_arena = take(dv, sizeof(double) * arena);
    const size_t o_hist = take(dv, sizeof(double) * hist);
    long long misc = 0;
    for (auto& p : b.plans) {
        const long long tn = (p.nao + 63) / 64;
        const long long sp2part = 2 * std::max<long long>(sp2_nblk, tn * (tn + 1) / 2);
        const long long cpart = CP_N * tn * (tn + 1) / 2;
        misc += p.nch * (5LL * p.nao + p.npad + (long long)nblk * (RED_N + 1) + sp2part + cpart + 4 + 128);
    }
    const size_t o_misc = take(dv, sizeof(double) * misc);
    const size_t o_colid = take(dv, sizeof(int) * (size_t)(nch_total * (b.maxn + 64)));
    const size_t o_res = take(dv, sizeof(double) * RES_N * b.nmol);
    const size_t o_chg = take(dv, sizeof(double) * std::max<long long>(natoms, 1));
    long long eps_total = 0;
    for (auto& p : b.plans) eps_total += (long long)p.nch * p.nao;
    const size_t o_eps = take(dv, sizeof(double) * std::max<long long>(eps_total, 1));
    const size_t o_grad = take(dv, sizeof(double) * 3 * std::max<long long>(natoms, 1));
    const size_t o_bstall = take(dv, sizeof(int) * std::max<long long>(nch_total, 1));
    const size_t o_loop = take(dv, sizeof(GraphLoop));
    const size_t o_dq = take(dv, (size_t)std::max<long long>(dq_bytes, 16));
    const size_t dtotal = align256(dv);
    // pinned staging also receives the outputs
    size_t hs = staged;
    const size_t h_o_active = take(hs, sizeof(int) * 4);
    const size_t h_o_work = take(hs, sizeof(double) * kWorkN);
    const size_t h_o_res = take(hs, sizeof(double) * RES_N * b.nmol);
    const size_t h_o_chg = take(hs, sizeof(double) * std::max<long long>(natoms, 1));
    const size_t h_o_eps = take(hs, sizeof(double) * std::max<long long>(eps_total, 1));
    const size_t h_o_grad = take(hs, sizeof(double) * 3 * std::max<long long>(natoms, 1));
    const size_t h_o_loop = take(hs, sizeof(GraphLoop));
    int rc = mem_ensure(mem, dtotal, align256(hs));
    if (rc) return rc;
    Mem* ws = &mem;
    char* D = ws->dpool;
    char* Hs = ws->hpin;
    auto dptr = [D](size_t off) { return (void*)(D + off); };
    b.d_mols = (MolDesc*)dptr(o_mols);
    b.d_atom_z = (int*)dptr(o_z);
    b.d_atom_mol = (int*)dptr(o_am);
    b.d_atom_xyz = (double*)dptr(o_xyz);
    b.d_pair_prefix = (long long*)dptr(o_pp);
    b.d_jobs = (ChanJob*)dptr(o_jobs);
    b.d_job0 = (int*)dptr(o_job0);
    b.d_gj_gt = (GemmJob*)dptr(o_ggt);
    b.d_gj_dn = (GemmJob*)dptr(o_gdn);
    b.d_gt_gt = (GemmTile*)dptr(o_tgt);
    b.d_gt_dn = (GemmTile*)dptr(o_tdn);
    b.d_eig = (EigJob*)dptr(o_eig);
    b.d_sp2 = (Sp2Job*)dptr(o_sp2);
    b.d_sp2_tiles = (GemmTile*)dptr(o_sp2t);
    b.d_sp2_maps = (TmaDesc*)dptr(o_maps);
    TmaDesc* hmaps = (TmaDesc*)(Hs + o_maps);
    b.sp2_tma = tma_encoder() != nullptr;
    b.d_xf_maps = (TmaDesc*)dptr(o_xfmaps);
    TmaDesc* hxfmaps = (TmaDesc*)(Hs + o_xfmaps);
    b.d_tc_tiles = (GemmTile*)dptr(o_tct);
    GemmTile* htct = (GemmTile*)(Hs + o_tct);
    int ntc = 0;
    b.d_oz_tiles = (GemmTile*)dptr(o_ozt);
    GemmTile* hozt = (GemmTile*)(Hs + o_ozt);
    int noz = 0;
    long long dq_off = 0;
    b.d_tri = (TriJob*)dptr(o_tri);
    b.d_sp2_big = (int*)dptr(o_sp2big);
    b.d_need_eigen = (int*)dptr(o_need);
    b.d_sp2_active = (int*)dptr(o_sp2a);
    b.d_work = (double*)dptr(o_work);
    b.d_sp2_state = (Sp2State*)dptr(o_sp2s);
    b.sp2_nblk = sp2_nblk;
    b.d_st = (MolState*)dptr(o_st);
    b.d_status = (int*)dptr(o_status);
    b.d_active = (int*)dptr(o_active);
    b.d_wstore = (double*)dptr(o_w);
    b.d_ecc = (double*)dptr(o_ecc);
    b.d_arena = (double*)dptr(o_arena);
    double* d_hist = (double*)dptr(o_hist);
    double* d_misc = (double*)dptr(o_misc);
    int* d_colid = (int*)dptr(o_colid);
    b.d_res = (double*)dptr(o_res);
    b.d_charges = (double*)dptr(o_chg);
    b.d_eps = (double*)dptr(o_eps);
    b.d_grad = (double*)dptr(o_grad);
    b.d_big_stall = (int*)dptr(o_bstall);
    b.d_loop = (GraphLoop*)dptr(o_loop);
    b.h_loop = (GraphLoop*)(Hs + h_o_loop);
    b.eps_total = eps_total;
    b.h_active = (int*)(Hs + h_o_active);
    b.h_work = (double*)(Hs + h_o_work);
    b.h_res = (double*)(Hs + h_o_res);
    b.h_charges = (double*)(Hs + h_o_chg);
    b.h_eps = (double*)(Hs + h_o_eps);
    b.h_grad = (double*)(Hs + h_o_grad);
    b.d_params = nullptr;
    if (host_tab) {
        std::memcpy(Hs + o_par, host_tab, par_bytes);
        b.d_params = (const DevElem*)dptr(o_par);
    }
    // ---- fill the staged region
    MolDesc* hm = (MolDesc*)(Hs + o_mols);
    int* hz = (int*)(Hs + o_z);
    int* ham = (int*)(Hs + o_am);
    double* hxyz = (double*)(Hs + o_xyz);
    long long* hpp = (long long*)(Hs + o_pp);
    ChanJob* hj = (ChanJob*)(Hs + o_jobs);
    int* hj0 = (int*)(Hs + o_job0);
    GemmJob* hggt = (GemmJob*)(Hs + o_ggt);
    GemmJob* hgdn = (GemmJob*)(Hs + o_gdn);
    GemmTile* htgt = (GemmTile*)(Hs + o_tgt);
    GemmTile* htdn = (GemmTile*)(Hs + o_tdn);
    EigJob* heig = (EigJob*)(Hs + o_eig);
    Sp2Job* hsp2 = (Sp2Job*)(Hs + o_sp2);
    GemmTile* hsp2t = (GemmTile*)(Hs + o_sp2t);
    TriJob* htri = (TriJob*)(Hs + o_tri);
    std::vector<GemmTile> tiles_pairs, tiles_other;  // jobs with even n and 16-byte aligned slots / the rest
    MolState* hst = (MolState*)(Hs + o_st);
    long long a_off = 0, w_off = 0, ar_off = 0, hi_off = 0, mi_off = 0, eps_off = 0;
    int atom_base = 0, job = 0, ntile = 0, cid_off = 0;
    std::vector<EigJob> eig_all;
    std::vector<int> eig_cluster;
    std::vector<TriJob> tri_all;
    b.sp2_big.clear();
    for (int mi = 0; mi < b.nmol; ++mi) {
        MolPlan& p = b.plans[mi];
        const am1gpu_molecule& m = in[p.user];
        MolDesc md{};
        md.natoms = p.natoms;
        md.nheavy = p.nheavy;
        md.nao = p.nao;
        md.nch = p.nch;
        md.n_occ[0] = p.n_occ[0];
        md.n_occ[1] = p.n_occ[1];
        md.method = method;
        md.atom_base = atom_base;
        md.pair_base = a_off;
        md.w_base = w_off;
        md.spin_scale = p.nch == 2 ? 1.0 : 0.5;
        md.occ_weight = p.nch == 2 ? 1.0 : 2.0;
        if (spin_scale_override >= 0.0) md.spin_scale = spin_scale_override;
        const long long n = p.nao, nn = n * n;
        md.h_base = ar_off;
        long long cur = ar_off + nn;
        for (int c = 0; c < p.nch; ++c) {
            md.ch_base[c] = cur;
            cur += 5 * nn + (long long)vs_rows(p) * n;
        }
        ar_off = (cur + 31) & ~31LL;
        for (int ia = 0; ia < p.natoms; ++ia) {
            const int u = p.order[ia];
            hz[atom_base + ia] = m.z[u];
            ham[atom_base + ia] = mi;
            for (int k = 0; k < 3; ++k) hxyz[3 * (atom_base + ia) + k] = m.xyz_bohr[3 * u + k];
        }
        hpp[mi] = a_off;
        const long long h = p.nheavy, H = p.natoms - p.nheavy;
        a_off += (long long)p.natoms * (p.natoms - 1) / 2;
        w_off += 100 * h * (h - 1) / 2 + 10 * h * H + H * (H - 1) / 2;
        atom_base += p.natoms;
        hj0[mi] = job;
        const long long ls = packed_sym_len((int)n), la = packed_anti_len((int)n);
        for (int c = 0; c < p.nch; ++c) {
            double* base = b.d_arena + md.ch_base[c];
            ChanJob cj{};
            cj.mol = mi;
            cj.ch = c;
            cj.n = (int)n;
            cj.F = base + SLOT_F * nn;
            cj.Fx = base + SLOT_FX * nn;
            cj.P = base + SLOT_P * nn;
            cj.Ct = base + SLOT_CT * nn;
            cj.Pnew = base + SLOT_GT * nn;
            cj.H = b.d_arena + md.h_base;
            md.pk_base[c] = hi_off;
            cj.hF = d_hist + hi_off;
            hi_off += MAX_DIIS * ls;
            cj.hE = d_hist + hi_off;
            hi_off += MAX_DIIS * la;
            cj.hD = nullptr;
            if (adiis && p.nch == 1) {
                cj.hD = d_hist + hi_off;
                hi_off += MAX_DIIS * ls;
            }
            hi_off = (hi_off + 31) & ~31LL;
            cj.rowmin = d_misc + mi_off;
            mi_off += n;
            cj.rowmax = d_misc + mi_off;
            mi_off += n;
            cj.rowdf = d_misc + mi_off;
            mi_off += n;
            cj.eps = b.d_eps + eps_off;
            eps_off += n;
            double* tri_d = d_misc + mi_off;
            mi_off += n;
            double* tri_e = d_misc + mi_off;
            mi_off += n;
            const long long tn_ = (n + 63) / 64;
            double* sp2part = d_misc + mi_off;
            mi_off += 2 * std::max<long long>(sp2_nblk, tn_ * (tn_ + 1) / 2);
            double* sp2bounds = d_misc + mi_off;
            mi_off += 4;
            double* lam = d_misc + mi_off;
            mi_off += p.npad;
            cj.red = d_misc + mi_off;
            mi_off += (long long)nblk * RED_N;
            cj.red2 = d_misc + mi_off;
            mi_off += nblk;
            cj.ntiles = (int)(tn_ * (tn_ + 1) / 2);
            cj.cpart = d_misc + mi_off;
            mi_off += (long long)CP_N * cj.ntiles;
            mi_off = (mi_off + 31) & ~31LL;
            hj[job] = cj;
            Sp2Job sj{};
            sj.F = cj.Fx;
            sj.rowmin = cj.rowmin;
            sj.rowmax = cj.rowmax;
            sj.rowdf = cj.rowdf;
            sj.X0 = base + SLOT_GT * nn;
            sj.X1 = base + SLOT_VS * nn;
            sj.P = cj.Pnew;
            sj.part = sp2part;
            sj.bounds = sp2bounds;
            sj.nocc = (double)p.n_occ[c];
            sj.weight = md.occ_weight;
            sj.n = (int)n;
            sj.mol = mi;
            // the purification and commutator kernels copy 16-byte pairs when every row of X0, X1,
            // F and P starts on 16 bytes: even n (slot bases are then 16-byte aligned too)
            const bool pairs = n % 2 == 0 && aligned16(sj.X0) && aligned16(sj.X1) && aligned16(cj.F) && aligned16(cj.P);
            std::vector<GemmTile>& tl = pairs ? tiles_pairs : tiles_other;
            if (pairs && b.sp2_tma)
                b.sp2_tma = encode_square_map(&hmaps[4 * job], sj.X0, (int)n) && encode_square_map(&hmaps[4 * job + 1], sj.X1, (int)n) &&
                            encode_square_map(&hmaps[4 * job + 2], cj.F, (int)n) && encode_square_map(&hmaps[4 * job + 3], cj.P, (int)n);
            sj.fallback = p.cluster > 0;
            sj.ldf = (int)((n + 3) & ~3LL);  // FP32 iterates of the mixed path: in the VS slot, 16-byte aligned
            sj.Xf0 = (float*)(((uintptr_t)(base + SLOT_VS * nn) + 15) & ~(uintptr_t)15);
            sj.Xf1 = sj.Xf0 + n * sj.ldf;
            sj.lowp_tc = mixed ? lowp_tc_for((int)n) : 0;
            if (sj.lowp_tc == 2 && !(encode_rows_map_f32(&hxfmaps[2 * job], sj.Xf0, sj.ldf, (int)n) &&
                                     encode_rows_map_f32(&hxfmaps[2 * job + 1], sj.Xf1, sj.ldf, (int)n)))
                sj.lowp_tc = 1;  // no tensor maps: the 3xTF32 kernel
            if (sj.lowp_tc == 1) b.has_tc3 = true;
            if (sj.lowp_tc == 2) b.has_tc1 = true;
            sj.tc_tile0 = ntc;
            if (sj.lowp_tc) {
                const int tc = (int)((n + 127) / 128);
                for (int x = 0; x < tc; ++x)
                    for (int y = x; y < tc; ++y) htct[ntc++] = GemmTile{job, x, y};
            }
            sj.tc_ntiles = ntc - sj.tc_tile0;
            sj.oz = fp64_oz_for((int)n) ? 1 : 0;
            sj.oz_tile0 = noz;
            sj.ldq = oz_ldq((int)n);
            sj.Dq0 = sj.Dq1 = nullptr;
            if (sj.oz) {
                for (int tm = 0; tm < (int)((n + 127) / 128); ++tm)
                    for (int tn = 0; tn < (int)((n + 47) / 48); ++tn)
                        if (48 * tn + 47 >= 128 * tm) hozt[noz++] = GemmTile{job, tm, tn};
                const long long pl = (long long)kOzPlanes * n * sj.ldq;
                sj.Dq0 = (int8_t*)dptr(o_dq) + dq_off;
                sj.Dq1 = sj.Dq0 + pl;
                dq_off += 2 * pl + 256;
            }
            sj.oz_ntiles = noz - sj.oz_tile0;
            if (!sj.fallback) b.sp2_big.push_back(job);
            sj.tile0 = (int)tl.size();  // tile index inside its own launch
            for (int x = 0; x < (int)tn_; ++x)
                for (int y = x; y < (int)tn_; ++y) tl.push_back(GemmTile{job, x, y});
            sj.ntiles = (int)tl.size() - sj.tile0;
            hsp2[job] = sj;
            TriJob tj{};
            tj.A = cj.Fx;
            tj.W = base + SLOT_GT * nn;    // large matrices: the working copy (free after the SCF)
            tj.work = base + SLOT_VS * nn;  // and the scratch vectors
            tj.d = tri_d;
            tj.e = tri_e;
            tj.eps = cj.eps;
            tj.n = (int)n;
            tj.mol = mi;
            tri_all.push_back(tj);
            // GEMMs of the eigensolver path: C^T F*, w C_occ^T C_occ
            hggt[job] = GemmJob{cj.Ct, cj.Fx, base + SLOT_GT * nn, (int)n, (int)n, (int)n, (int)n, (int)n, (int)n, 1.0, mi};
            hgdn[job] = GemmJob{cj.Ct, cj.Ct, cj.Pnew, (int)n, (int)n, p.n_occ[c], (int)n, (int)n, (int)n, md.occ_weight, mi};
            const int tn = (int)((n + 63) / 64);
            for (int x = 0; x < tn; ++x)
                for (int y = 0; y < tn; ++y) {
                    htgt[ntile] = GemmTile{job, x, y};
                    htdn[ntile] = GemmTile{job, x, y};
                    ++ntile;
                }
            EigJob ej{};
            ej.Gt = base + SLOT_GT * nn;
            ej.Ct = cj.Ct;
            ej.Vs = base + SLOT_VS * nn;
            ej.lam = lam;
            ej.colid_out = d_colid + cid_off;
            cid_off += p.npad + 32;
            ej.eps = cj.eps;
            ej.Ct_out = cj.Ct;
            ej.rowmin = cj.rowmin;
            ej.sweeps_out = nullptr;
            ej.n = (int)n;
            ej.npad = p.npad;
            ej.mol = mi;
            if (p.cluster > 0) {  // large molecules have no eigensolver job
                eig_all.push_back(ej);
                eig_cluster.push_back(p.cluster);
            }
            ++job;
        }
        hm[mi] = md;
        MolState s{};
        s.active = 1;
        s.e_old = 0.0;
        s.residual = INFINITY;
        hst[mi] = s;
    }
    hpp[b.nmol] = a_off;
    b.nt_gt = b.nt_dn = ntile;
    // each launch takes its jobs' tiles largest matrix first (a job's tiles stay contiguous, in the
    // same order, so its partial sums are unchanged): the long k-loops start in the first waves and
    // the last wave holds short ones
    auto largest_first = [&](std::vector<GemmTile>& v) {
        std::vector<std::pair<int, int>> blocks;  // (first tile, job), one per job
        for (size_t i = 0; i < v.size(); ++i)
            if (i == 0 || v[i].job != v[i - 1].job) blocks.push_back({(int)i, v[i].job});
        std::stable_sort(blocks.begin(), blocks.end(),
                         [&](const std::pair<int, int>& x, const std::pair<int, int>& y) { return hsp2[x.second].n > hsp2[y.second].n; });
        std::vector<GemmTile> out;
        out.reserve(v.size());
        for (auto& bk : blocks) {
            hsp2[bk.second].tile0 = (int)out.size();
            for (int i = bk.first; i < bk.first + hsp2[bk.second].ntiles; ++i) out.push_back(v[i]);
        }
        v.swap(out);
    };
    largest_first(tiles_pairs);
    largest_first(tiles_other);
    for (size_t i = 0; i < tiles_pairs.size(); ++i) hsp2t[i] = tiles_pairs[i];
    for (size_t i = 0; i < tiles_other.size(); ++i) hsp2t[tiles_pairs.size() + i] = tiles_other[i];
    b.nt_sp2_pairs = (int)tiles_pairs.size();
    b.nt_tc = ntc;
    b.nt_oz = noz;
    b.nt_sp2 = (int)(tiles_pairs.size() + tiles_other.size());
    // eigen jobs grouped by cluster size, largest first inside a group
    std::vector<int> idx(eig_all.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
        if (eig_cluster[x] != eig_cluster[y]) return eig_cluster[x] > eig_cluster[y];
        return eig_all[x].n > eig_all[y].n;
    });
    b.buckets.clear();
    for (size_t i = 0; i < idx.size(); ++i) {
        heig[i] = eig_all[idx[i]];
        const int C = eig_cluster[idx[i]];
        const size_t sm = jacobi_smem_bytes(eig_all[idx[i]].n, eig_all[idx[i]].npad, C);
        if (b.buckets.empty() || b.buckets.back().C != C) b.buckets.push_back({(int)i, 0, C, 0});
        b.buckets.back().count++;
        b.buckets.back().smem = std::max(b.buckets.back().smem, sm);
    }
    b.neig = (int)idx.size();
    // tridiagonalisation jobs grouped by cluster size, largest first
    std::vector<int> tix(tri_all.size());
    for (size_t i = 0; i < tix.size(); ++i) tix[i] = (int)i;
    std::stable_sort(tix.begin(), tix.end(), [&](int x, int y) { return tri_all[x].n > tri_all[y].n; });
    b.tri_buckets.clear();
    b.tri_big.clear();
    // A cluster reduction of C CTAs stops once its trailing block fits C / 2 CTAs, writes it to the
    // channel's free GT slot (W), and a job on C / 2 CTAs continues from there (A = W), down to one
    // CTA: each level frees SMs for the other matrices.  Launch order: per cluster size, largest
    // first, the matrices of that size, then the continuations into it (each after its parent).
    std::vector<TriJob> conts[5];  // continuations into 1, 2, 4, 8, 16 CTAs
    int first_of[5], count_of[5];
    for (int k = 0; k < 5; ++k) first_of[k] = -1, count_of[k] = 0;
    auto lg = [](int C) { return C == 1 ? 0 : C == 2 ? 1 : C == 4 ? 2 : C == 8 ? 3 : 4; };
    for (size_t i = 0; i < tix.size(); ++i) {
        const TriJob& tj = tri_all[tix[i]];
        htri[i] = tj;
        const int C = tridiag_cluster(tj.n);
        if (!C) {  // too large for a cluster: the grid-wide kernel (these sort first)
            b.tri_big.push_back(tj);
            continue;
        }
        if (first_of[lg(C)] < 0) first_of[lg(C)] = (int)i;
        count_of[lg(C)]++;
        TriJob* parent = &htri[i];
        int n_cur = tj.n;
        for (int c = C; c > 1; c /= 2) {
            const int m = tridiag_cluster_max(c / 2);
            if (m < 8 || m >= n_cur) break;
            parent->stop = n_cur - m;
            TriJob h2 = *parent;
            h2.A = tj.W;
            h2.W = tj.W;
            h2.work = nullptr;
            h2.d = parent->d + parent->stop;
            h2.e = parent->e + parent->stop;
            h2.eps = nullptr;
            h2.n = m;
            h2.stop = 0;
            conts[lg(c / 2)].push_back(h2);
            parent = &conts[lg(c / 2)].back();
            n_cur = m;
        }
    }
    {
        // continuations go after the jobs (k_bisect reads jobs 0 .. njobs - 1), largest cluster first;
        // a parent's stop is final before it is copied, since a job's continuation is pushed after it
        size_t at = tix.size();
        int cont_first[5];
        for (int k = 4; k >= 0; --k) {
            cont_first[k] = (int)at;
            for (const TriJob& h2 : conts[k]) htri[at++] = h2;
        }
        for (int k = 4; k >= 0; --k) {
            const int C = 1 << k;
            if (count_of[k] > 0) {
                size_t sm = 0;
                for (int i = first_of[k]; i < first_of[k] + count_of[k]; ++i) sm = std::max(sm, tridiag_smem_bytes(htri[i].n, C));
                b.tri_buckets.push_back({first_of[k], count_of[k], C, sm});
            }
            if (!conts[k].empty()) {
                size_t sm = 0;
                for (const TriJob& h2 : conts[k]) sm = std::max(sm, tridiag_smem_bytes(h2.n, C));
                b.tri_buckets.push_back({cont_first[k], (int)conts[k].size(), C, sm});
            }
        }
    }
    std::stable_sort(b.sp2_big.begin(), b.sp2_big.end(), [&](int x, int y) { return hsp2[x].n > hsp2[y].n; });
    std::copy(b.sp2_big.begin(), b.sp2_big.end(), (int*)(Hs + o_sp2big));
    b.mols.assign(hm, hm + b.nmol);
    b.jobs.assign(hj, hj + job);
    b.job0.assign(hj0, hj0 + b.nmol);
    b.arena_doubles = arena;
    CK(cudaMemcpyAsync(D, Hs, staged, cudaMemcpyHostToDevice, ws->stream));
    if (stats) stats->h2d_bytes += (int64_t)staged;
    CK(cudaMemsetAsync(b.d_status, 0, sizeof(int) * b.nmol, ws->stream));
    CK(cudaMemsetAsync(b.d_arena, 0, sizeof(double) * arena, ws->stream));
    CK(cudaMemsetAsync(b.d_big_stall, 0, sizeof(int) * std::max<long long>(nch_total, 1), ws->stream));
    return AM1GPU_OK;
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

// Where the device part of the large-matrix eigensolver (eigen_large_run) leaves its results: Z
// (n x n, component i of vector k at i * n + k), the ascending eigenvalues, the two failure
// counters, and a scratch region of at least n * n doubles that is free once Z is formed.
struct LargeEig {
    double* Z;
    double* eps;
    int* counts;
    double* spare;
};

// The device part of symmetric_eigen_large.  The matrix comes from host memory (a_host, staged
// through m's pinned buffer) or from device memory (a_dev, copied on the device); everything runs
// on stream s in m's device pool, and nothing is read back.
int eigen_large_run(int n, const double* a_host, const double* a_dev, Mem& m, cudaStream_t s, LargeEig* out);

// Stalled purifications of molecules above 448 orbitals: P from the large-matrix eigensolver.
int big_fallback(Batch& b, Mem* ws);

namespace {

// The upper-triangle tile kernels run as up to two launches: the 16-byte-copy tiles, then the rest.
template <class F>
void launch_tiles(const Batch& b, cudaStream_t, F&& launch) {
    if (b.nt_sp2_pairs > 0) launch(b.d_sp2_tiles, b.nt_sp2_pairs, true);
    if (b.nt_sp2 > b.nt_sp2_pairs) launch(b.d_sp2_tiles + b.nt_sp2_pairs, b.nt_sp2 - b.nt_sp2_pairs, false);
}

int launch_core(Batch& b, Mem* ws, const DevElem* dp, Run* run) {
    cudaStream_t s = ws->stream;
    int k = 0;
    if (b.npairs > 0) {
        k_pair_integrals<<<cdiv(b.npairs, 128), 128, 0, s>>>(b.d_mols, b.nmol, b.d_pair_prefix, b.npairs, dp, b.d_atom_z,
                                                            b.d_atom_xyz, b.d_wstore, b.d_arena, b.d_ecc, b.d_status);
        ++k;
    }
    if (b.natoms > 0) {
        k_core_diag<<<cdiv(b.natoms, 128), 128, 0, s>>>(b.d_mols, b.d_atom_mol, b.natoms, dp, b.d_atom_z, b.d_wstore, b.d_arena);
        ++k;
    }
    k_core_energy<<<b.nmol, 256, 0, s>>>(b.d_mols, b.d_ecc, b.d_st);
    ++k;
    CK(cudaGetLastError());
    if (run) run->launched(AM1GPU_PHASE_CORE, k);
    return AM1GPU_OK;
}

// One cluster of C CTAs per matrix, one launch per cluster size.
int launch_tridiag(Batch& b, Mem* ws) {
    for (auto& bk : b.tri_buckets) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(bk.count * bk.C, 1, 1);
        cfg.blockDim = dim3(512, 1, 1);
        cfg.dynamicSmemBytes = bk.smem;
        cfg.stream = ws->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = bk.C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, k_tridiag, (const TriJob*)(b.d_tri + bk.off), (const int*)nullptr));
    }
    return AM1GPU_OK;
}

// Matrices on the grid-wide path: the leading ones (sizes n_of(i) descending) of at least kBigGridN
template <class NOf>
int big_split(int count, NOf n_of) {
    int k = 0;
    while (k < count && big_on_grid(n_of(k))) ++k;
    return k;
}

// one launch per grid matrix and one for all the rest
int big_launches(int grid_count, int count) { return grid_count + (count > grid_count ? 1 : 0); }

cudaError_t launch_clusters(const void* f, int C, int count, int threads, size_t smem, cudaStream_t s, void** args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(C, count, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, f, args);
}

// Lanczos bounds of the matrices without an eigensolver fallback (b.sp2_big, largest first)
int launch_big_bounds(Batch& b, cudaStream_t s) {
    const int count = (int)b.sp2_big.size();
    if (count == 0) return AM1GPU_OK;
    const Sp2Job* jobs = b.d_sp2;
    const MolState* stp = b.d_st;
    const int k = big_split(count, [&](int i) { return b.jobs[b.sp2_big[i]].n; });
    for (int i = 0; i < k; ++i) {  // one cooperative launch per matrix
        int jbig = b.sp2_big[i];
        void* args[] = {&jobs, &jbig, &stp};
        CK(cudaLaunchCooperativeKernel((const void*)k_sp2_bounds_big, dim3(g_sp2b_grid), dim3(512), args, 0, s));
    }
    if (k < count) {
        const int* big = b.d_sp2_big + k;
        void* args[] = {&jobs, &big, &stp};
        CK(launch_clusters((const void*)k_sp2_bounds_cl, big_cluster(count - k, g_sms), count - k, 512, 0, s, args));
    }
    return AM1GPU_OK;
}

// Householder reduction of the matrices too large for a cluster's shared memory (the first
// entries of d_tri, largest first)
// The whole-GPU reduction of one matrix: blocked (panels of TRP_B columns with tensor-core
// trailing updates) unless AM1GPU_TRIDIAG=unblocked selects the one-column-per-step kernel (kept
// for comparison).
bool tridiag_blocked() {
    static const bool v = [] {
        const char* e = std::getenv("AM1GPU_TRIDIAG");
        return !(e && std::strcmp(e, "unblocked") == 0);
    }();
    return v;
}

int blocked_tridiag(TriJob tj, cudaStream_t s, int64_t* launches) {
    const int n = tj.n;
    tj.work = (double*)(((uintptr_t)tj.work + 15) & ~(uintptr_t)15);  // 16-byte copies of V, W
    CK(cudaMemcpyAsync(tj.W, tj.A, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, s));
    const size_t smem = tridiag_panel_smem_bytes(n);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tridiag_panel, TRIB_THREADS, smem));
    const int grid = std::min(per_sm, 2) * g_sms;
    if (per_sm < 1 || (long long)grid * 64 < n) return fail(AM1GPU_DEVICE_ERROR, "blocked tridiagonalisation does not fit the GPU");
    for (int k = 0; k < n - 1; k += TRP_B) {
        int bw = std::min(TRP_B, n - 1 - k);
        void* args[] = {&tj, &k, &bw};
        CK(cudaLaunchCooperativeKernel((const void*)k_tridiag_panel, dim3(grid), dim3(TRIB_THREADS), args, smem, s));
        ++*launches;
        if (k + bw < n - 1) {  // not the last panel: the trailing update of [k + TRP_B, n)
            const int t0 = k + TRP_B, nt = (n - t0 + 64 - 1) / 64;
            const unsigned tiles = (unsigned)nt * (nt + 1) / 2;
            if (n % 2 == 0) k_tridiag_syr2k16<<<tiles, 128, dgemm_smem_bytes(), s>>>(tj, t0);  // 16-byte copies
            else k_tridiag_syr2k8<<<tiles, 128, dgemm_smem_bytes(), s>>>(tj, t0);
            CK(cudaGetLastError());
            ++*launches;
        }
    }
    return AM1GPU_OK;
}

int launch_big_tridiag(Batch& b, cudaStream_t s, int64_t* launches) {
    const int count = (int)b.tri_big.size();
    if (count == 0) return AM1GPU_OK;
    const int k = big_split(count, [&](int i) { return b.tri_big[i].n; });
    for (int i = 0; i < k; ++i) {  // the whole GPU per matrix
        if (tridiag_blocked()) {
            int rc = blocked_tridiag(b.tri_big[i], s, launches);
            if (rc) return rc;
            continue;
        }
        TriJob arg = b.tri_big[i];
        ++*launches;
        const size_t smem = tridiag_big_smem_bytes(arg.n);
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tridiag_big, TRIB_THREADS, smem));
        if (per_sm < 1) return fail(AM1GPU_DEVICE_ERROR, "grid tridiagonalisation does not fit an SM");
        const int grid = std::min(per_sm, 2) * g_sms;
        void* args[] = {&arg};
        CK(cudaLaunchCooperativeKernel((const void*)k_tridiag_big, dim3(grid), dim3(TRIB_THREADS), args, smem, s));
    }
    if (k < count) {
        const TriJob* jobs = b.d_tri + k;
        void* args[] = {&jobs};
        CK(launch_clusters((const void*)k_tridiag_cl, big_cluster(count - k, g_sms), count - k, TRIB_THREADS,
                           tridiag_big_smem_bytes(b.tri_big[k].n), s, args));
        ++*launches;
    }
    return AM1GPU_OK;
}

// stream: where to launch (NULL: the workspace's own stream)
int launch_jacobi(Batch& b, Mem* ws, int force, const int* mask = nullptr, cudaStream_t stream = nullptr) {
    for (auto& bk : b.buckets) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(bk.count * bk.C, 1, 1);
        cfg.blockDim = dim3(256, 1, 1);
        cfg.dynamicSmemBytes = bk.smem;
        cfg.stream = stream ? stream : ws->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = bk.C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, k_jacobi, (const EigJob*)(b.d_eig + bk.off), (const MolState*)b.d_st, b.d_status, force,
                              mask));
    }
    return AM1GPU_OK;
}

// One SCF iteration's launches, shared by the host-driven loop and the captured graph.
struct IterEnq {
    Batch& b;
    Mem* ws;
    cudaStream_t s;
    const DevElem* dp;
    ScfParams prm;
    int nblk, rowblk, njobs;
    Run* run;
    size_t ph;  // start event of the phase being timed
};

// Fock build, commutator and history, extrapolation, and (purification path) the spectral bounds
// and the start of the purification.
int enq_head(IterEnq& e, bool lowp_left) {
    (void)lowp_left;
    Batch& b = e.b;
    const cudaStream_t s = e.s;
    Run& run = *e.run;
    int rc;
    CK(cudaMemsetAsync(b.d_active, 0, 4 * sizeof(int), s));
    if ((rc = run.begin(&e.ph))) return rc;
    k_fock<<<cdiv(b.natoms, 8), 256, 0, s>>>(b.d_mols, b.d_atom_mol, b.natoms, e.dp, b.d_atom_z, b.d_wstore, b.d_arena, b.d_st, 0);
    run.launched(AM1GPU_PHASE_FOCK);
    if ((rc = run.end(AM1GPU_PHASE_FOCK, e.ph)) || (rc = run.begin(&e.ph))) return rc;
    launch_tiles(b, s, [&](const GemmTile* t, int nt, bool pairs) {
        if (pairs && b.sp2_tma)
            k_commutator_tma<<<nt, 128, dgemm_tma_smem_bytes(), s>>>(b.d_jobs, t, nt, b.d_st, b.d_sp2_maps, b.d_sp2_active + 2);
        else if (pairs)
            k_commutator16<<<nt, 128, dgemm_smem_bytes(), s>>>(b.d_jobs, t, nt, b.d_st);
        else
            k_commutator8<<<nt, 128, dgemm_smem_bytes(), s>>>(b.d_jobs, t, nt, b.d_st);
    });
    k_post_fock<<<dim3(e.nblk, e.njobs), 256, 0, s>>>(b.d_jobs, b.d_mols, b.d_st, e.nblk, 0, 0);
    run.launched(AM1GPU_PHASE_COMMUTATOR, 2);
    if ((rc = run.end(AM1GPU_PHASE_COMMUTATOR, e.ph)) || (rc = run.begin(&e.ph))) return rc;
    k_diis_solve<<<cdiv(b.nmol, 64), 64, 0, s>>>(b.d_mols, b.d_jobs, b.d_job0, b.nmol, b.d_st, b.d_status, e.nblk, e.prm);
    k_combine<<<dim3(e.rowblk, e.njobs), 256, 0, s>>>(b.d_jobs, b.d_st, 0);
    run.launched(AM1GPU_PHASE_ACCEL, 2);
    if ((rc = run.end(AM1GPU_PHASE_ACCEL, e.ph)) || (rc = run.begin(&e.ph))) return rc;
    if (density_mode() == 0) {
        // purification: P from F* by SP2, eigensolver only for molecules whose purification stalls
        k_sp2_bounds<<<e.njobs, 512, 3 * sizeof(double) * b.maxn, s>>>(b.d_sp2, b.d_st);
        if ((rc = launch_big_bounds(b, s))) return rc;
        k_sp2_init<<<dim3(b.sp2_nblk, e.njobs), 256, 0, s>>>(b.d_sp2, b.d_sp2_state, b.d_st, b.sp2_nblk);
        k_sp2_start<<<cdiv(e.njobs, 128), 128, 0, s>>>(b.d_sp2, b.d_sp2_state, b.d_st, e.njobs, b.sp2_nblk);
        CK(cudaMemsetAsync(b.d_need_eigen, 0, sizeof(int) * b.nmol, s));
        run.launched(AM1GPU_PHASE_EIGEN,
                     3 + big_launches(big_split((int)b.sp2_big.size(), [&](int i) { return b.jobs[b.sp2_big[i]].n; }),
                                      (int)b.sp2_big.size()));
    }
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

// One purification step of every channel still purifying: the FP64 products (and the TF32 ones
// while any molecule may be in its TF32 phase), then the trace bookkeeping.  zero_count: clear the
// count of channels still purifying first (the captured loop's condition kernel clears it instead).
// cond (captured solve only): the update also takes the loop's decision on that handle
// (k_sp2_update_cond, batches of at most SP2_UPDATE_ONE channels), so no k_sp2_cond follows.
int enq_step(IterEnq& e, int sp2_max, bool lowp_left, bool zero_count, const cudaGraphConditionalHandle* cond = nullptr) {
    Batch& b = e.b;
    const cudaStream_t s = e.s;
    Run& run = *e.run;
    int rc;
    size_t pc;
    if ((rc = run.begin(&pc))) return rc;
    int nl = 0;
    launch_tiles(b, s, [&](const GemmTile* t, int nt, bool pairs) {
        if (pairs && b.sp2_tma)
            k_sp2_step_tma<<<nt, 128, dgemm_tma_smem_bytes(), s>>>(b.d_sp2, t, nt, b.d_sp2_state, b.d_sp2_maps, b.d_sp2_active + 2);
        else if (pairs)
            k_sp2_step16<<<nt, 128, dgemm_smem_bytes(), s>>>(b.d_sp2, t, nt, b.d_sp2_state);
        else
            k_sp2_step8<<<nt, 128, dgemm_smem_bytes(), s>>>(b.d_sp2, t, nt, b.d_sp2_state);
        ++nl;
    });
    if (b.nt_oz > 0) {
        k_sp2_step_oz<<<b.nt_oz, 128, oz_smem_bytes(), s>>>(b.d_sp2, b.d_oz_tiles, b.nt_oz, b.d_sp2_state, b.d_sp2_active + 2);
        ++nl;
    }
    if (lowp_left) {
        launch_tiles(b, s, [&](const GemmTile* t, int nt, bool) {
            k_sp2_step_tf32<<<nt, 128, tf32_smem_bytes(), s>>>(b.d_sp2, t, nt, b.d_sp2_state);
            ++nl;
        });
        if (b.nt_tc > 0 && b.has_tc3) {
            k_sp2_step_tc<<<b.nt_tc, 128, tc_smem_bytes(), s>>>(b.d_sp2, b.d_tc_tiles, b.nt_tc, b.d_sp2_state, b.d_sp2_active + 2);
            ++nl;
        }
        if (b.nt_tc > 0 && b.has_tc1) {
            k_sp2_step_tc1<<<b.nt_tc, 128, tc1_smem_bytes(), s>>>(b.d_sp2, b.d_tc_tiles, b.nt_tc, b.d_sp2_state, b.d_xf_maps,
                                                                  b.d_sp2_active + 2);
            ++nl;
        }
    }
    run.launched(AM1GPU_PHASE_DENSITY_CORE, nl);
    if ((rc = run.end(AM1GPU_PHASE_DENSITY_CORE, pc))) return rc;
    if (cond) {
        k_sp2_update_cond<<<1, SP2_UPDATE_ONE, 0, s>>>(b.d_sp2, b.d_sp2_state, e.njobs, sp2_max, b.d_work, *cond, b.d_loop);
    } else {
        if (zero_count) CK(cudaMemsetAsync(b.d_sp2_active, 0, sizeof(int), s));
        k_sp2_update<<<cdiv(e.njobs, 128), 128, 0, s>>>(b.d_sp2, b.d_sp2_state, e.njobs, sp2_max, b.d_sp2_active, b.d_work);
    }
    run.launched(AM1GPU_PHASE_EIGEN);
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

// The density of the iteration (the purified X, or the eigensolver for stalled and Jacobi-path
// molecules), the density change and the convergence test, in three parts: the purified density
// (enq_tail_finish), the eigensolver for the molecules whose purification stalled (enq_tail_stall:
// its kernels skip every other molecule, and the captured solve runs it only in iterations where
// some purification stalled), and the rest (enq_tail_rest).  The Jacobi density path (density_mode
// != 0) is all in enq_tail_finish.
int enq_tail_finish(IterEnq& e) {
    Batch& b = e.b;
    const cudaStream_t s = e.s;
    Run& run = *e.run;
    int rc;
    if (density_mode() == 0) {
        const unsigned fin_blocks = std::max(8u, std::min(256u, cdiv((long long)b.maxn * b.maxn, 65536)));
        k_sp2_finish<<<dim3(fin_blocks, e.njobs), 256, 0, s>>>(b.d_sp2, b.d_sp2_state, b.d_st, b.d_need_eigen, b.d_work,
                                                               b.d_big_stall, b.d_active + 3);
        run.launched(AM1GPU_PHASE_EIGEN);
        if (!b.sp2_big.empty() && (rc = big_fallback(b, e.ws))) return rc;
    } else {
        k_gemm_nn<<<b.nt_gt, 256, 0, s>>>(b.d_gj_gt, b.d_gt_gt, b.nt_gt, b.d_st, 0, nullptr);
        CK(cudaGetLastError());
        size_t pj;
        if ((rc = run.begin(&pj))) return rc;
        if ((rc = launch_jacobi(b, e.ws, 0, nullptr, e.s))) return rc;
        run.launched(AM1GPU_PHASE_DENSITY_CORE, (int)b.buckets.size());
        if ((rc = run.end(AM1GPU_PHASE_DENSITY_CORE, pj))) return rc;
        if (b.neig > 0) k_eig_sort<<<b.neig, 512, 0, s>>>(b.d_eig, b.d_st, 0, nullptr);
        run.launched(AM1GPU_PHASE_EIGEN, 2);
        if ((rc = run.end(AM1GPU_PHASE_EIGEN, e.ph)) || (rc = run.begin(&e.ph))) return rc;
        k_gemm_tn<<<b.nt_dn, 256, 0, s>>>(b.d_gj_dn, b.d_gt_dn, b.nt_dn, b.d_st, 0, nullptr);
        run.launched(AM1GPU_PHASE_DENSITY);
    }
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

// Stalled purifications: warm-started Jacobi + C_occ C_occ^T for those molecules only
// (need_eigen); nothing on the Jacobi density path.
int enq_tail_stall(IterEnq& e) {
    Batch& b = e.b;
    const cudaStream_t s = e.s;
    Run& run = *e.run;
    int rc;
    if (density_mode() != 0) return AM1GPU_OK;
    k_gemm_nn<<<b.nt_gt, 256, 0, s>>>(b.d_gj_gt, b.d_gt_gt, b.nt_gt, b.d_st, 0, b.d_need_eigen);
    if ((rc = launch_jacobi(b, e.ws, 0, b.d_need_eigen, e.s))) return rc;
    run.launched(AM1GPU_PHASE_EIGEN, (int)b.buckets.size());
    if (b.neig > 0) k_eig_sort<<<b.neig, 512, 0, s>>>(b.d_eig, b.d_st, 0, b.d_need_eigen);
    k_gemm_tn<<<b.nt_dn, 256, 0, s>>>(b.d_gj_dn, b.d_gt_dn, b.nt_dn, b.d_st, 0, b.d_need_eigen);
    run.launched(AM1GPU_PHASE_EIGEN, 3);
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

int enq_tail_rest(IterEnq& e) {
    Batch& b = e.b;
    const cudaStream_t s = e.s;
    Run& run = *e.run;
    int rc;
    if (density_mode() == 0 && ((rc = run.end(AM1GPU_PHASE_EIGEN, e.ph)) || (rc = run.begin(&e.ph)))) return rc;
    k_density_post<<<dim3(e.nblk, e.njobs), 256, 0, s>>>(b.d_jobs, b.d_st, e.nblk);
    k_converge<<<cdiv(b.nmol, 128), 128, 0, s>>>(b.d_mols, b.d_jobs, b.d_job0, b.nmol, b.d_st, b.d_status, e.nblk, e.prm,
                                                 b.d_active);
    run.launched(AM1GPU_PHASE_DENSITY, 2);
    if ((rc = run.end(AM1GPU_PHASE_DENSITY, e.ph))) return rc;
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

int enq_tail(IterEnq& e) {
    int rc;
    if ((rc = enq_tail_finish(e)) || (rc = enq_tail_stall(e)) || (rc = enq_tail_rest(e))) return rc;
    return AM1GPU_OK;
}

// The captured solve (AM1GPU_GRAPH, default on): the SCF loop runs as one graph launch whose loops
// are decided on the device, so the host reads nothing until the solve ends.  Not for batches
// with molecules above 448 orbitals (their purification bounds and reductions take cooperative
// launches, and their fallback reads flags on the host), the mixed path (whose TF32 launches the
// host drops once no molecule is in its TF32 phase), the Jacobi density path, or when phase timing
// is on (the phase events sit between launches).
bool graph_ok(const Batch& b, const am1gpu_options& o, bool timed) {
    static const int env = [] {
        const char* v = std::getenv("AM1GPU_GRAPH");
        return v ? std::atoi(v) : 1;
    }();
    return env != 0 && !timed && density_mode() == 0 && o.precision != AM1GPU_PRECISION_MIXED && b.sp2_big.empty() &&
           b.tri_big.empty() && b.nmol > 0 && o.max_scf > 0;
}

// Adds the work `fn` enqueues on stream cs to graph g after `deps` (capture into the graph), and
// returns the single node the captured sequence ends on.
template <class F>
int capture_into(cudaStream_t cs, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps, cudaGraphNode_t* last, F&& fn) {
    CK(cudaStreamBeginCaptureToGraph(cs, g, deps, nullptr, ndeps, cudaStreamCaptureModeRelaxed));
    int rc = fn();
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* tail = nullptr;
    size_t ntail = 0;
    cudaError_t e1 = cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &tail, &ntail);
    cudaGraphNode_t last_node = (e1 == cudaSuccess && ntail == 1) ? tail[0] : nullptr;
    cudaGraph_t out = g;
    cudaError_t e2 = cudaStreamEndCapture(cs, &out);
    if (rc) return rc;
    if (e1 != cudaSuccess) return fail(AM1GPU_DEVICE_ERROR, std::string("capture info: ") + cudaGetErrorString(e1));
    if (e2 != cudaSuccess) return fail(AM1GPU_DEVICE_ERROR, std::string("end capture: ") + cudaGetErrorString(e2));
    if (!last_node) return fail(AM1GPU_DEVICE_ERROR, "captured sequence does not end on one node");
    *last = last_node;
    return AM1GPU_OK;
}

// A WHILE node after `dep` in g, with handle h; its body graph in *body.
int add_while(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h, cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    CK(cudaGraphAddNode(node, g, &dep, 1, &np));
    *body = np.conditional.phGraph_out[0];
    return AM1GPU_OK;
}

// An IF node after `dep` in g, with handle h; its body graph in *body.
int add_if(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h, cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    CK(cudaGraphAddNode(node, g, &dep, 1, &np));
    *body = np.conditional.phGraph_out[0];
    return AM1GPU_OK;
}

// The SCF loop of run_device as one graph launch:
//   k_scf_arm -> WHILE(scf) { head -> k_sp2_arm -> WHILE(sp2) { step -> k_sp2_cond } -> tail -> k_scf_cond }
// (for batches of at most SP2_UPDATE_ONE channels the step's update kernel sets the purification
// loop's condition itself, k_sp2_update_cond, in place of k_sp2_update + k_sp2_cond) and, in a graph
// kept for a resident batch's later runs, the tail split as
//   finish -> k_stall_arm -> IF(stall) { stalled-purification eigensolver } -> rest -> k_scf_cond.
// The kernels are the eager loop's, in the same order; only the loop decisions moved to the device
// (k_graph.cu), and the eigensolver kernels for stalled purifications, which change nothing in an
// iteration where no purification stalled, run only in iterations where one did.  So the results
// are the same bit for bit.  The purification loop stops as soon as no
// channel purifies (the eager loop looks every six steps from the twelfth on); the extra eager
// steps change nothing, because finished channels skip their products.
// *launched: the graph was launched (an error before that leaves the stream untouched).
int scf_loop_graph(IterEnq& e, const am1gpu_options& o, bool* launched) {
    Batch& b = e.b;
    Mem& m = *e.ws;
    const int sp2_max = sp2_max_steps();
    if (!m.cap_stream) CK(cudaStreamCreateWithFlags(&m.cap_stream, cudaStreamNonBlocking));
    const cudaStream_t cs = m.cap_stream;
    if (b.graph_cacheable && b.graph_exec) {  // a resident batch's graph, captured on its first run
        *launched = true;
        CK(cudaGraphLaunch(b.graph_exec, e.s));
        CK(cudaMemcpyAsync(b.h_loop, b.d_loop, sizeof(GraphLoop), cudaMemcpyDeviceToHost, e.s));
        return AM1GPU_OK;
    }
    am1gpu_call_stats cnt{};  // launches per captured sequence
    Run crun{e.ws, &cnt, false};
    IterEnq ce = e;
    ce.s = cs;
    ce.run = &crun;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    struct GraphGuard {
        cudaGraph_t g;
        ~GraphGuard() {
            if (g) cudaGraphDestroy(g);
        }
    } guard{g};
    cudaGraphConditionalHandle h_scf, h_sp2;
    CK(cudaGraphConditionalHandleCreate(&h_scf, g, 0, 0));
    int rc;
    cudaGraphNode_t arm, w_scf, head, w_sp2, step, tail;
    if ((rc = capture_into(cs, g, nullptr, 0, &arm, [&]() -> int {
             k_scf_arm<<<1, 32, 0, cs>>>(h_scf, b.d_loop, o.max_scf);
             return AM1GPU_OK;
         })))
        return rc;
    cudaGraph_t body = nullptr, body2 = nullptr;
    if ((rc = add_while(g, arm, h_scf, &w_scf, &body))) return rc;
    CK(cudaGraphConditionalHandleCreate(&h_sp2, body, 0, 0));
    const int64_t head0 = cnt.kernel_launches;
    if ((rc = capture_into(cs, body, nullptr, 0, &head, [&]() -> int {
             int r = enq_head(ce, false);
             if (r) return r;
             k_sp2_arm<<<1, 32, 0, cs>>>(h_sp2, b.d_loop, b.d_sp2_active);
             return AM1GPU_OK;
         })))
        return rc;
    const int64_t per_head = cnt.kernel_launches - head0 + 1;
    if ((rc = add_while(body, head, h_sp2, &w_sp2, &body2))) return rc;
    const int64_t step0 = cnt.kernel_launches;
    const bool fused = e.njobs <= SP2_UPDATE_ONE;  // the update takes the loop's decision itself
    if ((rc = capture_into(cs, body2, nullptr, 0, &step, [&]() -> int {
             int r = enq_step(ce, sp2_max, false, false, fused ? &h_sp2 : nullptr);
             if (r) return r;
             if (!fused) k_sp2_cond<<<1, 32, 0, cs>>>(h_sp2, b.d_loop, b.d_sp2_active, sp2_max);
             return AM1GPU_OK;
         })))
        return rc;
    const int64_t per_step = cnt.kernel_launches - step0 + (fused ? 0 : 1);
    const int64_t tail0 = cnt.kernel_launches;
    int64_t per_stall = 0, per_tail = 0;
    if (b.graph_cacheable) {
        // a graph kept for the batch's later runs: the stalled-purification eigensolver behind an IF
        // node (its extra capture and instantiation cost more than they save in a one-off graph)
        cudaGraphConditionalHandle h_stall;
        CK(cudaGraphConditionalHandleCreate(&h_stall, body, 0, 0));
        cudaGraphNode_t fin, w_stall, stall_last;
        if ((rc = capture_into(cs, body, &w_sp2, 1, &fin, [&]() -> int {
                 int r = enq_tail_finish(ce);
                 if (r) return r;
                 k_stall_arm<<<1, 256, 0, cs>>>(h_stall, b.d_loop, b.d_need_eigen, b.nmol);
                 return AM1GPU_OK;
             })))
            return rc;
        const int64_t stall0 = cnt.kernel_launches;
        cudaGraph_t body3 = nullptr;
        if ((rc = add_if(body, fin, h_stall, &w_stall, &body3))) return rc;
        if ((rc = capture_into(cs, body3, nullptr, 0, &stall_last, [&]() -> int { return enq_tail_stall(ce); }))) return rc;
        per_stall = cnt.kernel_launches - stall0;
        if ((rc = capture_into(cs, body, &w_stall, 1, &tail, [&]() -> int {
                 int r = enq_tail_rest(ce);
                 if (r) return r;
                 k_scf_cond<<<1, 32, 0, cs>>>(h_scf, b.d_loop, b.d_active, o.max_scf);
                 return AM1GPU_OK;
             })))
            return rc;
        per_tail = cnt.kernel_launches - tail0 + 2 - per_stall;
    } else {
        if ((rc = capture_into(cs, body, &w_sp2, 1, &tail, [&]() -> int {
                 int r = enq_tail(ce);
                 if (r) return r;
                 k_scf_cond<<<1, 32, 0, cs>>>(h_scf, b.d_loop, b.d_active, o.max_scf);
                 return AM1GPU_OK;
             })))
            return rc;
        per_tail = cnt.kernel_launches - tail0 + 1;
    }
    cudaGraphExec_t ge = nullptr;
    CK(cudaGraphInstantiate(&ge, g, 0));
    *launched = true;
    const cudaError_t le = cudaGraphLaunch(ge, e.s);
    if (b.graph_cacheable && le == cudaSuccess) b.graph_exec = ge;
    else cudaGraphExecDestroy(ge);  // an executable graph still running is freed once it completes
    CK(le);
    CK(cudaMemcpyAsync(b.h_loop, b.d_loop, sizeof(GraphLoop), cudaMemcpyDeviceToHost, e.s));
    b.graph_counts[0] = per_head;
    b.graph_counts[1] = per_step;
    b.graph_counts[2] = per_tail;
    b.graph_counts[3] = per_stall;
    return AM1GPU_OK;
}

// The whole solve on the device: state reset, integrals, SCF iterations, final energy and the
// result records.  Inputs must already be resident (build_batch); nothing but the count of
// molecules still iterating is read back.
int run_device(Batch& b, Mem& mem, const DevElem* dp, const am1gpu_options& o, am1gpu_call_stats* stats) {
    Mem* ws = &mem;
    cudaStream_t s = ws->stream;
    Run run{ws, stats, timing_on()};
    int rc;
    size_t t0, ph;
    if ((rc = run.event(&t0))) return rc;
    if ((rc = run.begin(&ph))) return rc;
    CK(cudaMemsetAsync(b.d_status, 0, sizeof(int) * b.nmol, s));
    CK(cudaMemsetAsync(b.d_work, 0, sizeof(double) * kWorkN, s));
    CK(cudaMemsetAsync(b.d_sp2_active, 0, 4 * sizeof(int), s));  // [2]: error word of the tensor-core steps
    CK(cudaMemsetAsync(b.d_arena, 0, sizeof(double) * b.arena_doubles, s));
    // mixed precision: every molecule starts with TF32 purification (k_converge ends that phase)
    const bool mixed = o.precision == AM1GPU_PRECISION_MIXED && density_mode() == 0;
    bool lowp_left = mixed;  // some molecule may still be in its TF32 phase
    k_state_init<<<cdiv(b.nmol, 128), 128, 0, s>>>(b.d_st, b.d_mols, b.nmol, mixed ? 1 : 0);
    run.launched(AM1GPU_PHASE_CORE);
    rc = launch_core(b, ws, dp, &run);
    if (rc) return rc;
    const int njobs = (int)b.jobs.size();
    if (b.natoms > 0) {
        k_sad_init<<<cdiv(b.natoms, 128), 128, 0, s>>>(b.d_mols, b.d_atom_mol, b.natoms, dp, b.d_atom_z, b.d_arena);
        run.launched(AM1GPU_PHASE_CORE);
    }
    k_identity<<<dim3(cdiv(b.maxn, 256), njobs), 256, 0, s>>>(b.d_jobs);
    run.launched(AM1GPU_PHASE_CORE);
    CK(cudaGetLastError());
    if ((rc = run.end(AM1GPU_PHASE_CORE, ph))) return rc;
    ScfParams prm{o.max_scf, o.use_diis, o.accelerator, o.e_tol, o.p_tol, o.adiis_switch, lowp_switch(), lowp_max_iter()};
    IterEnq e{b, ws, s, dp, prm, b.nblk, std::max(1, std::min(64, (b.maxn + 7) / 8)), njobs, &run, 0};
    int done = 0;
    bool graph = graph_ok(b, o, run.timed);
    if (graph) {
        bool launched = false;
        rc = scf_loop_graph(e, o, &launched);
        if (rc && launched) return rc;
        if (rc) {  // the graph could not be built here: the host-driven loop runs the same kernels
            graph = false;
            cudaGetLastError();
        }
    }
    if (!graph) {
        const int check = b.nmol > 64 ? 4 : 1;
        while (done < o.max_scf) {
            for (int k = 0; k < check && done < o.max_scf; ++k, ++done) {
                if ((rc = enq_head(e, lowp_left))) return rc;
                if (density_mode() == 0) {
                    const int sp2_max = sp2_max_steps();
                    for (int step = 0; step < sp2_max; ++step) {
                        if ((rc = enq_step(e, sp2_max, lowp_left, true))) return rc;
                        if (step >= 12 && (step % 6) == 5) {
                            CK(cudaMemcpyAsync(b.h_active + 1, b.d_sp2_active, sizeof(int), cudaMemcpyDeviceToHost, s));
                            CK(cudaStreamSynchronize(s));
                            if (b.h_active[1] == 0) break;
                        }
                    }
                }
                if ((rc = enq_tail(e))) return rc;
            }
            CK(cudaMemcpyAsync(b.h_active, b.d_active, sizeof(int), cudaMemcpyDeviceToHost, s));
            if (lowp_left) CK(cudaMemcpyAsync(b.h_active + 2, b.d_active + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (*b.h_active == 0) break;
            if (lowp_left && b.h_active[2] == 0) lowp_left = false;  // no molecule returns to TF32
        }
    }
    stats->scf_cycles = done;
    const int nblk = b.nblk;
    // final energy at the final density (src/scf.rs:698-701, 835-839) and the result records
    if ((rc = run.begin(&ph))) return rc;
    k_fock<<<cdiv(b.natoms, 8), 256, 0, s>>>(b.d_mols, b.d_atom_mol, b.natoms, dp, b.d_atom_z, b.d_wstore, b.d_arena, b.d_st, 1);
    k_post_fock<<<dim3(nblk, njobs), 256, 0, s>>>(b.d_jobs, b.d_mols, b.d_st, nblk, 1, 1);
    k_final_energy<<<cdiv(b.nmol, 128), 128, 0, s>>>(b.d_mols, b.d_jobs, b.d_job0, b.nmol, b.d_st, nblk);
    // eigenvalues of the last F* (mo_energies, HOMO/LUMO): tridiagonalisation + bisection
    if ((rc = launch_tridiag(b, ws))) return rc;
    int64_t big_tri_launches = 0;
    if ((rc = launch_big_tridiag(b, s, &big_tri_launches))) return rc;
    bisect_launch(b.d_tri, njobs, b.maxn, s, true);
    k_results<<<cdiv(b.nmol, 128), 128, 0, s>>>(b.d_mols, b.d_jobs, b.d_job0, b.nmol, b.d_st, b.d_status, dp, b.d_atom_z,
                                                 b.d_atom_xyz, b.d_res, b.d_charges);
    run.launched(AM1GPU_PHASE_FINAL, 5 + (int)b.tri_buckets.size() + (int)big_tri_launches);
    CK(cudaGetLastError());
    if ((rc = run.end(AM1GPU_PHASE_FINAL, ph))) return rc;
    size_t t1;
    if ((rc = run.event(&t1))) return rc;
    CK(cudaMemcpyAsync(b.h_work, b.d_work, sizeof(double) * kWorkN, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(b.h_active + 2, b.d_sp2_active + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (b.h_active[2] & (1 << 10)) return fail(AM1GPU_LINALG, "a purification iterate left the range of its digit planes (|x| >= 2)");
    if (b.h_active[2]) return fail(AM1GPU_DEVICE_ERROR, "a tensor-core step gave up waiting for its MMAs or operand copies");
    stats->purification_steps += b.h_work[0];
    stats->purification_flops += b.h_work[1];
    stats->purification_bytes += b.h_work[3];
    stats->eigen_fallbacks += (int32_t)b.h_work[2];
    stats->lowp_purification_steps += b.h_work[4];
    stats->lowp_purification_flops += b.h_work[5];
    if (graph) {  // what the captured loops launched
        const GraphLoop lp = *b.h_loop;
        stats->scf_cycles = lp.scf_iter;
        stats->kernel_launches += 1 + (int64_t)lp.scf_iter * (b.graph_counts[0] + b.graph_counts[2]) +
                                  (int64_t)lp.sp2_total * b.graph_counts[1] + (int64_t)lp.eig_runs * b.graph_counts[3];
        stats->graph_launches += 1;
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, mem.events[t0], mem.events[t1]));
    stats->device_ms += ms;
    return run.collect();
}

// Nuclear gradient at the converged densities (closed_form_gradient, src/gradient.rs:173-253),
// fetched into b.h_grad.
int run_gradient(Batch& b, Mem& mem, const DevElem* dp, am1gpu_call_stats* stats) {
    cudaStream_t s = mem.stream;
    if (b.natoms > 0) {
        k_gradient<<<cdiv(b.natoms, 8), 256, 0, s>>>(b.d_mols, b.d_atom_mol, b.natoms, dp, b.d_atom_z, b.d_atom_xyz, b.d_jobs, b.d_job0,
                                                     b.d_grad, b.d_status);
        CK(cudaGetLastError());
        stats->kernel_launches += 1;
    }
    CK(cudaMemcpyAsync(b.h_grad, b.d_grad, sizeof(double) * 3 * std::max(b.natoms, 1), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    stats->d2h_bytes += (int64_t)(sizeof(double) * 3 * std::max(b.natoms, 1));
    return AM1GPU_OK;
}

int fetch_results(Batch& b, Mem& mem, am1gpu_call_stats* stats) {
    cudaStream_t s = mem.stream;
    CK(cudaMemcpyAsync(b.h_res, b.d_res, sizeof(double) * RES_N * b.nmol, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(b.h_charges, b.d_charges, sizeof(double) * std::max(b.natoms, 1), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(b.h_eps, b.d_eps, sizeof(double) * std::max(b.eps_total, 1LL), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    stats->d2h_bytes += (int64_t)(sizeof(double) * RES_N * b.nmol + sizeof(double) * std::max(b.natoms, 1) +
                                  sizeof(double) * std::max(b.eps_total, 1LL));
    return AM1GPU_OK;
}

// Copies one device matrix (internal AO order) out to the caller's order.
int fetch_matrix(Mem* ws, const double* dsrc, int n, std::vector<double>& tmp, am1gpu_call_stats* stats = nullptr) {
    tmp.resize((size_t)n * n);
    CK(cudaMemcpyAsync(tmp.data(), dsrc, sizeof(double) * n * n, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaStreamSynchronize(ws->stream));
    if (stats) stats->d2h_bytes += (int64_t)sizeof(double) * n * n;
    return AM1GPU_OK;
}

}  // namespace
int symmetric_eigen_one(int n, const double* a, double* w, double* v, Mem* mem_override);
namespace {
thread_local Mem tl_mem_eig;  // on-demand eigenvectors: separate from the batch's memory
int density_mode();

int write_result(Batch& b, Mem* ws, int mi, am1gpu_result* r, am1gpu_call_stats* stats) {
    const MolPlan& p = b.plans[mi];
    const double* rec = b.h_res + (size_t)mi * RES_N;
    r->electronic_ev = rec[RES_ELEC];
    r->core_ev = rec[RES_CORE];
    r->total_ev = rec[RES_TOTAL];
    r->heat_of_formation_kcal = rec[RES_HOF];
    for (int k = 0; k < 3; ++k) r->dipole_debye[k] = rec[RES_DIP + k];
    r->dipole_magnitude = rec[RES_DIPMAG];
    r->homo_ev = rec[RES_HOMO];
    r->lumo_ev = rec[RES_LUMO];
    r->homo_beta_ev = rec[RES_HOMO_B];
    r->lumo_beta_ev = rec[RES_LUMO_B];
    r->residual = rec[RES_RESID];
    r->nao = p.nao;
    r->n_occ = p.n_occ[0];
    r->n_occ_beta = p.n_occ[1];
    r->iterations = (int)rec[RES_ITER];
    r->converged = (int)rec[RES_CONV];
    r->unrestricted = p.nch == 2 ? 1 : 0;
    const MolDesc& md = b.mols[mi];
    if (r->charges)
        for (int ia = 0; ia < p.natoms; ++ia) r->charges[p.order[ia]] = b.h_charges[md.atom_base + ia];
    const int n = p.nao;
    const auto& map = p.ao_map;
    std::vector<double> t0, t1;
    const ChanJob& j0 = b.jobs[b.job0[mi]];
    if (r->density || r->spin_density) {
        int rc = fetch_matrix(ws, j0.P, n, t0, stats);
        if (rc) return rc;
        if (p.nch == 2) {
            rc = fetch_matrix(ws, b.jobs[b.job0[mi] + 1].P, n, t1, stats);
            if (rc) return rc;
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const size_t s = (size_t)i * n + j, d = (size_t)map[i] * n + map[j];
                if (r->density) r->density[d] = p.nch == 2 ? t0[s] + t1[s] : t0[s];
                if (r->spin_density && p.nch == 2) r->spin_density[d] = t0[s] - t1[s];
            }
    }
    for (int c = 0; c < p.nch; ++c) {
        double* e_out = c == 0 ? r->mo_energies : r->beta_energies;
        double* c_out = c == 0 ? r->mo_coeff : r->beta_coeff;
        const ChanJob& jc = b.jobs[b.job0[mi] + c];
        if (e_out) std::memcpy(e_out, b.h_eps + (jc.eps - b.d_eps), sizeof(double) * n);  // fetched in bulk
        if (c_out) {
            if (density_mode() == 0 || p.cluster == 0) {
                // the purification path has no eigenvectors: diagonalise the last F* now
                int rc = fetch_matrix(ws, jc.Fx, n, t0, stats);
                if (rc) return rc;
                std::vector<double> wv(n), vv((size_t)n * n);
                rc = symmetric_eigen_one(n, t0.data(), wv.data(), vv.data(), &tl_mem_eig);
                if (rc) return rc;
                for (int mu = 0; mu < n; ++mu)
                    for (int k = 0; k < n; ++k) c_out[(size_t)map[mu] * n + k] = vv[(size_t)mu * n + k];
            } else {
                int rc = fetch_matrix(ws, jc.Ct, n, t0, stats);
                if (rc) return rc;
                for (int k = 0; k < n; ++k)
                    for (int mu = 0; mu < n; ++mu) c_out[(size_t)map[mu] * n + k] = t0[(size_t)k * n + mu];
            }
        }
    }
    const int status = (int)rec[RES_STATUS];
    if (status == AM1GPU_SCF_DIVERGED)
        return fail(AM1GPU_SCF_DIVERGED, "the AM1 SCF diverged at iteration " + std::to_string(r->iterations) +
                                             ": a non-finite energy or density appeared");
    if (status == AM1GPU_LINALG) return fail(AM1GPU_LINALG, "the eigensolver refused a non-finite or unconverged matrix");
    if (status == AM1GPU_UNSUPPORTED) return fail(AM1GPU_UNSUPPORTED, "overlap not covered for an element of this molecule");
    if (!r->converged) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "AM1 SCF did not converge after %d iterations (error=%.3e)", r->iterations, r->residual);
        return fail(AM1GPU_SCF_NOT_CONVERGED, buf);
    }
    return AM1GPU_OK;
}

void fill_empty(am1gpu_result* r) {
    // a molecule with no atoms: nothing to solve (run_am1 converges at its second iteration)
    r->electronic_ev = r->core_ev = r->total_ev = r->heat_of_formation_kcal = 0.0;
    r->dipole_debye[0] = r->dipole_debye[1] = r->dipole_debye[2] = r->dipole_magnitude = 0.0;
    r->homo_ev = r->lumo_ev = r->homo_beta_ev = r->lumo_beta_ev = NAN;
    r->residual = 0.0;
    r->nao = r->n_occ = r->n_occ_beta = 0;
    r->iterations = 2;
    r->converged = 1;
    r->unrestricted = 0;
}

}  // namespace

// grads (optional): one caller buffer of 3 * natoms doubles per molecule for the nuclear gradient
int density_purify_one(int n, const double* F, double nocc, double weight, int precision, double* P, int* steps_out,
                       Mem* mem_override);

// The autotuner of the reduced-precision purification kernel: for each size class not yet tuned on
// this device, one AM1-like matrix of the class's size (spectrum in [-40, -12] eV occupied and
// [1, 10] eV virtual, the same matrix for all) is purified with each of the three kernels after a
// warm-up, and the fastest is kept for the process.  The mma.sync and single-pass tcgen05 kernels
// work at TF32 precision, the 3xTF32 one at FP32 accuracy; every one of them only starts the FP64
// iterations, which take the SCF to convergence.  Runs in its own device pool, before the batch is
// laid out.
int tune_lowp_kernels(const std::vector<MolPlan>& plans) {
    if (lowp_tc_env() >= 0) return AM1GPU_OK;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return AM1GPU_OK;
    LowpTune& t = g_lowp_tune[dev];
    bool need[kTuneClasses] = {false, false, false, false};
    for (const auto& p : plans) need[tune_class(p.nao)] = true;
    std::lock_guard<std::mutex> lock(t.mu);
    const std::string saved = g_err;
    for (int c = 0; c < kTuneClasses; ++c) {
        if (!need[c] || t.choice[c] >= 0) continue;
        const int n = kTuneSize[c], nocc = (2 * n) / 3;
        std::vector<double> f((size_t)n * n, 0.0), p((size_t)n * n);
        // F = diag(spectrum) + a small symmetric coupling: a gapped, dense matrix
        for (int i = 0; i < n; ++i) {
            f[(size_t)i * n + i] = i < nocc ? -40.0 + 28.0 * i / std::max(1, nocc - 1) : 1.0 + 9.0 * (i - nocc) / std::max(1, n - nocc - 1);
            for (int j = 0; j < i; ++j) {
                const double v = 0.05 * std::sin(0.37 * i + 0.91 * j);
                f[(size_t)i * n + j] = f[(size_t)j * n + i] = v;
            }
        }
        float best[3] = {0.f, 0.f, 0.f};
        bool ok[3] = {true, true, tma_encoder() != nullptr};
        // kind 0: mma.sync TF32 (precision 2), 1: tcgen05 3xTF32 (precision 1), 2: tcgen05 TF32 (precision 4)
        const int prec_of[3] = {2, 1, 4};
        for (int kind = 0; kind < 3; ++kind) {
            for (int rep = 0; rep < 3 && ok[kind]; ++rep) {
                const auto t0 = std::chrono::steady_clock::now();
                int steps = 0;
                if (density_purify_one(n, f.data(), nocc, 2.0, prec_of[kind], p.data(), &steps, &tl_mem_eig)) ok[kind] = false;
                const float ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
                if (rep > 0) best[kind] = rep == 1 ? ms : std::min(best[kind], ms);
            }
        }
        int pick = -1;
        for (int kind = 0; kind < 3; ++kind)
            if (ok[kind] && (pick < 0 || best[kind] < best[pick])) pick = kind;
        for (int kind = 0; kind < 3; ++kind) t.ms[c][kind] = ok[kind] ? best[kind] : 0.f;
        t.choice[c] = pick >= 0 ? pick : 1;
    }
    g_err = saved;
    return AM1GPU_OK;
}

// params (optional): the caller's parameter set, whose method replaces opts->method
int scf_batch(int nmol, const am1gpu_molecule* mols, const am1gpu_options* opts_in, am1gpu_result* res, int* status,
              double* const* grads = nullptr, const am1gpu_param_table* params = nullptr) {
    g_err.clear();
    tl_stats = am1gpu_call_stats{};
    if (nmol < 0 || (nmol > 0 && (!mols || !res)) || !opts_in) return fail(AM1GPU_INVALID_INPUT, "null argument");
    am1gpu_options opts_v = *opts_in;
    const am1gpu_options* opts = &opts_v;
    std::vector<DevElem> custom;
    int rc;
    if (params) {
        int method = 0;
        if ((rc = custom_param_table(params, custom, &method))) {
            for (int i = 0; i < nmol; ++i)
                if (status) status[i] = rc;
            return rc;
        }
        opts_v.method = method == 1 ? AM1GPU_METHOD_RM1 : AM1GPU_METHOD_AM1;
    }
    const DevElem* tab_all = params ? custom.data() : nullptr;
    DeviceCtx* ctx;
    rc = device_ctx(&ctx);
    if (rc) {
        for (int i = 0; i < nmol; ++i)
            if (status) status[i] = rc;
        return rc;
    }
    // plan every molecule (validation, atom order, AO map): independent per molecule, so large
    // batches plan on several host threads; results and the first error are taken in input order
    std::vector<MolPlan> all(nmol);
    std::vector<int> rcs(nmol, AM1GPU_OK);
    std::vector<std::string> msgs(nmol);
    auto plan_range = [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            if (mols[i].natoms == 0 && mols[i].multiplicity >= 1 && std::fabs(mols[i].charge) < 1e-6) {
                fill_empty(&res[i]);
                rcs[i] = -1;  // solved: nothing to plan
                continue;
            }
            rcs[i] = plan_molecule(mols[i], *opts, i, all[i], tab_all);
            if (rcs[i]) msgs[i] = g_err;
        }
    };
    const int nthr = nmol >= 512 ? (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    if (nthr > 1) {
        std::vector<std::thread> pool;
        const int chunk = (nmol + nthr - 1) / nthr;
        for (int t = 0; t < nthr; ++t) pool.emplace_back(plan_range, t * chunk, std::min(nmol, (t + 1) * chunk));
        for (auto& th : pool) th.join();
    } else {
        plan_range(0, nmol);
    }
    std::vector<MolPlan> plans;
    plans.reserve(nmol);
    int first = AM1GPU_OK;
    std::string first_msg;
    for (int i = 0; i < nmol; ++i) {
        const int r = rcs[i] < 0 ? AM1GPU_OK : rcs[i];
        if (rcs[i] == AM1GPU_OK) plans.push_back(std::move(all[i]));
        if (status) status[i] = r;
        if (r && !first) {
            first = r;
            first_msg = msgs[i];
        }
    }
    if (!plans.empty()) {
        Batch b;
        Workspace* ws;
        rc = workspace(&ws, 0, 0);
        if (!rc && opts->precision == AM1GPU_PRECISION_MIXED) rc = tune_lowp_kernels(plans);
        if (!rc) rc = build_batch(mols, *opts, std::move(plans), b, *ws, &tl_stats, -1.0, tab_all);
        const DevElem* dp = b.d_params ? b.d_params : ctx->d_params;
        if (!rc) rc = run_device(b, *ws, dp, *opts, &tl_stats);
        if (!rc && grads) rc = run_gradient(b, *ws, dp, &tl_stats);
        if (!rc) rc = fetch_results(b, *ws, &tl_stats);
        if (rc) {
            for (auto& p : b.plans)
                if (status) status[p.user] = rc;
            return rc;
        }
        for (int mi = 0; mi < b.nmol; ++mi) {
            const int u = b.plans[mi].user;
            if (grads && grads[u]) {  // caller atom order
                const MolPlan& p = b.plans[mi];
                const double* g = b.h_grad + 3LL * b.mols[mi].atom_base;
                for (int ia = 0; ia < p.natoms; ++ia)
                    for (int k = 0; k < 3; ++k) grads[u][3 * p.order[ia] + k] = g[3 * ia + k];
            }
            int r = write_result(b, ws, mi, &res[u], &tl_stats);
            if (status) status[u] = r;
            if (r && !first) {
                first = r;
                first_msg = g_err;
            }
        }
    }
    if (first) g_err = first_msg;
    return first;
}

int build_core_one(const am1gpu_molecule* mol, int method, double* h_core, double* core_ev) {
    g_err.clear();
    if (!mol) return fail(AM1GPU_INVALID_INPUT, "null argument");
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    am1gpu_options o;
    am1gpu_default_options(&o);
    o.method = method;
    o.reference = AM1GPU_REF_UHF;  // geometry only; the spin choice does not matter here
    am1gpu_molecule m = *mol;
    MolPlan p;
    // the electron count is irrelevant for H_core: validate elements with a neutral closed shell
    m.multiplicity = 1;
    m.charge = 0.0;
    double ne = 0.0;
    for (int i = 0; i < m.natoms; ++i)
        if (m.z[i] >= 0 && m.z[i] <= MAX_Z) ne += helem(method == 1, m.z[i]).core_charge;
    if (((long long)std::llround(ne)) % 2) m.multiplicity = 2;
    rc = plan_molecule(m, o, 0, p);
    if (rc) return rc;
    std::vector<MolPlan> plans{std::move(p)};
    Batch b;
    Workspace* ws;
    tl_stats = am1gpu_call_stats{};
    rc = workspace(&ws, 0, 0);
    if (!rc) rc = build_batch(&m, o, std::move(plans), b, *ws, &tl_stats);
    if (rc) return rc;
    rc = launch_core(b, ws, ctx->d_params, nullptr);
    if (rc) return rc;
    MolState st;
    CK(cudaMemcpyAsync(&st, b.d_st, sizeof(MolState), cudaMemcpyDeviceToHost, ws->stream));
    std::vector<double> t;
    rc = fetch_matrix(ws, b.d_arena + b.mols[0].h_base, b.plans[0].nao, t);
    if (rc) return rc;
    const int n = b.plans[0].nao;
    const auto& map = b.plans[0].ao_map;
    if (h_core)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) h_core[(size_t)map[i] * n + map[j]] = t[(size_t)i * n + j];
    if (core_ev) *core_ev = st.core_ev;
    return AM1GPU_OK;
}

int build_fock_one(const am1gpu_molecule* mol, int method, const double* p_tot, const double* p_spin, double spin_scale,
                   double* fock) {
    g_err.clear();
    if (!mol || !p_tot || !p_spin || !fock) return fail(AM1GPU_INVALID_INPUT, "null argument");
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    am1gpu_options o;
    am1gpu_default_options(&o);
    o.method = method;
    o.reference = AM1GPU_REF_UHF;  // two density slots: P0 = p_spin, P1 = p_tot - p_spin
    am1gpu_molecule m = *mol;
    m.charge = 0.0;
    double ne = 0.0;
    for (int i = 0; i < m.natoms; ++i)
        if (m.z[i] >= 0 && m.z[i] <= MAX_Z) ne += helem(method == 1, m.z[i]).core_charge;
    m.multiplicity = ((long long)std::llround(ne)) % 2 ? 2 : 1;
    MolPlan p;
    rc = plan_molecule(m, o, 0, p);
    if (rc) return rc;
    std::vector<MolPlan> plans{std::move(p)};
    Batch b;
    Workspace* ws;
    tl_stats = am1gpu_call_stats{};
    rc = workspace(&ws, 0, 0);
    if (!rc) rc = build_batch(&m, o, std::move(plans), b, *ws, &tl_stats, spin_scale);
    if (rc) return rc;
    rc = launch_core(b, ws, ctx->d_params, nullptr);
    if (rc) return rc;
    const int n = b.plans[0].nao;
    const auto& map = b.plans[0].ao_map;
    std::vector<double> p0((size_t)n * n), p1((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const size_t u = (size_t)map[i] * n + map[j];
            p0[(size_t)i * n + j] = p_spin[u];
            p1[(size_t)i * n + j] = p_tot[u] - p_spin[u];
        }
    CK(cudaMemcpyAsync(b.jobs[0].P, p0.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice, ws->stream));
    CK(cudaMemcpyAsync(b.jobs[1].P, p1.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice, ws->stream));
    k_fock<<<cdiv(b.natoms, 8), 256, 0, ws->stream>>>(b.d_mols, b.d_atom_mol, b.natoms, ctx->d_params, b.d_atom_z, b.d_wstore,
                                                      b.d_arena, b.d_st, 1);
    CK(cudaGetLastError());
    std::vector<double> t;
    rc = fetch_matrix(ws, b.jobs[0].F, n, t);
    if (rc) return rc;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) fock[(size_t)map[i] * n + map[j]] = t[(size_t)i * n + j];
    return AM1GPU_OK;
}

// G(P_r) = J(P_r) - K(P_r / 2) for nrhs densities of one molecule (build_g_matrix,
// src/fock.rs:556-575, FockBase::Zero).  The right-hand sides become copies of the molecule in one
// batch, in chunks of at most kGChunk, each with its own closed-shell channel: the pair integrals
// are formed once per copy (cheap next to the Fock build), H_core is zeroed, and one k_fock launch
// builds every copy's matrix, so F = 0 + J(P_r) - 1/2 K(P_r) exactly.
constexpr int kGChunk = 64;

int g_matrix_batch(const am1gpu_molecule* mol, int method, int nrhs, const double* dens, double* g) {
    g_err.clear();
    if (!mol || nrhs < 0 || (nrhs > 0 && (!dens || !g))) return fail(AM1GPU_INVALID_INPUT, "null argument");
    if (nrhs == 0) return AM1GPU_OK;
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    am1gpu_options o;
    am1gpu_default_options(&o);
    o.method = method;
    o.reference = AM1GPU_REF_RHF;  // one channel per copy: spin scale 1/2
    am1gpu_molecule m = *mol;
    double ne = 0.0;
    for (int i = 0; i < m.natoms; ++i)
        if (m.z[i] >= 0 && m.z[i] <= MAX_Z) ne += helem(method == 1, m.z[i]).core_charge;
    m.charge = ((long long)std::llround(ne)) % 2 ? 1.0 : 0.0;  // any closed shell: the electron count plays no part
    m.multiplicity = 1;
    MolPlan p;
    rc = plan_molecule(m, o, 0, p);
    if (rc) return rc;
    const int n = p.nao;
    const size_t nn = (size_t)n * n;
    Workspace* ws;
    tl_stats = am1gpu_call_stats{};
    rc = workspace(&ws, 0, 0);
    if (rc) return rc;
    std::vector<double> t(nn);
    for (int r0 = 0; r0 < nrhs; r0 += kGChunk) {
        const int cnt = std::min(kGChunk, nrhs - r0);
        std::vector<am1gpu_molecule> copies(cnt, m);
        std::vector<MolPlan> plans(cnt, p);
        for (int c = 0; c < cnt; ++c) plans[c].user = c;
        Batch b;
        rc = build_batch(copies.data(), o, std::move(plans), b, *ws, &tl_stats);
        if (!rc) rc = launch_core(b, ws, ctx->d_params, nullptr);
        if (rc) return rc;
        const auto& map = b.plans[0].ao_map;
        for (int c = 0; c < cnt; ++c) {
            const double* pr = dens + (size_t)(r0 + c) * nn;
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) t[(size_t)i * n + j] = pr[(size_t)map[i] * n + map[j]];
            CK(cudaMemcpyAsync(b.jobs[c].P, t.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, ws->stream));
            CK(cudaMemsetAsync(const_cast<double*>(b.jobs[c].H), 0, sizeof(double) * nn, ws->stream));  // the copy's own H_core
            CK(cudaStreamSynchronize(ws->stream));  // t is reused for the next copy
        }
        k_fock<<<cdiv(b.natoms, 8), 256, 0, ws->stream>>>(b.d_mols, b.d_atom_mol, b.natoms, ctx->d_params, b.d_atom_z, b.d_wstore,
                                                          b.d_arena, b.d_st, 1);
        CK(cudaGetLastError());
        tl_stats.kernel_launches += 1;
        for (int c = 0; c < cnt; ++c) {
            rc = fetch_matrix(ws, b.jobs[c].F, n, t, &tl_stats);
            if (rc) return rc;
            double* gr = g + (size_t)(r0 + c) * nn;
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) gr[(size_t)map[i] * n + map[j]] = t[(size_t)i * n + j];
        }
    }
    return AM1GPU_OK;
}

// C_z (=, or -= when sub) A_z B_z for z < batch on the FP64 tensor cores, in the 64 x 64 output
// tiles of 128 threads of dmma_gemm.cuh (k_dgemm16 when both operands allow 16-byte copies).
int dgemm(cudaStream_t s, const double* A, int lda, long long sA, const double* B, int ldb, long long sB, double* C, int ldc,
          long long sC, int M, int N, int K, int sub, int batch) {
    if (M <= 0 || N <= 0 || batch <= 0) return AM1GPU_OK;
    const dim3 grid((unsigned)cdiv(N, 64), (unsigned)cdiv(M, 64), (unsigned)batch);
    const bool pairs = ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0) && lda % 2 == 0 && ldb % 2 == 0 && K % 2 == 0 &&
                       N % 2 == 0 && sA % 2 == 0 && sB % 2 == 0;
    if (pairs) k_dgemm16<<<grid, 128, dgemm_smem_bytes(), s>>>(A, lda, sA, B, ldb, sB, C, ldc, sC, M, N, K, sub);
    else k_dgemm8<<<grid, 128, dgemm_smem_bytes(), s>>>(A, lda, sA, B, ldb, sB, C, ldc, sC, M, N, K, sub);
    CK(cudaGetLastError());
    return AM1GPU_OK;
}

// Eigenvalues and eigenvectors of one symmetric matrix above the cluster Jacobi's capacity (up to
// kMaxAo rows; `a` finite, its lower triangle read): the global-memory Householder reduction of
// the final-spectrum path (a cluster per matrix below kBigGridN rows, the blocked whole-GPU
// reduction above; both leave the reflectors in W), bisection, inverse iteration on the
// tridiagonal and the compact-WY back-transformation (k_stein.cu).  v[i * n + k] = component i of
// eigenvector k, eigenvalues ascending in w.
int symmetric_eigen_large(int n, const double* a, double* w, double* v, Mem* mem_override) {
    Workspace* ws;
    int rc;
    if (mem_override) {
        rc = mem_ensure(*mem_override, 0, 0);
        ws = mem_override;
    } else {
        rc = workspace(&ws, 0, 0);
    }
    if (rc) return rc;
    LargeEig r{};
    if ((rc = eigen_large_run(n, a, nullptr, *ws, ws->stream, &r))) return rc;
    const cudaStream_t s = ws->stream;
    const size_t nn = (size_t)n * n;
    int counts[2] = {0, 0};
    CK(cudaMemcpyAsync(w, r.eps, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(v, r.Z, nn * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(counts, r.counts, sizeof counts, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (counts[1] & 3) return fail(AM1GPU_LINALG, "inverse iteration produced an eigenvector of zero or non-finite norm");
    if (counts[1] & 4) return fail(AM1GPU_LINALG, "inverse iteration did not converge for an eigenvector (growth below the dstein threshold)");
    return AM1GPU_OK;
}

int eigen_large_run(int n, const double* a_host, const double* a_dev, Mem& m, cudaStream_t s, LargeEig* out) {
    const size_t nn = (size_t)n * n;
    const int nref = n - 2;
    const int P = cdiv(nref, kWyNb) * kWyNb, nblk = P / kWyNb;
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        off = align256(off);
        const size_t o2 = off;
        off += bytes;
        return o2;
    };
    const size_t kwork = (size_t)4 * TRP_B * n + 2 * (size_t)n + 1024 * (2 * TRP_B + 2) + 8;
    const size_t o_a = take(nn * 8), o_w = take(nn * 8), o_k = take(kwork * 8), o_z = take(nn * 8),
                 o_u = take(3 * std::max(nn, (size_t)P * n) * 8), o_s = take((size_t)2 * nblk * kWyNb * kWyNb * 8),
                 o_y = take((size_t)kWyNb * n * 8), o_d = take((size_t)n * 8), o_e = take((size_t)n * 8),
                 o_eps = take((size_t)n * 8), o_sh = take((size_t)n * 8), o_sc = take((size_t)n * 8), o_cl = take((size_t)n * 4),
                 o_cll = take((size_t)n * 4), o_cnt = take(16), o_tn = take(16), o_job = take(sizeof(TriJob));
    const size_t hbytes = align256(nn * 8) + 256;
    int rc = mem_ensure(m, align256(off), hbytes);
    if (rc) return rc;
    Workspace* ws = &m;
    char* D = ws->dpool;
    TriJob tj{};
    tj.A = (const double*)(D + o_a);
    tj.W = (double*)(D + o_w);
    tj.work = (double*)(D + o_k);
    tj.d = (double*)(D + o_d);
    tj.e = (double*)(D + o_e);
    tj.eps = (double*)(D + o_eps);
    tj.n = n;
    tj.mol = 0;
    if (a_host) {
        std::memcpy(ws->hpin, a_host, nn * 8);
        CK(cudaMemcpyAsync(D + o_a, ws->hpin, nn * 8, cudaMemcpyHostToDevice, s));
    } else {
        CK(cudaMemcpyAsync(D + o_a, a_dev, nn * 8, cudaMemcpyDeviceToDevice, s));
    }
    std::memcpy(ws->hpin + align256(nn * 8), &tj, sizeof tj);
    CK(cudaMemcpyAsync(D + o_job, ws->hpin + align256(nn * 8), sizeof tj, cudaMemcpyHostToDevice, s));
    // the lower triangle, mirrored (the reference's Side::Lower)
    k_mirror_lower<<<dim3((unsigned)cdiv(n, 32), (unsigned)cdiv(n, 32)), dim3(32, 8), 0, s>>>((double*)(D + o_a), n);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(D + o_cnt, 0, 16, s));
    Batch b;
    b.d_tri = (TriJob*)(D + o_job);
    b.maxn = n;
    b.tri_big = {tj};
    int64_t launches = 0;
    if ((rc = launch_big_tridiag(b, s, &launches))) return rc;
    bisect_launch(b.d_tri, 1, n, s, false);
    CK(cudaGetLastError());
    SteinJob sj{};
    sj.d = tj.d;
    sj.e = tj.e;
    sj.eps = tj.eps;
    sj.shift = (double*)(D + o_sh);
    sj.cl = (int*)(D + o_cl);
    sj.cl_list = (int*)(D + o_cll);
    sj.counts = (int*)(D + o_cnt);
    sj.scale = (double*)(D + o_sc);
    sj.tn = (double*)(D + o_tn);
    sj.Z = (double*)(D + o_z);
    sj.U = (double*)(D + o_u);
    sj.Zt = (double*)(D + o_a);  // the input is dead after the reduction
    sj.n = n;
    k_stein_prep<<<1, 1024, 0, s>>>(sj);
    for (int it = 0; it < 4; ++it) {
        k_stein_solve<<<cdiv(n, 64), 64, 0, s>>>(sj, it == 0 ? 1 : 0, it == 3 ? 1 : 0);
        k_stein_orth<<<std::max(1, n / 2), 256, sizeof(double) * n, s>>>(sj);
    }
    k_stein_scale<<<8 * g_sms, 256, 0, s>>>(sj);
    CK(cudaGetLastError());
    // back-transformation: Vt | V | U_wy in the (now dead) factor storage, then S | T, Y
    double* Vt = (double*)(D + o_u);
    double* V = Vt + (size_t)P * n;
    double* Uw = V + (size_t)n * P;
    double* S = (double*)(D + o_s);
    double* T = S + (size_t)nblk * kWyNb * kWyNb;
    double* Y = (double*)(D + o_y);
    double* Z = sj.Z;
    const long long blk = (long long)kWyNb * kWyNb, panel = (long long)kWyNb * n;
    k_wy_split<<<dim3((unsigned)cdiv(n, 32), (unsigned)(P / 32)), dim3(32, 8), 0, s>>>(tj.W, n, nref, P, Vt, V);
    CK(cudaGetLastError());
    if ((rc = dgemm(s, Vt, n, panel, V, P, kWyNb, S, kWyNb, blk, kWyNb, kWyNb, n, 0, nblk))) return rc;  // S_b = Vt_b V_b
    k_wy_tfactor<<<nblk, kWyNb, 0, s>>>(S, tj.W, tj.e, n, nref, T);
    CK(cudaGetLastError());
    if ((rc = dgemm(s, T, kWyNb, blk, Vt, n, panel, Uw, n, panel, kWyNb, n, kWyNb, 0, nblk))) return rc;  // U_b = T_b Vt_b
    for (int bi = nblk - 1; bi >= 0; --bi) {
        const int k = bi * kWyNb;  // column k of U_b and row k of V_b are zero: the products start there
        if ((rc = dgemm(s, Uw + (size_t)bi * panel + k, n, 0, Z + (size_t)k * n, n, 0, Y, n, 0, kWyNb, n, n - k, 0, 1))) return rc;
        if ((rc = dgemm(s, V + (size_t)k * P + k, P, 0, Y, n, 0, Z + (size_t)k * n, n, 0, n - k, n, kWyNb, 1, 1))) return rc;
    }
    out->Z = Z;
    out->eps = (double*)(D + o_eps);
    out->counts = (int*)(D + o_cnt);
    out->spare = (double*)(D + o_w);  // the reduction's working copy: free after the back-transformation
    return AM1GPU_OK;
}

// A molecule above 448 orbitals has no cluster Jacobi job, so when its purification stalls (a
// tiny HOMO-LUMO gap) its density comes from the large-matrix eigensolver instead: the
// eigenvectors Z of its F* and P = w Z_occ Z_occ^T, as the reference forms every density from
// an eigendecomposition (src/scf.rs:503-524, 654-657).  One flag read per iteration, only in
// batches that hold such molecules; the rare stalled molecule is then solved on the batch's
// stream, one at a time, in a separate device pool.
int big_fallback(Batch& b, Mem* ws) {
    const cudaStream_t s = ws->stream;
    CK(cudaMemcpyAsync(b.h_active + 3, b.d_active + 3, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (b.h_active[3] == 0) return AM1GPU_OK;
    std::vector<int> flags(b.jobs.size(), 0);
    CK(cudaMemcpyAsync(flags.data(), b.d_big_stall, sizeof(int) * flags.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    static const int kLinalg = AM1GPU_LINALG;
    for (size_t j = 0; j < flags.size(); ++j) {
        if (!flags[j]) continue;
        const ChanJob& cj = b.jobs[j];
        const MolDesc& md = b.mols[cj.mol];
        const int n = cj.n, nocc = md.n_occ[cj.ch];
        LargeEig r{};
        int rc = eigen_large_run(n, nullptr, cj.Fx, tl_mem_eig, s, &r);
        if (rc) return rc;
        if (nocc > 0) {
            k_transpose_cols<<<dim3(cdiv(n, 32), cdiv(nocc, 32)), dim3(32, 8), 0, s>>>(r.Z, n, nocc, r.spare);
            CK(cudaGetLastError());
            if ((rc = dgemm(s, r.Z, n, 0, r.spare, n, 0, cj.Pnew, n, 0, n, n, nocc, 0, 1))) return rc;
            k_sym_scale<<<dim3(cdiv(n, 32), cdiv(n, 32)), dim3(32, 8), 0, s>>>(cj.Pnew, n, md.occ_weight);
            CK(cudaGetLastError());
        } else {
            CK(cudaMemsetAsync(cj.Pnew, 0, sizeof(double) * n * n, s));
        }
        int counts[2] = {0, 0};
        CK(cudaMemcpyAsync(counts, r.counts, sizeof counts, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (counts[1])  // no usable eigenvectors: the molecule ends with LINALG, as it did before this fallback
            CK(cudaMemcpyAsync(b.d_status + cj.mol, &kLinalg, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(b.d_big_stall + j, 0, sizeof(int), s));
    }
    CK(cudaMemsetAsync(b.d_active + 3, 0, sizeof(int), s));
    CK(cudaStreamSynchronize(s));
    return AM1GPU_OK;
}

// Density of one symmetric matrix F by purification, P = w * (projector onto its nocc lowest
// eigenvectors): the step an SCF iteration takes after the extrapolation (the reference's
// symmetric_eigen + density_from_coeff, src/scf.rs:654-661, 503-524), alone, at the precision of
// the batched path's products: 0 FP64 tensor cores (k_sp2_step_tma/16/8), 1 FP32-accurate products on
// tcgen05 (k_sp2_step_tc, 3xTF32), 2 TF32 mma.sync (k_sp2_step_tf32), 3 FP64 from digit planes
// (k_sp2_step_oz), 4 TF32 on tcgen05 in one pass (k_sp2_step_tc1).  The reduced-precision runs
// stop at their own rounding floor and are rescaled to the exact trace, as in the mixed SCF.
int density_purify_one(int n, const double* F, double nocc, double weight, int precision, double* P, int* steps_out,
                       Mem* mem_override = nullptr) {
    g_err.clear();
    if (n < 1 || n > 448 || !F || !P) return fail(AM1GPU_INVALID_INPUT, "n must be 1..448 and the pointers non-null");
    if (precision < 0 || precision > 4) return fail(AM1GPU_INVALID_INPUT, "precision must be 0, 1, 2, 3 or 4");
    if (!(nocc >= 0.0 && nocc <= n)) return fail(AM1GPU_INVALID_INPUT, "nocc outside 0..n");
    for (long long i = 0; i < (long long)n * n; ++i)
        if (!std::isfinite(F[i])) return fail(AM1GPU_LINALG, "the matrix is not finite");
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    const long long nn = (long long)n * n;
    const int ldf = (n + 3) & ~3;
    const int t64 = (n + 63) / 64, t128 = (n + 127) / 128;
    const int nt64 = t64 * (t64 + 1) / 2, nt128 = t128 * (t128 + 1) / 2, ntoz = oz_tiles_of(n);
    const int ldq = oz_ldq(n);
    const int nblk = sp2_init_blocks(n);
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        off = align256(off);
        const size_t o = off;
        off += bytes;
        return o;
    };
    const size_t o_job = take(sizeof(Sp2Job)), o_maps = take(4 * sizeof(TmaDesc)), o_xfmaps = take(2 * sizeof(TmaDesc)),
                 o_t64 = take(sizeof(GemmTile) * nt64),
                 o_t128 = take(sizeof(GemmTile) * nt128),
                 o_toz = take(sizeof(GemmTile) * ntoz),
                 o_ms = take(sizeof(MolState)), o_f = take(8 * nn), o_rmin = take(8 * (size_t)n), o_rmax = take(8 * (size_t)n);
    const size_t staged = align256(off);
    const size_t o_sst = take(sizeof(Sp2State)), o_bnd = take(32), o_x0 = take(8 * nn), o_x1 = take(8 * nn), o_p = take(8 * nn),
                 o_part = take(16 * (size_t)std::max(32, nt64)), o_xf = take(8 * (size_t)n * ldf + 64), o_need = take(16),
                 o_work = take(8 * kWorkN), o_act = take(16), o_stall = take(16),
                 o_dq = take(2 * (size_t)kOzPlanes * n * ldq);
    Workspace* ws;
    if (mem_override) {
        if ((rc = mem_ensure(*mem_override, align256(off), staged + align256(sizeof(Sp2State)) + 256))) return rc;
        ws = mem_override;
    } else if ((rc = workspace(&ws, align256(off), staged + align256(sizeof(Sp2State)) + 256))) {
        return rc;
    }
    char* D = ws->dpool;
    char* H = ws->hpin;
    const cudaStream_t s = ws->stream;
    Sp2Job jb{};
    jb.F = (const double*)(D + o_f);
    jb.rowmin = (const double*)(D + o_rmin);
    jb.rowmax = (const double*)(D + o_rmax);
    jb.X0 = (double*)(D + o_x0);
    jb.X1 = (double*)(D + o_x1);
    jb.P = (double*)(D + o_p);
    jb.part = (double*)(D + o_part);
    jb.bounds = (double*)(D + o_bnd);
    jb.nocc = nocc;
    jb.weight = weight;
    jb.n = n;
    jb.mol = 0;
    jb.tile0 = 0;
    jb.ntiles = nt64;
    jb.fallback = 1;
    jb.ldf = ldf;
    jb.Xf0 = (float*)(((uintptr_t)(D + o_xf) + 15) & ~(uintptr_t)15);
    jb.Xf1 = jb.Xf0 + (size_t)n * ldf;
    jb.lowp_tc = precision == 1 ? 1 : precision == 4 ? 2 : 0;
    jb.tc_tile0 = 0;
    jb.tc_ntiles = (precision == 1 || precision == 4) ? nt128 : 0;
    jb.oz = precision == 3 ? 1 : 0;
    jb.oz_tile0 = 0;
    jb.oz_ntiles = precision == 3 ? ntoz : 0;
    jb.ldq = ldq;
    jb.Dq0 = (int8_t*)(D + o_dq);
    jb.Dq1 = jb.Dq0 + (size_t)kOzPlanes * n * ldq;
    std::memcpy(H + o_job, &jb, sizeof jb);
    TmaDesc* hmaps = (TmaDesc*)(H + o_maps);
    const bool tma = encode_square_map(&hmaps[0], jb.X0, n) && encode_square_map(&hmaps[1], jb.X1, n);
    TmaDesc* hxfmaps = (TmaDesc*)(H + o_xfmaps);
    if (precision == 4 && !(encode_rows_map_f32(&hxfmaps[0], jb.Xf0, ldf, n) && encode_rows_map_f32(&hxfmaps[1], jb.Xf1, ldf, n)))
        return fail(AM1GPU_UNSUPPORTED, "no tensor-map encoder on this device: the single-pass tcgen05 products are not available");
    GemmTile* hoz = (GemmTile*)(H + o_toz);
    int koz = 0;
    for (int tm = 0; tm < t128; ++tm)
        for (int tn = 0; tn < (n + 47) / 48; ++tn)
            if (48 * tn + 47 >= 128 * tm) hoz[koz++] = GemmTile{0, tm, tn};
    GemmTile* h64 = (GemmTile*)(H + o_t64);
    GemmTile* h128 = (GemmTile*)(H + o_t128);
    int k = 0;
    for (int x = 0; x < t64; ++x)
        for (int y = x; y < t64; ++y) h64[k++] = GemmTile{0, x, y};
    k = 0;
    for (int x = 0; x < t128; ++x)
        for (int y = x; y < t128; ++y) h128[k++] = GemmTile{0, x, y};
    MolState ms{};
    ms.active = 1;
    ms.lowp = (precision == 1 || precision == 2 || precision == 4) ? 1 : 0;
    std::memcpy(H + o_ms, &ms, sizeof ms);
    double* hf = (double*)(H + o_f);
    double* hmin = (double*)(H + o_rmin);
    double* hmax = (double*)(H + o_rmax);
    for (int r = 0; r < n; ++r) {  // the lower triangle, mirrored (Side::Lower), and its Gershgorin row bounds
        double bound = 0.0;
        for (int c = 0; c < n; ++c) {
            const double v = r >= c ? F[(size_t)r * n + c] : F[(size_t)c * n + r];
            hf[(size_t)r * n + c] = v;
            if (c != r) bound += std::fabs(v);
        }
        hmin[r] = hf[(size_t)r * n + r] - bound;
        hmax[r] = hf[(size_t)r * n + r] + bound;
    }
    CK(cudaMemcpyAsync(D, H, staged, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(D + o_work, 0, 8 * kWorkN, s));
    CK(cudaMemsetAsync(D + o_need, 0, 16, s));
    CK(cudaMemsetAsync(D + o_act, 0, 16, s));
    CK(cudaMemsetAsync(D + o_stall, 0, 16, s));
    const Sp2Job* dj = (const Sp2Job*)(D + o_job);
    Sp2State* dsst = (Sp2State*)(D + o_sst);
    const MolState* dms = (const MolState*)(D + o_ms);
    const GemmTile* d64 = (const GemmTile*)(D + o_t64);
    const GemmTile* d128 = (const GemmTile*)(D + o_t128);
    int* dact = (int*)(D + o_act);
    k_sp2_bounds<<<1, 512, 3 * sizeof(double) * n, s>>>(dj, dms);
    k_sp2_init<<<dim3(nblk, 1), 256, 0, s>>>(dj, dsst, dms, nblk);
    k_sp2_start<<<1, 128, 0, s>>>(dj, dsst, dms, 1, nblk);
    CK(cudaGetLastError());
    const bool pairs = n % 2 == 0;  // every slot here starts on 256 bytes
    int* hact = (int*)(H + staged);
    for (int step = 0; step < kSp2MaxSteps; ++step) {
        if (precision == 0) {
            if (tma)
                k_sp2_step_tma<<<nt64, 128, dgemm_tma_smem_bytes(), s>>>(dj, d64, nt64, dsst, (const TmaDesc*)(D + o_maps), dact + 2);
            else if (pairs)
                k_sp2_step16<<<nt64, 128, dgemm_smem_bytes(), s>>>(dj, d64, nt64, dsst);
            else
                k_sp2_step8<<<nt64, 128, dgemm_smem_bytes(), s>>>(dj, d64, nt64, dsst);
        } else if (precision == 3) {
            k_sp2_step_oz<<<ntoz, 128, oz_smem_bytes(), s>>>(dj, (const GemmTile*)(D + o_toz), ntoz, dsst, dact + 2);
        } else if (precision == 2) {
            k_sp2_step_tf32<<<nt64, 128, tf32_smem_bytes(), s>>>(dj, d64, nt64, dsst);
        } else if (precision == 4) {
            k_sp2_step_tc1<<<nt128, 128, tc1_smem_bytes(), s>>>(dj, d128, nt128, dsst, (const TmaDesc*)(D + o_xfmaps), dact + 2);
        } else {
            k_sp2_step_tc<<<nt128, 128, tc_smem_bytes(), s>>>(dj, d128, nt128, dsst, dact + 2);
        }
        CK(cudaMemsetAsync(dact, 0, sizeof(int), s));
        k_sp2_update<<<1, 128, 0, s>>>(dj, dsst, 1, kSp2MaxSteps, dact, (double*)(D + o_work));
        CK(cudaGetLastError());
        if (step >= 12 && (step % 6) == 5) {
            CK(cudaMemcpyAsync(hact, dact, 16, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (hact[0] == 0) break;
        }
    }
    k_sp2_finish<<<dim3(std::max(8u, std::min(256u, cdiv(nn, 65536))), 1), 256, 0, s>>>(dj, dsst, dms, (int*)(D + o_need),
                                                                                       (double*)(D + o_work), (int*)(D + o_stall),
                                                                                       dact + 3);
    CK(cudaGetLastError());
    Sp2State* hs = (Sp2State*)(H + staged + 256);
    CK(cudaMemcpyAsync(hs, dsst, sizeof(Sp2State), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hact, dact, 16, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(P, D + o_p, 8 * nn, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (steps_out) *steps_out = hs->steps;
    if (hact[2] & (1 << 10)) return fail(AM1GPU_LINALG, "a purification iterate left the range of its digit planes (|x| >= 2)");
    if (hact[2]) return fail(AM1GPU_DEVICE_ERROR, "a tensor-core step gave up waiting for its MMAs or operand copies");
    if (!hs->converged) return fail(AM1GPU_LINALG, "the purification did not reach idempotency (gap too small)");
    return AM1GPU_OK;
}

int symmetric_eigen_one(int n, const double* a, double* w, double* v, Mem* mem_override = nullptr) {
    g_err.clear();
    if (n < 0 || (n > 0 && (!a || !w || !v))) return fail(AM1GPU_INVALID_INPUT, "null argument");
    if (n == 0) return AM1GPU_OK;
    for (long long i = 0; i < (long long)n * n; ++i)
        if (!std::isfinite(a[i])) {
            return fail(AM1GPU_LINALG, "the " + std::to_string(n) + "x" + std::to_string(n) +
                                           " matrix handed to the eigensolver is not finite: element (" + std::to_string(i / n) +
                                           ", " + std::to_string(i % n) + ")");
        }
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    int npad, C;
    if (!choose_cluster(n, &npad, &C)) {
        if (n > kMaxAo) return fail(AM1GPU_UNSUPPORTED, "matrix with " + std::to_string(n) + " rows exceeds " + std::to_string(kMaxAo));
        return symmetric_eigen_large(n, a, w, v, mem_override);
    }
    // layout: Gt (n*n, the lower triangle mirrored), Ct (n*n identity), Vs (npad*n), lam, colid, eps, rowmin, state
    const size_t nn = (size_t)n * n;
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        off = align256(off);
        const size_t o2 = off;
        off += bytes;
        return o2;
    };
    const size_t o_g = take(nn * 8), o_c = take(nn * 8), o_v = take((size_t)npad * n * 8), o_l = take(npad * 8),
                 o_id = take(npad * 4), o_e = take(n * 8), o_r = take(n * 8), o_st = take(sizeof(MolState)),
                 o_status = take(16), o_job = take(sizeof(EigJob));
    Workspace* ws;
    if (mem_override) {
        rc = mem_ensure(*mem_override, align256(off), align256(off));
        ws = mem_override;
    } else {
        rc = workspace(&ws, align256(off), align256(off));
    }
    if (rc) return rc;
    char* D = ws->dpool;
    char* Hh = ws->hpin;
    double* g = (double*)(Hh + o_g);
    double* c = (double*)(Hh + o_c);
    double* rmin = (double*)(Hh + o_r);
    for (int i = 0; i < n; ++i) {
        double bound = 0.0;
        for (int j = 0; j < n; ++j) {
            const double x = i >= j ? a[(size_t)i * n + j] : a[(size_t)j * n + i];  // lower triangle
            g[(size_t)i * n + j] = x;
            c[(size_t)i * n + j] = i == j ? 1.0 : 0.0;
            if (i != j) bound += std::fabs(x);
        }
        rmin[i] = g[(size_t)i * n + i] - bound;
    }
    MolState* hs = (MolState*)(Hh + o_st);
    *hs = MolState{};
    hs->active = 1;
    EigJob* ej = (EigJob*)(Hh + o_job);
    *ej = EigJob{};
    ej->Gt = (double*)(D + o_g);
    ej->Ct = (double*)(D + o_c);
    ej->Vs = (double*)(D + o_v);
    ej->lam = (double*)(D + o_l);
    ej->colid_out = (int*)(D + o_id);
    ej->eps = (double*)(D + o_e);
    ej->Ct_out = (double*)(D + o_c);
    ej->rowmin = (double*)(D + o_r);
    ej->n = n;
    ej->npad = npad;
    ej->mol = 0;
    std::memset(Hh + o_status, 0, 16);
    CK(cudaMemcpyAsync(D, Hh, align256(off), cudaMemcpyHostToDevice, ws->stream));
    Batch b;
    b.d_eig = (EigJob*)(D + o_job);
    b.d_st = (MolState*)(D + o_st);
    b.d_status = (int*)(D + o_status);
    b.buckets = {{0, 1, C, jacobi_smem_bytes(n, npad, C)}};
    b.neig = 1;
    rc = launch_jacobi(b, ws, 1);
    if (rc) return rc;
    k_eig_sort<<<1, 512, 0, ws->stream>>>(b.d_eig, b.d_st, 1, nullptr);
    CK(cudaGetLastError());
    std::vector<double> ct(nn);
    int st = 0;
    CK(cudaMemcpyAsync(w, D + o_e, n * 8, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaMemcpyAsync(ct.data(), D + o_c, nn * 8, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaMemcpyAsync(&st, D + o_status, 4, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaStreamSynchronize(ws->stream));
    if (st) return fail(AM1GPU_LINALG, "Jacobi eigensolver did not converge");
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) v[(size_t)i * n + k] = ct[(size_t)k * n + i];
    return AM1GPU_OK;
}

// Eigenvalues only, of one symmetric matrix of up to kMaxAo rows: the final-spectrum path of the
// SCF (on-chip cluster reduction while the matrix fits a cluster's shared memory, a cluster over
// global memory below kBigGridN rows, the blocked whole-GPU reduction above), then bisection.
int symmetric_eigenvalues_one(int n, const double* a, double* w) {
    g_err.clear();
    if (n < 0 || (n > 0 && (!a || !w))) return fail(AM1GPU_INVALID_INPUT, "null argument");
    if (n == 0) return AM1GPU_OK;
    if (n > kMaxAo) return fail(AM1GPU_UNSUPPORTED, "matrix with " + std::to_string(n) + " rows exceeds " + std::to_string(kMaxAo));
    for (long long i = 0; i < (long long)n * n; ++i)
        if (!std::isfinite(a[i])) return fail(AM1GPU_LINALG, "the matrix handed to the eigensolver is not finite");
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    const size_t nn = (size_t)n * n;
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        off = align256(off);
        const size_t o2 = off;
        off += bytes;
        return o2;
    };
    const size_t o_a = take(nn * 8), o_w = take(nn * 8), o_k = take(std::max(nn, (size_t)4 * TRP_B * n + 2 * n + 1024 * (2 * TRP_B + 2)) * 8),
                 o_d = take((size_t)n * 8), o_e = take((size_t)n * 8), o_eps = take((size_t)n * 8), o_job = take(sizeof(TriJob));
    Workspace* ws;
    rc = workspace(&ws, align256(off), align256(o_k));
    if (rc) return rc;
    char* D = ws->dpool;
    TriJob tj{};
    tj.A = (const double*)(D + o_a);
    tj.W = (double*)(D + o_w);
    tj.work = (double*)(D + o_k);
    tj.d = (double*)(D + o_d);
    tj.e = (double*)(D + o_e);
    tj.eps = (double*)(D + o_eps);
    tj.n = n;
    tj.mol = 0;
    std::memcpy(ws->hpin, a, nn * 8);  // the matrix through pinned staging, then the job record
    std::memcpy(ws->hpin + align256(nn * 8), &tj, sizeof tj);
    CK(cudaMemcpyAsync(D + o_a, ws->hpin, nn * 8, cudaMemcpyHostToDevice, ws->stream));
    CK(cudaMemcpyAsync(D + o_job, ws->hpin + align256(nn * 8), sizeof tj, cudaMemcpyHostToDevice, ws->stream));
    // the lower triangle, mirrored (the reference's Side::Lower, as am1gpu_symmetric_eigen)
    k_mirror_lower<<<dim3((unsigned)cdiv(n, 32), (unsigned)cdiv(n, 32)), dim3(32, 8), 0, ws->stream>>>((double*)(D + o_a), n);
    CK(cudaGetLastError());
    Batch b;
    b.d_tri = (TriJob*)(D + o_job);
    b.maxn = n;
    const int C = tridiag_cluster(n);
    if (C) {
        b.tri_buckets = {{0, 1, C, tridiag_smem_bytes(n, C)}};
        rc = launch_tridiag(b, ws);
    } else {
        b.tri_big = {tj};
        int64_t launches = 0;
        rc = launch_big_tridiag(b, ws->stream, &launches);
    }
    if (rc) return rc;
    bisect_launch(b.d_tri, 1, n, ws->stream, true);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(w, D + o_eps, (size_t)n * 8, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaStreamSynchronize(ws->stream));
    return AM1GPU_OK;
}

// Many independent symmetric eigenproblems in one set of launches: the subsystem blocks of the
// divide-and-conquer SCF (solve_subsystems, src/divide_conquer.rs:587-617), each of which the
// reference diagonalises with its own symmetric_eigen call.  Every matrix gets the cluster Jacobi
// job symmetric_eigen_one would give it (same cluster size, same arithmetic), the jobs are
// grouped by cluster size and launched together, then sorted.  status[i] receives matrix i's
// code; the return value is the first nonzero one.
int symmetric_eigen_batch(int count, const int32_t* ns, const double* const* a, double* const* w, double* const* v, int32_t* status) {
    g_err.clear();
    if (count < 0 || (count > 0 && (!ns || !a || !w || !v))) return fail(AM1GPU_INVALID_INPUT, "null argument");
    int first = AM1GPU_OK;
    std::string first_msg;
    auto set = [&](int i, int code, const std::string& msg) {
        if (status) status[i] = code;
        if (code && !first) {
            first = code;
            first_msg = msg;
        }
    };
    struct Item {
        int i, n, npad, C;
        size_t o_g, o_c, o_v, o_l, o_id, o_e, o_r;
    };
    std::vector<Item> items;
    std::vector<int> large;
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        off = align256(off);
        const size_t o2 = off;
        off += bytes;
        return o2;
    };
    for (int i = 0; i < count; ++i) {
        const int n = ns[i];
        set(i, AM1GPU_OK, "");
        if (n < 0 || (n > 0 && (!a[i] || !w[i] || !v[i]))) {
            set(i, AM1GPU_INVALID_INPUT, "matrix " + std::to_string(i) + ": null argument or negative size");
            continue;
        }
        if (n == 0) continue;
        bool finite = true;
        for (long long k = 0; k < (long long)n * n && finite; ++k) finite = std::isfinite(a[i][k]);
        if (!finite) {
            set(i, AM1GPU_LINALG, "matrix " + std::to_string(i) + " handed to the eigensolver is not finite");
            continue;
        }
        Item it{i, n, 0, 0};
        if (!choose_cluster(n, &it.npad, &it.C)) {
            if (n > kMaxAo)
                set(i, AM1GPU_UNSUPPORTED, "matrix " + std::to_string(i) + " has more than " + std::to_string(kMaxAo) + " rows");
            else
                large.push_back(i);  // past the cluster Jacobi: the large-matrix path, one at a time, after the batch
            continue;
        }
        const size_t nn = (size_t)n * n;
        it.o_g = take(nn * 8);
        it.o_c = take(nn * 8);
        it.o_v = take((size_t)it.npad * n * 8);
        it.o_l = take((size_t)it.npad * 8);
        it.o_id = take((size_t)it.npad * 4);
        it.o_e = take((size_t)n * 8);
        it.o_r = take((size_t)n * 8);
        items.push_back(it);
    }
    if (!items.empty()) {
        // cluster-size groups, largest clusters (and matrices) first, as the batched SCF orders them
        std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.C != y.C ? x.C > y.C : x.n > y.n; });
        const int m = (int)items.size();
        const size_t o_st = take(sizeof(MolState) * m), o_status = take(sizeof(int) * m), o_job = take(sizeof(EigJob) * m);
        DeviceCtx* ctx;
        int rc = device_ctx(&ctx);
        if (rc) return rc;
        Workspace* ws;
        rc = workspace(&ws, align256(off), align256(off));
        if (rc) return rc;
        char* D = ws->dpool;
        char* Hh = ws->hpin;
        Batch b;
        b.buckets.clear();
        for (int k = 0; k < m; ++k) {
            const Item& it = items[k];
            const int n = it.n;
            const double* ak = a[it.i];
            double* g = (double*)(Hh + it.o_g);
            double* c = (double*)(Hh + it.o_c);
            double* rmin = (double*)(Hh + it.o_r);
            for (int r = 0; r < n; ++r) {
                double bound = 0.0;
                for (int q = 0; q < n; ++q) {
                    const double x = r >= q ? ak[(size_t)r * n + q] : ak[(size_t)q * n + r];  // lower triangle
                    g[(size_t)r * n + q] = x;
                    c[(size_t)r * n + q] = r == q ? 1.0 : 0.0;
                    if (r != q) bound += std::fabs(x);
                }
                rmin[r] = g[(size_t)r * n + r] - bound;
            }
            MolState* hs = (MolState*)(Hh + o_st) + k;
            *hs = MolState{};
            hs->active = 1;
            EigJob* ej = (EigJob*)(Hh + o_job) + k;
            *ej = EigJob{};
            ej->Gt = (double*)(D + it.o_g);
            ej->Ct = (double*)(D + it.o_c);
            ej->Vs = (double*)(D + it.o_v);
            ej->lam = (double*)(D + it.o_l);
            ej->colid_out = (int*)(D + it.o_id);
            ej->eps = (double*)(D + it.o_e);
            ej->Ct_out = (double*)(D + it.o_c);
            ej->rowmin = (double*)(D + it.o_r);
            ej->n = n;
            ej->npad = it.npad;
            ej->mol = k;
            const size_t sm = jacobi_smem_bytes(n, it.npad, it.C);
            if (b.buckets.empty() || b.buckets.back().C != it.C) b.buckets.push_back({k, 0, it.C, 0});
            b.buckets.back().count++;
            b.buckets.back().smem = std::max(b.buckets.back().smem, sm);
        }
        std::memset(Hh + o_status, 0, sizeof(int) * m);
        CK(cudaMemcpyAsync(D, Hh, align256(off), cudaMemcpyHostToDevice, ws->stream));
        b.d_eig = (EigJob*)(D + o_job);
        b.d_st = (MolState*)(D + o_st);
        b.d_status = (int*)(D + o_status);
        b.neig = m;
        rc = launch_jacobi(b, ws, 1);
        if (rc) return rc;
        k_eig_sort<<<m, 512, 0, ws->stream>>>(b.d_eig, b.d_st, 1, nullptr);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(Hh, D, align256(off), cudaMemcpyDeviceToHost, ws->stream));
        CK(cudaStreamSynchronize(ws->stream));
        for (int k = 0; k < m; ++k) {
            const Item& it = items[k];
            const int n = it.n;
            if (((int*)(Hh + o_status))[k]) {
                set(it.i, AM1GPU_LINALG, "matrix " + std::to_string(it.i) + ": Jacobi eigensolver did not converge");
                continue;
            }
            std::memcpy(w[it.i], Hh + it.o_e, sizeof(double) * n);
            const double* ct = (const double*)(Hh + it.o_c);
            for (int q = 0; q < n; ++q)
                for (int r = 0; r < n; ++r) v[it.i][(size_t)r * n + q] = ct[(size_t)q * n + r];
        }
    }
    if (!large.empty()) {
        DeviceCtx* ctx;
        const int rc = device_ctx(&ctx);
        if (rc) return rc;
    }
    for (int i : large) {
        const int rc = symmetric_eigen_large(ns[i], a[i], w[i], v[i], nullptr);
        if (rc == AM1GPU_DEVICE_ERROR) return rc;
        set(i, rc, rc ? "matrix " + std::to_string(i) + ": " + g_err : std::string());
    }
    if (first) g_err = first_msg;
    return first;
}

}  // namespace am1

// A resident batch: inputs uploaded once, device memory and stream owned by the handle.
struct am1gpu_batch {
    am1::Mem mem;
    am1::Batch b;
    am1gpu_options opts;
    std::vector<int> status;   // validation result per caller molecule
    std::vector<int> planned;  // caller index -> batch index, or -1
    int nmol = 0;
    am1gpu_call_stats stats{};
    const am1::DevElem* dp = nullptr;
    bool ran = false;
};

void am1::set_last_error(const std::string& msg) { am1::g_err = msg; }

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" {

void am1gpu_default_options(am1gpu_options* o) {
    if (!o) return;
    o->reference = AM1GPU_REF_AUTO;
    o->method = AM1GPU_METHOD_AM1;
    o->max_scf = 200;
    o->use_diis = 1;
    o->accelerator = AM1GPU_ACCEL_ADIIS_CDIIS;
    o->precision = AM1GPU_PRECISION_FP64;
    o->e_tol = 1.0e-8;
    o->p_tol = 1.0e-7;
    o->adiis_switch = 0.1;
}

int am1gpu_basis_size(int32_t natoms, const int32_t* z, int32_t method, int32_t* nao) {
    if (natoms < 0 || (natoms > 0 && !z) || !nao) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    int tot = 0;
    for (int i = 0; i < natoms; ++i) {
        if (z[i] < 0 || z[i] > am1::MAX_Z || !am1::helem(method == 1, z[i]).present)
            return am1::fail(AM1GPU_ELEMENT_NOT_PARAMETERIZED, "element Z=" + std::to_string(z[i]) + " is not parameterized");
        tot += am1::helem(method == 1, z[i]).norb;
    }
    *nao = tot;
    return AM1GPU_OK;
}

int am1gpu_element_params(int32_t method, int32_t z, am1gpu_element* out) {
    if (!out) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    if (method != AM1GPU_METHOD_AM1 && method != AM1GPU_METHOD_RM1) return am1::fail(AM1GPU_INVALID_INPUT, "unknown method");
    if (z < 1 || z > am1::MAX_Z || !am1::helem(method == 1, z).present)
        return am1::fail(AM1GPU_ELEMENT_NOT_PARAMETERIZED, std::string(method == 1 ? "RM1" : "AM1") + " has no parameters for element Z=" +
                                                               std::to_string(z));
    am1::element_to_abi(am1::helem(method == 1, z), z, out);
    return AM1GPU_OK;
}

int am1gpu_derive_element(int32_t z, const double raw[12], const double gauss[12], am1gpu_element* out) {
    if (!raw || !gauss || !out) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    if (z < 1 || z > am1::MAX_Z) return am1::fail(AM1GPU_INVALID_INPUT, "atomic number outside 1..86");
    am1::element_to_abi(am1::derive_from_raw(z, raw, gauss), z, out);
    return AM1GPU_OK;
}

int am1gpu_scf_params(const am1gpu_molecule* mol, const am1gpu_param_table* params, const am1gpu_options* opts, am1gpu_result* res) {
    if (!mol || !opts || !res) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    int32_t st = 0;
    am1gpu_options o = *opts;
    o.precision = AM1GPU_PRECISION_FP64;  // the plain path is FP64 throughout
    return am1::scf_batch(1, mol, &o, res, &st, nullptr, params);
}

int am1gpu_scf_batch_params(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_param_table* params, const am1gpu_options* opts,
                            am1gpu_result* results, int32_t* status) {
    return am1::scf_batch(nmol, mols, opts, results, status, nullptr, params);
}

int am1gpu_gradient_batch_params(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_param_table* params,
                                 const am1gpu_options* opts, am1gpu_result* results, double* const* gradients, int32_t* status) {
    if (nmol > 0 && !gradients) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    return am1::scf_batch(nmol, mols, opts, results, status, gradients, params);
}

int am1gpu_scf(const am1gpu_molecule* mol, const am1gpu_options* opts, am1gpu_result* res) {
    if (!mol || !opts || !res) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    int32_t st = 0;
    am1gpu_options o = *opts;
    o.precision = AM1GPU_PRECISION_FP64;  // the plain path is FP64 throughout
    return am1::scf_batch(1, mol, &o, res, &st);
}

int am1gpu_gradient(const am1gpu_molecule* mol, const am1gpu_options* opts, am1gpu_result* res, double* gradient) {
    if (!mol || !opts || !res || !gradient) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    int32_t st = 0;
    am1gpu_options o = *opts;
    o.precision = AM1GPU_PRECISION_FP64;
    double* const g[1] = {gradient};
    return am1::scf_batch(1, mol, &o, res, &st, g);
}

int am1gpu_gradient_batch(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts, am1gpu_result* results,
                          double* const* gradients, int32_t* status) {
    if (nmol > 0 && !gradients) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    return am1::scf_batch(nmol, mols, opts, results, status, gradients);
}

int am1gpu_scf_batch(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts, am1gpu_result* results,
                     int32_t* status) {
    return am1::scf_batch(nmol, mols, opts, results, status);
}

int am1gpu_build_core(const am1gpu_molecule* mol, int32_t method, double* h_core, double* core_ev) {
    return am1::build_core_one(mol, method, h_core, core_ev);
}

int am1gpu_build_fock(const am1gpu_molecule* mol, int32_t method, const double* p_tot, const double* p_spin,
                      double spin_scale, double* fock) {
    return am1::build_fock_one(mol, method, p_tot, p_spin, spin_scale, fock);
}

int am1gpu_g_matrix_batch(const am1gpu_molecule* mol, int32_t method, int32_t nrhs, const double* densities, double* g) {
    return am1::g_matrix_batch(mol, method, nrhs, densities, g);
}

int am1gpu_symmetric_eigen_batch(int32_t count, const int32_t* n, const double* const* a, double* const* w, double* const* v,
                                 int32_t* status) {
    return am1::symmetric_eigen_batch(count, n, a, w, v, status);
}

int am1gpu_symmetric_eigenvalues(int32_t n, const double* a, double* w) { return am1::symmetric_eigenvalues_one(n, a, w); }

int am1gpu_lowp_tuning(int32_t* choice, float* ms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return am1::fail(AM1GPU_DEVICE_ERROR, "no CUDA device");
    am1::LowpTune& t = am1::g_lowp_tune[dev];
    std::lock_guard<std::mutex> lock(t.mu);
    for (int c = 0; c < am1::kTuneClasses; ++c) {
        if (choice) choice[c] = t.choice[c];
        if (ms)
            for (int k = 0; k < 3; ++k) ms[3 * c + k] = t.ms[c][k];
    }
    return AM1GPU_OK;
}

int am1gpu_density_purify(int32_t n, const double* f, double n_occ, double weight, int32_t precision, double* p, int32_t* steps) {
    int st = 0;
    const int rc = am1::density_purify_one(n, f, n_occ, weight, precision, p, &st);
    if (steps) *steps = st;
    return rc;
}

int am1gpu_symmetric_eigen(int32_t n, const double* a, double* w, double* v) {
    return am1::symmetric_eigen_one(n, a, w, v);
}

const char* am1gpu_last_error(void) { return am1::g_err.c_str(); }

int am1gpu_batch_create(int32_t nmol, const am1gpu_molecule* mols, const am1gpu_options* opts, am1gpu_batch** out) {
    using namespace am1;
    g_err.clear();
    if (!out || !opts || nmol < 0 || (nmol > 0 && !mols)) return fail(AM1GPU_INVALID_INPUT, "null argument");
    *out = nullptr;
    DeviceCtx* ctx;
    int rc = device_ctx(&ctx);
    if (rc) return rc;
    auto* h = new am1gpu_batch();
    h->opts = *opts;
    h->nmol = nmol;
    h->status.assign(nmol, AM1GPU_OK);
    h->planned.assign(nmol, -1);
    h->dp = ctx->d_params;
    std::vector<MolPlan> plans;
    for (int i = 0; i < nmol; ++i) {
        MolPlan p;
        const int r = plan_molecule(mols[i], *opts, i, p);
        h->status[i] = r;
        if (r == AM1GPU_OK) {
            h->planned[i] = (int)plans.size();
            plans.push_back(std::move(p));
        }
    }
    if (!plans.empty()) {
        if (opts->precision == AM1GPU_PRECISION_MIXED) rc = tune_lowp_kernels(plans);
        if (!rc) rc = build_batch(mols, *opts, std::move(plans), h->b, h->mem, &h->stats);
        h->b.graph_cacheable = true;
        if (!rc && cudaStreamSynchronize(h->mem.stream) != cudaSuccess) rc = fail(AM1GPU_DEVICE_ERROR, "upload failed");
        if (rc) {
            mem_release(h->mem);
            delete h;
            return rc;
        }
    }
    *out = h;
    return AM1GPU_OK;
}

int am1gpu_batch_run(am1gpu_batch* h) {
    using namespace am1;
    g_err.clear();
    if (!h) return fail(AM1GPU_INVALID_INPUT, "null batch");
    h->stats = am1gpu_call_stats{};
    if (h->b.nmol == 0) return AM1GPU_OK;
    int rc = run_device(h->b, h->mem, h->dp, h->opts, &h->stats);
    tl_stats = h->stats;
    h->ran = rc == AM1GPU_OK;
    return rc;
}

int am1gpu_batch_results(am1gpu_batch* h, am1gpu_result* results, int32_t* status) {
    using namespace am1;
    g_err.clear();
    if (!h || (h->nmol > 0 && !results)) return fail(AM1GPU_INVALID_INPUT, "null argument");
    if (h->b.nmol > 0 && !h->ran) return fail(AM1GPU_INVALID_INPUT, "am1gpu_batch_run has not completed");
    int rc = h->b.nmol > 0 ? fetch_results(h->b, h->mem, &h->stats) : AM1GPU_OK;
    if (rc) return rc;
    int first = AM1GPU_OK;
    std::string msg;
    for (int i = 0; i < h->nmol; ++i) {
        int r = h->status[i];
        if (r == AM1GPU_OK) r = write_result(h->b, &h->mem, h->planned[i], &results[i], &h->stats);
        if (status) status[i] = r;
        if (r && !first) {
            first = r;
            msg = g_err;
        }
    }
    tl_stats = h->stats;
    if (first) g_err = msg;
    return first;
}

void am1gpu_batch_destroy(am1gpu_batch* h) {
    if (!h) return;
    if (h->b.graph_exec) {
        cudaStreamSynchronize(h->mem.stream);
        cudaGraphExecDestroy(h->b.graph_exec);
    }
    am1::mem_release(h->mem);
    delete h;
}

void am1gpu_set_timing(int32_t enable) { am1::g_timing.store(enable ? 1 : 0); }

int am1gpu_set_stream_priority(int32_t priority) {
    using namespace am1;
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));  // lo: least (0), hi: greatest (negative)
    const int p = std::max(hi, std::min(lo, (int)priority));
    tl_priority = p;
    Mem& w = tl_mem;
    if (w.stream && w.priority != p) {  // the thread's stream so far: replace it (nothing is in flight between calls)
        CK(cudaStreamSynchronize(w.stream));
        CK(cudaStreamDestroy(w.stream));
        w.stream = nullptr;
        CK(cudaStreamCreateWithPriority(&w.stream, cudaStreamNonBlocking, p));
        w.priority = p;
    }
    return AM1GPU_OK;
}

int am1gpu_last_call_stats(am1gpu_call_stats* out) {
    if (!out) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    *out = am1::tl_stats;
    return AM1GPU_OK;
}

int am1gpu_batch_stats(const am1gpu_batch* h, am1gpu_call_stats* out) {
    if (!h || !out) return am1::fail(AM1GPU_INVALID_INPUT, "null argument");
    *out = h->stats;
    return AM1GPU_OK;
}

}  // extern "C"
