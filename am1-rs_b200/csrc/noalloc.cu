// am1gpu_symmetric_eigen_noalloc: the Jacobi eigensolver for callers that cannot allocate.
//
// Some callers must not allocate device memory at all: code that runs while another framework
// owns the device memory pool (a deep-learning runtime with a caching allocator it does not
// share, an MPI/NCCL application that has carved out all of HBM), real-time loops where an
// allocation would be an unbounded stall, and library code inside such hosts that is only
// handed device buffers.  They can pass the input and output buffers they already own, but
// not let this library call cudaMalloc.  For them the eigensolver's scratch (the warm-start
// copies, the slot-ordered vectors, the eigenvalue list, the job record) lives in one
// file-scope device array of fixed size, NOALLOC_SCRATCH_DOUBLES doubles (512 KiB), which
// bounds the matrix to NOALLOC_MAX_N = 128.  Every GPU that loads the library holds this array
// until the process exits.
//
// The host cannot use the array's name as a device address (in host code it names a host-side
// stand-in), so at set-up -- on the first call on each device, with that device current -- the
// address is fetched with cudaGetSymbolAddress and kept per device (a set-up that fails is not
// kept: the next call tries again).  That first call must come before any stream capture.  Every
// call waits for its stream to finish before it returns, because it reads the solver's status
// word back to the host.  All calls share the one array: two calls whose kernels overlap on the
// GPU (different streams, different host threads) race on it, so callers serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/am1gpu.h"
#include "am1gpu_internal.h"
#include "kernels.h"

namespace am1 {

constexpr int NOALLOC_MAX_N = 128;
constexpr int NOALLOC_MAX_NPAD = 160;  // n padded to a multiple of 2 x cluster size (<= n + 31)
constexpr size_t NOALLOC_SCRATCH_DOUBLES = 65536;

// Layout (doubles): Gt n*n | Ct n*n | Vs npad*n | lam npad | eps n | rowmin n | state | job | colid
struct NoallocLayout {
    size_t gt, ct, vs, lam, eps, rowmin, state, status, job, colid, end;
};

__host__ __device__ inline NoallocLayout noalloc_layout() {
    NoallocLayout L{};
    const size_t n = NOALLOC_MAX_N, np = NOALLOC_MAX_NPAD;
    L.gt = 0;
    L.ct = L.gt + n * n;
    L.vs = L.ct + n * n;
    L.lam = L.vs + np * n;
    L.eps = L.lam + np;
    L.rowmin = L.eps + n;
    L.state = L.rowmin + n;
    L.status = L.state + (sizeof(MolState) + 7) / 8;
    L.job = L.status + 1;
    L.colid = L.job + (sizeof(EigJob) + 7) / 8;
    L.end = L.colid + (np * sizeof(int) + 7) / 8;
    return L;
}

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Gt = A (its lower triangle, mirrored: symmetric_eigen reads Side::Lower), Ct = I, Gershgorin
// row bounds, a fresh job record and state; status 5 (LINALG) if A holds a non-finite element.
__global__ void k_noalloc_prepare(const double* __restrict__ a, int n, int npad) {
    double* s = g_noalloc_scratch;
    const NoallocLayout L = noalloc_layout();
    const int tid = threadIdx.x;
    __shared__ int bad;
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int i = tid; i < n * n; i += blockDim.x) {
        const int r = i / n, c = i % n;
        if (!isfinite(a[i])) bad = 1;
        s[L.gt + i] = r >= c ? a[i] : a[(size_t)c * n + r];
        s[L.ct + i] = r == c ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int r = tid; r < n; r += blockDim.x) {
        double bound = 0.0;
        for (int c = 0; c < n; ++c)
            if (c != r) bound += fabs(s[L.gt + (size_t)r * n + c]);
        s[L.rowmin + r] = s[L.gt + (size_t)r * n + r] - bound;
    }
    if (tid == 0) {
        MolState st{};
        st.active = 1;
        *reinterpret_cast<MolState*>(s + L.state) = st;
        *reinterpret_cast<int*>(s + L.status) = bad ? 5 : 0;
        EigJob jb{};
        jb.Gt = s + L.gt;
        jb.Ct = s + L.ct;
        jb.Vs = s + L.vs;
        jb.lam = s + L.lam;
        jb.colid_out = reinterpret_cast<int*>(s + L.colid);
        jb.eps = s + L.eps;
        jb.Ct_out = s + L.ct;
        jb.rowmin = s + L.rowmin;
        jb.sweeps_out = nullptr;
        jb.n = n;
        jb.npad = npad;
        jb.mol = 0;
        *reinterpret_cast<EigJob*>(s + L.job) = jb;
    }
}

// w = sorted eigenvalues, v[i][k] = component i of eigenvector k (columns are vectors).
__global__ void k_noalloc_finish(double* __restrict__ w, double* __restrict__ v, int n) {
    const double* s = g_noalloc_scratch;
    const NoallocLayout L = noalloc_layout();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
        const int r = i / n, k = i % n;
        v[i] = s[L.ct + (size_t)k * n + r];
        if (r == 0) w[k] = s[L.eps + k];
    }
}

namespace {

// Per-device set-up, kept only once it has succeeded: a failed attempt (a transient error, or
// a call made during someone else's stream capture) is retried by the next call.
struct NoallocDevice {
    std::mutex mu;
    bool done = false;
    double* scratch = nullptr;
    int smem_budget = 0;
};
NoallocDevice g_noalloc_dev[64];

cudaError_t noalloc_setup(NoallocDevice& d, int dev) {
    std::lock_guard<std::mutex> lock(d.mu);
    if (d.done) return cudaSuccess;
    // with that device current: the scratch array's device address and the eigensolver's launch
    // attributes (no allocation)
    double* scratch = nullptr;
    cudaError_t rc;
    if ((rc = cudaGetSymbolAddress((void**)&scratch, g_noalloc_scratch)) != cudaSuccess) return rc;
    int optin = 0;
    if ((rc = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return rc;
    cudaFuncAttributes fa{};
    if ((rc = cudaFuncGetAttributes(&fa, k_jacobi)) != cudaSuccess) return rc;
    const int budget = optin - (int)fa.sharedSizeBytes;
    if ((rc = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, budget)) != cudaSuccess) return rc;
    if ((rc = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess) return rc;
    if (!scratch) return cudaErrorInvalidSymbol;
    d.scratch = scratch;
    d.smem_budget = budget;
    d.done = true;
    return cudaSuccess;
}

// errors are reported through am1gpu_last_error, like every other entry point
int noalloc_fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

}  // namespace

}  // namespace am1

extern "C" int am1gpu_symmetric_eigen_noalloc(int32_t n, const double* a, double* w, double* v, void* stream) {
    using namespace am1;
    static_assert(NOALLOC_SCRATCH_DOUBLES * sizeof(double) >= 8, "scratch");
    if (noalloc_layout().end > NOALLOC_SCRATCH_DOUBLES) return noalloc_fail(AM1GPU_INVALID_INPUT, "scratch layout overflow");
    if (n < 1 || !a || !w || !v) return noalloc_fail(AM1GPU_INVALID_INPUT, "null argument or n < 1");
    if (n > NOALLOC_MAX_N)
        return noalloc_fail(AM1GPU_INVALID_INPUT, "n = " + std::to_string(n) + " exceeds the allocation-free eigensolver's maximum of " +
                                                      std::to_string(NOALLOC_MAX_N));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return noalloc_fail(AM1GPU_DEVICE_ERROR, "no CUDA device");
    NoallocDevice& d = g_noalloc_dev[dev];
    if ((e = noalloc_setup(d, dev)) != cudaSuccess)
        return noalloc_fail(AM1GPU_DEVICE_ERROR, std::string("set-up failed: ") + cudaGetErrorString(e));
    // cluster size and padding as the batched solver chooses them
    int npad = 0, C = 0;
    static const int cs[5] = {1, 2, 4, 8, 16};
    for (int k = 0; k < 5 && !C; ++k) {
        const int c = cs[k];
        const int np = ((n < 2 ? 2 : n) + 2 * c - 1) / (2 * c) * (2 * c);
        if (c > 1 && np / 2 / c < 2) continue;
        if ((long long)jacobi_smem_bytes(n, np, c) <= d.smem_budget) {
            npad = np;
            C = c;
        }
    }
    if (!C || npad > NOALLOC_MAX_NPAD) return noalloc_fail(AM1GPU_INVALID_INPUT, "no eigensolver configuration for this size");
    cudaStream_t s = (cudaStream_t)stream;
    const NoallocLayout L = noalloc_layout();
    double* base = d.scratch;
    k_noalloc_prepare<<<1, 256, 0, s>>>(a, n, npad);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = jacobi_smem_bytes(n, npad, C);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const EigJob* job = reinterpret_cast<const EigJob*>(base + L.job);
    const MolState* st = reinterpret_cast<const MolState*>(base + L.state);
    int* status = reinterpret_cast<int*>(base + L.status);
    e = cudaLaunchKernelEx(&cfg, k_jacobi, job, st, status, 1, (const int*)nullptr);
    if (e != cudaSuccess) return noalloc_fail(AM1GPU_DEVICE_ERROR, std::string("jacobi launch: ") + cudaGetErrorString(e));
    k_eig_sort<<<1, 512, 0, s>>>(job, st, 1, nullptr);
    k_noalloc_finish<<<(n * n + 255) / 256, 256, 0, s>>>(w, v, n);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_fail(AM1GPU_DEVICE_ERROR, cudaGetErrorString(e));
    int host_status = 0;
    if ((e = cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return noalloc_fail(AM1GPU_DEVICE_ERROR, cudaGetErrorString(e));
    if (host_status) return noalloc_fail(AM1GPU_LINALG, "the matrix handed to the eigensolver is not finite, or Jacobi did not converge");
    set_last_error("");
    return AM1GPU_OK;
}
