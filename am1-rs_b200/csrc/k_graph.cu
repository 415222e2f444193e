// Control kernels of the captured SCF solve (CUDA graph with device-side loops).
//
// The graph path runs a whole batched solve as one graph launch: the SCF iterations are the body
// of a conditional WHILE node, and inside it the purification steps are the body of a second one.
// These single-thread kernels decide, on the device, whether a loop goes round again, so the host
// reads nothing until the solve is done.  Each loop carries its own counter, and a loop ends when
// the counter reaches its cap whatever the other conditions say: the SCF loop after max_scf
// iterations, the purification loop after max_steps products, exactly as the host-driven loop of
// the eager path is bounded.
#include <cuda_runtime.h>

#include "kernels.h"

namespace am1 {

// Before the SCF loop: iteration counter and total-step counter to 0, the loop armed when any
// iteration is allowed at all.
__global__ void k_scf_arm(cudaGraphConditionalHandle h, GraphLoop* loop, int max_scf) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    loop->scf_iter = 0;
    loop->sp2_total = 0;
    loop->eig_runs = 0;
    cudaGraphSetConditional(h, max_scf > 0 ? 1u : 0u);
}

// Before each purification loop: its step counter and active count to 0, the loop armed.
__global__ void k_sp2_arm(cudaGraphConditionalHandle h, GraphLoop* loop, int* active_count) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    loop->sp2_step = 0;
    *active_count = 0;
    cudaGraphSetConditional(h, 1u);
}

// After each purification step (k_sp2_update has counted the channels still purifying): go round
// again while any is and fewer than max_steps steps were taken; the count restarts at 0.
__global__ void k_sp2_cond(cudaGraphConditionalHandle h, GraphLoop* loop, int* active_count, int max_steps) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int step = loop->sp2_step + 1;
    loop->sp2_step = step;
    loop->sp2_total += 1;
    const int more = *active_count > 0 && step < max_steps;
    *active_count = 0;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

// After the purified densities of an iteration: the stalled-purification eigensolver runs only if
// some molecule's purification stalled (need_eigen set by k_sp2_finish).  One CTA.
__global__ void k_stall_arm(cudaGraphConditionalHandle h, GraphLoop* loop, const int* need_eigen, int nmol) {
    int any = 0;
    for (int i = threadIdx.x; i < nmol; i += blockDim.x) any |= need_eigen[i] != 0;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        if (any) loop->eig_runs += 1;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// After each SCF iteration (k_converge has counted the molecules still iterating in active[0]):
// go round again while any is and fewer than max_scf iterations were done.
__global__ void k_scf_cond(cudaGraphConditionalHandle h, GraphLoop* loop, const int* active, int max_scf) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int it = loop->scf_iter + 1;
    loop->scf_iter = it;
    cudaGraphSetConditional(h, (active[0] > 0 && it < max_scf) ? 1u : 0u);
}

}  // namespace am1
