// fdtd_fp32.cu — FP32 fused step kernels with compensated (increment-form)
// pressure accumulation.  Built with -fmad=false like every device unit: the
// FP32 kernels request their FMAs explicitly (fmaf), so no result depends on
// how the compiler contracts one instantiation or another.
#include <cuda_runtime.h>

#include "fdtd_device.cuh"
#include "fdtd_launch.hpp"
#include "fdtd_stencil.cuh"

namespace fdtd {

cudaError_t launch_prologue_fp32(const SolveParams* dP, int cur, int advance, int n_solid_pml, cudaStream_t s) {
    int blocks = 1;
    if (n_solid_pml > 0) blocks = (n_solid_pml + 255) / 256 > 2368 ? 2368 : (n_solid_pml + 255) / 256;
    k_prologue<float><<<blocks, 256, 0, s>>>(dP, cur, advance);
    return cudaGetLastError();
}

}  // namespace fdtd

#include "fdtd_hot.cuh"
namespace fdtd {
cudaError_t launch_step_regions_fp32(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                                     const StepStreams& S, int* launches) {
    return launch_regions<float>(dP, hP, R, cur, S, launches);
}
}  // namespace fdtd

#include "fdtd_batch.cuh"
namespace fdtd {
// The reduced-state shell kernels stage their loads in more than the default
// 48 KB of dynamic shared memory: raise their limit on the current device.
cudaError_t prepare_fp32_kernels() {
    // the TMA-staged shell: a ring of up to 24 KB stages
    cudaError_t e = cudaFuncSetAttribute(k_pml_shell_tma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TMA_STAGES * 24 * 1024 + 16 * TMA_STAGES);
    if (e != cudaSuccess) return e;
    if (shell_smem_bytes<float>() > 0) {
        e = cudaFuncSetAttribute(k_pml_shell<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 shell_smem_bytes<float>());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_batch_shell<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     shell_smem_bytes<float>());
        if (e != cudaSuccess) return e;
    }
    if (red_smem_bytes() > 0) {
        e = cudaFuncSetAttribute(k_pml_shell_red<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, red_smem_bytes());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_batch_shell_red<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     red_smem_bytes());
    }
    return e;
}

int tma_blocks_per_sm(int smem_bytes) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pml_shell_tma<float>, TMA_BLOCK, smem_bytes) != cudaSuccess)
        return 1;
    return n;
}

cudaError_t launch_batch_fp32(const BatchLaunch& L, const StepStreams& S, int* launches) {
    return launch_batch<float>(L, S, launches);
}
}  // namespace fdtd
