// step_launch.h -- host-side launchers of the step and ensemble kernels,
// whose instantiations live in a translation unit of their own (k_scalar.cu)
// that compiles in parallel with the rest.  Every launcher with launch =
// false only sets the kernel's shared-memory attribute (before a stream
// capture, for instance).
#pragma once
#include <cuda_runtime.h>

#include "tslb_step.cuh"

namespace tslb_launch {

// set the dynamic shared-memory limit of kernel fn once per device (tslb.cu)
cudaError_t ensure_smem_attr(const void* fn, size_t bytes);

// step kernel (tslb_step.cuh): every storage type, x alignment,
// tau correction and interior solid mask
cudaError_t scalar_step(const tslb::StepArgs& a, int mode, int prec, cudaStream_t st, bool launch);
cudaError_t scalar_ensemble(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                            int prec, bool vec, unsigned int* step, cudaStream_t st, bool launch);

}  // namespace tslb_launch
