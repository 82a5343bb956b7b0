// k_pair_bf16.cu -- the paired-column step and ensemble kernels with __nv_bfloat16 storage.
#include "k_pair.cuh"

namespace tslb_launch {

cudaError_t pair_step_bf16(const tslb::StepArgs& a, int mode, cudaStream_t st, bool launch) {
    return pair_step_t<__nv_bfloat16>(a, mode, st, launch);
}

cudaError_t pair_ensemble_bf16(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                             cudaStream_t st, bool launch) {
    return pair_ensemble_t<__nv_bfloat16>(args, work, nwork, grid, mode, st, launch);
}

}  // namespace tslb_launch
