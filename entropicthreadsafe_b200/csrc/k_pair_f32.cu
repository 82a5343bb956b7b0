// k_pair_f32.cu -- the paired-column step and ensemble kernels with float storage.
#include "k_pair.cuh"

namespace tslb_launch {

cudaError_t pair_step_f32(const tslb::StepArgs& a, int mode, cudaStream_t st, bool launch) {
    return pair_step_t<float>(a, mode, st, launch);
}

cudaError_t pair_ensemble_f32(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                             cudaStream_t st, bool launch) {
    return pair_ensemble_t<float>(args, work, nwork, grid, mode, st, launch);
}

}  // namespace tslb_launch
