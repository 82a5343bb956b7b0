// k_pair_f16.cu -- the paired-column step and ensemble kernels with __half storage.
#include "k_pair.cuh"

namespace tslb_launch {

cudaError_t pair_step_f16(const tslb::StepArgs& a, int mode, cudaStream_t st, bool launch) {
    return pair_step_t<__half>(a, mode, st, launch);
}

cudaError_t pair_ensemble_f16(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                             cudaStream_t st, bool launch) {
    return pair_ensemble_t<__half>(args, work, nwork, grid, mode, st, launch);
}

}  // namespace tslb_launch
