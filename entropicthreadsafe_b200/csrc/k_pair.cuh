// k_pair.cuh -- launch templates of the paired-column kernels, instantiated
// once per storage type by k_pair_f32.cu, k_pair_bf16.cu and k_pair_f16.cu.
#pragma once
#include "step_launch.h"
#include "tslb_pair.cuh"

namespace tslb_launch {

template <class T>
cudaError_t pair_step_t(const tslb::StepArgs& a, int mode, cudaStream_t st, bool launch) {
    using namespace tslb;
    const dim3 block(PH, PY, 1);
    const dim3 grid((a.nx + PX - 1) / PX, (a.ny + PY - 1) / PY, (a.zt1 - a.zt0 + a.zchunk - 1) / a.zchunk);
    const size_t sm = pair_smem_bytes(mode, (int)sizeof(T));
    cudaError_t err = cudaSuccess;
    auto go = [&](void (*kernel)(const StepArgs)) {
        err = ensure_smem_attr((const void*)kernel, sm);
        if (err == cudaSuccess && launch) kernel<<<grid, block, sm, st>>>(a);
    };
    if constexpr (std::is_same<T, float>::value) {
        // per-node tau correction: FP32 storage, colour mode (checked by the callers)
        if (mode == TSLB_MODE_COLOUR && a.dtau) {
            go(pair_kernel<TSLB_MODE_COLOUR, float, true>);
            return err;
        }
    }
    if (mode == TSLB_MODE_COLOUR) go(pair_kernel<TSLB_MODE_COLOUR, T>);
    else if (mode == TSLB_MODE_SINGLE) go(pair_kernel<TSLB_MODE_SINGLE, T>);
    else go(pair_kernel<TSLB_MODE_PHASEFIELD, T>);
    return err;
}

template <class T>
cudaError_t pair_ensemble_t(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                            cudaStream_t st, bool launch) {
    using namespace tslb;
    const size_t sm = pair_smem_bytes(mode, (int)sizeof(T));
    cudaError_t err = cudaSuccess;
    auto go = [&](void (*kernel)(const StepArgs*, const WorkItem*, int)) {
        err = ensure_smem_attr((const void*)kernel, sm);
        if (err == cudaSuccess && launch) kernel<<<grid, dim3(PH, PY, 1), sm, st>>>(args, work, nwork);
    };
    if (mode == TSLB_MODE_COLOUR) go(ensemble_pair_kernel<TSLB_MODE_COLOUR, T>);
    else go(ensemble_pair_kernel<TSLB_MODE_PHASEFIELD, T>);
    return err;
}

}  // namespace tslb_launch
