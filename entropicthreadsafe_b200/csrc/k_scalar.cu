// k_scalar.cu -- the scalar step kernel (tslb_step.cuh, one x column per
// thread) in every variant: storage type, rows that are whole 16-byte chunks
// or not, per-node tau correction, interior solid mask; and its ensemble form.
#include "step_launch.h"

namespace tslb_launch {

namespace {
template <class Fn>
void with_storage(int prec, Fn&& fn) {
    if (prec == TSLB_PREC_BF16) fn(__nv_bfloat16{});
    else if (prec == TSLB_PREC_FP16S) fn(__half{});
    else fn(float{});
}
}  // namespace

cudaError_t scalar_step(const tslb::StepArgs& a, int mode, int prec, cudaStream_t st, bool launch) {
    using namespace tslb;
    const dim3 block(TX, TY, 1);
    const dim3 grid((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY, (a.zt1 - a.zt0 + a.zchunk - 1) / a.zchunk);
    cudaError_t err = cudaSuccess;
    with_storage(prec, [&](auto tag) {
        using T = decltype(tag);
        const bool vec = a.nx % (16 / (int)sizeof(T)) == 0;
        const size_t sm = step_smem_bytes_es(mode, (int)sizeof(T));
        auto go = [&](void (*kernel)(const StepArgs)) {
            err = ensure_smem_attr((const void*)kernel, sm);
            if (err == cudaSuccess && launch) kernel<<<grid, block, sm, st>>>(a);
        };
        if (a.solid && std::is_same<T, float>::value) {
            // interior solid nodes (FP32 storage, no tau correction; checked by tslb_set_solid_mask)
            if (mode == TSLB_MODE_COLOUR) go(vec ? step_kernel<TSLB_MODE_COLOUR, true, float, false, true>
                                                 : step_kernel<TSLB_MODE_COLOUR, false, float, false, true>);
            else if (mode == TSLB_MODE_SINGLE) go(vec ? step_kernel<TSLB_MODE_SINGLE, true, float, false, true>
                                                      : step_kernel<TSLB_MODE_SINGLE, false, float, false, true>);
            else go(vec ? step_kernel<TSLB_MODE_PHASEFIELD, true, float, false, true>
                        : step_kernel<TSLB_MODE_PHASEFIELD, false, float, false, true>);
        } else if (mode == TSLB_MODE_COLOUR && a.dtau && std::is_same<T, float>::value) {
            // per-node tau correction (FP32 storage only; checked by the callers)
            go(vec ? step_kernel<TSLB_MODE_COLOUR, true, float, true> : step_kernel<TSLB_MODE_COLOUR, false, float, true>);
        } else if (mode == TSLB_MODE_COLOUR) {
            go(vec ? step_kernel<TSLB_MODE_COLOUR, true, T> : step_kernel<TSLB_MODE_COLOUR, false, T>);
        } else if (mode == TSLB_MODE_SINGLE) {
            go(vec ? step_kernel<TSLB_MODE_SINGLE, true, T> : step_kernel<TSLB_MODE_SINGLE, false, T>);
        } else {
            go(vec ? step_kernel<TSLB_MODE_PHASEFIELD, true, T> : step_kernel<TSLB_MODE_PHASEFIELD, false, T>);
        }
    });
    return err;
}

cudaError_t scalar_ensemble(const tslb::StepArgs* args, const tslb::WorkItem* work, int nwork, int grid, int mode,
                            int prec, bool vec, unsigned int* step, cudaStream_t st, bool launch) {
    using namespace tslb;
    cudaError_t err = cudaSuccess;
    with_storage(prec, [&](auto tag) {
        using T = decltype(tag);
        const size_t sm = step_smem_bytes_es(mode, (int)sizeof(T));
        auto go = [&](void (*kernel)(const StepArgs*, const WorkItem*, int, unsigned int*)) {
            err = ensure_smem_attr((const void*)kernel, sm);
            if (err == cudaSuccess && launch) kernel<<<grid, dim3(TX, TY, 1), sm, st>>>(args, work, nwork, step);
        };
        if (mode == TSLB_MODE_COLOUR) go(vec ? ensemble_kernel<TSLB_MODE_COLOUR, true, T> : ensemble_kernel<TSLB_MODE_COLOUR, false, T>);
        else go(vec ? ensemble_kernel<TSLB_MODE_PHASEFIELD, true, T> : ensemble_kernel<TSLB_MODE_PHASEFIELD, false, T>);
    });
    return err;
}

}  // namespace tslb_launch
