// tslb_internal.h -- the lattice context shared by the translation units of
// libtslb.so (tslb.cu: step and diagnostics; closure.cu: the learned
// eddy-viscosity closure).  Not part of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/tslb.h"
#include "tslb_device.cuh"

struct tslb_closure;

struct tslb_ctx {
    tslb_params p;
    int nx, ny, nz;
    long long n;        // nodes
    long long N;        // padded field stride
    int device;
    cudaStream_t stream = nullptr;
    void* state[2] = {nullptr, nullptr};   // ping-pong, 11 fields each, storage type
    int esize = 4;                         // bytes per stored element
    float* io = nullptr;                   // FP32 conversion buffer (bf16/fp16 storage)
    float* rho_out = nullptr;              // rho = 1 + d for downloads
    float scale[tslb::NF];                 // fp16 storage: stored = value * scale
    int cur = 0;
    float* nrm = nullptr;                  // 3 fields
    float* inlet[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    unsigned int* flags = nullptr;
    // FP64 diagnostics: red_blocks x RED_PARTS per-block partials, then the
    // RED_PARTS results and the last-block ticket; red_host is pinned
    double* red = nullptr;
    double* red_host = nullptr;
    double* red_ring = nullptr;            // tslb_reduce_async results (pinned, TSLB_REDUCE_QUEUE slots)
    int red_queued = 0;
    int red_blocks = 0;
    bool loaded = false;
    int zchunk = 32;
    // z slab of a larger lattice (tslb_create_slab): the local array holds
    // halo_lo + owned + halo_hi planes; a step updates planes [zt0, zt1)
    int zt0 = 0, zt1 = 0;                  // zt1 = 0: all planes
    int nz_global = 0, z_begin = 0, halo = 0, halo_lo = 0, halo_hi = 0;
    long long launches = 0;
    // per-node tau correction (colour mode, FP32 storage): dtau_base is the
    // static field of tslb_set_tau_correction (e.g. a sponge layer); with a
    // closure attached the closure writes dtau = dtau_base + its output and
    // the step reads dtau, otherwise the step reads dtau_base
    float* dtau = nullptr;
    float* dtau_base = nullptr;
    bool base_on = false;
    // interior solid nodes (tslb_set_solid_mask): bit masks of solid nodes and
    // of fluid nodes with a solid neighbour
    unsigned int* solid = nullptr;
    unsigned int* near = nullptr;
    bool solid_on = false;
    // moment-space boundary planes (tslb_set_moment_bc), per face
    int mbc_kind[6] = {0, 0, 0, 0, 0, 0};
    float mbc_uwall[6], mbc_radius[6], mbc_amp[6];
    tslb_closure* closure = nullptr;       // attached closure (not owned)
    int closure_interval = 1;
    long long steps_done = 0;
    // running sums of u, v, w, phi, w^2 (tslb_stats_*)
    float* stats = nullptr;
    long long stats_count = 0;
    std::string err;
};

namespace tslb_internal {
// record msg as the context's (or, for ctx == NULL, the creation) error; returns code
int fail(tslb_ctx* c, int code, const std::string& msg);
// FP32 view of the current state (converted through io for bf16/fp16 storage)
int fp32_view(tslb_ctx* c, const float** out);
// allocate the per-node tau correction buffer (zeroed) if absent
int ensure_dtau(tslb_ctx* c);
// closure.cu: refresh c->dtau from the attached closure before a step
int closure_before_step(tslb_ctx* c);
// set the shared-memory attribute of the step kernel the context launches
// next (its mode, storage, tau correction and solid mask)
int prepare_step_kernel(tslb_ctx* c);
}  // namespace tslb_internal
