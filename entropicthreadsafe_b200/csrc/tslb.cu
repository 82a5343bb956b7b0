// tslb.cu -- C-ABI (include/tslb.h) of the B200 TSLB step: context,
// device state, uploads/downloads, the step launch and FP64 diagnostics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/tslb.h"
#include "../../include/tslb_io.h"
#include "step_launch.h"
#include "tslb_internal.h"
#include "tslb_step.cuh"

using namespace tslb;

// message of this thread's last failed creation (tslb_create, tslb_ensemble_create,
// tslb_step_noalloc): per thread, so concurrent failures do not race
static thread_local std::string g_create_error;

namespace tslb_internal {

int fail(tslb_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

}  // namespace tslb_internal

namespace {

using tslb_internal::fail;

#define CUDA_TRY(ctx, call)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(ctx, TSLB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

long long face_area(const tslb_ctx* c, int face) {
    int ax = face / 2;
    return ax == 0 ? (long long)c->ny * c->nz : ax == 1 ? (long long)c->nx * c->nz : (long long)c->nx * c->ny;
}

int validate(const tslb_params* p, int nx, int ny, int nz, std::string& why) {
    if (!p) { why = "params is NULL"; return TSLB_ERR_ARG; }
    if (nx < 1 || ny < 1 || nz < 1) { why = "sizes must be >= 1"; return TSLB_ERR_ARG; }
    if ((long long)nx * ny * nz > (1LL << 36)) { why = "lattice too large"; return TSLB_ERR_ARG; }
    if (p->mode != TSLB_MODE_PHASEFIELD && p->mode != TSLB_MODE_COLOUR && p->mode != TSLB_MODE_SINGLE) {
        why = "unknown mode"; return TSLB_ERR_ARG;
    }
    if (p->precision != TSLB_PREC_FP32 && p->precision != TSLB_PREC_BF16 && p->precision != TSLB_PREC_FP16S) {
        why = "unknown precision"; return TSLB_ERR_ARG;
    }
    if (!(p->tau_a > 0.5f) || !std::isfinite(p->tau_a)) { why = "tau_a must be > 0.5"; return TSLB_ERR_ARG; }
    if (p->mode == TSLB_MODE_COLOUR && (!(p->tau_b > 0.5f) || !std::isfinite(p->tau_b))) { why = "tau_b must be > 0.5"; return TSLB_ERR_ARG; }
    if (!std::isfinite(p->sigma) || !std::isfinite(p->beta) || !std::isfinite(p->sharp_c) || !std::isfinite(p->grad_threshold)) {
        why = "non-finite parameter"; return TSLB_ERR_ARG;
    }
    for (int a = 0; a < 3; ++a)
        if (!std::isfinite(p->force[a])) { why = "non-finite force"; return TSLB_ERR_ARG; }
    for (int f = 0; f < 6; ++f) {
        if (p->bc[f] < TSLB_BC_PERIODIC || p->bc[f] > TSLB_BC_PRESSURE) { why = "unknown boundary kind"; return TSLB_ERR_ARG; }
        for (int a = 0; a < 3; ++a)
            if (!std::isfinite(p->bc_u[f][a])) { why = "non-finite wall velocity"; return TSLB_ERR_ARG; }
    }
    for (int ax = 0; ax < 3; ++ax) {
        bool pm = p->bc[2 * ax] == TSLB_BC_PERIODIC, pp = p->bc[2 * ax + 1] == TSLB_BC_PERIODIC;
        if (pm != pp) { why = "periodic faces must come in pairs"; return TSLB_ERR_ARG; }
    }
    if (p->wall_phi_mode != 0 && p->wall_phi_mode != 1) { why = "wall_phi_mode must be 0 or 1"; return TSLB_ERR_ARG; }
    return TSLB_OK;
}

StepArgs make_args(tslb_ctx* c, const void* in, void* out) {
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.nx = c->nx; a.ny = c->ny; a.nz = c->nz; a.N = c->N;
    a.in = in; a.out = out; a.nrm = c->nrm;
    a.zchunk = c->zchunk;
    a.zt0 = c->zt0;
    a.zt1 = c->zt1 > 0 ? c->zt1 : c->nz;
    a.zoff = c->z_begin - c->zt0;
    a.mode = c->p.mode;
    a.omega_pf = 1.0f / c->p.tau_a;
    a.inv_nu_a = 3.0f / (c->p.tau_a - 0.5f);
    a.inv_nu_b = 3.0f / ((c->p.mode == TSLB_MODE_COLOUR ? c->p.tau_b : c->p.tau_a) - 0.5f);
    a.sigma = c->p.sigma; a.beta = c->p.beta; a.sharp = c->p.sharp_c; a.thr = c->p.grad_threshold;
    a.acoef = 4.5f;  // A = 9/2 sigma omega gives the Laplace jump 2 sigma / R for phi in [-1, 1]
    for (int k = 0; k < 3; ++k) a.force[k] = c->p.force[k];
    a.wall_phi_mode = c->p.wall_phi_mode;
    for (int f = 0; f < 6; ++f) {
        a.face[f].kind = c->p.bc[f];
        for (int k = 0; k < 3; ++k) a.face[f].u[k] = c->p.bc_u[f][k];
        a.face[f].phi = c->p.bc_phi[f];
        a.face[f].plane = c->inlet[f];
    }
    a.flags = c->flags;
    a.dtau = c->closure ? c->dtau : (c->base_on ? c->dtau_base : nullptr);
    a.solid = c->solid_on ? c->solid : nullptr;
    a.near = c->solid_on ? c->near : nullptr;
    a.sr = 1;
    a.sr_step = (unsigned int)c->steps_done;
    a.sr_counter = nullptr;
    for (int f = 0; f < NF; ++f) {
        a.scale[f] = c->scale[f];
        a.iscale[f] = 1.0f / c->scale[f];
    }
    return a;
}

// ---------------------------------------------------------------- kernels
template <class T>
__global__ void normals_kernel(const StepArgs a, float* nrm) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = (long long)a.nx * a.ny * a.nz;
    if (i >= n) return;
    const int x = (int)(i % a.nx), y = (int)((i / a.nx) % a.ny), z = (int)(i / ((long long)a.nx * a.ny));
    float g[3];
    grad_phi<T>(a, x, y, z, g);
    if (a.solid && bit_at(a.solid, i)) g[0] = g[1] = g[2] = 0.f;   // normals of solid nodes are 0
    const float den = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) + 1e-9f;
    nrm[i] = g[0] / den;
    nrm[a.N + i] = g[1] / den;
    nrm[2 * a.N + i] = g[2] / den;
}

// rho (host layout) -> rho - 1 in place
__global__ void shift_rho_kernel(float* d, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) d[i] = d[i] - 1.0f;
}

// rho = 1 + d into a separate field (the state keeps d)
__global__ void rho_from_d_kernel(const float* __restrict__ d, float* __restrict__ rho, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) rho[i] = 1.0f + d[i];
}

// FP32 fields (rho already shifted to rho - 1) -> storage type
template <class T>
__global__ void to_storage_kernel(const float* __restrict__ src, T* __restrict__ dst, long long N, long long n, StepArgs a) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int f = 0; f < NF; ++f) dst[f * N + i] = cvt_out<T>(src[f * N + i], a, f);
}
// storage type -> FP32 fields (rho stays rho - 1)
template <class T>
__global__ void from_storage_kernel(const T* __restrict__ src, float* __restrict__ dst, long long N, long long n, StepArgs a) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int f = 0; f < NF; ++f) dst[f * N + i] = cvt_in<T>(src[f * N + i], a, f);
}

// Moments pass of the reference on populations in its halo layout
// (recursive_2c_TSLB3D.f90:351-539; colour: both sets, recursive_colorTSLB3D.f90:482-671).
__constant__ int c_cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ int c_cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1};
__constant__ int c_cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ int c_piorder[26] = {1, 2, 3, 4, 5, 6, 7, 8, 10, 9, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26};

__device__ float feq_over_w_dev(int q, float rho, float u, float v, float w) {
    const float cx = (float)c_cx[q], cy = (float)c_cy[q], cz = (float)c_cz[q];
    const float t = 1.f / 3.f;
    const float cu = cx * u + cy * v + cz * w, uu = u * u + v * v + w * w;
    const float h3 = 13.5f * ((cx * cx - t) * cy * u * u * v + (cx * cx - t) * cz * u * u * w +
                              (cy * cy - t) * cx * u * v * v + (cy * cy - t) * cz * v * v * w +
                              (cz * cz - t) * cx * u * w * w + (cz * cz - t) * cy * v * w * w) +
                     27.f * cx * cy * cz * u * v * w;
    return rho * (1.f + 3.f * cu + 4.5f * cu * cu - 1.5f * uu + h3);
}

__global__ void pops_to_moments_kernel(int nx, int ny, int nz, long long N, int colour,
                                       const float* __restrict__ f, const float* __restrict__ g, float* out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = (long long)nx * ny * nz;
    if (i >= n) return;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const long long sx = nx + 2, sy = ny + 2, vol = sx * sy * (nz + 2);
    const long long h = (x + 1) + sx * ((y + 1) + sy * (long long)(z + 1));
    float tot[27];
    float ra = 0.f, rb = 0.f, phi = 0.f;
    for (int q = 0; q < 27; ++q) { tot[q] = f[q * vol + h]; ra += tot[q]; }
    if (colour) {
        for (int q = 0; q < 27; ++q) { float gb = g[q * vol + h]; rb += gb; tot[q] += gb; }
    } else if (g) {
        for (int q = 0; q < 7; ++q) phi += g[q * vol + h];
    } else {
        phi = 1.f;   // single component
    }
    const float rho = colour ? ra + rb : ra;
    if (colour) phi = (ra - rb) / rho;
    float sp[3] = {0.f, 0.f, 0.f}, sm[3] = {0.f, 0.f, 0.f};
    for (int q = 1; q < 27; ++q) {
        const int c[3] = {c_cx[q], c_cy[q], c_cz[q]};
        for (int a = 0; a < 3; ++a) {
            if (c[a] > 0) sp[a] += tot[q];
            if (c[a] < 0) sm[a] += tot[q];
        }
    }
    const float u = (sp[0] - sm[0]) / rho, v = (sp[1] - sm[1]) / rho, w = (sp[2] - sm[2]) / rho;
    float P[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < 26; ++k) {
        const int q = c_piorder[k];
        const float wq = wclass(c_cx[q] * c_cx[q] + c_cy[q] * c_cy[q] + c_cz[q] * c_cz[q]);
        const float fneq = tot[q] - wq * feq_over_w_dev(q, rho, u, v, w);
        const int cx = c_cx[q], cy = c_cy[q], cz = c_cz[q];
        if (cx) P[0] += fneq;
        if (cx * cy > 0) P[1] += fneq; else if (cx * cy < 0) P[1] -= fneq;
        if (cx * cz > 0) P[2] += fneq; else if (cx * cz < 0) P[2] -= fneq;
        if (cy) P[3] += fneq;
        if (cy * cz > 0) P[4] += fneq; else if (cy * cz < 0) P[4] -= fneq;
        if (cz) P[5] += fneq;
    }
    out[F_D * N + i] = rho - 1.0f;
    out[F_U * N + i] = u; out[F_V * N + i] = v; out[F_W * N + i] = w;
    out[F_XX * N + i] = P[0]; out[F_XY * N + i] = P[1]; out[F_XZ * N + i] = P[2];
    out[F_YY * N + i] = P[3]; out[F_YZ * N + i] = P[4]; out[F_ZZ * N + i] = P[5];
    out[F_PHI * N + i] = phi;
}

// FP64 diagnostics: sums in TSLB_RED_* order (8..9 hold sums of rho and
// counts inside/outside; finalised on the host) and, in part RED_SLOTS, the
// maximum of |u|^2.  Every block writes its partials; the last block to
// finish (ticket) adds them up in block order, so the result depends only on
// the state and the grid, never on the order in which blocks finish.
constexpr int RED_SLOTS = 12, RED_PARTS = RED_SLOTS + 1, RED_THREADS = 256;
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(const float* __restrict__ s, long long n, long long N,
                                                             int colour, double* part, double* out,
                                                             unsigned int* ticket) {
    __shared__ double sh[RED_PARTS][RED_THREADS / 32];
    __shared__ bool last;
    double acc[RED_SLOTS];
    for (int k = 0; k < RED_SLOTS; ++k) acc[k] = 0.0;
    float umax2 = 0.f;
    const float lo = colour ? -0.9f : 0.1f;
    auto node = [&](double d, double u, double v, double w, double phi) {
        const double rho = 1.0 + d;
        acc[0] += d;  // mass - n, exact for small deviations
        if (colour) { acc[1] += rho * (1.0 + phi) * 0.5; acc[2] += rho * (1.0 - phi) * 0.5; }
        else { acc[1] += phi; acc[2] += 1.0 - phi; }
        acc[3] += rho * u; acc[4] += rho * v; acc[5] += rho * w;
        const double uu = u * u + v * v + w * w;
        acc[6] += 0.5 * rho * uu;
        umax2 = fmaxf(umax2, (float)uu);
        if (phi > 0.9) { acc[7] += rho; acc[8] += 1.0; }
        if (phi < lo) { acc[9] += rho; acc[10] += 1.0; }
    };
    // four nodes' loads in flight per thread, then their FP64 accumulation
    constexpr int U4 = 4;
    const long long S = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + (U4 - 1) * S < n; i += U4 * S) {
        float x[U4][5];
#pragma unroll
        for (int q = 0; q < U4; ++q) {
            const long long j = i + q * S;
            x[q][0] = __ldcs(s + F_D * N + j);
            x[q][1] = __ldcs(s + F_U * N + j);
            x[q][2] = __ldcs(s + F_V * N + j);
            x[q][3] = __ldcs(s + F_W * N + j);
            x[q][4] = __ldcs(s + F_PHI * N + j);
        }
#pragma unroll
        for (int q = 0; q < U4; ++q) node(x[q][0], x[q][1], x[q][2], x[q][3], x[q][4]);
    }
    for (; i < n; i += S) node(s[F_D * N + i], s[F_U * N + i], s[F_V * N + i], s[F_W * N + i], s[F_PHI * N + i]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // block partials: a fixed shuffle tree per warp, then the warps in order
    for (int k = 0; k < RED_PARTS; ++k) {
        double vv = k < RED_SLOTS ? acc[k] : (double)umax2;
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_down_sync(0xffffffffu, vv, o);
            vv = k < RED_SLOTS ? vv + t : fmax(vv, t);
        }
        if (lane == 0) sh[k][warp] = vv;
    }
    __syncthreads();
    if (threadIdx.x < RED_PARTS) {
        const int k = threadIdx.x;
        double t = sh[k][0];
        for (int w8 = 1; w8 < RED_THREADS / 32; ++w8) t = k < RED_SLOTS ? t + sh[k][w8] : fmax(t, sh[k][w8]);
        part[(long long)blockIdx.x * RED_PARTS + k] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block: thread t takes blocks t, t + 256, ... in order, then the same trees
    for (int k = 0; k < RED_PARTS; ++k) {
        double vv = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += RED_THREADS) {
            const double p = __ldcg(part + (long long)b * RED_PARTS + k);
            vv = k < RED_SLOTS ? vv + p : fmax(vv, p);
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_down_sync(0xffffffffu, vv, o);
            vv = k < RED_SLOTS ? vv + t : fmax(vv, t);
        }
        if (lane == 0) sh[k][warp] = vv;
    }
    __syncthreads();
    if (threadIdx.x < RED_PARTS) {
        const int k = threadIdx.x;
        double t = sh[k][0];
        for (int w8 = 1; w8 < RED_THREADS / 32; ++w8) t = k < RED_SLOTS ? t + sh[k][w8] : fmax(t, sh[k][w8]);
        out[k] = t;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014)
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Jet inlet plane: inside the disc normal velocity speed (1 + amp xi) and
// phi = +1, outside zero velocity and phi = -1; xi in [-1, 1) from a hash of
// (seed, counter, plane index).  n0 is the first in-plane extent; `axis` and
// `sign` give the normal component and its direction into the lattice.
__global__ void inlet_disc_kernel(float* plane, int n0, int n1, int axis, float sign, float c0, float c1, float r2,
                                  float speed, float amp, unsigned long long seed, unsigned long long counter) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long pa = (long long)n0 * n1;
    if (i >= pa) return;
    const float d0 = (float)(i % n0) - c0, d1 = (float)(i / n0) - c1;
    const bool in = __fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)) <= r2;
    const unsigned long long h = mix64(mix64(seed * 0x9E3779B97F4A7C15ull + counter) ^ (unsigned long long)i);
    const float xi = __fsub_rn(__fmul_rn((float)(h >> 40), 1.0f / 8388608.0f), 1.0f);
    const float wn = in ? __fmul_rn(sign * speed, __fadd_rn(1.0f, __fmul_rn(amp, xi))) : 0.0f;
    for (int k = 0; k < 3; ++k) plane[k * pa + i] = k == axis ? wn : 0.0f;
    plane[3 * pa + i] = in ? 1.0f : -1.0f;
}

// moment-space boundary plane of face (4: z = 0, 5: z = nz - 1), see tslb_set_moment_bc
template <class T>
__global__ void moment_bc_kernel(StepArgs a, T* st, int face, int kind, float uwall, float r2, float amp, int step) {
    const long long plane = (long long)a.nx * a.ny;
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= plane) return;
    const int k0 = face == 4 ? 0 : a.nz - 1, k1 = face == 4 ? 1 : a.nz - 2;
    const long long i0 = (long long)k0 * plane + p, i1 = (long long)k1 * plane + p;
    if (kind == TSLB_MBC_COPY) {
        for (int f = 0; f < NF; ++f) st[f * a.N + i0] = st[f * a.N + i1];
        return;
    }
    // TSLB_MBC_JET: rho - 1 and Pi from the next plane, tangential velocity 0
    st[F_D * a.N + i0] = st[F_D * a.N + i1];
    for (int f = F_XX; f <= F_ZZ; ++f) st[f * a.N + i0] = st[f * a.N + i1];
    st[F_U * a.N + i0] = cvt_out<T>(0.f, a, F_U);
    st[F_V * a.N + i0] = cvt_out<T>(0.f, a, F_V);
    if (step % 10 == 0) {
        const int i = (int)(p % a.nx) + 1, j = (int)(p / a.nx) + 1;   // 1-based
        const float dx = (float)i - a.nx / 2.0f, dy = (float)j - a.ny / 2.0f;
        if (dx * dx + dy * dy <= r2) {
            const float r = fmaxf(rand_noseeded(i, j, 1, step), 2.98023224e-8f);
            const float w = uwall + amp * sqrtf(-2.0f * logf(r)) * cosf(6.283185307179586f * r);
            st[F_W * a.N + i0] = cvt_out<T>(w, a, F_W);
        }
    }
}

// solid bit mask from isfluid bytes: word w holds nodes 32w .. 32w+31
__global__ void solid_bits_kernel(const unsigned char* __restrict__ isfluid, long long n, unsigned int* solid) {
    const long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (w * 32 >= n) return;
    unsigned int b = 0;
    for (int k = 0; k < 32; ++k) {
        const long long i = w * 32 + k;
        if (i < n && isfluid[i] == 0) b |= 1u << k;
    }
    solid[w] = b;
}

// fluid nodes with a solid node among their 26 neighbours (periodic axes wrap;
// a neighbour behind a non-periodic face is not an interior solid)
__global__ void near_bits_kernel(const unsigned char* __restrict__ isfluid, int nx, int ny, int nz, int px, int py,
                                 int pz, unsigned int* near) {
    const long long n = (long long)nx * ny * nz;
    const long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (w * 32 >= n) return;
    unsigned int b = 0;
    for (int k = 0; k < 32; ++k) {
        const long long i = w * 32 + k;
        if (i >= n || isfluid[i] == 0) continue;
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
        bool hit = false;
        for (int dz = -1; dz <= 1 && !hit; ++dz)
            for (int dy = -1; dy <= 1 && !hit; ++dy)
                for (int dx = -1; dx <= 1 && !hit; ++dx) {
                    int sx = x + dx, sy = y + dy, sz = z + dz;
                    if (sx < 0 || sx >= nx) { if (!px) continue; sx = (sx + nx) % nx; }
                    if (sy < 0 || sy >= ny) { if (!py) continue; sy = (sy + ny) % ny; }
                    if (sz < 0 || sz >= nz) { if (!pz) continue; sz = (sz + nz) % nz; }
                    hit = isfluid[sx + (long long)nx * (sy + (long long)ny * sz)] == 0;
                }
        if (hit) b |= 1u << k;
    }
    near[w] = b;
}

// running sums (time averages of the jet statistics): slots u, v, w, phi,
// ww, then uu, uv, uw, vv, vw and the six Pi^neq components
constexpr int NSTATS = 16;
__global__ void stats_accumulate_kernel(const float* __restrict__ s, long long n, long long N, float* __restrict__ acc) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float u = s[F_U * N + i], v = s[F_V * N + i], w = s[F_W * N + i];
    acc[i] += u;
    acc[N + i] += v;
    acc[2 * N + i] += w;
    acc[3 * N + i] += s[F_PHI * N + i];
    acc[4 * N + i] += w * w;
    acc[5 * N + i] += u * u;
    acc[6 * N + i] += u * v;
    acc[7 * N + i] += u * w;
    acc[8 * N + i] += v * v;
    acc[9 * N + i] += v * w;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[(10 + k) * N + i] += s[(F_XX + k) * N + i];
}

// means over cf^3 blocks of the running sums k0 .. k0 + nk - 1: out[(k - k0) * nc + j]
__global__ void stats_coarsen_kernel(const float* __restrict__ acc, int nx, int ny, int nz, long long N, int cf, int k0,
                                     int nk, float inv, float* __restrict__ out) {
    const int cx = nx / cf, cy = ny / cf, cz = nz / cf;
    const long long nc = (long long)cx * cy * cz;
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= nc) return;
    const int X = (int)(j % cx), Y = (int)((j / cx) % cy), Z = (int)(j / ((long long)cx * cy));
    for (int k = k0; k < k0 + nk; ++k) {
        float sum = 0.f;
        for (int dz = 0; dz < cf; ++dz)
            for (int dy = 0; dy < cf; ++dy)
                for (int dx = 0; dx < cf; ++dx)
                    sum += acc[k * N + (long long)(cf * X + dx) + (long long)nx * ((cf * Y + dy) + (long long)ny * (cf * Z + dz))];
        out[(k - k0) * nc + j] = sum * inv;
    }
}

int check_flags(tslb_ctx* c) {
    unsigned int h = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&h, c->flags, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (h) CUDA_TRY(c, cudaMemsetAsync(c->flags, 0, sizeof(unsigned int), c->stream));
    if (h & 2u) return fail(c, TSLB_ERR_TIMEOUT, "a bounded wait of the closure kernel ran out");
    if (h & 1u) return fail(c, TSLB_ERR_NAN, "the step produced a non-finite moment");
    return TSLB_OK;
}

int storage_bytes(int prec) { return prec == TSLB_PREC_FP32 ? 4 : 2; }

// Call fn with a value of the storage type of precision `prec`.
template <class Fn>
void with_storage(int prec, Fn&& fn) {
    if (prec == TSLB_PREC_BF16) fn(__nv_bfloat16{});
    else if (prec == TSLB_PREC_FP16S) fn(__half{});
    else fn(float{});
}


}  // namespace

// The step kernels use more than 48 KB of dynamic shared memory, which needs
// a function attribute once per kernel and device.  Modules load lazily, so
// the attribute is set only for the instantiations a lattice launches: at
// its first launch, or earlier through prepare_step_kernel (before a stream
// capture, for instance).
namespace tslb_launch {
namespace {
std::mutex g_attr_mu;
std::vector<std::pair<int, const void*>> g_attr_done;
}  // namespace

cudaError_t ensure_smem_attr(const void* fn, size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto& d : g_attr_done)
        if (d.first == dev && d.second == fn) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) g_attr_done.emplace_back(dev, fn);
    return e;
}
}  // namespace tslb_launch

namespace {

// The lattices' large buffers (state, conversion and output fields, normals)
// come from one memory pool per device that keeps freed memory for the next
// lattice: a lattice created after another was destroyed reuses its pages
// instead of mapping new ones.  Allocation and release are ordered on the
// lattice's stream.  The pool keeps at most 1/8 of the device's memory
// cached (the excess goes back at synchronisation points); a failed
// allocation first returns all cached memory and is tried once more, and
// tslb_release_memory returns it on request.
std::mutex g_pool_mu;
constexpr int MAX_DEVICES = 64;
cudaMemPool_t g_pool[MAX_DEVICES] = {};

cudaError_t pool_alloc(void** ptr, size_t bytes, int dev, cudaStream_t st) {
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
        if (!g_pool[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaError_t e = cudaMemPoolCreate(&pool, &props);
            if (e != cudaSuccess) return e;
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            unsigned long long keep = (unsigned long long)total_b / 8;
            e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) {
                cudaMemPoolDestroy(pool);
                return e;
            }
            g_pool[dev] = pool;
        }
        pool = g_pool[dev];
    }
    cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, st);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocFromPoolAsync(ptr, bytes, pool, st);
    }
    return e;
}

void pool_free(void* ptr, cudaStream_t st) {
    if (ptr) cudaFreeAsync(ptr, st);
}

// Page-locked host blocks of the contexts (diagnostics results and ring):
// cudaHostAlloc and cudaFreeHost take milliseconds, so freed blocks are
// kept (up to kPinnedKeep bytes, process-wide) and handed out again to
// requests of the same size.
std::mutex g_pin_mu;
std::vector<std::pair<size_t, void*>> g_pin_free;
size_t g_pin_kept = 0;
constexpr size_t kPinnedKeep = 64u << 20;

cudaError_t pinned_get(void** p, size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        for (size_t i = 0; i < g_pin_free.size(); ++i)
            if (g_pin_free[i].first == bytes) {
                *p = g_pin_free[i].second;
                g_pin_free.erase(g_pin_free.begin() + (long)i);
                g_pin_kept -= bytes;
                return cudaSuccess;
            }
    }
    return cudaHostAlloc(p, bytes, cudaHostAllocPortable);
}

void pinned_put(void* p, size_t bytes) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        if (g_pin_kept + bytes <= kPinnedKeep) {
            g_pin_free.emplace_back(bytes, p);
            g_pin_kept += bytes;
            return;
        }
    }
    cudaFreeHost(p);
}
constexpr size_t kRingBytes = sizeof(double) * RED_PARTS * TSLB_REDUCE_QUEUE;
constexpr size_t kRedHostBytes = sizeof(double) * RED_PARTS;

int ensure_normals(tslb_ctx* c) {
    if (c->nrm) return TSLB_OK;
    CUDA_TRY(c, pool_alloc(reinterpret_cast<void**>(&c->nrm), sizeof(float) * 3 * c->N, c->device, c->stream));
    return TSLB_OK;
}

// tile columns of the step grid
long long step_tiles(int nx, int ny) { return (long long)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY); }
constexpr int kStepBlocksPerSM = 2;   // resident step blocks per SM (registers and shared memory)

// Target planes per block.  Each chunk also reads the source planes just
// outside it, so long chunks repeat less work; the chunks per tile column
// are the fewest whose blocks fill the resident slots (bps blocks per SM) in
// whole waves to at least 90%, with chunks of at least 8 planes.
int choose_zchunk(long long tiles, int nz, int sms, int bps, int mode) {
    const long long slots = (long long)bps * sms;
    const int max_chunks = std::max(1, nz / 8);
    int best = 1;
    double best_fill = -1.0;
    for (int nc = 1; nc <= max_chunks; ++nc) {
        const int zc = (nz + nc - 1) / nc;
        const long long blocks = tiles * ((nz + zc - 1) / zc);
        const long long waves = (blocks + slots - 1) / slots;
        const double fill = (double)blocks / (double)(waves * slots);
        if (fill > best_fill + 1e-9) {
            best_fill = fill;
            best = nc;
        }
        if (fill >= 0.9) break;
    }
    const int zc = (nz + best - 1) / best;
    // Phase field: the curvature makes planes with interface nodes slower, so
    // tile columns crossing droplets take longer; chunks of 16 planes give
    // several waves of blocks that the scheduler balances (0.591 -> 0.567 ms on
    // the 384 x 192 x 128 channel).  The uniform colour step is fastest with
    // the fewest chunks.
    if (mode == TSLB_MODE_PHASEFIELD) return std::min(zc, std::max(16, (nz + 7) / 8));
    return zc;
}

int launch_normals(tslb_ctx* c) {
    int rc = ensure_normals(c);
    if (rc) return rc;
    StepArgs a = make_args(c, c->state[c->cur], nullptr);
    const int bs = 256;
    const long long grid = (c->n + bs - 1) / bs;
    with_storage(c->p.precision, [&](auto tag) {
        normals_kernel<decltype(tag)><<<(unsigned)grid, bs, 0, c->stream>>>(a, c->nrm);
    });
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

// The step kernel on one lattice (shared by the context and the no-alloc
// paths): the instantiation for the mode, storage, x alignment, tau
// correction and solid mask of `a`.  launch = false only sets its shared
// memory attribute.  Returns the error of that attribute; launch errors are
// left to cudaGetLastError.
cudaError_t launch_step_kernel(const StepArgs& a, int mode, int prec, cudaStream_t st, bool launch = true) {
    return tslb_launch::scalar_step(a, mode, prec, st, launch);
}

int launch_moment_bcs(tslb_ctx* c) {
    for (int face = 4; face < 6; ++face) {
        if (c->mbc_kind[face] == TSLB_MBC_NONE) continue;
        StepArgs a = make_args(c, nullptr, nullptr);
        const long long plane = (long long)c->nx * c->ny;
        const int step = (int)((c->steps_done + 1) % 2000000000LL);
        with_storage(c->p.precision, [&](auto tag) {
            using T = decltype(tag);
            moment_bc_kernel<T><<<(unsigned)((plane + 255) / 256), 256, 0, c->stream>>>(
                a, static_cast<T*>(c->state[c->cur]), face, c->mbc_kind[face], c->mbc_uwall[face],
                c->mbc_radius[face] * c->mbc_radius[face], c->mbc_amp[face], step);
        });
        c->launches++;
        CUDA_TRY(c, cudaGetLastError());
    }
    return TSLB_OK;
}

int launch_step(tslb_ctx* c) {
    {
        int rc = launch_moment_bcs(c);
        if (rc) return rc;
    }
    if (c->closure) {
        int rc = tslb_internal::closure_before_step(c);
        if (rc) return rc;
    }
    StepArgs a = make_args(c, c->state[c->cur], c->state[c->cur ^ 1]);
    CUDA_TRY(c, launch_step_kernel(a, c->p.mode, c->p.precision, c->stream));
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    c->cur ^= 1;
    c->steps_done++;
    return TSLB_OK;
}

// FP32 fields in io (rho already shifted) -> the state in its storage type
int io_to_state(tslb_ctx* c) {
    StepArgs a = make_args(c, nullptr, nullptr);
    const int bs = 256;
    with_storage(c->p.precision, [&](auto tag) {
        using T = decltype(tag);
        to_storage_kernel<T><<<(unsigned)((c->n + bs - 1) / bs), bs, 0, c->stream>>>(c->io, reinterpret_cast<T*>(c->state[c->cur]), c->N, c->n, a);
    });
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

// the state -> FP32 fields in io (rho stays rho - 1)
int state_to_io(tslb_ctx* c) {
    StepArgs a = make_args(c, nullptr, nullptr);
    const int bs = 256;
    with_storage(c->p.precision, [&](auto tag) {
        using T = decltype(tag);
        from_storage_kernel<T><<<(unsigned)((c->n + bs - 1) / bs), bs, 0, c->stream>>>(reinterpret_cast<const T*>(c->state[c->cur]), c->io, c->N, c->n, a);
    });
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

}  // namespace

namespace tslb_internal {

// FP32 view of the current state: the state itself, or io after conversion
int fp32_view(tslb_ctx* c, const float** out) {
    if (c->p.precision == TSLB_PREC_FP32) {
        *out = static_cast<const float*>(c->state[c->cur]);
        return TSLB_OK;
    }
    int rc = state_to_io(c);
    *out = c->io;
    return rc;
}

// single-component mode: phi is held at 1 and the step does not write it,
// so both ping-pong buffers carry the same phi field
int single_phi_both(tslb_ctx* c) {
    if (c->p.mode != TSLB_MODE_SINGLE) return TSLB_OK;
    const size_t off = (size_t)F_PHI * c->N * c->esize, bytes = (size_t)c->n * c->esize;
    CUDA_TRY(c, cudaMemcpyAsync(static_cast<char*>(c->state[c->cur ^ 1]) + off, static_cast<char*>(c->state[c->cur]) + off,
                                bytes, cudaMemcpyDeviceToDevice, c->stream));
    return TSLB_OK;
}

int ensure_dtau(tslb_ctx* c) {
    if (c->dtau) return TSLB_OK;
    CUDA_TRY(c, cudaMalloc(&c->dtau, sizeof(float) * c->N));
    CUDA_TRY(c, cudaMemsetAsync(c->dtau, 0, sizeof(float) * c->N, c->stream));
    return TSLB_OK;
}

int prepare_step_kernel(tslb_ctx* c) {
    StepArgs a = make_args(c, c->state[c->cur], c->state[c->cur ^ 1]);
    CUDA_TRY(c, launch_step_kernel(a, c->p.mode, c->p.precision, c->stream, false));
    return TSLB_OK;
}

}  // namespace tslb_internal

namespace {

using tslb_internal::fp32_view;

// Default power-of-two scales of fp16 storage: stored magnitudes near 2^10
// for typical moments (|rho - 1| < 1/16, |u| < 1/4, |Pi^neq| < 1/16, |phi| <= 1).
void default_scales(tslb_ctx* c) {
    for (int f = 0; f < NF; ++f) c->scale[f] = 1.0f;
    if (c->p.precision != TSLB_PREC_FP16S) return;
    c->scale[F_D] = 16384.f;
    c->scale[F_U] = c->scale[F_V] = c->scale[F_W] = 4096.f;
    for (int f = F_XX; f <= F_ZZ; ++f) c->scale[f] = 16384.f;
    c->scale[F_PHI] = 1024.f;
}

}  // namespace

// ------------------------------------------------------------------ C-ABI
extern "C" {

void tslb_default_params(tslb_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->mode = TSLB_MODE_PHASEFIELD;
    p->precision = TSLB_PREC_FP32;
    p->tau_a = 0.5004f;  // recursive_2c_TSLB3D.f90:21
    p->tau_b = 0.5004f;
    p->sigma = 0.001f;   // :27
    p->beta = 0.7f;
    p->sharp_c = 0.3f * 3;  // :28
    p->grad_threshold = 1e-3f;  // recursive_colorTSLB3D.f90:763
    for (int f = 0; f < 6; ++f) { p->bc[f] = TSLB_BC_PERIODIC; p->bc_phi[f] = 0.f; }
    p->wall_phi_mode = 0;
}

int tslb_create(const tslb_params* p, int nx, int ny, int nz, tslb_ctx** out) {
    if (!out) return fail(nullptr, TSLB_ERR_ARG, "out is NULL");
    *out = nullptr;
    std::string why;
    int rc = validate(p, nx, ny, nz, why);
    if (rc) return fail(nullptr, rc, why);
    tslb_ctx* c = new (std::nothrow) tslb_ctx();
    if (!c) return fail(nullptr, TSLB_ERR_ARG, "out of host memory");
    c->p = *p;
    c->nx = nx; c->ny = ny; c->nz = nz;
    c->n = (long long)nx * ny * nz;
    c->N = (c->n + 31) / 32 * 32;
    auto bail = [&](cudaError_t e, const char* what) {
        g_create_error = std::string(what) + ": " + cudaGetErrorString(e);
        tslb_destroy(c);
        return TSLB_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaGetDevice(&c->device)) != cudaSuccess) return bail(e, "cudaGetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "cudaStreamCreate");
    c->esize = storage_bytes(p->precision);
    default_scales(c);
    for (int b = 0; b < 2; ++b)
        if ((e = pool_alloc(&c->state[b], (size_t)c->esize * NF * c->N, c->device, c->stream)) != cudaSuccess)
            return bail(e, "allocation (state)");
    if (p->precision != TSLB_PREC_FP32)
        if ((e = pool_alloc(reinterpret_cast<void**>(&c->io), sizeof(float) * NF * c->N, c->device, c->stream)) != cudaSuccess)
            return bail(e, "allocation (io)");
    // rho = 1 + d for downloads (with the lattice, so lattices of one size
    // allocate alike and reuse each other's pool memory)
    if ((e = pool_alloc(reinterpret_cast<void**>(&c->rho_out), sizeof(float) * c->N, c->device, c->stream)) != cudaSuccess)
        return bail(e, "allocation (rho)");
    // the step forms the interface normals it needs itself; the normal field
    // is allocated when tslb_download_normals asks for it
    {
        int sm_count = 148;
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, c->device);
        c->red_blocks = 4 * sm_count;
        // reduction partials, results and ticket (one more double), then the
        // non-finite flag: one pool block, cleared on the stream
        const size_t red_bytes = (sizeof(double) * ((size_t)c->red_blocks * RED_PARTS + RED_PARTS + 1) + 15) / 16 * 16;
        if ((e = pool_alloc(reinterpret_cast<void**>(&c->red), red_bytes + 16, c->device, c->stream)) != cudaSuccess)
            return bail(e, "allocation (reduce)");
        c->flags = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(c->red) + red_bytes);
        if ((e = cudaMemsetAsync(c->red, 0, red_bytes + 16, c->stream)) != cudaSuccess) return bail(e, "cudaMemsetAsync(reduce)");
        if ((e = pinned_get(reinterpret_cast<void**>(&c->red_host), kRedHostBytes)) != cudaSuccess)
            return bail(e, "cudaHostAlloc(reduce)");
    }
    for (int f = 0; f < 6; ++f) {
        if (p->bc[f] != TSLB_BC_INLET) continue;
        size_t bytes = sizeof(float) * 4 * face_area(c, f);
        if ((e = pool_alloc(reinterpret_cast<void**>(&c->inlet[f]), bytes, c->device, c->stream)) != cudaSuccess)
            return bail(e, "allocation (inlet)");
        if ((e = cudaMemsetAsync(c->inlet[f], 0, bytes, c->stream)) != cudaSuccess) return bail(e, "cudaMemsetAsync(inlet)");
    }
    // the pool's allocations and the clears are ordered on the lattice's stream: complete them for every stream
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return bail(e, "cudaStreamSynchronize");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    c->zchunk = choose_zchunk(step_tiles(nx, ny), nz, sms, kStepBlocksPerSM, p->mode);
    if ((e = launch_step_kernel(make_args(c, c->state[0], c->state[1]), p->mode, p->precision, c->stream, false)) != cudaSuccess)
        return bail(e, "cudaFuncSetAttribute");
    *out = c;
    return TSLB_OK;
}

void tslb_destroy(tslb_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int b = 0; b < 2; ++b) pool_free(c->state[b], c->stream);
    pool_free(c->io, c->stream);
    pool_free(c->rho_out, c->stream);
    pool_free(c->nrm, c->stream);
    pool_free(c->red, c->stream);   // with the flag word
    for (int f = 0; f < 6; ++f) pool_free(c->inlet[f], c->stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    pinned_put(c->red_host, kRedHostBytes);
    pinned_put(c->red_ring, kRingBytes);
    cudaFree(c->dtau);
    cudaFree(c->dtau_base);
    cudaFree(c->solid);
    cudaFree(c->near);
    cudaFree(c->stats);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int tslb_upload_moments(tslb_ctx* c, const float* rho, const float* u, const float* v, const float* w,
                        const float* pxx, const float* pxy, const float* pxz, const float* pyy,
                        const float* pyz, const float* pzz, const float* phi) {
    if (!c) return TSLB_ERR_ARG;
    const float* src[NF] = {rho, u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi};
    std::vector<float> ones;
    if (c->p.mode == TSLB_MODE_SINGLE) {
        // single component: phi is held at 1 (the argument may be NULL)
        ones.assign((size_t)c->n, 1.0f);
        src[F_PHI] = ones.data();
    }
    for (int f = 0; f < NF; ++f)
        if (!src[f]) return fail(c, TSLB_ERR_ARG, "tslb_upload_moments: NULL field");
    const bool fp32 = c->p.precision == TSLB_PREC_FP32;
    float* s = fp32 ? static_cast<float*>(c->state[c->cur]) : c->io;
    if (c->p.precision == TSLB_PREC_FP16S) {
        // per-field power-of-two scales from the data: largest |value| near 2^10
        default_scales(c);
        for (int f = 0; f < NF; ++f) {
            double mx = 0.0;
            for (long long i = 0; i < c->n; ++i) {
                const double v = f == F_D ? (double)src[f][i] - 1.0 : (double)src[f][i];
                mx = std::max(mx, std::fabs(v));
            }
            if (mx > 0.0 && std::isfinite(mx)) {
                const int k = std::max(-8, std::min(24, (int)std::floor(std::log2(1024.0 / mx))));
                c->scale[f] = std::ldexp(1.0f, k);
            }
        }
    }
    for (int f = 0; f < NF; ++f)
        CUDA_TRY(c, cudaMemcpyAsync(s + f * c->N, src[f], sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
    const int bs = 256;
    shift_rho_kernel<<<(unsigned)((c->n + bs - 1) / bs), bs, 0, c->stream>>>(s + F_D * c->N, c->n);
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    if (!fp32) {
        int rc = io_to_state(c);
        if (rc) return rc;
    }
    int rc = tslb_internal::single_phi_both(c);
    if (rc) return rc;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->loaded = true;
    return TSLB_OK;
}

int tslb_upload_pops(tslb_ctx* c, const float* f, const float* g) {
    if (!c) return TSLB_ERR_ARG;
    const bool single = c->p.mode == TSLB_MODE_SINGLE;
    if (!f || (!g && !single)) return fail(c, TSLB_ERR_ARG, "tslb_upload_pops: NULL populations");
    const long long vol = (long long)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
    const int nqg = c->p.mode == TSLB_MODE_COLOUR ? 27 : 7;
    float *df = nullptr, *dg = nullptr;
    CUDA_TRY(c, cudaMalloc(&df, sizeof(float) * 27 * vol));
    cudaError_t e = single ? cudaSuccess : cudaMalloc(&dg, sizeof(float) * nqg * vol);
    if (e != cudaSuccess) { cudaFree(df); return fail(c, TSLB_ERR_CUDA, std::string("cudaMalloc(g): ") + cudaGetErrorString(e)); }
    e = cudaMemcpyAsync(df, f, sizeof(float) * 27 * vol, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && !single) e = cudaMemcpyAsync(dg, g, sizeof(float) * nqg * vol, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        const int bs = 128;
        const bool fp32 = c->p.precision == TSLB_PREC_FP32;
        float* dst = fp32 ? static_cast<float*>(c->state[c->cur]) : c->io;
        pops_to_moments_kernel<<<(unsigned)((c->n + bs - 1) / bs), bs, 0, c->stream>>>(
            c->nx, c->ny, c->nz, c->N, c->p.mode == TSLB_MODE_COLOUR, df, dg, dst);
        c->launches++;
        e = cudaGetLastError();
        if (e == cudaSuccess && !fp32) {
            default_scales(c);
            if (io_to_state(c) != TSLB_OK) e = cudaGetLastError();
        }
        if (e == cudaSuccess && tslb_internal::single_phi_both(c) != TSLB_OK) e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(df);
    cudaFree(dg);
    if (e != cudaSuccess) return fail(c, TSLB_ERR_CUDA, std::string("tslb_upload_pops: ") + cudaGetErrorString(e));
    c->loaded = true;
    return TSLB_OK;
}

int tslb_step(tslb_ctx* c, int nsteps) {
    if (!c) return TSLB_ERR_ARG;
    if (nsteps < 0) return fail(c, TSLB_ERR_ARG, "nsteps < 0");
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "tslb_step before an upload");
    for (int s = 0; s < nsteps; ++s) {
        int rc = launch_step(c);
        if (rc) return rc;
    }
    return TSLB_OK;
}

int tslb_download_moments(tslb_ctx* c, float* rho, float* u, float* v, float* w, float* pxx, float* pxy,
                          float* pxz, float* pyy, float* pyz, float* pzz, float* phi) {
    if (!c) return TSLB_ERR_ARG;
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "download before an upload");
    float* dst[NF] = {rho, u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi};
    const float* s = nullptr;
    int rc = fp32_view(c, &s);
    if (rc) return rc;
    for (int f = 0; f < NF; ++f) {
        if (!dst[f]) continue;
        const float* src = s + f * c->N;
        if (f == F_D) {
            // the state holds d = rho - 1: rho is formed on the device
            const int bs = 256;
            rho_from_d_kernel<<<(unsigned)((c->n + bs - 1) / bs), bs, 0, c->stream>>>(src, c->rho_out, c->n);
            c->launches++;
            CUDA_TRY(c, cudaGetLastError());
            src = c->rho_out;
        }
        CUDA_TRY(c, cudaMemcpyAsync(dst[f], src, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

void* tslb_host_alloc(long long bytes) {
    if (bytes <= 0) return nullptr;
    void* p = nullptr;
    if (cudaMallocHost(&p, (size_t)bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void tslb_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

int tslb_download_normals(tslb_ctx* c, float* nx, float* ny, float* nz) {
    if (!c) return TSLB_ERR_ARG;
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "download before an upload");
    int rc = launch_normals(c);
    if (rc) return rc;
    float* dst[3] = {nx, ny, nz};
    for (int k = 0; k < 3; ++k)
        if (dst[k]) CUDA_TRY(c, cudaMemcpyAsync(dst[k], c->nrm + k * c->N, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return TSLB_OK;
}

}  // extern "C"

namespace {

// the nodes a context owns: all of them, or a z slab's own planes
void owned_nodes(const tslb_ctx* c, long long* off, long long* n) {
    const long long plane = (long long)c->nx * c->ny;
    const int zt1 = c->zt1 > 0 ? c->zt1 : c->nz;
    *off = (long long)c->zt0 * plane;
    *n = (long long)(zt1 - c->zt0) * plane;
}

// queue the FP64 reduction of the current state and its copy into host_dst
// (RED_PARTS doubles; page-locked for an asynchronous copy)
int enqueue_reduce(tslb_ctx* c, double* host_dst) {
    const float* view = nullptr;
    int rc = fp32_view(c, &view);
    if (rc) return rc;
    long long off = 0, n = 0;
    owned_nodes(c, &off, &n);
    double* results = c->red + (size_t)c->red_blocks * RED_PARTS;
    unsigned int* ticket = reinterpret_cast<unsigned int*>(results + RED_PARTS);
    reduce_kernel<<<(unsigned)c->red_blocks, RED_THREADS, 0, c->stream>>>(view + off, n, c->N, c->p.mode == TSLB_MODE_COLOUR,
                                                                          c->red, results, ticket);
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(host_dst, results, sizeof(double) * RED_PARTS, cudaMemcpyDeviceToHost, c->stream));
    return TSLB_OK;
}

// the TSLB_RED_* values of one copied reduction
void finish_reduce(const tslb_ctx* c, const double* h, double* out) {
    long long off = 0, n = 0;
    owned_nodes(c, &off, &n);
    const double umax2 = h[RED_SLOTS];
    out[TSLB_RED_MASS] = (double)n + h[0];
    out[TSLB_RED_MASS_A] = h[1];
    out[TSLB_RED_MASS_B] = h[2];
    out[TSLB_RED_MOM_X] = h[3];
    out[TSLB_RED_MOM_Y] = h[4];
    out[TSLB_RED_MOM_Z] = h[5];
    out[TSLB_RED_KINETIC] = h[6];
    out[TSLB_RED_UMAX] = std::sqrt(umax2);
    out[TSLB_RED_RHO_IN] = h[8] > 0 ? h[7] / h[8] : 0.0;
    out[TSLB_RED_RHO_OUT] = h[10] > 0 ? h[9] / h[10] : 0.0;
    out[TSLB_RED_DP] = (h[8] > 0 && h[10] > 0) ? (out[TSLB_RED_RHO_IN] - out[TSLB_RED_RHO_OUT]) / 3.0 : 0.0;
    out[TSLB_RED_N_IN] = h[8];
}

}  // namespace

extern "C" {

int tslb_reduce(tslb_ctx* c, double out[TSLB_NREDUCE]) {
    if (!c || !out) return fail(c, TSLB_ERR_ARG, "tslb_reduce: NULL");
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "reduce before an upload");
    int rc = enqueue_reduce(c, c->red_host);
    if (rc) return rc;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    finish_reduce(c, c->red_host, out);
    return check_flags(c);
}

int tslb_reduce_async(tslb_ctx* c) {
    if (!c) return TSLB_ERR_ARG;
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "reduce before an upload");
    if (c->red_queued >= TSLB_REDUCE_QUEUE)
        return fail(c, TSLB_ERR_STATE, "tslb_reduce_async: TSLB_REDUCE_QUEUE results wait; call tslb_reduce_collect");
    if (!c->red_ring)
        CUDA_TRY(c, pinned_get(reinterpret_cast<void**>(&c->red_ring), kRingBytes));
    int rc = enqueue_reduce(c, c->red_ring + (size_t)c->red_queued * RED_PARTS);
    if (rc) return rc;
    c->red_queued++;
    return TSLB_OK;
}

int tslb_reduce_collect(tslb_ctx* c, double* out, int max, int* count) {
    if (!c) return TSLB_ERR_ARG;
    if (count) *count = 0;
    if (max > 0 && !out) return fail(c, TSLB_ERR_ARG, "tslb_reduce_collect: NULL output");
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const int k = std::min(std::max(max, 0), c->red_queued);
    for (int i = 0; i < k; ++i) finish_reduce(c, c->red_ring + (size_t)i * RED_PARTS, out + (size_t)i * TSLB_NREDUCE);
    if (count) *count = k;
    c->red_queued = 0;
    return check_flags(c);
}

int tslb_set_inlet(tslb_ctx* c, int face, const float* uvw_phi) {
    if (!c) return TSLB_ERR_ARG;
    if (face < 0 || face > 5 || !uvw_phi) return fail(c, TSLB_ERR_ARG, "tslb_set_inlet: bad face or NULL plane");
    if (c->p.bc[face] != TSLB_BC_INLET || !c->inlet[face]) return fail(c, TSLB_ERR_ARG, "tslb_set_inlet: face is not an inlet");
    CUDA_TRY(c, cudaMemcpyAsync(c->inlet[face], uvw_phi, sizeof(float) * 4 * face_area(c, face), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return TSLB_OK;
}

int tslb_set_inlet_disc(tslb_ctx* c, int face, float c0, float c1, float radius, float speed, float amp,
                        unsigned long long seed, unsigned long long counter) {
    if (!c) return TSLB_ERR_ARG;
    if (face < 0 || face > 5) return fail(c, TSLB_ERR_ARG, "tslb_set_inlet_disc: bad face");
    if (c->p.bc[face] != TSLB_BC_INLET || !c->inlet[face]) return fail(c, TSLB_ERR_ARG, "tslb_set_inlet_disc: face is not an inlet");
    if (!std::isfinite(c0) || !std::isfinite(c1) || !std::isfinite(radius) || !std::isfinite(speed) || !std::isfinite(amp))
        return fail(c, TSLB_ERR_ARG, "tslb_set_inlet_disc: non-finite argument");
    const int ax = face / 2;
    const int n0 = ax == 0 ? c->ny : c->nx, n1 = ax == 2 ? c->ny : c->nz;
    const long long pa = (long long)n0 * n1;
    inlet_disc_kernel<<<(unsigned)((pa + 255) / 256), 256, 0, c->stream>>>(c->inlet[face], n0, n1, ax, (face & 1) ? -1.f : 1.f, c0, c1,
                                                                          radius * radius, speed, amp, seed, counter);
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

float tslb_rand_noseeded(int i, int j, int k, int l) { return rand_noseeded(i, j, k, l); }

int tslb_set_moment_bc(tslb_ctx* c, int face, int kind, float uwall, float radius, float amp) {
    if (!c) return TSLB_ERR_ARG;
    if (face != 4 && face != 5) return fail(c, TSLB_ERR_UNSUPPORTED, "tslb_set_moment_bc: z faces (4, 5) only");
    if (kind < TSLB_MBC_NONE || kind > TSLB_MBC_JET) return fail(c, TSLB_ERR_ARG, "tslb_set_moment_bc: unknown kind");
    if (c->nz < 3) return fail(c, TSLB_ERR_ARG, "tslb_set_moment_bc: nz must be >= 3");
    if ((face == 4 && c->halo_lo) || (face == 5 && c->halo_hi))
        return fail(c, TSLB_ERR_UNSUPPORTED, "tslb_set_moment_bc: the face belongs to a neighbouring slab");
    if (!std::isfinite(uwall) || !std::isfinite(radius) || !std::isfinite(amp))
        return fail(c, TSLB_ERR_ARG, "tslb_set_moment_bc: non-finite argument");
    c->mbc_kind[face] = kind;
    c->mbc_uwall[face] = uwall;
    c->mbc_radius[face] = radius;
    c->mbc_amp[face] = amp;
    return TSLB_OK;
}

int tslb_set_solid_mask(tslb_ctx* c, const unsigned char* isfluid) {
    if (!c) return TSLB_ERR_ARG;
    if (!isfluid) {
        c->solid_on = false;
        return TSLB_OK;
    }
    if (c->p.precision != TSLB_PREC_FP32)
        return fail(c, TSLB_ERR_UNSUPPORTED, "tslb_set_solid_mask: FP32 storage only");
    if (c->base_on || c->closure)
        return fail(c, TSLB_ERR_UNSUPPORTED, "tslb_set_solid_mask: not combined with a tau correction or closure");
    const long long words = (c->n + 31) / 32;
    if (!c->solid) CUDA_TRY(c, cudaMalloc(&c->solid, sizeof(unsigned int) * words));
    if (!c->near) CUDA_TRY(c, cudaMalloc(&c->near, sizeof(unsigned int) * words));
    unsigned char* d = nullptr;
    CUDA_TRY(c, cudaMalloc(&d, (size_t)c->n));
    cudaError_t e = cudaMemcpyAsync(d, isfluid, (size_t)c->n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        const unsigned g = (unsigned)((words + 255) / 256);
        solid_bits_kernel<<<g, 256, 0, c->stream>>>(d, c->n, c->solid);
        near_bits_kernel<<<g, 256, 0, c->stream>>>(d, c->nx, c->ny, c->nz, c->p.bc[0] == TSLB_BC_PERIODIC,
                                                  c->p.bc[2] == TSLB_BC_PERIODIC, c->p.bc[4] == TSLB_BC_PERIODIC, c->near);
        c->launches += 2;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(c, TSLB_ERR_CUDA, std::string("tslb_set_solid_mask: ") + cudaGetErrorString(e));
    c->solid_on = true;
    return tslb_internal::prepare_step_kernel(c);
}

int tslb_set_tau_correction(tslb_ctx* c, const float* dtau) {
    if (!c) return TSLB_ERR_ARG;
    if (c->solid_on && dtau) return fail(c, TSLB_ERR_UNSUPPORTED, "tslb_set_tau_correction: not combined with solid nodes");
    if (!dtau) {
        c->base_on = false;
        return TSLB_OK;
    }
    if (c->p.mode != TSLB_MODE_COLOUR || c->p.precision != TSLB_PREC_FP32)
        return fail(c, TSLB_ERR_ARG, "tslb_set_tau_correction: colour mode with FP32 storage only");
    const float lo = -(std::min(c->p.tau_a, c->p.tau_b) - 0.5f);
    for (long long i = 0; i < c->n; ++i)
        if (!std::isfinite(dtau[i]) || !(dtau[i] > lo))
            return fail(c, TSLB_ERR_ARG, "tslb_set_tau_correction: non-finite value or tau + dtau <= 1/2");
    if (!c->dtau_base) CUDA_TRY(c, cudaMalloc(&c->dtau_base, sizeof(float) * c->N));
    CUDA_TRY(c, cudaMemcpyAsync(c->dtau_base, dtau, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->base_on = true;
    return tslb_internal::prepare_step_kernel(c);
}

int tslb_download_tau_correction(tslb_ctx* c, float* dtau) {
    if (!c || !dtau) return fail(c, TSLB_ERR_ARG, "tslb_download_tau_correction: NULL");
    const float* src = c->closure ? c->dtau : (c->base_on ? c->dtau_base : nullptr);
    if (!src) {
        for (long long i = 0; i < c->n; ++i) dtau[i] = 0.f;
        return TSLB_OK;
    }
    CUDA_TRY(c, cudaMemcpyAsync(dtau, src, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return TSLB_OK;
}

int tslb_stats_reset(tslb_ctx* c) {
    if (!c) return TSLB_ERR_ARG;
    if (!c->stats) CUDA_TRY(c, cudaMalloc(&c->stats, sizeof(float) * NSTATS * c->N));
    CUDA_TRY(c, cudaMemsetAsync(c->stats, 0, sizeof(float) * NSTATS * c->N, c->stream));
    c->stats_count = 0;
    return TSLB_OK;
}

int tslb_stats_accumulate(tslb_ctx* c) {
    if (!c) return TSLB_ERR_ARG;
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "tslb_stats_accumulate before an upload");
    if (!c->stats) {
        int rc = tslb_stats_reset(c);
        if (rc) return rc;
    }
    const float* view = nullptr;
    int rc = fp32_view(c, &view);
    if (rc) return rc;
    stats_accumulate_kernel<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(view, c->n, c->N, c->stats);
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    c->stats_count++;
    return TSLB_OK;
}

namespace {
// block means of running-sum slots k0 .. k0 + nk - 1 into the host arrays dst[0 .. nk-1] (NULL: skipped)
int stats_fetch(tslb_ctx* c, const char* who, int coarsen, int k0, int nk, float* const* dst, long long* count) {
    if (coarsen < 1 || c->nx % coarsen || c->ny % coarsen || c->nz % coarsen)
        return fail(c, TSLB_ERR_ARG, std::string(who) + ": coarsening factor must divide the lattice sizes");
    if (count) *count = c->stats_count;
    if (!c->stats || c->stats_count == 0) return fail(c, TSLB_ERR_STATE, std::string(who) + ": no accumulated samples");
    const long long nc = c->n / ((long long)coarsen * coarsen * coarsen);
    float* tmp = nullptr;
    CUDA_TRY(c, cudaMalloc(&tmp, sizeof(float) * nk * nc));
    const float inv = 1.0f / ((float)c->stats_count * coarsen * coarsen * coarsen);
    stats_coarsen_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(c->stats, c->nx, c->ny, c->nz, c->N, coarsen,
                                                                            k0, nk, inv, tmp);
    c->launches++;
    cudaError_t e = cudaGetLastError();
    for (int k = 0; k < nk && e == cudaSuccess; ++k)
        if (dst[k]) e = cudaMemcpyAsync(dst[k], tmp + k * nc, sizeof(float) * nc, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return fail(c, TSLB_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
    return TSLB_OK;
}
}  // namespace

int tslb_stats_download(tslb_ctx* c, int coarsen, float* u, float* v, float* w, float* phi, float* ww, long long* count) {
    if (!c) return TSLB_ERR_ARG;
    float* const dst[5] = {u, v, w, phi, ww};
    return stats_fetch(c, "tslb_stats_download", coarsen, 0, 5, dst, count);
}

int tslb_stats_download_stress(tslb_ctx* c, int coarsen, float* uu, float* pineq, long long* count) {
    if (!c) return TSLB_ERR_ARG;
    if (coarsen < 1 || c->nx % coarsen || c->ny % coarsen || c->nz % coarsen)
        return fail(c, TSLB_ERR_ARG, "tslb_stats_download_stress: coarsening factor must divide the lattice sizes");
    const long long nc = c->n / ((long long)coarsen * coarsen * coarsen);
    // uu: (uu, uv, uw, vv, vw, ww) as six consecutive arrays of nc values
    float* const d1[6] = {uu ? uu : nullptr, uu ? uu + nc : nullptr, uu ? uu + 2 * nc : nullptr,
                          uu ? uu + 3 * nc : nullptr, uu ? uu + 4 * nc : nullptr, uu ? uu + 5 * nc : nullptr};
    int rc = stats_fetch(c, "tslb_stats_download_stress", coarsen, 5, 5, d1, count);
    if (rc) return rc;
    float* const d2[1] = {uu ? uu + 5 * nc : nullptr};
    rc = stats_fetch(c, "tslb_stats_download_stress", coarsen, 4, 1, d2, count);
    if (rc) return rc;
    float* const d3[6] = {pineq ? pineq : nullptr, pineq ? pineq + nc : nullptr, pineq ? pineq + 2 * nc : nullptr,
                          pineq ? pineq + 3 * nc : nullptr, pineq ? pineq + 4 * nc : nullptr, pineq ? pineq + 5 * nc : nullptr};
    return stats_fetch(c, "tslb_stats_download_stress", coarsen, 10, 6, d3, count);
}

int tslb_synchronize(tslb_ctx* c) {
    if (!c) return TSLB_ERR_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

void* tslb_stream(tslb_ctx* c) { return c ? (void*)c->stream : nullptr; }

int tslb_release_memory(void) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (int d = 0; d < MAX_DEVICES; ++d)
        if (g_pool[d] && cudaMemPoolTrimTo(g_pool[d], 0) != cudaSuccess) return TSLB_ERR_CUDA;
    return TSLB_OK;
}

long long tslb_launch_count(tslb_ctx* c) { return c ? c->launches : 0; }

const char* tslb_last_error(tslb_ctx* c) {
    if (!c) return g_create_error.c_str();
    return c->err.c_str();
}

}  // extern "C"

// ---- checkpoints (include/tslb_io.h) ----
namespace {
struct CkptHeader {
    char magic[8];
    int32_t version, nx, ny, nz, mode, precision, esize, nfields;
    long long steps_done;
    float scale[NF];
    tslb_params params;
};
const char kCkptMagic[8] = {'T', 'S', 'L', 'B', 'C', 'K', 'P', '1'};
}  // namespace

extern "C" {

long long tslb_steps_done(tslb_ctx* c) { return c ? c->steps_done : 0; }

int tslb_checkpoint_save(tslb_ctx* c, const char* path) {
    if (!c || !path) return fail(c, TSLB_ERR_ARG, "tslb_checkpoint_save: NULL");
    if (!c->loaded) return fail(c, TSLB_ERR_STATE, "tslb_checkpoint_save before an upload");
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = 1; h.nx = c->nx; h.ny = c->ny; h.nz = c->nz; h.mode = c->p.mode; h.precision = c->p.precision;
    h.esize = c->esize; h.nfields = NF; h.steps_done = c->steps_done;
    for (int f = 0; f < NF; ++f) h.scale[f] = c->scale[f];
    h.params = c->p;
    std::vector<char> buf((size_t)c->esize * c->n);
    FILE* fh = std::fopen(path, "wb");
    if (!fh) return fail(c, TSLB_ERR_ARG, std::string("tslb_checkpoint_save: cannot open ") + path);
    bool ok = std::fwrite(&h, sizeof(h), 1, fh) == 1;
    for (int f = 0; f < NF && ok; ++f) {
        const char* src = static_cast<const char*>(c->state[c->cur]) + (size_t)f * c->N * c->esize;
        cudaError_t e = cudaMemcpyAsync(buf.data(), src, buf.size(), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            std::fclose(fh);
            return fail(c, TSLB_ERR_CUDA, std::string("tslb_checkpoint_save: ") + cudaGetErrorString(e));
        }
        ok = std::fwrite(buf.data(), 1, buf.size(), fh) == buf.size();
    }
    if (std::fclose(fh) != 0 || !ok) return fail(c, TSLB_ERR_ARG, std::string("tslb_checkpoint_save: write failed: ") + path);
    return TSLB_OK;
}

int tslb_checkpoint_load(tslb_ctx* c, const char* path) {
    if (!c || !path) return fail(c, TSLB_ERR_ARG, "tslb_checkpoint_load: NULL");
    FILE* fh = std::fopen(path, "rb");
    if (!fh) return fail(c, TSLB_ERR_ARG, std::string("tslb_checkpoint_load: cannot open ") + path);
    CkptHeader h;
    if (std::fread(&h, sizeof(h), 1, fh) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1 ||
        h.nfields != NF) {
        std::fclose(fh);
        return fail(c, TSLB_ERR_ARG, "tslb_checkpoint_load: not a TSLB checkpoint");
    }
    if (h.nx != c->nx || h.ny != c->ny || h.nz != c->nz || h.mode != c->p.mode || h.precision != c->p.precision ||
        h.esize != c->esize) {
        std::fclose(fh);
        return fail(c, TSLB_ERR_ARG, "tslb_checkpoint_load: sizes, mode or precision differ from the lattice's");
    }
    std::vector<char> buf((size_t)c->esize * c->n);
    for (int f = 0; f < NF; ++f) {
        if (std::fread(buf.data(), 1, buf.size(), fh) != buf.size()) {
            std::fclose(fh);
            return fail(c, TSLB_ERR_ARG, "tslb_checkpoint_load: truncated file");
        }
        char* dst = static_cast<char*>(c->state[c->cur]) + (size_t)f * c->N * c->esize;
        cudaError_t e = cudaMemcpyAsync(dst, buf.data(), buf.size(), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            std::fclose(fh);
            return fail(c, TSLB_ERR_CUDA, std::string("tslb_checkpoint_load: ") + cudaGetErrorString(e));
        }
    }
    std::fclose(fh);
    for (int f = 0; f < NF; ++f) c->scale[f] = h.scale[f];
    c->steps_done = h.steps_done;
    int rc = tslb_internal::single_phi_both(c);
    if (rc) return rc;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->loaded = true;
    return TSLB_OK;
}

}  // extern "C"


// ------------------------------------------------- step without allocation
// Scratch of tslb_step_noalloc: the step kernel's non-finite flag, in a fixed
// device array of this file (TSLB_NOALLOC_SCRATCH_WORDS words; the step
// needs no scratch that grows with the lattice).  In host code the name is a
// host-side stand-in, not a device address; the address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned int g_noalloc_flags[TSLB_NOALLOC_SCRATCH_WORDS];

namespace {
constexpr int kMaxDevices = 64;
struct NoallocScratch {
    bool ready = false;
    unsigned int* flags = nullptr;
};
NoallocScratch g_noalloc[kMaxDevices];
std::mutex g_noalloc_mu;

// context-free failures report through tslb_last_error(NULL)
int noalloc_fail(int code, const std::string& msg) {
    g_create_error = msg;
    return code;
}

// Once per device, with that device current: resolve the scratch address
// and set the shared-memory attribute of every step kernel the entry point
// can launch (FP32 storage, the three modes, x aligned to 16 bytes or not),
// so later calls make no first-use runtime calls of their own.
int noalloc_setup(int dev, NoallocScratch** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocScratch& s = g_noalloc[dev];
    if (!s.ready) {
        cudaError_t e = cudaGetSymbolAddress((void**)&s.flags, g_noalloc_flags);
        if (e != cudaSuccess) return noalloc_fail(TSLB_ERR_CUDA, std::string("cudaGetSymbolAddress(flags): ") + cudaGetErrorString(e));
        const int modes[3] = {TSLB_MODE_PHASEFIELD, TSLB_MODE_COLOUR, TSLB_MODE_SINGLE};
        for (int mode : modes) {
            for (int nx : {4, 3}) {   // 16-byte aligned rows, and not
                StepArgs a;
                std::memset(&a, 0, sizeof(a));
                a.nx = nx; a.ny = 1; a.nz = 1; a.zchunk = 1;
                e = launch_step_kernel(a, mode, TSLB_PREC_FP32, nullptr, false);
                if (e != cudaSuccess) return noalloc_fail(TSLB_ERR_CUDA, std::string("step kernel attribute: ") + cudaGetErrorString(e));
            }
        }
        s.ready = true;
    }
    *out = &s;
    return TSLB_OK;
}

// [a, a + bytes) and [b, b + bytes) share a byte
bool ranges_overlap(const void* a, const void* b, unsigned long long bytes) {
    const unsigned long long x = (unsigned long long)(uintptr_t)a, y = (unsigned long long)(uintptr_t)b;
    return x < y + bytes && y < x + bytes;
}
}  // namespace

extern "C" int tslb_step_noalloc(const tslb_params* p, int nx, int ny, int nz, const float* d_in, float* d_out,
                                 long long field_stride, void* stream) {
    std::string why;
    int rc = validate(p, nx, ny, nz, why);
    if (rc) return noalloc_fail(rc, "tslb_step_noalloc: " + why);
    const long long n = (long long)nx * ny * nz;
    if (!d_in || !d_out) return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: NULL device buffer");
    if (field_stride < n || field_stride % 4 != 0)
        return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: field_stride must be >= nx*ny*nz and a multiple of 4");
    if (field_stride > (1LL << 40)) return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: field_stride too large");
    // the step reads halo neighbours of d_in after it has written d_out: the
    // two 11-field ranges must not share a byte
    if (ranges_overlap(d_in, d_out, (unsigned long long)NF * (unsigned long long)field_stride * sizeof(float)))
        return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: d_in and d_out overlap (each spans 11 * field_stride floats)");
    if (((uintptr_t)d_in | (uintptr_t)d_out) % 16 != 0)
        return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: d_in and d_out must be 16-byte aligned");
    for (int f = 0; f < 6; ++f)
        if (p->bc[f] == TSLB_BC_INLET) return noalloc_fail(TSLB_ERR_UNSUPPORTED, "tslb_step_noalloc: inlet faces are not supported");
    if (p->precision != TSLB_PREC_FP32) return noalloc_fail(TSLB_ERR_UNSUPPORTED, "tslb_step_noalloc: FP32 storage only");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(TSLB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(TSLB_ERR_ARG, "tslb_step_noalloc: device ordinal out of range");
    NoallocScratch* sc = nullptr;
    rc = noalloc_setup(dev, &sc);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The non-finite flag (zero when the library loads) collects every call's
    // result until tslb_noalloc_check reads and clears it.
    // a context-free view of the lattice for make_args
    tslb_ctx view;
    view.p = *p;
    view.nx = nx; view.ny = ny; view.nz = nz;
    view.n = n; view.N = field_stride;
    view.flags = sc->flags;
    view.stream = st;
    for (int f = 0; f < NF; ++f) view.scale[f] = 1.0f;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = step_tiles(nx, ny);
    const long long want = 4LL * kStepBlocksPerSM * sms;
    view.zchunk = (int)std::min<long long>(nz, std::max<long long>(8, (tiles * nz + want - 1) / want));
    StepArgs a = make_args(&view, d_in, d_out);
    if ((e = launch_step_kernel(a, p->mode, TSLB_PREC_FP32, st)) != cudaSuccess)
        return noalloc_fail(TSLB_ERR_CUDA, std::string("step kernel attribute: ") + cudaGetErrorString(e));
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_fail(TSLB_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
    return TSLB_OK;
}

extern "C" int tslb_noalloc_check(void* stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(TSLB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(TSLB_ERR_ARG, "tslb_noalloc_check: device ordinal out of range");
    NoallocScratch* sc = nullptr;
    int rc = noalloc_setup(dev, &sc);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned int h = 0;
    // a plain host word: the copy waits for the steps queued before it on the stream
    if ((e = cudaMemcpyAsync(&h, sc->flags, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return noalloc_fail(TSLB_ERR_CUDA, std::string("tslb_noalloc_check: ") + cudaGetErrorString(e));
    if (h) {
        if ((e = cudaMemsetAsync(sc->flags, 0, sizeof(unsigned int), st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return noalloc_fail(TSLB_ERR_CUDA, std::string("tslb_noalloc_check: ") + cudaGetErrorString(e));
        return noalloc_fail(TSLB_ERR_NAN, "tslb_step_noalloc: a step produced a non-finite moment");
    }
    return TSLB_OK;
}


// ---------------------------------------------------------------- z slabs
// A lattice split into z slabs, one per GPU (the reference's MPI domain
// decomposition, TSLB_2C-mpi/mpi_module.f90:2120-2258: pack, isend/irecv,
// wait, unpack).  A slab context's device array holds its own planes and
// `halo` copies of the neighbours' planes on each side that has a
// neighbour; the step kernels update the own planes only (zt0 .. zt1).  A
// step reads the moments of one plane beyond its targets and phi of `halo`
// planes beyond (colour: the gradient at the source plane; phase field: the
// normals there, from phi one plane further), so the exchange carries the
// 10 non-phi moments of the edge plane and phi of `halo` edge planes.

namespace {

int slab_halo_planes(int mode) { return mode == TSLB_MODE_PHASEFIELD ? 3 : mode == TSLB_MODE_COLOUR ? 2 : 1; }
int slab_phi_planes(const tslb_ctx* c) { return c->p.mode == TSLB_MODE_SINGLE ? 0 : c->halo; }

// buffer: [10 moment fields of one plane][nphi phi planes], storage type
template <class T>
__global__ void halo_pack_kernel(const T* __restrict__ st, long long N, long long plane, int zmom, int zphi0, int nphi,
                                 T* __restrict__ buf) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)(NMOM + nphi) * plane) return;
    const long long k = i / plane, p = i - k * plane;
    buf[i] = k < NMOM ? st[k * N + (long long)zmom * plane + p] : st[F_PHI * N + (long long)(zphi0 + k - NMOM) * plane + p];
}
template <class T>
__global__ void halo_unpack_kernel(T* __restrict__ st, long long N, long long plane, int zmom, int zphi0, int nphi,
                                   const T* __restrict__ buf) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)(NMOM + nphi) * plane) return;
    const long long k = i / plane, p = i - k * plane;
    if (k < NMOM) st[k * N + (long long)zmom * plane + p] = buf[i];
    else st[F_PHI * N + (long long)(zphi0 + k - NMOM) * plane + p] = buf[i];
}

// side 0: the slab's bottom (z-), side 1: its top (z+).  pack: the own edge
// planes the neighbour on that side needs; unpack: the halo planes there.
int halo_copy(tslb_ctx* c, int side, bool pack, void* buf) {
    if (!c) return TSLB_ERR_ARG;
    if (side != 0 && side != 1) return fail(c, TSLB_ERR_ARG, "halo: side must be 0 (z-) or 1 (z+)");
    if (!buf) return fail(c, TSLB_ERR_ARG, "halo: NULL buffer");
    if (c->halo == 0) return fail(c, TSLB_ERR_STATE, "halo: not a slab context (tslb_create_slab)");
    if (pack ? false : (side == 0 ? c->halo_lo == 0 : c->halo_hi == 0))
        return fail(c, TSLB_ERR_STATE, "halo: the slab has no neighbour on this side");
    const long long plane = (long long)c->nx * c->ny;
    const int H = c->halo, nphi = slab_phi_planes(c);
    int zmom, zphi0;
    if (pack) {
        zmom = side == 0 ? c->zt0 : c->zt1 - 1;
        zphi0 = side == 0 ? c->zt0 : c->zt1 - H;
    } else {
        zmom = side == 0 ? c->zt0 - 1 : c->zt1;
        zphi0 = side == 0 ? c->zt0 - H : c->zt1;
    }
    const long long total = (long long)(NMOM + nphi) * plane;
    const int bs = 256;
    with_storage(c->p.precision, [&](auto tag) {
        using T = decltype(tag);
        T* st = static_cast<T*>(c->state[c->cur]);
        if (pack)
            halo_pack_kernel<T><<<(unsigned)((total + bs - 1) / bs), bs, 0, c->stream>>>(st, c->N, plane, zmom, zphi0, nphi,
                                                                                        static_cast<T*>(buf));
        else
            halo_unpack_kernel<T><<<(unsigned)((total + bs - 1) / bs), bs, 0, c->stream>>>(st, c->N, plane, zmom, zphi0, nphi,
                                                                                          static_cast<const T*>(buf));
    });
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

}  // namespace

extern "C" {

int tslb_create_slab(const tslb_params* p, int nx, int ny, int nz, int z_begin, int z_end, tslb_ctx** out) {
    if (!out) return fail(nullptr, TSLB_ERR_ARG, "out is NULL");
    *out = nullptr;
    std::string why;
    int rc = validate(p, nx, ny, nz, why);
    if (rc) return fail(nullptr, rc, "tslb_create_slab: " + why);
    const int H = slab_halo_planes(p->mode);
    if (z_begin < 0 || z_end > nz || z_end - z_begin < H)
        return fail(nullptr, TSLB_ERR_ARG, "tslb_create_slab: need 0 <= z_begin, z_end <= nz and at least " +
                                               std::to_string(H) + " own planes");
    const bool zper = p->bc[4] == TSLB_BC_PERIODIC;
    const bool whole = z_begin == 0 && z_end == nz;
    const int lo = whole ? 0 : (z_begin > 0 || zper ? H : 0);
    const int hi = whole ? 0 : (z_end < nz || zper ? H : 0);
    tslb_params lp = *p;
    if (lo || hi) {
        // a side with a halo has no boundary condition of its own: the step never
        // reaches it (its faces stay non-periodic placeholders, in pairs)
        if (lo) lp.bc[4] = TSLB_BC_BOUNCEBACK;
        if (hi) lp.bc[5] = TSLB_BC_BOUNCEBACK;
        if (lp.bc[4] == TSLB_BC_PERIODIC) lp.bc[4] = TSLB_BC_BOUNCEBACK;
        if (lp.bc[5] == TSLB_BC_PERIODIC) lp.bc[5] = TSLB_BC_BOUNCEBACK;
        for (int f = 4; f < 6; ++f)
            if ((f == 4 ? lo : hi) && p->bc[f] == TSLB_BC_INLET)
                return fail(nullptr, TSLB_ERR_ARG, "tslb_create_slab: an inlet face must belong to the slab that owns it");
    }
    const int nzl = lo + (z_end - z_begin) + hi;
    tslb_ctx* c = nullptr;
    rc = tslb_create(&lp, nx, ny, nzl, &c);
    if (rc) return rc;
    c->nz_global = nz;
    c->z_begin = z_begin;
    c->halo = whole ? 0 : H;
    c->halo_lo = lo;
    c->halo_hi = hi;
    c->zt0 = lo;
    c->zt1 = lo + (z_end - z_begin);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    c->zchunk = choose_zchunk(step_tiles(nx, ny), z_end - z_begin, sms, kStepBlocksPerSM, p->mode);
    *out = c;
    return TSLB_OK;
}

int tslb_slab_geometry(const tslb_ctx* c, int out[6]) {
    if (!c || !out) return TSLB_ERR_ARG;
    out[0] = c->nz_global > 0 ? c->nz_global : c->nz;
    out[1] = c->z_begin;
    out[2] = c->z_begin + ((c->zt1 > 0 ? c->zt1 : c->nz) - c->zt0);
    out[3] = c->halo_lo;
    out[4] = c->halo_hi;
    out[5] = c->halo;
    return TSLB_OK;
}

long long tslb_halo_bytes(const tslb_ctx* c) {
    if (!c || c->halo == 0) return 0;
    return (long long)(NMOM + slab_phi_planes(c)) * c->nx * c->ny * c->esize;
}

int tslb_halo_pack(tslb_ctx* c, int side, void* d_buf) { return halo_copy(c, side, true, d_buf); }
int tslb_halo_unpack(tslb_ctx* c, int side, const void* d_buf) { return halo_copy(c, side, false, const_cast<void*>(d_buf)); }

}  // extern "C"

// ------------------------------------------------------ batched ensemble
constexpr int kEnsStepWords = 4;   // the ensemble kernel's step counter, ticket and work counter, padded

struct tslb_ensemble {
    std::vector<tslb_ctx*> m;          // member lattices (own state, own params)
    int mode = 0, precision = 0;
    bool vec = true;
    cudaStream_t stream = nullptr;
    StepArgs* d_args[2] = {nullptr, nullptr};  // per step parity: member args
    WorkItem* d_work = nullptr;
    int nwork = 0;
    int zchunk = 16;
    int grid = 0;                      // 0: one block per work item
    int sms = 148;
    int parity = 0;                    // steps taken mod 2 since the last args upload
    unsigned int* d_step = nullptr;    // {step counter of the stochastic rounding, launch ticket, work counter, 0}
    struct TuneRow { int zchunk, grid; float ms; };
    std::vector<TuneRow> tuned;        // the autotuner's timings, in the order it ran them
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    std::string err;
};

namespace {

int efail(tslb_ensemble* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    else g_create_error = msg;
    return code;
}

#define ECUDA_TRY(e, call)                                                               \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return efail(e, TSLB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void ens_drop_graph(tslb_ensemble* e) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    e->graph_steps = 0;
}

// Rebuild the work list and both parities of the member arguments for the
// current z chunk and member buffers.
int ens_build(tslb_ensemble* e) {
    std::vector<WorkItem> work;
    std::vector<StepArgs> args[2];
    for (size_t d = 0; d < e->m.size(); ++d) {
        tslb_ctx* c = e->m[d];
        c->zchunk = std::min(e->zchunk, c->nz);
        const int gx = (c->nx + TX - 1) / TX, gy = (c->ny + TY - 1) / TY, gz = (c->nz + c->zchunk - 1) / c->zchunk;
        for (int bz = 0; bz < gz; ++bz)
            for (int by = 0; by < gy; ++by)
                for (int bx = 0; bx < gx; ++bx) work.push_back(WorkItem{(int)d, bx, by, bz});
        for (int par = 0; par < 2; ++par) {
            const int cur = c->cur ^ par;
            args[par].push_back(make_args(c, c->state[cur], c->state[cur ^ 1]));
            // the ensemble replays these arguments every step (CUDA graph): the step
            // that seeds the stochastic rounding comes from the device counter
            args[par].back().sr_counter = e->d_step;
        }
    }
    // largest items first (the planes a block marches through, its z chunk plus
    // the two source planes outside it): the last items of a step are then
    // the short ones, so the SMs run out of work at about the same time
    auto planes = [&](const WorkItem& w) {
        const tslb_ctx* c = e->m[w.dom];
        return std::min(c->zchunk, c->nz - w.bz * c->zchunk) + 2;
    };
    std::stable_sort(work.begin(), work.end(), [&](const WorkItem& a, const WorkItem& b) { return planes(a) > planes(b); });
    ens_drop_graph(e);
    cudaFree(e->d_work);
    for (int par = 0; par < 2; ++par) cudaFree(e->d_args[par]);
    e->d_work = nullptr;
    e->d_args[0] = e->d_args[1] = nullptr;
    e->nwork = (int)work.size();
    ECUDA_TRY(e, cudaMalloc(&e->d_work, sizeof(WorkItem) * work.size()));
    ECUDA_TRY(e, cudaMemcpy(e->d_work, work.data(), sizeof(WorkItem) * work.size(), cudaMemcpyHostToDevice));
    for (int par = 0; par < 2; ++par) {
        ECUDA_TRY(e, cudaMalloc(&e->d_args[par], sizeof(StepArgs) * args[par].size()));
        ECUDA_TRY(e, cudaMemcpy(e->d_args[par], args[par].data(), sizeof(StepArgs) * args[par].size(), cudaMemcpyHostToDevice));
    }
    e->parity = 0;
    return TSLB_OK;
}

// The ensemble kernel of the ensemble's mode, storage and x alignment:
// sets its shared-memory attribute and (launch) launches one step.
cudaError_t ens_kernel(tslb_ensemble* e, bool launch) {
    const int grid = e->grid > 0 ? std::min(e->grid, e->nwork) : e->nwork;
    const StepArgs* args = e->d_args[e->parity];
    return tslb_launch::scalar_ensemble(args, e->d_work, e->nwork, grid, e->mode, e->precision, e->vec, e->d_step,
                                        e->stream, launch);
}

// one ensemble step on the ensemble stream (no host synchronisation)
int ens_launch(tslb_ensemble* e) {
    ECUDA_TRY(e, ens_kernel(e, true));
    ECUDA_TRY(e, cudaGetLastError());
    e->parity ^= 1;
    return TSLB_OK;
}

// fold the steps taken into the members' current buffers
void ens_settle(tslb_ensemble* e) {
    if (e->parity) {
        for (tslb_ctx* c : e->m) c->cur ^= 1;
        // arguments of parity 0 must again start from the members' current buffers
        std::swap(e->d_args[0], e->d_args[1]);
        e->parity = 0;
    }
}

int ens_check(tslb_ensemble* e, int i) {
    if (!e) return TSLB_ERR_ARG;
    if (i < 0 || i >= (int)e->m.size()) return efail(e, TSLB_ERR_ARG, "member index out of range");
    return TSLB_OK;
}

}  // namespace

extern "C" {

int tslb_ensemble_create(const tslb_params* params, const int* dims, int n, tslb_ensemble** out) {
    if (!out) return efail(nullptr, TSLB_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!params || !dims || n < 1) return efail(nullptr, TSLB_ERR_ARG, "tslb_ensemble_create: need n >= 1 members");
    for (int i = 1; i < n; ++i)
        if (params[i].mode != params[0].mode || params[i].precision != params[0].precision)
            return efail(nullptr, TSLB_ERR_ARG, "tslb_ensemble_create: members must share mode and precision");
    if (params[0].mode == TSLB_MODE_SINGLE)
        return efail(nullptr, TSLB_ERR_UNSUPPORTED, "tslb_ensemble_create: single-component members are not supported");
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < 6; ++f)
            if (params[i].bc[f] == TSLB_BC_INLET)
                return efail(nullptr, TSLB_ERR_UNSUPPORTED, "tslb_ensemble_create: inlet faces are not supported in ensembles");
    tslb_ensemble* e = new (std::nothrow) tslb_ensemble();
    if (!e) return efail(nullptr, TSLB_ERR_ARG, "out of host memory");
    e->mode = params[0].mode;
    e->precision = params[0].precision;
    for (int i = 0; i < n; ++i) {
        tslb_ctx* c = nullptr;
        int rc = tslb_create(&params[i], dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], &c);
        if (rc) {
            std::string msg = "member " + std::to_string(i) + ": " + g_create_error;
            tslb_ensemble_destroy(e);
            return efail(nullptr, rc, msg);
        }
        e->m.push_back(c);
        const int epc = 16 / storage_bytes(e->precision);
        if (dims[3 * i] % epc) e->vec = false;
    }
    cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    // step counter of the stochastic rounding (members start at step 0) and launch ticket
    if (ce == cudaSuccess) ce = cudaMalloc(&e->d_step, kEnsStepWords * sizeof(unsigned int));
    if (ce == cudaSuccess) ce = cudaMemset(e->d_step, 0, kEnsStepWords * sizeof(unsigned int));
    if (ce == cudaSuccess) ce = ens_kernel(e, false);
    int dev = 0;
    if (ce == cudaSuccess) ce = cudaGetDevice(&dev);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, dev);
    if (ce != cudaSuccess) {
        std::string msg = std::string("tslb_ensemble_create: ") + cudaGetErrorString(ce);
        tslb_ensemble_destroy(e);
        return efail(nullptr, TSLB_ERR_CUDA, msg);
    }
    e->grid = kStepBlocksPerSM * e->sms;  // persistent: the resident blocks walk the work list
    int rc = ens_build(e);
    if (rc) {
        std::string msg = e->err;
        tslb_ensemble_destroy(e);
        return efail(nullptr, rc, msg);
    }
    *out = e;
    return TSLB_OK;
}

void tslb_ensemble_destroy(tslb_ensemble* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    ens_drop_graph(e);
    cudaFree(e->d_work);
    for (int par = 0; par < 2; ++par) cudaFree(e->d_args[par]);
    cudaFree(e->d_step);
    for (tslb_ctx* c : e->m) tslb_destroy(c);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int tslb_ensemble_upload_moments(tslb_ensemble* e, int i, const float* rho, const float* u, const float* v,
                                 const float* w, const float* pxx, const float* pxy, const float* pxz,
                                 const float* pyy, const float* pyz, const float* pzz, const float* phi) {
    int rc = ens_check(e, i);
    if (rc) return rc;
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    rc = tslb_upload_moments(e->m[i], rho, u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi);
    if (rc) return efail(e, rc, e->m[i]->err);
    // fp16 scales may have changed: refresh the member arguments
    return ens_build(e);
}

int tslb_ensemble_step(tslb_ensemble* e, int nsteps) {
    if (!e) return TSLB_ERR_ARG;
    if (nsteps < 0) return efail(e, TSLB_ERR_ARG, "nsteps < 0");
    for (tslb_ctx* c : e->m)
        if (!c->loaded) return efail(e, TSLB_ERR_STATE, "tslb_ensemble_step before every member is uploaded");
    for (int s = 0; s < nsteps; ++s) {
        int rc = ens_launch(e);
        if (rc) return rc;
    }
    return TSLB_OK;
}

int tslb_ensemble_step_graph(tslb_ensemble* e, int nsteps) {
    if (!e) return TSLB_ERR_ARG;
    if (nsteps < 1) return efail(e, TSLB_ERR_ARG, "nsteps < 1");
    for (tslb_ctx* c : e->m)
        if (!c->loaded) return efail(e, TSLB_ERR_STATE, "tslb_ensemble_step_graph before every member is uploaded");
    if (!e->graph || e->graph_steps != nsteps || e->parity != 0) {
        ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
        ens_settle(e);
        ens_drop_graph(e);
        cudaGraph_t g = nullptr;
        ECUDA_TRY(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        int rc = TSLB_OK;
        for (int s = 0; s < nsteps && rc == TSLB_OK; ++s) rc = ens_launch(e);
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        e->parity = 0;  // capture records launches; they have not run
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (ce != cudaSuccess) return efail(e, TSLB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return efail(e, TSLB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce));
        e->graph_steps = nsteps;
    }
    ECUDA_TRY(e, cudaGraphLaunch(e->graph, e->stream));
    // the graph starts and ends on parity 0 only for even nsteps
    if (nsteps % 2) {
        ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
        for (tslb_ctx* c : e->m) c->cur ^= 1;
        std::swap(e->d_args[0], e->d_args[1]);
        ens_drop_graph(e);
    }
    return TSLB_OK;
}

int tslb_ensemble_download_moments(tslb_ensemble* e, int i, float* rho, float* u, float* v, float* w, float* pxx,
                                   float* pxy, float* pxz, float* pyy, float* pyz, float* pzz, float* phi) {
    int rc = ens_check(e, i);
    if (rc) return rc;
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    rc = tslb_download_moments(e->m[i], rho, u, v, w, pxx, pxy, pxz, pyy, pyz, pzz, phi);
    if (rc) return efail(e, rc, e->m[i]->err);
    return TSLB_OK;
}

int tslb_ensemble_reduce(tslb_ensemble* e, int i, double out[TSLB_NREDUCE]) {
    int rc = ens_check(e, i);
    if (rc) return rc;
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    rc = tslb_reduce(e->m[i], out);
    if (rc) return efail(e, rc, e->m[i]->err);
    return TSLB_OK;
}

int tslb_ensemble_tune(tslb_ensemble* e, int* zchunk_out, int* grid_out) {
    if (!e) return TSLB_ERR_ARG;
    for (tslb_ctx* c : e->m)
        if (!c->loaded) return efail(e, TSLB_ERR_STATE, "tslb_ensemble_tune before every member is uploaded");
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    // back up every member's current state; tuning steps run on it and it is restored
    std::vector<void*> backup(e->m.size(), nullptr);
    auto release = [&]() { for (void* b : backup) cudaFree(b); };
    for (size_t d = 0; d < e->m.size(); ++d) {
        tslb_ctx* c = e->m[d];
        const size_t bytes = (size_t)c->esize * NF * c->N;
        cudaError_t ce = cudaMalloc(&backup[d], bytes);
        if (ce == cudaSuccess) ce = cudaMemcpy(backup[d], c->state[c->cur], bytes, cudaMemcpyDeviceToDevice);
        if (ce != cudaSuccess) { release(); return efail(e, TSLB_ERR_CUDA, std::string("tune backup: ") + cudaGetErrorString(ce)); }
    }
    // and the rounding's step counter, which the tuning steps advance
    unsigned int step_backup[kEnsStepWords] = {0, 0, 0, 0};
    {
        cudaError_t ce = cudaMemcpy(step_backup, e->d_step, sizeof(step_backup), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) { release(); return efail(e, TSLB_ERR_CUDA, std::string("tune backup: ") + cudaGetErrorString(ce)); }
    }
    // the persistent kernel: two or one resident blocks per SM taking the work
    // items as they finish (one block per item, grid 0, is a tslb_ensemble_set_launch choice)
    const int zcands[] = {8, 16, 32, 64, 128, 1 << 20};
    const int gcands[] = {kStepBlocksPerSM * e->sms, e->sms};
    float best = 1e30f;
    int bz = e->zchunk, bg = e->grid;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    int rc = TSLB_OK;
    e->tuned.clear();
    for (int zc : zcands) {
        for (int gr : gcands) {
            e->zchunk = zc;
            e->grid = gr;
            rc = ens_build(e);
            if (rc) break;
            const int reps = 10;
            rc = ens_launch(e);  // warm-up
            cudaEventRecord(t0, e->stream);
            for (int r = 0; r < reps && rc == TSLB_OK; ++r) rc = ens_launch(e);
            cudaEventRecord(t1, e->stream);
            cudaError_t ce = cudaEventSynchronize(t1);
            if (rc == TSLB_OK && ce != cudaSuccess) rc = efail(e, TSLB_ERR_CUDA, std::string("tune: ") + cudaGetErrorString(ce));
            if (rc) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            e->tuned.push_back({zc, gr, ms / reps});
            if (ms < best) { best = ms; bz = zc; bg = gr; }
            // keep the members' buffers consistent with their cur index
            ens_settle(e);
        }
        if (rc) break;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    // restore the uploaded state
    for (size_t d = 0; d < e->m.size() && rc == TSLB_OK; ++d) {
        tslb_ctx* c = e->m[d];
        cudaError_t ce = cudaMemcpy(c->state[c->cur], backup[d], (size_t)c->esize * NF * c->N, cudaMemcpyDeviceToDevice);
        if (ce != cudaSuccess) rc = efail(e, TSLB_ERR_CUDA, std::string("tune restore: ") + cudaGetErrorString(ce));
    }
    if (rc == TSLB_OK) {
        cudaError_t ce = cudaMemcpy(e->d_step, step_backup, sizeof(step_backup), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) rc = efail(e, TSLB_ERR_CUDA, std::string("tune restore: ") + cudaGetErrorString(ce));
    }
    release();
    if (rc) return rc;
    e->zchunk = bz;
    e->grid = bg;
    rc = ens_build(e);
    if (rc) return rc;
    if (zchunk_out) *zchunk_out = bz;
    if (grid_out) *grid_out = bg;
    return TSLB_OK;
}

int tslb_ensemble_tune_results(tslb_ensemble* e, int max, int* count, int* zchunk, int* grid, float* ms_per_step) {
    if (!e || !count || max < 0) return TSLB_ERR_ARG;
    const int n = (int)e->tuned.size();
    *count = n;
    for (int i = 0; i < n && i < max; ++i) {
        if (zchunk) zchunk[i] = e->tuned[i].zchunk;
        if (grid) grid[i] = e->tuned[i].grid;
        if (ms_per_step) ms_per_step[i] = e->tuned[i].ms;
    }
    return TSLB_OK;
}

int tslb_ensemble_set_launch(tslb_ensemble* e, int zchunk, int grid) {
    if (!e) return TSLB_ERR_ARG;
    if (zchunk < 1 || grid < 0) return efail(e, TSLB_ERR_ARG, "tslb_ensemble_set_launch: need zchunk >= 1 and grid >= 0");
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    e->zchunk = zchunk;
    e->grid = grid;
    return ens_build(e);
}

int tslb_ensemble_synchronize(tslb_ensemble* e) {
    if (!e) return TSLB_ERR_ARG;
    ECUDA_TRY(e, cudaStreamSynchronize(e->stream));
    ens_settle(e);
    for (tslb_ctx* c : e->m) {
        int rc = check_flags(c);
        if (rc) return efail(e, rc, c->err);
    }
    return TSLB_OK;
}

void* tslb_ensemble_stream(tslb_ensemble* e) { return e ? (void*)e->stream : nullptr; }

const char* tslb_ensemble_last_error(tslb_ensemble* e) {
    if (!e) return g_create_error.c_str();
    return e->err.c_str();
}

}  // extern "C"
