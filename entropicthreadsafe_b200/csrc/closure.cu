// closure.cu -- learned eddy-viscosity closure (include/tslb_closure.h):
// tensor-core inference on a lattice, tensor-core training (forward +
// backward, Adam), the fine-to-coarse training-set filter.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/tslb_closure.h"
#include "closure_mlp.cuh"
#include "tslb_internal.h"

using namespace clo;
using tslb::F_PHI;
using tslb::F_U;
using tslb::F_V;
using tslb::F_W;
using tslb::F_XX;

struct tslb_closure {
    int device = 0;
    int sms = 148;
    int infer_per_sm = 1, train_per_sm = 1;   // resident CTAs per SM (occupancy API)
    cudaStream_t stream = nullptr;
    float* params = nullptr;   // FP32 master, NPARAM_PAD
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    Image* img = nullptr;
    float* partial = nullptr;  // max_ctas * PSTRIDE
    int max_ctas = 0;
    float* loss_dev = nullptr;
    int loss_cap = 0;
    unsigned int* flags = nullptr;
    float mu[NFEAT], sd[NFEAT], dtau_max = 0.01f, dtau_min = 0.f;
    long long adam_t = 0;
    // training set
    float* ds_feat = nullptr;
    float* ds_tgt = nullptr;
    float* ds_wgt = nullptr;
    long long ds_n = 0, ds_cap = 0;
    int fine_adds = 0;
    std::string err;
};

// message of this thread's last failed tslb_closure_create (per thread)
static thread_local std::string g_closure_create_error;

namespace {

constexpr int TRAIN_SMEM = 104 * 1024;   // caps residency at 2 CTAs/SM (256 TMEM columns each)
constexpr int OFF_ACT = IMG_BYTES, OFF_DZ = IMG_BYTES + ACT_BYTES;
constexpr int OFF_MISC_TRAIN = OFF_DZ + DZ_BYTES, OFF_MISC_INFER = OFF_ACT + Act<NCH_INFER>::BYTES;
// image + 10-chunk ACT + barrier words: at most 7 CTAs/SM (64 TMEM columns each)
constexpr int INFER_SMEM = OFF_MISC_INFER + 64;
static_assert(OFF_MISC_TRAIN + 2048 + 32 * 1024 <= TRAIN_SMEM, "training tail space");
static_assert(8 * (INFER_SMEM + 1024) > 228 * 1024 && 7 * 64 <= 512, "inference residency vs TMEM columns");

int cfail(tslb_closure* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_closure_create_error = msg;
    return code;
}

#define CL_TRY(c, call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return cfail(c, TSLB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------ kernels
// master parameters -> the kernels' image (BF16 weights in the core-matrix layout)
__global__ void image_kernel(const float* __restrict__ params, Image* img) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    const float v = params[p];
    __nv_bfloat16* w1 = reinterpret_cast<__nv_bfloat16*>(img->w1);
    __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(img->w2);
    if (p < P_B1) {
        const int n = p / KIN, k = p % KIN;
        if (k != NFEAT) w1[w1_chunk(n, k >> 3) * 8 + (k & 7)] = __float2bfloat16_rn(k < NFEAT ? v : 0.f);
    } else if (p < P_W2) {
        img->b1[p - P_B1] = v;
        w1[w1_chunk(p - P_B1, 1) * 8 + (NFEAT & 7)] = __float2bfloat16_rn(v);   // bias column
    } else if (p < P_B2) {
        const int n = (p - P_W2) / NH, k = (p - P_W2) % NH;
        w2[w2_chunk(n, k >> 3) * 8 + (k & 7)] = __float2bfloat16_rn(v);
    } else if (p < P_W3) {
        img->b2[p - P_B2] = v;
    } else if (p < P_B3) {
        img->w3[p - P_W3] = __bfloat162float(__float2bfloat16_rn(v));
    } else {
        img->b3 = v;
    }
}

// Shared-memory prologue of the MLP kernels: image copy, mbarrier, TMEM.
struct Smem {
    Image* im;
    uint4* act;
    uint4* dz;
    uint64_t* bar;
    uint32_t* tslot;
    int* abort_s;
    float* red;
};

__device__ __forceinline__ Smem smem_setup(uint8_t* sm, const Image* gimg, int off_misc, bool train, uint32_t ncols) {
    Smem S;
    S.im = reinterpret_cast<Image*>(sm);
    S.act = reinterpret_cast<uint4*>(sm + OFF_ACT);
    S.dz = reinterpret_cast<uint4*>(sm + OFF_DZ);
    S.bar = reinterpret_cast<uint64_t*>(sm + off_misc);
    S.tslot = reinterpret_cast<uint32_t*>(sm + off_misc + 8);
    S.abort_s = reinterpret_cast<int*>(sm + off_misc + 12);
    S.red = reinterpret_cast<float*>(sm + off_misc + 64);
    const int tid = threadIdx.x;
    const uint4* src = reinterpret_cast<const uint4*>(gimg);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (int i = tid; i < (int)(sizeof(Image) / 16); i += blockDim.x) dst[i] = src[i];
    if (train) {
        // constant chunks of ACT: a 1 in the first column of chunk 10, zeros in chunk 11
        const float one[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        S.act[act_chunk(tid, 10)] = pack8(one);
        S.act[act_chunk(tid, 11)] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid == 0) {
        tc::mbar_init(S.bar, 1);
        *S.abort_s = 0;
    }
    if ((tid >> 5) == 0) tc::tmem_alloc(S.tslot, ncols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    return S;
}

// Free the TMEM after all threads' accesses; after a timeout first give the
// MMAs in flight another bounded wait.
__device__ __forceinline__ void smem_teardown(const Smem& S, uint32_t tb, uint32_t ncols, uint32_t ph) {
    if (*S.abort_s && threadIdx.x == 0) tc::mbar_wait_bounded(S.bar, ph, 4000000000LL);
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_free(tb, ncols);
    }
}

// feature rows from a device array
struct ArraySrc {
    const float* feat;
    float* out;
    long long n;
    struct Raw {
        float f[NFEAT];
    };
    __device__ void load(long long i, Raw& r) const {
        if (i >= n) return;
#pragma unroll
        for (int k = 0; k < NFEAT; ++k) r.f[k] = feat[i * NFEAT + k];
    }
    __device__ bool features(const Raw& r, long long, float* f) const {
        bool ok = true;
#pragma unroll
        for (int k = 0; k < NFEAT; ++k) {
            f[k] = r.f[k];
            ok = ok && isfinite(f[k]);
        }
        return ok;
    }
    __device__ float keep(const Raw&) const { return 0.f; }
    __device__ void store(long long i, float y, float) const { out[i] = y; }
};

// features of lattice node i from the FP32 moment state; dtau is read (the
// previous correction) and rewritten by the same thread
struct LatticeSrc {
    const float* st;
    long long N, n;
    int nx, ny, nz;
    int px, py, pz;
    float inv_nu_a, inv_nu_b;
    float* dtau;         // total correction of the previous refresh, rewritten (null: none)
    const float* base;   // static correction (tslb_set_tau_correction) or null
    Divider dx, dy;      // division by nx, ny
    struct Raw {
        float P[6], phi, u, v, w, ph[6], dprev, dbase;
    };
    __device__ float phi_at(int x, int y, int z) const {
        return st[F_PHI * N + x + (long long)nx * (y + (long long)ny * z)];
    }
    __device__ void load(long long i, Raw& r) const {
        if (i >= n) return;
        int x, y, z;
        if (n < (1LL << 31)) {
            const int ii = (int)i, q = dx.div(ii);
            x = ii - q * nx;
            z = dy.div(q);
            y = q - z * ny;
        } else {
            x = (int)(i % nx); y = (int)((i / nx) % ny); z = (int)(i / ((long long)nx * ny));
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) r.P[k] = st[(F_XX + k) * N + i];
        r.phi = st[F_PHI * N + i];
        r.u = st[F_U * N + i]; r.v = st[F_V * N + i]; r.w = st[F_W * N + i];
        r.ph[0] = phi_at(nbr(x, 1, nx, px), y, z);
        r.ph[1] = phi_at(nbr(x, -1, nx, px), y, z);
        r.ph[2] = phi_at(x, nbr(y, 1, ny, py), z);
        r.ph[3] = phi_at(x, nbr(y, -1, ny, py), z);
        r.ph[4] = phi_at(x, y, nbr(z, 1, nz, pz));
        r.ph[5] = phi_at(x, y, nbr(z, -1, nz, pz));
        r.dprev = dtau ? dtau[i] : 0.f;
        r.dbase = base ? base[i] : 0.f;
    }
    __device__ bool features(const Raw& r, long long, float* f) const {
        const float gx = 0.5f * (r.ph[0] - r.ph[1]), gy = 0.5f * (r.ph[2] - r.ph[3]), gz = 0.5f * (r.ph[4] - r.ph[5]);
        // plain tau of the node's mixture: 1/omega = (6 + q)/(2q), and
        // s = tau / (tau + dprev) = (6 + q) / (6 + q + 2 q dprev)
        const float q = 0.5f * ((inv_nu_a + inv_nu_b) + r.phi * (inv_nu_a - inv_nu_b));
        const float s = (6.f + q) / fmaf(2.f * q, r.dprev, 6.f + q);
        make_features(s, r.P, r.phi, sqrtf(gx * gx + gy * gy + gz * gz), sqrtf(r.u * r.u + r.v * r.v + r.w * r.w), f);
        bool ok = true;
#pragma unroll
        for (int k = 0; k < NFEAT; ++k) ok = ok && isfinite(f[k]);
        return ok;
    }
    // the static correction, read with the inputs so the store waits on nothing
    __device__ float keep(const Raw& r) const { return r.dbase; }
    __device__ void store(long long i, float y, float b) const { dtau[i] = y + b; }
};

// Inference: dtau = dtau_min + (dtau_max - dtau_min) sigmoid(o) for every row of the source, 128
// rows per tile, tiles strided over a persistent grid.  The next tile's
// inputs are loaded while this tile's MMAs run; both layers accumulate in
// the same 64 TMEM columns, so up to 7 CTAs share an SM.
template <class Src>
__global__ void __launch_bounds__(TILE, 6) infer_kernel(const Image* __restrict__ gimg, Src src, long long n,
                                                        unsigned int* gflag) {
    extern __shared__ __align__(1024) uint8_t sm[];
    Smem S = smem_setup(sm, gimg, OFF_MISC_INFER, false, 64);
    const uint32_t tb = *S.tslot;
    const Image& im = *S.im;
    const int tid = threadIdx.x;
    const uint32_t act_a = tc::smem_u32(S.act), w1_a = tc::smem_u32(im.w1), w2_a = tc::smem_u32(im.w2);
    uint32_t ph = 0;
    const long long ntiles = (n + TILE - 1) / TILE;
    typename Src::Raw raw;
    if ((long long)blockIdx.x < ntiles) src.load((long long)blockIdx.x * TILE + tid, raw);
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long i = t * TILE + tid;
        const bool valid = i < n;
        float f[NFEAT];
        const bool fin = valid && src.features(raw, i, f);
        const float kept = src.keep(raw);
        if (t + gridDim.x < ntiles) src.load((t + gridDim.x) * TILE + tid, raw);
        put_x<NCH_INFER>(S.act, tid, f, im, fin);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_fwd1<NCH_INFER>(tb, act_a, w1_a, 0);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, gflag)) break;
        epi_h1<NCH_INFER, false>(tb, S.act, tid, 0);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_fwd2<NCH_INFER>(tb, act_a, w2_a, 0);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, gflag)) break;
        const float o = epi_out(tb, im, 0);
        float y = im.dtau_min + (im.dtau_max - im.dtau_min) / (1.f + expf(-o));
        // stability clamp: the plain tau where anything is not finite
        if (!fin || !isfinite(y)) y = 0.f;
        y = fminf(fmaxf(y, im.dtau_min), im.dtau_max);
        if (valid) src.store(i, y, kept);
    }
    smem_teardown(S, tb, 64, ph);
}

struct TrainArgs {
    const Image* img;
    const float* feat;
    const float* tgt;
    const float* wgt;
    long long ndata;    // rows of the sample arrays
    long long nrows;    // rows of this batch
    int random;         // 1: row slot -> hash-drawn sample; 0: row slot = sample
    unsigned long long seed;
    int step;
    float inv_batch;
    float* partial;     // [gridDim.x][PSTRIDE]
    unsigned int* flags;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Forward + backward of the batch; each CTA writes its partial gradient
// (summed over its tiles in tensor memory) and loss to a.partial.
__global__ void __launch_bounds__(TILE, 1) train_kernel(const TrainArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    Smem S = smem_setup(sm, a.img, OFF_MISC_TRAIN, true, 256);
    const uint32_t tb = *S.tslot;
    const Image& im = *S.im;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t act_a = tc::smem_u32(S.act), dz_a = tc::smem_u32(S.dz);
    const uint32_t w1_a = tc::smem_u32(im.w1), w2_a = tc::smem_u32(im.w2);
    uint32_t ph = 0;
    float dw3[NH];
#pragma unroll
    for (int j = 0; j < NH; ++j) dw3[j] = 0.f;
    float db3 = 0.f, lsum = 0.f;
    bool first = true;
    const long long ntiles = (a.nrows + TILE - 1) / TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long slot = t * TILE + tid;
        const bool valid = slot < a.nrows;
        long long idx = slot;
        if (a.random)
            idx = (long long)(mix64(a.seed * 0x100000001B3ull ^ ((unsigned long long)a.step << 40) ^ (unsigned long long)slot) %
                              (unsigned long long)a.ndata);
        float f[NFEAT], tg = 0.f, wg = 0.f;
#pragma unroll
        for (int k = 0; k < NFEAT; ++k) f[k] = valid ? a.feat[idx * NFEAT + k] : 0.f;
        if (valid) { tg = a.tgt[idx]; wg = a.wgt[idx]; }
        put_x(S.act, tid, f, im, valid);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_fwd1(tb, act_a, w1_a);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, a.flags)) break;
        const uint64_t m1 = epi_h1<NCH_TRAIN, true>(tb, S.act, tid, COL_Z1);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_fwd2(tb, act_a, w2_a);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, a.flags)) break;
        const float o = epi_out(tb, im);
        const float sg = 1.f / (1.f + expf(-o));
        const float y = im.dtau_min + (im.dtau_max - im.dtau_min) * sg;
        const float r = valid ? y - tg : 0.f;
        lsum = fmaf(a.inv_batch * wg * r, r, lsum);
        // dL/do = 2/B a (y - t) dy/do, dy/do = (dtau_max - dtau_min) sigmoid (1 - sigmoid)
        const float g = valid ? 2.f * a.inv_batch * wg * r * (y - im.dtau_min) * (1.f - sg) : 0.f;
        db3 += g;
        epi_dz2(tb, S.dz, tid, im, g, dw3);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_bwd_dh1(tb, dz_a, w2_a);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, a.flags)) break;
        epi_dz1(tb, S.dz, tid, m1);
        sync_for_mma();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_bwd_dw(tb, dz_a, act_a, first);
            tc::mma_commit(S.bar);
        }
        if (!wait_mma(S.bar, ph, S.abort_s, a.flags)) break;
        first = false;
    }
    float* part = a.partial + (size_t)blockIdx.x * PSTRIDE;
    // weight and bias gradients of the two hidden layers from tensor memory
    const int row = 32 * warp + lane;
    const bool have = !first && *S.abort_s == 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        float d[32];
        if (have) tc::tmem_ld32(lane_addr(tb, COL_DW + 32 * q), d);
        else {
#pragma unroll
            for (int j = 0; j < 32; ++j) d[j] = 0.f;
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int col = 32 * q + j;
            if (row < NH) {
                if (col < NH) part[P_W2 + row * NH + col] = d[j];
                else if (col == 80) part[P_B2 + row] = d[j];
            } else {
                const int u = row - NH;
                if (col >= 64 && col < 80) part[P_W1 + u * KIN + (col - 64)] = d[j];
                else if (col == 80) part[P_B1 + u] = d[j];
            }
        }
    }
    // output-layer gradient and loss: block sums
#pragma unroll
    for (int j = 0; j < NH + 2; ++j) {
        float v = j < NH ? dw3[j] : (j == NH ? db3 : lsum);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) S.red[warp * (NH + 2) + j] = v;
    }
    __syncthreads();
    if (tid < NH + 2) {
        const float v = S.red[tid] + S.red[(NH + 2) + tid] + S.red[2 * (NH + 2) + tid] + S.red[3 * (NH + 2) + tid];
        part[tid < NH ? P_W3 + tid : (tid == NH ? P_B3 : NPARAM_PAD)] = v;
    }
    smem_teardown(S, tb, 256, ph);
}

// Sum the CTAs' partials in a fixed order; gradient mode writes the
// gradient, training mode takes one Adam step on the master parameters and
// rewrites their image.
struct AdamArgs {
    const float* partial;
    int nctas;
    float* params;
    float* m;
    float* v;
    Image* img;
    float lr, b1, b2, eps;
    float bc1, bc2;       // 1 - b1^t, 1 - b2^t
    float* grad_out;      // gradient mode when non-null
    float* loss_out;
};
__global__ void adam_kernel(const AdamArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && a.loss_out) {
        float l = 0.f;
        for (int c = 0; c < a.nctas; ++c) l += a.partial[(size_t)c * PSTRIDE + NPARAM_PAD];
        *a.loss_out = l;
    }
    if (p >= NPARAM) return;
    float g = 0.f;
    for (int c = 0; c < a.nctas; ++c) g += a.partial[(size_t)c * PSTRIDE + p];
    if (p < P_B1 && (p % KIN) >= NFEAT) g = 0.f;   // padding inputs
    if (a.grad_out) {
        a.grad_out[p] = g;
        return;
    }
    const float m = a.b1 * a.m[p] + (1.f - a.b1) * g;
    const float v = a.b2 * a.v[p] + (1.f - a.b2) * g * g;
    a.m[p] = m;
    a.v[p] = v;
    float w = a.params[p] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
    if (p < P_B1 && (p % KIN) >= NFEAT) w = 0.f;
    a.params[p] = w;
    __nv_bfloat16* w1 = reinterpret_cast<__nv_bfloat16*>(a.img->w1);
    __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(a.img->w2);
    if (p < P_B1) {
        const int n = p / KIN, k = p % KIN;
        if (k != NFEAT) w1[w1_chunk(n, k >> 3) * 8 + (k & 7)] = __float2bfloat16_rn(w);
    } else if (p < P_W2) {
        a.img->b1[p - P_B1] = w;
        w1[w1_chunk(p - P_B1, 1) * 8 + (NFEAT & 7)] = __float2bfloat16_rn(w);   // bias column
    } else if (p < P_B2) {
        const int n = (p - P_W2) / NH, k = (p - P_W2) % NH;
        w2[w2_chunk(n, k >> 3) * 8 + (k & 7)] = __float2bfloat16_rn(w);
    } else if (p < P_W3) {
        a.img->b2[p - P_B2] = w;
    } else if (p < P_B3) {
        a.img->w3[p - P_W3] = __bfloat162float(__float2bfloat16_rn(w));
    } else {
        a.img->b3 = w;
    }
}

// ---- training set from a fine lattice ----
// block means over 2x2x2 fine nodes: u, v, w, phi, pi_scale * Pi (6),
// uu, uv, uw, vv, vw, ww -> inter[k * nc + J]
constexpr int NINTER = 16;
__global__ void coarsen_kernel(const float* __restrict__ st, long long N, int nxf, int nyf, int nzf, float pi_scale,
                               float* __restrict__ inter) {
    const int cx = nxf / 2, cy = nyf / 2, cz = nzf / 2;
    const long long nc = (long long)cx * cy * cz;
    const long long J = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (J >= nc) return;
    const int X = (int)(J % cx), Y = (int)((J / cx) % cy), Z = (int)(J / ((long long)cx * cy));
    float s[NINTER];
#pragma unroll
    for (int k = 0; k < NINTER; ++k) s[k] = 0.f;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const long long i = (2 * X + dx) + (long long)nxf * ((2 * Y + dy) + (long long)nyf * (2 * Z + dz));
                const float u = st[F_U * N + i], v = st[F_V * N + i], w = st[F_W * N + i];
                s[0] += u; s[1] += v; s[2] += w;
                s[3] += st[F_PHI * N + i];
#pragma unroll
                for (int k = 0; k < 6; ++k) s[4 + k] += st[(F_XX + k) * N + i];
                s[10] += u * u; s[11] += u * v; s[12] += u * w;
                s[13] += v * v; s[14] += v * w; s[15] += w * w;
            }
#pragma unroll
    for (int k = 0; k < NINTER; ++k) inter[k * nc + J] = s[k] * (k >= 4 && k < 10 ? 0.125f * pi_scale : 0.125f);
}

// samples of the coarse nodes J = phase (mod keep): features, target
// t = 3 nu_t = -3 (tau_dev : S)/(2 S : S) and weight a = S : S (0 on
// non-periodic boundary planes, where the differences are one-sided)
__global__ void samples_kernel(const float* __restrict__ inter, int cx, int cy, int cz, int px, int py, int pz, int keep,
                               long long J0, long long J1, long long base, float* __restrict__ feat,
                               float* __restrict__ tgt, float* __restrict__ wgt) {
    const long long nc = (long long)cx * cy * cz;
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long J = J0 + r * keep;
    if (J >= J1) return;
    const int X = (int)(J % cx), Y = (int)((J / cx) % cy), Z = (int)(J / ((long long)cx * cy));
    auto at = [&](int k, int x, int y, int z) { return inter[k * nc + x + (long long)cx * (y + (long long)cy * z)]; };
    const int xp = nbr(X, 1, cx, px), xm = nbr(X, -1, cx, px);
    const int yp = nbr(Y, 1, cy, py), ym = nbr(Y, -1, cy, py);
    const int zp = nbr(Z, 1, cz, pz), zm = nbr(Z, -1, cz, pz);
    float G[3][3];   // G[a][b] = d u_b / d x_a
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        G[0][b] = 0.5f * (at(b, xp, Y, Z) - at(b, xm, Y, Z));
        G[1][b] = 0.5f * (at(b, X, yp, Z) - at(b, X, ym, Z));
        G[2][b] = 0.5f * (at(b, X, Y, zp) - at(b, X, Y, zm));
    }
    const float gx = 0.5f * (at(3, xp, Y, Z) - at(3, xm, Y, Z));
    const float gy = 0.5f * (at(3, X, yp, Z) - at(3, X, ym, Z));
    const float gz = 0.5f * (at(3, X, Y, zp) - at(3, X, Y, zm));
    const float u = at(0, X, Y, Z), v = at(1, X, Y, Z), w = at(2, X, Y, Z);
    float P[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) P[k] = at(4 + k, X, Y, Z);
    float f[NFEAT];
    make_features(1.f, P, at(3, X, Y, Z), sqrtf(gx * gx + gy * gy + gz * gz), sqrtf(u * u + v * v + w * w), f);
    // strain rate and subgrid stress, components (xx, xy, xz, yy, yz, zz)
    const float S6[6] = {G[0][0], 0.5f * (G[0][1] + G[1][0]), 0.5f * (G[0][2] + G[2][0]),
                         G[1][1], 0.5f * (G[1][2] + G[2][1]), G[2][2]};
    float T6[6] = {at(10, X, Y, Z) - u * u, at(11, X, Y, Z) - u * v, at(12, X, Y, Z) - u * w,
                   at(13, X, Y, Z) - v * v, at(14, X, Y, Z) - v * w, at(15, X, Y, Z) - w * w};
    const float tr = (T6[0] + T6[3] + T6[5]) * (1.f / 3.f);
    T6[0] -= tr; T6[3] -= tr; T6[5] -= tr;
    const float SS = S6[0] * S6[0] + S6[3] * S6[3] + S6[5] * S6[5] + 2.f * (S6[1] * S6[1] + S6[2] * S6[2] + S6[4] * S6[4]);
    const float TS = T6[0] * S6[0] + T6[3] * S6[3] + T6[5] * S6[5] + 2.f * (T6[1] * S6[1] + T6[2] * S6[2] + T6[4] * S6[4]);
    const bool edge = (!px && (X == 0 || X == cx - 1)) || (!py && (Y == 0 || Y == cy - 1)) || (!pz && (Z == 0 || Z == cz - 1));
    const bool ok = SS > 1e-30f && !edge;
    const long long o = base + r;
#pragma unroll
    for (int k = 0; k < NFEAT; ++k) feat[o * NFEAT + k] = f[k];
    tgt[o] = ok ? -3.f * TS / (2.f * SS) : 0.f;
    wgt[o] = ok ? SS : 0.f;
}

// per-block FP64 sums of f_k, f_k^2 (k < 10) and the weight
constexpr int NSUM = 2 * NFEAT + 1;
__global__ void norm_partial_kernel(const float* __restrict__ feat, const float* __restrict__ wgt, long long n,
                                    double* __restrict__ part) {
    __shared__ double sh[NSUM][8];
    double acc[NSUM];
    for (int k = 0; k < NSUM; ++k) acc[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        for (int k = 0; k < NFEAT; ++k) {
            const double x = feat[i * NFEAT + k];
            acc[k] += x;
            acc[NFEAT + k] += x * x;
        }
        acc[2 * NFEAT] += wgt[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < NSUM; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NSUM) {
        double t = 0.0;
        for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) t += sh[threadIdx.x][w8];
        part[blockIdx.x * NSUM + threadIdx.x] = t;
    }
}

__global__ void scale_kernel(float* x, long long n, float s) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) x[i] *= s;
}

__global__ void features_kernel(LatticeSrc src, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= src.n) return;
    float f[NFEAT];
    LatticeSrc::Raw r;
    src.load(i, r);
    src.features(r, i, f);
#pragma unroll
    for (int k = 0; k < NFEAT; ++k) out[i * NFEAT + k] = f[k];
}

// ------------------------------------------------------------ host helpers
cudaError_t set_attributes() {
    const cudaFuncAttribute dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    const cudaFuncAttribute carve = cudaFuncAttributePreferredSharedMemoryCarveout;
    cudaError_t e = cudaFuncSetAttribute(train_kernel, dyn, TRAIN_SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(infer_kernel<ArraySrc>, dyn, INFER_SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(infer_kernel<LatticeSrc>, dyn, INFER_SMEM);
    // all of the unified L1/shared storage as shared memory, so residency is set by the
    // kernels' shared memory and registers (and the occupancy query agrees with the launch)
    if (e == cudaSuccess) e = cudaFuncSetAttribute(train_kernel, carve, (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(infer_kernel<ArraySrc>, carve, (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(infer_kernel<LatticeSrc>, carve, (int)cudaSharedmemCarveoutMaxShared);
    return e;
}

// CTAs of TILE threads that fit on one SM by registers (allocated per warp
// in units of 8 per thread), shared memory (plus the per-block reserve) and
// threads.  The runtime's occupancy query under-reports for these kernels.
cudaError_t resident_ctas(int dev, const void* fn, int smem, int* out) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    int regs_sm = 65536, smem_sm = 233472, reserve = 1024, thr_sm = 2048;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserve, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    const int regs_warp = ((fa.numRegs + 7) / 8) * 8 * 32;
    const int warps = TILE / 32;
    int n = regs_sm / (regs_warp * warps);
    n = std::min(n, smem_sm / (smem + (int)fa.sharedSizeBytes + reserve));
    n = std::min(n, thr_sm / TILE);
    *out = std::max(n, 1);
    return cudaSuccess;
}

int upload_meta(tslb_closure* c) {
    float isd[KIN], mu[KIN];
    for (int k = 0; k < KIN; ++k) {
        mu[k] = k < NFEAT ? c->mu[k] : 0.f;
        isd[k] = k < NFEAT ? 1.0f / c->sd[k] : 0.f;
    }
    char* base = reinterpret_cast<char*>(c->img);
    CL_TRY(c, cudaMemcpyAsync(base + offsetof(Image, dtau_max), &c->dtau_max, sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(base + offsetof(Image, dtau_min), &c->dtau_min, sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(base + offsetof(Image, mu), mu, sizeof(mu), cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(base + offsetof(Image, isd), isd, sizeof(isd), cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    return TSLB_OK;
}

int rebuild_image(tslb_closure* c) {
    image_kernel<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(c->params, c->img);
    CL_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

int check_cflags(tslb_closure* c) {
    unsigned int h = 0;
    CL_TRY(c, cudaMemcpyAsync(&h, c->flags, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    if (h & 2u) {
        CL_TRY(c, cudaMemsetAsync(c->flags, 0, sizeof(unsigned int), c->stream));
        CL_TRY(c, cudaStreamSynchronize(c->stream));
        return cfail(c, TSLB_ERR_TIMEOUT, "a bounded wait on the tensor cores ran out");
    }
    return TSLB_OK;
}

int ensure_partial(tslb_closure* c, int nctas) {
    if (nctas <= c->max_ctas) return TSLB_OK;
    cudaFree(c->partial);
    c->partial = nullptr;
    CL_TRY(c, cudaMalloc(&c->partial, sizeof(float) * (size_t)nctas * PSTRIDE));
    c->max_ctas = nctas;
    return TSLB_OK;
}

// one pass of train_kernel + adam_kernel on the given sample arrays (device)
int train_pass(tslb_closure* c, const float* feat, const float* tgt, const float* wgt, long long ndata, long long nrows,
               int random, unsigned long long seed, int step, float lr, float* grad_out, float* loss_out) {
    const long long ntiles = (nrows + TILE - 1) / TILE;
    const int grid = (int)std::min<long long>(ntiles, (long long)c->train_per_sm * c->sms);
    int rc = ensure_partial(c, grid);
    if (rc) return rc;
    TrainArgs a;
    a.img = c->img; a.feat = feat; a.tgt = tgt; a.wgt = wgt;
    a.ndata = ndata; a.nrows = nrows; a.random = random; a.seed = seed; a.step = step;
    a.inv_batch = 1.0f / (float)nrows;
    a.partial = c->partial; a.flags = c->flags;
    train_kernel<<<grid, TILE, TRAIN_SMEM, c->stream>>>(a);
    CL_TRY(c, cudaGetLastError());
    AdamArgs d;
    d.partial = c->partial; d.nctas = grid;
    d.params = c->params; d.m = c->adam_m; d.v = c->adam_v; d.img = c->img;
    d.lr = lr; d.b1 = 0.9f; d.b2 = 0.999f; d.eps = 1e-8f;
    if (!grad_out) c->adam_t++;
    d.bc1 = 1.0f - std::pow(0.9f, (float)std::max<long long>(c->adam_t, 1));
    d.bc2 = 1.0f - std::pow(0.999f, (float)std::max<long long>(c->adam_t, 1));
    d.grad_out = grad_out; d.loss_out = loss_out;
    adam_kernel<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(d);
    CL_TRY(c, cudaGetLastError());
    return TSLB_OK;
}

LatticeSrc lattice_src(tslb_ctx* L, const float* view) {
    LatticeSrc s;
    s.st = view; s.N = L->N; s.n = L->n;
    s.nx = L->nx; s.ny = L->ny; s.nz = L->nz;
    s.px = L->p.bc[0] == TSLB_BC_PERIODIC;
    s.py = L->p.bc[2] == TSLB_BC_PERIODIC;
    s.pz = L->p.bc[4] == TSLB_BC_PERIODIC;
    s.inv_nu_a = 3.0f / (L->p.tau_a - 0.5f);
    s.inv_nu_b = 3.0f / (L->p.tau_b - 0.5f);
    s.dtau = L->dtau;
    s.base = L->base_on ? L->dtau_base : nullptr;
    s.dx = Divider::make(L->nx);
    s.dy = Divider::make(L->ny);
    return s;
}

int grow_dataset(tslb_closure* c, long long need) {
    if (need <= c->ds_cap) return TSLB_OK;
    long long cap = std::max<long long>(need, std::max<long long>(1 << 20, 2 * c->ds_cap));
    float *f = nullptr, *t = nullptr, *w = nullptr;
    CL_TRY(c, cudaMalloc(&f, sizeof(float) * NFEAT * cap));
    CL_TRY(c, cudaMalloc(&t, sizeof(float) * cap));
    CL_TRY(c, cudaMalloc(&w, sizeof(float) * cap));
    if (c->ds_n) {
        CL_TRY(c, cudaMemcpyAsync(f, c->ds_feat, sizeof(float) * NFEAT * c->ds_n, cudaMemcpyDeviceToDevice, c->stream));
        CL_TRY(c, cudaMemcpyAsync(t, c->ds_tgt, sizeof(float) * c->ds_n, cudaMemcpyDeviceToDevice, c->stream));
        CL_TRY(c, cudaMemcpyAsync(w, c->ds_wgt, sizeof(float) * c->ds_n, cudaMemcpyDeviceToDevice, c->stream));
        CL_TRY(c, cudaStreamSynchronize(c->stream));
    }
    cudaFree(c->ds_feat); cudaFree(c->ds_tgt); cudaFree(c->ds_wgt);
    c->ds_feat = f; c->ds_tgt = t; c->ds_wgt = w;
    c->ds_cap = cap;
    return TSLB_OK;
}

// temporary device copies of host sample arrays
struct DevSamples {
    float *f = nullptr, *t = nullptr, *w = nullptr, *y = nullptr;
    ~DevSamples() { cudaFree(f); cudaFree(t); cudaFree(w); cudaFree(y); }
};

}  // namespace

namespace tslb_internal {

int closure_before_step(tslb_ctx* L) {
    tslb_closure* c = L->closure;
    if (L->steps_done % L->closure_interval != 0) return TSLB_OK;
    const float* view = nullptr;
    int rc = fp32_view(L, &view);
    if (rc) return rc;
    const long long ntiles = (L->n + TILE - 1) / TILE;
    const int grid = (int)std::min<long long>(ntiles, (long long)c->infer_per_sm * c->sms);
    infer_kernel<LatticeSrc><<<grid, TILE, INFER_SMEM, L->stream>>>(c->img, lattice_src(L, view), L->n, L->flags);
    L->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(L, TSLB_ERR_CUDA, std::string("closure kernel: ") + cudaGetErrorString(e));
    return TSLB_OK;
}

}  // namespace tslb_internal

// ------------------------------------------------------------------ C-ABI
extern "C" {

int tslb_closure_create(tslb_closure** out) {
    if (!out) return cfail(nullptr, TSLB_ERR_ARG, "out is NULL");
    *out = nullptr;
    tslb_closure* c = new (std::nothrow) tslb_closure();
    if (!c) return cfail(nullptr, TSLB_ERR_ARG, "out of host memory");
    for (int k = 0; k < NFEAT; ++k) { c->mu[k] = 0.f; c->sd[k] = 1.f; }
    auto bail = [&](cudaError_t e, const char* what) {
        g_closure_create_error = std::string(what) + ": " + cudaGetErrorString(e);
        tslb_closure_destroy(c);
        return TSLB_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaGetDevice(&c->device)) != cudaSuccess) return bail(e, "cudaGetDevice");
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "cudaStreamCreate");
    if ((e = cudaMalloc(&c->params, sizeof(float) * NPARAM_PAD)) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&c->adam_m, sizeof(float) * NPARAM_PAD)) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&c->adam_v, sizeof(float) * NPARAM_PAD)) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&c->img, sizeof(Image))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&c->flags, sizeof(unsigned int))) != cudaSuccess) return bail(e, "cudaMalloc");
    cudaMemset(c->params, 0, sizeof(float) * NPARAM_PAD);
    cudaMemset(c->adam_m, 0, sizeof(float) * NPARAM_PAD);
    cudaMemset(c->adam_v, 0, sizeof(float) * NPARAM_PAD);
    cudaMemset(c->img, 0, sizeof(Image));
    cudaMemset(c->flags, 0, sizeof(unsigned int));
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(e, "cudaMemset");
    if ((e = set_attributes()) != cudaSuccess) return bail(e, "cudaFuncSetAttribute");
    // persistent grids: exactly the CTAs that can be resident at once
    if ((e = resident_ctas(c->device, (const void*)infer_kernel<LatticeSrc>, INFER_SMEM, &c->infer_per_sm)) != cudaSuccess)
        return bail(e, "resident_ctas");
    if ((e = resident_ctas(c->device, (const void*)train_kernel, TRAIN_SMEM, &c->train_per_sm)) != cudaSuccess)
        return bail(e, "resident_ctas");
    if (rebuild_image(c) || upload_meta(c)) {
        g_closure_create_error = c->err;
        tslb_closure_destroy(c);
        return TSLB_ERR_CUDA;
    }
    *out = c;
    return TSLB_OK;
}

void tslb_closure_destroy(tslb_closure* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->params); cudaFree(c->adam_m); cudaFree(c->adam_v); cudaFree(c->img);
    cudaFree(c->partial); cudaFree(c->loss_dev); cudaFree(c->flags);
    cudaFree(c->ds_feat); cudaFree(c->ds_tgt); cudaFree(c->ds_wgt);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int tslb_closure_set_params(tslb_closure* c, const float* params, const float* mu, const float* sd, float dtau_max) {
    if (!c) return TSLB_ERR_ARG;
    if (!(dtau_max > 0.f) || !std::isfinite(dtau_max)) return cfail(c, TSLB_ERR_ARG, "dtau_max must be finite and > 0");
    if (params)
        for (int p = 0; p < NPARAM; ++p)
            if (!std::isfinite(params[p])) return cfail(c, TSLB_ERR_ARG, "non-finite parameter");
    if (sd)
        for (int k = 0; k < NFEAT; ++k)
            if (!(sd[k] > 0.f) || !std::isfinite(sd[k])) return cfail(c, TSLB_ERR_ARG, "sd must be finite and > 0");
    if (mu)
        for (int k = 0; k < NFEAT; ++k)
            if (!std::isfinite(mu[k])) return cfail(c, TSLB_ERR_ARG, "non-finite mu");
    if (params) {
        std::vector<float> h(NPARAM_PAD, 0.f);
        std::memcpy(h.data(), params, sizeof(float) * NPARAM);
        for (int n = 0; n < NH; ++n)
            for (int k = NFEAT; k < KIN; ++k) h[P_W1 + n * KIN + k] = 0.f;
        CL_TRY(c, cudaMemcpyAsync(c->params, h.data(), sizeof(float) * NPARAM_PAD, cudaMemcpyHostToDevice, c->stream));
        CL_TRY(c, cudaMemsetAsync(c->adam_m, 0, sizeof(float) * NPARAM_PAD, c->stream));
        CL_TRY(c, cudaMemsetAsync(c->adam_v, 0, sizeof(float) * NPARAM_PAD, c->stream));
        c->adam_t = 0;
        int rc = rebuild_image(c);
        if (rc) return rc;
    }
    if (mu) std::memcpy(c->mu, mu, sizeof(c->mu));
    if (sd) std::memcpy(c->sd, sd, sizeof(c->sd));
    c->dtau_max = dtau_max;
    return upload_meta(c);
}

int tslb_closure_get_params(tslb_closure* c, float* params, float* mu, float* sd, float* dtau_max) {
    if (!c) return TSLB_ERR_ARG;
    if (params) {
        CL_TRY(c, cudaMemcpyAsync(params, c->params, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, c->stream));
        CL_TRY(c, cudaStreamSynchronize(c->stream));
    }
    if (mu) std::memcpy(mu, c->mu, sizeof(c->mu));
    if (sd) std::memcpy(sd, c->sd, sizeof(c->sd));
    if (dtau_max) *dtau_max = c->dtau_max;
    return TSLB_OK;
}

int tslb_closure_set_dtau_min(tslb_closure* c, float dtau_min) {
    if (!c) return TSLB_ERR_ARG;
    if (!(dtau_min <= 0.f) || !std::isfinite(dtau_min)) return cfail(c, TSLB_ERR_ARG, "dtau_min must be finite and <= 0");
    c->dtau_min = dtau_min;
    return upload_meta(c);
}

float tslb_closure_dtau_min(const tslb_closure* c) { return c ? c->dtau_min : 0.f; }

int tslb_closure_forward(tslb_closure* c, const float* features, long long n, float* dtau) {
    if (!c) return TSLB_ERR_ARG;
    if (n < 0 || (n > 0 && (!features || !dtau))) return cfail(c, TSLB_ERR_ARG, "tslb_closure_forward: bad arguments");
    if (n == 0) return TSLB_OK;
    DevSamples d;
    CL_TRY(c, cudaMalloc(&d.f, sizeof(float) * NFEAT * n));
    CL_TRY(c, cudaMalloc(&d.y, sizeof(float) * n));
    CL_TRY(c, cudaMemcpyAsync(d.f, features, sizeof(float) * NFEAT * n, cudaMemcpyHostToDevice, c->stream));
    ArraySrc src{d.f, d.y, n};
    const long long ntiles = (n + TILE - 1) / TILE;
    const int grid = (int)std::min<long long>(ntiles, (long long)c->infer_per_sm * c->sms);
    infer_kernel<ArraySrc><<<grid, TILE, INFER_SMEM, c->stream>>>(c->img, src, n, c->flags);
    CL_TRY(c, cudaGetLastError());
    CL_TRY(c, cudaMemcpyAsync(dtau, d.y, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    return check_cflags(c);
}

int tslb_closure_gradient(tslb_closure* c, const float* features, const float* target, const float* weight, long long n,
                          float* grad, double* loss) {
    if (!c) return TSLB_ERR_ARG;
    if (n <= 0 || !features || !target || !weight || !grad) return cfail(c, TSLB_ERR_ARG, "tslb_closure_gradient: bad arguments");
    DevSamples d;
    CL_TRY(c, cudaMalloc(&d.f, sizeof(float) * NFEAT * n));
    CL_TRY(c, cudaMalloc(&d.t, sizeof(float) * n));
    CL_TRY(c, cudaMalloc(&d.w, sizeof(float) * n));
    CL_TRY(c, cudaMalloc(&d.y, sizeof(float) * (NPARAM_PAD + 8)));
    CL_TRY(c, cudaMemcpyAsync(d.f, features, sizeof(float) * NFEAT * n, cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(d.t, target, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(d.w, weight, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    int rc = train_pass(c, d.f, d.t, d.w, n, n, 0, 0, 0, 0.f, d.y, d.y + NPARAM_PAD);
    if (rc) return rc;
    float l = 0.f;
    CL_TRY(c, cudaMemcpyAsync(grad, d.y, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaMemcpyAsync(&l, d.y + NPARAM_PAD, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    if (loss) *loss = l;
    return check_cflags(c);
}

int tslb_closure_dataset_clear(tslb_closure* c) {
    if (!c) return TSLB_ERR_ARG;
    c->ds_n = 0;
    c->fine_adds = 0;
    return TSLB_OK;
}

int tslb_closure_dataset_add(tslb_closure* c, const float* features, const float* target, const float* weight, long long n) {
    if (!c) return TSLB_ERR_ARG;
    if (n < 0 || (n > 0 && (!features || !target || !weight))) return cfail(c, TSLB_ERR_ARG, "tslb_closure_dataset_add: bad arguments");
    int rc = grow_dataset(c, c->ds_n + n);
    if (rc) return rc;
    CL_TRY(c, cudaMemcpyAsync(c->ds_feat + NFEAT * c->ds_n, features, sizeof(float) * NFEAT * n, cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(c->ds_tgt + c->ds_n, target, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaMemcpyAsync(c->ds_wgt + c->ds_n, weight, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    c->ds_n += n;
    return TSLB_OK;
}

int tslb_closure_dataset_add_fine(tslb_closure* c, tslb_ctx* fine, float pi_scale, int keep_every, int z_lo, int z_hi,
                                  long long* added) {
    if (!c || !fine) return cfail(c, TSLB_ERR_ARG, "tslb_closure_dataset_add_fine: NULL");
    if (added) *added = 0;
    if (fine->p.mode != TSLB_MODE_COLOUR) return cfail(c, TSLB_ERR_ARG, "the fine lattice must be in colour mode");
    if ((fine->nx | fine->ny | fine->nz) & 1) return cfail(c, TSLB_ERR_ARG, "the fine lattice sizes must be even");
    if (keep_every < 1 || !std::isfinite(pi_scale)) return cfail(c, TSLB_ERR_ARG, "keep_every >= 1 and a finite pi_scale");
    if (!fine->loaded) return cfail(c, TSLB_ERR_STATE, "the fine lattice has no state");
    const float* view = nullptr;
    if (tslb_internal::fp32_view(fine, &view)) return cfail(c, TSLB_ERR_CUDA, "fine state: " + fine->err);
    CL_TRY(c, cudaStreamSynchronize(fine->stream));
    const int cx = fine->nx / 2, cy = fine->ny / 2, cz = fine->nz / 2;
    const long long nc = (long long)cx * cy * cz;
    if (z_hi <= 0 || z_hi > cz) z_hi = cz;
    if (z_lo < 0 || z_lo >= z_hi) return cfail(c, TSLB_ERR_ARG, "tslb_closure_dataset_add_fine: empty z range");
    const int phase = c->fine_adds % keep_every;
    const long long plane = (long long)cx * cy;
    const long long J0 = z_lo * plane + phase, J1 = z_hi * plane;
    const long long nadd = J1 > J0 ? (J1 - J0 + keep_every - 1) / keep_every : 0;
    int rc = grow_dataset(c, c->ds_n + nadd);
    if (rc) return rc;
    float* inter = nullptr;
    CL_TRY(c, cudaMalloc(&inter, sizeof(float) * NINTER * nc));
    coarsen_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(view, fine->N, fine->nx, fine->ny, fine->nz, pi_scale, inter);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && nadd > 0) {
        samples_kernel<<<(unsigned)((nadd + 255) / 256), 256, 0, c->stream>>>(
            inter, cx, cy, cz, fine->p.bc[0] == TSLB_BC_PERIODIC, fine->p.bc[2] == TSLB_BC_PERIODIC,
            fine->p.bc[4] == TSLB_BC_PERIODIC, keep_every, J0, J1, c->ds_n, c->ds_feat, c->ds_tgt, c->ds_wgt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(inter);
    if (e != cudaSuccess) return cfail(c, TSLB_ERR_CUDA, std::string("dataset filter: ") + cudaGetErrorString(e));
    c->ds_n += nadd;
    c->fine_adds++;
    if (added) *added = nadd;
    return TSLB_OK;
}

long long tslb_closure_dataset_size(tslb_closure* c) { return c ? c->ds_n : 0; }

int tslb_closure_dataset_download(tslb_closure* c, float* features, float* target, float* weight) {
    if (!c) return TSLB_ERR_ARG;
    if (c->ds_n == 0) return TSLB_OK;
    if (features) CL_TRY(c, cudaMemcpyAsync(features, c->ds_feat, sizeof(float) * NFEAT * c->ds_n, cudaMemcpyDeviceToHost, c->stream));
    if (target) CL_TRY(c, cudaMemcpyAsync(target, c->ds_tgt, sizeof(float) * c->ds_n, cudaMemcpyDeviceToHost, c->stream));
    if (weight) CL_TRY(c, cudaMemcpyAsync(weight, c->ds_wgt, sizeof(float) * c->ds_n, cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    return TSLB_OK;
}

int tslb_closure_normalize(tslb_closure* c) {
    if (!c) return TSLB_ERR_ARG;
    if (c->ds_n < 2) return cfail(c, TSLB_ERR_STATE, "tslb_closure_normalize: the training set is empty");
    const int blocks = 2 * c->sms;
    double* part = nullptr;
    CL_TRY(c, cudaMalloc(&part, sizeof(double) * blocks * NSUM));
    norm_partial_kernel<<<blocks, 256, 0, c->stream>>>(c->ds_feat, c->ds_wgt, c->ds_n, part);
    std::vector<double> h((size_t)blocks * NSUM);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(part);
    if (e != cudaSuccess) return cfail(c, TSLB_ERR_CUDA, std::string("normalize: ") + cudaGetErrorString(e));
    double s[NSUM] = {0.0};
    for (int b = 0; b < blocks; ++b)
        for (int k = 0; k < NSUM; ++k) s[k] += h[(size_t)b * NSUM + k];
    const double n = (double)c->ds_n;
    for (int k = 0; k < NFEAT; ++k) {
        const double m = s[k] / n;
        const double var = std::max(0.0, s[NFEAT + k] / n - m * m);
        c->mu[k] = (float)m;
        c->sd[k] = var > 1e-24 ? (float)std::sqrt(var) : 1.0f;
    }
    if (!(s[2 * NFEAT] > 0.0)) return cfail(c, TSLB_ERR_STATE, "tslb_closure_normalize: all sample weights are zero");
    const float ws = (float)(n / s[2 * NFEAT]);
    scale_kernel<<<(unsigned)((c->ds_n + 255) / 256), 256, 0, c->stream>>>(c->ds_wgt, c->ds_n, ws);
    CL_TRY(c, cudaGetLastError());
    return upload_meta(c);
}

int tslb_closure_train(tslb_closure* c, int steps, int batch, float lr, unsigned long long seed, float* loss_history) {
    if (!c) return TSLB_ERR_ARG;
    if (steps < 0 || batch < TILE || batch % TILE || !(lr > 0.f))
        return cfail(c, TSLB_ERR_ARG, "tslb_closure_train: steps >= 0, batch a positive multiple of 128, lr > 0");
    if (c->ds_n == 0) return cfail(c, TSLB_ERR_STATE, "tslb_closure_train: the training set is empty");
    if (steps > c->loss_cap) {
        cudaFree(c->loss_dev);
        c->loss_dev = nullptr;
        CL_TRY(c, cudaMalloc(&c->loss_dev, sizeof(float) * steps));
        c->loss_cap = steps;
    }
    for (int s = 0; s < steps; ++s) {
        const float cosf_ = 0.5f * (1.0f + std::cos(3.14159265358979f * (float)s / (float)std::max(steps, 1)));
        const float lr_s = lr * (0.1f + 0.9f * cosf_);
        int rc = train_pass(c, c->ds_feat, c->ds_tgt, c->ds_wgt, c->ds_n, batch, 1, seed, s, lr_s, nullptr, c->loss_dev + s);
        if (rc) return rc;
    }
    if (loss_history && steps > 0)
        CL_TRY(c, cudaMemcpyAsync(loss_history, c->loss_dev, sizeof(float) * steps, cudaMemcpyDeviceToHost, c->stream));
    CL_TRY(c, cudaStreamSynchronize(c->stream));
    return check_cflags(c);
}

int tslb_closure_features(tslb_closure* c, tslb_ctx* L, float* features) {
    if (!c || !L || !features) return cfail(c, TSLB_ERR_ARG, "tslb_closure_features: NULL");
    if (L->p.mode != TSLB_MODE_COLOUR || L->p.precision != TSLB_PREC_FP32)
        return cfail(c, TSLB_ERR_ARG, "tslb_closure_features: colour mode with FP32 storage only");
    if (!L->loaded) return cfail(c, TSLB_ERR_STATE, "the lattice has no state");
    const float* view = nullptr;
    if (tslb_internal::fp32_view(L, &view)) return cfail(c, TSLB_ERR_CUDA, L->err);
    float* d = nullptr;
    CL_TRY(c, cudaMalloc(&d, sizeof(float) * NFEAT * L->n));
    // the correction in effect: the closure's total, the static field, or none
    LatticeSrc src = lattice_src(L, view);
    src.dtau = L->closure ? L->dtau : (L->base_on ? L->dtau_base : nullptr);
    features_kernel<<<(unsigned)((L->n + 255) / 256), 256, 0, L->stream>>>(src, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(features, d, sizeof(float) * NFEAT * L->n, cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cfail(c, TSLB_ERR_CUDA, std::string("features: ") + cudaGetErrorString(e));
    return TSLB_OK;
}

int tslb_attach_closure(tslb_ctx* L, tslb_closure* c, int interval) {
    if (!L) return TSLB_ERR_ARG;
    if (!c) {
        L->closure = nullptr;
        return TSLB_OK;
    }
    if (interval < 1) return tslb_internal::fail(L, TSLB_ERR_ARG, "tslb_attach_closure: interval must be >= 1");
    if (L->p.mode != TSLB_MODE_COLOUR || L->p.precision != TSLB_PREC_FP32)
        return tslb_internal::fail(L, TSLB_ERR_ARG, "tslb_attach_closure: colour mode with FP32 storage only");
    if (c->device != L->device) return tslb_internal::fail(L, TSLB_ERR_ARG, "tslb_attach_closure: closure and lattice on different devices");
    if (L->solid_on) return tslb_internal::fail(L, TSLB_ERR_UNSUPPORTED, "tslb_attach_closure: not combined with solid nodes");
    // a negative correction must leave tau above 1/2 (omega below 2) for either component
    if (!(std::min(L->p.tau_a, L->p.tau_b) + c->dtau_min > 0.5f))
        return tslb_internal::fail(L, TSLB_ERR_ARG, "tslb_attach_closure: tau + dtau_min must stay above 1/2");
    int rc = tslb_internal::ensure_dtau(L);
    if (rc) return rc;
    // the first refresh sees the static correction as the previous total
    if (L->base_on) {
        if (cudaMemcpyAsync(L->dtau, L->dtau_base, sizeof(float) * L->n, cudaMemcpyDeviceToDevice, L->stream) != cudaSuccess)
            return tslb_internal::fail(L, TSLB_ERR_CUDA, "tslb_attach_closure: copy of the static correction");
    } else if (cudaMemsetAsync(L->dtau, 0, sizeof(float) * L->N, L->stream) != cudaSuccess) {
        return tslb_internal::fail(L, TSLB_ERR_CUDA, "tslb_attach_closure: clearing the correction");
    }
    // the closure's own queued work (parameter uploads, training) precedes the lattice's use of it
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return tslb_internal::fail(L, TSLB_ERR_CUDA, "closure stream");
    L->closure = c;
    L->closure_interval = interval;
    return tslb_internal::prepare_step_kernel(L);
}

const char* tslb_closure_last_error(tslb_closure* c) {
    if (!c) return g_closure_create_error.c_str();
    return c->err.c_str();
}

}  // extern "C"
