// closure_mlp.cuh -- the closure network 10 -> 64 -> 64 -> 1 on the sm_100a
// tensor cores, one tile of 128 rows (nodes or samples) per CTA of 128
// threads; thread s owns row s, which is also TMEM lane s.
//
// Shared-memory operand buffers (core-matrix layout, see tcgen05.cuh):
//   ACT [16 row groups][12 chunks][8 rows][16 B]: chunks 0..7 hold h1
//       (64 hidden values), chunks 8..9 the normalised input x (16 values,
//       10 used), chunk 10 a constant 1 in its first column, chunk 11 zeros.
//       Forward: K-major A of x W1^T (chunks 8..9) and of h1 W2^T.
//       Backward: MN-major B (N = 96: h1 | x | 1) of the weight gradient.
//   DZ  [16 row groups][16 chunks][8 rows][16 B]: chunks 0..7 dL/dz2,
//       chunks 8..15 dL/dz1.  K-major A of dz2 W2 (chunks 0..7); MN-major A
//       (M = 128: dz2 | dz1) of the weight gradient.
//   Image: W1 as a K-major B (n = 64 units, k = 16 inputs), W2 as a K-major
//       B (n = 64, k = 64) and, read MN-major, as the B of dz2 W2.
// Weight gradient in one accumulator (M = 128, N = 96, K = samples):
//   D = [dz2 | dz1]^T [h1 | x | 1]: rows 0..63 x cols 0..63 = dW2,
//   rows 64..127 x cols 64..79 = dW1, column 80 = db2 (rows 0..63), db1
//   (rows 64..127).  It accumulates over all tiles a CTA processes.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "tcgen05.cuh"

namespace clo {

constexpr int NFEAT = 10, KIN = 16, NH = 64, TILE = 128;
constexpr int P_W1 = 0, P_B1 = 1024, P_W2 = 1088, P_B2 = 5184, P_W3 = 5248, P_B3 = 5312, NPARAM = 5313;
constexpr int NPARAM_PAD = 5320;
constexpr int PSTRIDE = NPARAM_PAD + 8;  // per-CTA partial gradient; loss sum at NPARAM_PAD

// TMEM columns of the training kernel (inference uses column 0 for both layers)
constexpr uint32_t COL_Z1 = 0, COL_Z2 = 64, COL_DH1 = 0, COL_DW = 128;

// ACT holds NCH 16-byte chunks per row: 12 in training (h1 | x | 1 | 0),
// 10 in inference (h1 | x)
constexpr int NCH_TRAIN = 12, NCH_INFER = 10;
template <int NCH>
struct Act {
    static constexpr int GROUP = NCH * 128;   // bytes per row group of 8 rows
    static constexpr int BYTES = 16 * GROUP;
    __device__ static __forceinline__ int chunk(int s, int c) { return (s >> 3) * (NCH * 8) + c * 8 + (s & 7); }
};
constexpr int ACT_GROUP = Act<NCH_TRAIN>::GROUP, DZ_GROUP = 16 * 128;   // bytes per row group
constexpr int ACT_BYTES = Act<NCH_TRAIN>::BYTES, DZ_BYTES = 16 * DZ_GROUP;

// The network in the form the kernels read it (device memory; copied into
// shared memory at kernel start).
struct __align__(128) Image {
    uint4 w1[128];   // W1, K-major B: 16-byte chunk (unit n, k-chunk kc) at (n/8)*16 + kc*8 + n%8;
                     // column 10 holds b1 (input 10 is a constant 1)
    uint4 w2[512];   // W2, K-major B: chunk (n, kc) at (n/8)*64 + kc*8 + n%8
    float b1[NH], b2[NH], w3[NH];   // w3 holds BF16-rounded values
    float b3, dtau_max, dtau_min, pad0;
    float mu[KIN], isd[KIN];
};
constexpr int IMG_BYTES = (int)((sizeof(Image) + 127) / 128 * 128);

__host__ __device__ constexpr int w1_chunk(int n, int kc) { return (n >> 3) * 16 + kc * 8 + (n & 7); }
__host__ __device__ constexpr int w2_chunk(int n, int kc) { return (n >> 3) * 64 + kc * 8 + (n & 7); }
__device__ __forceinline__ int act_chunk(int s, int c) { return Act<NCH_TRAIN>::chunk(s, c); }
__device__ __forceinline__ int dz_chunk(int s, int c) { return (s >> 3) * 128 + c * 8 + (s & 7); }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ uint4 pack8(const float* v) {
    return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}
// bf16(max(a, 0)) | bf16(max(b, 0)) << 16 in one conversion (a in the low half,
// as pack2); for finite inputs equal to pack2(fmaxf(a, 0), fmaxf(b, 0))
__device__ __forceinline__ uint32_t pack2_relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}
__device__ __forceinline__ uint4 pack8_relu(const float* v) {
    return make_uint4(pack2_relu(v[0], v[1]), pack2_relu(v[2], v[3]), pack2_relu(v[4], v[5]), pack2_relu(v[6], v[7]));
}

// ---- MMA issue (one thread) ----
template <int NCH = NCH_TRAIN>
__device__ __forceinline__ void issue_fwd1(uint32_t tb, uint32_t act, uint32_t w1, uint32_t col = COL_Z1) {
    tc::mma_bf16(tb + col, tc::sdesc(act + 8 * 128, 128, Act<NCH>::GROUP), tc::sdesc(w1, 128, 256),
                 tc::idesc_bf16(128, 64, 0, 0), 0u);
}
template <int NCH = NCH_TRAIN>
__device__ __forceinline__ void issue_fwd2(uint32_t tb, uint32_t act, uint32_t w2, uint32_t col = COL_Z2) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
        tc::mma_bf16(tb + col, tc::sdesc(act + kk * 256, 128, Act<NCH>::GROUP), tc::sdesc(w2 + kk * 256, 128, 1024),
                     tc::idesc_bf16(128, 64, 0, 0), kk > 0 ? 1u : 0u);
}
// dL/dh1 = dz2 W2: A = dz2 (K-major, k = output unit), B = W2 read MN-major
// (n = input unit at 128-byte steps, k = output unit at 1024-byte steps)
__device__ __forceinline__ void issue_bwd_dh1(uint32_t tb, uint32_t dz, uint32_t w2) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
        tc::mma_bf16(tb + COL_DH1, tc::sdesc(dz + kk * 256, 128, DZ_GROUP), tc::sdesc(w2 + kk * 2048, 1024, 128),
                     tc::idesc_bf16(128, 64, 0, 1), kk > 0 ? 1u : 0u);
}
// weight gradient over the tile's 128 samples (K = samples)
__device__ __forceinline__ void issue_bwd_dw(uint32_t tb, uint32_t dz, uint32_t act, bool first) {
#pragma unroll
    for (int kk = 0; kk < 8; ++kk)
        tc::mma_bf16(tb + COL_DW, tc::sdesc(dz + kk * 2 * DZ_GROUP, DZ_GROUP, 128),
                     tc::sdesc(act + kk * 2 * ACT_GROUP, ACT_GROUP, 128), tc::idesc_bf16(128, 96, 1, 1),
                     (first && kk == 0) ? 0u : 1u);
}

// ---- CTA-wide steps ----
// Make this thread's shared-memory writes visible to the tensor core and
// its TMEM reads complete, then synchronise the CTA.
__device__ __forceinline__ void sync_for_mma() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
}

// Thread 0 waits (bounded) for the MMAs committed to `bar`; the result is
// CTA-uniform.  On a timeout bit 1 of *gflag is set.
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& ph, int* abort_s, unsigned int* gflag) {
    if (threadIdx.x == 0) {
        if (!tc::mbar_wait_bounded(bar, ph, 4000000000LL)) {
            *abort_s = 1;
            atomicOr(gflag, 2u);
        }
    }
    __syncthreads();
    const bool ok = *abort_s == 0;
    if (ok) ph ^= 1u;   // on a timeout ph stays the phase still pending
    tc::fence_after_sync();
    return ok;
}

// normalised input row -> ACT chunks 8, 9; input 10 is a constant 1 that
// carries the first layer's bias (stored in W1's column 10)
template <int NCH = NCH_TRAIN>
__device__ __forceinline__ void put_x(uint4* act, int s, const float* f, const Image& im, bool valid) {
    float x[KIN];
#pragma unroll
    for (int k = 0; k < KIN; ++k) x[k] = (valid && k < NFEAT) ? (f[k] - im.mu[k]) * im.isd[k] : 0.f;
    x[NFEAT] = valid ? 1.f : 0.f;
    act[Act<NCH>::chunk(s, 8)] = pack8(x);
    act[Act<NCH>::chunk(s, 9)] = pack8(x + 8);
}

__device__ __forceinline__ uint32_t lane_addr(uint32_t tb, uint32_t col) {
    const uint32_t warp = threadIdx.x >> 5;
    return tb + ((32u * warp) << 16) + col;
}

// z1 (bias included) -> h1 = relu(z1) into ACT chunks 0..7; MASK: also
// returns the bits z1 > 0 (training)
template <int NCH, bool MASK>
__device__ __forceinline__ uint64_t epi_h1(uint32_t tb, uint4* act, int s, uint32_t col) {
    uint64_t mask = 0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float z[32];
        tc::tmem_ld32(lane_addr(tb, col + 32 * q), z);
        if (MASK) {
            uint32_t m = 0;
#pragma unroll
            for (int j = 0; j < 32; ++j) m |= (z[j] > 0.f ? 1u : 0u) << j;
            mask |= (uint64_t)m << (32 * q);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) act[Act<NCH>::chunk(s, 4 * q + c)] = pack8_relu(z + 8 * c);
    }
    return mask;
}

// network output o = w3 . relu(z2 + b2) + b3 in four partial sums (units
// j = 0, 1, 2, 3 mod 4), the bias add and the products on the paired FP32
// instructions
__device__ __forceinline__ float epi_out(uint32_t tb, const Image& im, uint32_t col = COL_Z2) {
    float2 o[2] = {make_float2(im.b3, 0.f), make_float2(0.f, 0.f)};
    const float2* b2 = reinterpret_cast<const float2*>(im.b2);
    const float2* w3 = reinterpret_cast<const float2*>(im.w3);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float z[32];
        tc::tmem_ld32(lane_addr(tb, col + 32 * q), z);
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            float2 v = __fadd2_rn(make_float2(z[j], z[j + 1]), b2[(32 * q + j) >> 1]);
            v.x = fmaxf(v.x, 0.f);
            v.y = fmaxf(v.y, 0.f);
            o[(j >> 1) & 1] = __ffma2_rn(w3[(32 * q + j) >> 1], v, o[(j >> 1) & 1]);
        }
    }
    return (o[0].x + o[0].y) + (o[1].x + o[1].y);
}

// dz2 = g w3 [z2 + b2 > 0] into DZ chunks 0..7; dw3 += g h2
__device__ __forceinline__ void epi_dz2(uint32_t tb, uint4* dz, int s, const Image& im, float g, float* dw3) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float z[32], d[32];
        tc::tmem_ld32(lane_addr(tb, COL_Z2 + 32 * q), z);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float v = z[j] + im.b2[32 * q + j];
            const bool p = v > 0.f;
            dw3[32 * q + j] = fmaf(g, p ? v : 0.f, dw3[32 * q + j]);
            d[j] = p ? g * im.w3[32 * q + j] : 0.f;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) dz[dz_chunk(s, 4 * q + c)] = pack8(d + 8 * c);
    }
}

// dz1 = dh1 [z1 > 0] into DZ chunks 8..15
__device__ __forceinline__ void epi_dz1(uint32_t tb, uint4* dz, int s, uint64_t mask) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float z[32];
        tc::tmem_ld32(lane_addr(tb, COL_DH1 + 32 * q), z);
        const uint32_t m = (uint32_t)(mask >> (32 * q));
#pragma unroll
        for (int j = 0; j < 32; ++j) z[j] = ((m >> j) & 1u) ? z[j] : 0.f;
#pragma unroll
        for (int c = 0; c < 4; ++c) dz[dz_chunk(s, 8 + 4 * q + c)] = pack8(z + 8 * c);
    }
}

// ---- features ----
__device__ __forceinline__ float frob(const float* P) {
    return sqrtf(P[0] * P[0] + P[3] * P[3] + P[5] * P[5] + 2.f * (P[1] * P[1] + P[2] * P[2] + P[4] * P[4]));
}
// f0..5 = s Pi (xx, xy, xz, yy, yz, zz), f6 = phi, f7 = |grad phi|, f8 = |u|, f9 = s |Pi|_F
__device__ __forceinline__ void make_features(float s, const float* P, float phi, float gmag, float umag, float* f) {
#pragma unroll
    for (int k = 0; k < 6; ++k) f[k] = s * P[k];
    f[6] = phi;
    f[7] = gmag;
    f[8] = umag;
    f[9] = s * frob(P);
}
// Division by an invariant divisor d >= 1 of dividends 0 <= n < 2^31 with a
// multiply-high and a shift (the round-up method of Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994): with
// l = ceil(log2 d) and m = ceil(2^(31+l) / d) < 2^32, the error of m / 2^(31+l)
// against 1/d is below 1/(d n) for every n < 2^31, so
// n / d = floor(n m / 2^(31+l)) = umulhi(n, m) >> (l - 1).  d = 1 keeps m = 0.
struct Divider {
    uint32_t m = 0;
    int sh = 0;
    static Divider make(int d) {
        Divider r;
        if (d <= 1) return r;
        int l = 0;
        while ((1LL << l) < d) ++l;
        r.m = (uint32_t)((((unsigned long long)1 << (31 + l)) + (unsigned long long)d - 1) / (unsigned long long)d);
        r.sh = l - 1;
        return r;
    }
    __device__ __forceinline__ int div(int n) const { return m ? (int)(__umulhi((uint32_t)n, m) >> sh) : n; }
};

// neighbour coordinate: periodic axes wrap, others repeat the boundary node
__device__ __forceinline__ int nbr(int x, int d, int n, bool periodic) {
    int y = x + d;
    if (y < 0) y = periodic ? y + n : 0;
    else if (y >= n) y = periodic ? y - n : n - 1;
    return y;
}

}  // namespace clo
