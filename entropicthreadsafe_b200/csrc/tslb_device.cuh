// tslb_device.cuh -- device-side building blocks of the fused TSLB step.
//
// State layout in HBM: 11 SoA fields of nx*ny*nz floats (x fastest, field
// stride N padded to 32 floats):
//   0 d = rho - 1   1 u   2 v   3 w   4 pxx 5 pxy 6 pxz 7 pyy 8 pyz 9 pzz  10 phi
// p** is the non-equilibrium second moment Pi^neq.  Storing rho - 1 keeps
// the density's small deviations exact to FP32 round-off of the deviation.
//
// Post-collision populations are written as f_c = w_c (1 + P'(c)) where
// P'(c) is a polynomial in the components of c with 17 per-node
// coefficients (the monomials 1, cx, cy, cz, cx^2, ..., cx cy cz that
// survive on D3Q27 because c_a^3 = c_a).  The coefficients fold:
//   f^eq(rho, u_s) in third-order Hermite form
//     (recursive_2c_TSLB3D.f90:639-804 "feqs")
//   (1 - omega) w a^neq(Pi, u), the recursive regularized non-equilibrium
//     (recursive_2c_TSLB3D.f90:640-805 "fneq1")
//   colour mode: the perturbation operator and the force source of
//     turbulent_benchmark/couette/recursive_colorTSLB3D.f90:765-959
// so that every pulled population costs a handful of FMAs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

#include "../../include/tslb.h"

namespace tslb {

constexpr int NF = 11;
enum { F_D = 0, F_U, F_V, F_W, F_XX, F_XY, F_XZ, F_YY, F_YZ, F_ZZ, F_PHI };

// Coefficient slots (per node, shared memory), in five quads and one pair
// that the pull reads whole, so a source reads a quad with one 16-byte load:
//   q0 (0, z | zz, c0)        every source
//   q1 (x, xx | xz, xxz)      sources with cx != 0
//   q2 (y, yy | yz, yyz)      sources with cy != 0
//   q3 (xzz, c1 | yzz, c2)    the first half for cx != 0, the second for cy != 0
//   q4 (xy, xyz | xxy, xyy)   sources with cx != 0 and cy != 0
//   p5 (c3, c4)               every source (c4: the rest population's)
// Colour slots c0..c4: phi, Bx, By, Bz, delta0 | phase field: G0, G1x, G1y, G1z, -.
enum {
    K_0 = 0, K_Z, K_ZZ, K_C0,
    K_X, K_XX, K_XZ, K_XXZ,
    K_Y, K_YY, K_YZ, K_YYZ,
    K_XZZ, K_C1, K_YZZ, K_C2,
    K_XY, K_XYZ, K_XXY, K_XYY,
    K_C3, K_C4,
    NCOEF
};
constexpr int NQUAD = 5;   // quads q0..q4; slots 4 NQUAD.. form the pair p5
static_assert(NCOEF == 4 * NQUAD + 2, "coefficient slots: five quads and one pair");

// accumulator slots of a target node
enum { A_RHO = 0, A_JX, A_JY, A_JZ, A_XX, A_XY, A_XZ, A_YY, A_YZ, A_ZZ, A_COL, NACC };

constexpr int TX = 32;  // block tile in x (one warp row)
constexpr int TY = 8;   // block tile in y
constexpr int CW = TX + 2, CH = TY + 2, CAREA = CW * CH;

// lattice weights by |c|^2 (recursive_2c_TSLB3D.f90:71-74)
__host__ __device__ constexpr float wclass(int c2) {
    return c2 == 0 ? 8.0f / 27.0f : c2 == 1 ? 2.0f / 27.0f : c2 == 2 ? 1.0f / 54.0f : 1.0f / 216.0f;
}
// 1/|c| by |c|^2 for the recolouring cos(theta)
__host__ __device__ constexpr float invlen(int c2) {
    return c2 == 1 ? 1.0f : c2 == 2 ? 0.70710678118654752f : c2 == 3 ? 0.57735026918962576f : 0.0f;
}

struct FaceBC {
    int kind;          // TSLB_BC_*
    float u[3];        // wall velocity
    float phi;         // colour of incoming populations (< -2: own phi); ghost phi on solid faces
    const float* plane;  // TSLB_BC_INLET: u, v, w, phi planes of the face
};

struct StepArgs {
    int nx, ny, nz;
    long long N;            // field stride (elements)
    const void* in;         // 11 fields of the storage type
    void* out;              // 11 fields of the storage type
    float scale[NF];        // stored = value * scale (fp16 storage; 1 otherwise)
    float iscale[NF];       // value = stored * iscale
    const float* nrm;       // phase field: interface normals (3 fields of stride N)
    int zchunk;             // target planes per block
    int mode;
    float omega_pf;         // 1/tau (phase field)
    float inv_nu_a, inv_nu_b;  // colour: 1/nu of each component
    float sigma, beta, sharp, thr, acoef;
    float force[3];
    int wall_phi_mode;
    FaceBC face[6];
    unsigned int* flags;    // bit 0: non-finite moment produced
    const float* dtau;      // colour: per-node correction of tau (stride N), or null
    const unsigned int* solid;  // interior solid nodes, one bit per node (bit i & 31 of word i >> 5), or null
    const unsigned int* near;   // fluid nodes with a solid one among their 26 neighbours, same layout
    int zt0, zt1;           // target planes [zt0, zt1) a step updates (a z slab: its own planes;
                            // the planes outside them are halo copies of the neighbours')
    int zoff;               // global index of local plane 0 (a z slab's offset; seeds the rounding)
    int sr;                 // 16-bit storage: store the moments with stochastic rounding
    unsigned int sr_step;   // step counter that seeds the rounding (with the node and the field)
    const unsigned int* sr_counter;  // ensembles: device step counter read instead of sr_step, or null
};

// Counter-based uniform in [0, 1) of four integers: the reference's
// rand_noseeded (TSLB_2C-mpi/vars_single_3D_module.f90:150-215), which seeds
// the two lagged generators of the Marsaglia-Zaman "universal" method from
// (i, j, k, l) in 24 rounds each and returns one output.  Every FP32 value
// is a multiple of 2^-24 in [-1, 2), so the arithmetic is exact and equal
// on the host, on the device and in the Fortran original.
__host__ __device__ inline float rand_noseeded(int i, int j, int k, int l) {
    int isub = i % 178 + 1, jsub = j % 178 + 1, ksub = k % 178 + 1, lsub = l % 169;
    float u[2];
    for (int g = 0; g < 2; ++g) {
        float s = 0.f, t = 0.5f;
        for (int jj = 0; jj < 24; ++jj) {
            const int msub = ((isub * jsub) % 179) * ksub % 179;
            isub = jsub;
            jsub = ksub;
            ksub = msub;
            lsub = (53 * lsub + 1) % 169;
            if ((lsub * msub) % 64 >= 32) s += t;
            t *= 0.5f;
        }
        u[g] = s;   // u97, then u33
    }
    float uni = u[0] - u[1];
    if (uni < 0.f) uni += 1.f;
    const float c = 362436.0f / 16777216.0f, cd = 7654321.0f / 16777216.0f, cm = 16777213.0f / 16777216.0f;
    float csub = c - cd;
    if (csub < 0.f) csub += cm;
    uni -= csub;
    if (uni < 0.f) uni += 1.f;
    return uni;
}

__device__ __forceinline__ bool bit_at(const unsigned int* b, long long i) {
    return (__ldg(b + (i >> 5)) >> (i & 31)) & 1u;
}

// Storage types of the moment state: FP32, BF16 or FP16 (scaled).  All
// arithmetic is FP32; conversion happens on load and store.
template <class T>
struct Stor;
template <>
struct Stor<float> {
    static __device__ __forceinline__ float ld(float v) { return v; }
    static __device__ __forceinline__ float st(float v) { return v; }
};
template <>
struct Stor<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(__nv_bfloat16 v) { return __bfloat162float(v); }
    static __device__ __forceinline__ __nv_bfloat16 st(float v) { return __float2bfloat16_rn(v); }
};
template <>
struct Stor<__half> {
    static __device__ __forceinline__ float ld(__half v) { return __half2float(v); }
    static __device__ __forceinline__ __half st(float v) { return __float2half_rn(v); }
};

__device__ __forceinline__ long long nidx(const StepArgs& a, int x, int y, int z) {
    return (long long)x + (long long)a.nx * ((long long)y + (long long)a.ny * z);
}
// periodic wrap of any coordinate into [0, n) (tiles may reach several periods out on tiny lattices)
__device__ __forceinline__ int wrapi(int c, int n) {
    c %= n;
    return c < 0 ? c + n : c;
}
__device__ __forceinline__ int dimn(const StepArgs& a, int ax) { return ax == 0 ? a.nx : ax == 1 ? a.ny : a.nz; }

__device__ __forceinline__ long long plane_index(const StepArgs& a, int face, int x, int y, int z) {
    int ax = face >> 1;
    if (ax == 0) return (long long)y + (long long)a.ny * z;
    if (ax == 1) return (long long)x + (long long)a.nx * z;
    return (long long)x + (long long)a.nx * y;
}
__device__ __forceinline__ long long plane_area(const StepArgs& a, int face) {
    int ax = face >> 1;
    return ax == 0 ? (long long)a.ny * a.nz : ax == 1 ? (long long)a.nx * a.nz : (long long)a.nx * a.ny;
}

// phi at any node of the halo'd lattice: periodic axes wrap; on solid faces
// the inlet plane's phi (inlet faces), bc phi (wall_phi_mode 0) or the
// nearest fluid value (mirror).  The first out-of-range non-periodic axis in
// x, y, z order names the face.
// stored value -> FP32 value of field f (fp16 storage carries a per-field scale)
template <class T>
__device__ __forceinline__ float cvt_in(T v, const StepArgs& a, int f) {
    if constexpr (std::is_same<T, __half>::value) return Stor<T>::ld(v) * a.iscale[f];
    else return Stor<T>::ld(v);
}
template <class T>
__device__ __forceinline__ T cvt_out(float v, const StepArgs& a, int f) {
    if constexpr (std::is_same<T, __half>::value) return Stor<T>::st(v * a.scale[f]);
    else return Stor<T>::st(v);
}

// largest finite value of a 16-bit storage type (bf16: FP32's range)
template <class T>
struct Stor16Max;
template <>
struct Stor16Max<__half> {
    static constexpr float value = 65504.0f;
};
template <>
struct Stor16Max<__nv_bfloat16> {
    static constexpr float value = 3.3895313892515355e38f;
};
template <class T>
__device__ __forceinline__ T bits_as(unsigned short u);
template <>
__device__ __forceinline__ __half bits_as<__half>(unsigned short u) { return __ushort_as_half(u); }
template <>
__device__ __forceinline__ __nv_bfloat16 bits_as<__nv_bfloat16>(unsigned short u) { return __ushort_as_bfloat16(u); }

// Stochastic rounding of the 16-bit stored moments: a value rounds away from
// zero with the probability of its distance from the value toward zero, so
// the expected stored value is the FP32 one.  Rounding to nearest drops every
// change smaller than half a unit in the last place at every step - the body
// force of the channel adds about 2.5e-6 to u per step, 1/200 of a BF16 unit
// at u = 0.07 - and the stored flow stops following the forcing.  The step
// stores two fields with one stochastically rounded hardware conversion
// (cvt.rs.bf16x2.f32 / cvt.rs.f16x2.f32, sm_100a) whose random bits hash the
// node, the pair's first field and the step counter, so a run (and its
// restart from a checkpoint) is reproducible.
__device__ __forceinline__ unsigned int sr_node(unsigned int node, unsigned int step) {
    unsigned int h = node * 0x9E3779B1u ^ (step * 0x85EBCA77u + 0x165667B1u);
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}
__device__ __forceinline__ unsigned int sr_field(unsigned int hnode, int f) {
    unsigned int h = (hnode + (unsigned int)f * 0x9E3779B9u) * 0x85EBCA6Bu;
    return h ^ (h >> 16);
}
// Store fields f and g (g == f: f alone) of one node in 16-bit storage with
// one paired conversion: cvt.rn / cvt.rs (stochastic, random bits r) to
// f16x2 or bf16x2 of the stored values (fp16: value * per-field scale).
// Returns the largest stored magnitude before rounding, for the range check.
template <class T>
__device__ __forceinline__ float store_pair16(T* po, const StepArgs& a, int f, int g, float vf, float vg, int sr,
                                              unsigned int r) {
    constexpr bool H = std::is_same<T, __half>::value;
    const float xf = H ? vf * a.scale[f] : vf, xg = H ? vg * a.scale[g] : vg;
    unsigned int d;
    if (sr) {
        if (H) asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(xg), "f"(xf), "r"(r));
        else asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(xg), "f"(xf), "r"(r));
    } else {
        if (H) asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(xg), "f"(xf));
        else asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(xg), "f"(xf));
    }
    // the low half holds field f, the high half field g
    po[f * a.N] = bits_as<T>((unsigned short)(d & 0xFFFFu));
    if (g != f) po[g * a.N] = bits_as<T>((unsigned short)(d >> 16));
    return fmaxf(fabsf(xf), fabsf(xg));
}

template <class T>
__device__ __forceinline__ float ld_field(const StepArgs& a, int f, long long idx) {
    return cvt_in<T>(__ldg(reinterpret_cast<const T*>(a.in) + f * a.N + idx), a, f);
}

template <class T>
__device__ float phi_at(const StepArgs& a, int x, int y, int z) {
    int c[3] = {x, y, z};
    int face = -1;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        int n = dimn(a, ax);
        if (c[ax] < 0 || c[ax] >= n) {
            if (a.face[2 * ax].kind == TSLB_BC_PERIODIC) {
                c[ax] = wrapi(c[ax], n);
            } else {
                if (face < 0) face = 2 * ax + (c[ax] >= n ? 1 : 0);
                c[ax] = c[ax] < 0 ? 0 : n - 1;
            }
        }
    }
    if (face < 0) return ld_field<T>(a, F_PHI, nidx(a, c[0], c[1], c[2]));
    const FaceBC& fb = a.face[face];
    if (fb.kind == TSLB_BC_INLET) return __ldg(fb.plane + 3 * plane_area(a, face) + plane_index(a, face, c[0], c[1], c[2]));
    if (a.wall_phi_mode == 0) return fb.phi;
    return ld_field<T>(a, F_PHI, nidx(a, c[0], c[1], c[2]));
}

__device__ __forceinline__ bool interior1(const StepArgs& a, int x, int y, int z) {
    return x >= 1 && x < a.nx - 1 && y >= 1 && y < a.ny - 1 && z >= 1 && z < a.nz - 1;
}

// isotropic gradient 3 sum_i p_i c_i s(x+c_i) of phi
// (recursive_2c_TSLB3D.f90:555-565; recursive_colorTSLB3D.f90:726-744)
template <class T>
__device__ void grad_phi(const StepArgs& a, int x, int y, int z, float g[3]) {
    float gx = 0.f, gy = 0.f, gz = 0.f;
    const bool fast = interior1(a, x, y, z);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                const float wv = wclass(dx * dx + dy * dy + dz * dz);
                float s = fast ? ld_field<T>(a, F_PHI, nidx(a, x + dx, y + dy, z + dz)) : phi_at<T>(a, x + dx, y + dy, z + dz);
                s *= wv;
                if (dx) gx += dx > 0 ? s : -s;
                if (dy) gy += dy > 0 ? s : -s;
                if (dz) gz += dz > 0 ? s : -s;
            }
    g[0] = 3.f * gx;
    g[1] = 3.f * gy;
    g[2] = 3.f * gz;
}

// Arithmetic of the coefficient phase, one operation at a time.  The step
// computes a node's coefficients in every tile whose coefficient tile holds
// it: as an own node of one tile and as a rim node of its neighbours.  The
// populations it sends into different tiles must be the same numbers, or
// mass is not conserved exactly, so no operation is left for the compiler
// to contract: Ar1 evaluates one node in FP32, Ar2 two nodes at once on the
// paired FP32 instructions of sm_100 (one node per lane), and both round
// every operation identically, lane by lane.
struct Ar1 {
    using V = float;
    static __device__ __forceinline__ V c(float x) { return x; }
    static __device__ __forceinline__ V add(V x, V y) { return __fadd_rn(x, y); }
    static __device__ __forceinline__ V sub(V x, V y) { return __fsub_rn(x, y); }
    static __device__ __forceinline__ V mul(V x, V y) { return __fmul_rn(x, y); }
    static __device__ __forceinline__ V fma(V x, V y, V z) { return __fmaf_rn(x, y, z); }
    // lane-wise functions (square root, division, selection)
    template <class F>
    static __device__ __forceinline__ V map(V x, F f) { return f(x); }
    template <class F>
    static __device__ __forceinline__ V map2(V x, V y, F f) { return f(x, y); }
};
struct Ar2 {
    using V = float2;
    static __device__ __forceinline__ V c(float x) { return make_float2(x, x); }
    static __device__ __forceinline__ V add(V x, V y) { return __fadd2_rn(x, y); }
    // x - y rounded once: fma(y, -1, x)
    static __device__ __forceinline__ V sub(V x, V y) { return __ffma2_rn(y, make_float2(-1.f, -1.f), x); }
    static __device__ __forceinline__ V mul(V x, V y) { return __fmul2_rn(x, y); }
    static __device__ __forceinline__ V fma(V x, V y, V z) { return __ffma2_rn(x, y, z); }
    template <class F>
    static __device__ __forceinline__ V map(V x, F f) { return make_float2(f(x.x), f(x.y)); }
    template <class F>
    static __device__ __forceinline__ V map2(V x, V y, F f) { return make_float2(f(x.x, y.x), f(x.y, y.y)); }
};

// Per-node coefficients of P'(c) = f_c / w_c - 1 and the colour terms, for
// one node (Ar1) or two (Ar2).  m[] are the node's 11 moments (m[F_D] =
// rho - 1).  gphi: colour mode, the gradient of phi; phase field, the
// interface normal n, with curv the curvature -div n where the interface
// indicator exceeds 0.2 (else 0).  TAU: the node's relaxation time is
// tau(phi) + dt (a local eddy-viscosity correction); the surface-tension
// coefficient follows the corrected omega.
template <int MODE, bool TAU, class Ar>
__device__ __forceinline__ void node_coefs_v(const StepArgs& a, const typename Ar::V* m, const typename Ar::V* gphi,
                                             typename Ar::V curv, typename Ar::V dt, typename Ar::V* K) {
    using V = typename Ar::V;
    auto c = [](float x) { return Ar::c(x); };
    const V d = m[F_D], rho = Ar::add(c(1.f), d);
    const V u = m[F_U], v = m[F_V], w = m[F_W];
    const V pxx = m[F_XX], pxy = m[F_XY], pxz = m[F_XZ], pyy = m[F_YY], pyz = m[F_YZ], pzz = m[F_ZZ];
    const V phi = m[F_PHI];
    V omega, U, W_, Vv, A = c(0.f), mg = c(0.f), nx_ = c(0.f), ny_ = c(0.f), nz_ = c(0.f);
    if (MODE == TSLB_MODE_COLOUR) {
        const V g0 = gphi[0], g1 = gphi[1], g2 = gphi[2];
        const V m2 = Ar::fma(g2, g2, Ar::fma(g1, g1, Ar::mul(g0, g0)));
        const float thr2 = a.thr * a.thr;
        const V rs = Ar::map(m2, [](float x) { return rsqrtf(x); });
        // branch-free: outside the interface (|g|^2 <= thr^2) A = 0 and n = 0
        mg = Ar::map2(m2, rs, [thr2](float x, float r) { return x > thr2 ? __fmul_rn(x, r) : 0.f; });
        const V inv = Ar::map2(m2, rs, [thr2](float x, float r) { return x > thr2 ? r : 0.f; });
        // 1/nu = (rhoA/rho)/nu_a + (rhoB/rho)/nu_b ; omega = 2/(6 nu + 1) = 2q/(6 + q)
        const float qa = 0.5f * (a.inv_nu_a + a.inv_nu_b), qd = 0.5f * (a.inv_nu_a - a.inv_nu_b);
        const V q = Ar::fma(phi, c(qd), c(qa));
        const V q2 = Ar::add(q, q);
        // TAU: 1/omega = (6 + q)/(2q) + dtau
        const V den = TAU ? Ar::fma(q2, dt, Ar::add(q, c(6.f))) : Ar::add(q, c(6.f));
        omega = Ar::map2(q2, den, [](float n, float e) { return __fdividef(n, e); });
        nx_ = Ar::mul(g0, inv); ny_ = Ar::mul(g1, inv); nz_ = Ar::mul(g2, inv);
        const float acs = a.acoef * a.sigma;
        A = Ar::map2(m2, omega, [thr2, acs](float x, float o) { return x > thr2 ? __fmul_rn(acs, o) : 0.f; });
        U = u; Vv = v; W_ = w;
    } else if (MODE == TSLB_MODE_SINGLE) {
        // fused_TSLB_force_1c: equilibrium at the shifted velocity u + F
        omega = c(a.omega_pf);
        U = Ar::add(u, c(a.force[0]));
        Vv = Ar::add(v, c(a.force[1]));
        W_ = Ar::add(w, c(a.force[2]));
    } else {
        // CSF velocity shift u + sigma kappa n (+ F) (recursive_2c_TSLB3D.f90:630-636,
        // lb_kernels_module.f90:769)
        omega = c(a.omega_pf);
        const V sk = Ar::mul(c(a.sigma), curv);
        U = Ar::add(Ar::fma(sk, gphi[0], u), c(a.force[0]));
        Vv = Ar::add(Ar::fma(sk, gphi[1], v), c(a.force[1]));
        W_ = Ar::add(Ar::fma(sk, gphi[2], w), c(a.force[2]));
        nx_ = gphi[0]; ny_ = gphi[1]; nz_ = gphi[2];
    }
    const V om1 = Ar::sub(c(1.f), omega);
    // recursive third-order non-equilibrium moments a3 = u_a Pi_bc + perms
    const V u2 = Ar::add(u, u), v2 = Ar::add(v, v), w2 = Ar::add(w, w);
    const V a_xxy = Ar::fma(v, pxx, Ar::mul(u2, pxy));
    const V a_xxz = Ar::fma(w, pxx, Ar::mul(u2, pxz));
    const V a_xyy = Ar::fma(v2, pxy, Ar::mul(u, pyy));
    const V a_yyz = Ar::fma(w, pyy, Ar::mul(v2, pyz));
    const V a_xzz = Ar::fma(w2, pxz, Ar::mul(u, pzz));
    const V a_yzz = Ar::fma(w2, pyz, Ar::mul(v, pzz));
    const V a_xyz = Ar::fma(w, pxy, Ar::fma(v, pxz, Ar::mul(u, pyz)));
    const V rU = Ar::mul(rho, U), rV = Ar::mul(rho, Vv), rW = Ar::mul(rho, W_);
    // second-order equilibrium products rho U_a U_b
    const V rUU = Ar::mul(rU, U), rVV = Ar::mul(rV, Vv), rWW = Ar::mul(rW, W_);
    const V rUV = Ar::mul(rU, Vv), rUW = Ar::mul(rU, W_), rVW = Ar::mul(rV, W_);
    // full third-order coefficients: rho U_a U_b U_c + (1 - omega) a3
    const V t_xxy = Ar::fma(om1, a_xxy, Ar::mul(rUU, Vv)), t_xxz = Ar::fma(om1, a_xxz, Ar::mul(rUU, W_));
    const V t_xyy = Ar::fma(om1, a_xyy, Ar::mul(rUV, Vv)), t_yyz = Ar::fma(om1, a_yyz, Ar::mul(rVV, W_));
    const V t_xzz = Ar::fma(om1, a_xzz, Ar::mul(rUW, W_)), t_yzz = Ar::fma(om1, a_yzz, Ar::mul(rVW, W_));
    const V t_xyz = Ar::fma(om1, a_xyz, Ar::mul(rUV, W_));
    const V tr = Ar::add(Ar::add(pxx, pyy), pzz);
    // K0 = d - 1.5 (rho |U|^2 + (1 - omega) tr Pi)
    K[K_0] = Ar::fma(Ar::mul(c(-1.5f), om1), tr, Ar::fma(c(-1.5f), Ar::add(Ar::add(rUU, rVV), rWW), d));
    K[K_X] = Ar::fma(c(-4.5f), Ar::add(t_xyy, t_xzz), Ar::mul(c(3.f), rU));
    K[K_Y] = Ar::fma(c(-4.5f), Ar::add(t_xxy, t_yzz), Ar::mul(c(3.f), rV));
    K[K_Z] = Ar::fma(c(-4.5f), Ar::add(t_xxz, t_yyz), Ar::mul(c(3.f), rW));
    K[K_XX] = Ar::mul(c(4.5f), Ar::fma(om1, pxx, rUU));
    K[K_YY] = Ar::mul(c(4.5f), Ar::fma(om1, pyy, rVV));
    K[K_ZZ] = Ar::mul(c(4.5f), Ar::fma(om1, pzz, rWW));
    K[K_XY] = Ar::mul(c(9.f), Ar::fma(om1, pxy, rUV));
    K[K_XZ] = Ar::mul(c(9.f), Ar::fma(om1, pxz, rUW));
    K[K_YZ] = Ar::mul(c(9.f), Ar::fma(om1, pyz, rVW));
    K[K_XXY] = Ar::mul(c(13.5f), t_xxy);
    K[K_XXZ] = Ar::mul(c(13.5f), t_xxz);
    K[K_XYY] = Ar::mul(c(13.5f), t_xyy);
    K[K_YYZ] = Ar::mul(c(13.5f), t_yyz);
    K[K_XZZ] = Ar::mul(c(13.5f), t_xzz);
    K[K_YZZ] = Ar::mul(c(13.5f), t_yzz);
    K[K_XYZ] = Ar::mul(c(27.f), t_xyz);
    if (MODE == TSLB_MODE_COLOUR) {
        // force as population source 3 w c.F (recursive_colorTSLB3D.f90:776)
        K[K_X] = Ar::add(K[K_X], c(3.f * a.force[0]));
        K[K_Y] = Ar::add(K[K_Y], c(3.f * a.force[1]));
        K[K_Z] = Ar::add(K[K_Z], c(3.f * a.force[2]));
        // perturbation (A/2)|g| [w (c.n)^2 - B_i], B_i = w_i for i >= 1 (A = 0 off the interface)
        const V h = Ar::mul(Ar::mul(c(0.5f), A), mg), h2 = Ar::add(h, h);
        K[K_0] = Ar::sub(K[K_0], h);
        K[K_XX] = Ar::fma(Ar::mul(h, nx_), nx_, K[K_XX]);
        K[K_YY] = Ar::fma(Ar::mul(h, ny_), ny_, K[K_YY]);
        K[K_ZZ] = Ar::fma(Ar::mul(h, nz_), nz_, K[K_ZZ]);
        K[K_XY] = Ar::fma(Ar::mul(h2, nx_), ny_, K[K_XY]);
        K[K_XZ] = Ar::fma(Ar::mul(h2, nx_), nz_, K[K_XZ]);
        K[K_YZ] = Ar::fma(Ar::mul(h2, ny_), nz_, K[K_YZ]);
        // rest population: B_0 = -10/27 instead of w_0
        const V d0 = Ar::mul(Ar::mul(A, c(1.f / 3.f)), mg);
        // recolouring 2 beta (rhoA rhoB / rho) n  (published form, cos theta; n = 0 off the interface)
        const V bb = Ar::mul(Ar::mul(c(0.5f * a.beta), rho), Ar::fma(Ar::mul(c(-1.f), phi), phi, c(1.f)));
        K[K_C0] = phi; K[K_C1] = Ar::mul(bb, nx_); K[K_C2] = Ar::mul(bb, ny_); K[K_C3] = Ar::mul(bb, nz_); K[K_C4] = d0;
    } else if (MODE == TSLB_MODE_SINGLE) {
        K[K_C0] = c(0.f); K[K_C1] = c(0.f); K[K_C2] = c(0.f); K[K_C3] = c(0.f); K[K_C4] = c(0.f);
    } else if (MODE == TSLB_MODE_PHASEFIELD) {
        // D3Q7 phase field: g_q = G0 + e_q.G1 (recursive_2c_TSLB3D.f90:808-831)
        const V sh = Ar::mul(Ar::mul(c(0.125f * a.sharp), phi), Ar::sub(c(1.f), phi));
        const V p3 = Ar::mul(c(0.375f), phi);
        K[K_C0] = Ar::mul(c(0.125f), phi);
        K[K_C1] = Ar::fma(sh, nx_, Ar::mul(p3, u));
        K[K_C2] = Ar::fma(sh, ny_, Ar::mul(p3, v));
        K[K_C3] = Ar::fma(sh, nz_, Ar::mul(p3, w));
        K[K_C4] = c(0.f);
    }
}

// one node (the call sites of the phase field and of single lattices)
template <int MODE, bool TAU = false>
__device__ __forceinline__ void node_coefs(const StepArgs& a, const float* m, const float* gphi, float curv, float* K,
                                           long long id = 0) {
    const float dt = TAU ? __ldg(a.dtau + id) : 0.f;
    node_coefs_v<MODE, TAU, Ar1>(a, m, gphi, curv, dt, K);
}

// P'(c) for a runtime direction (boundary paths)
__device__ __forceinline__ float eval_P(const float* K, long long stride, int cx, int cy, int cz) {
    const float fx = (float)cx, fy = (float)cy, fz = (float)cz;
    const float ax = (float)(cx * cx), ay = (float)(cy * cy), az = (float)(cz * cz);
    return K[K_0 * stride] + fx * K[K_X * stride] + fy * K[K_Y * stride] + fz * K[K_Z * stride] +
           ax * K[K_XX * stride] + ay * K[K_YY * stride] + az * K[K_ZZ * stride] +
           fx * fy * K[K_XY * stride] + fx * fz * K[K_XZ * stride] + fy * fz * K[K_YZ * stride] +
           ax * fy * K[K_XXY * stride] + ax * fz * K[K_XXZ * stride] + fx * ay * K[K_XYY * stride] +
           ay * fz * K[K_YYZ * stride] + fx * az * K[K_XZZ * stride] + fy * az * K[K_YZZ * stride] +
           fx * fy * fz * K[K_XYZ * stride];
}

// accumulate population value f (already weighted) of direction c into acc
__device__ __forceinline__ void acc_dir_rt(float* acc, int cx, int cy, int cz, float f) {
    acc[A_RHO] += f;
    acc[A_JX] += cx * f; acc[A_JY] += cy * f; acc[A_JZ] += cz * f;
    acc[A_XX] += (cx * cx) * f; acc[A_YY] += (cy * cy) * f; acc[A_ZZ] += (cz * cz) * f;
    acc[A_XY] += (cx * cy) * f; acc[A_XZ] += (cx * cz) * f; acc[A_YZ] += (cy * cz) * f;
}

}  // namespace tslb
