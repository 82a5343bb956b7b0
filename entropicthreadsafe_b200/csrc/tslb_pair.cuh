// tslb_pair.cuh -- the fused pull step with two x columns per thread.
//
// The same step as tslb_step.cuh (moments in, moments out; every target
// pulls its 27 post-collision populations from the per-node coefficients
// of P'(c), tslb_device.cuh), laid out so that the coefficient phase and
// the pull run on the paired FP32 instructions of sm_100 (FFMA2, FADD2,
// FMUL2: one instruction, two independent IEEE FP32 lanes):
//
//   * lane l of warp w owns the target columns x0 + l ("A") and
//     x0 + l + 32 ("B") of row y0 + w of a 64 x 8 tile; every value the
//     thread computes is a float2 (A, B);
//   * the coefficient tile stores each slot pair (a, b) of the pair node
//     (column x, column x + 32) as one float4 (a_A, a_B, b_A, b_B), so a
//     single 16-byte shared load returns two operand pairs ready for the
//     paired instructions.  Pair node q of a tile row holds columns
//     x0 + q - 1 and x0 + q + 31 (q = 0 .. 33), so the three sources
//     x - 1, x, x + 1 of a target pair are the pair nodes q - 1, q, q + 1.
//
// Each block marches a z chunk of its tile column as the scalar kernel
// does: cp.async staging of the next plane's moments (and phi two planes
// ahead), the coefficients of the current source plane into a double
// buffered tile, one CTA barrier, the pull into three target planes of
// accumulators, face conditions, and the store of the completed plane.
// The plane loop is unrolled three times so the three accumulator planes
// change roles by renaming instead of register moves.
//
// Target-relative accumulation: the density deviation d = rho - 1 of a node
// is stored apart from its coefficients (K_0 holds K_0 - d), and every
// pulled population is accumulated as P'(c) - d_t, d_t the target's own
// deviation: (K_0 - d_s) + (d_s - d_t) + (the c-dependent terms).  All the
// summed terms are then small (velocity and stress sized), not of the size
// of d, so the new d = d_t + sum w (P' - d_t), the momentum and the second
// moments keep FP32 round-off of their own size instead of that of d.
//
// Requirements: nx a multiple of the 16-byte staging chunk (4 FP32 or 8
// 16-bit values), no interior solid mask (the scalar kernel covers both).
#pragma once

#include "tslb_step.cuh"

namespace tslb {

// ---- paired FP32 arithmetic: .x = column A, .y = column B ----
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
// a + s b for a compile-time sign s = +-1
template <int S>
__device__ __forceinline__ float2 addsgn(float2 a, float2 b) { return S > 0 ? add2(a, b) : sub2(a, b); }

// ---- tile geometry ----
constexpr int PH = 32;               // columns per half tile (one warp row)
constexpr int PX = 2 * PH;           // tile width in x
constexpr int PY = 8;                // tile rows, one warp each
constexpr int PTHR = PH * PY;        // threads per block
constexpr int CQ = PH + 2;           // pair nodes per coefficient row (x0-1 .. x0+32 and +32)
constexpr int CR = PY + 2;           // coefficient rows (y0-1 .. y0+PY)
constexpr int CN = CQ * CR;          // pair nodes of one coefficient plane
constexpr int NSP = NCOEF / 2 + 1;   // slot pairs: the 11 of the scalar tile with (c3, c4) split
                                     // into (c3, d) and (c4, 0)
constexpr int PRIM = CN - PTHR;      // pair nodes of the tile rim

template <int ES>   // element size of the stored state in bytes
struct PGeo {
    static constexpr int EPC = 16 / ES;            // elements per 16-byte chunk
    static constexpr int SW = PX + 2 * EPC;        // staged row: columns x0-EPC .. x0+PX+EPC-1
    static constexpr int NCH = SW / EPC;           // chunks per staged row
    static constexpr int MROWS = CR;               // staged moment rows y0-1 .. y0+PY
    static constexpr int PROWS = PY + 4;           // staged phi rows y0-2 .. y0+PY+1
    static constexpr int MAREA = MROWS * SW, PAREA = PROWS * SW;
    static constexpr int MCELLS = MROWS * NCH;     // 16-byte cells of one staged moment plane
    static constexpr int MGROUPS = PTHR / MCELLS;  // thread (g, cell) copies fields g, g + MGROUPS, ...
    static constexpr int MFIELDS = (NMOM + MGROUPS - 1) / MGROUPS;
    static constexpr int PCOPIES = PROWS * NCH;    // 16-byte cells of one staged phi plane
    static_assert(MGROUPS >= 1, "a staged moment plane has more cells than the block has threads");
    static_assert(PCOPIES <= PTHR, "a staged phi plane has more cells than the block has threads");
};

__host__ __device__ constexpr size_t pair_smem_bytes(int mode, int es) {
    return sizeof(float4) * 2 * NSP * CN + (size_t)es * 2 * NMOM * CR * (PX + 2 * (16 / es)) +
           (mode == TSLB_MODE_COLOUR ? (size_t)es * PRING * (PY + 4) * (PX + 2 * (16 / es)) : 0);
}

// Coefficients of P'(c) of a pair node (tslb_device.cuh node_coefs, paired).
// m: the node's moments (m[F_D] = rho - 1, m[F_PHI] = phi); g: colour-mode
// gradient of phi; U, V, W (phase field, single component): the equilibrium
// velocity and n the normal, formed per column by the caller; om: omega.
template <int MODE>
__device__ __forceinline__ void pair_coefs(const StepArgs& a, const float2* m, const float2* g, float2 omega, float2 U,
                                           float2 V, float2 W, float2 nx_, float2 ny_, float2 nz_, float2 A, float2 mg,
                                           float2* K) {
    const float2 d = m[F_D], rho = add2(bc2(1.f), d);
    const float2 u = m[F_U], v = m[F_V], w = m[F_W];
    const float2 pxx = m[F_XX], pxy = m[F_XY], pxz = m[F_XZ], pyy = m[F_YY], pyz = m[F_YZ], pzz = m[F_ZZ];
    const float2 om1 = sub2(bc2(1.f), omega);
    const float2 u2 = add2(u, u), v2 = add2(v, v), w2 = add2(w, w);
    // recursive third-order non-equilibrium moments a3 = u_a Pi_bc + perms
    const float2 a_xxy = fma2(u2, pxy, mul2(v, pxx));
    const float2 a_xxz = fma2(u2, pxz, mul2(w, pxx));
    const float2 a_xyy = fma2(v2, pxy, mul2(u, pyy));
    const float2 a_yyz = fma2(v2, pyz, mul2(w, pyy));
    const float2 a_xzz = fma2(w2, pxz, mul2(u, pzz));
    const float2 a_yzz = fma2(w2, pyz, mul2(v, pzz));
    const float2 a_xyz = fma2(u, pyz, fma2(v, pxz, mul2(w, pxy)));
    const float2 rU = mul2(rho, U), rV = mul2(rho, V), rW = mul2(rho, W);
    const float2 rUU = mul2(rU, U), rVV = mul2(rV, V), rWW = mul2(rW, W);
    const float2 rUV = mul2(rU, V), rUW = mul2(rU, W), rVW = mul2(rV, W);
    // full third-order coefficients: rho U_a U_b U_c + (1 - omega) a3
    const float2 t_xxy = fma2(om1, a_xxy, mul2(rUU, V));
    const float2 t_xxz = fma2(om1, a_xxz, mul2(rUU, W));
    const float2 t_xyy = fma2(om1, a_xyy, mul2(rVV, U));
    const float2 t_yyz = fma2(om1, a_yyz, mul2(rVV, W));
    const float2 t_xzz = fma2(om1, a_xzz, mul2(rWW, U));
    const float2 t_yzz = fma2(om1, a_yzz, mul2(rWW, V));
    const float2 t_xyz = fma2(om1, a_xyz, mul2(rUV, W));
    const float2 tr = add2(add2(pxx, pyy), pzz);
    const float2 ke = add2(add2(rUU, rVV), rWW);
    K[K_0] = mul2(bc2(-1.5f), fma2(om1, tr, ke));   // K_0 - d (the pull adds d_s - d_t)
    K[K_X] = fma2(bc2(3.f), rU, mul2(bc2(-4.5f), add2(t_xyy, t_xzz)));
    K[K_Y] = fma2(bc2(3.f), rV, mul2(bc2(-4.5f), add2(t_xxy, t_yzz)));
    K[K_Z] = fma2(bc2(3.f), rW, mul2(bc2(-4.5f), add2(t_xxz, t_yyz)));
    K[K_XX] = mul2(bc2(4.5f), fma2(om1, pxx, rUU));
    K[K_YY] = mul2(bc2(4.5f), fma2(om1, pyy, rVV));
    K[K_ZZ] = mul2(bc2(4.5f), fma2(om1, pzz, rWW));
    K[K_XY] = mul2(bc2(9.f), fma2(om1, pxy, rUV));
    K[K_XZ] = mul2(bc2(9.f), fma2(om1, pxz, rUW));
    K[K_YZ] = mul2(bc2(9.f), fma2(om1, pyz, rVW));
    K[K_XXY] = mul2(bc2(13.5f), t_xxy);
    K[K_XXZ] = mul2(bc2(13.5f), t_xxz);
    K[K_XYY] = mul2(bc2(13.5f), t_xyy);
    K[K_YYZ] = mul2(bc2(13.5f), t_yyz);
    K[K_XZZ] = mul2(bc2(13.5f), t_xzz);
    K[K_YZZ] = mul2(bc2(13.5f), t_yzz);
    K[K_XYZ] = mul2(bc2(27.f), t_xyz);
    const float2 phi = m[F_PHI];
    if (MODE == TSLB_MODE_COLOUR) {
        // force as population source 3 w c.F (recursive_colorTSLB3D.f90:776)
        K[K_X] = fma2(bc2(3.f), bc2(a.force[0]), K[K_X]);
        K[K_Y] = fma2(bc2(3.f), bc2(a.force[1]), K[K_Y]);
        K[K_Z] = fma2(bc2(3.f), bc2(a.force[2]), K[K_Z]);
        // perturbation (A/2)|g| [w (c.n)^2 - B_i] (A = 0 off the interface)
        const float2 h = mul2(mul2(bc2(0.5f), A), mg);
        const float2 h2 = add2(h, h);
        K[K_0] = sub2(K[K_0], h);
        K[K_XX] = fma2(mul2(h, nx_), nx_, K[K_XX]);
        K[K_YY] = fma2(mul2(h, ny_), ny_, K[K_YY]);
        K[K_ZZ] = fma2(mul2(h, nz_), nz_, K[K_ZZ]);
        K[K_XY] = fma2(mul2(h2, nx_), ny_, K[K_XY]);
        K[K_XZ] = fma2(mul2(h2, nx_), nz_, K[K_XZ]);
        K[K_YZ] = fma2(mul2(h2, ny_), nz_, K[K_YZ]);
        // recolouring 2 beta (rhoA rhoB / rho) n (published cos theta form)
        const float2 bb = mul2(mul2(bc2(0.5f * a.beta), rho), fma2(neg2(phi), phi, bc2(1.f)));
        K[K_C0] = phi;
        K[K_C1] = mul2(bb, nx_);
        K[K_C2] = mul2(bb, ny_);
        K[K_C3] = mul2(bb, nz_);
        K[K_C4] = mul2(mul2(A, bc2(1.f / 3.f)), mg);   // rest population: B_0 = -10/27 instead of w_0
    } else if (MODE == TSLB_MODE_PHASEFIELD) {
        // D3Q7 phase field: g_q = G0 + e_q.G1 (recursive_2c_TSLB3D.f90:808-831)
        const float2 sh = mul2(mul2(bc2(0.125f * a.sharp), phi), sub2(bc2(1.f), phi));
        const float2 p3 = mul2(bc2(0.375f), phi);
        K[K_C0] = mul2(bc2(0.125f), phi);
        K[K_C1] = fma2(p3, u, mul2(sh, nx_));
        K[K_C2] = fma2(p3, v, mul2(sh, ny_));
        K[K_C3] = fma2(p3, w, mul2(sh, nz_));
        K[K_C4] = bc2(0.f);
    } else {
        K[K_C0] = bc2(0.f); K[K_C1] = bc2(0.f); K[K_C2] = bc2(0.f); K[K_C3] = bc2(0.f); K[K_C4] = bc2(0.f);
    }
}

// Gradient 3 sum_i p_i c_i phi(x + c_i) of a pair node from the staged phi
// planes z-1, z, z+1 (pm, p0, pp point at column A; column B is PH further).
template <int SWv, class T>
__device__ __forceinline__ void pair_grad(const T* pm, const T* p0, const T* pp, float2 g[3]) {
    auto P = [&](const T* pl, int dx, int dy) {
        return make_float2(Stor<T>::ld(pl[dy * SWv + dx]), Stor<T>::ld(pl[dy * SWv + dx + PH]));
    };
    const float2 x1 = sub2(P(p0, 1, 0), P(p0, -1, 0));
    const float2 x2 = sub2(add2(add2(P(p0, 1, 1), P(p0, 1, -1)), add2(P(pp, 1, 0), P(pm, 1, 0))),
                           add2(add2(P(p0, -1, 1), P(p0, -1, -1)), add2(P(pp, -1, 0), P(pm, -1, 0))));
    const float2 x3 = sub2(add2(add2(P(pp, 1, 1), P(pp, 1, -1)), add2(P(pm, 1, 1), P(pm, 1, -1))),
                           add2(add2(P(pp, -1, 1), P(pp, -1, -1)), add2(P(pm, -1, 1), P(pm, -1, -1))));
    const float2 y1 = sub2(P(p0, 0, 1), P(p0, 0, -1));
    const float2 y2 = sub2(add2(add2(P(p0, 1, 1), P(p0, -1, 1)), add2(P(pp, 0, 1), P(pm, 0, 1))),
                           add2(add2(P(p0, 1, -1), P(p0, -1, -1)), add2(P(pp, 0, -1), P(pm, 0, -1))));
    const float2 y3 = sub2(add2(add2(P(pp, 1, 1), P(pp, -1, 1)), add2(P(pm, 1, 1), P(pm, -1, 1))),
                           add2(add2(P(pp, 1, -1), P(pp, -1, -1)), add2(P(pm, 1, -1), P(pm, -1, -1))));
    const float2 z1 = sub2(P(pp, 0, 0), P(pm, 0, 0));
    const float2 z2 = sub2(add2(add2(P(pp, 1, 0), P(pp, -1, 0)), add2(P(pp, 0, 1), P(pp, 0, -1))),
                           add2(add2(P(pm, 1, 0), P(pm, -1, 0)), add2(P(pm, 0, 1), P(pm, 0, -1))));
    const float2 z3 = sub2(add2(add2(P(pp, 1, 1), P(pp, 1, -1)), add2(P(pp, -1, 1), P(pp, -1, -1))),
                           add2(add2(P(pm, 1, 1), P(pm, 1, -1)), add2(P(pm, -1, 1), P(pm, -1, -1))));
    constexpr float c1 = 3.f * wclass(1), c2 = 3.f * wclass(2), c3 = 3.f * wclass(3);
    g[0] = fma2(bc2(c1), x1, fma2(bc2(c2), x2, mul2(bc2(c3), x3)));
    g[1] = fma2(bc2(c1), y1, fma2(bc2(c2), y2, mul2(bc2(c3), y3)));
    g[2] = fma2(bc2(c1), z1, fma2(bc2(c2), z2, mul2(bc2(c3), z3)));
}

// P' - d_t = Q0 + cz Q1 + cz^2 Q2 + (d_s - d_t) of the directions (CXv, CYv,
// cz) from one source pair node (K: its slot pair 0; slot pair p at K[p CN]),
// for the targets of the planes cz = -1, 0, 1 (deviations dm, d0, dp), and
// the colour slots the pull uses: C[0] phi (or G0), C[1] Bx, C[2] By, C[3]
// Bz, C[4] the rest population's delta (the centre source only).
template <int CXv, int CYv>
__device__ __forceinline__ void pair_eval(const float4* __restrict__ K, float2 dm, float2 d0, float2 dp, float2& Pm,
                                          float2& P0, float2& Pp, float2* C) {
    const float4 k0z = K[0];              // (0 - d, z)
    const float4 kzz = K[CN];             // (zz, c0)
    float2 q0 = lo2(k0z), q1 = hi2(k0z), q2 = lo2(kzz);
    C[0] = hi2(kzz);
    if (CXv) {
        const float4 kx = K[2 * CN];      // (x, xx)
        const float4 kxz = K[3 * CN];     // (xz, xxz)
        const float4 kxzz = K[4 * CN];    // (xzz, c1)
        q0 = add2(q0, addsgn<CXv>(hi2(kx), lo2(kx)));
        q1 = add2(q1, addsgn<CXv>(hi2(kxz), lo2(kxz)));
        q2 = addsgn<CXv>(q2, lo2(kxzz));
        C[1] = hi2(kxzz);
    }
    if (CYv) {
        const float4 ky = K[5 * CN];      // (y, yy)
        const float4 kyz = K[6 * CN];     // (yz, yyz)
        const float4 kyzz = K[7 * CN];    // (yzz, c2)
        q0 = add2(q0, addsgn<CYv>(hi2(ky), lo2(ky)));
        q1 = add2(q1, addsgn<CYv>(hi2(kyz), lo2(kyz)));
        q2 = addsgn<CYv>(q2, lo2(kyzz));
        C[2] = hi2(kyzz);
    }
    if (CXv && CYv) {
        const float4 kxy = K[8 * CN];     // (xy, xyz)
        const float4 kxxy = K[9 * CN];    // (xxy, xyy)
        // cx cy K_xy + cy K_xxy + cx K_xyy = cy ((K_xxy + cx K_xy) + cx cy K_xyy)
        q0 = addsgn<CYv>(q0, addsgn<CXv * CYv>(addsgn<CXv>(lo2(kxxy), lo2(kxy)), hi2(kxxy)));
        q1 = addsgn<CXv * CYv>(q1, hi2(kxy));
    }
    const float4 kc = K[10 * CN];         // (c3, d)
    C[3] = lo2(kc);
    const float2 ds = hi2(kc);
    if (CXv == 0 && CYv == 0) C[4] = lo2(K[11 * CN]);   // (c4, -)
    const float2 t = add2(q0, q2);
    Pm = add2(sub2(t, q1), sub2(ds, dm));
    P0 = add2(q0, sub2(ds, d0));
    Pp = add2(add2(t, q1), sub2(ds, dp));
}

// Moments of the three populations of one (cy, cz) group -- directions
// (+1, cy, cz), (0, cy, cz), (-1, cy, cz) with unweighted P' values a, c0,
// b -- through S = a + b, D = a - b, T = S + (wC/wE) c0, each accumulated
// with the weight wE.  FIRST: the group is the first to touch this target
// plane, so it assigns instead of adding.
template <int CYv, int CZv, bool FIRST>
__device__ __forceinline__ void pair_acc_group(float2* acc, float2 a, float2 c0, float2 b) {
    constexpr float wE = w1d(1) * w1d(CYv) * w1d(CZv), rC = w1d(0) / w1d(1);
    const float2 S = add2(a, b), D = sub2(a, b), T = fma2(bc2(rC), c0, S);
    const float2 pe = bc2(wE), ne = bc2(-wE);
    auto put = [&](int i, float2 wv, float2 x) { acc[i] = FIRST ? mul2(wv, x) : fma2(wv, x, acc[i]); };
    put(A_RHO, pe, T);
    put(A_JX, pe, D);
    put(A_XX, pe, S);
    if (CYv) { put(A_JY, CYv > 0 ? pe : ne, T); put(A_YY, pe, T); put(A_XY, CYv > 0 ? pe : ne, D); }
    if (CZv) { put(A_JZ, CZv > 0 ? pe : ne, T); put(A_ZZ, pe, T); put(A_XZ, CZv > 0 ? pe : ne, D); }
    if (CYv && CZv) put(A_YZ, CYv * CZv > 0 ? pe : ne, T);
}

// colour of one (cy, cz) group as an increment over the target's phi (the
// scalar col_group, paired)
template <int CYv, int CZv, bool FIRST>
__device__ __forceinline__ void pair_col_group(float2* acc, float2 ha, float2 hc, float2 hb, float2 Ex, float2 Ey,
                                               float2 Ez, float2 By0, float2 Bz0) {
    constexpr int cE = 1 + CYv * CYv + CZv * CZv, cC = CYv * CYv + CZv * CZv;
    constexpr float wE = w1d(1) * w1d(CYv) * w1d(CZv), wC = w1d(0) * w1d(CYv) * w1d(CZv);
    float2 r = Ex;
    if (CYv) r = addsgn<CYv>(r, Ey);
    if (CZv) r = addsgn<CZv>(r, Ez);
    float2 v = fma2(bc2(wE), add2(ha, hb), mul2(bc2(wC), hc));
    v = fma2(bc2(wE * invlen(cE)), r, v);
    if (cC) {
        float2 rc;
        if (CYv && CZv) rc = addsgn<CZv>(CYv > 0 ? By0 : neg2(By0), Bz0);
        else if (CYv) rc = CYv > 0 ? By0 : neg2(By0);
        else rc = CZv > 0 ? Bz0 : neg2(Bz0);
        v = fma2(bc2(wC * invlen(cC)), rc, v);
    }
    acc[A_COL] = FIRST ? v : add2(acc[A_COL], v);
}

// All populations that leave source row y - CYv of plane s toward the
// column pair's targets in planes s-1 (accm), s (acc0), s+1 (accp).  Kc:
// the target pair node's slot pair 0.  FIRST: row -1 is the first to write
// accp.  phm, ph0, php: the targets' own phi (colour mode).
template <int MODE, int CYv, bool FIRST>
__device__ __forceinline__ void pair_pull_row(const float4* __restrict__ Kc, float2* accm, float2* acc0, float2* accp,
                                              float2 dm, float2 d0, float2 dp, float2 phm, float2 ph0, float2 php) {
    const float4* Ka = Kc - CYv * CQ - 1;   // source of cx = +1 (x - 1)
    const float4* Kz = Kc - CYv * CQ;       // source of cx = 0
    const float4* Kb = Kc - CYv * CQ + 1;   // source of cx = -1 (x + 1)
    float2 am, a0, ap, cm, c0, cp, bm, b0, bp;
    float2 Ca[5], Cz[5], Cb[5];
    pair_eval<1, CYv>(Ka, dm, d0, dp, am, a0, ap, Ca);
    pair_eval<0, CYv>(Kz, dm, d0, dp, cm, c0, cp, Cz);
    pair_eval<-1, CYv>(Kb, dm, d0, dp, bm, b0, bp, Cb);
    pair_acc_group<CYv, -1, false>(accm, am, cm, bm);
    pair_acc_group<CYv, 0, false>(acc0, a0, c0, b0);
    pair_acc_group<CYv, 1, FIRST>(accp, ap, cp, bp);
    if (MODE == TSLB_MODE_COLOUR) {
        const float2 pa = Ca[0], pz = Cz[0], pb = Cb[0];
        // recolouring sums over the cx = +1 / -1 sources
        const float2 Ex = sub2(Ca[1], Cb[1]);
        const float2 Ey = CYv ? add2(Ca[2], Cb[2]) : bc2(0.f);
        const float2 Ez = add2(Ca[3], Cb[3]);
        const float2 By0 = CYv ? Cz[2] : bc2(0.f);
        const float2 Bz0 = Cz[3];
        // (phi_s - phi_t)(1 + P') = (phi_s - phi_t)(rho_t + (P' - d_t)) for the three
        // sources and the three target planes
        const float2 rm = add2(bc2(1.f), dm), r0 = add2(bc2(1.f), d0), rp = add2(bc2(1.f), dp);
        auto h = [](float2 ps, float2 pt, float2 rt, float2 P) { return mul2(sub2(ps, pt), add2(rt, P)); };
        pair_col_group<CYv, -1, false>(accm, h(pa, phm, rm, am), h(pz, phm, rm, cm), h(pb, phm, rm, bm), Ex, Ey, Ez, By0, Bz0);
        pair_col_group<CYv, 0, false>(acc0, h(pa, ph0, r0, a0), h(pz, ph0, r0, c0), h(pb, ph0, r0, b0), Ex, Ey, Ez, By0, Bz0);
        pair_col_group<CYv, 1, FIRST>(accp, h(pa, php, rp, ap), h(pz, php, rp, cp), h(pb, php, rp, bp), Ex, Ey, Ez, By0, Bz0);
        // rest population: f_0 += delta0 (the perturbation's B_0); no colour increment
        if (CYv == 0) acc0[A_RHO] = add2(acc0[A_RHO], Cz[4]);
    } else if (MODE == TSLB_MODE_PHASEFIELD) {
        // phase field g (D3Q7): axis directions and the rest population
        if (CYv == 0) {
            const float2 g0 = Cz[0], gz = Cz[3];
            accm[A_COL] = add2(accm[A_COL], sub2(g0, gz));            // q = 6, (0,0,-1)
            accp[A_COL] = add2(accp[A_COL], add2(g0, gz));            // q = 5, (0,0,+1)
            acc0[A_COL] = add2(acc0[A_COL], add2(Ca[0], Ca[1]));      // q = 1 from x - 1
            acc0[A_COL] = add2(acc0[A_COL], sub2(Cb[0], Cb[1]));      // q = 2 from x + 1
            acc0[A_COL] = fma2(bc2(2.f), g0, acc0[A_COL]);            // q = 0: p0g phi = 2 G0
        } else {
            acc0[A_COL] = add2(acc0[A_COL], addsgn<CYv>(Cz[0], Cz[2]));  // q = 3 / 4
        }
    }
}

// One block's work: tile (bx, by) of 64 x 8 columns and z chunk bz of lattice a.
template <int MODE, class T, bool TAU = false>
__device__ __forceinline__ void pair_block(const StepArgs& a, int bx, int by, int bz) {
    using G = PGeo<sizeof(T)>;
    constexpr int SW = G::SW, EPC = G::EPC, MAREA = G::MAREA, PAREA = G::PAREA;
    extern __shared__ float4 smem4[];
    float4* coef_base = smem4;                                           // [2][NSP][CN]
    T* mst = reinterpret_cast<T*>(coef_base + 2 * NSP * CN);             // [2][NMOM][MROWS][SW]
    T* phis = mst + 2 * NMOM * MAREA;                                    // colour: [PRING][PROWS][SW]
    const T* gin = reinterpret_cast<const T*>(a.in);
    T* gout = reinterpret_cast<T*>(a.out);
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * PH + lane;
    const int x0 = bx * PX, y0 = by * PY;
    const int z0 = a.zt0 + bz * a.zchunk;
    const int z1 = min(z0 + a.zchunk, a.zt1);
    const int XA = x0 + lane, XB = XA + PH, Y = y0 + wy;
    const bool actA = XA < a.nx && Y < a.ny, actB = XB < a.nx && Y < a.ny;
    const bool xper = a.face[0].kind == TSLB_BC_PERIODIC;
    const bool yper = a.face[2].kind == TSLB_BC_PERIODIC;
    const bool zper = a.face[4].kind == TSLB_BC_PERIODIC;
    const long long plane = (long long)a.nx * a.ny;

    // faces each target column touches (z faces are added per plane)
    unsigned maskA = 0, maskB = 0;
    if (!xper) {
        if (XA == 0) maskA |= 1u;
        if (XA == a.nx - 1) maskA |= 2u;
        if (XB == a.nx - 1) maskB |= 2u;
    }
    if (!yper) {
        if (Y == 0) { maskA |= 4u; maskB |= 4u; }
        if (Y == a.ny - 1) { maskA |= 8u; maskB |= 8u; }
    }

    // pair nodes of this thread: its own (row wy + 1, q = lane + 1) and, for
    // tid < PRIM, one rim node
    const bool has_rim = tid < PRIM;
    int r1, q1;
    {
        const int k = has_rim ? tid : 0;
        if (k < CQ) { r1 = 0; q1 = k; }
        else if (k < 2 * CQ) { r1 = CR - 1; q1 = k - CQ; }
        else if (k < 2 * CQ + PY) { r1 = 1 + (k - 2 * CQ); q1 = 0; }
        else { r1 = 1 + (k - 2 * CQ - PY); q1 = CQ - 1; }
    }
    const int r0 = wy + 1, q0 = lane + 1;
    const XYNode nA0 = xy_node(a, x0 + q0 - 1, y0 - 1 + r0, xper, yper);
    const XYNode nB0 = xy_node(a, x0 + q0 - 1 + PH, y0 - 1 + r0, xper, yper);
    const XYNode nA1 = xy_node(a, x0 + q1 - 1, y0 - 1 + r1, xper, yper);
    const XYNode nB1 = xy_node(a, x0 + q1 - 1 + PH, y0 - 1 + r1, xper, yper);
    // staged position (column A) of a pair node: moments row r, column q - 1 + EPC; phi row r + 1
    const int mi0 = r0 * SW + q0 - 1 + EPC, mi1 = r1 * SW + q1 - 1 + EPC;
    const int ci0 = r0 * CQ + q0, ci1 = r1 * CQ + q1;

    auto zwrap = [&](int z, bool& out) {
        out = false;
        if (z < 0 || z >= a.nz) { if (zper) return wrapi(z, a.nz); out = true; }
        return z;
    };

    // ---- staging of phi planes (colour mode): thread tid < PCOPIES owns cell (row, chunk) ----
    int pch_off = 0, pch_dst = 0;
    bool pch_out = true;
    if (MODE == TSLB_MODE_COLOUR && tid < G::PCOPIES) {
        const int row = tid / G::NCH, ch = tid % G::NCH;
        const XYNode nd = xy_node(a, x0 - EPC + EPC * ch, y0 - 2 + row, xper, yper);
        pch_off = nd.off;
        pch_out = nd.out;
        pch_dst = row * SW + EPC * ch;
    }
    const T* pg0 = gin + F_PHI * a.N + pch_off;
    const unsigned ps0 = (unsigned)__cvta_generic_to_shared(phis) + (unsigned)(pch_dst * sizeof(T));
    auto stage_phi = [&](int z) {
        if (tid >= G::PCOPIES) return;
        bool zout;
        const int gz = zwrap(z, zout);
        if (!pch_out && !zout) {
            cp_async16s(ps0 + (unsigned)((z & (PRING - 1)) * (PAREA * (int)sizeof(T))), pg0 + (long long)gz * plane);
        } else {
            T* dst = phis + (z & (PRING - 1)) * PAREA + pch_dst;
            const int row = tid / G::NCH, ch = tid % G::NCH;
#pragma unroll
            for (int e = 0; e < EPC; ++e)
                dst[e] = cvt_out<T>(phi_at<T>(a, x0 - EPC + EPC * ch + e, y0 - 2 + row, z), a, F_PHI);
        }
    };

    // ---- staging of the 10 non-phi moments: thread tid < MGROUPS MCELLS owns one cell ----
    int mcell_dst = 0, mcell_off = 0, mfg = 0;
    bool mcell_ok = false;
    if (tid < G::MGROUPS * G::MCELLS) {
        const int cell = tid % G::MCELLS, row = cell / G::NCH, ch = cell % G::NCH;
        mfg = tid / G::MCELLS;
        const XYNode nd = xy_node(a, x0 - EPC + EPC * ch, y0 - 1 + row, xper, yper);
        mcell_off = nd.off;
        mcell_ok = !nd.out;
        mcell_dst = mfg * MAREA + row * SW + EPC * ch;
    }
    const T* mg0 = gin + mfg * a.N + mcell_off;
    const long long mfstride = (long long)G::MGROUPS * a.N;
    const unsigned ms0 = (unsigned)__cvta_generic_to_shared(mst) + (unsigned)(mcell_dst * sizeof(T));
    auto stage_mom = [&](int z) {
        bool zout;
        const int gz = zwrap(z, zout);
        if (zout || !mcell_ok) return;
        const unsigned d = ms0 + (unsigned)((z & 1) * (NMOM * MAREA * (int)sizeof(T)));
        const T* g = mg0 + (long long)gz * plane;
#pragma unroll
        for (int k = 0; k < G::MFIELDS; ++k) {
            if (G::MGROUPS * G::MFIELDS == NMOM || mfg + k * G::MGROUPS < NMOM)
                cp_async16s(d + (unsigned)(k * G::MGROUPS * MAREA * (int)sizeof(T)), g + k * mfstride);
        }
    };

    if (MODE == TSLB_MODE_COLOUR) {
        stage_phi(z0 - 2);
        stage_phi(z0 - 1);
        stage_phi(z0);
    }
    stage_mom(z0 - 1);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    // coefficients of one pair node of source plane s (nodes behind a face,
    // or in a solid plane, send nothing)
    auto coef_node = [&](int s, int gz, const XYNode& nA, const XYNode& nB, int mi, int ci) {
        const T* ms = mst + (s & 1) * (NMOM * MAREA) + mi;
        float2 m[NF];
#pragma unroll
        for (int f = 0; f < NMOM; ++f)
            m[f] = make_float2(cvt_in<T>(ms[f * MAREA], a, f), cvt_in<T>(ms[f * MAREA + PH], a, f));
        float2 g[3] = {bc2(0.f), bc2(0.f), bc2(0.f)};
        float2 omega, U, V, W, nx_ = bc2(0.f), ny_ = bc2(0.f), nz_ = bc2(0.f), A = bc2(0.f), mg = bc2(0.f);
        if (MODE == TSLB_MODE_COLOUR) {
            const int pi = mi + SW;
            const T* p0 = phis + (s & (PRING - 1)) * PAREA + pi;
            const T* pm = phis + ((s - 1) & (PRING - 1)) * PAREA + pi;
            const T* pp = phis + ((s + 1) & (PRING - 1)) * PAREA + pi;
            m[F_PHI] = make_float2(cvt_in<T>(p0[0], a, F_PHI), cvt_in<T>(p0[PH], a, F_PHI));
            pair_grad<SW>(pm, p0, pp, g);
            if constexpr (std::is_same<T, __half>::value) {
                const float2 is = bc2(a.iscale[F_PHI]);
                g[0] = mul2(g[0], is); g[1] = mul2(g[1], is); g[2] = mul2(g[2], is);
            }
            const float2 m2 = fma2(g[0], g[0], fma2(g[1], g[1], mul2(g[2], g[2])));
            const float thr2 = a.thr * a.thr;
            const bool ifA = m2.x > thr2, ifB = m2.y > thr2;
            const float rsA = rsqrtf(m2.x), rsB = rsqrtf(m2.y);
            mg = make_float2(ifA ? m2.x * rsA : 0.f, ifB ? m2.y * rsB : 0.f);
            const float2 inv = make_float2(ifA ? rsA : 0.f, ifB ? rsB : 0.f);
            nx_ = mul2(g[0], inv); ny_ = mul2(g[1], inv); nz_ = mul2(g[2], inv);
            // 1/nu = (rhoA/rho)/nu_a + (rhoB/rho)/nu_b ; omega = 2/(6 nu + 1) = 2q/(6 + q)
            const float2 q = fma2(m[F_PHI], bc2(0.5f * (a.inv_nu_a - a.inv_nu_b)), bc2(0.5f * (a.inv_nu_a + a.inv_nu_b)));
            const float2 q2 = add2(q, q);
            if (TAU) {
                // 1/omega = (6 + q)/(2q) + dtau
                const float dtA = __ldg(a.dtau + (long long)gz * plane + nA.off);
                const float dtB = __ldg(a.dtau + (long long)gz * plane + nB.off);
                const float2 den = fma2(q2, make_float2(dtA, dtB), add2(bc2(6.f), q));
                omega = make_float2(__fdividef(q2.x, den.x), __fdividef(q2.y, den.y));
            } else {
                const float2 den = add2(bc2(6.f), q);
                omega = make_float2(__fdividef(q2.x, den.x), __fdividef(q2.y, den.y));
            }
            const float sa = a.acoef * a.sigma;
            A = make_float2(ifA ? sa * omega.x : 0.f, ifB ? sa * omega.y : 0.f);
            U = m[F_U]; V = m[F_V]; W = m[F_W];
        } else if (MODE == TSLB_MODE_SINGLE) {
            // fused_TSLB_force_1c: equilibrium at the shifted velocity u + F
            omega = bc2(a.omega_pf);
            m[F_PHI] = bc2(1.f);
            U = add2(m[F_U], bc2(a.force[0]));
            V = add2(m[F_V], bc2(a.force[1]));
            W = add2(m[F_W], bc2(a.force[2]));
        } else {
            // phase field: normals of the separate normals pass, curvature where
            // phi (1 - phi) |n|^2 > 0.2, CSF velocity shift u + sigma kappa n + F
            omega = bc2(a.omega_pf);
            const long long idA = (long long)gz * plane + nA.off, idB = (long long)gz * plane + nB.off;
            const float phA = ld_field<T>(a, F_PHI, idA), phB = ld_field<T>(a, F_PHI, idB);
            m[F_PHI] = make_float2(phA, phB);
            float n[2][3];
            float sk[2];
            const long long ids[2] = {idA, idB};
            const float phs[2] = {phA, phB};
            const XYNode* nds[2] = {&nA, &nB};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                n[h][0] = __ldg(a.nrm + ids[h]);
                n[h][1] = __ldg(a.nrm + a.N + ids[h]);
                n[h][2] = __ldg(a.nrm + 2 * a.N + ids[h]);
                const float ind = phs[h] * (1.f - phs[h]) * (n[h][0] * n[h][0] + n[h][1] * n[h][1] + n[h][2] * n[h][2]);
                float curv = 0.f;
                if (ind > 0.2f) curv = curvature_at(a, nds[h]->off % a.nx, nds[h]->off / a.nx, gz);
                sk[h] = a.sigma * curv;
            }
            nx_ = make_float2(n[0][0], n[1][0]);
            ny_ = make_float2(n[0][1], n[1][1]);
            nz_ = make_float2(n[0][2], n[1][2]);
            const float2 skv = make_float2(sk[0], sk[1]);
            U = add2(fma2(skv, nx_, m[F_U]), bc2(a.force[0]));
            V = add2(fma2(skv, ny_, m[F_V]), bc2(a.force[1]));
            W = add2(fma2(skv, nz_, m[F_W]), bc2(a.force[2]));
        }
        float2 K[NCOEF];
        pair_coefs<MODE>(a, m, g, omega, U, V, W, nx_, ny_, nz_, A, mg, K);
        float2 dn = m[F_D];
        if (nA.out) {
#pragma unroll
            for (int c = 0; c < NCOEF; ++c) K[c].x = 0.f;
            dn.x = 0.f;
        }
        if (nB.out) {
#pragma unroll
            for (int c = 0; c < NCOEF; ++c) K[c].y = 0.f;
            dn.y = 0.f;
        }
        float4* dst = coef_base + (s & 1) * (NSP * CN) + ci;
#pragma unroll
        for (int p = 0; p < K_C3 / 2; ++p) dst[p * CN] = make_float4(K[2 * p].x, K[2 * p].y, K[2 * p + 1].x, K[2 * p + 1].y);
        dst[10 * CN] = make_float4(K[K_C3].x, K[K_C3].y, dn.x, dn.y);
        dst[11 * CN] = make_float4(K[K_C4].x, K[K_C4].y, 0.f, 0.f);
    };

    // staged-phi offset of the thread's own target columns (row wy + 2)
    const int pown = (wy + 2) * SW + lane + EPC;
    auto own_phi = [&](int z) {
        const T* p = phis + (z & (PRING - 1)) * PAREA + pown;
        return make_float2(cvt_in<T>(p[0], a, F_PHI), cvt_in<T>(p[PH], a, F_PHI));
    };

    // the targets' own d = rho - 1 in plane z, from the staged moments (row wy + 1)
    const int mown = (wy + 1) * SW + lane + EPC;
    auto own_d = [&](int z) {
        const T* p = mst + (z & 1) * (NMOM * MAREA) + F_D * MAREA + mown;
        return make_float2(cvt_in<T>(p[0], a, F_D), cvt_in<T>(p[PH], a, F_D));
    };

    // one source plane s with target accumulators M (s-1), Z (s), P (s+1) and
    // the targets' deviations dM, dZ (set by the two previous planes) and dP
    auto body = [&](int s, float2* M, float2* Z, float2* P, float2& dM, float2& dZ, float2& dP) {
        const bool more = s < z1;
        // ---- 0. prefetch: phi of plane s+2, moments of plane s+1 ----
        if (MODE == TSLB_MODE_COLOUR && more) stage_phi(s + 2);
        if (more) stage_mom(s + 1);
        cp_async_commit();
        // ---- 1. coefficients of source plane s ----
        bool zsolid;
        const int gz = zwrap(s, zsolid);
        if (!zsolid) {
            coef_node(s, gz, nA0, nB0, mi0, ci0);
            if (has_rim) coef_node(s, gz, nA1, nB1, mi1, ci1);
        }
        // the copies issued above land before the barrier, which publishes them
        // together with the coefficients
        cp_async_wait<0>();
        __syncthreads();
        // ---- 2. pull ----
        // d of target plane s+1 (staged with plane s+1's moments; unused when
        // that plane lies behind a z face)
        dP = own_d(s + 1);
        if (zsolid) {
#pragma unroll
            for (int i = 0; i < NACC; ++i) P[i] = bc2(0.f);
        } else {
            const float4* Kc = coef_base + (s & 1) * (NSP * CN) + (wy + 1) * CQ + (lane + 1);
            float2 phm = bc2(0.f), ph0 = bc2(0.f), php = bc2(0.f);
            if (MODE == TSLB_MODE_COLOUR) { phm = own_phi(s - 1); ph0 = own_phi(s); php = own_phi(s + 1); }
            if (MODE != TSLB_MODE_COLOUR) P[A_COL] = bc2(0.f);
            pair_pull_row<MODE, -1, true>(Kc, M, Z, P, dM, dZ, dP, phm, ph0, php);
            pair_pull_row<MODE, 0, false>(Kc, M, Z, P, dM, dZ, dP, phm, ph0, php);
            pair_pull_row<MODE, 1, false>(Kc, M, Z, P, dM, dZ, dP, phm, ph0, php);
        }
        // ---- 3. populations from behind non-periodic faces, target plane s ----
        if (s >= z0 && s < z1) {
            unsigned zmask = 0;
            if (!zper && s == 0) zmask |= 16u;
            if (!zper && s == a.nz - 1) zmask |= 32u;
            const unsigned mA = actA ? (maskA | zmask) : 0u, mB = actB ? (maskB | zmask) : 0u;
            if (mA | mB) {
                const float4* Kc = coef_base + (s & 1) * (NSP * CN) + (wy + 1) * CQ + (lane + 1);
#pragma unroll 1
                for (int h = 0; h < 2; ++h) {
                    const unsigned mk = h ? mB : mA;
                    if (!mk) continue;
                    float Kp[NCOEF], acc[NACC];
#pragma unroll
                    for (int c = 0; c < K_C3; c += 2) {
                        const float4 v = Kc[(c >> 1) * CN];
                        Kp[c] = h ? v.y : v.x;
                        Kp[c + 1] = h ? v.w : v.z;
                    }
                    {
                        const float4 v3 = Kc[10 * CN], v4 = Kc[11 * CN];   // (c3, d), (c4, -)
                        Kp[K_C3] = h ? v3.y : v3.x;
                        Kp[K_C4] = h ? v4.y : v4.x;
                    }
#pragma unroll
                    for (int i = 0; i < NACC; ++i) acc[i] = h ? Z[i].y : Z[i].x;
                    boundary_target_k<MODE, T, TAU, false, true>(a, Kp, mk, h ? XB : XA, Y, s, acc, h ? dZ.y : dZ.x);
#pragma unroll
                    for (int i = 0; i < NACC; ++i) { if (h) Z[i].y = acc[i]; else Z[i].x = acc[i]; }
                }
            }
        }
        // ---- 4. target plane s-1 is complete ----
        const int t = s - 1;
        if (t >= z0 && t < z1 && (actA || actB)) {
            // M[A_RHO] = d_new - d_t; the second moments collected P' - d_t too, so
            // Pi_aa = M_aa - (d_new - d_t)/3 - rho u_a u_a
            const float2 d = add2(dM, M[A_RHO]), rho = add2(bc2(1.f), d);
            const float2 inv = make_float2(1.f / rho.x, 1.f / rho.y);
            const float2 u = mul2(M[A_JX], inv), v = mul2(M[A_JY], inv), w = mul2(M[A_JZ], inv);
            const float2 d3 = mul2(M[A_RHO], bc2(1.f / 3.f));
            const float2 ru = neg2(mul2(rho, u)), rv = neg2(mul2(rho, v)), rw = neg2(mul2(rho, w));
            float2 o[NF];
            o[F_D] = d;
            o[F_U] = u; o[F_V] = v; o[F_W] = w;
            o[F_XX] = fma2(ru, u, sub2(M[A_XX], d3));
            o[F_YY] = fma2(rv, v, sub2(M[A_YY], d3));
            o[F_ZZ] = fma2(rw, w, sub2(M[A_ZZ], d3));
            o[F_XY] = fma2(ru, v, M[A_XY]);
            o[F_XZ] = fma2(ru, w, M[A_XZ]);
            o[F_YZ] = fma2(rv, w, M[A_YZ]);
            // colour mode: phi_t + (colour increment) / rho
            o[F_PHI] = MODE == TSLB_MODE_COLOUR ? fma2(M[A_COL], inv, own_phi(t)) : M[A_COL];
            constexpr int nout = MODE == TSLB_MODE_SINGLE ? F_PHI : NF;
            const long long rowoff = (long long)t * plane + (long long)Y * a.nx;
            T* poA = gout + rowoff + XA;
            float2 chk = bc2(0.f);
            if constexpr (sizeof(T) == 2) {
                // 16-bit storage: both columns of a field in one stochastically rounded
                // conversion, seeded by the node (column A) and the step
                const unsigned int hnode = sr_node((unsigned int)(rowoff + (long long)a.zoff * plane + XA), a.sr_step);
#pragma unroll
                for (int f = 0; f < nout; ++f) {
                    float2 val = o[f];
                    if constexpr (std::is_same<T, __half>::value) val = mul2(val, bc2(a.scale[f]));
                    unsigned int pk;
                    if (a.sr) {
                        const unsigned int rb = sr_field(hnode, f);
                        if constexpr (std::is_same<T, __half>::value)
                            asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(pk) : "f"(val.y), "f"(val.x), "r"(rb));
                        else
                            asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(pk) : "f"(val.y), "f"(val.x), "r"(rb));
                    } else {
                        if constexpr (std::is_same<T, __half>::value)
                            asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(pk) : "f"(val.y), "f"(val.x));
                        else
                            asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(pk) : "f"(val.y), "f"(val.x));
                    }
                    const unsigned short lo = (unsigned short)(pk & 0xFFFFu), hi = (unsigned short)(pk >> 16);
                    T sA, sB;
                    if constexpr (std::is_same<T, __half>::value) { sA = __ushort_as_half(lo); sB = __ushort_as_half(hi); }
                    else { sA = __ushort_as_bfloat16(lo); sB = __ushort_as_bfloat16(hi); }
                    if (actA) poA[f * a.N] = sA;
                    if (actB) poA[f * a.N + PH] = sB;
                    chk = add2(chk, make_float2(Stor<T>::ld(sA), Stor<T>::ld(sB)));
                }
            } else {
#pragma unroll
                for (int f = 0; f < nout; ++f) {
                    if (actA) poA[f * a.N] = o[f].x;
                    if (actB) poA[f * a.N + PH] = o[f].y;
                    chk = add2(chk, o[f]);
                }
            }
            if ((actA && !isfinite(chk.x)) || (actB && !isfinite(chk.y))) atomicOr(a.flags, 1u);
        }
    };

    float2 accA[NACC], accB[NACC], accC[NACC];
#pragma unroll
    for (int i = 0; i < NACC; ++i) { accA[i] = bc2(0.f); accB[i] = bc2(0.f); accC[i] = bc2(0.f); }
    float2 dA = bc2(0.f), dB = own_d(z0 - 1), dC = bc2(0.f);
    int s = z0 - 1;
    for (; s + 2 <= z1; s += 3) {
        body(s, accA, accB, accC, dA, dB, dC);
        body(s + 1, accB, accC, accA, dB, dC, dA);
        body(s + 2, accC, accA, accB, dC, dA, dB);
    }
    if (s <= z1) { body(s, accA, accB, accC, dA, dB, dC); ++s; }
    if (s <= z1) body(s, accB, accC, accA, dB, dC, dA);
    cp_async_wait<0>();
}

template <int MODE, class T, bool TAU = false>
__global__ void __launch_bounds__(PTHR, 1) pair_kernel(const StepArgs a) {
    pair_block<MODE, T, TAU>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Ensemble step (the scalar ensemble_kernel of tslb_step.cuh with the paired
// block): blocks walk a work list of (lattice, 64 x 8 tile, z chunk) items,
// staging each lattice's arguments in shared memory when they move to it.
template <int MODE, class T>
__global__ void __launch_bounds__(PTHR, 1) ensemble_pair_kernel(const StepArgs* __restrict__ args,
                                                               const WorkItem* __restrict__ work, int nwork) {
    __shared__ StepArgs sa;
    int cur = -1;
    for (int it = blockIdx.x; it < nwork; it += gridDim.x) {
        const WorkItem w = work[it];
        if (w.dom != cur) {
            __syncthreads();
            const int words = (int)(sizeof(StepArgs) / sizeof(int));
            const int* src = reinterpret_cast<const int*>(args + w.dom);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.y * PH + threadIdx.x; i < words; i += PTHR) dst[i] = src[i];
            __syncthreads();
            cur = w.dom;
        }
        pair_block<MODE, T>(sa, w.bx, w.by, w.bz);
        __syncthreads();
    }
}

}  // namespace tslb
