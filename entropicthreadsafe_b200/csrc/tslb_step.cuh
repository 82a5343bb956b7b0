// tslb_step.cuh -- the fused pull step kernel.
//
// One CUDA block owns a TX x TY tile of (x, y) columns and a chunk of
// `zchunk` target planes.  It marches through the source planes
// s = z0-1 .. z1 of the chunk; for each:
//   0. the moments of plane s+1 and phi of plane s+2 are copied into shared
//      memory with cp.async (16-byte chunks when nx % 4 == 0), overlapping
//      the work on plane s;
//   1. every thread computes the coefficients of P'(c) (tslb_device.cuh) of
//      one or two nodes of plane s (the tile plus a one-node rim) into
//      shared memory (double buffered);
//   2. every thread pulls, for its own column, the 27 populations that
//      leave the 9 source nodes (x-ox, y-oy, s) and land on targets
//      (x, y, s-1), (x, y, s), (x, y, s+1), accumulating the targets'
//      moments in registers;
//   3. populations whose source lies behind a non-periodic face are
//      supplied at the target from its own node (bounce-back, regularized
//      velocity faces);
//   4. target plane s-1 is complete: its 11 moments are written out.
// One CTA barrier per plane, between 1 and 2: before it every thread waits
// for its own copies of step 0, so the barrier publishes the coefficients of
// plane s and the staged data of plane s+1 alike.
// Reading moments and writing moments is all the HBM traffic there is:
// the populations f, g of the reference (recursive_2c_TSLB3D.f90:54) never
// exist in memory.
#pragma once

#include "tslb_device.cuh"

namespace tslb {

// Coefficients live in shared memory as NQUAD planes of CAREA float4 and one
// plane of CAREA float2: node n's quad q is at float offset q * 4 CAREA + 4 n,
// its pair p5 at PAIR_OFF + 2 n.  A source loads each quad its directions use
// with one 16-byte load (lanes, consecutive x, read consecutive 16-byte
// words), or the half of q3 it uses with an 8-byte load.
constexpr int PAIR_OFF = 4 * NQUAD * CAREA;
// a node of the coefficient tile: its quad-plane and pair-plane addresses
struct CNode {
    const float* q;   // coef + 4 n
    const float* p;   // coef + PAIR_OFF + 2 n
    __device__ __forceinline__ CNode at(int dn) const { return CNode{q + 4 * dn, p + 2 * dn}; }
};
__device__ __forceinline__ CNode cnode(const float* coef, int n) { return CNode{coef + 4 * n, coef + PAIR_OFF + 2 * n}; }
__device__ __forceinline__ float comp4(const float4& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
// slot of node c: HALF reads the half of its quad that holds it (8 bytes)
template <bool HALF = false>
__device__ __forceinline__ float coef_at(const CNode& c, int slot) {
    if (slot >= 4 * NQUAD) {
        const float2 v = *reinterpret_cast<const float2*>(c.p);
        return slot & 1 ? v.y : v.x;
    }
    const float* b = c.q + (slot >> 2) * (4 * CAREA);
    if (HALF) {
        const float2 v = *reinterpret_cast<const float2*>(b + (slot & 2));
        return slot & 1 ? v.y : v.x;
    }
    return comp4(*reinterpret_cast<const float4*>(b), slot & 3);
}
// (single-component mode leaves the colour slots unset: stored, never read)
template <int MODE>
__device__ __forceinline__ void store_coefs(float* coef, int n, const float* K) {
#pragma unroll
    for (int q = 0; q < NQUAD; ++q)
        *reinterpret_cast<float4*>(coef + q * (4 * CAREA) + 4 * n) = make_float4(K[4 * q], K[4 * q + 1], K[4 * q + 2], K[4 * q + 3]);
    *reinterpret_cast<float2*>(coef + PAIR_OFF + 2 * n) = make_float2(K[4 * NQUAD], K[4 * NQUAD + 1]);
}

// P' = Q0 + cz Q1 + cz^2 Q2 of the directions (CXv, CYv, cz), cz = -1, 0, 1,
// of the source at coefficient node Kp
template <int CXv, int CYv>
struct Src {
    CNode Kp;
    // q3 is read whole only by sources that use both of its halves
    __device__ __forceinline__ float L(int slot) const {
        return (slot >> 2) == 3 && !(CXv && CYv) ? coef_at<true>(Kp, slot) : coef_at<false>(Kp, slot);
    }
    __device__ __forceinline__ void eval(float& Pm, float& P0, float& Pp) const {
        float q0 = L(K_0);
        if (CXv) q0 += CXv * L(K_X) + L(K_XX);
        if (CYv) q0 += CYv * L(K_Y) + L(K_YY);
        if (CXv && CYv) q0 += (CXv * CYv) * L(K_XY) + CYv * L(K_XXY) + CXv * L(K_XYY);
        float q1 = L(K_Z);
        if (CXv) q1 += CXv * L(K_XZ) + L(K_XXZ);
        if (CYv) q1 += CYv * L(K_YZ) + L(K_YYZ);
        if (CXv && CYv) q1 += (CXv * CYv) * L(K_XYZ);
        float q2 = L(K_ZZ);
        if (CXv) q2 += CXv * L(K_XZZ);
        if (CYv) q2 += CYv * L(K_YZZ);
        const float t = q0 + q2;
        Pm = t - q1;
        P0 = q0;
        Pp = t + q1;
    }
};

// The mirror sources of cx = +1 and cx = -1 (same cy) evaluated together as
// one float2 on the paired FP32 instructions of sm_100 (x: cx = +1, y: cx = -1);
// the factors +-1 are exact, so each lane is the scalar evaluation.
template <int CYv>
struct SrcPair {
    Src<1, CYv> A;    // source of cx = +1
    Src<-1, CYv> B;   // source of cx = -1
    __device__ __forceinline__ float2 L(int slot) const { return make_float2(A.L(slot), B.L(slot)); }
    __device__ __forceinline__ void eval(float2& Pm, float2& P0, float2& Pp) const {
        const float2 sx = make_float2(1.f, -1.f);
        float2 q0 = __fadd2_rn(L(K_0), __ffma2_rn(sx, L(K_X), L(K_XX)));
        float2 q1 = __fadd2_rn(L(K_Z), __ffma2_rn(sx, L(K_XZ), L(K_XXZ)));
        float2 q2 = __ffma2_rn(sx, L(K_XZZ), L(K_ZZ));
        if (CYv) {
            const float2 cy = make_float2((float)CYv, (float)CYv), sxy = make_float2((float)CYv, (float)-CYv);
            q0 = __fadd2_rn(q0, __ffma2_rn(cy, L(K_Y), L(K_YY)));
            q0 = __fadd2_rn(q0, __ffma2_rn(sxy, L(K_XY), __ffma2_rn(cy, L(K_XXY), __fmul2_rn(sx, L(K_XYY)))));
            q1 = __fadd2_rn(q1, __ffma2_rn(cy, L(K_YZ), L(K_YYZ)));
            q1 = __ffma2_rn(sxy, L(K_XYZ), q1);
            q2 = __ffma2_rn(cy, L(K_YZZ), q2);
        }
        const float2 t = __fadd2_rn(q0, q2);
        Pm = __ffma2_rn(make_float2(-1.f, -1.f), q1, t);
        P0 = q0;
        Pp = __fadd2_rn(t, q1);
    }
};

__host__ __device__ constexpr float w1d(int c) { return c == 0 ? 2.0f / 3.0f : 1.0f / 6.0f; }

// Moments of the three populations of one (cy, cz) group: directions
// (+1, cy, cz), (0, cy, cz), (-1, cy, cz) with values a, c0, b (unweighted
// P'), folded through S = a + b, D = a - b and T = S + (wC/wE) c0, each
// accumulated with the weight wE of the x-moving directions (wC/wE = 4).
template <int CYv, int CZv>
__device__ __forceinline__ void acc_group(float* acc, float a, float c0, float b) {
    constexpr float wE = w1d(1) * w1d(CYv) * w1d(CZv);
    constexpr float pe = wE, ne = -wE;
    const float S = a + b, D = a - b, T = fmaf(w1d(0) / w1d(1), c0, S);
    acc[A_RHO] = fmaf(pe, T, acc[A_RHO]);
    acc[A_JX] = fmaf(pe, D, acc[A_JX]);
    acc[A_XX] = fmaf(pe, S, acc[A_XX]);
    if (CYv) {
        acc[A_JY] = fmaf(CYv > 0 ? pe : ne, T, acc[A_JY]);
        acc[A_YY] = fmaf(pe, T, acc[A_YY]);
        acc[A_XY] = fmaf(CYv > 0 ? pe : ne, D, acc[A_XY]);
    }
    if (CZv) {
        acc[A_JZ] = fmaf(CZv > 0 ? pe : ne, T, acc[A_JZ]);
        acc[A_ZZ] = fmaf(pe, T, acc[A_ZZ]);
        acc[A_XZ] = fmaf(CZv > 0 ? pe : ne, D, acc[A_XZ]);
    }
    if (CYv && CZv) acc[A_YZ] = fmaf(CYv * CZv > 0 ? pe : ne, T, acc[A_YZ]);
}

// colour of one (cy, cz) group, as an increment over the target's own
// phi: w ((phi_s - phi_t)(1 + P') + (B.c)/|c|) summed over cx.  Uniform
// colour regions then keep phi exactly.
template <int CYv, int CZv>
__device__ __forceinline__ void col_group(float* acc, float ha, float hc, float hb, float Ex, float Ey, float Ez,
                                          float By0, float Bz0) {
    constexpr int cE = 1 + CYv * CYv + CZv * CZv, cC = CYv * CYv + CZv * CZv;
    constexpr float wE = w1d(1) * w1d(CYv) * w1d(CZv), wC = w1d(0) * w1d(CYv) * w1d(CZv);
    float r = Ex;
    if (CYv) r += CYv > 0 ? Ey : -Ey;
    if (CZv) r += CZv > 0 ? Ez : -Ez;
    // summed in units of wE (wC = 4 wE), one weighting into the accumulator
    float v = fmaf(wC / wE, hc, ha + hb);
    v = fmaf(invlen(cE), r, v);
    if (cC) {
        float rc = 0.f;
        if (CYv) rc += CYv > 0 ? By0 : -By0;
        if (CZv) rc += CZv > 0 ? Bz0 : -Bz0;
        v = fmaf((wC / wE) * invlen(cC), rc, v);
    }
    acc[A_COL] = fmaf(wE, v, acc[A_COL]);
}

// All populations that leave the source row y - CYv of plane s and land on
// the column's targets in planes s-1 (accm), s (acc0), s+1 (accp).  Kc
// points at the column's own node in the coefficient tile; phm, ph0, php
// are the column's own phi in the three target planes (colour mode).
template <int MODE, int CYv>
__device__ __forceinline__ void pull_row(const CNode& Kc, float* accm, float* acc0, float* accp,
                                         float phm, float ph0, float php) {
    const Src<1, CYv> sa{Kc.at(-(CYv * CW + 1))};   // source of cx = +1 (x - 1)
    const Src<0, CYv> sz{Kc.at(-(CYv * CW))};       // source of cx = 0
    const Src<-1, CYv> sb{Kc.at(-(CYv * CW - 1))};  // source of cx = -1 (x + 1)
    float am, a0, ap, cm, c0, cp, bm, b0, bp;
    {
        float2 pm, p0, pp;
        SrcPair<CYv>{sa, sb}.eval(pm, p0, pp);
        am = pm.x; bm = pm.y; a0 = p0.x; b0 = p0.y; ap = pp.x; bp = pp.y;
    }
    sz.eval(cm, c0, cp);
    acc_group<CYv, -1>(accm, am, cm, bm);
    acc_group<CYv, 0>(acc0, a0, c0, b0);
    acc_group<CYv, 1>(accp, ap, cp, bp);
    if (MODE == TSLB_MODE_COLOUR) {
        const float pa = sa.L(K_C0), pz = sz.L(K_C0), pb = sb.L(K_C0);
        // recolouring sums over the cx = +1 / -1 sources
        const float Ex = sa.L(K_C1) - sb.L(K_C1);
        const float Ey = CYv ? sa.L(K_C2) + sb.L(K_C2) : 0.f;
        const float Ez = sa.L(K_C3) + sb.L(K_C3);
        const float By0 = CYv ? sz.L(K_C2) : 0.f;
        const float Bz0 = sz.L(K_C3);
        // (phi_s - phi_t)(1 + P') for the three sources and the three target planes
        auto h = [](float ps, float pt, float P) { const float d = ps - pt; return fmaf(d, P, d); };
        col_group<CYv, -1>(accm, h(pa, phm, am), h(pz, phm, cm), h(pb, phm, bm), Ex, Ey, Ez, By0, Bz0);
        col_group<CYv, 0>(acc0, h(pa, ph0, a0), h(pz, ph0, c0), h(pb, ph0, b0), Ex, Ey, Ez, By0, Bz0);
        col_group<CYv, 1>(accp, h(pa, php, ap), h(pz, php, cp), h(pb, php, bp), Ex, Ey, Ez, By0, Bz0);
        if (CYv == 0) {
            // rest population: f_0 += delta0 (perturbation with B_0 = -10/27); its
            // colour is the target's own, so it adds no colour increment
            acc0[A_RHO] += sz.L(K_C4);
        }
    } else if (MODE == TSLB_MODE_PHASEFIELD) {
        // phase field g (D3Q7): axis directions and the rest population
        if (CYv == 0) {
            const float g0 = sz.L(K_C0), gz = sz.L(K_C3);
            accm[A_COL] += g0 - gz;                        // q = 6, (0,0,-1)
            accp[A_COL] += g0 + gz;                        // q = 5, (0,0,+1)
            acc0[A_COL] += sa.L(K_C0) + sa.L(K_C1);        // q = 1 from x - 1
            acc0[A_COL] += sb.L(K_C0) - sb.L(K_C1);        // q = 2 from x + 1
            acc0[A_COL] = fmaf(2.f, g0, acc0[A_COL]);      // q = 0: p0g phi = 2 G0
        } else {
            acc0[A_COL] += sz.L(K_C0) + CYv * sz.L(K_C2);  // q = 3 / 4
        }
    }
}

// Regularized or bounce-back populations entering target (x,y,z) from
// behind non-periodic faces; Kp holds the target's own coefficients.
template <int MODE, class T, bool TAU = false, bool SOLID = false>
__device__ void boundary_target_k(const StepArgs& a, const float* Kp, unsigned mask, int x, int y, int z, float* acc) {
    // colour mode accumulates colour increments over the target's own phi
    const float pht = Kp[K_C0];
    // own raw moments (velocity faces only)
    float m[NF];
    bool have_m = false;
    for (int q = 0; q < 27; ++q) {
        // the 26 moving directions as a 3x3x3 index (q == 13 is the rest population)
        const int dx = (q % 3) - 1, dy = ((q / 3) % 3) - 1, dz = (q / 9) - 1;
        if (dx == 0 && dy == 0 && dz == 0) continue;
        const int c[3] = {dx, dy, dz};
        // face through which the source x - c lies: axis a, side (c>0 -> minus face)
        int vface = -1;
        bool solid = false;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (c[ax] == 0) continue;
            const int f = 2 * ax + (c[ax] > 0 ? 0 : 1);
            if (mask & (1u << f)) {
                solid = true;
                const int k = a.face[f].kind;
                // a later velocity face wins, as the oracle's face loop overwrites in face order
                if (k == TSLB_BC_VELOCITY || k == TSLB_BC_INLET || k == TSLB_BC_OUTLET || k == TSLB_BC_PRESSURE) vface = f;
            }
        }
        // an interior solid source node (the lattice's solid mask), periodic axes wrapped
        bool msolid = false;
        if (SOLID && !solid) {
            const int sx = x - dx, sy = y - dy, sz = z - dz;
            msolid = bit_at(a.solid, nidx(a, sx < 0 ? sx + a.nx : (sx >= a.nx ? sx - a.nx : sx),
                                          sy < 0 ? sy + a.ny : (sy >= a.ny ? sy - a.ny : sy),
                                          sz < 0 ? sz + a.nz : (sz >= a.nz ? sz - a.nz : sz)));
        }
        if (!solid && !msolid) continue;
        const int c2 = dx * dx + dy * dy + dz * dz;
        const float wq = wclass(c2);
        // The pull skips whole solid z planes, but a source behind an x or y
        // face, or an interior solid node, is a zero-coefficient node it visited.
        const bool xy_solid = (dx && (mask & (1u << (dx > 0 ? 0 : 1)))) || (dy && (mask & (1u << (dy > 0 ? 2 : 3))));
        const bool zplane_solid = a.face[4].kind != TSLB_BC_PERIODIC && (z - dz < 0 || z - dz >= a.nz);
        const bool visited = (xy_solid && !zplane_solid) || msolid;
        // colour mode: the visited zero node added w (0 - phi_t): undo it
        if (MODE == TSLB_MODE_COLOUR && visited) acc[A_COL] += wq * pht;
        if (vface < 0) {
            // half-way bounce-back: f_c(x) = f^post_{-c}(x)
            const float P = eval_P(Kp, 1, -dx, -dy, -dz);
            acc_dir_rt(acc, dx, dy, dz, wq * P);
            if (MODE == TSLB_MODE_COLOUR) {
                // the reflected population carries the target's own colour: only the recolouring term
                const float bc = -(dx * Kp[K_C1] + dy * Kp[K_C2] + dz * Kp[K_C3]);
                acc[A_COL] += wq * invlen(c2) * bc;
            } else if (MODE == TSLB_MODE_PHASEFIELD && c2 == 1) {
                const float ge = -(dx * Kp[K_C1] + dy * Kp[K_C2] + dz * Kp[K_C3]);
                acc[A_COL] += Kp[K_C0] + ge;
            }
        } else {
            if (!have_m) {
                const long long id = nidx(a, x, y, z);
#pragma unroll
                for (int f = 0; f < NF; ++f) m[f] = ld_field<T>(a, f, id);
                have_m = true;
            }
            const FaceBC& fb = a.face[vface];
            const int ax = vface >> 1;
            float Ub[3] = {fb.u[0], fb.u[1], fb.u[2]};
            float phib = fb.phi < -2.f ? m[F_PHI] : fb.phi;
            // in-plane position of the ghost node the population leaves, x - c
            // (periodic axes wrap, a non-periodic axis clamps), in the target's layer
            int g[3] = {x, y, z};
            {
                const int cc[3] = {dx, dy, dz};
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    if (b == ax) continue;
                    const int n = dimn(a, b), v = g[b] - cc[b];
                    g[b] = (v >= 0 && v < n) ? v : (a.face[2 * b].kind == TSLB_BC_PERIODIC ? wrapi(v, n) : (v < 0 ? 0 : n - 1));
                }
            }
            if (fb.kind == TSLB_BC_INLET) {
                // the inlet plane at the ghost node (boundary_cds_3D_module.f90:934-986:
                // u, v, w of node (i, j, 1) feed the populations it sends)
                const long long pa = plane_area(a, vface), pi = plane_index(a, vface, g[0], g[1], g[2]);
                Ub[0] = __ldg(fb.plane + pi);
                Ub[1] = __ldg(fb.plane + pa + pi);
                Ub[2] = __ldg(fb.plane + 2 * pa + pi);
                phib = __ldg(fb.plane + 3 * pa + pi);
            } else if (fb.kind == TSLB_BC_OUTLET || fb.kind == TSLB_BC_PRESSURE) {
                phib = m[F_PHI];
            }
            float Uf[3] = {Ub[0], Ub[1], Ub[2]};  // velocity of the f equilibrium
            if (fb.kind == TSLB_BC_OUTLET) {
                // outlet: the normal velocity of the fluid node next to the ghost
                // node (zero gradient, :992 w(i,j,nz) = w(i,j,nz-1))
                Uf[ax] = ld_field<T>(a, F_U + ax, nidx(a, g[0], g[1], g[2]));
            } else if (fb.kind == TSLB_BC_PRESSURE) {
                // pressure outlet: the fluid node's velocity at density 1
                Uf[0] = m[F_U]; Uf[1] = m[F_V]; Uf[2] = m[F_W];
            }
            const float d = fb.kind == TSLB_BC_PRESSURE ? 0.f : m[F_D], rho = 1.f + d;
            float omega;
            if (MODE == TSLB_MODE_COLOUR) {
                const float ca = 0.5f * (1.f + m[F_PHI]), cb = 0.5f * (1.f - m[F_PHI]);
                const float nu = 1.f / (ca * a.inv_nu_a + cb * a.inv_nu_b);
                const float dt = TAU ? __ldg(a.dtau + nidx(a, x, y, z)) : 0.f;
                omega = 2.f / (6.f * nu + 1.f + 2.f * dt);
            } else {
                omega = a.omega_pf;
            }
            // f^eq(rho, Ub)/w - 1 (boundary_cds_3D_module.f90:461-507)
            const float cu = dx * Uf[0] + dy * Uf[1] + dz * Uf[2];
            const float uu = Uf[0] * Uf[0] + Uf[1] * Uf[1] + Uf[2] * Uf[2];
            const float t3 = 1.f / 3.f;
            const float hxxy = (dx * dx - t3) * dy, hxxz = (dx * dx - t3) * dz, hxyy = (dy * dy - t3) * dx;
            const float hyyz = (dy * dy - t3) * dz, hxzz = (dz * dz - t3) * dx, hyzz = (dz * dz - t3) * dy;
            const float hxyz = (float)(dx * dy * dz);
            const float U = Uf[0], V = Uf[1], W = Uf[2];
            const float h3e = 13.5f * (hxxy * U * U * V + hxxz * U * U * W + hxyy * U * V * V + hyyz * V * V * W +
                                       hxzz * U * W * W + hyzz * V * W * W) + 27.f * hxyz * U * V * W;
            const float feqm1 = d + rho * (3.f * cu + 4.5f * cu * cu - 1.5f * uu + h3e);
            // a^neq(Pi, u) of the fluid node
            const float u = m[F_U], v = m[F_V], w = m[F_W];
            const float pxx = m[F_XX], pxy = m[F_XY], pxz = m[F_XZ], pyy = m[F_YY], pyz = m[F_YZ], pzz = m[F_ZZ];
            const float h2 = (dx * dx - t3) * pxx + (dy * dy - t3) * pyy + (dz * dz - t3) * pzz +
                             2.f * (dx * dy * pxy + dx * dz * pxz + dy * dz * pyz);
            const float an = 4.5f * h2 +
                             13.5f * (hxxy * (2.f * u * pxy + v * pxx) + hxxz * (2.f * u * pxz + w * pxx) +
                                      hxyy * (u * pyy + 2.f * v * pxy) + hyyz * (2.f * v * pyz + w * pyy) +
                                      hxzz * (u * pzz + 2.f * w * pxz) + hyzz * (v * pzz + 2.f * w * pyz)) +
                             27.f * hxyz * (u * pyz + v * pxz + w * pxy);
            const float P = feqm1 + (1.f - omega) * an;
            acc_dir_rt(acc, dx, dy, dz, wq * P);
            if (MODE == TSLB_MODE_COLOUR) {
                const float dphi = phib - pht;
                acc[A_COL] += wq * fmaf(dphi, P, dphi);
            } else if (MODE == TSLB_MODE_PHASEFIELD && c2 == 1) {
                // g entering from the face (:984-986, :1044-1045)
                const float eu = dx * Ub[0] + dy * Ub[1] + dz * Ub[2];
                acc[A_COL] += 0.125f * phib * (1.f + 3.f * eu);
            }
        }
    }
}

// the same, with the target's coefficients read from the coefficient tile at Kc
template <int MODE, class T, bool TAU = false, bool SOLID = false>
__device__ __forceinline__ void boundary_target(const StepArgs& a, const CNode& Kc, unsigned mask, int x, int y,
                                                int z, float* acc) {
    float Kp[NCOEF];
#pragma unroll
    for (int c = 0; c < NCOEF; ++c) Kp[c] = coef_at(Kc, c);
    boundary_target_k<MODE, T, TAU, SOLID>(a, Kp, mask, x, y, z, acc);
}

// ---- shared-memory staging geometry ----
// Moments and phi are staged with the tile's x range widened to whole
// 16-byte chunks of EPC elements: columns x0-EPC .. x0+TX+EPC-1.
constexpr int NTHR = TX * TY;
constexpr int NHALO = CAREA - NTHR;           // coefficient nodes on the tile rim (84)
constexpr int NMOM = NF - 1;                  // moments staged per node (phi comes from the phi ring)
// Phi rows staged beyond the tile in y (and planes held beyond the source
// plane in z): colour mode reads the gradient at the coefficient nodes (the
// tile plus a one-node rim), 2; the phase field also the normals of their
// neighbours for the curvature, 3.
__host__ __device__ constexpr int phi_halo(int mode) { return mode == TSLB_MODE_PHASEFIELD ? 3 : 2; }
template <int ES, int PHR = 2>   // element size in bytes, phi halo
struct Geo {
    static constexpr int EPC = 16 / ES;               // elements per 16-byte chunk
    static constexpr int SW = TX + 2 * EPC;           // staged row width
    static constexpr int OFF = EPC - 1;               // staged column of tile column 0 (x0 - 1)
    static constexpr int NCH = SW / EPC;              // chunks per row
    static constexpr int MROWS = CH;                  // moment rows: y0-1 .. y0+TY
    static constexpr int PROWS = TY + 2 * PHR;        // phi rows: y0-PHR .. y0+TY+PHR-1
    static constexpr int MAREA = MROWS * SW, PAREA = PROWS * SW;
    static constexpr int MCELLS = MROWS * NCH;        // 16-byte cells of one staged moment plane
    static constexpr int MGROUPS = NTHR / MCELLS;     // thread (g, cell) copies fields g, g + MGROUPS, ...
    static constexpr int MFIELDS = (NMOM + MGROUPS - 1) / MGROUPS;
    static_assert(MGROUPS >= 1, "a staged moment plane has more cells than the block has threads");
    static constexpr int PCOPIES = PROWS * NCH;
    static constexpr int PELEMS = PROWS * SW;
    static constexpr int PEROUNDS = (PELEMS + NTHR - 1) / NTHR;
};

// Phi ring: slot z & (PRING - 1) holds phi plane z.  Iteration s stages plane
// s+PHR while other threads may still read planes from s-PHR on (the previous
// iteration's pull or curvature), so the ring holds at least 2 PHR + 1 planes.
constexpr int PRING = 8;
// Phase field: the curvature work list of the block (section 4 of step_block):
// the candidate nodes' tile indices for two planes, their curvatures, two counts
constexpr size_t CURV_LIST_BYTES = sizeof(float) * CAREA + sizeof(unsigned short) * 2 * CAREA + sizeof(int) * 2;
__host__ __device__ constexpr size_t step_smem_bytes_es(int mode, int es) {
    return sizeof(float) * 2 * NCOEF * CAREA + (size_t)es * 2 * NMOM * CH * (TX + 2 * (16 / es)) +
           (mode != TSLB_MODE_SINGLE ? (size_t)es * PRING * (TY + 2 * phi_halo(mode)) * (TX + 2 * (16 / es)) : 0) +
           (mode == TSLB_MODE_PHASEFIELD ? CURV_LIST_BYTES : 0);
}
__host__ __device__ constexpr size_t step_smem_bytes(int mode) { return step_smem_bytes_es(mode, 4); }

// gradient 3 sum_i p_i c_i phi(x+c_i) of one node (Ar1) or two (Ar2) from
// phi planes held in shared memory: P(dz, dx, dy) returns phi at offset
// (dx, dy, dz) of the node(s).  Every operation is explicit (see Ar1).
template <class Ar, class LD>
__device__ __forceinline__ void grad_v(LD P, typename Ar::V g[3]) {
    using V = typename Ar::V;
    auto S4 = [](V a, V b, V c, V d) { return Ar::add(Ar::add(Ar::add(a, b), c), d); };
    const V x1 = Ar::sub(P(0, 1, 0), P(0, -1, 0));
    const V x2 = Ar::sub(S4(P(0, 1, 1), P(0, 1, -1), P(1, 1, 0), P(-1, 1, 0)),
                         S4(P(0, -1, 1), P(0, -1, -1), P(1, -1, 0), P(-1, -1, 0)));
    const V x3 = Ar::sub(S4(P(1, 1, 1), P(1, 1, -1), P(-1, 1, 1), P(-1, 1, -1)),
                         S4(P(1, -1, 1), P(1, -1, -1), P(-1, -1, 1), P(-1, -1, -1)));
    const V y1 = Ar::sub(P(0, 0, 1), P(0, 0, -1));
    const V y2 = Ar::sub(S4(P(0, 1, 1), P(0, -1, 1), P(1, 0, 1), P(-1, 0, 1)),
                         S4(P(0, 1, -1), P(0, -1, -1), P(1, 0, -1), P(-1, 0, -1)));
    const V y3 = Ar::sub(S4(P(1, 1, 1), P(1, -1, 1), P(-1, 1, 1), P(-1, -1, 1)),
                         S4(P(1, 1, -1), P(1, -1, -1), P(-1, 1, -1), P(-1, -1, -1)));
    const V z1 = Ar::sub(P(1, 0, 0), P(-1, 0, 0));
    const V z2 = Ar::sub(S4(P(1, 1, 0), P(1, -1, 0), P(1, 0, 1), P(1, 0, -1)),
                         S4(P(-1, 1, 0), P(-1, -1, 0), P(-1, 0, 1), P(-1, 0, -1)));
    const V z3 = Ar::sub(S4(P(1, 1, 1), P(1, 1, -1), P(1, -1, 1), P(1, -1, -1)),
                         S4(P(-1, 1, 1), P(-1, 1, -1), P(-1, -1, 1), P(-1, -1, -1)));
    const V c1 = Ar::c(3.f * wclass(1)), c2 = Ar::c(3.f * wclass(2)), c3 = Ar::c(3.f * wclass(3));
    g[0] = Ar::fma(c3, x3, Ar::fma(c2, x2, Ar::mul(c1, x1)));
    g[1] = Ar::fma(c3, y3, Ar::fma(c2, y2, Ar::mul(c1, y1)));
    g[2] = Ar::fma(c3, z3, Ar::fma(c2, z2, Ar::mul(c1, z1)));
}
// one node; pm, p0, pp point at it in planes z-1, z, z+1 (row pitch SWv).
// fp16 storage: the caller multiplies the result by the phi scale.
template <int SWv, class T>
__device__ __forceinline__ void grad_smem(const T* pm, const T* p0, const T* pp, float g[3]) {
    grad_v<Ar1>([&](int dz, int dx, int dy) {
        const T* pl = dz < 0 ? pm : dz > 0 ? pp : p0;
        return Stor<T>::ld(pl[dy * SWv + dx]);
    }, g);
}

// Phase-field interface normal n = g / (|g| + 1e-9) from the staged phi
// planes (ring slots of plane z and its neighbours), at staged offset pi
// (recursive_2c_TSLB3D.f90:555-571).
// n = g / (|g| + 1e-9) of one node (Ar1) or two (Ar2), operation by operation
template <class Ar>
__device__ __forceinline__ void normalize_v(typename Ar::V n[3]) {
    const typename Ar::V m2 = Ar::fma(n[2], n[2], Ar::fma(n[1], n[1], Ar::mul(n[0], n[0])));
    const typename Ar::V inv = Ar::map(m2, [](float x) { return __frcp_rn(__fadd_rn(sqrtf(x), 1e-9f)); });
    n[0] = Ar::mul(n[0], inv); n[1] = Ar::mul(n[1], inv); n[2] = Ar::mul(n[2], inv);
}
// the phase field's interface indicator phi (1 - phi) |n|^2 (recursive_2c_TSLB3D.f90:614)
template <class Ar>
__device__ __forceinline__ typename Ar::V pf_indicator(typename Ar::V phi, const typename Ar::V n[3]) {
    const typename Ar::V nn = Ar::fma(n[2], n[2], Ar::fma(n[1], n[1], Ar::mul(n[0], n[0])));
    return Ar::mul(Ar::mul(phi, Ar::sub(Ar::c(1.f), phi)), nn);
}

template <int SWv, class T>
__device__ __forceinline__ void pf_normal(const T* ring, int parea, int z, int pi, const StepArgs& a, float n[3]) {
    const T* p0 = ring + (z & (PRING - 1)) * parea + pi;
    const T* pm = ring + ((z - 1) & (PRING - 1)) * parea + pi;
    const T* pp = ring + ((z + 1) & (PRING - 1)) * parea + pi;
    grad_smem<SWv>(pm, p0, pp, n);
    if constexpr (std::is_same<T, __half>::value) {
        n[0] = __fmul_rn(n[0], a.iscale[F_PHI]); n[1] = __fmul_rn(n[1], a.iscale[F_PHI]);
        n[2] = __fmul_rn(n[2], a.iscale[F_PHI]);
    }
    normalize_v<Ar1>(n);
}


struct XYNode {
    int off;      // gx + nx * gy (wrapped/clamped)
    int gx, gy;   // raw coordinates (may be out of range)
    bool out;     // behind a non-periodic x or y face
};

__device__ __forceinline__ XYNode xy_node(const StepArgs& a, int gx, int gy, bool xper, bool yper) {
    XYNode n;
    n.gx = gx; n.gy = gy; n.out = false;
    int cx = gx, cy = gy;
    if (cx < 0 || cx >= a.nx) { if (xper) cx = wrapi(cx, a.nx); else { n.out = true; cx = cx < 0 ? 0 : a.nx - 1; } }
    if (cy < 0 || cy >= a.ny) { if (yper) cy = wrapi(cy, a.ny); else { n.out = true; cy = cy < 0 ? 0 : a.ny - 1; } }
    n.off = cx + a.nx * cy;
    return n;
}

// Phase-field curvature -div n of one coefficient node, computed by a whole
// warp: the isotropic stencil over the node's 26 neighbours
// (recursive_2c_TSLB3D.f90:617-627), each neighbour's normal recomputed from
// the staged phi (pf_normal); a neighbour behind a non-periodic face, or an
// interior solid one, has n = 0.  Lane j < 26 computes neighbour j and a
// butterfly sums the 26 terms; every lane returns the sum.  z is the source
// plane (ring index), gz its lattice plane, pi the node's staged offset and
// (gx, gy) its lattice coordinates (may lie beyond a periodic face).
static_assert(TX == 32, "a warp is one tile row: the lane is threadIdx.x");
template <int SWv, bool SOLID, class T>
__device__ float node_curvature(const T* ring, int parea, int z, int pi, int gx, int gy, int gz, const StepArgs& a,
                                bool xper, bool yper, bool zper) {
    const int lane = threadIdx.x;
    const int j = lane < 13 ? lane : lane + 1;   // 3 x 3 x 3 index of the neighbour, the centre (13) skipped
    const int dx = j % 3 - 1, dy = (j / 3) % 3 - 1, dz = j / 9 - 1;
    const int xn = gx + dx, yn = gy + dy, zn = gz + dz;
    bool ok = lane < 26 && (zper || (zn >= 0 && zn < a.nz)) && (xper || (xn >= 0 && xn < a.nx)) &&
              (yper || (yn >= 0 && yn < a.ny));
    if (SOLID && ok) ok = !bit_at(a.solid, nidx(a, wrapi(xn, a.nx), wrapi(yn, a.ny), wrapi(zn, a.nz)));
    float t = 0.f;
    if (ok) {
        float n[3];
        pf_normal<SWv>(ring, parea, z + dz, pi + dy * SWv + dx, a, n);
        t = wclass(dx * dx + dy * dy + dz * dz) * ((float)dx * n[0] + (float)dy * n[1] + (float)dz * n[2]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return -3.f * t;
}

__device__ __forceinline__ void cp_async4(float* sdst, const float* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16s(unsigned sa, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// T: storage type of the moment state (float, __nv_bfloat16, __half).
// VEC: nx is a multiple of the 16-byte chunk, so chunks never straddle the
// x faces and planes are staged with 16-byte cp.async copies.
// One block's work: tile (bx, by) of columns and z chunk bz of lattice a.
// SOLID: the lattice has interior solid nodes (bit masks a.solid, a.near).
// PAIR: the warps holding rim nodes compute their two coefficient nodes at
// once (coef_pair); the results are the same numbers either way, so a form
// whose registers are short (the phase field inside an ensemble) leaves it.
template <int MODE, bool VEC, class T, bool TAU = false, bool SOLID = false, bool PAIR = true>
__device__ __forceinline__ void step_block(const StepArgs& a, int bx, int by, int bz) {
    constexpr int PHR = phi_halo(MODE);
    constexpr bool PHI = MODE != TSLB_MODE_SINGLE;   // phi is staged (colour, phase field)
    using G = Geo<sizeof(T), PHR>;
    constexpr int SW = G::SW, EPC = G::EPC, MAREA = G::MAREA, PAREA = G::PAREA;
    extern __shared__ float4 smem4[];
    float* coef_base = reinterpret_cast<float*>(smem4);               // [2][NQUAD quads + pair][CAREA]
    T* mst = reinterpret_cast<T*>(coef_base + 2 * NCOEF * CAREA);     // [2][NMOM][MROWS][SW]
    T* phis = mst + 2 * NMOM * MAREA;                                 // [PRING][PROWS][SW] (not single)
    // phase field: curvature work list (curvatures of plane s, candidates of planes s and s+1, their counts)
    float* cq_curv = reinterpret_cast<float*>(phis + PRING * PAREA);  // [CAREA]
    unsigned short* cq_list = reinterpret_cast<unsigned short*>(cq_curv + CAREA);   // [2][CAREA]
    int* cq_n = reinterpret_cast<int*>(cq_list + 2 * CAREA);          // [2]
    const T* gin = reinterpret_cast<const T*>(a.in);
    T* gout = reinterpret_cast<T*>(a.out);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = bx * TX, y0 = by * TY;
    const int z0 = a.zt0 + bz * a.zchunk;
    const int z1 = min(z0 + a.zchunk, a.zt1);
    const int X = x0 + tx, Y = y0 + ty;
    const bool active = X < a.nx && Y < a.ny;
    const bool xper = a.face[0].kind == TSLB_BC_PERIODIC;
    const bool yper = a.face[2].kind == TSLB_BC_PERIODIC;
    const bool zper = a.face[4].kind == TSLB_BC_PERIODIC;
    const long long plane = (long long)a.nx * a.ny;
    // the step that seeds the stochastic rounding of 16-bit stores (an ensemble
    // advances a device counter after each step: its graph replays fixed arguments)
    const unsigned int sr_step = a.sr_counter ? *a.sr_counter : a.sr_step;

    // faces the column touches (z faces are added per plane)
    unsigned colmask = 0;
    if (active) {
        if (!xper && X == 0) colmask |= 1u;
        if (!xper && X == a.nx - 1) colmask |= 2u;
        if (!yper && Y == 0) colmask |= 4u;
        if (!yper && Y == a.ny - 1) colmask |= 8u;
    }

    // coefficient nodes of this thread: its own column (r = 0) and one rim node (r = 1)
    const bool has_rim = tid < NHALO;
    XYNode cn0 = xy_node(a, X, Y, xper, yper), cn1;
    const int ci0 = (ty + 1) * CW + (tx + 1);
    int ci1;
    {
        int h = has_rim ? tid : 0, cx, cy;
        if (h < CW) { cx = h; cy = 0; }
        else if (h < 2 * CW) { cx = h - CW; cy = CH - 1; }
        else if (h < 2 * CW + TY) { cx = 0; cy = h - 2 * CW + 1; }
        else { cx = CW - 1; cy = h - 2 * CW - TY + 1; }
        cn1 = xy_node(a, x0 - 1 + cx, y0 - 1 + cy, xper, yper);
        ci1 = cy * CW + cx;
    }
    // position of a coefficient node (cx, cy) in the staged planes: moments
    // row cy, column cx + OFF; phi row cy + PHR - 1, same column
    const int mi0 = (ci0 / CW) * SW + (ci0 % CW) + G::OFF, mi1 = (ci1 / CW) * SW + (ci1 % CW) + G::OFF;
    const int pi0 = mi0 + (PHR - 1) * SW, pi1 = mi1 + (PHR - 1) * SW;
    const int nnodes = has_rim ? 2 : 1;

    auto zwrap = [&](int z, bool& out) {
        out = false;
        if (z < 0 || z >= a.nz) { if (zper) return wrapi(z, a.nz); out = true; }
        return z;
    };

    // ---- staging of phi planes (colour and phase-field modes) ----
    // VEC: copy j < PCOPIES is the 16-byte chunk (row j / NCH, chunk j % NCH);
    // a chunk is either fully inside the domain (after the periodic wrap) or
    // fully behind a non-periodic face, whose ghost values are computed.
    int pch_off = 0, pch_dst = 0;
    bool pch_out = true;
    if (VEC && tid < G::PCOPIES) {
        const int row = tid / G::NCH, ch = tid % G::NCH;
        const XYNode nd = xy_node(a, x0 - EPC + EPC * ch, y0 - PHR + row, xper, yper);
        pch_off = nd.off;
        pch_out = nd.out;
        pch_dst = row * SW + EPC * ch;
    }
    const T* pg0 = gin + F_PHI * a.N + pch_off;
    const unsigned ps0 = (unsigned)__cvta_generic_to_shared(phis) + (unsigned)(pch_dst * sizeof(T));
    auto ghost = [&](float v) { return cvt_out<T>(v, a, F_PHI); };
    auto stage_phi = [&](int z) {
        bool zout;
        const int gz = zwrap(z, zout);
        T* slot = phis + (z & (PRING - 1)) * PAREA;
        const T* ph = gin + F_PHI * a.N + (long long)gz * plane;
        if (VEC) {
            if (tid < G::PCOPIES) {
                T* dst = slot + pch_dst;
                if (!pch_out && !zout) {
                    cp_async16s(ps0 + (unsigned)((z & (PRING - 1)) * (PAREA * (int)sizeof(T))), pg0 + (long long)gz * plane);
                } else {
                    const int row = tid / G::NCH, ch = tid % G::NCH;
#pragma unroll
                    for (int e = 0; e < EPC; ++e) dst[e] = ghost(phi_at<T>(a, x0 - EPC + EPC * ch + e, y0 - PHR + row, z));
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < G::PEROUNDS; ++r) {
                const int j = tid + r * NTHR;
                if (j < G::PELEMS) {
                    const int row = j / SW, col = j % SW;
                    const XYNode nd = xy_node(a, x0 - EPC + col, y0 - PHR + row, xper, yper);
                    if (!nd.out && !zout) {
                        if constexpr (sizeof(T) == 4) cp_async4(reinterpret_cast<float*>(slot + j), reinterpret_cast<const float*>(ph + nd.off));
                        else slot[j] = ph[nd.off];
                    } else {
                        slot[j] = ghost(phi_at<T>(a, nd.gx, nd.gy, z));
                    }
                }
            }
        }
    };

    // ---- staging of the 10 non-phi moments of plane z ----
    // VEC: thread tid < MGROUPS MCELLS owns cell tid % MCELLS (row, chunk) of the
    // staged plane and copies it for the fields tid / MCELLS + k MGROUPS; the
    // addresses are fixed per thread, only the plane changes.
    int mcell_dst = 0, mcell_off = 0, mfg = 0;
    bool mcell_ok = false;
    if (VEC && tid < G::MGROUPS * G::MCELLS) {
        const int cell = tid % G::MCELLS, row = cell / G::NCH, ch = cell % G::NCH;
        mfg = tid / G::MCELLS;
        const XYNode nd = xy_node(a, x0 - EPC + EPC * ch, y0 - 1 + row, xper, yper);
        mcell_off = nd.off;
        mcell_ok = !nd.out;
        mcell_dst = mfg * MAREA + row * SW + EPC * ch;
    }
    // per-thread staging bases: global (field group, cell) and shared (cell)
    const T* mg0 = gin + mfg * a.N + mcell_off;
    const long long mfstride = (long long)G::MGROUPS * a.N;
    const unsigned ms0 = (unsigned)__cvta_generic_to_shared(mst) + (unsigned)(mcell_dst * sizeof(T));

    auto stage_mom = [&](int z) {
        bool zout;
        const int gz = zwrap(z, zout);
        if (zout) return;
        T* dst = mst + (z & 1) * (NMOM * MAREA);
        const T* src = gin + (long long)gz * plane;
        if (VEC) {
            if (mcell_ok) {
                const unsigned d = ms0 + (unsigned)((z & 1) * (NMOM * MAREA * (int)sizeof(T)));
                const T* g = mg0 + (long long)gz * plane;
#pragma unroll
                for (int k = 0; k < G::MFIELDS; ++k) {
                    if (G::MGROUPS * G::MFIELDS == NMOM || mfg + k * G::MGROUPS < NMOM)
                        cp_async16s(d + (unsigned)(k * G::MGROUPS * MAREA * (int)sizeof(T)), g + k * mfstride);
                }
            }
        } else {
            for (int r = 0; r < nnodes; ++r) {
                const XYNode nd = r ? cn1 : cn0;
                if (nd.out) continue;
                const T* p = src + nd.off;
                T* d = dst + (r ? mi1 : mi0);
#pragma unroll
                for (int f = 0; f < NMOM; ++f) {
                    if constexpr (sizeof(T) == 4) cp_async4(reinterpret_cast<float*>(d + f * MAREA), reinterpret_cast<const float*>(p + f * a.N));
                    else d[f * MAREA] = p[f * a.N];
                }
            }
        }
    };

    // phi of the planes the first source plane z0 - 1 reads: z0 - PHR .. z0 + PHR - 2
    if (PHI)
        for (int z = z0 - PHR; z <= z0 + PHR - 2; ++z) stage_phi(z);
    stage_mom(z0 - 1);
    cp_async_commit();
    if (MODE == TSLB_MODE_PHASEFIELD && tid == 0) cq_n[0] = cq_n[1] = 0;
    cp_async_wait<0>();
    __syncthreads();

    // Phase field: the curvature of a plane's interface nodes is shared by all
    // warps of the block.  The coefficient phase of plane s lists the nodes of
    // plane s+1 that may need it (candidates: phi (1 - phi) above the
    // indicator's threshold, a superset of the nodes where phi (1 - phi) |n|^2
    // exceeds it); the next coefficient phase, after the plane barrier, first
    // computes their curvatures warp by warp, then (one more barrier) the
    // coefficients.  A node's position in its plane's list: slot0 / slot1.
    int slot0 = -1, slot1 = -1;
    auto list_candidates = [&](int z) {
        bool zs;
        const int gzc = zwrap(z, zs);
        if (zs) { slot0 = slot1 = -1; return; }
        auto cand = [&](const bool has, const XYNode& nd, const int ci, const int pi) {
            if (!has || nd.out || (SOLID && bit_at(a.solid, (long long)gzc * plane + nd.off))) return -1;
            const float ph = cvt_in<T>(phis[(z & (PRING - 1)) * PAREA + pi], a, F_PHI);
            if (!(ph * (1.f - ph) > 0.2f * (1.f - 1e-5f))) return -1;
            const int e = atomicAdd(&cq_n[z & 1], 1);
            cq_list[(z & 1) * CAREA + e] = (unsigned short)ci;
            return e;
        };
        slot0 = cand(true, cn0, ci0, pi0);
        slot1 = cand(has_rim, cn1, ci1, pi1);
    };
    if (MODE == TSLB_MODE_PHASEFIELD) {
        list_candidates(z0 - 1);
        __syncthreads();
    }

    float accm[NACC], acc0[NACC], accp[NACC];
#pragma unroll
    for (int i = 0; i < NACC; ++i) { accm[i] = 0.f; acc0[i] = 0.f; accp[i] = 0.f; }

    int buf = 0;
    for (int s = z0 - 1; s <= z1; ++s) {
        float* coef = coef_base + buf * (NCOEF * CAREA);
        const bool more = s < z1;
        // ---- 0. prefetch: phi of plane s+PHR, moments of plane s+1 ----
        if (PHI && more) stage_phi(s + PHR);
        cp_async_commit();
        if (more) stage_mom(s + 1);
        cp_async_commit();
        // non-VEC: this thread's own moment copies of plane s; VEC: every copy of
        // plane s was waited for before the previous plane's pre-pull barrier
        if (!VEC) cp_async_wait<2>();
        // ---- 1. coefficients of source plane s: own column and one rim node ----
        bool zsolid;
        const int gz = zwrap(s, zsolid);
        const T* ms = mst + (s & 1) * (NMOM * MAREA);
        // a solid source plane sends nothing: no coefficients, no pull
        auto coef_node = [&](const XYNode& nd, const int ci, const int mi, const int pi) {
            float K[NCOEF];
            // solid nodes (behind a face, or interior solids) send nothing
            if (nd.out || (SOLID && bit_at(a.solid, (long long)gz * plane + nd.off))) {
#pragma unroll
                for (int c = 0; c < NCOEF; ++c) K[c] = 0.f;
            } else {
                float m[NF];
#pragma unroll
                for (int f = 0; f < NMOM; ++f) m[f] = cvt_in<T>(ms[f * MAREA + mi], a, f);
                float g[3] = {0.f, 0.f, 0.f};
                if (MODE == TSLB_MODE_COLOUR) {
                    const T* p0 = phis + (s & (PRING - 1)) * PAREA + pi;
                    const T* pm = phis + ((s - 1) & (PRING - 1)) * PAREA + pi;
                    const T* pp = phis + ((s + 1) & (PRING - 1)) * PAREA + pi;
                    m[F_PHI] = cvt_in<T>(*p0, a, F_PHI);
                    grad_smem<SW>(pm, p0, pp, g);
                    if constexpr (std::is_same<T, __half>::value) {
                        g[0] = __fmul_rn(g[0], a.iscale[F_PHI]); g[1] = __fmul_rn(g[1], a.iscale[F_PHI]);
                        g[2] = __fmul_rn(g[2], a.iscale[F_PHI]);
                    }
                } else {
                    m[F_PHI] = 1.f;
                }
                node_coefs<MODE, TAU>(a, m, g, 0.f, K, TAU ? (long long)gz * plane + nd.off : 0);
            }
            store_coefs<MODE>(coef, ci, K);
        };
        // The warps that hold rim nodes (rows 0-2 of the tile: threads tid < NHALO)
        // have two coefficient nodes per plane and set the length of the phase
        // before the plane barrier.  They evaluate both at once on the paired
        // FP32 instructions: lane x the own node, lane y the rim node (a thread
        // without one repeats its own node in y and stores x alone).  Every
        // operation rounds as in coef_node, so a node gets the same coefficients
        // as an own node of one tile and as a rim node of another.
        auto coef_pair = [&]() {
            const XYNode nb = has_rim ? cn1 : cn0;
            const int miB = has_rim ? mi1 : mi0, piB = has_rim ? pi1 : pi0;
            Ar2::V m[NF], g[3] = {Ar2::c(0.f), Ar2::c(0.f), Ar2::c(0.f)};
#pragma unroll
            for (int f = 0; f < NMOM; ++f)
                m[f] = make_float2(cvt_in<T>(ms[f * MAREA + mi0], a, f), cvt_in<T>(ms[f * MAREA + miB], a, f));
            if (MODE == TSLB_MODE_COLOUR) {
                const T* r0 = phis + (s & (PRING - 1)) * PAREA;
                const T* rm = phis + ((s - 1) & (PRING - 1)) * PAREA;
                const T* rp = phis + ((s + 1) & (PRING - 1)) * PAREA;
                m[F_PHI] = make_float2(cvt_in<T>(r0[pi0], a, F_PHI), cvt_in<T>(r0[piB], a, F_PHI));
                grad_v<Ar2>([&](int dz, int dx, int dy) {
                    const T* pl = dz < 0 ? rm : dz > 0 ? rp : r0;
                    const int o = dy * SW + dx;
                    return make_float2(Stor<T>::ld(pl[pi0 + o]), Stor<T>::ld(pl[piB + o]));
                }, g);
                if constexpr (std::is_same<T, __half>::value) {
                    const Ar2::V sc = Ar2::c(a.iscale[F_PHI]);
                    g[0] = Ar2::mul(g[0], sc); g[1] = Ar2::mul(g[1], sc); g[2] = Ar2::mul(g[2], sc);
                }
            } else {
                m[F_PHI] = Ar2::c(1.f);
            }
            const long long pz = (long long)gz * plane;
            const Ar2::V dt = TAU ? make_float2(__ldg(a.dtau + pz + cn0.off), __ldg(a.dtau + pz + nb.off)) : Ar2::c(0.f);
            Ar2::V K2[NCOEF];
            node_coefs_v<MODE, TAU, Ar2>(a, m, g, Ar2::c(0.f), dt, K2);
            // solid nodes (behind a face, or interior solids) send nothing
            const bool s0 = cn0.out || (SOLID && bit_at(a.solid, pz + cn0.off));
            const bool s1 = nb.out || (SOLID && bit_at(a.solid, pz + nb.off));
            float K[NCOEF];
#pragma unroll
            for (int c = 0; c < NCOEF; ++c) K[c] = s0 ? 0.f : K2[c].x;
            store_coefs<MODE>(coef, ci0, K);
            if (has_rim) {
#pragma unroll
                for (int c = 0; c < NCOEF; ++c) K[c] = s1 ? 0.f : K2[c].y;
                store_coefs<MODE>(coef, ci1, K);
            }
        };
        // Phase field: the interface normal n = grad phi / (|grad phi| + 1e-9) of
        // the node (recursive_2c_TSLB3D.f90:555-571) and, where the indicator
        // phi (1 - phi) |n|^2 exceeds 0.2, the curvature -div n over the 26
        // neighbours' normals (:614-629), taken from the block's work list.
        auto coef_node_pf = [&](const XYNode& nd, const int ci, const int mi, const int pi, const int slot) {
            float K[NCOEF];
            if (nd.out || (SOLID && bit_at(a.solid, (long long)gz * plane + nd.off))) {
#pragma unroll
                for (int c = 0; c < NCOEF; ++c) K[c] = 0.f;
            } else {
                float m[NF], g[3];
#pragma unroll
                for (int f = 0; f < NMOM; ++f) m[f] = cvt_in<T>(ms[f * MAREA + mi], a, f);
                const float phi = cvt_in<T>(phis[(s & (PRING - 1)) * PAREA + pi], a, F_PHI);
                m[F_PHI] = phi;
                pf_normal<SW>(phis, PAREA, s, pi, a, g);
                const bool need = pf_indicator<Ar1>(phi, g) > 0.2f;
                // a node that needs the curvature was listed as a candidate (slot >= 0)
                const float curv = need && slot >= 0 ? cq_curv[slot] : 0.f;
                node_coefs<MODE, TAU>(a, m, g, curv, K, TAU ? (long long)gz * plane + nd.off : 0);
            }
            store_coefs<MODE>(coef, ci, K);
        };
        // the same two nodes at once for the phase field (coef_node_pf per lane)
        auto coef_pair_pf = [&]() {
            const XYNode nb = has_rim ? cn1 : cn0;
            const int miB = has_rim ? mi1 : mi0, piB = has_rim ? pi1 : pi0, slotB = has_rim ? slot1 : slot0;
            Ar2::V m[NF], g[3];
#pragma unroll
            for (int f = 0; f < NMOM; ++f)
                m[f] = make_float2(cvt_in<T>(ms[f * MAREA + mi0], a, f), cvt_in<T>(ms[f * MAREA + miB], a, f));
            const T* r0 = phis + (s & (PRING - 1)) * PAREA;
            const T* rm = phis + ((s - 1) & (PRING - 1)) * PAREA;
            const T* rp = phis + ((s + 1) & (PRING - 1)) * PAREA;
            const Ar2::V phi = make_float2(cvt_in<T>(r0[pi0], a, F_PHI), cvt_in<T>(r0[piB], a, F_PHI));
            m[F_PHI] = phi;
            grad_v<Ar2>([&](int dz, int dx, int dy) {
                const T* pl = dz < 0 ? rm : dz > 0 ? rp : r0;
                const int o = dy * SW + dx;
                return make_float2(Stor<T>::ld(pl[pi0 + o]), Stor<T>::ld(pl[piB + o]));
            }, g);
            if constexpr (std::is_same<T, __half>::value) {
                const Ar2::V sc = Ar2::c(a.iscale[F_PHI]);
                g[0] = Ar2::mul(g[0], sc); g[1] = Ar2::mul(g[1], sc); g[2] = Ar2::mul(g[2], sc);
            }
            normalize_v<Ar2>(g);
            const Ar2::V ind = pf_indicator<Ar2>(phi, g);
            // a node that needs the curvature was listed as a candidate (slot >= 0)
            const Ar2::V curv = make_float2(ind.x > 0.2f && slot0 >= 0 ? cq_curv[slot0] : 0.f,
                                            ind.y > 0.2f && slotB >= 0 ? cq_curv[slotB] : 0.f);
            const long long pz = (long long)gz * plane;
            const Ar2::V dt = TAU ? make_float2(__ldg(a.dtau + pz + cn0.off), __ldg(a.dtau + pz + nb.off)) : Ar2::c(0.f);
            Ar2::V K2[NCOEF];
            node_coefs_v<MODE, TAU, Ar2>(a, m, g, curv, dt, K2);
            const bool s0 = cn0.out || (SOLID && bit_at(a.solid, pz + cn0.off));
            const bool s1 = nb.out || (SOLID && bit_at(a.solid, pz + nb.off));
            float K[NCOEF];
#pragma unroll
            for (int c = 0; c < NCOEF; ++c) K[c] = s0 ? 0.f : K2[c].x;
            store_coefs<MODE>(coef, ci0, K);
            if (has_rim) {
#pragma unroll
                for (int c = 0; c < NCOEF; ++c) K[c] = s1 ? 0.f : K2[c].y;
                store_coefs<MODE>(coef, ci1, K);
            }
        };
        if (MODE == TSLB_MODE_PHASEFIELD) {
            // curvatures of this plane's candidates, warp w taking entries w, w + 8, ...
            // (the count is the same for every thread: the list was completed before
            // the previous plane's barrier)
            const int cnt = cq_n[s & 1];
            if (cnt > 0) {
                for (int e = ty; e < cnt; e += TY) {
                    const int ci = cq_list[(s & 1) * CAREA + e];
                    const int cx = ci % CW, cy = ci / CW;
                    const float k = node_curvature<SW, SOLID>(phis, PAREA, s, cy * SW + cx + G::OFF + (PHR - 1) * SW,
                                                              x0 - 1 + cx, y0 - 1 + cy, gz, a, xper, yper, zper);
                    if (tx == 0) cq_curv[e] = k;
                }
                __syncthreads();
                // every thread has read cnt; the next entries of this parity come after the plane barrier
                if (tid == 0) cq_n[s & 1] = 0;
            }
        }
        if (!zsolid) {
            if constexpr (MODE == TSLB_MODE_PHASEFIELD) {
                if (PAIR && ty * TX < NHALO) {
                    coef_pair_pf();
                } else {
                    coef_node_pf(cn0, ci0, mi0, pi0, slot0);
                    if (!PAIR && has_rim) coef_node_pf(cn1, ci1, mi1, pi1, slot1);
                }
            } else if (PAIR && ty * TX < NHALO) {
                coef_pair();
            } else {
                coef_node(cn0, ci0, mi0, pi0);
                if (!PAIR && has_rim) coef_node(cn1, ci1, mi1, pi1);
            }
        }
        // phase field: candidates of the next source plane (its phi is staged)
        if (MODE == TSLB_MODE_PHASEFIELD) {
            if (more) list_candidates(s + 1);
            else slot0 = slot1 = -1;
        }
        // VEC: all copies issued so far (moments of s+1, phi of s+2) land before the
        // barrier, which also makes them visible for the next plane's coefficients
        if (VEC) cp_async_wait<0>();
        else cp_async_wait<1>();  // this thread's phi copies of plane s+2 have landed
        __syncthreads();
        // ---- 2. pull ----
        if (active) {
            const CNode Kc = cnode(coef, (ty + 1) * CW + (tx + 1));
            float phm = 0.f, ph0 = 0.f, php = 0.f;
            if (MODE == TSLB_MODE_COLOUR) {
                // own-column phi of the target planes s-1 .. s+1
                const int po = (ty + PHR) * SW + (tx + EPC);
                phm = cvt_in<T>(phis[((s - 1) & (PRING - 1)) * PAREA + po], a, F_PHI);
                ph0 = cvt_in<T>(phis[(s & (PRING - 1)) * PAREA + po], a, F_PHI);
                php = cvt_in<T>(phis[((s + 1) & (PRING - 1)) * PAREA + po], a, F_PHI);
            }
            if (!zsolid) {
                pull_row<MODE, -1>(Kc, accm, acc0, accp, phm, ph0, php);
                pull_row<MODE, 0>(Kc, accm, acc0, accp, phm, ph0, php);
                pull_row<MODE, 1>(Kc, accm, acc0, accp, phm, ph0, php);
            }
            // ---- 3. populations from behind non-periodic faces, target plane s ----
            if (s >= z0 && s < z1) {
                unsigned mask = colmask;
                if (!zper && s == 0) mask |= 16u;
                if (!zper && s == a.nz - 1) mask |= 32u;
                const bool near_solid = SOLID && bit_at(a.near, (long long)s * plane + cn0.off);
                if (mask || near_solid) boundary_target<MODE, T, TAU, SOLID>(a, Kc, mask, X, Y, s, acc0);
            }
            // ---- 4. target plane s-1 is complete ----
            const int t = s - 1;
            if (t >= z0 && t < z1) {
                const float d = accm[A_RHO], rho = 1.f + d, inv = 1.f / rho;
                const float u = accm[A_JX] * inv, v = accm[A_JY] * inv, w = accm[A_JZ] * inv;
                const float d3 = d * (1.f / 3.f);
                float o[NF];
                o[F_D] = d;
                o[F_U] = u; o[F_V] = v; o[F_W] = w;
                o[F_XX] = accm[A_XX] - d3 - rho * u * u;
                o[F_YY] = accm[A_YY] - d3 - rho * v * v;
                o[F_ZZ] = accm[A_ZZ] - d3 - rho * w * w;
                o[F_XY] = accm[A_XY] - rho * u * v;
                o[F_XZ] = accm[A_XZ] - rho * u * w;
                o[F_YZ] = accm[A_YZ] - rho * v * w;
                // colour mode: phi_t + (colour increment) / rho
                o[F_PHI] = MODE == TSLB_MODE_COLOUR ? fmaf(accm[A_COL], inv, phm) : accm[A_COL];
                T* po = gout + (long long)t * plane + cn0.off;
                if (SOLID && bit_at(a.solid, (long long)t * plane + cn0.off)) {
                    // interior solid nodes keep their moments
                    const T* pi = gin + (long long)t * plane + cn0.off;
#pragma unroll
                    for (int f = 0; f < NF; ++f) po[f * a.N] = pi[f * a.N];
                } else {
                // single-component mode does not step phi (held at 1 in both buffers)
                constexpr int nout = MODE == TSLB_MODE_SINGLE ? F_PHI : NF;
                bool bad;
                if constexpr (sizeof(T) == 2) {
                    // 16-bit storage: two fields per conversion (store_pair16), stochastic
                    // rounding seeded by the node (its index in the whole lattice) and the step
                    const unsigned int hnode = sr_node((unsigned int)((t + a.zoff) * plane + cn0.off), sr_step);
                    float vmax = 0.f;
#pragma unroll
                    for (int f = 0; f < nout; f += 2) {
                        const int g = f + 1 < nout ? f + 1 : f;
                        vmax = fmaxf(vmax, store_pair16<T>(po, a, f, g, o[f], o[g], a.sr, sr_field(hnode, f)));
                    }
                    // non-finite, or beyond the storage's range (NaN fails the comparison)
                    bad = !(vmax <= Stor16Max<T>::value);
                } else {
                    float chk = 0.f;
#pragma unroll
                    for (int f = 0; f < nout; ++f) {
                        po[f * a.N] = o[f];
                        chk += o[f];
                    }
                    bad = !isfinite(chk);
                }
                if (bad) atomicOr(a.flags, 1u);
                }
            }
        }
        // rotate the target slots
#pragma unroll
        for (int i = 0; i < NACC; ++i) { accm[i] = acc0[i]; acc0[i] = accp[i]; accp[i] = 0.f; }
        buf ^= 1;
    }
    cp_async_wait<0>();
}

template <int MODE, bool VEC, class T, bool TAU = false, bool SOLID = false>
__global__ void __launch_bounds__(NTHR, 2) step_kernel(const StepArgs a) {
    step_block<MODE, VEC, T, TAU, SOLID>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Work item of the ensemble kernel: lattice, tile column, z chunk.
struct WorkItem {
    int dom, bx, by, bz;
};

// Ensemble step: blocks walk a list of work items over many independent
// lattices; each item is one tile column and z chunk of one lattice.  Block
// b starts with item b; later items go, in list order (longest first), to
// whichever block asks next (a work counter), so a grid smaller than the
// list balances items of uneven length.  The lattice's arguments are staged
// in shared memory when the block moves to a new lattice.  All lattices
// share MODE, VEC and T.  step[0] is the step counter that seeds the
// stochastic rounding (every member's arguments point at it), step[1] a
// ticket and step[2] the work counter: the last block of the launch to
// finish, after every block has read the step and taken its last item,
// advances the step and clears the other two for the next launch.
template <int MODE, bool VEC, class T>
__global__ void __launch_bounds__(NTHR, 2) ensemble_kernel(const StepArgs* __restrict__ args,
                                                          const WorkItem* __restrict__ work, int nwork,
                                                          unsigned int* step) {
    __shared__ StepArgs sa;
    __shared__ int next;
    int cur = -1;
    for (int it = blockIdx.x; it < nwork;) {
        const WorkItem w = work[it];
        if (w.dom != cur) {
            __syncthreads();
            const int words = (int)(sizeof(StepArgs) / sizeof(int));
            const int* src = reinterpret_cast<const int*>(args + w.dom);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.y * TX + threadIdx.x; i < words; i += NTHR) dst[i] = src[i];
            __syncthreads();
            cur = w.dom;
        }
        step_block<MODE, VEC, T, false, false, MODE != TSLB_MODE_PHASEFIELD>(sa, w.bx, w.by, w.bz);
        __syncthreads();
        // every thread has read `next` (it was read before this item's barriers)
        if (step) {
            if (threadIdx.x == 0 && threadIdx.y == 0) next = (int)gridDim.x + (int)atomicAdd(step + 2, 1u);
            __syncthreads();
            it = next;
        } else {
            it += gridDim.x;
        }
    }
    if (step && threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        if (atomicAdd(step + 1, 1u) == gridDim.x - 1) {
            step[1] = 0;
            step[2] = 0;
            step[0] += 1;
            __threadfence();
        }
    }
}

}  // namespace tslb
