// tslb_step.cuh -- the fused pull step kernel.
//
// One CUDA block owns a TX x TY tile of (x, y) columns and a chunk of
// `zchunk` target planes.  It marches through the source planes
// s = z0-1 .. z1 of the chunk; for each:
//   1. every thread computes the coefficients of P'(c) (tslb_device.cuh) of
//      some nodes of plane s (tile plus a one-node halo) into shared memory
//      (double buffered, one __syncthreads per plane);
//   2. every thread pulls, for its own column, the 27 populations that
//      leave the 9 source nodes (x-ox, y-oy, s) and land on targets
//      (x, y, s-1), (x, y, s), (x, y, s+1), accumulating the targets'
//      moments in registers;
//   3. populations whose source lies behind a non-periodic face are
//      supplied at the target from its own node (bounce-back, regularized
//      velocity faces);
//   4. target plane s-1 is complete: its 11 moments are written out.
// Reading moments and writing moments is all the HBM traffic there is:
// the populations f, g of the reference (recursive_2c_TSLB3D.f90:54) never
// exist in memory.
#pragma once

#include "tslb_device.cuh"

namespace tslb {

// Populations leaving the source node whose coefficients start at Kp
// (stride CAREA) in directions (-OX, -OY, cz), cz = -1, 0, 1.
template <int MODE, int OX, int OY>
__device__ __forceinline__ void pull_lateral(const float* __restrict__ Kp, float* accm, float* acc0, float* accp) {
    constexpr int CXv = -OX, CYv = -OY;
    constexpr int AX = CXv * CXv, AY = CYv * CYv;
    auto L = [&](int slot) { return Kp[slot * CAREA]; };
    // P'(cx,cy,cz) = Q0 + cz Q1 + cz^2 Q2
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
    const float Pm = t - q1, P0 = q0, Pp = t + q1;   // cz = -1, 0, +1
    constexpr float w0 = wclass(AX + AY), w1 = wclass(AX + AY + 1);
    const float fm = w1 * Pm, f0 = w0 * P0, fp = w1 * Pp;
    acc_dir<CXv, CYv, -1>(accm, fm);
    acc_dir<CXv, CYv, 0>(acc0, f0);
    acc_dir<CXv, CYv, 1>(accp, fp);
    if (MODE == TSLB_MODE_COLOUR) {
        // colour: w (phi (1 + P') + (B.c)/|c|); rest population adds delta0
        const float ph = L(K_C0);
        const float bl = (CXv ? CXv * L(K_C1) : 0.f) + (CYv ? CYv * L(K_C2) : 0.f);
        const float bz = L(K_C3);
        constexpr float il0 = invlen(AX + AY), il1 = invlen(AX + AY + 1);
        accm[A_COL] += w1 * fmaf(ph, Pm, ph) + (w1 * il1) * (bl - bz);
        accp[A_COL] += w1 * fmaf(ph, Pp, ph) + (w1 * il1) * (bl + bz);
        if (AX + AY == 0) {
            const float d0 = L(K_C4);
            acc0[A_RHO] += d0;
            acc0[A_COL] += w0 * fmaf(ph, P0, ph) + ph * d0;
        } else {
            acc0[A_COL] += w0 * fmaf(ph, P0, ph) + (w0 * il0) * bl;
        }
    } else {
        // phase field g: axis directions and the rest population only
        if (AX + AY == 0) {
            const float g0 = L(K_C0), gz = L(K_C3);
            accm[A_COL] += g0 - gz;      // q = 6 (-z) leaves the source below... direction (0,0,-1)
            accp[A_COL] += g0 + gz;      // q = 5 (+z)
            acc0[A_COL] += 2.f * g0;     // q = 0: p0g phi = 2 G0
        } else if (AX + AY == 1) {
            const float g0 = L(K_C0);
            const float ge = CXv ? CXv * L(K_C1) : CYv * L(K_C2);
            acc0[A_COL] += g0 + ge;
        }
    }
}

// Regularized or bounce-back populations entering target (x,y,z) from
// behind non-periodic faces; Kp points at the target's own coefficients.
template <int MODE>
__device__ void boundary_target(const StepArgs& a, const float* __restrict__ Kp, unsigned mask, int x, int y, int z, float* acc) {
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
                if (k == TSLB_BC_VELOCITY || k == TSLB_BC_INLET || k == TSLB_BC_OUTLET) vface = f;
            }
        }
        if (!solid) continue;
        const int c2 = dx * dx + dy * dy + dz * dz;
        const float wq = wclass(c2);
        if (vface < 0) {
            // half-way bounce-back: f_c(x) = f^post_{-c}(x)
            const float P = eval_P(Kp, CAREA, -dx, -dy, -dz);
            acc_dir_rt(acc, dx, dy, dz, wq * P);
            if (MODE == TSLB_MODE_COLOUR) {
                const float ph = Kp[K_C0 * CAREA];
                const float bc = -(dx * Kp[K_C1 * CAREA] + dy * Kp[K_C2 * CAREA] + dz * Kp[K_C3 * CAREA]);
                acc[A_COL] += wq * fmaf(ph, P, ph) + wq * invlen(c2) * bc;
            } else if (c2 == 1) {
                const float ge = -(dx * Kp[K_C1 * CAREA] + dy * Kp[K_C2 * CAREA] + dz * Kp[K_C3 * CAREA]);
                acc[A_COL] += Kp[K_C0 * CAREA] + ge;
            }
        } else {
            if (!have_m) {
                const long long id = nidx(a, x, y, z);
#pragma unroll
                for (int f = 0; f < NF; ++f) m[f] = __ldg(a.in + f * a.N + id);
                have_m = true;
            }
            const FaceBC& fb = a.face[vface];
            const int ax = vface >> 1;
            float Ub[3] = {fb.u[0], fb.u[1], fb.u[2]};
            float phib = fb.phi < -2.f ? m[F_PHI] : fb.phi;
            if (fb.kind == TSLB_BC_INLET) {
                const long long pa = plane_area(a, vface), pi = plane_index(a, vface, x, y, z);
                Ub[0] = __ldg(fb.plane + pi);
                Ub[1] = __ldg(fb.plane + pa + pi);
                Ub[2] = __ldg(fb.plane + 2 * pa + pi);
                phib = __ldg(fb.plane + 3 * pa + pi);
            } else if (fb.kind == TSLB_BC_OUTLET) {
                phib = m[F_PHI];
            }
            float Uf[3] = {Ub[0], Ub[1], Ub[2]};  // velocity of the f equilibrium
            if (fb.kind == TSLB_BC_OUTLET) Uf[ax] = m[F_U + ax];
            const float d = m[F_D], rho = 1.f + d;
            float omega;
            if (MODE == TSLB_MODE_COLOUR) {
                const float ca = 0.5f * (1.f + m[F_PHI]), cb = 0.5f * (1.f - m[F_PHI]);
                const float nu = 1.f / (ca * a.inv_nu_a + cb * a.inv_nu_b);
                omega = 2.f / (6.f * nu + 1.f);
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
                acc[A_COL] += wq * fmaf(phib, P, phib);
            } else if (c2 == 1) {
                // g entering from the face (:984-986, :1044-1045)
                const float eu = dx * Ub[0] + dy * Ub[1] + dz * Ub[2];
                acc[A_COL] += 0.125f * phib * (1.f + 3.f * eu);
            }
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(TX * TY, 2) step_kernel(const StepArgs a) {
    extern __shared__ float smem[];  // 2 buffers x NCOEF x CAREA
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * a.zchunk;
    const int z1 = min(z0 + a.zchunk, a.nz);
    const int X = x0 + tx, Y = y0 + ty;
    const bool active = X < a.nx && Y < a.ny;
    const bool xper = a.face[0].kind == TSLB_BC_PERIODIC;
    const bool yper = a.face[2].kind == TSLB_BC_PERIODIC;
    const bool zper = a.face[4].kind == TSLB_BC_PERIODIC;
    // faces the column touches (z faces are added per plane)
    unsigned colmask = 0;
    if (active) {
        if (!xper && X == 0) colmask |= 1u;
        if (!xper && X == a.nx - 1) colmask |= 2u;
        if (!yper && Y == 0) colmask |= 4u;
        if (!yper && Y == a.ny - 1) colmask |= 8u;
    }

    float accm[NACC], acc0[NACC], accp[NACC];
#pragma unroll
    for (int i = 0; i < NACC; ++i) { accm[i] = 0.f; acc0[i] = 0.f; accp[i] = 0.f; }

    int buf = 0;
    for (int s = z0 - 1; s <= z1; ++s) {
        float* coef = smem + buf * (NCOEF * CAREA);
        // ---- 1. coefficients of source plane s (tile + halo) ----
        int gz = s;
        bool zsolid = false;
        if (gz < 0 || gz >= a.nz) {
            if (zper) gz = wrapi(gz, a.nz); else zsolid = true;
        }
        for (int idx = tid; idx < CAREA; idx += TX * TY) {
            const int cyy = idx / CW, cxx = idx - cyy * CW;
            int gx = x0 - 1 + cxx, gy = y0 - 1 + cyy;
            bool solid = zsolid;
            if (gx < 0 || gx >= a.nx) { if (xper) gx = wrapi(gx, a.nx); else solid = true; }
            if (gy < 0 || gy >= a.ny) { if (yper) gy = wrapi(gy, a.ny); else solid = true; }
            float K[NCOEF];
            if (solid) {
#pragma unroll
                for (int c = 0; c < NCOEF; ++c) K[c] = 0.f;
            } else {
                float m[NF];
                const long long id = nidx(a, gx, gy, gz);
#pragma unroll
                for (int f = 0; f < NF; ++f) m[f] = __ldg(a.in + f * a.N + id);
                node_coefs<MODE>(a, m, gx, gy, gz, K);
            }
#pragma unroll
            for (int c = 0; c < NCOEF; ++c) coef[c * CAREA + idx] = K[c];
        }
        __syncthreads();
        // ---- 2. pull ----
        if (active) {
            const float* Kc = coef + (ty + 1) * CW + (tx + 1);
            pull_lateral<MODE, -1, -1>(Kc - CW - 1, accm, acc0, accp);
            pull_lateral<MODE, 0, -1>(Kc - CW, accm, acc0, accp);
            pull_lateral<MODE, 1, -1>(Kc - CW + 1, accm, acc0, accp);
            pull_lateral<MODE, -1, 0>(Kc - 1, accm, acc0, accp);
            pull_lateral<MODE, 0, 0>(Kc, accm, acc0, accp);
            pull_lateral<MODE, 1, 0>(Kc + 1, accm, acc0, accp);
            pull_lateral<MODE, -1, 1>(Kc + CW - 1, accm, acc0, accp);
            pull_lateral<MODE, 0, 1>(Kc + CW, accm, acc0, accp);
            pull_lateral<MODE, 1, 1>(Kc + CW + 1, accm, acc0, accp);
            // ---- 3. populations from behind non-periodic faces, target plane s ----
            if (s >= z0 && s < z1) {
                unsigned mask = colmask;
                if (!zper && s == 0) mask |= 16u;
                if (!zper && s == a.nz - 1) mask |= 32u;
                if (mask) boundary_target<MODE>(a, Kc, mask, X, Y, s, acc0);
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
                o[F_PHI] = MODE == TSLB_MODE_COLOUR ? accm[A_COL] * inv : accm[A_COL];
                const long long id = nidx(a, X, Y, t);
                float chk = 0.f;
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    a.out[f * a.N + id] = o[f];
                    chk += o[f];
                }
                if (!isfinite(chk)) atomicOr(a.flags, 1u);
            }
        }
        // rotate the target slots
#pragma unroll
        for (int i = 0; i < NACC; ++i) { accm[i] = acc0[i]; acc0[i] = accp[i]; accp[i] = 0.f; }
        buf ^= 1;
    }
}

}  // namespace tslb
