// tslb_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's two-component TSLB step, used as the
// parity checker of the CUDA path.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg use it; nothing in the product links it.
//
// It keeps the reference's structure: populations f (D3Q27) and g (D3Q7
// in phase-field mode, a second D3Q27 set in colour mode) stored with a
// one-node halo, a moments pass, a normals pass, a collision that PUSHES
// post-collision populations to x+c_i, and boundary conditions applied to
// the pushed populations.  Paths below are relative to the reference repo.
//
//   lattice, weights          recursive_2c_TSLB3D.f90:71-77, vars_single_3D_module.f90
//   moments pass              recursive_2c_TSLB3D.f90:346-542
//   normals pass              recursive_2c_TSLB3D.f90:543-577
//   collision + push          recursive_2c_TSLB3D.f90:607-836
//   body force (velocity shift) TSLB_2C-mpi/lb_kernels_module.f90:769
//   colour-gradient operator  turbulent_benchmark/couette/recursive_colorTSLB3D.f90:468-1108
//                             (with the fixes listed at colour_collide_push)
//   bounce-back               boundary_cds_3D_module.f90:10-76
//   regularized velocity faces boundary_cds_3D_module.f90:405-629 (Couette),
//                             :931-1048 (jet inlet / outlet)
//   periodic wrap             TSLB_2C-mpi/mpi_module.f90:2083-2118
//
// The equilibrium f^eq_i(rho,u) and the regularized non-equilibrium
// a^neq_i(Pi,u) are evaluated from their third-order Hermite form
// (w_i [rho + 3 c.u + 4.5 H2:uu + H3 terms]); the reference writes the same
// polynomials expanded per direction.  Agreement of the two forms is pinned
// by tests/golden (the reference's own statements evaluated with numpy).
//
// Templated on the real type: float restates the reference's db=4 build,
// double its PRC=8 build.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/tslb.h"

namespace orc {

// D3Q27 in the reference's numbering (recursive_2c_TSLB3D.f90:549-552).
static const int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1};
static const int CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1};
static const int CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1};
static const int OPP[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
// Order in which the moments pass accumulates Pi^neq (recursive_2c_TSLB3D.f90:377-536).
static const int PI_ORDER[26] = {1, 2, 3, 4, 5, 6, 7, 8, 10, 9, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26};
// D3Q7 of the phase field g (recursive_2c_TSLB3D.f90:808-831).
static const int GX[7] = {0, 1, -1, 0, 0, 0, 0};
static const int GY[7] = {0, 0, 0, 1, -1, 0, 0};
static const int GZ[7] = {0, 0, 0, 0, 0, 1, -1};
static const int GOPP[7] = {0, 2, 1, 4, 3, 6, 5};

enum Field { RHO = 0, UX, UY, UZ, PXX, PXY, PXZ, PYY, PYZ, PZZ, PHI, NFIELD };

inline int cls(int i) { return CX[i] * CX[i] + CY[i] * CY[i] + CZ[i] * CZ[i]; }

template <class R>
struct Weights {
    R p[4];   // by |c|^2: p0 = 8/27, p1 = 2/27, p2 = 1/54, p3 = 1/216
    R b0;     // colour perturbation B_0 = -10/27 (recursive_colorTSLB3D.f90:81)
    Weights() {
        p[0] = R(8) / R(27);
        p[1] = R(2) / R(27);
        p[2] = R(1) / R(54);
        p[3] = R(1) / R(216);
        b0 = R(-10) / R(27);
    }
    R w(int i) const { return p[cls(i)]; }
};

// Third-order Hermite polynomials of direction i (D3Q27 supports
// xxy, xxz, xyy, yyz, xzz, yzz, xyz).
template <class R>
struct Herm {
    R h2xx, h2yy, h2zz, h2xy, h2xz, h2yz;
    R hxxy, hxxz, hxyy, hyyz, hxzz, hyzz, hxyz;
    explicit Herm(int i) {
        const R cx = R(CX[i]), cy = R(CY[i]), cz = R(CZ[i]);
        const R t = R(1) / R(3);
        h2xx = cx * cx - t; h2yy = cy * cy - t; h2zz = cz * cz - t;
        h2xy = cx * cy; h2xz = cx * cz; h2yz = cy * cz;
        hxxy = (cx * cx - t) * cy; hxxz = (cx * cx - t) * cz;
        hxyy = (cy * cy - t) * cx; hyyz = (cy * cy - t) * cz;
        hxzz = (cz * cz - t) * cx; hyzz = (cz * cz - t) * cy;
        hxyz = cx * cy * cz;
    }
};

// f^eq_i(rho,u) / w_i: the expanded per-direction polynomials of
// recursive_2c_TSLB3D.f90:113-252 (and :378-529), in Hermite form.
template <class R>
inline R feq_over_w(int i, R rho, R u, R v, R w) {
    const Herm<R> H(i);
    const R cu = R(CX[i]) * u + R(CY[i]) * v + R(CZ[i]) * w;
    const R uu = u * u + v * v + w * w;
    const R h3 = R(13.5) * (H.hxxy * u * u * v + H.hxxz * u * u * w + H.hxyy * u * v * v +
                            H.hyyz * v * v * w + H.hxzz * u * w * w + H.hyzz * v * w * w) +
                 R(27) * H.hxyz * u * v * w;
    return rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uu + h3);
}

// a^neq_i(Pi,u): the "fneq1" polynomials of recursive_2c_TSLB3D.f90:640-805,
// i.e. 4.5 H2:Pi + recursive third-order terms (u_a Pi_bc + perms).
template <class R>
inline R aneq(int i, const R* P /*xx,xy,xz,yy,yz,zz*/, R u, R v, R w) {
    const Herm<R> H(i);
    const R pxx = P[0], pxy = P[1], pxz = P[2], pyy = P[3], pyz = P[4], pzz = P[5];
    const R h2 = H.h2xx * pxx + H.h2yy * pyy + H.h2zz * pzz +
                 R(2) * (H.h2xy * pxy + H.h2xz * pxz + H.h2yz * pyz);
    const R a_xxy = R(2) * u * pxy + v * pxx;
    const R a_xxz = R(2) * u * pxz + w * pxx;
    const R a_xyy = u * pyy + R(2) * v * pxy;
    const R a_yyz = R(2) * v * pyz + w * pyy;
    const R a_xzz = u * pzz + R(2) * w * pxz;
    const R a_yzz = v * pzz + R(2) * w * pyz;
    const R a_xyz = u * pyz + v * pxz + w * pxy;
    const R h3 = R(13.5) * (H.hxxy * a_xxy + H.hxxz * a_xxz + H.hxyy * a_xyy +
                            H.hyyz * a_yyz + H.hxzz * a_xzz + H.hyzz * a_yzz) +
                 R(27) * H.hxyz * a_xyz;
    return R(4.5) * h2 + h3;
}

template <class R>
struct Oracle {
    tslb_params prm;
    int nx, ny, nz, sx, sy, sz;
    size_t vol;
    bool colour;
    Weights<R> W;
    std::vector<R> f, g;                 // populations with halo
    std::vector<R> M[NFIELD];            // moment fields with halo
    std::vector<R> nrm[3];               // interface normals with halo (phase field)
    std::vector<R> inlet[6];             // per-face inlet planes: u,v,w,phi
    int nq_g;

    Oracle(const tslb_params& p, int nx_, int ny_, int nz_)
        : prm(p), nx(nx_), ny(ny_), nz(nz_), sx(nx_ + 2), sy(ny_ + 2), sz(nz_ + 2) {
        vol = size_t(sx) * sy * sz;
        colour = p.mode == TSLB_MODE_COLOUR;
        // TSLB_MODE_SINGLE runs as the phase-field step: at sigma = 0 (or with a uniform
        // phi) the CSF force vanishes and its f step is fused_TSLB_force_1c
        // (TSLB_2C-mpi/lb_kernels_module.f90:574-736)
        nq_g = colour ? 27 : 7;
        f.assign(27 * vol, R(0));
        g.assign(size_t(nq_g) * vol, R(0));
        for (auto& m : M) m.assign(vol, R(0));
        for (auto& n : nrm) n.assign(vol, R(0));
        for (int fc = 0; fc < 6; ++fc) {
            int a = fc / 2;
            size_t area = a == 0 ? size_t(ny) * nz : a == 1 ? size_t(nx) * nz : size_t(nx) * ny;
            inlet[fc].assign(4 * area, R(0));
        }
    }

    // ---- indexing (0-based interior i in [0,nx), halo -1 and nx) ----
    size_t id(int i, int j, int k) const {
        return size_t(i + 1) + size_t(sx) * (size_t(j + 1) + size_t(sy) * size_t(k + 1));
    }
    size_t iid(int i, int j, int k) const {  // interior Fortran-order index
        return size_t(i) + size_t(nx) * (size_t(j) + size_t(ny) * size_t(k));
    }
    int dim(int a) const { return a == 0 ? nx : a == 1 ? ny : nz; }
    bool periodic(int a) const { return prm.bc[2 * a] == TSLB_BC_PERIODIC; }
    static bool velocity_kind(int bc) {
        return bc == TSLB_BC_VELOCITY || bc == TSLB_BC_INLET || bc == TSLB_BC_OUTLET || bc == TSLB_BC_PRESSURE;
    }
    R& F(int q, int i, int j, int k) { return f[size_t(q) * vol + id(i, j, k)]; }
    R& G(int q, int i, int j, int k) { return g[size_t(q) * vol + id(i, j, k)]; }
    R omega_pf() const { return R(1) / R(prm.tau_a); }

    // interior solid nodes (the reference's isfluid == 0; empty: none).  Solid
    // nodes are not stepped (moments kept, no push), their normals are 0, and
    // populations entering fluid nodes from them are bounced back
    // (boundary_cds_3D_module.f90:11-76 applied at every isfluid == 0 node).
    std::vector<unsigned char> isfluid;
    bool solid_at(int i, int j, int k) const { return !isfluid.empty() && !isfluid[iid(i, j, k)]; }

    // per-node correction of the colour-mode relaxation time (empty: none);
    // the B200 path's tslb_set_tau_correction and learned closure
    std::vector<R> dtau;
    R node_dtau(int i, int j, int k) const { return dtau.empty() ? R(0) : dtau[iid(i, j, k)]; }
    // omega = 1/tau with tau = 3 nu + 1/2 (+ dtau)
    R omega_colour(R nu, int i, int j, int k) const {
        if (dtau.empty()) return R(2) / (R(6) * nu + R(1));
        return R(1) / (R(3) * nu + R(0.5) + node_dtau(i, j, k));
    }

    // inlet plane value of face fc at the in-plane coordinates of node (i,j,k)
    size_t plane_index(int fc, int i, int j, int k) const {
        int a = fc / 2;
        if (a == 0) return size_t(j) + size_t(ny) * size_t(k);
        if (a == 1) return size_t(i) + size_t(nx) * size_t(k);
        return size_t(i) + size_t(nx) * size_t(j);
    }
    R inlet_val(int fc, int comp, int i, int j, int k) const {
        int a = fc / 2;
        size_t area = a == 0 ? size_t(ny) * nz : a == 1 ? size_t(nx) * nz : size_t(nx) * ny;
        return inlet[fc][size_t(comp) * area + plane_index(fc, i, j, k)];
    }

    // ---- halo fill of a scalar field ----
    // Periodic axes wrap (the MPI exchange_float / intpbc semantics); solid
    // faces get the ghost value: the inlet plane's phi on inlet faces, else
    // bc_phi[face] (wall_phi_mode 0), the nearest interior value (mirror,
    // wall_phi_mode 1), or `solid_value` when use_solid_value is set.
    void fill_halo(std::vector<R>& fld, bool is_phi, bool use_solid_value, R solid_value) {
        for (int k = -1; k <= nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    bool inside = i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
                    if (inside) continue;
                    int c[3] = {i, j, k};
                    int wall_face = -1;
                    for (int a = 0; a < 3; ++a) {
                        int n = dim(a);
                        if (c[a] < 0 || c[a] >= n) {
                            if (periodic(a)) {
                                c[a] = (c[a] + n) % n;
                            } else {
                                if (wall_face < 0) wall_face = 2 * a + (c[a] >= n ? 1 : 0);
                                c[a] = c[a] < 0 ? 0 : n - 1;
                            }
                        }
                    }
                    R val;
                    if (wall_face < 0) {
                        val = fld[id(c[0], c[1], c[2])];
                    } else if (use_solid_value) {
                        val = solid_value;
                    } else if (is_phi && prm.bc[wall_face] == TSLB_BC_INLET) {
                        val = inlet_val(wall_face, 3, c[0], c[1], c[2]);
                    } else if (is_phi && prm.wall_phi_mode == 0) {
                        val = R(prm.bc_phi[wall_face]);
                    } else {
                        val = fld[id(c[0], c[1], c[2])];
                    }
                    fld[id(i, j, k)] = val;
                }
    }

    // isotropic 26-neighbour gradient 3 sum_i p_i c_i s(x+c_i)
    // (recursive_2c_TSLB3D.f90:555-565, recursive_colorTSLB3D.f90:726-744)
    void grad(const std::vector<R>& s, int i, int j, int k, R out[3]) const {
        R gx = 0, gy = 0, gz = 0;
        for (int q = 1; q < 27; ++q) {
            R val = W.w(q) * s[id(i + CX[q], j + CY[q], k + CZ[q])];
            gx += R(CX[q]) * val;
            gy += R(CY[q]) * val;
            gz += R(CZ[q]) * val;
        }
        out[0] = R(3) * gx;
        out[1] = R(3) * gy;
        out[2] = R(3) * gz;
    }

    // ------------------------------------------------------------------
    // Moments pass (recursive_2c_TSLB3D.f90:346-542; colour form
    // recursive_colorTSLB3D.f90:482-671 with u from the total populations
    // of both sets divided by their total density).
    void moments_pass() {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    if (solid_at(i, j, k)) continue;  // solid nodes keep their moments
                    size_t x = id(i, j, k);
                    R tot[27];
                    R rho_a = 0, rho_b = 0;
                    for (int q = 0; q < 27; ++q) {
                        R fa = f[size_t(q) * vol + x];
                        rho_a += fa;
                        tot[q] = fa;
                    }
                    R phi = 0;
                    if (colour) {
                        for (int q = 0; q < 27; ++q) {
                            R gb = g[size_t(q) * vol + x];
                            rho_b += gb;
                            tot[q] += gb;
                        }
                    } else {
                        for (int q = 0; q < 7; ++q) phi += g[size_t(q) * vol + x];
                    }
                    R rho = colour ? rho_a + rho_b : rho_a;
                    if (colour) phi = (rho_a - rho_b) / rho;
                    R sp[3] = {0, 0, 0}, sm[3] = {0, 0, 0};
                    for (int q = 1; q < 27; ++q) {
                        const int c[3] = {CX[q], CY[q], CZ[q]};
                        for (int a = 0; a < 3; ++a) {
                            if (c[a] > 0) sp[a] += tot[q];
                            if (c[a] < 0) sm[a] += tot[q];
                        }
                    }
                    R u = (sp[0] - sm[0]) / rho, v = (sp[1] - sm[1]) / rho, w = (sp[2] - sm[2]) / rho;
                    R P[6] = {0, 0, 0, 0, 0, 0};
                    for (int n = 0; n < 26; ++n) {
                        int q = PI_ORDER[n];
                        R fneq = tot[q] - W.w(q) * feq_over_w<R>(q, rho, u, v, w);
                        const int cx = CX[q], cy = CY[q], cz = CZ[q];
                        if (cx) P[0] += fneq;
                        if (cx * cy > 0) P[1] += fneq; else if (cx * cy < 0) P[1] -= fneq;
                        if (cx * cz > 0) P[2] += fneq; else if (cx * cz < 0) P[2] -= fneq;
                        if (cy) P[3] += fneq;
                        if (cy * cz > 0) P[4] += fneq; else if (cy * cz < 0) P[4] -= fneq;
                        if (cz) P[5] += fneq;
                    }
                    M[RHO][x] = rho;
                    M[UX][x] = u; M[UY][x] = v; M[UZ][x] = w;
                    for (int c = 0; c < 6; ++c) M[PXX + c][x] = P[c];
                    M[PHI][x] = phi;
                }
    }

    // Normals pass (recursive_2c_TSLB3D.f90:543-577): n = grad phi / (|grad phi| + 1e-9).
    void normals_pass() {
        fill_halo(M[PHI], true, false, R(0));
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    R gr[3];
                    grad(M[PHI], i, j, k, gr);
                    R mod = std::sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
                    R den = mod + R(1e-9);
                    size_t x = id(i, j, k);
                    if (solid_at(i, j, k)) gr[0] = gr[1] = gr[2] = R(0);
                    nrm[0][x] = gr[0] / den;
                    nrm[1][x] = gr[1] / den;
                    nrm[2][x] = gr[2] / den;
                }
        for (int a = 0; a < 3; ++a) fill_halo(nrm[a], false, true, R(0));
    }

    // Phase-field collision + push (recursive_2c_TSLB3D.f90:607-836).
    void phasefield_collide_push() {
        const R omega = omega_pf();
        const R sigma = R(prm.sigma), sharp = R(prm.sharp_c);
        const R p0g = R(1) / R(4), p1g = R(1) / R(8);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    if (solid_at(i, j, k)) continue;
                    size_t x = id(i, j, k);
                    const R rho = M[RHO][x], u = M[UX][x], v = M[UY][x], w = M[UZ][x];
                    const R P[6] = {M[PXX][x], M[PXY][x], M[PXZ][x], M[PYY][x], M[PYZ][x], M[PZZ][x]};
                    const R phi = M[PHI][x];
                    const R n0 = nrm[0][x], n1 = nrm[1][x], n2 = nrm[2][x];
                    R curv = 0;
                    R ind = phi * (R(1) - phi) * (n0 * n0 + n1 * n1 + n2 * n2);
                    if (ind > R(0.2)) {
                        R gx[3], gy[3], gz[3];
                        grad(nrm[0], i, j, k, gx);
                        grad(nrm[1], i, j, k, gy);
                        grad(nrm[2], i, j, k, gz);
                        curv = -(gx[0] + gy[1] + gz[2]);
                    }
                    const R us = u + sigma * curv * n0 + R(prm.force[0]);
                    const R vs = v + sigma * curv * n1 + R(prm.force[1]);
                    const R ws = w + sigma * curv * n2 + R(prm.force[2]);
                    for (int q = 0; q < 27; ++q) {
                        R val = W.w(q) * feq_over_w<R>(q, rho, us, vs, ws) +
                                (R(1) - omega) * aneq<R>(q, P, u, v, w) * W.w(q);
                        F(q, i + CX[q], j + CY[q], k + CZ[q]) = val;
                    }
                    G(0, i, j, k) = p0g * phi;
                    const R uvw[3] = {u, v, w};
                    const R nn[3] = {n0, n1, n2};
                    for (int q = 1; q < 7; ++q) {
                        int a = (q - 1) / 2;
                        R sgn = (q % 2 == 1) ? R(1) : R(-1);
                        R eq = p1g * phi * (R(1) + sgn * R(3) * uvw[a]);
                        R sh = p1g * sharp * phi * (R(1) - phi) * nn[a];
                        G(q, i + GX[q], j + GY[q], k + GZ[q]) = eq + sgn * sh;
                    }
                }
    }

    // Colour-gradient collision + push: the operator of
    // recursive_colorTSLB3D.f90:719-1104 with these fixes (the draft does
    // not compile):
    //  - psi = (rhoA - rhoB)/(rhoA + rhoB) (the draft inverts it, :511);
    //  - every f^eq uses the total density (the draft mixes in an
    //    undeclared `rho`, :534,774,...);
    //  - the perturbation is the published form
    //    (A/2)|grad psi| [w_i (c_i.grad psi)^2/|grad psi|^2 - B_i]
    //    (the draft omits the square, :772);
    //  - the recolouring is beta (rhoA rhoB/rho^2) w_i rho cos(theta_i),
    //    cos(theta_i) = c_i.grad psi/(|c_i||grad psi|) (the draft divides
    //    by |grad psi|^2, :773);
    //  - all 27 directions of both components are written in both the
    //    interface and the bulk branch (the draft drops g in several).
    // The force is the draft's population source p_i c_i.F / cs^2 (:776).
    // A = colour_surface_coeff * sigma * omega.
    R colour_surface_coeff() const { return R(4.5); }

    void colour_collide_push() {
        fill_halo(M[PHI], true, false, R(0));
        const R nu_a = (R(prm.tau_a) - R(0.5)) / R(3);
        const R nu_b = (R(prm.tau_b) - R(0.5)) / R(3);
        const R beta = R(prm.beta), sigma = R(prm.sigma), thr = R(prm.grad_threshold);
        const R Fx = R(prm.force[0]), Fy = R(prm.force[1]), Fz = R(prm.force[2]);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    if (solid_at(i, j, k)) continue;
                    size_t x = id(i, j, k);
                    const R rho = M[RHO][x], u = M[UX][x], v = M[UY][x], w = M[UZ][x];
                    const R P[6] = {M[PXX][x], M[PXY][x], M[PXZ][x], M[PYY][x], M[PYZ][x], M[PZZ][x]};
                    const R phi = M[PHI][x];
                    const R ca = (R(1) + phi) / R(2), cb = (R(1) - phi) / R(2);  // rhoA/rho, rhoB/rho
                    R gp[3];
                    grad(M[PHI], i, j, k, gp);
                    const R m2 = gp[0] * gp[0] + gp[1] * gp[1] + gp[2] * gp[2];
                    const R m = std::sqrt(m2);
                    const R nu = R(1) / (ca / nu_a + cb / nu_b);
                    // tau = 3 nu + 1/2, plus the per-node correction when set
                    const R omega = omega_colour(nu, i, j, k);
                    const R A = colour_surface_coeff() * sigma * omega;
                    const bool iface = m > thr;
                    const R rec = beta * ca * cb * rho;  // beta rhoA rhoB / rho
                    for (int q = 0; q < 27; ++q) {
                        const R wq = W.w(q);
                        R fpc = wq * feq_over_w<R>(q, rho, u, v, w) +
                                (R(1) - omega) * aneq<R>(q, P, u, v, w) * wq +
                                R(3) * wq * (R(CX[q]) * Fx + R(CY[q]) * Fy + R(CZ[q]) * Fz);
                        R om2 = 0;
                        if (iface) {
                            const R cg = R(CX[q]) * gp[0] + R(CY[q]) * gp[1] + R(CZ[q]) * gp[2];
                            const R bq = q == 0 ? W.b0 : wq;
                            fpc += R(0.5) * A * m * (wq * cg * cg / m2 - bq);
                            if (q != 0) om2 = rec * wq * cg / (std::sqrt(R(cls(q))) * m);
                        }
                        const int ti = i + CX[q], tj = j + CY[q], tk = k + CZ[q];
                        F(q, ti, tj, tk) = fpc * ca + om2;
                        G(q, ti, tj, tk) = fpc * cb - om2;
                    }
                }
    }

    // ------------------------------------------------------------------
    // Boundary conditions on the pushed populations.
    bool out_of_range(int i, int j, int k) const {
        return i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz;
    }

    // Faces of the out-of-range axes of halo node (i,j,k) that are not periodic.
    int wall_faces(int i, int j, int k, int faces[3]) const {
        int c[3] = {i, j, k}, n = 0;
        for (int a = 0; a < 3; ++a) {
            if (periodic(a)) continue;
            if (c[a] < 0) faces[n++] = 2 * a;
            else if (c[a] >= dim(a)) faces[n++] = 2 * a + 1;
        }
        return n;
    }

    // in-plane coordinate of the ghost node a population comes from: periodic
    // axes wrap, a non-periodic axis clamps to the lattice
    int src_coord(int axis, int c) const {
        const int n = dim(axis);
        if (c >= 0 && c < n) return c;
        if (periodic(axis)) return (c % n + n) % n;
        return c < 0 ? 0 : n - 1;
    }

    // Regularized population entering fluid node (i,j,k) from a velocity
    // face in direction q: f^eq(rho_x, U_b) + (1-omega) w a^neq(Pi_x, u_x)
    // (boundary_cds_3D_module.f90:454-629, 931-1048).  U_b is the velocity of
    // the ghost node the population leaves, (i,j,k) - c_q: the inlet plane at
    // that node's in-plane position (:934, w(i,j,k) of the ghost node i,j,1),
    // and for the outlet the normal velocity of the fluid node next to it
    // (:992, w(i,j,nz) = w(i,j,nz-1)).
    void velocity_face_value(int fc, int q, int i, int j, int k) {
        size_t x = id(i, j, k);
        const R rho = M[RHO][x], u = M[UX][x], v = M[UY][x], w = M[UZ][x];
        const R P[6] = {M[PXX][x], M[PXY][x], M[PXZ][x], M[PYY][x], M[PYZ][x], M[PZZ][x]};
        const R phi = M[PHI][x];
        const int bc = prm.bc[fc];
        const int axis = fc / 2;
        R Ub[3] = {R(prm.bc_u[fc][0]), R(prm.bc_u[fc][1]), R(prm.bc_u[fc][2])};
        R phib = prm.bc_phi[fc] < -2.0f ? phi : R(prm.bc_phi[fc]);
        // the ghost node's in-plane position; the layer coordinate stays the target's
        int g[3] = {i, j, k};
        const int cq[3] = {CX[q], CY[q], CZ[q]};
        for (int a = 0; a < 3; ++a)
            if (a != axis) g[a] = src_coord(a, g[a] - cq[a]);
        if (bc == TSLB_BC_INLET) {
            for (int a = 0; a < 3; ++a) Ub[a] = inlet_val(fc, a, g[0], g[1], g[2]);
            phib = inlet_val(fc, 3, g[0], g[1], g[2]);
        } else if (bc == TSLB_BC_OUTLET) {
            Ub[axis] = M[UX + axis][id(g[0], g[1], g[2])];
            phib = phi;
        }
        R rho_b = rho;
        if (bc == TSLB_BC_PRESSURE) {
            // pressure outlet (no reference counterpart): density 1, the node's velocity and phi
            const R uvw[3] = {u, v, w};
            for (int a = 0; a < 3; ++a) Ub[a] = uvw[a];
            phib = phi;
            rho_b = R(1);
        }
        R omega;
        if (colour) {
            const R nu_a = (R(prm.tau_a) - R(0.5)) / R(3), nu_b = (R(prm.tau_b) - R(0.5)) / R(3);
            const R ca = (R(1) + phi) / R(2), cb = (R(1) - phi) / R(2);
            const R nu = R(1) / (ca / nu_a + cb / nu_b);
            omega = omega_colour(nu, i, j, k);
        } else {
            omega = omega_pf();
        }
        const R wq = W.w(q);
        R val = wq * feq_over_w<R>(q, rho_b, Ub[0], Ub[1], Ub[2]) + (R(1) - omega) * wq * aneq<R>(q, P, u, v, w);
        if (colour) {
            F(q, i, j, k) = val * (R(1) + phib) / R(2);
            G(q, i, j, k) = val * (R(1) - phib) / R(2);
        } else {
            F(q, i, j, k) = val;
        }
    }

    // phase-field g entering from a velocity face (jet inlet g5 :984-986,
    // outlet g6 :1044-1045)
    void velocity_face_g(int fc, int q, int i, int j, int k) {
        size_t x = id(i, j, k);
        const R phi = M[PHI][x];
        const int bc = prm.bc[fc];
        R Ub[3] = {R(prm.bc_u[fc][0]), R(prm.bc_u[fc][1]), R(prm.bc_u[fc][2])};
        R phib = prm.bc_phi[fc] < -2.0f ? phi : R(prm.bc_phi[fc]);
        if (bc == TSLB_BC_INLET) {
            for (int a = 0; a < 3; ++a) Ub[a] = inlet_val(fc, a, i, j, k);
            phib = inlet_val(fc, 3, i, j, k);
        } else if (bc == TSLB_BC_OUTLET || bc == TSLB_BC_PRESSURE) {
            phib = phi;
        }
        const R eu = R(GX[q]) * Ub[0] + R(GY[q]) * Ub[1] + R(GZ[q]) * Ub[2];
        G(q, i, j, k) = (R(1) / R(8)) * phib * (R(1) + R(3) * eu);
    }

    void boundary_conditions() {
        // (1) bounce-back from solid halo nodes of bounce-back faces:
        //     f(x+c_i, i) = f(x, opp(i)) (boundary_cds_3D_module.f90:11-76).
        for (int k = -1; k <= nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    if (!out_of_range(i, j, k)) continue;
                    int faces[3];
                    int nf = wall_faces(i, j, k, faces);
                    if (nf == 0) continue;
                    bool bb = false;
                    for (int n = 0; n < nf; ++n) bb |= prm.bc[faces[n]] == TSLB_BC_BOUNCEBACK;
                    if (!bb) continue;
                    for (int q = 1; q < 27; ++q) {
                        int ti = i + CX[q], tj = j + CY[q], tk = k + CZ[q];
                        if (out_of_range(ti, tj, tk)) continue;
                        F(q, ti, tj, tk) = F(OPP[q], i, j, k);
                        if (colour) G(q, ti, tj, tk) = G(OPP[q], i, j, k);
                    }
                    if (!colour)
                        for (int q = 1; q < 7; ++q) {
                            int ti = i + GX[q], tj = j + GY[q], tk = k + GZ[q];
                            if (out_of_range(ti, tj, tk)) continue;
                            G(q, ti, tj, tk) = G(GOPP[q], i, j, k);
                        }
                }
        // (2) regularized velocity faces overwrite every population whose
        //     source lies in the face layer.
        for (int fc = 0; fc < 6; ++fc) {
            if (!velocity_kind(prm.bc[fc])) continue;
            const int a = fc / 2, side = fc % 2;
            const int layer = side ? dim(a) - 1 : 0;
            const int inward = side ? -1 : 1;
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        int c[3] = {i, j, k};
                        if (c[a] != layer) continue;
                        for (int q = 1; q < 27; ++q) {
                            const int cq[3] = {CX[q], CY[q], CZ[q]};
                            if (cq[a] != inward) continue;
                            velocity_face_value(fc, q, i, j, k);
                        }
                        if (!colour)
                            for (int q = 1; q < 7; ++q) {
                                const int cq[3] = {GX[q], GY[q], GZ[q]};
                                if (cq[a] != inward) continue;
                                velocity_face_g(fc, q, i, j, k);
                            }
                    }
        }
        // (3) periodic wrap of populations that left through periodic faces
        //     only (mpi_module.f90:2083-2118: oi = mod(oi+nx-1,nx)+1).
        for (int k = -1; k <= nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    if (!out_of_range(i, j, k)) continue;
                    int faces[3];
                    if (wall_faces(i, j, k, faces) > 0) continue;
                    int wi = (i + nx) % nx, wj = (j + ny) % ny, wk = (k + nz) % nz;
                    for (int q = 1; q < 27; ++q) {
                        // only populations that were pushed into this halo node
                        int si = i - CX[q], sj = j - CY[q], sk = k - CZ[q];
                        if (out_of_range(si, sj, sk)) continue;
                        F(q, wi, wj, wk) = F(q, i, j, k);
                        if (colour) G(q, wi, wj, wk) = G(q, i, j, k);
                    }
                    if (!colour)
                        for (int q = 1; q < 7; ++q) {
                            int si = i - GX[q], sj = j - GY[q], sk = k - GZ[q];
                            if (out_of_range(si, sj, sk)) continue;
                            G(q, wi, wj, wk) = G(q, i, j, k);
                        }
                }
        // (4) half-way bounce-back at interior solid nodes, after the wrap so
        //     that populations that crossed a periodic face have arrived:
        //     f(x+c_i, i) = f(x, opp(i)) for fluid x+c_i (periodic axes wrap)
        if (!isfluid.empty()) {
            auto wrap = [&](int v, int a, bool& ok) {
                const int n = dim(a);
                if (v >= 0 && v < n) return v;
                if (periodic(a)) return (v + n) % n;
                ok = false;
                return v;
            };
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        if (!solid_at(i, j, k)) continue;
                        for (int q = 1; q < 27; ++q) {
                            bool ok = true;
                            const int ti = wrap(i + CX[q], 0, ok), tj = wrap(j + CY[q], 1, ok), tk = wrap(k + CZ[q], 2, ok);
                            if (!ok || solid_at(ti, tj, tk)) continue;
                            F(q, ti, tj, tk) = F(OPP[q], i, j, k);
                            if (colour) G(q, ti, tj, tk) = G(OPP[q], i, j, k);
                        }
                        if (!colour)
                            for (int q = 1; q < 7; ++q) {
                                bool ok = true;
                                const int ti = wrap(i + GX[q], 0, ok), tj = wrap(j + GY[q], 1, ok), tk = wrap(k + GZ[q], 2, ok);
                                if (!ok || solid_at(ti, tj, tk)) continue;
                                G(q, ti, tj, tk) = G(GOPP[q], i, j, k);
                            }
                    }
        }
    }

    // ------------------------------------------------------------------
    // One time step with the state held as moments: the reference loop
    // (moments -> normals -> collision -> BC) re-cut so that the moments
    // pass closes the step.
    void step() {
        if (colour) {
            colour_collide_push();
        } else {
            normals_pass();
            phasefield_collide_push();
        }
        boundary_conditions();
        moments_pass();
    }

    // Populations of a moment state: f_i = f^eq_i + w_i a^neq_i at the node,
    // so that the moments pass returns (rho,u,Pi,phi) (lb_kernels_module.f90
    // initial_conditions builds f the same way from rho, u).
    void set_moments(const std::vector<R> in[NFIELD]) {
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t x = id(i, j, k), s = iid(i, j, k);
                    for (int c = 0; c < NFIELD; ++c) M[c][x] = in[c][s];
                }
    }

    void set_pops(const std::vector<R>& fin, const std::vector<R>& gin) {
        size_t n = size_t(nx) * ny * nz;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t x = id(i, j, k), s = iid(i, j, k);
                    for (int q = 0; q < 27; ++q) f[size_t(q) * vol + x] = fin[size_t(q) * n + s];
                    for (int q = 0; q < nq_g; ++q) g[size_t(q) * vol + x] = gin[size_t(q) * n + s];
                }
        moments_pass();
    }

    void get_moments(std::vector<R> out[NFIELD]) const {
        size_t n = size_t(nx) * ny * nz;
        for (int c = 0; c < NFIELD; ++c) out[c].resize(n);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int c = 0; c < NFIELD; ++c) out[c][iid(i, j, k)] = M[c][id(i, j, k)];
    }

    void get_normals(std::vector<R> out[3]) {
        normals_pass();
        size_t n = size_t(nx) * ny * nz;
        for (int c = 0; c < 3; ++c) out[c].resize(n);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int c = 0; c < 3; ++c) out[c][iid(i, j, k)] = nrm[c][id(i, j, k)];
    }

    // FP64 diagnostics in the TSLB_RED_* layout.
    void reduce(double out[TSLB_NREDUCE]) const {
        double s[TSLB_NREDUCE] = {0};
        double umax = 0, rin = 0, rout = 0, nin = 0, nout = 0;
        const double lo = colour ? -0.9 : 0.1;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    size_t x = id(i, j, k);
                    double rho = M[RHO][x], u = M[UX][x], v = M[UY][x], w = M[UZ][x], phi = M[PHI][x];
                    s[TSLB_RED_MASS] += rho;
                    if (colour) {
                        s[TSLB_RED_MASS_A] += rho * (1 + phi) / 2;
                        s[TSLB_RED_MASS_B] += rho * (1 - phi) / 2;
                    } else {
                        s[TSLB_RED_MASS_A] += phi;
                        s[TSLB_RED_MASS_B] += 1 - phi;
                    }
                    s[TSLB_RED_MOM_X] += rho * u;
                    s[TSLB_RED_MOM_Y] += rho * v;
                    s[TSLB_RED_MOM_Z] += rho * w;
                    double uu = u * u + v * v + w * w;
                    s[TSLB_RED_KINETIC] += 0.5 * rho * uu;
                    umax = std::max(umax, std::sqrt(uu));
                    if (phi > 0.9) { rin += rho; nin += 1; }
                    if (phi < lo) { rout += rho; nout += 1; }
                }
        s[TSLB_RED_UMAX] = umax;
        s[TSLB_RED_RHO_IN] = nin > 0 ? rin / nin : 0;
        s[TSLB_RED_RHO_OUT] = nout > 0 ? rout / nout : 0;
        s[TSLB_RED_DP] = (nin > 0 && nout > 0) ? (s[TSLB_RED_RHO_IN] - s[TSLB_RED_RHO_OUT]) / 3.0 : 0;
        s[TSLB_RED_N_IN] = nin;
        std::memcpy(out, s, sizeof(s));
    }
};

}  // namespace orc
