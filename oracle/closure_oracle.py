"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the learned closure.

The reference has no closure (its coarse jet, boundary_cds_3D_module.f90:862-1119
with recursive_2c_TSLB3D.f90's loop, runs with the plain tau); this module
restates the B200 closure's definition (include/tslb_closure.h) so the tests
can check the CUDA kernels:

- features of a lattice state (10 per node),
- the fine-to-coarse training samples (box filter of factor 2, subgrid
  stress, least-squares eddy viscosity),
- the network's forward pass and the gradient of the weighted squared loss.

`emulate=True` rounds exactly where the tensor-core kernels round to BF16
(the weights W1, W2, w3, the first bias b1, which the kernels carry as a
weight column against a constant input 1, the normalised input, the hidden
activation h1 and the back-propagated dz2, dz1); everything else is FP64.  `emulate=False` is
the exact FP64 network (used for finite-difference checks of the backward
pass).  Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

NFEAT = 10
NH = 64
OFF = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "w3": 5248, "b3": 5312}
NPARAM = 5313


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (round to nearest even) via FP32; returns float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    bits = a.view(np.uint32).astype(np.uint64)
    lsb = (bits >> 16) & 1
    r = ((bits + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p) -> dict:
    p = np.asarray(p, np.float64)
    return {
        "W1": p[OFF["W1"]:OFF["b1"]].reshape(NH, 16)[:, :NFEAT],
        "b1": p[OFF["b1"]:OFF["W2"]],
        "W2": p[OFF["W2"]:OFF["b2"]].reshape(NH, NH),
        "b2": p[OFF["b2"]:OFF["w3"]],
        "w3": p[OFF["w3"]:OFF["b3"]],
        "b3": p[OFF["b3"]],
    }


def pack_grad(dW1, db1, dW2, db2, dw3, db3) -> np.ndarray:
    g = np.zeros(NPARAM, np.float64)
    w1 = np.zeros((NH, 16))
    w1[:, :NFEAT] = dW1
    g[OFF["W1"]:OFF["b1"]] = w1.reshape(-1)
    g[OFF["b1"]:OFF["W2"]] = db1
    g[OFF["W2"]:OFF["b2"]] = dW2.reshape(-1)
    g[OFF["b2"]:OFF["w3"]] = db2
    g[OFF["w3"]:OFF["b3"]] = dw3
    g[OFF["b3"]] = db3
    return g


def normalised_input(F, mu, sd, emulate: bool) -> np.ndarray:
    F = np.asarray(F, np.float64).reshape(-1, NFEAT)
    if emulate:
        # the kernel computes (f - mu) * (1/sd) in FP32, then rounds to BF16
        f32 = F.astype(np.float32)
        isd = (np.float32(1.0) / np.asarray(sd, np.float32)).astype(np.float32)
        x = ((f32 - np.asarray(mu, np.float32)) * isd).astype(np.float32)
        return bf16(x)
    return (F - np.asarray(mu, np.float64)) / np.asarray(sd, np.float64)


def forward(p, mu, sd, dtau_max, F, emulate: bool = True, dtau_min: float = 0.0):
    """dtau = dtau_min + (dtau_max - dtau_min) sigmoid(o) for feature rows F; returns (y, cache)."""
    w = unpack(p)
    W1, W2, w3, b1 = w["W1"], w["W2"], w["w3"], w["b1"]
    if emulate:
        W1, W2, w3, b1 = bf16(W1), bf16(W2), bf16(w3), bf16(b1)
    x = normalised_input(F, mu, sd, emulate)
    z1 = x @ W1.T + b1
    m1 = z1 > 0
    h1 = np.where(m1, z1, 0.0)
    if emulate:
        h1 = bf16(h1)
    z2 = h1 @ W2.T + w["b2"]
    m2 = z2 > 0
    h2 = np.where(m2, z2, 0.0)
    o = h2 @ w3 + w["b3"]
    sg = 1.0 / (1.0 + np.exp(-o))
    y = dtau_min + (dtau_max - dtau_min) * sg
    cache = dict(x=x, m1=m1, h1=h1, m2=m2, h2=h2, sg=sg, W2=W2, w3=w3, o=o)
    return y, cache


def loss_and_grad(p, mu, sd, dtau_max, F, t, a, emulate: bool = True, dtau_min: float = 0.0):
    """Mean of a (y - t)^2 and its gradient with respect to the parameter vector."""
    y, c = forward(p, mu, sd, dtau_max, F, emulate, dtau_min)
    t = np.asarray(t, np.float64).reshape(-1)
    a = np.asarray(a, np.float64).reshape(-1)
    B = y.shape[0]
    r = y - t
    loss = float(np.sum(a * r * r) / B)
    g = 2.0 / B * a * r * (y - dtau_min) * (1.0 - c["sg"])
    dw3 = c["h2"].T @ g
    db3 = g.sum()
    dz2 = g[:, None] * c["w3"][None, :] * c["m2"]
    if emulate:
        dz2 = bf16(dz2)
    dW2 = dz2.T @ c["h1"]
    db2 = dz2.sum(0)
    dh1 = dz2 @ c["W2"]
    dz1 = dh1 * c["m1"]
    if emulate:
        dz1 = bf16(dz1)
    dW1 = dz1.T @ c["x"]
    db1 = dz1.sum(0)
    return loss, pack_grad(dW1, db1, dW2, db2, dw3, db3)


# ---------------------------------------------------------------- features
def _nbr(x, d, n, periodic):
    y = x + d
    if periodic:
        return y % n
    return np.clip(y, 0, n - 1)


def _central(f, axis, periodic):
    n = f.shape[axis]
    idx = np.arange(n)
    fp = np.take(f, _nbr(idx, 1, n, periodic), axis=axis)
    fm = np.take(f, _nbr(idx, -1, n, periodic), axis=axis)
    return 0.5 * (fp - fm)


def _frob(P):
    return np.sqrt(P[0] ** 2 + P[3] ** 2 + P[5] ** 2 + 2.0 * (P[1] ** 2 + P[2] ** 2 + P[4] ** 2))


def _features(P, phi, gmag, speed, s):
    f = np.empty(phi.shape + (NFEAT,), np.float64)
    for k in range(6):
        f[..., k] = s * P[k]
    f[..., 6] = phi
    f[..., 7] = gmag
    f[..., 8] = speed
    f[..., 9] = s * _frob(P)
    return f


def lattice_features(fields: dict, tau_a: float, tau_b: float, periodic, dtau_prev=None) -> np.ndarray:
    """Features of every node of a colour-mode state (arrays (nz, ny, nx));
    periodic = (px, py, pz).  Returns (n, 10) in node order (x fastest)."""
    px, py, pz = periodic
    phi = np.asarray(fields["phi"], np.float64)
    P = [np.asarray(fields[k], np.float64) for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz")]
    u, v, w = (np.asarray(fields[k], np.float64) for k in ("u", "v", "w"))
    gx = _central(phi, 2, px)
    gy = _central(phi, 1, py)
    gz = _central(phi, 0, pz)
    ia, ib = 3.0 / (tau_a - 0.5), 3.0 / (tau_b - 0.5)
    q = 0.5 * ((ia + ib) + phi * (ia - ib))
    tau = (6.0 + q) / (2.0 * q)
    dt = 0.0 if dtau_prev is None else np.asarray(dtau_prev, np.float64).reshape(phi.shape)
    s = tau / (tau + dt)
    f = _features(P, phi, np.sqrt(gx * gx + gy * gy + gz * gz), np.sqrt(u * u + v * v + w * w), s)
    return f.reshape(-1, NFEAT)


def fine_samples(fields: dict, pi_scale: float, periodic):
    """Training samples of every coarse node of a fine colour-mode state
    (arrays (nz, ny, nx), even sizes): features, target 3 nu_t, weight S:S.
    Returns (features (nc, 10), target (nc,), weight (nc,)) in coarse node order."""
    px, py, pz = periodic

    def blk(a):
        a = np.asarray(a, np.float64)
        nz, ny, nx = a.shape
        return a.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).mean(axis=(1, 3, 5))

    u, v, w = (np.asarray(fields[k], np.float64) for k in ("u", "v", "w"))
    U, V, W = blk(u), blk(v), blk(w)
    PHI = blk(fields["phi"])
    P = [pi_scale * blk(fields[k]) for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz")]
    UU = [blk(u * u), blk(u * v), blk(u * w), blk(v * v), blk(v * w), blk(w * w)]
    vel = (U, V, W)
    # G[a][b] = d u_b / d x_a on the coarse grid; axes of the arrays are (z, y, x)
    ax = {0: (2, px), 1: (1, py), 2: (0, pz)}
    G = [[_central(vel[b], ax[a][0], ax[a][1]) for b in range(3)] for a in range(3)]
    gphi = [_central(PHI, ax[a][0], ax[a][1]) for a in range(3)]
    f = _features(P, PHI, np.sqrt(sum(g * g for g in gphi)), np.sqrt(U * U + V * V + W * W), 1.0)
    S = [G[0][0], 0.5 * (G[0][1] + G[1][0]), 0.5 * (G[0][2] + G[2][0]), G[1][1], 0.5 * (G[1][2] + G[2][1]), G[2][2]]
    T = [UU[0] - U * U, UU[1] - U * V, UU[2] - U * W, UU[3] - V * V, UU[4] - V * W, UU[5] - W * W]
    tr = (T[0] + T[3] + T[5]) / 3.0
    T[0], T[3], T[5] = T[0] - tr, T[3] - tr, T[5] - tr
    SS = S[0] ** 2 + S[3] ** 2 + S[5] ** 2 + 2.0 * (S[1] ** 2 + S[2] ** 2 + S[4] ** 2)
    TS = T[0] * S[0] + T[3] * S[3] + T[5] * S[5] + 2.0 * (T[1] * S[1] + T[2] * S[2] + T[4] * S[4])
    cz, cy, cx = PHI.shape
    Z, Y, X = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    edge = np.zeros(PHI.shape, bool)
    if not px:
        edge |= (X == 0) | (X == cx - 1)
    if not py:
        edge |= (Y == 0) | (Y == cy - 1)
    if not pz:
        edge |= (Z == 0) | (Z == cz - 1)
    ok = (SS > 1e-30) & ~edge
    tgt = np.where(ok, -3.0 * TS / (2.0 * np.where(ok, SS, 1.0)), 0.0)
    wgt = np.where(ok, SS, 0.0)
    return f.reshape(-1, NFEAT), tgt.reshape(-1), wgt.reshape(-1)
