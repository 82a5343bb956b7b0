"""Initial states and parameters of the benchmark workloads.

Each builder returns (params, fields) where fields holds the 11 moment
arrays of shape (nz, ny, nx).  All noise is seeded and counter-based, so a
workload is the same on every machine and for every rank.

  droplet  64^3 fully periodic static droplet, colour gradient
  channel  384x192x128 two-component channel: x, y periodic, bounce-back
           walls at z, body force gx, 40 droplets of radius 8
  jet      two-component round jet: 192x192x384 (coarse) or 384x384x768
           (fine, factor 2 in space and time), disc inlet at z = 0,
           zero-gradient outlet, x, y periodic
"""
from __future__ import annotations

import numpy as np

from . import capi


def counter_uniform(seed: int, *keys: np.ndarray) -> np.ndarray:
    """Uniform [0,1) from a splitmix64 hash of (seed, keys...), elementwise."""
    with np.errstate(over="ignore"):
        h = np.full(np.broadcast(*keys).shape, np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15), np.uint64)
        for k in keys:
            h = h ^ (np.asarray(k).astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15) + (h << np.uint64(6)) + (h >> np.uint64(2)))
            z = h + np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            h = z ^ (z >> np.uint64(31))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def empty_fields(nx: int, ny: int, nz: int) -> dict:
    f = {k: np.zeros((nz, ny, nx), np.float32) for k in capi.FIELDS}
    f["rho"][:] = 1.0
    return f


def droplet(n: int = 64, radius: float = 16.0, tau: float = 0.8, sigma: float = 0.01,
            beta: float = 0.7, width: float = 2.0, mode: int = capi.MODE_COLOUR, sharp_c: float = 0.9):
    """Static droplet at the box centre, fully periodic.

    Colour mode: phi = tanh((R - r)/2) in [-1, 1].  Phase-field mode: the
    reference's [0, 1] convention, phi = (1 + tanh((R - r)/2))/2, with the
    reference's sharpening coefficient 0.3 * 3 (recursive_2c_TSLB3D.f90:28)."""
    if mode == capi.MODE_PHASEFIELD:
        p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=tau, tau_b=tau, sigma=sigma, sharp_c=sharp_c)
    else:
        p = capi.make_params(mode=capi.MODE_COLOUR, tau_a=tau, tau_b=tau, sigma=sigma, beta=beta,
                             grad_threshold=1e-3)
    f = empty_fields(n, n, n)
    c = (n - 1) / 2.0  # (n+1)/2 in 1-based indices
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
    t = np.tanh((radius - r) / width)
    f["phi"][:] = 0.5 * (1.0 + t) if mode == capi.MODE_PHASEFIELD else t
    return p, f


CHANNEL = dict(nx=384, ny=192, nz=128, gx=2.5e-6, nu=0.0015, u_centre=0.05, noise=0.05,
               ndrops=40, radius=8.0, wall_gap=12.0, sigma=0.005, beta=0.7, seed=1234)


def droplet_centres(nx, ny, nz, ndrops, radius, wall_gap, seed, min_sep=None):
    """Seeded rejection sampling of non-overlapping centres (periodic in x, y)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    min_sep = 2 * radius + 4 if min_sep is None else min_sep
    zlo, zhi = wall_gap + radius, nz - 1 - wall_gap - radius
    centres = []
    tries = 0
    while len(centres) < ndrops:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place droplets")
        c = np.array([rng.uniform(0, nx), rng.uniform(0, ny), rng.uniform(zlo, zhi)])
        ok = True
        for q in centres:
            dx = abs(c[0] - q[0]); dx = min(dx, nx - dx)
            dy = abs(c[1] - q[1]); dy = min(dy, ny - dy)
            if dx * dx + dy * dy + (c[2] - q[2]) ** 2 < min_sep ** 2:
                ok = False
                break
        if ok:
            centres.append(c)
    return np.array(centres)


def channel(nx: int | None = None, ny: int | None = None, nz: int | None = None, **over):
    """Two-component channel: x, y periodic, half-way bounce-back walls at z.

    The laminar profile of this force and viscosity would peak at
    gx H^2 / (8 nu) = 3.4 lattice units, far outside the stable range, so
    the initial mean flow is the parabolic shape scaled to u_centre = 0.05
    (Mach 0.087), plus counter-based uniform noise of +-5% of u_centre in
    all three components (key = (x, y, z, component), seed 1234)."""
    cfg = dict(CHANNEL)
    cfg.update(over)
    nx = nx or cfg["nx"]; ny = ny or cfg["ny"]; nz = nz or cfg["nz"]
    tau = 3 * cfg["nu"] + 0.5
    p = capi.make_params(mode=capi.MODE_COLOUR, tau_a=tau, tau_b=tau, sigma=cfg["sigma"], beta=cfg["beta"],
                         grad_threshold=1e-3, force=(cfg["gx"], 0.0, 0.0),
                         bc=[capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK] * 2,
                         bc_phi=[-1.0] * 6, wall_phi_mode=1)
    f = empty_fields(nx, ny, nz)
    z = (np.arange(nz) + 0.5).reshape(nz, 1, 1)
    prof = 4.0 * z * (nz - z) / nz ** 2
    zi, yi, xi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    uc, amp = cfg["u_centre"], cfg["noise"] * cfg["u_centre"]
    for comp, name in enumerate(("u", "v", "w")):
        noise = amp * (2.0 * counter_uniform(cfg["seed"], xi, yi, zi, comp) - 1.0)
        base = uc * prof if name == "u" else 0.0
        f[name][:] = (base + noise).astype(np.float32)
    cen = droplet_centres(nx, ny, nz, cfg["ndrops"], cfg["radius"], cfg["wall_gap"], cfg["seed"])
    phi = np.full((nz, ny, nx), -1.0)
    R = cfg["radius"]
    for cx, cy, cz in cen:
        # only the droplet's bounding box, with periodic images in x and y
        for sx in (-nx, 0, nx):
            for sy in (-ny, 0, ny):
                x0, x1 = int(np.floor(cx + sx - R - 4)), int(np.ceil(cx + sx + R + 4))
                y0, y1 = int(np.floor(cy + sy - R - 4)), int(np.ceil(cy + sy + R + 4))
                z0, z1 = int(np.floor(cz - R - 4)), int(np.ceil(cz + R + 4))
                xs = np.arange(max(x0, 0), min(x1, nx - 1) + 1)
                ys = np.arange(max(y0, 0), min(y1, ny - 1) + 1)
                zs = np.arange(max(z0, 0), min(z1, nz - 1) + 1)
                if xs.size == 0 or ys.size == 0 or zs.size == 0:
                    continue
                Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
                r = np.sqrt((X - cx - sx) ** 2 + (Y - cy - sy) ** 2 + (Z - cz) ** 2)
                blob = np.tanh((R - r) / 2.0)
                sub = phi[np.ix_(zs, ys, xs)]
                phi[np.ix_(zs, ys, xs)] = np.maximum(sub, blob)
    f["phi"][:] = phi.astype(np.float32)
    return p, f


# ---- round jet (the learned-closure workload) ----
JET = dict(nx=192, ny=192, nz=384, diameter=16.0, w_in=0.08, noise=0.03, nu=8e-4, sigma=0.002, beta=0.7,
           refresh=10)


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def inlet_disc(n0: int, n1: int, axis: int, sign: float, c0: float, c1: float, radius: float, speed: float,
               amp: float, seed: int, counter: int) -> np.ndarray:
    """Host mirror of tslb_set_inlet_disc: the (4, n1, n0) plane (u, v, w, phi)."""
    i = np.arange(n0 * n1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        k = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(counter)
    h = _mix64(_mix64(np.array([k], np.uint64))[0] ^ i)
    xi = (h >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 8388608.0) - np.float32(1.0)
    d0 = (np.arange(n0 * n1) % n0).astype(np.float32) - np.float32(c0)
    d1 = (np.arange(n0 * n1) // n0).astype(np.float32) - np.float32(c1)
    inside = d0 * d0 + d1 * d1 <= np.float32(radius) * np.float32(radius)
    wn = (np.float32(sign) * np.float32(speed)) * (np.float32(1.0) + np.float32(amp) * xi)
    out = np.zeros((4, n0 * n1), np.float32)
    out[axis] = np.where(inside, wn, np.float32(0.0))
    out[3] = np.where(inside, np.float32(1.0), np.float32(-1.0))
    return out.reshape(4, n1, n0)


def jet(scale: int = 1, **over):
    """Round jet of component A (phi = +1) into quiescent B (phi = -1).

    scale 1: 192 x 192 x 384, disc diameter 16, nu 8e-4, sigma 0.002.
    scale 2: 384 x 384 x 768 at the same Reynolds and Weber numbers under
    acoustic scaling (dx and dt halved, lattice velocities unchanged):
    diameter 32, nu and sigma doubled, and the inlet noise refreshed every
    2 x 10 steps.  x, y periodic; inlet face z- (TSLB_BC_INLET, drawn by
    jet_inlet); outlet z+ with zero-gradient velocity and phi at density 1
    (TSLB_BC_PRESSURE: the reference's zero-gradient outlet, which also
    copies the density, grows without bound at this viscosity).  Returns
    (params, fields, spec)."""
    cfg = dict(JET)
    cfg.update(over)
    nx, ny, nz = scale * cfg["nx"], scale * cfg["ny"], scale * cfg["nz"]
    nu = cfg["nu"] * scale
    tau = 3.0 * nu + 0.5
    p = capi.make_params(mode=capi.MODE_COLOUR, tau_a=tau, tau_b=tau, sigma=cfg["sigma"] * scale, beta=cfg["beta"],
                         grad_threshold=1e-3, bc=[capi.BC_PERIODIC] * 4 + [capi.BC_INLET, capi.BC_PRESSURE],
                         bc_phi=[-1.0] * 6, wall_phi_mode=1)
    f = empty_fields(nx, ny, nz)
    f["phi"][:] = -1.0
    spec = dict(nx=nx, ny=ny, nz=nz, scale=scale, diameter=cfg["diameter"] * scale, w_in=cfg["w_in"],
                noise=cfg["noise"], refresh=cfg["refresh"] * scale, cx=nx / 2 - 0.5, cy=ny / 2 - 0.5, tau=tau)
    return p, f, spec


def jet_sponge(spec: dict, frac: float = 0.15, amp: float = 0.3) -> np.ndarray:
    """Sponge layer in front of the outlet: a static tau correction rising as
    amp * scale * s^2 over the last `frac` of the length (s from 0 to 1), so
    eddies are damped before the outlet.  (nz, ny, nx) float32."""
    nz, ny, nx = spec["nz"], spec["ny"], spec["nx"]
    z0 = (1.0 - frac) * nz
    z = np.arange(nz) + 0.5
    prof = np.where(z > z0, ((z - z0) / (nz - z0)) ** 2, 0.0) * amp * spec["scale"]
    return np.broadcast_to(prof.astype(np.float32)[:, None, None], (nz, ny, nx))


def jet_inlet(lat, spec: dict, seed: int, step: int) -> None:
    """Draw the jet inlet of `step` on the device (refreshed every spec['refresh'] steps)."""
    lat.set_inlet_disc(4, spec["cx"], spec["cy"], spec["diameter"] / 2, spec["w_in"], spec["noise"], seed,
                       step // spec["refresh"])
