"""CPU check of the oracle's interior solids: a channel whose walls are
bounce-back faces equals, to FP64 round-off, the same channel in a box
periodic in z whose walls are two planes of solid nodes (isfluid = 0), for
the single-component step and for the colour-gradient step (wall phi given
as the solid nodes' frozen phi = the faces' bc_phi)."""
import numpy as np
import pytest

import oracle
from entropicthreadsafe_b200 import capi, workloads


def state(nx, ny, nz, seed, colour):
    rng = np.random.default_rng(seed)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.01, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    if colour:
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        r = np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2)
        f["phi"][:] = np.tanh((3.5 - r) / 2.0)
    else:
        f["phi"][:] = 1.0
    return {k: v.astype(np.float64) for k, v in f.items()}


@pytest.mark.parametrize("colour", [False, True])
def test_solid_planes_equal_bounceback_faces(colour):
    nx, ny, H, steps = 12, 10, 10, 40
    mode = capi.MODE_COLOUR if colour else capi.MODE_SINGLE
    common = dict(mode=mode, tau_a=0.7, tau_b=0.8, sigma=0.01 if colour else 0.0, beta=0.7,
                  force=(2e-5, 0.0, 1e-5), bc_phi=[-1.0] * 6, wall_phi_mode=0)
    pf = capi.make_params(bc=[capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK] * 2, **common)
    pm = capi.make_params(bc=[capi.BC_PERIODIC] * 6, **common)
    f = state(nx, ny, H, 1, colour)
    a = oracle.Oracle(pf, nx, ny, H, fp64=True)
    a.set_moments(f)
    a.step(steps)
    ra = a.get_moments()
    a.close()
    # the same fluid between two solid planes, z periodic
    g = {k: np.concatenate([v[:1] * 0 + (1.0 if k == "rho" else 0.0), v, v[:1] * 0 + (1.0 if k == "rho" else 0.0)])
         for k, v in f.items()}
    g["phi"][0] = g["phi"][-1] = -1.0 if colour else 1.0   # the faces' bc_phi (wall_phi_mode 0)
    iso = np.ones((H + 2, ny, nx), np.uint8)
    iso[0] = iso[-1] = 0
    b = oracle.Oracle(pm, nx, ny, H + 2, fp64=True)
    b.set_isfluid(iso)
    b.set_moments(g)
    b.step(steps)
    rb = b.get_moments()
    b.close()
    for k in capi.FIELDS:
        if k == "phi" and not colour:
            continue
        ref = ra[k]
        err = np.abs(rb[k][1:-1] - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err < 1e-12, (k, err)
        # solid nodes keep their moments
        assert np.array_equal(rb[k][0], g[k][0]) and np.array_equal(rb[k][-1], g[k][-1])
