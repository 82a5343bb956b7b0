"""Interior solid nodes (tslb_set_solid_mask, the reference's isfluid): the
CUDA step against the oracle with the same mask in the three modes, an
all-fluid mask changing nothing, solid planes equal to bounce-back faces,
and mass conservation around an obstacle."""
import numpy as np
import pytest

import oracle
from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice
from helpers import rel_err

pytestmark = pytest.mark.gpu

TARGET, TOL_FACTOR = 1e-5, 4.0


def obstacle(nx, ny, nz):
    """A cube and a thin plate of solid nodes."""
    iso = np.ones((nz, ny, nx), np.uint8)
    iso[nz // 2 - 2:nz // 2 + 2, ny // 2 - 3:ny // 2 + 1, 3:7] = 0
    iso[2:nz - 2, 1, nx - 5] = 0
    return iso


def case(mode, nx=20, ny=18, nz=16, seed=4):
    rng = np.random.default_rng(seed)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.01, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - 13.5) ** 2 + (y - 8) ** 2 + (z - 8) ** 2)
    if mode == capi.MODE_COLOUR:
        f["phi"][:] = np.tanh((4.0 - r) / 2.0)
        p = capi.make_params(mode=mode, tau_a=0.7, tau_b=0.8, sigma=0.01, beta=0.7, force=(1e-5, 0, 0))
    elif mode == capi.MODE_PHASEFIELD:
        f["phi"][:] = 0.5 * (1 + np.tanh((4.0 - r) / 1.5))
        p = capi.make_params(mode=mode, tau_a=0.7, sigma=0.01, sharp_c=0.9, force=(1e-5, 0, 0))
    else:
        f["phi"][:] = 1.0
        p = capi.make_params(mode=mode, tau_a=0.7, sigma=0.0, force=(1e-5, 0, 0))
    iso = obstacle(nx, ny, nz)
    f["phi"][iso == 0] = -1.0 if mode == capi.MODE_COLOUR else (0.0 if mode == capi.MODE_PHASEFIELD else 1.0)
    return p, f, iso


def run_oracle(p, f, iso, steps, fp64):
    nz, ny, nx = f["rho"].shape
    o = oracle.Oracle(p, nx, ny, nz, fp64=fp64)
    o.set_isfluid(iso)
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    o.step(steps)
    out = o.get_moments()
    o.close()
    return out


@pytest.mark.parametrize("mode", [capi.MODE_COLOUR, capi.MODE_PHASEFIELD, capi.MODE_SINGLE])
def test_solids_match_oracle(mode):
    p, f, iso = case(mode)
    nz, ny, nx = f["rho"].shape
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        lat.set_solid_mask(iso)
        lat.step(60)
        gpu = lat.download()
    o64 = run_oracle(p, f, iso, 60, True)
    o32 = run_oracle(p, f, iso, 60, False)
    if mode == capi.MODE_SINGLE:
        for d in (gpu, o64, o32):
            d.pop("phi")
    eg = {k: rel_err(gpu[k], o64[k]) for k in gpu}
    e32 = {k: rel_err(o32[k], o64[k]) for k in gpu}
    bad = {k: (eg[k], e32[k]) for k in gpu if eg[k] > max(TARGET, TOL_FACTOR * e32[k])}
    assert not bad, bad
    for k in gpu:   # solid nodes keep their moments
        assert np.array_equal(gpu[k][iso == 0], f[k][iso == 0].astype(np.float32)), k


def test_all_fluid_mask_changes_nothing():
    p, f, _ = case(capi.MODE_COLOUR)
    nz, ny, nx = f["rho"].shape
    outs = []
    for mask in (None, np.ones((nz, ny, nx), np.uint8)):
        with Lattice(p, nx, ny, nz) as lat:
            lat.upload_moments(f)
            if mask is not None:
                lat.set_solid_mask(mask)
            lat.step(30)
            outs.append(lat.download())
    for k in capi.FIELDS:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_solid_planes_equal_bounceback_faces():
    nx, ny, H = 16, 12, 14
    rng = np.random.default_rng(2)
    f = workloads.empty_fields(nx, ny, H)
    f["u"][:] = rng.normal(0, 0.01, f["u"].shape)
    common = dict(mode=capi.MODE_SINGLE, tau_a=0.7, sigma=0.0, force=(2e-5, 0, 0))
    with Lattice(capi.make_params(bc=[capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK] * 2, **common), nx, ny, H) as a:
        a.upload_moments(f)
        a.step(50)
        ra = a.download()
    g = {k: np.concatenate([np.full((1, ny, nx), 1.0 if k in ("rho", "phi") else 0.0, np.float32), v,
                            np.full((1, ny, nx), 1.0 if k in ("rho", "phi") else 0.0, np.float32)]) for k, v in f.items()}
    iso = np.ones((H + 2, ny, nx), np.uint8)
    iso[0] = iso[-1] = 0
    with Lattice(capi.make_params(bc=[capi.BC_PERIODIC] * 6, **common), nx, ny, H + 2) as b:
        b.upload_moments(g)
        b.set_solid_mask(iso)
        b.step(50)
        rb = b.download()
    for k in ("rho", "u", "v", "w", "pxx", "pxz", "pzz"):
        err = np.abs(rb[k][1:-1].astype(np.float64) - ra[k]).max() / max(np.abs(ra[k]).max(), 1e-30)
        assert err < 1e-5, (k, err)


def test_mass_is_conserved_around_an_obstacle():
    p, f, iso = case(capi.MODE_SINGLE, nx=32, ny=24, nz=24)
    with Lattice(p, 32, 24, 24) as lat:
        lat.upload_moments(f)
        lat.set_solid_mask(iso)
        m0 = lat.reduce()["mass"]
        lat.step(500)
        r = lat.reduce()
        out = lat.download()
    assert abs(r["mass"] - m0) / m0 < 1e-6
    # the force drives a flow that the obstacle slows: fluid next to the cube moves slower than the bulk
    assert out["u"][iso == 1].mean() > 0
