"""The paired-column step kernel against the scalar step kernel.

Lattices whose rows are whole 16-byte chunks (and that have no interior
solid mask) are stepped by the paired-column kernel (tslb_pair.cuh: two x
columns per thread, paired FP32 instructions, 64 x 8 tiles); the others by
the scalar kernel (tslb_step.cuh).  TSLB_STEP_KERNEL=scalar at creation
forces the scalar kernel, so the two can be compared on the same input.
Both are FP32 evaluations of the same step in different operation orders:
they agree to FP32 round-off, and both are held to the oracle elsewhere.
The shapes cover partial tiles in x and y, periodic and wall faces, and
every mode and storage form.
"""
import os

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice
from helpers import rel_err

pytestmark = pytest.mark.gpu


def run(p, f, nsteps, scalar):
    nz, ny, nx = f["rho"].shape
    old = os.environ.get("TSLB_STEP_KERNEL")
    if scalar:
        os.environ["TSLB_STEP_KERNEL"] = "scalar"
    else:
        os.environ.pop("TSLB_STEP_KERNEL", None)
    try:
        with Lattice(p, nx, ny, nz) as lat:
            lat.upload_moments(f)
            lat.step(nsteps)
            return lat.download()
    finally:
        if old is None:
            os.environ.pop("TSLB_STEP_KERNEL", None)
        else:
            os.environ["TSLB_STEP_KERNEL"] = old


def compare(p, f, nsteps, tol):
    a = run(p, f, nsteps, scalar=False)
    b = run(p, f, nsteps, scalar=True)
    errs = {k: rel_err(a[k], b[k]) for k in capi.FIELDS}
    errs["rho-1"] = rel_err(np.asarray(a["rho"], np.float64) - 1, np.asarray(b["rho"], np.float64) - 1)
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, bad
    return errs


@pytest.mark.parametrize("shape", [(64, 16, 12), (40, 12, 10), (136, 20, 9)])
def test_colour_channel_walls_force(shape):
    nx, ny, nz = shape
    p, f = workloads.channel(nx=nx, ny=ny, nz=nz, ndrops=2, radius=3.0, wall_gap=1.0, gx=2.5e-5)
    compare(p, f, 30, 2e-5)


def test_colour_droplet_periodic():
    p, f = workloads.droplet(n=32, radius=8.0)
    compare(p, f, 40, 2e-5)


def test_colour_moving_walls_and_x_walls():
    p, f = workloads.droplet(n=32, radius=7.0)
    p.tau_b = 1.1
    for face in (capi.FACE_XM, capi.FACE_XP):
        p.bc[face] = capi.BC_BOUNCEBACK
    for face, u in ((capi.FACE_ZM, -0.05), (capi.FACE_ZP, 0.05)):
        p.bc[face] = capi.BC_VELOCITY
        p.bc_u[face][0] = u
        p.bc_phi[face] = -1.0
    p.wall_phi_mode = 1
    compare(p, f, 30, 2e-5)


def test_phasefield_droplet_walls():
    p, f = workloads.droplet(n=32, radius=8.0, mode=capi.MODE_PHASEFIELD)
    p.bc[capi.FACE_ZM] = p.bc[capi.FACE_ZP] = capi.BC_BOUNCEBACK
    p.force[0] = 1e-5
    compare(p, f, 30, 2e-5)


def test_single_component_channel():
    p, f = workloads.channel(nx=64, ny=24, nz=16, ndrops=0, gx=2.5e-5)
    p.mode = capi.MODE_SINGLE
    f["phi"][:] = 1.0
    compare(p, f, 30, 2e-5)


@pytest.mark.parametrize("prec", [capi.PREC_BF16, capi.PREC_FP16S])
def test_sixteen_bit_storage_forms(prec):
    """16-bit forms: one step from the same stored state (the stochastic
    rounding draws differ between the kernels, so only one store is compared,
    to the storage's own resolution)."""
    p, f = workloads.channel(nx=64, ny=16, nz=12, ndrops=2, radius=3.0, wall_gap=1.0, gx=2.5e-5)
    p.precision = prec
    a = run(p, f, 1, scalar=False)
    b = run(p, f, 1, scalar=True)
    tol = 2.0 ** -6 if prec == capi.PREC_BF16 else 2.0 ** -9   # two units of the stored precision
    for k in ("u", "v", "w", "phi"):
        assert rel_err(a[k], b[k]) <= tol, k
