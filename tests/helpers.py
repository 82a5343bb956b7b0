"""Shared helpers of the parity tests (oracle vs CUDA path)."""
from __future__ import annotations

import json
import os

import numpy as np

from entropicthreadsafe_b200 import capi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# golden cases given as the reference's populations after its initial conditions
GOLDEN_CASES = ("pf_periodic", "pf_walls_force", "couette", "pf_jet")
# the 32^3, 100-step phase-field droplet, given as its initial moments
GOLDEN_MOMENT_CASE = "pf_droplet32"


def golden_params(meta):
    bc = [capi.BC_PERIODIC] * 6
    bcu = [[0.0, 0.0, 0.0]] * 6
    if meta["walls"] == "bounceback":
        bc[4] = bc[5] = capi.BC_BOUNCEBACK
    elif meta["walls"] == "couette":
        bc[4] = bc[5] = capi.BC_VELOCITY
        bcu = [[0, 0, 0]] * 4 + [[-meta["uwall"], 0, 0], [meta["uwall"], 0, 0]]
    elif meta["walls"] == "jet":
        # bcs_2c_turbulent_jet: inlet plane at z-, zero-gradient outlet at z+ whose
        # g6 carries phi at the fixed speed 0.05 (boundary_cds_3D_module.f90:1044-1045)
        bc[4], bc[5] = capi.BC_INLET, capi.BC_OUTLET
        bcu = [[0, 0, 0]] * 5 + [[0, 0, 0.05]]
    return capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=meta["tau"], sigma=meta["sigma"],
                            sharp_c=meta["sharp_c"], force=meta["force"], bc=bc, bc_u=bcu,
                            bc_phi=[0.0] * 6, wall_phi_mode=0)


def golden_inlet(d):
    """{face: planes} of a golden case with an inlet plane (the jet), else None."""
    return {capi.FACE_ZM: np.asarray(d["inlet"], np.float32)} if "inlet" in d.files else None


def golden_initial_moments(d):
    """The 11 initial moment fields of a moments-only golden case (the first
    moments pass of the reference's initial populations, rounded to FP32)."""
    return {k: np.asarray(d["ic_" + k], np.float32) for k in capi.FIELDS}


def load_golden(case):
    d = np.load(os.path.join(GOLDEN, case + ".npz"))
    return d, json.loads(str(d["meta"]))


def rel_err(a, b):
    """max |a - b| / max |b| (the field-wise metric of the parity tests)."""
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def with_halo(pops: np.ndarray) -> np.ndarray:
    """(Q, nz, ny, nx) interior populations -> the reference's halo layout."""
    q, nz, ny, nx = pops.shape
    out = np.zeros((q, nz + 2, ny + 2, nx + 2), pops.dtype)
    out[:, 1:-1, 1:-1, 1:-1] = pops
    return out


def run_oracle(params, fields, nsteps, fp64=True, inlet=None):
    import oracle
    nz, ny, nx = fields["rho"].shape
    o = oracle.Oracle(params, nx, ny, nz, fp64=fp64)
    if inlet:
        for face, planes in inlet.items():
            o.set_inlet(face, planes)
    o.set_moments({k: np.asarray(v, np.float64) for k, v in fields.items()})
    o.step(nsteps)
    out = o.get_moments()
    red = o.reduce()
    o.close()
    return out, red


def run_gpu(params, fields, nsteps, inlet=None):
    from entropicthreadsafe_b200.solver import Lattice
    nz, ny, nx = fields["rho"].shape
    with Lattice(params, nx, ny, nz) as lat:
        if inlet:
            for face, planes in inlet.items():
                lat.set_inlet(face, planes)
        lat.upload_moments(fields)
        lat.step(nsteps)
        out = lat.download()
        red = lat.reduce()
    return out, red


def field_errors(a, b):
    errs = {k: rel_err(a[k], b[k]) for k in capi.FIELDS}
    errs["rho-1"] = rel_err(np.asarray(a["rho"], np.float64) - 1.0, np.asarray(b["rho"], np.float64) - 1.0)
    return errs
