"""The CPU oracle against golden vectors of the reference's own statements.

tests/golden/*.npz hold populations and moments produced by evaluating the
reference's Fortran statements with numpy (tests/golden/make_golden.py):
the phase-field step recursive_2c_TSLB3D.f90:351-832, the forced collision
TSLB_2C-mpi/lb_kernels_module.f90:747-931, bounce-back
boundary_cds_3D_module.f90:18-70, the moving-wall condition
boundary_cds_3D_module.f90:413-571 and the jet's inlet and outlet
boundary_cds_3D_module.f90:885-1050 (with a fixed inlet plane); and the
single-component program's moments_TSLB, fused_TSLB_1c and
fused_TSLB_force_1c (TSLB_2C-mpi/lb_kernels_module.f90:21-206, 423-566,
583-730), stepped from a moment state.
"""
import json

import numpy as np
import pytest

import oracle
from entropicthreadsafe_b200 import capi

from helpers import (GOLDEN_CASES as CASES, GOLDEN_MOMENT_CASE, golden_initial_moments, golden_inlet, golden_params,
                     load_golden as load, rel_err)


def make_oracle(d, meta, nx, ny, nz, fp64):
    o = oracle.Oracle(golden_params(meta), nx, ny, nz, fp64=fp64)
    for face, planes in (golden_inlet(d) or {}).items():
        o.set_inlet(face, planes)
    return o


@pytest.mark.parametrize("case", CASES)
def test_oracle_fp64_matches_reference_statements(case):
    d, meta = load(case)
    nz, ny, nx = d["rho_fp64"].shape
    o = make_oracle(d, meta, nx, ny, nz, True)
    o.set_pops(d["f_fp64"], d["g_fp64"])
    o.step(meta["nsteps"])
    out = o.get_moments()
    for m in capi.FIELDS:
        # double-precision round-off only: the two forms of the polynomials differ
        assert rel_err(out[m], d[m + "_fp64"]) < 1e-12, m


@pytest.mark.parametrize("case", CASES)
def test_oracle_fp32_matches_reference_statements(case):
    d, meta = load(case)
    nz, ny, nx = d["rho_fp32"].shape
    o = make_oracle(d, meta, nx, ny, nz, False)
    o.set_pops(d["f_fp32"], d["g_fp32"])
    o.step(meta["nsteps"])
    out = o.get_moments()
    # FP32 round-off of two algebraically equal forms, relative to each field's max
    tol = {"rho": 2e-6, "u": 2e-5, "v": 2e-5, "w": 5e-5, "phi": 2e-6}
    for m in capi.FIELDS:
        assert rel_err(out[m], d[m + "_fp32"]) < tol.get(m, 2e-4), m


def test_reference_fp32_noise_is_what_the_gpu_tolerance_assumes():
    # the reference's own FP32 statements against its FP64 statements: the
    # noise floor that any FP32 implementation of this step shares
    d, _ = load("pf_periodic")
    for m in capi.FIELDS:
        assert rel_err(d[m + "_fp32"], d[m + "_fp64"]) < 2e-4, m


@pytest.mark.slow
def test_oracle_fp64_matches_reference_statements_32cube_100_steps():
    """The 32^3 droplet over 100 steps: the oracle from the initial moments
    against the reference statements from their initial populations (FP64,
    the golden rounded to FP32 when stored)."""
    d, meta = load(GOLDEN_MOMENT_CASE)
    nz, ny, nx = d["rho_fp64"].shape
    o = make_oracle(d, meta, nx, ny, nz, True)
    o.set_moments({k: v.astype(np.float64) for k, v in golden_initial_moments(d).items()})
    o.step(meta["nsteps"])
    out = o.get_moments()
    for m in capi.FIELDS:
        a, b = out[m], d[m + "_fp64"].astype(np.float64)
        if m == "rho":
            a, b = a - 1.0, b - 1.0
        assert rel_err(a, b) < 1e-6, m
    spread = json.loads(str(d["fp32_spread"]))
    assert set(spread) == set(capi.FIELDS)


# the single-component program's own statements (moments_TSLB, fused_TSLB_1c,
# fused_TSLB_force_1c of TSLB_2C-mpi/lb_kernels_module.f90)
SC_CASES = ("sc_periodic", "sc_force")
SC_FIELDS = tuple(f for f in capi.FIELDS if f != "phi")


@pytest.mark.parametrize("fp64", [True, False], ids=["fp64", "fp32"])
@pytest.mark.parametrize("case", SC_CASES)
def test_single_component_oracle_matches_reference_statements(case, fp64):
    """TSLB_MODE_SINGLE of the oracle (the phase-field step at sigma = 0 with
    a uniform phi, as the GPU single-component kernel is checked against)
    from the fixture's initial moments, against the reference's
    single-component statements over the same steps: unforced (sc_periodic)
    and with the forced collision's velocity shift (sc_force)."""
    d, meta = load(case)
    ic = {k: d["ic_" + k].astype(np.float64) for k in SC_FIELDS}
    nz, ny, nx = ic["rho"].shape
    ic["phi"] = np.ones((nz, ny, nx))
    p = capi.make_params(mode=capi.MODE_SINGLE, tau_a=meta["tau"], sigma=0.0, force=meta["force"])
    o = oracle.Oracle(p, nx, ny, nz, fp64=fp64)
    o.set_moments(ic)
    o.step(meta["nsteps"])
    out = o.get_moments()
    o.close()
    tag = "fp64" if fp64 else "fp32"
    for m in SC_FIELDS:
        a, b = out[m], d[m + "_" + tag].astype(np.float64)
        if m == "rho":
            a, b = a - 1.0, b - 1.0
        if fp64:
            # double-precision round-off of two algebraically equal forms (the
            # non-equilibrium moments are sums of O(1) populations of size 1e-4)
            assert rel_err(a, b) < 1e-11, (m, rel_err(a, b))
        else:
            # FP32 round-off relative to each field's max (rho - 1 and Pi^neq of
            # size 1e-3 and 1e-4): the reference's own FP32 statements differ
            # from their FP64 run by up to 4e-4
            assert rel_err(a, b) < 1e-3, (m, rel_err(a, b))


@pytest.mark.parametrize("fp64", [True, False], ids=["fp64", "fp32"])
def test_interior_obstacle_matches_reference_statements(fp64):
    """A droplet against an obstacle of solid nodes (isfluid = 0) inside a
    fully periodic box: the oracle's interior solids (moments kept, no
    collision, normals 0, half-way bounce-back after the periodic exchange)
    against the reference's bounce-back block boundary_cds_3D_module.f90:18-70
    applied at every solid node."""
    d, meta = load("pf_obstacle")
    tag = "fp64" if fp64 else "fp32"
    nz, ny, nx = d["rho_" + tag].shape
    i0, i1, j0, j1, k0, k1 = meta["obstacle"]
    isfluid = np.ones((nz, ny, nx), np.uint8)
    isfluid[k0 - 1:k1, j0 - 1:j1, i0 - 1:i1] = 0
    o = make_oracle(d, meta, nx, ny, nz, fp64)
    o.set_isfluid(isfluid)
    o.set_pops(d["f_" + tag], d["g_" + tag])
    o.step(meta["nsteps"])
    out = o.get_moments()
    o.close()
    tol = 1e-12 if fp64 else None
    for m in capi.FIELDS:
        err = rel_err(out[m], d[m + "_" + tag])
        if fp64:
            assert err < tol, (m, err)
        else:
            assert err < {"rho": 2e-6, "u": 2e-5, "v": 2e-5, "w": 5e-5, "phi": 2e-6}.get(m, 2e-4), (m, err)
