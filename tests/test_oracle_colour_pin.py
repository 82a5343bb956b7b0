"""The colour-gradient restatement reduces to the golden-pinned path.

The reference's colour-gradient step exists only as a draft that does not
compile, so no golden vector covers it.  Where the colour plays no part -
one colour everywhere, no body force, equal relaxation times - the colour
step's f part (equilibrium, recursive regularization, streaming, walls)
must equal the phase-field step at sigma = 0, whose f step is the
reference's fused_TSLB_1c and is pinned by the golden vectors
(tests/test_oracle_golden.py).  The GPU colour kernel is held to this
colour restatement by the parity tests, so this pins its f part too.
CPU only, FP64."""
import numpy as np
import pytest

import oracle
from entropicthreadsafe_b200 import capi, workloads


def state(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.02, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    return f


@pytest.mark.parametrize("walls", ["periodic", "bounceback_z", "moving_wall_z"])
def test_single_colour_step_equals_pinned_phase_field_step(walls):
    nx, ny, nz = 16, 12, 10
    bc = [capi.BC_PERIODIC] * 6
    bcu = [[0.0, 0.0, 0.0]] * 6
    if walls != "periodic":
        bc[capi.FACE_ZM] = capi.BC_BOUNCEBACK
        bc[capi.FACE_ZP] = capi.BC_BOUNCEBACK if walls == "bounceback_z" else capi.BC_VELOCITY
        if walls == "moving_wall_z":
            bcu = [[0.0, 0.0, 0.0]] * 5 + [[0.03, 0.0, 0.0]]
    f = state(nx, ny, nz, 7)
    pc = capi.make_params(mode=capi.MODE_COLOUR, tau_a=0.7, tau_b=0.7, sigma=0.01, beta=0.7, bc=bc, bc_u=bcu,
                          bc_phi=[1.0] * 6, wall_phi_mode=1)
    pp = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.0, bc=bc, bc_u=bcu, bc_phi=[1.0] * 6)
    fc = dict(f)
    fc["phi"] = np.ones_like(f["phi"])      # colour convention: +1 is component A
    fp = dict(f)
    fp["phi"] = np.ones_like(f["phi"])      # phase field: phi = 1 is component A
    out = {}
    for name, p, fi in (("colour", pc, fc), ("phase field", pp, fp)):
        o = oracle.Oracle(p, nx, ny, nz, fp64=True)
        o.set_moments({k: v.astype(np.float64) for k, v in fi.items()})
        o.step(40)
        out[name] = o.get_moments()
        o.close()
    c, q = out["colour"], out["phase field"]
    assert np.all(c["phi"] == 1.0)
    for k in ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        scale = max(np.abs(q[k]).max(), 1e-12)
        err = np.abs(c[k] - q[k]).max() / scale
        assert err < 1e-10, (walls, k, err)
