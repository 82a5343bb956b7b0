"""Moment-space boundary planes (tslb_set_moment_bc, the reference's
bcs_TSLB_only_z_turbojet): 25 single-component steps with the jet plane at
z = 0 and the copy plane at z = nz - 1 against the oracle stepping with the
same plane rewrites (oracle/newbcs.py) before each step."""
import numpy as np
import pytest

import oracle
from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice
from helpers import rel_err
from oracle import newbcs

pytestmark = pytest.mark.gpu


def test_moment_planes_match_oracle():
    nx, ny, nz, steps = 20, 18, 24, 25
    rng = np.random.default_rng(8)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v"):
        f[k][:] = rng.normal(0, 0.005, f[k].shape)
    f["w"][:] = 0.02 + rng.normal(0, 0.005, f["w"].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    f["phi"][:] = 1.0
    p = capi.make_params(mode=capi.MODE_SINGLE, tau_a=0.6, sigma=0.0,
                         bc=[capi.BC_PERIODIC] * 4 + [capi.BC_PRESSURE] * 2)
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        lat.set_moment_bc(4, capi.MBC_JET, 0.05, 4.0, 0.004)
        lat.set_moment_bc(5, capi.MBC_COPY)
        lat.step(steps)
        gpu = lat.download()
    o = oracle.Oracle(p, nx, ny, nz, fp64=True)
    m = {k: np.asarray(v, np.float64) for k, v in f.items()}
    for s in range(steps):
        newbcs.moment_bc(m, 4, "jet", s + 1, 0.05, 4.0, 0.004)
        newbcs.moment_bc(m, 5, "copy", s + 1)
        o.set_moments(m)
        o.step(1)
        m = o.get_moments()
    o.close()
    for k in ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        assert rel_err(gpu[k], m[k]) < 5e-5, (k, rel_err(gpu[k], m[k]))
    # the inlet disc carries the jet velocity after the refreshes at steps 10 and 20
    assert gpu["w"][1, ny // 2, nx // 2] > 0.03
