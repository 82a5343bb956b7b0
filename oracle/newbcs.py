"""TEST INFRASTRUCTURE ONLY: restatements of the reference's moment-space
boundary planes for the parity tests.

- rand_noseeded: the statements of TSLB_2C-mpi/vars_single_3D_module.f90:150-215
  one by one (integer mods, real(4) accumulators as numpy float32);
- moment_bc: bcs_TSLB_only_z_turbojet (TSLB_newBCS/boundary_cds_3D_module.f90:1233-1292)
  on a dict of moment arrays (nz, ny, nx), face 4 (k = 1) as the jet side and
  face 5 (k = nz) as the copy side, with the step numbering of the library
  (include/tslb.h, tslb_set_moment_bc).
"""
from __future__ import annotations

import numpy as np

F32 = np.float32


def rand_noseeded(i: int, j: int, k: int, l: int) -> np.float32:
    isub = i % 178 + 1
    jsub = j % 178 + 1
    ksub = k % 178 + 1
    lsub = l % 169
    s, t = F32(0.0), F32(0.5)
    for _ in range(24):
        msub = ((isub * jsub) % 179 * ksub) % 179
        isub, jsub, ksub = jsub, ksub, msub
        lsub = (53 * lsub + 1) % 169
        if (lsub * msub) % 64 >= 32:
            s = F32(s + t)
        t = F32(F32(0.5) * t)
    u97 = s
    s, t = F32(0.0), F32(0.5)
    for _ in range(24):
        msub = ((isub * jsub) % 179 * ksub) % 179
        isub, jsub, ksub = jsub, ksub, msub
        lsub = (53 * lsub + 1) % 169
        if (lsub * msub) % 64 >= 32:
            s = F32(s + t)
        t = F32(F32(0.5) * t)
    u33 = s
    uni = F32(u97 - u33)
    if uni < 0:
        uni = F32(uni + F32(1.0))
    c, cd, cm = F32(362436.0 / 16777216.0), F32(7654321.0 / 16777216.0), F32(16777213.0 / 16777216.0)
    csub = F32(c - cd)
    if csub < 0:
        csub = F32(csub + cm)
    uni = F32(uni - csub)
    if uni < 0:
        uni = F32(uni + F32(1.0))
    return uni


def moment_bc(fields: dict, face: int, kind: str, step: int, uwall=0.0, radius=10.0, amp=0.004) -> None:
    nz, ny, nx = fields["rho"].shape
    k0, k1 = (0, 1) if face == 4 else (nz - 1, nz - 2)
    if kind == "copy":
        for f in fields.values():
            f[k0] = f[k1]
        return
    for name in ("rho", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        fields[name][k0] = fields[name][k1]
    fields["u"][k0] = 0.0
    fields["v"][k0] = 0.0
    if step % 10 == 0:
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                dx, dy = F32(i) - F32(nx / 2.0), F32(j) - F32(ny / 2.0)
                if dx * dx + dy * dy <= F32(radius) * F32(radius):
                    r = max(float(rand_noseeded(i, j, 1, step)), 2.98023224e-8)
                    fields["w"][k0, j - 1, i - 1] = uwall + amp * np.sqrt(-2.0 * np.log(r)) * np.cos(2 * np.pi * r)
