"""Batched ensembles of independent lattices (config 4) over the C-ABI.

`Ensemble` wraps tslb_ensemble_*: members of different sizes advanced by
one kernel launch per step (optionally K steps from a CUDA graph), with a
timing autotuner for the z chunk and the resident grid of the persistent
kernel.  `couette_droplets` draws
the droplet-in-Couette domains of config 4 from a seed, and `deformation`
measures the Taylor deformation D = (L - B)/(L + B) of a droplet.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi, workloads
from .solver import TslbError


class Ensemble:
    def __init__(self, params: list, dims: list):
        self.L = capi.lib()
        self.n = len(params)
        self.dims = [tuple(int(v) for v in d) for d in dims]
        arr = (capi.TslbParams * self.n)(*params)
        self._params = arr
        d = (ctypes.c_int * (3 * self.n))(*[v for dd in self.dims for v in dd])
        h = ctypes.c_void_p()
        rc = self.L.tslb_ensemble_create(ctypes.addressof(arr), d, self.n, ctypes.byref(h))
        if rc != capi.OK:
            raise TslbError(rc, self.L.tslb_ensemble_last_error(None).decode())
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.tslb_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != capi.OK:
            raise TslbError(rc, self.L.tslb_ensemble_last_error(self.h).decode())

    def shape(self, i: int):
        nx, ny, nz = self.dims[i]
        return (nz, ny, nx)

    def upload_moments(self, i: int, fields: dict) -> None:
        arrs = [np.ascontiguousarray(fields[k], np.float32).reshape(self.shape(i)) for k in capi.FIELDS]
        self._check(self.L.tslb_ensemble_upload_moments(self.h, i, *[capi.fptr(a) for a in arrs]))

    def download(self, i: int) -> dict:
        out = {k: np.empty(self.shape(i), np.float32) for k in capi.FIELDS}
        self._check(self.L.tslb_ensemble_download_moments(self.h, i, *[capi.fptr(out[k]) for k in capi.FIELDS]))
        return out

    def step(self, nsteps: int = 1) -> None:
        self._check(self.L.tslb_ensemble_step(self.h, nsteps))

    def step_graph(self, nsteps: int) -> None:
        self._check(self.L.tslb_ensemble_step_graph(self.h, nsteps))

    def reduce(self, i: int) -> dict:
        out = np.zeros(capi.NREDUCE, np.float64)
        self._check(self.L.tslb_ensemble_reduce(self.h, i, capi.dptr(out)))
        return dict(zip(capi.RED_NAMES, out.tolist()))

    def tune(self):
        zc, gr = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.tslb_ensemble_tune(self.h, ctypes.byref(zc), ctypes.byref(gr)))
        return zc.value, gr.value

    def tune_results(self) -> list:
        """The last tune()'s timings: dicts of zchunk (1 << 20: whole
        lattices), grid (resident blocks of the persistent kernel) and ms
        per step."""
        n = ctypes.c_int()
        self._check(self.L.tslb_ensemble_tune_results(self.h, 0, ctypes.byref(n), None, None, None))
        zc = (ctypes.c_int * max(n.value, 1))()
        gr = (ctypes.c_int * max(n.value, 1))()
        ms = (ctypes.c_float * max(n.value, 1))()
        self._check(self.L.tslb_ensemble_tune_results(self.h, n.value, ctypes.byref(n), zc, gr, ms))
        return [dict(zchunk=zc[i], grid=gr[i], ms=ms[i]) for i in range(n.value)]

    def set_launch(self, zchunk: int, grid: int) -> None:
        """Fix the z chunk and the grid (0: one block per work item; > 0:
        that many blocks taking the items as they finish) without tuning."""
        self._check(self.L.tslb_ensemble_set_launch(self.h, int(zchunk), int(grid)))

    def synchronize(self) -> None:
        self._check(self.L.tslb_ensemble_synchronize(self.h))

    @property
    def stream(self) -> int:
        return int(self.L.tslb_ensemble_stream(self.h) or 0)

    @property
    def nodes(self) -> int:
        return sum(a * b * c for a, b, c in self.dims)


def couette_droplets(n: int = 48, seed: int = 2024, uwall: float = 0.05, tau_matrix: float = 1.0):
    """Config 4 domains: Lx in [48, 128], Ly = Lz in [32, 96] (multiples of 8),
    walls at z moving at -+uwall, x and y periodic, a centred droplet of
    radius U[0.2, 0.3] Lz, capillary number U[0.1, 0.5] and viscosity ratio
    (droplet / matrix) U[1, 4].  Component A (phi = +1) is the droplet."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nu_m = (tau_matrix - 0.5) / 3.0
    domains = []
    for _ in range(n):
        lx = int(rng.integers(6, 17)) * 8
        lz = int(rng.integers(4, 13)) * 8
        ly = lz
        R = float(rng.uniform(0.2, 0.3)) * lz
        ca = float(rng.uniform(0.1, 0.5))
        lam = float(rng.uniform(1.0, 4.0))
        shear = 2.0 * uwall / lz
        sigma = nu_m * shear * R / ca
        tau_d = 3.0 * lam * nu_m + 0.5
        p = capi.make_params(mode=capi.MODE_COLOUR, tau_a=tau_d, tau_b=tau_matrix, sigma=sigma, beta=0.7,
                             grad_threshold=1e-3,
                             bc=[capi.BC_PERIODIC] * 4 + [capi.BC_VELOCITY] * 2,
                             bc_u=[[0, 0, 0]] * 4 + [[-uwall, 0, 0], [uwall, 0, 0]],
                             bc_phi=[-1.0] * 6, wall_phi_mode=1)
        f = workloads.empty_fields(lx, ly, lz)
        z, y, x = np.meshgrid(np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
        r = np.sqrt((x - (lx - 1) / 2) ** 2 + (y - (ly - 1) / 2) ** 2 + (z - (lz - 1) / 2) ** 2)
        f["phi"][:] = np.tanh((R - r) / 2.0)
        # linear Couette flow as the initial velocity
        f["u"][:] = (uwall * (2.0 * (z + 0.5) / lz - 1.0)).astype(np.float32)
        domains.append(dict(params=p, dims=(lx, ly, lz), fields=f, radius=R, ca=ca, lam=lam, sigma=sigma))
    return domains


def deformation(phi: np.ndarray) -> float:
    """Taylor deformation D = (L - B)/(L + B) of the phi > 0 region, from the
    eigenvalues of its second-moment tensor (L, B: longest and shortest axes)."""
    w = np.clip(np.asarray(phi, np.float64), 0.0, None)
    if w.sum() <= 0:
        return 0.0
    nz, ny, nx = w.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m = w.sum()
    c = [float((w * q).sum() / m) for q in (x, y, z)]
    d = [x - c[0], y - c[1], z - c[2]]
    S = np.array([[float((w * d[i] * d[j]).sum() / m) for j in range(3)] for i in range(3)])
    ev = np.sort(np.linalg.eigvalsh(S))
    Lr, Br = np.sqrt(ev[-1]), np.sqrt(max(ev[0], 0.0))
    return float((Lr - Br) / (Lr + Br))
