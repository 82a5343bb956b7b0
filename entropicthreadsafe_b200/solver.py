"""Host-side handle of one TSLB lattice on the GPU, over the C-ABI.

Mirrors the reference driver's view of the state (the vars-module arrays of
recursive_2c_TSLB3D.f90 / TSLB_2C-mpi/vars_single_3D_module.f90): fields are
numpy arrays of shape (nz, ny, nx) in C order, which is exactly Fortran's
column-major (1:nx,1:ny,1:nz) with x fastest.  Every method is one call
through libtslb.so; errors raise TslbError with the library's message.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi


class TslbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tslb error {code}: {msg}")
        self.code = code


class Lattice:
    def __init__(self, params: capi.TslbParams, nx: int, ny: int, nz: int):
        self.L = capi.lib()
        self.params = params
        self.shape = (nz, ny, nx)
        self.n = nx * ny * nz
        h = ctypes.c_void_p()
        rc = self.L.tslb_create(ctypes.addressof(params), nx, ny, nz, ctypes.byref(h))
        if rc != capi.OK:
            raise TslbError(rc, self.L.tslb_last_error(None).decode())
        self.h = h

    # -- lifetime --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.tslb_destroy(self.h)
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
            raise TslbError(rc, self.L.tslb_last_error(self.h).decode())

    # -- state -----------------------------------------------------------
    def upload_moments(self, fields: dict) -> None:
        arrs = [np.ascontiguousarray(fields[k], np.float32).reshape(self.shape) for k in capi.FIELDS]
        self._check(self.L.tslb_upload_moments(self.h, *[capi.fptr(a) for a in arrs]))

    def upload_pops(self, f: np.ndarray, g: np.ndarray) -> None:
        """f: (27, nz+2, ny+2, nx+2), g: (7|27, nz+2, ny+2, nx+2) -- the reference's
        f(0:nx+1,0:ny+1,0:nz+1,0:26) in memory order."""
        f = np.ascontiguousarray(f, np.float32)
        g = np.ascontiguousarray(g, np.float32)
        self._check(self.L.tslb_upload_pops(self.h, capi.fptr(f), capi.fptr(g)))

    def download(self, out: dict | None = None) -> dict:
        if out is None:
            out = {k: np.empty(self.shape, np.float32) for k in capi.FIELDS}
        self._check(self.L.tslb_download_moments(self.h, *[capi.fptr(out[k]) for k in capi.FIELDS]))
        return out

    def normals(self) -> np.ndarray:
        out = np.empty((3,) + self.shape, np.float32)
        self._check(self.L.tslb_download_normals(self.h, capi.fptr(out[0]), capi.fptr(out[1]), capi.fptr(out[2])))
        return out

    def set_inlet(self, face: int, planes: np.ndarray) -> None:
        planes = np.ascontiguousarray(planes, np.float32)
        self._check(self.L.tslb_set_inlet(self.h, face, capi.fptr(planes)))

    def set_inlet_disc(self, face: int, c0: float, c1: float, radius: float, speed: float, amp: float,
                       seed: int, counter: int) -> None:
        """Jet inlet drawn on the device (see tslb_set_inlet_disc; workloads.inlet_disc is its host mirror)."""
        self._check(self.L.tslb_set_inlet_disc(self.h, face, c0, c1, radius, speed, amp, int(seed), int(counter)))

    def set_moment_bc(self, face: int, kind: int, uwall: float = 0.0, radius: float = 10.0, amp: float = 0.004) -> None:
        """Moment-space boundary plane of a z face (tslb_set_moment_bc)."""
        self._check(self.L.tslb_set_moment_bc(self.h, face, kind, uwall, radius, amp))

    def set_solid_mask(self, isfluid) -> None:
        """Interior solid nodes: isfluid (nz, ny, nx), 1 fluid / 0 solid, or None."""
        if isfluid is None:
            self._check(self.L.tslb_set_solid_mask(self.h, None))
            return
        m = np.ascontiguousarray(isfluid, np.uint8).reshape(self.shape)
        self._check(self.L.tslb_set_solid_mask(self.h, m.ctypes.data))

    def set_tau_correction(self, dtau) -> None:
        """Per-node relaxation-time correction (nz, ny, nx), or None to switch it off."""
        if dtau is None:
            self._check(self.L.tslb_set_tau_correction(self.h, None))
            return
        d = np.ascontiguousarray(dtau, np.float32).reshape(self.shape)
        self._check(self.L.tslb_set_tau_correction(self.h, capi.fptr(d)))

    def tau_correction(self) -> np.ndarray:
        out = np.empty(self.shape, np.float32)
        self._check(self.L.tslb_download_tau_correction(self.h, capi.fptr(out)))
        return out

    # -- checkpoints (include/tslb_io.h) --------------------------------
    def checkpoint_save(self, path: str) -> None:
        self._check(self.L.tslb_checkpoint_save(self.h, str(path).encode()))

    def checkpoint_load(self, path: str) -> None:
        self._check(self.L.tslb_checkpoint_load(self.h, str(path).encode()))

    @property
    def steps_done(self) -> int:
        return int(self.L.tslb_steps_done(self.h))

    # -- time averages ---------------------------------------------------
    def stats_reset(self) -> None:
        self._check(self.L.tslb_stats_reset(self.h))

    def stats_accumulate(self) -> None:
        self._check(self.L.tslb_stats_accumulate(self.h))

    def stats(self, coarsen: int = 1) -> dict:
        """Means of u, v, w, phi, w^2 over the accumulated samples, averaged over coarsen^3 blocks."""
        nz, ny, nx = self.shape
        shp = (nz // coarsen, ny // coarsen, nx // coarsen)
        out = {k: np.empty(shp, np.float32) for k in ("u", "v", "w", "phi", "ww")}
        cnt = ctypes.c_longlong()
        self._check(self.L.tslb_stats_download(self.h, coarsen, *[capi.fptr(out[k]) for k in ("u", "v", "w", "phi", "ww")],
                                               ctypes.byref(cnt)))
        out["count"] = int(cnt.value)
        return out

    def stats_stress(self, coarsen: int = 1) -> dict:
        """Means of the products u_a u_b ("uu": uu, uv, uw, vv, vw, ww) and of
        Pi^neq ("pineq": xx, xy, xz, yy, yz, zz) over the accumulated samples,
        averaged over coarsen^3 blocks; arrays of shape (6, nz', ny', nx')."""
        nz, ny, nx = self.shape
        shp = (6, nz // coarsen, ny // coarsen, nx // coarsen)
        uu, pi = np.empty(shp, np.float32), np.empty(shp, np.float32)
        cnt = ctypes.c_longlong()
        self._check(self.L.tslb_stats_download_stress(self.h, coarsen, capi.fptr(uu), capi.fptr(pi), ctypes.byref(cnt)))
        return {"uu": uu, "pineq": pi, "count": int(cnt.value)}

    # -- time stepping ---------------------------------------------------
    def step(self, nsteps: int = 1) -> None:
        self._check(self.L.tslb_step(self.h, nsteps))

    def synchronize(self) -> None:
        self._check(self.L.tslb_synchronize(self.h))

    def reduce(self) -> dict:
        out = np.zeros(capi.NREDUCE, np.float64)
        self._check(self.L.tslb_reduce(self.h, capi.dptr(out)))
        return dict(zip(capi.RED_NAMES, out.tolist()))

    def reduce_async(self) -> None:
        """Queue the diagnostics of the state after the queued steps (no wait)."""
        self._check(self.L.tslb_reduce_async(self.h))

    def reduce_collect(self) -> list:
        """Wait and return the queued diagnostics, oldest first."""
        out = np.zeros((capi.REDUCE_QUEUE, capi.NREDUCE), np.float64)
        cnt = ctypes.c_int()
        self._check(self.L.tslb_reduce_collect(self.h, capi.dptr(out), capi.REDUCE_QUEUE, ctypes.byref(cnt)))
        return [dict(zip(capi.RED_NAMES, row.tolist())) for row in out[:cnt.value]]

    @property
    def stream(self) -> int:
        return int(self.L.tslb_stream(self.h) or 0)

    @property
    def launches(self) -> int:
        return int(self.L.tslb_launch_count(self.h))
