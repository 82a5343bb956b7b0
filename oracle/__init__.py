"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle.

The oracle restates the reference's two-component TSLB step on the CPU
(see tslb_oracle.hpp for the reference file:line map).  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this
package; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
NFIELD = 11
FIELDS = ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "phi")


def build(quiet: bool = True) -> None:
    """Compile the oracle libraries with its Makefile (g++, OpenMP)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_LIBS: dict = {}


def _lib(fast: bool = False) -> ctypes.CDLL:
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name not in _LIBS:
        path = os.path.join(_BUILD, name)
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        lib.orc_create.restype = vp
        lib.orc_create.argtypes = [vp, ip, ip, ip, ip]
        lib.orc_destroy.argtypes = [vp]
        for fn in ("orc_set_moments", "orc_get_moments", "orc_get_normals", "orc_reduce"):
            getattr(lib, fn).argtypes = [vp, dp]
            getattr(lib, fn).restype = ip
        lib.orc_set_pops.argtypes = [vp, dp, dp]
        lib.orc_set_pops.restype = ip
        lib.orc_set_inlet.argtypes = [vp, ip, dp]
        lib.orc_set_inlet.restype = ip
        lib.orc_set_isfluid.argtypes = [vp, vp]
        lib.orc_set_isfluid.restype = ip
        lib.orc_set_dtau.argtypes = [vp, dp]
        lib.orc_set_dtau.restype = ip
        lib.orc_step.argtypes = [vp, ip]
        lib.orc_step.restype = ip
        _LIBS[name] = lib
    return _LIBS[name]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """CPU restatement of the step; state = moments (see tslb_oracle.hpp).

    params: a ctypes tslb_params structure (entropicthreadsafe_b200 defines it).
    Fields are numpy arrays of shape (nz, ny, nx) (C order == Fortran x-fastest).
    """

    def __init__(self, params, nx: int, ny: int, nz: int, fp64: bool = True, fast: bool = False):
        self.lib = _lib(fast)
        self.shape = (nz, ny, nx)
        self.n = nx * ny * nz
        self.fp64 = fp64
        self.h = self.lib.orc_create(ctypes.addressof(params), nx, ny, nz, int(fp64))
        if not self.h:
            raise ValueError("orc_create failed")

    def close(self) -> None:
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(f"oracle call failed: {rc}")

    def set_moments(self, fields: dict) -> None:
        buf = np.empty((NFIELD,) + self.shape, np.float64)
        for c, name in enumerate(FIELDS):
            buf[c] = fields[name]
        self._check(self.lib.orc_set_moments(self.h, _dptr(buf)))

    def get_moments(self) -> dict:
        buf = np.empty((NFIELD,) + self.shape, np.float64)
        self._check(self.lib.orc_get_moments(self.h, _dptr(buf)))
        return {name: buf[c].copy() for c, name in enumerate(FIELDS)}

    def set_pops(self, f: np.ndarray, g: np.ndarray) -> None:
        """f: (27, nz, ny, nx); g: (7 or 27, nz, ny, nx), interior nodes."""
        f = np.ascontiguousarray(f, np.float64)
        g = np.ascontiguousarray(g, np.float64)
        self._check(self.lib.orc_set_pops(self.h, _dptr(f), _dptr(g)))

    def set_inlet(self, face: int, planes: np.ndarray) -> None:
        planes = np.ascontiguousarray(planes, np.float64)
        self._check(self.lib.orc_set_inlet(self.h, face, _dptr(planes)))

    def set_isfluid(self, isfluid) -> None:
        """Interior solid nodes: isfluid (nz, ny, nx), 1 fluid / 0 solid, or None."""
        if isfluid is None:
            self._check(self.lib.orc_set_isfluid(self.h, None))
            return
        m = np.ascontiguousarray(isfluid, np.uint8).reshape(self.shape)
        self._check(self.lib.orc_set_isfluid(self.h, m.ctypes.data))

    def set_tau_correction(self, dtau) -> None:
        """Per-node correction of the colour-mode relaxation time, (nz, ny, nx), or None."""
        if dtau is None:
            self._check(self.lib.orc_set_dtau(self.h, None))
            return
        d = np.ascontiguousarray(dtau, np.float64).reshape(self.shape)
        self._check(self.lib.orc_set_dtau(self.h, _dptr(d)))

    def normals(self) -> np.ndarray:
        buf = np.empty((3,) + self.shape, np.float64)
        self._check(self.lib.orc_get_normals(self.h, _dptr(buf)))
        return buf

    def step(self, nsteps: int = 1) -> None:
        self._check(self.lib.orc_step(self.h, nsteps))

    def reduce(self) -> np.ndarray:
        out = np.zeros(12, np.float64)
        self._check(self.lib.orc_reduce(self.h, _dptr(out)))
        return out
