"""Learned eddy-viscosity closure over the C-ABI (include/tslb_closure.h).

A `Closure` holds the network 10 -> 64 -> 64 -> 1 and its training set on
the GPU.  It corrects the relaxation time of a coarse colour-mode lattice:
`lattice_attach(lat, closure)` makes every step start with the tensor-core
inference kernel writing dtau per node.  The reference has no closure; its
coarse jet (boundary_cds_3D_module.f90:862-1119) runs with the plain tau.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi
from .solver import Lattice, TslbError

NFEAT = capi.CLOSURE_NFEAT
NH = capi.CLOSURE_HIDDEN
NPARAM = capi.CLOSURE_NPARAM
OFF = capi.CLOSURE_OFF
FEATURE_NAMES = ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "phi", "grad_phi", "speed", "pi_norm")


def pack(W1, b1, W2, b2, w3, b3) -> np.ndarray:
    """Parameter vector from the layer arrays (W1 64x10 or 64x16, W2 64x64)."""
    p = np.zeros(NPARAM, np.float32)
    w1 = np.zeros((NH, 16), np.float32)
    W1 = np.asarray(W1, np.float32)
    w1[:, :W1.shape[1]] = W1
    w1[:, NFEAT:] = 0.0
    p[OFF["W1"]:OFF["b1"]] = w1.reshape(-1)
    p[OFF["b1"]:OFF["W2"]] = b1
    p[OFF["W2"]:OFF["b2"]] = np.asarray(W2, np.float32).reshape(-1)
    p[OFF["b2"]:OFF["w3"]] = b2
    p[OFF["w3"]:OFF["b3"]] = w3
    p[OFF["b3"]] = b3
    return p


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p)
    return {
        "W1": p[OFF["W1"]:OFF["b1"]].reshape(NH, 16)[:, :NFEAT].copy(),
        "b1": p[OFF["b1"]:OFF["W2"]].copy(),
        "W2": p[OFF["W2"]:OFF["b2"]].reshape(NH, NH).copy(),
        "b2": p[OFF["b2"]:OFF["w3"]].copy(),
        "w3": p[OFF["w3"]:OFF["b3"]].copy(),
        "b3": float(p[OFF["b3"]]),
    }


def init_params(seed: int = 0, out_bias: float = -4.0) -> np.ndarray:
    """He-initialised hidden layers, small output layer, output bias giving
    dtau near dtau_max * sigmoid(out_bias) at the start."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, np.sqrt(2.0 / NFEAT), (NH, NFEAT))
    W2 = rng.normal(0.0, np.sqrt(2.0 / NH), (NH, NH))
    w3 = rng.normal(0.0, np.sqrt(1.0 / NH), NH) * 0.1
    return pack(W1, np.zeros(NH), W2, np.zeros(NH), w3, out_bias)


class Closure:
    def __init__(self):
        self.L = capi.lib()
        h = ctypes.c_void_p()
        rc = self.L.tslb_closure_create(ctypes.byref(h))
        if rc != capi.OK:
            raise TslbError(rc, self.L.tslb_closure_last_error(None).decode())
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.tslb_closure_destroy(self.h)
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
            raise TslbError(rc, self.L.tslb_closure_last_error(self.h).decode())

    # -- parameters -------------------------------------------------------
    def set_params(self, params=None, mu=None, sd=None, dtau_max: float | None = None) -> None:
        if dtau_max is None:
            dtau_max = self.get_params()["dtau_max"]
        arrs = []
        for a, n in ((params, NPARAM), (mu, NFEAT), (sd, NFEAT)):
            arrs.append(None if a is None else np.ascontiguousarray(a, np.float32).reshape(n))
        ptrs = [None if a is None else capi.fptr(a) for a in arrs]
        self._check(self.L.tslb_closure_set_params(self.h, *ptrs, float(dtau_max)))

    def get_params(self) -> dict:
        p = np.empty(NPARAM, np.float32)
        mu = np.empty(NFEAT, np.float32)
        sd = np.empty(NFEAT, np.float32)
        dm = ctypes.c_float()
        self._check(self.L.tslb_closure_get_params(self.h, capi.fptr(p), capi.fptr(mu), capi.fptr(sd), ctypes.byref(dm)))
        return {"params": p, "mu": mu, "sd": sd, "dtau_max": float(dm.value),
                "dtau_min": float(self.L.tslb_closure_dtau_min(self.h))}

    def set_dtau_min(self, dtau_min: float) -> None:
        """Lower bound of the output (<= 0): dtau = lo + (hi - lo) sigmoid(o)."""
        self._check(self.L.tslb_closure_set_dtau_min(self.h, float(dtau_min)))

    # -- evaluation ---------------------------------------------------------
    def forward(self, features: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32).reshape(-1, NFEAT)
        out = np.empty(f.shape[0], np.float32)
        self._check(self.L.tslb_closure_forward(self.h, capi.fptr(f), f.shape[0], capi.fptr(out)))
        return out

    def gradient(self, features, target, weight):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, NFEAT)
        t = np.ascontiguousarray(target, np.float32).reshape(-1)
        w = np.ascontiguousarray(weight, np.float32).reshape(-1)
        g = np.empty(NPARAM, np.float32)
        loss = ctypes.c_double()
        self._check(self.L.tslb_closure_gradient(self.h, capi.fptr(f), capi.fptr(t), capi.fptr(w), f.shape[0],
                                                 capi.fptr(g), ctypes.byref(loss)))
        return g, float(loss.value)

    def features(self, lat: Lattice) -> np.ndarray:
        out = np.empty((lat.n, NFEAT), np.float32)
        self._check(self.L.tslb_closure_features(self.h, lat.h, capi.fptr(out)))
        return out

    # -- training set ---------------------------------------------------------
    def dataset_clear(self) -> None:
        self._check(self.L.tslb_closure_dataset_clear(self.h))

    def dataset_add(self, features, target, weight) -> None:
        f = np.ascontiguousarray(features, np.float32).reshape(-1, NFEAT)
        t = np.ascontiguousarray(target, np.float32).reshape(-1)
        w = np.ascontiguousarray(weight, np.float32).reshape(-1)
        self._check(self.L.tslb_closure_dataset_add(self.h, capi.fptr(f), capi.fptr(t), capi.fptr(w), f.shape[0]))

    def dataset_add_fine(self, fine: Lattice, pi_scale: float, keep_every: int = 1, z_range=(0, 0)) -> int:
        """Samples of the fine lattice on the coarse planes z_range[0] <= z < z_range[1] (0: to the end)."""
        n = ctypes.c_longlong()
        self._check(self.L.tslb_closure_dataset_add_fine(self.h, fine.h, float(pi_scale), int(keep_every),
                                                         int(z_range[0]), int(z_range[1]), ctypes.byref(n)))
        return int(n.value)

    @property
    def dataset_size(self) -> int:
        return int(self.L.tslb_closure_dataset_size(self.h))

    def dataset(self):
        n = self.dataset_size
        f = np.empty((n, NFEAT), np.float32)
        t = np.empty(n, np.float32)
        w = np.empty(n, np.float32)
        if n:
            self._check(self.L.tslb_closure_dataset_download(self.h, capi.fptr(f), capi.fptr(t), capi.fptr(w)))
        return f, t, w

    def normalize(self) -> None:
        self._check(self.L.tslb_closure_normalize(self.h))

    def train(self, steps: int, batch: int = 16384, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        hist = np.empty(max(steps, 1), np.float32)
        self._check(self.L.tslb_closure_train(self.h, int(steps), int(batch), float(lr), int(seed), capi.fptr(hist)))
        return hist[:steps]


TRAINED_JET = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "closure_jet_192.npz")


def load_trained(path: str = TRAINED_JET) -> dict:
    """A trained network: params, mu, sd, dtau_max, the calibrated output
    gain and (optional) the output's lower bound dtau_min.  The packaged file
    is the network of the round-jet study (closure_study: trained on
    box-filtered 384 x 384 x 768 runs; gain 1 and dtau_min = -0.00075 chosen a
    posteriori on coarse 192 x 192 x 384 runs, closure_study --calibrate)."""
    d = np.load(path)
    return {k: d[k] for k in d.files}


def trained_closure(path: str = TRAINED_JET) -> "Closure":
    """A Closure loaded with a trained network, its output scaled by the calibrated gain."""
    t = load_trained(path)
    c = Closure()
    c.set_params(t["params"], t["mu"], t["sd"], float(t["dtau_max"]) * float(t["gain"]))
    if "dtau_min" in t:
        c.set_dtau_min(float(t["dtau_min"]) * float(t["gain"]))
    return c


def lattice_attach(lat: Lattice, closure: Closure | None, interval: int = 1) -> None:
    """Attach (or with None detach) the closure to a colour-mode FP32 lattice."""
    rc = lat.L.tslb_attach_closure(lat.h, closure.h if closure is not None else None, int(interval))
    lat._check(rc)
