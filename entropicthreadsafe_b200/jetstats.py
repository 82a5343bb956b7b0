"""Statistics of the round jet from time-averaged fields.

The reference's drivers average frames written by print_module.f90 on the
host; here the library accumulates the means on the device
(tslb_stats_accumulate) and these functions reduce them to the jet's
statistics, all in units of the coarse grid (the fine grid's means are
averaged over 2x2x2 blocks first):

  centreline velocity  w_c(z): mean w over the nodes within 1 of the axis;
  half-width           r_half(z): radius where the azimuthally averaged
                       excess velocity falls to half of its axis value;
  spreading rate       d r_half / dz, least squares over the window;
  decay rate           d (w_in / w_c) / d(z / D), least squares;
  mixing thickness     delta(z) = integral over r of (1 - mean phi^2),
                       zero for an unmixed sharp interface.
"""
from __future__ import annotations

import numpy as np


def radial(mean: np.ndarray, cx: float, cy: float, rmax: float):
    """Azimuthal averages in unit-wide radius bins: (r_bin_mean, prof[z, bin])."""
    nz, ny, nx = mean.shape
    y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    nb = int(rmax)
    b = np.floor(r).astype(np.int64)
    m = b < nb
    cnt = np.bincount(b[m], minlength=nb).astype(np.float64)
    rb = np.bincount(b[m], weights=r[m], minlength=nb) / np.maximum(cnt, 1)
    flat = mean.reshape(nz, -1)[:, m.reshape(-1)]
    idx = b[m]
    prof = np.stack([np.bincount(idx, weights=flat[k], minlength=nb) / np.maximum(cnt, 1) for k in range(nz)])
    return rb, prof


def half_width(rb: np.ndarray, prof_w: np.ndarray) -> np.ndarray:
    amb = prof_w[:, -4:].mean(axis=1, keepdims=True)
    ex = prof_w - amb
    out = np.full(prof_w.shape[0], np.nan)
    for k in range(prof_w.shape[0]):
        e = ex[k]
        if e[0] <= 0:
            continue
        h = 0.5 * e[0]
        below = np.nonzero(e < h)[0]
        if below.size == 0 or below[0] == 0:
            continue
        j = below[0]
        out[k] = rb[j - 1] + (e[j - 1] - h) / (e[j - 1] - e[j]) * (rb[j] - rb[j - 1])
    return out


def jet_statistics(mean_w: np.ndarray, mean_phi: np.ndarray, cx: float, cy: float, diameter: float, w_in: float,
                   window=(6.0, 20.0), rmax: float | None = None) -> dict:
    """Scalars and profiles of the jet; window in diameters from the inlet."""
    nz, ny, nx = mean_w.shape
    rmax = rmax or 0.5 * min(nx, ny)
    rb, pw = radial(mean_w, cx, cy, rmax)
    _, pp = radial(mean_phi, cx, cy, rmax)
    z = np.arange(nz) + 0.5
    wc = pw[:, 0]
    rh = half_width(rb, pw)
    delta = np.sum(1.0 - np.clip(pp, -1, 1) ** 2, axis=1)   # unit-wide bins
    z0, z1 = window[0] * diameter, window[1] * diameter
    sel = (z >= z0) & (z <= z1) & np.isfinite(rh) & (wc > 0)
    out = dict(z=z, wc=wc, r_half=rh, delta=delta, window=[z0, z1])
    if sel.sum() >= 4:
        out["spreading_rate"] = float(np.polyfit(z[sel], rh[sel], 1)[0])
        out["decay_rate"] = float(np.polyfit(z[sel] / diameter, w_in / wc[sel], 1)[0])
        out["mixing_thickness"] = float(np.mean(delta[sel]))
        out["centreline_mean"] = float(np.mean(wc[sel]))
    else:
        out["spreading_rate"] = out["decay_rate"] = out["mixing_thickness"] = out["centreline_mean"] = float("nan")
    return out


def compare(stats: dict, ref: dict) -> dict:
    """Relative differences of the scalar statistics and profiles against the reference (fine-grid) run."""
    res = {}
    for k in ("spreading_rate", "decay_rate", "mixing_thickness", "centreline_mean"):
        a, b = stats[k], ref[k]
        res[k] = float(abs(a - b) / abs(b)) if np.isfinite(a) and np.isfinite(b) and b != 0 else float("nan")
    z0, z1 = ref["window"]
    sel = (ref["z"] >= z0) & (ref["z"] <= z1)
    for k in ("wc", "r_half", "delta"):
        a, b = np.asarray(stats[k])[sel], np.asarray(ref[k])[sel]
        ok = np.isfinite(a) & np.isfinite(b)
        res[k + "_profile"] = float(np.linalg.norm(a[ok] - b[ok]) / max(np.linalg.norm(b[ok]), 1e-30)) if ok.any() else float("nan")
    return res
