"""Long-run effect of the 16-bit moment storage on the channel flow.

    python -m entropicthreadsafe_b200.precision_study [--steps 20000] [--every 500] [--avg 5000] [--out result.json]
    python -m entropicthreadsafe_b200.precision_study --table200 [--out result.json]

The two-component channel (workloads.channel, 384 x 192 x 128, 40 droplets)
is advanced with the moments stored in FP32, in BF16 and in FP16 with a
per-field power-of-two scale (collision in FP32 throughout).  Over the last
`avg` steps, every `every` steps, the velocity is read back and reduced to

  * the mean streamwise velocity profile u_x(z): u averaged over x and y,
    then over the snapshots;
  * the streamwise energy spectrum E(k_x) of the velocity fluctuations,
    E(k) = sum over u, v, w of |FFT_x(u_i - <u_i>_x)|^2 / nx^2, averaged over
    y, over the channel core (the middle half in z) and over the snapshots.

The 16-bit runs are compared with the FP32 run: profile error
max_z |u_x - u_x,FP32| / max_z |u_x,FP32|, and spectrum deviation as the
mean over the resolved wavenumbers (1 <= k < nx/4) of |log10 E - log10 E_FP32|
together with the relative difference of the total fluctuation energy.
The FP32 run stands in for the FP64 solution here (there is no FP64 GPU
path); its own error against the FP64 oracle is measured over 200 steps by
tests/test_gpu_precision.py.  A second FP32 run whose initial velocity is
perturbed by 1e-6 (relative, uniform noise) measures how far two FP32
realisations of this droplet-laden flow drift apart by themselves: the
floor below which a storage form's deviation is not an error of its own.

--table200 measures the short-run errors on the same full channel: each
storage form (with its stochastic rounding) after 200 steps against the
FP64 oracle run of the same 200 steps, per moment field as max and L2
relative error (max|a - b| / max|b|, ||a - b||_2 / ||b||_2; rho as rho - 1).
The FP64 oracle takes a few minutes on the host cores.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def mean_profile(u: np.ndarray) -> np.ndarray:
    """u (nz, ny, nx) -> u averaged over x and y, one value per z."""
    return np.asarray(u, np.float64).mean(axis=(1, 2))


def spectrum_x(u: np.ndarray, v: np.ndarray, w: np.ndarray, core: tuple[int, int]) -> np.ndarray:
    """Streamwise energy spectrum of the fluctuations over the planes core[0] <= z < core[1]:
    E[k] for k = 0 .. nx/2, averaged over y and z."""
    z0, z1 = core
    e = None
    for comp in (u, v, w):
        a = np.asarray(comp[z0:z1], np.float64)
        a = a - a.mean(axis=2, keepdims=True)
        fk = np.fft.rfft(a, axis=2) / a.shape[2]
        p = (np.abs(fk) ** 2).mean(axis=(0, 1))
        e = p if e is None else e + p
    return e


def compare(prof: np.ndarray, spec: np.ndarray, prof_ref: np.ndarray, spec_ref: np.ndarray) -> dict:
    nk = len(spec_ref)
    kmax = max(2, (2 * (nk - 1)) // 4)            # k < nx / 4
    ks = slice(1, kmax)
    ok = (spec[ks] > 0) & (spec_ref[ks] > 0)
    dlog = np.abs(np.log10(spec[ks][ok]) - np.log10(spec_ref[ks][ok]))
    return {
        "profile_max_rel_err": float(np.abs(prof - prof_ref).max() / max(np.abs(prof_ref).max(), 1e-30)),
        "spectrum_mean_abs_dlog10": float(dlog.mean()) if dlog.size else float("nan"),
        "fluctuation_energy_rel_diff": float(abs(spec[1:].sum() - spec_ref[1:].sum()) / max(spec_ref[1:].sum(), 1e-30)),
    }


def run(precision: int, steps: int, every: int, avg: int, perturb: float = 0.0) -> dict:
    from entropicthreadsafe_b200 import workloads
    from entropicthreadsafe_b200.solver import Lattice
    p, f = workloads.channel()
    p.precision = precision
    if perturb:
        rng = np.random.default_rng(2024)
        for k in ("u", "v", "w"):
            f[k] = (f[k] * (1.0 + perturb * rng.uniform(-1, 1, f[k].shape))).astype(np.float32)
    nz, ny, nx = f["rho"].shape
    core = (nz // 4, 3 * nz // 4)
    profs, specs = [], []
    t0 = time.perf_counter()
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        done = 0
        start = steps - avg
        if start > 0:
            lat.step(start)
            done = start
        while done < steps:
            n = min(every, steps - done)
            lat.step(n)
            done += n
            st = lat.download()
            profs.append(mean_profile(st["u"]))
            specs.append(spectrum_x(st["u"], st["v"], st["w"], core))
        red = lat.reduce()
    return {"profile": np.mean(profs, axis=0), "spectrum": np.mean(specs, axis=0), "seconds": time.perf_counter() - t0,
            "snapshots": len(profs), "mass": red["mass"], "umax": red["umax"]}


def field_errors(a: dict, b: dict) -> dict:
    """Per moment field: (max, L2) relative error of a against b; rho as rho - 1."""
    from entropicthreadsafe_b200 import capi
    out = {}
    for k in capi.FIELDS:
        x, y = np.asarray(a[k], np.float64), np.asarray(b[k], np.float64)
        if k == "rho":
            x, y = x - 1.0, y - 1.0
        d = x - y
        out[k] = {"max": float(np.abs(d).max() / max(np.abs(y).max(), 1e-30)),
                  "l2": float(np.sqrt((d * d).sum() / max((y * y).sum(), 1e-60)))}
    return out


def table200(steps: int = 200) -> dict:
    """Every storage form on the full channel after `steps` steps against the FP64 oracle."""
    import oracle
    from entropicthreadsafe_b200 import capi, workloads
    from entropicthreadsafe_b200.solver import Lattice
    p, f = workloads.channel()
    nz, ny, nx = f["rho"].shape
    t0 = time.perf_counter()
    o = oracle.Oracle(p, nx, ny, nz, fp64=True, fast=True)
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    o.step(steps)
    ref = o.get_moments()
    o.close()
    res = {"steps": steps, "oracle_seconds": time.perf_counter() - t0, "forms": {}}
    for name, prec in (("fp32", capi.PREC_FP32), ("bf16", capi.PREC_BF16), ("fp16s", capi.PREC_FP16S)):
        p.precision = prec
        with Lattice(p, nx, ny, nz) as lat:
            lat.upload_moments(f)
            lat.step(steps)
            got = lat.download()
        res["forms"][name] = {"fields": field_errors(got, ref),
                              "mean_profile_max_rel_err": float(np.abs(mean_profile(got["u"]) - mean_profile(ref["u"])).max()
                                                                / np.abs(mean_profile(ref["u"])).max())}
    return res


def main(argv=None) -> int:
    from entropicthreadsafe_b200 import capi
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--avg", type=int, default=5000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--table200", action="store_true", help="200-step errors of every storage form against FP64")
    a = ap.parse_args(argv)
    if a.table200:
        res = table200()
        print(json.dumps(res))
        if a.out:
            with open(a.out, "w") as fh:
                json.dump(res, fh)
        return 0
    from entropicthreadsafe_b200.solver import TslbError
    res = {"steps": a.steps, "every": a.every, "avg": a.avg}
    runs = {}
    cases = (("fp32", capi.PREC_FP32, 0.0), ("fp32_perturbed", capi.PREC_FP32, 1e-6), ("bf16", capi.PREC_BF16, 0.0),
             ("fp16s", capi.PREC_FP16S, 0.0))
    for name, prec, pert in cases:
        try:
            runs[name] = run(prec, a.steps, a.every, a.avg, pert)
        except TslbError as e:   # e.g. the state became non-finite
            res[name] = {"failed": str(e)}
            continue
        res[name] = {"seconds": runs[name]["seconds"], "snapshots": runs[name]["snapshots"],
                     "mass": runs[name]["mass"], "umax": runs[name]["umax"],
                     "profile": runs[name]["profile"].tolist(), "spectrum": runs[name]["spectrum"].tolist()}
    for name in ("fp32_perturbed", "bf16", "fp16s"):
        if name in runs and "fp32" in runs:
            res[name]["vs_fp32"] = compare(runs[name]["profile"], runs[name]["spectrum"], runs["fp32"]["profile"],
                                           runs["fp32"]["spectrum"])
    summary = {k: res[k].get("vs_fp32", res[k].get("failed")) for k in ("fp32_perturbed", "bf16", "fp16s")}
    print(json.dumps({"steps": a.steps, "summary": summary,
                      "seconds": {k: res[k].get("seconds") for k, _, _ in cases}}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
