"""Per-domain deformation of the 48 droplet-in-Couette domains (config 4).

The ensemble (one launch per step, K steps replayed from a CUDA graph, z
chunk and grid from the autotuner) and each domain run alone through the
plain single-lattice step kernel are advanced the same number of steps;
for every domain the Taylor deformation D = (L - B)/(L + B) of the droplet
is measured on both, with Taylor's small-deformation estimate
D_T = Ca (19 lam + 16) / (16 lam + 16) beside them (unbounded shear; the
domains are confined, R / Lz in [0.2, 0.3], so it is an order of magnitude,
not a target).

    python -m entropicthreadsafe_b200.ensemble_study --steps 5000 --out ensemble_deformation.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import ensemble
from .solver import Lattice


def run(steps: int = 5000, n: int = 48, seed: int = 2024, chunk: int = 200) -> dict:
    """steps must be a multiple of chunk (the graph's length)."""
    import torch
    if steps % chunk or steps < 2 * chunk or chunk % 2:
        raise ValueError("steps must be a multiple (>= 2) of an even chunk")
    doms = ensemble.couette_droplets(n=n, seed=seed)
    nodes = sum(a * b * c for a, b, c in (d["dims"] for d in doms))
    with ensemble.Ensemble([d["params"] for d in doms], [d["dims"] for d in doms]) as ens:
        for i, d in enumerate(doms):
            ens.upload_moments(i, d["fields"])
        zc, gr = ens.tune()
        st = torch.cuda.ExternalStream(ens.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # the first `chunk` steps capture the graph (untimed); the rest replay it
        ens.step_graph(chunk)
        ens.synchronize()
        e0.record(st)
        for _ in range(steps // chunk - 1):
            ens.step_graph(chunk)
        e1.record(st)
        ens.synchronize()
        ms_ens = e0.elapsed_time(e1)
        phi_ens = [ens.download(i)["phi"] for i in range(n)]
    d_ens = [ensemble.deformation(p) for p in phi_ens]
    d_single, ms_single, same = [], 0.0, []
    for i, d in enumerate(doms):
        nx, ny, nz = d["dims"]
        with Lattice(d["params"], nx, ny, nz) as lat:
            lat.upload_moments(d["fields"])
            st = torch.cuda.ExternalStream(lat.stream)
            lat.step(chunk)
            e0.record(st)
            lat.step(steps - chunk)
            e1.record(st)
            lat.synchronize()
            ms_single += e0.elapsed_time(e1)
            phi = lat.download()["phi"]
            d_single.append(ensemble.deformation(phi))
            same.append(bool(np.array_equal(phi, phi_ens[i])))
    rows = []
    for i, d in enumerate(doms):
        lam, ca = d["lam"], d["ca"]
        rows.append(dict(domain=i, dims=list(d["dims"]), radius=d["radius"], ca=ca, lam=lam,
                         d_ensemble=d_ens[i], d_single=d_single[i], abs_diff=abs(d_ens[i] - d_single[i]),
                         phi_bit_equal=same[i], d_taylor=ca * (19 * lam + 16) / (16 * lam + 16)))
    return dict(steps=steps, domains=n, seed=seed, nodes=nodes, tuned=dict(zchunk=zc, grid=gr),
                ensemble_ms=ms_ens, single_ms=ms_single,
                ensemble_mlups=nodes * (steps - chunk) / (ms_ens * 1e-3) / 1e6,
                single_mlups=nodes * (steps - chunk) / (ms_single * 1e-3) / 1e6,
                all_phi_bit_equal=all(same),
                max_abs_diff=max(r["abs_diff"] for r in rows), rows=rows)


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--domains", type=int, default=48)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    t0 = time.perf_counter()
    r = run(args.steps, args.domains, args.seed)
    r["wall_s"] = time.perf_counter() - t0
    print(f"{r['domains']} domains, {r['steps']} steps: ensemble {r['ensemble_mlups']:.0f} MLUPS "
          f"(tuned {r['tuned']}), one at a time {r['single_mlups']:.0f} MLUPS, max |D_ens - D_single| "
          f"{r['max_abs_diff']:.3g}", flush=True)
    for row in r["rows"]:
        print("{domain:2d} {dims} Ca {ca:.3f} lam {lam:.2f} D {d_ensemble:.4f} single {d_single:.4f} "
              "Taylor {d_taylor:.3f}".format(**row))
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(r, fh, indent=1)
    return r


if __name__ == "__main__":
    main()
