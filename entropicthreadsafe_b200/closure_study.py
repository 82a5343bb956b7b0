"""Learned-closure study on the round jet (coarse + closure vs coarse plain
vs fine plain).

    python -m entropicthreadsafe_b200.closure_study [--out result.json] [--shrink K]

1. Fine plain runs (384 x 384 x 768, two inlet-noise seeds) feed the
   training set: snapshots of their state, box-filtered onto the coarse
   grid (tslb_closure_dataset_add_fine).
2. The network is trained on the GPU (tslb_closure_train).
3. A third fine plain run (another seed) is the judge: its time-averaged
   fields give the reference jet statistics, and snapshots of it give a
   held-out a-priori test of the network.
4. Coarse plain and coarse + closure runs (192 x 192 x 384, the judge's
   seed) are compared with the judge on spreading rate, centreline decay
   and mixing thickness; GPU time (CUDA events on each lattice's stream)
   is reported for every run.

Times are in coarse steps; the fine grid runs twice as many steps
(acoustic scaling).  --shrink K divides the lattice sizes and the jet
diameter by K and the step counts by K (a quick check of the pipeline;
the physics of a shrunk jet is not the configuration's).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import jetstats, workloads
from .closure import Closure, init_params, lattice_attach
from .solver import Lattice, TslbError


def _events(stream_handle):
    import torch
    st = torch.cuda.ExternalStream(stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return st, e0, e1


def run_jet(scale: int, seed: int, steps: int, avg_from: int, sample_every: int, over: dict, closure=None,
            interval: int = 1, dataset=None, snaps=(), keep_every: int = 8, pi_scale: float = 2.0,
            check_every: int = 500, sponge=(0.15, 0.3)) -> dict:
    """One jet run; returns its statistics (coarse units), GPU time and state.

    Training samples (dataset) are taken outside the sponge layer, whose
    added viscosity the fine stresses carry."""
    p, f, spec = workloads.jet(scale, **over)
    z_hi = int((1.0 - sponge[0]) * spec["nz"] / scale) if sponge is not None else 0
    res = dict(scale=scale, seed=seed, steps=steps, nodes=spec["nx"] * spec["ny"] * spec["nz"],
               closure=closure is not None, diverged_at=None, snapshots=0, samples=0)
    with Lattice(p, spec["nx"], spec["ny"], spec["nz"]) as lat:
        lat.upload_moments(f)
        if sponge is not None and sponge[1] > 0:
            lat.set_tau_correction(workloads.jet_sponge(spec, *sponge))
        if closure is not None:
            lattice_attach(lat, closure, interval)
        lat.stats_reset()
        st, e0, e1 = _events(lat.stream)
        t0 = time.perf_counter()
        e0.record(st)
        snaps = set(snaps)
        done = 0
        try:
            for s in range(steps):
                if s % spec["refresh"] == 0:
                    workloads.jet_inlet(lat, spec, seed, s)
                lat.step(1)
                done = s + 1
                if done >= avg_from and (done - avg_from) % sample_every == 0:
                    lat.stats_accumulate()
                if dataset is not None and done in snaps:
                    res["samples"] += dataset.dataset_add_fine(lat, pi_scale, keep_every, (0, z_hi))
                    res["snapshots"] += 1
                if done % check_every == 0:
                    lat.synchronize()
        except TslbError as e:
            res["diverged_at"] = done
            res["error"] = str(e)
        e1.record(st)
        e1.synchronize()
        res["gpu_s"] = e0.elapsed_time(e1) / 1e3
        res["wall_s"] = time.perf_counter() - t0
        res["mlups"] = res["nodes"] * steps / res["gpu_s"] / 1e6 if res["diverged_at"] is None else None
        if res["diverged_at"] is None:
            lat.synchronize()
            m = lat.stats(coarsen=scale)
            d = spec["diameter"] / scale
            cx, cy = spec["nx"] / scale / 2 - 0.5, spec["ny"] / scale / 2 - 0.5
            res["stats"] = jetstats.jet_statistics(m["w"], m["phi"], cx, cy, d, spec["w_in"])
            res["samples_averaged"] = m["count"]
        if closure is not None:
            lattice_attach(lat, None)
    return res


def a_priori(closure: Closure, F: np.ndarray, t: np.ndarray, a: np.ndarray) -> dict:
    """Weighted squared error of the network's dtau on held-out samples
    against the method without it (dtau = 0) and the best constant."""
    y = closure.forward(F).astype(np.float64)
    w = a.astype(np.float64)
    t = t.astype(np.float64)
    l_net = float(np.sum(w * (y - t) ** 2) / np.sum(w))
    l_zero = float(np.sum(w * t ** 2) / np.sum(w))
    c = float(np.clip(np.sum(w * t) / np.sum(w), 0.0, None))
    l_const = float(np.sum(w * (c - t) ** 2) / np.sum(w))
    return dict(loss_net=l_net, loss_plain=l_zero, loss_const=l_const, gain_vs_plain=1.0 - l_net / l_zero,
                gain_vs_const=1.0 - l_net / l_const, mean_dtau=float(np.sum(w * y) / np.sum(w)),
                mean_target=float(np.sum(w * t) / np.sum(w)))


def _strip(r: dict) -> dict:
    out = {k: v for k, v in r.items() if k != "stats"}
    if "stats" in r:
        s = r["stats"]
        out["stats"] = {k: s[k] for k in ("spreading_rate", "decay_rate", "mixing_thickness", "centreline_mean")}
        out["profiles"] = {k: np.asarray(s[k]).round(6).tolist() for k in ("wc", "r_half", "delta")}
    return out


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=None)
    ap.add_argument("--shrink", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16000, help="coarse steps per run")
    ap.add_argument("--avg-from", type=int, default=8000)
    ap.add_argument("--sample-every", type=int, default=10)
    ap.add_argument("--snap-every", type=int, default=1000)
    ap.add_argument("--keep-every", type=int, default=6)
    ap.add_argument("--train-seeds", type=int, nargs="*", default=[101, 102])
    ap.add_argument("--judge-seed", type=int, default=13)
    ap.add_argument("--train-steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--dtau-max", type=float, default=0.02)
    ap.add_argument("--intervals", type=int, nargs="*", default=[1, 2],
                    help="closure refresh intervals of the coarse + closure runs")
    args = ap.parse_args(argv)
    K = args.shrink
    over = {}
    if K > 1:
        J = workloads.JET
        over = dict(nx=J["nx"] // K, ny=J["ny"] // K, nz=J["nz"] // K, diameter=J["diameter"] / K)
    T, A, S = args.steps // K, args.avg_from // K, args.sample_every
    snaps = [2 * s for s in range(A, T + 1, max(args.snap_every // K, 1))][1:]
    _, _, cs = workloads.jet(1, **over)
    _, _, fs = workloads.jet(2, **over)
    pi_scale = 2.0 * cs["tau"] / fs["tau"]
    result = dict(config=dict(vars(args)), pi_scale=pi_scale, coarse=dict(cs), fine=dict(fs))

    closure = Closure()
    closure.set_params(init_params(0), np.zeros(10), np.ones(10), args.dtau_max)
    # 1. training data from fine plain runs
    train_runs = []
    for seed in args.train_seeds:
        r = run_jet(2, seed, 2 * T, 2 * A, 2 * S, over, dataset=closure, snaps=snaps, keep_every=args.keep_every,
                    pi_scale=pi_scale)
        train_runs.append(_strip(r))
        print(f"fine training run seed {seed}: {r['gpu_s']:.1f} s GPU, {r['samples']} samples", flush=True)
    result["train_runs"] = train_runs
    result["dataset_size"] = closure.dataset_size
    # 2. training
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    closure.normalize()
    hist = closure.train(args.train_steps, batch=args.batch, lr=args.lr, seed=7)
    train_s = time.perf_counter() - t0
    result["training"] = dict(gpu_s=train_s, steps=args.train_steps, batch=args.batch,
                              loss_first=float(hist[:20].mean()), loss_last=float(hist[-20:].mean()),
                              loss_curve=hist[:: max(1, len(hist) // 50)].round(9).tolist())
    print(f"training: {train_s:.1f} s, loss {hist[:20].mean():.3e} -> {hist[-20:].mean():.3e}", flush=True)
    # 3. judge: fine plain with a held-out seed; its snapshots test the network a priori
    ev = Closure()
    judge = run_jet(2, args.judge_seed, 2 * T, 2 * A, 2 * S, over, dataset=ev, snaps=snaps[-3:],
                    keep_every=4 * args.keep_every, pi_scale=pi_scale)
    F, t, a = ev.dataset()
    ev.close()
    result["a_priori"] = a_priori(closure, F, t, a)
    result["judge"] = _strip(judge)
    print(f"judge fine run: {judge['gpu_s']:.1f} s GPU; a priori {result['a_priori']}", flush=True)
    # 4. coarse runs
    runs = {"coarse_plain": run_jet(1, args.judge_seed, T, A, S, over)}
    for k in args.intervals:
        runs[f"coarse_closure_i{k}"] = run_jet(1, args.judge_seed, T, A, S, over, closure=closure, interval=k)
    for name, r in runs.items():
        result[name] = _strip(r)
        if "stats" in judge and "stats" in r:
            result[name]["vs_fine"] = jetstats.compare(r["stats"], judge["stats"])
        result[name]["gpu_time_ratio_fine_over_this"] = judge["gpu_s"] / r["gpu_s"]
    closure.close()
    print(json.dumps(result["a_priori"], indent=1))
    for name in runs:
        print(name, result[name].get("stats"), result[name].get("vs_fine"), f"{result[name]['gpu_s']:.2f} s", flush=True)
    print("judge", result["judge"].get("stats"), f"{result['judge']['gpu_s']:.2f} s")
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(result, fh, indent=1)
    return result


if __name__ == "__main__":
    main()
