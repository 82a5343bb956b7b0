"""Learned-closure study on the round jet (coarse + closure vs coarse plain
vs fine plain).

    python -m entropicthreadsafe_b200.closure_study [--out result.json] [--shrink K]
    python -m entropicthreadsafe_b200.closure_study --reference-only --out reference.json

1. Fine plain runs (384 x 384 x 768, three inlet-noise seeds) are the
   reference: their time-averaged fields, averaged over the seeds, give the
   reference jet statistics, and the spread over the seeds is the noise
   floor of one realisation.  Snapshots of two of them, box-filtered onto
   the coarse grid (tslb_closure_dataset_add_fine), are the training set;
   snapshots of the third test the network a priori.
2. The network is trained on the GPU (tslb_closure_train).
3. Coarse plain and coarse + closure runs (192 x 192 x 384, three seeds)
   are compared, as seed averages, with the fine average on spreading
   rate, centreline decay and mixing thickness.  The closure runs are
   repeated with the network's output scaled by a few global gains (an a
   posteriori calibration, as LES calibrates a Smagorinsky constant); the
   best gain on these seeds is then checked on three fresh seeds.  GPU time
   (CUDA events on each lattice's stream) is reported for every run.

Times are in coarse steps; the fine grid runs twice as many steps
(acoustic scaling).  --shrink K divides the lattice sizes and the jet
diameter by K and the step counts by K (a quick check of the pipeline;
the physics of a shrunk jet is not the configuration's).

--reference-only runs step 1 alone and writes the fine reference (seed
mean and spread of the statistics, and the mean profiles) that
gain_check() compares coarse runs with: the file shipped as
data/closure_jet_fine_reference.json.
"""
from __future__ import annotations

import argparse
import json
import os
import time
import warnings

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
            check_every: int = 500, sponge=(0.15, 0.3), z_lo: int = 0) -> dict:
    """One jet run; returns its statistics (coarse units), GPU time and state.

    Training samples (dataset) are taken from coarse plane z_lo on (past the
    inlet's top-hat edge) and outside the sponge layer, whose added
    viscosity the fine stresses carry."""
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
                    res["samples"] += dataset.dataset_add_fine(lat, pi_scale, keep_every, (z_lo, z_hi))
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


def _mean_stats(runs) -> dict | None:
    """Seed average of the runs' statistics and profiles; 'spread' is the
    standard deviation over the seeds relative to the mean."""
    keys = ("spreading_rate", "decay_rate", "mixing_thickness", "centreline_mean")
    ok = [r["stats"] for r in runs if "stats" in r]
    if not ok:
        return None
    out = {k: float(np.mean([s[k] for s in ok])) for k in keys}
    out["spread"] = {k: float(np.std([s[k] for s in ok]) / abs(out[k])) if len(ok) > 1 else 0.0 for k in keys}
    for k in ("wc", "r_half", "delta"):
        # planes where no run has a value (the half width beyond the jet) stay NaN
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", category=RuntimeWarning)
            out[k] = np.nanmean(np.stack([np.asarray(s[k], float) for s in ok]), axis=0)
    out["z"] = ok[0]["z"]
    out["window"] = ok[0]["window"]
    return out


SCALARS = ("spreading_rate", "decay_rate", "mixing_thickness", "centreline_mean")


def _summary(runs, ref) -> dict:
    ms = _mean_stats(runs)
    entry = dict(gpu_s=float(np.mean([r["gpu_s"] for r in runs])), diverged=[r["diverged_at"] for r in runs])
    if ms is not None:
        entry["mean"] = {k: ms[k] for k in SCALARS}
        entry["spread"] = ms["spread"]
        if ref is not None:
            entry["vs_fine"] = jetstats.compare(ms, ref)
            entry["score"] = float(np.mean([entry["vs_fine"][k] for k in SCALARS]))
    return entry


REFERENCE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "closure_jet_fine_reference.json")


def save_reference(ref: dict, fine_runs, path: str) -> None:
    """The fine reference as JSON: scalars, seed spread, profiles, window."""
    out = {k: ref[k] for k in SCALARS}
    out["spread"] = ref["spread"]
    out["window"] = [float(v) for v in ref["window"]]
    for k in ("z", "wc", "r_half", "delta"):
        out[k] = [None if not np.isfinite(v) else float(v) for v in np.asarray(ref[k], float)]
    out["seeds"] = [r["seed"] for r in fine_runs]
    out["gpu_s"] = float(np.mean([r["gpu_s"] for r in fine_runs]))
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)


def load_reference(path: str = REFERENCE) -> dict:
    with open(path) as fh:
        d = json.load(fh)
    for k in ("z", "wc", "r_half", "delta"):
        d[k] = np.array([np.nan if v is None else v for v in d[k]], float)
    return d


def gain_check(seeds, steps: int = 20000, avg_from: int = 8000, sample_every: int = 10, interval: int = 2,
               ref: dict | None = None) -> dict:
    """Coarse plain and coarse + the trained closure (closure.trained_closure,
    its calibrated gain and lower bound included) on the given inlet-noise seeds, against
    the stored fine reference: the seed means' relative errors of the four
    statistics and the profiles, and the GPU time of each form."""
    from .closure import trained_closure
    ref = load_reference() if ref is None else ref
    plain = [run_jet(1, sd, steps, avg_from, sample_every, {}) for sd in seeds]
    clo = trained_closure()
    try:
        closed = [run_jet(1, sd, steps, avg_from, sample_every, {}, closure=clo, interval=interval) for sd in seeds]
    finally:
        clo.close()
    return dict(seeds=list(seeds), plain=_summary(plain, ref), closure=_summary(closed, ref),
                fine_spread=ref["spread"], fine_gpu_s=ref["gpu_s"])


def calibrate(seeds, settings, steps: int = 20000, avg_from: int = 8000, sample_every: int = 10, interval: int = 2,
              ref: dict | None = None) -> dict:
    """Coarse runs with the packaged network (closure.load_trained) at each
    (gain, dtau_min) setting: dtau = dtau_min + (gain dtau_max - dtau_min)
    sigmoid(o).  A tiny gain with a negative dtau_min is the uniform
    viscosity change alone, the control for what the network adds."""
    from .closure import load_trained
    t = load_trained()
    ref = load_reference() if ref is None else ref
    out = {}
    c = Closure()
    try:
        for gain, lo in settings:
            c.set_params(t["params"], t["mu"], t["sd"], float(t["dtau_max"]) * float(gain))
            c.set_dtau_min(float(lo))
            runs = [run_jet(1, sd, steps, avg_from, sample_every, {}, closure=c, interval=interval) for sd in seeds]
            e = _summary(runs, ref)
            out[f"gain {gain} dtau_min {lo}"] = e
            print(f"gain {gain}, dtau_min {lo}:", {k: round(v, 4) for k, v in e.get("vs_fine", {}).items()},
                  {k: round(v, 5) for k, v in e.get("mean", {}).items()}, flush=True)
    finally:
        c.close()
    return out


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=None)
    ap.add_argument("--shrink", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000, help="coarse steps per run")
    ap.add_argument("--avg-from", type=int, default=8000)
    ap.add_argument("--sample-every", type=int, default=10)
    ap.add_argument("--snap-every", type=int, default=1000)
    ap.add_argument("--keep-every", type=int, default=6)
    ap.add_argument("--fine-seeds", type=int, nargs="*", default=[101, 102, 103])
    ap.add_argument("--train-seeds", type=int, nargs="*", default=[101, 102],
                    help="fine seeds whose snapshots train the network; the others test it a priori")
    ap.add_argument("--coarse-seeds", type=int, nargs="*", default=[101, 102, 103],
                    help="coarse seeds of the comparison and of the gain calibration")
    ap.add_argument("--check-seeds", type=int, nargs="*", default=[104, 105, 106],
                    help="fresh coarse seeds that check the calibrated gain")
    ap.add_argument("--z-lo", type=int, default=4, help="first coarse plane of the training samples")
    ap.add_argument("--train-steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--dtau-max", type=float, default=0.02)
    ap.add_argument("--interval", type=int, default=2, help="closure refresh interval of the coarse runs")
    ap.add_argument("--gains", type=float, nargs="*", default=[1.0, 2.0, 4.0, 8.0],
                    help="output gains of the a posteriori calibration")
    ap.add_argument("--reference-only", action="store_true",
                    help="only the fine runs: write their reference statistics to --out")
    ap.add_argument("--calibrate", nargs="*", default=None, metavar="GAIN:DTAU_MIN",
                    help="only coarse runs of the packaged network at these settings on --coarse-seeds")
    args = ap.parse_args(argv)
    if args.calibrate is not None:
        settings = [tuple(float(v) for v in c.split(":")) for c in args.calibrate]
        r = calibrate(args.coarse_seeds, settings, args.steps, args.avg_from, args.sample_every, args.interval)
        if args.out:
            with open(args.out, "w") as fh:
                json.dump(r, fh, indent=1, default=float)
        return r
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
    held = Closure()
    # 1. fine plain runs: training snapshots, held-out snapshots, reference statistics
    fine_runs = []
    for seed in args.fine_seeds:
        train = seed in args.train_seeds
        keep = None if args.reference_only else (closure if train else held)
        r = run_jet(2, seed, 2 * T, 2 * A, 2 * S, over, dataset=keep,
                    snaps=snaps if train else snaps[-3:],
                    keep_every=args.keep_every if train else 4 * args.keep_every, pi_scale=pi_scale,
                    z_lo=args.z_lo // K)
        fine_runs.append(r)
        print(f"fine run seed {seed} ({'training' if train else 'held out'}): {r['gpu_s']:.1f} s GPU, "
              f"{r['samples']} samples, diverged {r['diverged_at']}", flush=True)
    ref = _mean_stats(fine_runs)
    if args.reference_only:
        if args.out and ref is not None:
            save_reference(ref, fine_runs, args.out)
        print("fine mean:", {k: ref[k] for k in SCALARS} if ref else None, "spread", ref["spread"] if ref else None)
        return dict(reference={k: ref[k] for k in SCALARS} if ref else None, fine_runs=[_strip(r) for r in fine_runs])
    result["fine_runs"] = [_strip(r) for r in fine_runs]
    result["fine"]["mean"] = {k: ref[k] for k in SCALARS} if ref else None
    result["fine"]["spread"] = ref["spread"] if ref else None
    result["fine"]["gpu_s"] = float(np.mean([r["gpu_s"] for r in fine_runs]))
    result["dataset_size"] = closure.dataset_size
    # 2. training
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    closure.normalize()
    hist = closure.train(args.train_steps, batch=args.batch, lr=args.lr, seed=7)
    train_s = time.perf_counter() - t0
    result["training"] = dict(seconds=train_s, steps=args.train_steps, batch=args.batch,
                              loss_first=float(hist[:50].mean()), loss_last=float(hist[-50:].mean()),
                              loss_curve=hist[:: max(1, len(hist) // 50)].round(12).tolist())
    prm = closure.get_params()
    net = {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in prm.items()}
    result["network"] = net
    print(f"training: {train_s:.2f} s, loss {hist[:50].mean():.3e} -> {hist[-50:].mean():.3e}", flush=True)
    if held.dataset_size:
        F, t, a = held.dataset()
        result["a_priori_held_out"] = a_priori(closure, F, t, a)
        print("a priori (held-out fine seed):", result["a_priori_held_out"], flush=True)
    held.close()
    # 3. coarse plain, and coarse + closure at each gain, on the calibration seeds
    plain = [run_jet(1, sd, T, A, S, over) for sd in args.coarse_seeds]
    result["coarse_plain"] = _summary(plain, ref)
    result["coarse_plain"]["runs"] = [_strip(r) for r in plain]
    print("coarse plain:", result["coarse_plain"].get("vs_fine"), f"{result['coarse_plain']['gpu_s']:.1f} s", flush=True)

    def with_gain(seeds, gain):
        closure.set_params(np.asarray(net["params"], np.float32), np.asarray(net["mu"], np.float32),
                           np.asarray(net["sd"], np.float32), net["dtau_max"] * gain)
        return [run_jet(1, sd, T, A, S, over, closure=closure, interval=args.interval) for sd in seeds]

    result["coarse_closure"] = {}
    for g in args.gains:
        rs = with_gain(args.coarse_seeds, g)
        e = _summary(rs, ref)
        e["runs"] = [_strip(r) for r in rs]
        result["coarse_closure"][str(g)] = e
        print(f"coarse + closure, gain {g}:", e.get("vs_fine"), f"{e['gpu_s']:.1f} s", flush=True)
    # 4. the best gain on the calibration seeds, checked on fresh seeds
    scored = {g: e["score"] for g, e in result["coarse_closure"].items() if "score" in e}
    if scored and args.check_seeds:
        best = min(scored, key=scored.get)
        result["best_gain"] = float(best)
        cp = [run_jet(1, sd, T, A, S, over) for sd in args.check_seeds]
        cc = with_gain(args.check_seeds, float(best))
        result["check"] = dict(seeds=args.check_seeds, gain=float(best), plain=_summary(cp, ref),
                               closure=_summary(cc, ref))
        print("check seeds: plain", result["check"]["plain"].get("vs_fine"), "\n closure",
              result["check"]["closure"].get("vs_fine"), flush=True)
    result["gpu_time_ratio_fine_over_plain"] = result["fine"]["gpu_s"] / result["coarse_plain"]["gpu_s"]
    result["gpu_time_ratio_fine_over_closure"] = result["fine"]["gpu_s"] / np.mean(
        [e["gpu_s"] for e in result["coarse_closure"].values()])
    print("fine mean:", result["fine"]["mean"], "spread", result["fine"]["spread"], flush=True)
    closure.close()
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(result, fh, indent=1, default=float)
    return result


if __name__ == "__main__":
    main()
