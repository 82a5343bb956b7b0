"""GPU checks of the jet workload's device parts: the counter-based inlet
drawn on the device equals its host mirror, the device time averages equal
host averages of downloaded states, and the closure study runs end to end
on a shrunk jet."""
import numpy as np
import pytest

from entropicthreadsafe_b200 import workloads
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu


def small_jet():
    return workloads.jet(1, nx=24, ny=20, nz=32, diameter=6.0)


def test_device_inlet_equals_host_mirror():
    p, f, spec = small_jet()
    outs = []
    for device in (True, False):
        with Lattice(p, spec["nx"], spec["ny"], spec["nz"]) as lat:
            lat.upload_moments(f)
            for s in range(25):
                if s % spec["refresh"] == 0:
                    if device:
                        workloads.jet_inlet(lat, spec, 77, s)
                    else:
                        lat.set_inlet(4, workloads.inlet_disc(spec["nx"], spec["ny"], 2, 1.0, spec["cx"], spec["cy"],
                                                              spec["diameter"] / 2, spec["w_in"], spec["noise"], 77,
                                                              s // spec["refresh"]))
                lat.step(1)
            outs.append(lat.download())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k
    assert np.abs(outs[0]["w"]).max() > 0.01


def test_inlet_mirror_statistics():
    pl = workloads.inlet_disc(64, 48, 2, 1.0, 31.5, 23.5, 8.0, 0.08, 0.03, 5, 3)
    disc = pl[3] > 0
    assert abs(disc.sum() - np.pi * 64) < 12
    w = pl[2][disc]
    assert np.all(np.abs(w / 0.08 - 1) <= 0.03 + 1e-7)
    assert abs(w.mean() / 0.08 - 1) < 0.01 and w.std() / 0.08 > 0.01
    assert np.all(pl[2][~disc] == 0) and np.all(pl[3][~disc] == -1) and np.all(pl[:2] == 0)
    other = workloads.inlet_disc(64, 48, 2, 1.0, 31.5, 23.5, 8.0, 0.08, 0.03, 5, 4)
    assert not np.array_equal(other[2], pl[2])


def test_device_time_averages():
    p, f, spec = small_jet()
    with Lattice(p, spec["nx"], spec["ny"], spec["nz"]) as lat:
        lat.upload_moments(f)
        lat.stats_reset()
        acc = {k: 0.0 for k in ("u", "v", "w", "phi", "ww")}
        prods = [("u", "u"), ("u", "v"), ("u", "w"), ("v", "v"), ("v", "w"), ("w", "w")]
        pis = ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz")
        uu, pi = [0.0] * 6, [0.0] * 6
        for s in range(30):
            if s % spec["refresh"] == 0:
                workloads.jet_inlet(lat, spec, 3, s)
            lat.step(1)
            if s % 3 == 0:
                lat.stats_accumulate()
                d = lat.download()
                for k in ("u", "v", "w", "phi"):
                    acc[k] = acc[k] + d[k].astype(np.float64)
                acc["ww"] = acc["ww"] + d["w"].astype(np.float64) ** 2
                for j, (a, b) in enumerate(prods):
                    uu[j] = uu[j] + d[a].astype(np.float64) * d[b]
                for j, k in enumerate(pis):
                    pi[j] = pi[j] + d[k].astype(np.float64)
        m1 = lat.stats(1)
        m2 = lat.stats(2)
        s1 = lat.stats_stress(1)
        s2 = lat.stats_stress(2)
    assert m1["count"] == 10 and s1["count"] == 10
    refs = dict(acc)
    refs.update({f"uu{j}": uu[j] for j in range(6)})
    refs.update({f"pi{j}": pi[j] for j in range(6)})
    got1 = dict(m1)
    got1.update({f"uu{j}": s1["uu"][j] for j in range(6)})
    got1.update({f"pi{j}": s1["pineq"][j] for j in range(6)})
    got2 = dict(m2)
    got2.update({f"uu{j}": s2["uu"][j] for j in range(6)})
    got2.update({f"pi{j}": s2["pineq"][j] for j in range(6)})
    for k in refs:
        ref = refs[k] / 10
        assert np.abs(got1[k] - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1e-3), k
        nz, ny, nx = ref.shape
        blk = ref.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).mean(axis=(1, 3, 5))
        assert np.abs(got2[k] - blk).max() <= 1e-6 * max(np.abs(blk).max(), 1e-3), k


def test_closure_study_runs_on_a_shrunk_jet(tmp_path):
    from entropicthreadsafe_b200 import closure_study
    out = tmp_path / "study.json"
    r = closure_study.main(["--shrink", "8", "--steps", "8000", "--avg-from", "4000", "--snap-every", "800",
                            "--keep-every", "2", "--train-steps", "200", "--batch", "4096", "--fine-seeds", "1", "2",
                            "--train-seeds", "1", "--coarse-seeds", "3", "--check-seeds", "4", "--gains", "1", "2",
                            "--out", str(out)])
    assert out.exists()
    assert r["dataset_size"] > 1000
    # minibatch losses of a tiny shrunk set are noisy; learning itself is
    # tested in test_gpu_closure (Smagorinsky law)
    assert np.isfinite(r["training"]["loss_last"]) and r["training"]["loss_last"] > 0
    assert np.isfinite(r["a_priori_held_out"]["loss_net"])
    for run in r["fine_runs"]:
        assert run["diverged_at"] is None and run["gpu_s"] > 0
        # the averaging window holds the jet: every statistic is a number
        assert all(np.isfinite(run["stats"][k]) for k in closure_study.SCALARS), run["stats"]
    assert all(d is None for d in r["coarse_plain"]["diverged"])
    for g in ("1.0", "2.0"):
        assert all(d is None for d in r["coarse_closure"][g]["diverged"])
        assert "vs_fine" in r["coarse_closure"][g]
    assert r["best_gain"] in (1.0, 2.0) and "vs_fine" in r["check"]["closure"]
