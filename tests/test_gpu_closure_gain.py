"""What the trained closure gains over the method without it, on the
learned-closure jet: the coarse 192 x 192 x 384 jet run plain and with the
trained network attached (closure.trained_closure(): the network at gain 1
with its calibrated lower bound dtau_min), on two inlet-noise seeds that
neither the training (fine seeds 101-103) nor the calibration and its check
(coarse seeds 101-106) saw, each
compared with the fine-grid plain reference (384 x 384 x 768, seeds
101-103, the yardstick of the method) stored with the package
(data/closure_jet_fine_reference.json, written by
`closure_study --reference-only`).

The closure must bring the jet spreading rate and the centreline decay
rate closer to the fine grid than the plain coarse runs do, and the mean
relative error of the four statistics (spreading, decay, mixing thickness,
centreline velocity) down by at least half, at a GPU time still at least 5x
below the fine grid's.  About 80 s of GPU time.
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_trained_closure_beats_the_plain_coarse_jet():
    from entropicthreadsafe_b200 import closure_study
    r = closure_study.gain_check([107, 108])
    p, c = r["plain"]["vs_fine"], r["closure"]["vs_fine"]
    print("plain", {k: f"{v:.3f}" for k, v in p.items()})
    print("closure", {k: f"{v:.3f}" for k, v in c.items()})
    print("fine seed spread", r["fine_spread"], "GPU s: fine", r["fine_gpu_s"], "plain", r["plain"]["gpu_s"],
          "closure", r["closure"]["gpu_s"])
    assert all(d is None for d in r["plain"]["diverged"] + r["closure"]["diverged"])
    for k in ("spreading_rate", "decay_rate"):
        assert np.isfinite(c[k]) and c[k] < p[k], (k, c[k], p[k])
    assert r["closure"]["score"] <= 0.5 * r["plain"]["score"], (r["closure"]["score"], r["plain"]["score"])
    assert r["fine_gpu_s"] / r["closure"]["gpu_s"] >= 5.0
