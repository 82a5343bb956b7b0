"""The jet statistics of the closure study recover the known parameters of
an analytic self-similar round jet (CPU only)."""
import numpy as np

from entropicthreadsafe_b200 import jetstats


def analytic_jet(S=0.09, B=5.5, D=16.0, w_in=0.08, width=1.5, nx=160, nz=400, zv=-8.0):
    """Mean fields of a self-similar jet: w = w_c(z) exp(-ln2 (r / r_half)^2) with
    r_half = S (z - zv) and w_c = w_in B D / (z - zv); phi = tanh((r_half - r) / width)."""
    cx = cy = nx / 2 - 0.5
    z = np.arange(nz) + 0.5
    y, x = np.meshgrid(np.arange(nx), np.arange(nx), indexing="ij")
    r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    rh = S * (z - zv)
    wc = w_in * B * D / (z - zv)
    w = wc[:, None, None] * np.exp(-np.log(2.0) * (r[None] / rh[:, None, None]) ** 2)
    phi = np.tanh((rh[:, None, None] - r[None]) / width)
    return w, phi, cx, cy, dict(S=S, B=B, D=D, w_in=w_in, width=width)


def test_recovers_spreading_decay_and_mixing():
    w, phi, cx, cy, p = analytic_jet()
    st = jetstats.jet_statistics(w, phi, cx, cy, p["D"], p["w_in"])
    assert abs(st["spreading_rate"] - p["S"]) <= 0.03 * p["S"], st["spreading_rate"]
    # w_in / w_c = (z - zv) / (B D): slope 1 / B per diameter
    assert abs(st["decay_rate"] - 1.0 / p["B"]) <= 0.02 / p["B"], st["decay_rate"]
    # the integral of 1 - tanh^2 over r is 2 * width (unit-wide bins)
    assert abs(st["mixing_thickness"] - 2.0 * p["width"]) <= 0.05 * 2.0 * p["width"], st["mixing_thickness"]
    z0, z1 = st["window"]
    sel = (st["z"] >= z0) & (st["z"] <= z1)
    rh = p["S"] * (st["z"][sel] + 8.0)
    assert np.nanmax(np.abs(st["r_half"][sel] - rh) / rh) < 0.05


def test_compare_against_itself_and_a_scaled_jet():
    w, phi, cx, cy, p = analytic_jet()
    ref = jetstats.jet_statistics(w, phi, cx, cy, p["D"], p["w_in"])
    same = jetstats.compare(ref, ref)
    assert all(v == 0.0 for v in same.values()), same
    # a jet with 10% weaker velocities everywhere: same spreading, centreline 10% lower
    st = jetstats.jet_statistics(0.9 * w, phi, cx, cy, p["D"], p["w_in"])
    d = jetstats.compare(st, ref)
    assert abs(d["centreline_mean"] - 0.1) < 1e-6
    assert d["spreading_rate"] < 1e-6 and d["mixing_thickness"] < 1e-12
    assert abs(d["decay_rate"] - 1.0 / 9.0) < 1e-6   # w_in / w_c grows by 1 / 0.9


def test_no_jet_gives_nan_statistics():
    w = np.zeros((100, 64, 64))
    phi = -np.ones_like(w)
    st = jetstats.jet_statistics(w, phi, 31.5, 31.5, 16.0, 0.08)
    assert np.isnan(st["spreading_rate"]) and np.isnan(st["decay_rate"])
