"""Analysis functions of the precision study (CPU only)."""
import numpy as np

from entropicthreadsafe_b200 import precision_study as ps


def test_spectrum_of_a_single_mode():
    nz, ny, nx = 8, 4, 64
    x = np.arange(nx)
    u = np.broadcast_to(0.1 + 0.02 * np.sin(2 * np.pi * 5 * x / nx), (nz, ny, nx)).copy()
    z = np.zeros_like(u)
    e = ps.spectrum_x(u, z, z, (2, 6))
    assert e.shape == (nx // 2 + 1,)
    assert np.argmax(e) == 5 and e[0] < 1e-20            # the mean is removed
    # |FFT / nx|^2 of a sine of amplitude A at one positive k is (A/2)^2
    assert abs(e[5] - 0.01 ** 2) < 1e-12
    assert e.sum() - e[5] < 1e-20


def test_mean_profile_and_compare():
    nz, ny, nx = 16, 4, 32
    zz = np.arange(nz)[:, None, None] + np.zeros((1, ny, nx))
    u = 0.05 * zz * (nz - 1 - zz) / ((nz - 1) / 2) ** 2
    prof = ps.mean_profile(u)
    assert np.allclose(prof, u[:, 0, 0])
    rng = np.random.default_rng(1)
    v = rng.normal(0, 1e-3, u.shape)
    spec = ps.spectrum_x(u + v, v, v, (4, 12))
    same = ps.compare(prof, spec, prof, spec)
    assert same["profile_max_rel_err"] == 0 and same["spectrum_mean_abs_dlog10"] == 0
    d = ps.compare(1.01 * prof, 4.0 * spec, prof, spec)
    assert abs(d["profile_max_rel_err"] - 0.01) < 1e-12
    assert abs(d["spectrum_mean_abs_dlog10"] - np.log10(4.0)) < 1e-12
    assert abs(d["fluctuation_energy_rel_diff"] - 3.0) < 1e-12
