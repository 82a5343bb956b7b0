"""GPU checks of the learned closure (include/tslb_closure.h) against the
FP64 closure oracle (oracle/closure_oracle.py) and the step oracle.

- forward pass of the tensor-core kernel vs the oracle with the kernel's
  BF16 rounding points (tolerance in units of dtau_max);
- gradient of the training kernel vs the oracle (BF16-emulating: relative
  L2 error per parameter block <= 2e-3; exact FP64 network: <= 0.1, the
  size of BF16 rounding of activations and back-propagated errors, about
  5% on dW1 for this case);
- lattice features, fine-to-coarse samples and the tau-corrected step vs
  the oracles;
- the stability clamp, determinism of training, and that training fits a
  known eddy-viscosity law.
"""
import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.closure import Closure, init_params, lattice_attach
from entropicthreadsafe_b200.solver import Lattice
from oracle import closure_oracle as co

from helpers import field_errors

pytestmark = pytest.mark.gpu

BLOCKS = (("W1", 0, 1024), ("b1", 1024, 1088), ("W2", 1088, 5184), ("b2", 5184, 5248), ("w3", 5248, 5312),
          ("b3", 5312, 5313))


def random_case(seed, n, dtau_max=0.02):
    rng = np.random.default_rng(seed)
    p = init_params(seed, out_bias=-1.0).astype(np.float64)
    p[1024:1088] = rng.normal(0, 0.2, 64)
    p[5184:5248] = rng.normal(0, 0.2, 64)
    p[5248:5312] = rng.normal(0, 0.5, 64)
    mu = rng.normal(0, 1e-3, co.NFEAT)
    sd = rng.uniform(5e-4, 2e-3, co.NFEAT)
    F = mu + sd * rng.normal(0, 1.5, (n, co.NFEAT))
    t = rng.uniform(0, dtau_max, n)
    a = rng.uniform(0.1, 2.0, n)
    return p.astype(np.float32), mu.astype(np.float32), sd.astype(np.float32), dtau_max, F.astype(np.float32), \
        t.astype(np.float32), a.astype(np.float32)


def closure_with(p, mu, sd, dm):
    c = Closure()
    c.set_params(p, mu, sd, dm)
    return c


def test_forward_matches_oracle():
    p, mu, sd, dm, F, _, _ = random_case(1, 1000)
    with closure_with(p, mu, sd, dm) as c:
        y = c.forward(F)
    ref, _ = co.forward(p, mu, sd, dm, F, emulate=True)
    err = np.abs(y.astype(np.float64) - ref)
    assert np.median(err) <= 1e-5 * dm, np.median(err)
    assert err.max() <= 2e-3 * dm, err.max()
    # the spread of outputs is real (not a constant)
    assert ref.std() > 0.05 * dm


def test_gradient_matches_oracle():
    p, mu, sd, dm, F, t, a = random_case(2, 777)
    with closure_with(p, mu, sd, dm) as c:
        g, loss = c.gradient(F, t, a)
    le, ge = co.loss_and_grad(p, mu, sd, dm, F, t, a, emulate=True)
    lx, gx = co.loss_and_grad(p, mu, sd, dm, F, t, a, emulate=False)
    assert abs(loss - le) <= 1e-4 * le, (loss, le)
    for name, lo, hi in BLOCKS:
        gg, ee, xx = g[lo:hi].astype(np.float64), ge[lo:hi], gx[lo:hi]
        if name == "W1":
            gg, ee, xx = (v.reshape(64, 16)[:, :co.NFEAT] for v in (gg, ee, xx))
            assert np.all(g[lo:hi].reshape(64, 16)[:, co.NFEAT:] == 0)
        e_emu = np.linalg.norm(gg - ee) / np.linalg.norm(ee)
        e_ex = np.linalg.norm(gg - xx) / np.linalg.norm(xx)
        assert e_emu <= 2e-3, (name, e_emu)
        assert e_ex <= 0.1, (name, e_ex)


def test_forward_clamps_non_finite_rows():
    p, mu, sd, dm, F, _, _ = random_case(3, 300)
    F[5, 2] = np.nan
    F[77, 9] = np.inf
    with closure_with(p, mu, sd, dm) as c:
        y = c.forward(F)
    assert y[5] == 0.0 and y[77] == 0.0
    assert np.all(np.isfinite(y)) and np.all((y >= 0) & (y <= dm))


def test_signed_range_matches_oracle():
    """A negative lower bound: dtau = lo + (hi - lo) sigmoid(o), forward and
    gradient against the oracle, outputs inside [lo, hi], non-finite rows
    at 0; attaching checks that tau + lo stays above 1/2."""
    p, mu, sd, dm, F, t, a = random_case(4, 640)
    lo = -0.4 * dm
    t = (t - 0.5 * dm).astype(np.float32)
    F[3, 1] = np.nan
    with closure_with(p, mu, sd, dm) as c:
        c.set_dtau_min(lo)
        assert c.get_params()["dtau_min"] == np.float32(lo)
        y = c.forward(F)
        g, loss = c.gradient(F, t, a)
        lat = Lattice(jet_params(tau=0.5 - lo / 2), 16, 16, 16)
        with pytest.raises(Exception):
            lattice_attach(lat, c)
        lat.close()
    ref, _ = co.forward(p, mu, sd, dm, F, emulate=True, dtau_min=lo)
    # rows with a non-finite feature keep the plain tau in the kernel (the
    # oracle's ReLU would map the NaN to 0): compared apart
    keep = np.isfinite(F).all(axis=1)
    err = np.abs(y[keep].astype(np.float64) - ref[keep])
    assert y[3] == 0.0
    assert np.median(err) <= 1e-5 * (dm - lo) and err.max() <= 2e-3 * (dm - lo), (np.median(err), err.max())
    assert y.min() >= lo and y.max() <= dm and (y < 0).any()
    le, ge = co.loss_and_grad(p, mu, sd, dm, F[keep], t[keep], a[keep], emulate=True, dtau_min=lo)
    with closure_with(p, mu, sd, dm) as c:
        c.set_dtau_min(lo)
        g, loss = c.gradient(F[keep], t[keep], a[keep])
    assert abs(loss - le) <= 1e-4 * le, (loss, le)
    for name, b0, b1 in BLOCKS:
        gg, ee = g[b0:b1].astype(np.float64), ge[b0:b1]
        if name == "W1":
            gg, ee = (v.reshape(64, 16)[:, :co.NFEAT] for v in (gg, ee))
        assert np.linalg.norm(gg - ee) <= 2e-3 * np.linalg.norm(ee), name


def jet_like_state(nx, ny, nz, seed):
    """A colour state with a droplet, random velocity and stress fields."""
    rng = np.random.default_rng(seed)
    f = workloads.empty_fields(nx, ny, nz)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2)
    f["phi"][:] = np.tanh((0.3 * min(nx, ny, nz) - r) / 2.0)
    for k in ("u", "v", "w"):
        f[k][:] = 0.02 * np.sin(2 * np.pi * (x / nx + 2 * y / ny)) + rng.normal(0, 0.003, r.shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 2e-4, r.shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, r.shape)
    return f


def jet_params(nz_faces=(capi.BC_INLET, capi.BC_OUTLET), tau=0.52):
    bc = [capi.BC_PERIODIC] * 4 + list(nz_faces)
    return capi.make_params(mode=capi.MODE_COLOUR, tau_a=tau, tau_b=tau + 0.03, sigma=0.002, beta=0.7, bc=bc,
                            bc_phi=[-1.0] * 6, wall_phi_mode=1)


def inlet_planes(nx, ny, radius=4.0, w=0.05, seed=0):
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    disc = (x - nx / 2 + 0.5) ** 2 + (y - ny / 2 + 0.5) ** 2 <= radius ** 2
    pl = np.zeros((4, ny, nx), np.float32)
    pl[2] = np.where(disc, w * (1 + 0.03 * rng.uniform(-1, 1, disc.shape)), 0.0)
    pl[3] = np.where(disc, 1.0, -1.0)
    return pl


def test_lattice_features_match_oracle():
    nx, ny, nz = 24, 20, 28
    p = jet_params()
    f = jet_like_state(nx, ny, nz, 4)
    dt = np.random.default_rng(9).uniform(0, 0.01, (nz, ny, nx)).astype(np.float32)
    with Lattice(p, nx, ny, nz) as lat, Closure() as c:
        lat.upload_moments(f)
        g0 = c.features(lat)
        lat.set_tau_correction(dt)
        g1 = c.features(lat)
    for dtp, got in ((None, g0), (dt, g1)):
        ref = co.lattice_features({k: v.astype(np.float32) for k, v in f.items()}, p.tau_a, p.tau_b,
                                  (True, True, False), dtp)
        scale = np.abs(ref).max(axis=0) + 1e-30
        err = (np.abs(got.astype(np.float64) - ref) / scale).max()
        assert err <= 2e-6, err


def test_dataset_from_fine_lattice_matches_oracle():
    nx, ny, nz = 24, 20, 32
    p = jet_params()
    f = jet_like_state(nx, ny, nz, 5)
    with Lattice(p, nx, ny, nz) as lat, Closure() as c:
        lat.upload_moments(f)
        n0 = c.dataset_add_fine(lat, 1.9, keep_every=3)
        n1 = c.dataset_add_fine(lat, 1.9, keep_every=3, z_range=(2, 13))
        feat, tgt, wgt = c.dataset()
        assert c.dataset_size == n0 + n1
        c.dataset_clear()
        assert c.dataset_size == 0 and c.dataset()[0].shape[0] == 0
        # a cleared set fills again from the start
        assert c.dataset_add_fine(lat, 1.9, keep_every=3) == n0 and c.dataset_size == n0
    rf, rt, rw = co.fine_samples({k: v.astype(np.float32) for k, v in f.items()}, 1.9, (True, True, False))
    nc = rf.shape[0]
    plane = (nx // 2) * (ny // 2)
    sel = np.concatenate([np.arange(0, nc, 3), np.arange(2 * plane + 1, 13 * plane, 3)])
    assert n0 + n1 == len(sel) == feat.shape[0]
    scale = np.abs(rf).max(axis=0) + 1e-30
    assert (np.abs(feat - rf[sel]) / scale).max() <= 2e-6
    assert np.array_equal(wgt == 0, rw[sel] == 0)
    ok = rw[sel] > 1e-3 * rw.max()
    assert np.abs(wgt[ok] - rw[sel][ok]).max() <= 1e-4 * rw.max()
    assert np.abs(tgt[ok] - rt[sel][ok]).max() <= 1e-3 * np.abs(rt[sel][ok]).max()


def test_tau_correction_step_matches_oracle():
    import oracle
    nx, ny, nz = 24, 20, 28
    p = jet_params()
    f = jet_like_state(nx, ny, nz, 6)
    pl = inlet_planes(nx, ny)
    dt = np.random.default_rng(10).uniform(0, 0.02, (nz, ny, nx)).astype(np.float32)
    with Lattice(p, nx, ny, nz) as lat:
        lat.set_inlet(4, pl)
        lat.upload_moments(f)
        lat.set_tau_correction(dt)
        lat.step(5)
        got = lat.download()
    o = oracle.Oracle(p, nx, ny, nz, fp64=True)
    o.set_inlet(4, pl.astype(np.float64))
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    o.set_tau_correction(dt.astype(np.float64))
    o.step(5)
    ref = o.get_moments()
    o.close()
    errs = field_errors(got, ref)
    assert max(errs.values()) <= 2e-5, errs
    # the correction is not a no-op
    o = oracle.Oracle(p, nx, ny, nz, fp64=True)
    o.set_inlet(4, pl.astype(np.float64))
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    o.step(5)
    plain = o.get_moments()
    o.close()
    assert max(field_errors(plain, ref)[k] for k in ("pxx", "pxy", "u")) > 1e-3


def test_attached_closure_step_matches_oracle():
    """Three steps with the closure attached vs the oracle stepping with the
    closure oracle's dtau of each step's state."""
    import oracle
    nx, ny, nz = 24, 20, 28
    p = jet_params()
    f = jet_like_state(nx, ny, nz, 7)
    pl = inlet_planes(nx, ny)
    net, mu, sd, dm, _, _, _ = random_case(8, 10, dtau_max=0.03)
    # normalisation from the state's own features so the network is in its working range
    feats = co.lattice_features(f, p.tau_a, p.tau_b, (True, True, False))
    mu = feats.mean(0).astype(np.float32)
    sd = (feats.std(0) + 1e-12).astype(np.float32)
    nsteps = 3
    # a static correction (a sponge on the last planes) under the closure's output
    base = np.zeros((nz, ny, nx), np.float32)
    base[-6:] = np.linspace(0.01, 0.1, 6, dtype=np.float32)[:, None, None]
    with Lattice(p, nx, ny, nz) as lat, closure_with(net, mu, sd, dm) as c:
        lat.set_inlet(4, pl)
        lat.upload_moments(f)
        lat.set_tau_correction(base)
        lattice_attach(lat, c, 1)
        lat.step(nsteps)
        got = lat.download()
        dt_gpu = lat.tau_correction()
        lattice_attach(lat, None)
    o = oracle.Oracle(p, nx, ny, nz, fp64=True)
    o.set_inlet(4, pl.astype(np.float64))
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    dtp = base.astype(np.float64)
    for _ in range(nsteps):
        st = o.get_moments()
        y, _ = co.forward(net, mu, sd, dm, co.lattice_features(st, p.tau_a, p.tau_b, (True, True, False), dtp),
                          emulate=True)
        dtp = y.reshape(nz, ny, nx) + base
        o.set_tau_correction(dtp)
        o.step(1)
    ref = o.get_moments()
    o.close()
    assert np.abs(dt_gpu - dtp).max() <= 5e-3 * dm
    assert (dtp - base).std() > 0.02 * dm   # the correction varies in space
    errs = field_errors(got, ref)
    assert max(errs.values()) <= 1e-4, errs


def test_training_fits_a_smagorinsky_law_and_is_deterministic():
    """Targets t = clip(c |Pi|, 0, dtau_max) with noise: the trained network
    explains most of their weighted variance, and the same seed gives the
    same parameters bit for bit."""
    rng = np.random.default_rng(12)
    n = 60000
    F = np.zeros((n, co.NFEAT), np.float32)
    F[:, :6] = rng.normal(0, 1e-3, (n, 6))
    F[:, 6] = rng.uniform(-1, 1, n)
    F[:, 7] = np.abs(rng.normal(0, 0.2, n))
    F[:, 8] = np.abs(rng.normal(0.03, 0.02, n))
    F[:, 9] = np.sqrt(F[:, 0] ** 2 + F[:, 3] ** 2 + F[:, 5] ** 2 + 2 * (F[:, 1] ** 2 + F[:, 2] ** 2 + F[:, 4] ** 2))
    dm = 0.05
    t = np.clip(8.0 * F[:, 9], 0, dm) + rng.normal(0, 0.001, n)
    a = rng.uniform(0.5, 1.5, n).astype(np.float32)
    params = []
    for _ in range(2):
        with Closure() as c:
            c.set_params(init_params(0), np.zeros(co.NFEAT), np.ones(co.NFEAT), dm)
            c.dataset_add(F, t.astype(np.float32), a)
            c.normalize()
            hist = c.train(600, batch=8192, lr=3e-3, seed=5)
            y = c.forward(F)
            params.append(c.get_params()["params"])
    assert np.array_equal(params[0], params[1])
    w = a / a.mean()
    resid = np.sum(w * (y - t) ** 2)
    total = np.sum(w * (t - np.average(t, weights=w)) ** 2)
    assert 1 - resid / total > 0.9, 1 - resid / total
    assert hist[-50:].mean() < 0.1 * hist[:10].mean()
