"""CPU checks of the closure oracle (oracle/closure_oracle.py): its BF16
rounding against torch's, its backward pass against finite differences of
its own forward pass, its fine-to-coarse samples against a per-node loop,
and the C-ABI's argument checks that need no GPU."""
import numpy as np
import pytest

from oracle import closure_oracle as co


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-4, 5000), rng.uniform(-300, 300, 5000)]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    assert np.array_equal(co.bf16(x), ref)


def random_net(seed, dtau_max=0.02):
    rng = np.random.default_rng(seed)
    p = np.zeros(co.NPARAM)
    w1 = np.zeros((co.NH, 16))
    w1[:, :co.NFEAT] = rng.normal(0, 0.5, (co.NH, co.NFEAT))
    p[co.OFF["W1"]:co.OFF["b1"]] = w1.reshape(-1)
    p[co.OFF["b1"]:co.OFF["W2"]] = rng.normal(0, 0.1, co.NH)
    p[co.OFF["W2"]:co.OFF["b2"]] = rng.normal(0, 0.2, co.NH * co.NH)
    p[co.OFF["b2"]:co.OFF["w3"]] = rng.normal(0, 0.1, co.NH)
    p[co.OFF["w3"]:co.OFF["b3"]] = rng.normal(0, 0.3, co.NH)
    p[co.OFF["b3"]] = -1.0
    mu = rng.normal(0, 1e-3, co.NFEAT)
    sd = rng.uniform(5e-4, 2e-3, co.NFEAT)
    F = mu + sd * rng.normal(0, 1, (300, co.NFEAT))
    t = rng.uniform(0, dtau_max, 300)
    a = rng.uniform(0.1, 2.0, 300)
    return p, mu, sd, dtau_max, F, t, a


@pytest.mark.parametrize("lo", [0.0, -0.008])
def test_oracle_backward_matches_finite_differences(lo):
    """With and without a negative lower bound of the output (dtau_min)."""
    p, mu, sd, dm, F, t, a = random_net(7)
    t = t + lo / 2
    _, g = co.loss_and_grad(p, mu, sd, dm, F, t, a, emulate=False, dtau_min=lo)
    rng = np.random.default_rng(1)
    # every block of the parameter vector, a few entries each (W1 padding excluded)
    picks = []
    for name, b0, b1 in (("W1", 0, 1024), ("b1", 1024, 1088), ("W2", 1088, 5184), ("b2", 5184, 5248),
                         ("w3", 5248, 5312), ("b3", 5312, 5313)):
        cand = [i for i in range(b0, b1) if not (name == "W1" and i % 16 >= co.NFEAT)]
        picks += list(rng.choice(cand, size=min(6, len(cand)), replace=False))
    for i in picks:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = co.loss_and_grad(pp, mu, sd, dm, F, t, a, emulate=False, dtau_min=lo)
        lm, _ = co.loss_and_grad(pm, mu, sd, dm, F, t, a, emulate=False, dtau_min=lo)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(abs(fd), 1e-9) + 1e-12, (i, fd, g[i])
    assert np.all(g[0:1024].reshape(64, 16)[:, co.NFEAT:] == 0.0)


def test_emulated_gradient_is_close_to_exact():
    p, mu, sd, dm, F, t, a = random_net(11)
    le, ge = co.loss_and_grad(p, mu, sd, dm, F, t, a, emulate=True)
    lx, gx = co.loss_and_grad(p, mu, sd, dm, F, t, a, emulate=False)
    # BF16 operands move the gradient by O(2^-8) relative
    assert abs(le - lx) <= 0.02 * lx
    assert np.linalg.norm(ge - gx) <= 0.05 * np.linalg.norm(gx)


def test_fine_samples_match_a_per_node_loop():
    rng = np.random.default_rng(5)
    nz, ny, nx = 8, 6, 10
    names = ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "phi")
    f = {k: rng.normal(0, 0.01, (nz, ny, nx)) for k in names}
    f["phi"] = np.tanh(rng.normal(0, 1, (nz, ny, nx)))
    feat, tgt, wgt = co.fine_samples(f, 1.7, (True, True, False))
    cz, cy, cx = nz // 2, ny // 2, nx // 2

    def m(a, X, Y, Z):
        return a[2 * Z:2 * Z + 2, 2 * Y:2 * Y + 2, 2 * X:2 * X + 2].mean()

    for Z in range(cz):
        for Y in range(cy):
            for X in range(cx):
                J = X + cx * (Y + cy * Z)
                xp, xm = (X + 1) % cx, (X - 1) % cx
                yp, ym = (Y + 1) % cy, (Y - 1) % cy
                zp, zm = min(Z + 1, cz - 1), max(Z - 1, 0)
                vel = ("u", "v", "w")
                G = np.array([[0.5 * (m(f[vel[b]], xp, Y, Z) - m(f[vel[b]], xm, Y, Z)) for b in range(3)],
                              [0.5 * (m(f[vel[b]], X, yp, Z) - m(f[vel[b]], X, ym, Z)) for b in range(3)],
                              [0.5 * (m(f[vel[b]], X, Y, zp) - m(f[vel[b]], X, Y, zm)) for b in range(3)]])
                S = 0.5 * (G + G.T)
                ub = np.array([m(f[c], X, Y, Z) for c in vel])
                uu = np.array([[m(f[vel[a]] * f[vel[b]], X, Y, Z) for b in range(3)] for a in range(3)])
                T = uu - np.outer(ub, ub)
                T -= np.trace(T) / 3 * np.eye(3)
                SS = float(np.sum(S * S))
                edge = Z in (0, cz - 1)
                want_t = 0.0 if edge else -3 * float(np.sum(T * S)) / (2 * SS)
                want_w = 0.0 if edge else SS
                assert abs(tgt[J] - want_t) <= 1e-9 * max(1.0, abs(want_t)), (X, Y, Z)
                assert abs(wgt[J] - want_w) <= 1e-12 * max(1.0, want_w)
                P = [1.7 * m(f[k], X, Y, Z) for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz")]
                assert np.allclose(feat[J, :6], P, rtol=1e-12, atol=0)
                assert abs(feat[J, 8] - np.linalg.norm(ub)) <= 1e-12
