"""Lattices driven from several host threads at once.

Each context owns its stream and state, and the library's shared pieces (the
per-device memory pool, the per-kernel shared-memory attributes, the error
strings of failed creations) are guarded, so lattices stepped concurrently by
different threads give the results they give one at a time.  ctypes releases
the interpreter lock during every library call, so the threads really overlap.
"""
import threading

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu


def cases():
    """(name, params, fields): different modes and storage types, so that the
    threads launch different step-kernel instantiations for the first time."""
    out = []
    p, f = workloads.droplet(n=24, radius=6.0)
    out.append(("colour fp32", p, f))
    p, f = workloads.droplet(n=24, radius=6.0)
    p.precision = capi.PREC_BF16
    out.append(("colour bf16", p, f))
    p, f = workloads.droplet(n=32, radius=7.0)
    p.precision = capi.PREC_FP16S
    out.append(("colour fp16s", p, f))
    n = 20
    p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.01, sharp_c=0.9)
    f = workloads.empty_fields(n, n, n)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((x - 9.5) ** 2 + (y - 9.5) ** 2 + (z - 9.5) ** 2)
    f["phi"][:] = 0.5 * (1 + np.tanh((5 - r) / 1.5))
    out.append(("phase field", p, f))
    return out


def run_case(p, f, steps):
    nz, ny, nx = f["rho"].shape
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        lat.step(steps)
        red = lat.reduce()
        return lat.download(), red


def test_concurrent_lattices_match_sequential():
    cs = cases()
    ref = [run_case(p, f, 40) for _, p, f in cs]
    got = [None] * len(cs)
    errors = []

    def worker(i):
        try:
            for _ in range(2):   # create, step, destroy twice: pool reuse under concurrency
                got[i] = run_case(cs[i][1], cs[i][2], 40)
        except Exception as e:   # reported below, with the case name
            errors.append((cs[i][0], repr(e)))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(cs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a worker thread did not finish"
    assert not errors, errors
    for (name, _, _), (st_ref, red_ref), (st, red) in zip(cs, ref, got):
        for k in capi.FIELDS:
            assert np.array_equal(st[k], st_ref[k]), (name, k)
        assert red == red_ref, name


def test_concurrent_create_destroy():
    """Creation and destruction from several threads, lattices of several
    sizes: every lattice starts from its own upload."""
    p, f = workloads.droplet(n=24, radius=6.0)
    errors = []

    def worker(seed):
        rng = np.random.default_rng(seed)
        try:
            for _ in range(6):
                n = int(rng.choice([16, 24, 32]))
                pp, ff = workloads.droplet(n=n, radius=n / 4)
                with Lattice(pp, n, n, n) as lat:
                    lat.upload_moments(ff)
                    lat.step(2)
                    red = lat.reduce()
                    assert abs(red["mass"] - ff["rho"].astype(np.float64).sum()) < 1e-3 * n ** 3
        except Exception as e:
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
