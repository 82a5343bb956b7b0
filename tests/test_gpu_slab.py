"""z slabs on one GPU: a lattice cut into slabs that refresh their halos
every step gives the single lattice's result bit for bit.

Each slab runs in its own host thread and exchanges through
slab.exchange_halos with a mailbox of device buffers standing in for the
NCCL transfers (one GPU: the slabs' kernels never wait on one another; the
threads hand over buffers between launches).  This covers the slab
kernels' own-plane range, the halo pack and unpack kernels and the
message pairing, including two slabs of a periodic axis (both neighbours
the same slab) and the phase-field mode's three halo planes.
"""
import queue
import threading

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.slab import Slab, exchange_halos, partition
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu


def run_slabs(p, f, nslab, nsteps):
    import torch
    nz, ny, nx = f["rho"].shape
    zper = p.bc[capi.FACE_ZM] == capi.BC_PERIODIC
    slabs = [Slab(p, nx, ny, nz, *partition(nz, nslab, r)) for r in range(nslab)]
    for s in slabs:
        s.upload_moments(f)
    boxes = {(src, dst, tag): queue.Queue() for src in range(nslab) for dst in range(nslab) for tag in (0, 1)}
    bufs = [[torch.empty(max(s.halo_bytes, 1), dtype=torch.uint8, device="cuda") for _ in range(2)] for s in slabs]

    def worker(r):
        s = slabs[r]

        def pack(side):
            s.pack(side, bufs[r][side].data_ptr())
            s.synchronize()
            return bufs[r][side].clone()

        def unpack(side, buf):
            s.unpack(side, buf.data_ptr())
            s.synchronize()

        def sendrecv(sends, recvs):
            for buf, peer, tag in sends:
                boxes[(r, peer, tag)].put(buf)
            return [boxes[(peer, r, tag)].get(timeout=60) for _, peer, tag in recvs]

        for _ in range(nsteps):
            s.step(1)
            s.synchronize()
            exchange_halos(r, nslab, zper, pack, unpack, sendrecv)

    threads = [threading.Thread(target=worker, args=(r,)) for r in range(nslab)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    out = {k: np.concatenate([s.download()[k] for s in slabs]) for k in capi.FIELDS}
    red = [s.reduce() for s in slabs]
    for s in slabs:
        s.close()
    return out, red


def run_single(p, f, nsteps):
    nz, ny, nx = f["rho"].shape
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        lat.step(nsteps)
        return lat.download(), lat.reduce()


def assert_same(a, b):
    for k in capi.FIELDS:
        assert np.array_equal(a[k], b[k]), (k, float(np.abs(a[k] - b[k]).max()))


@pytest.mark.parametrize("nslab", [2, 3])
def test_colour_channel_walls(nslab):
    p, f = workloads.channel(nx=64, ny=16, nz=24, ndrops=3, radius=3.0, wall_gap=2.0, gx=2.5e-5)
    a, red = run_slabs(p, f, nslab, 12)
    b, red1 = run_single(p, f, 12)
    assert_same(a, b)
    # the slabs' own-plane diagnostics add up to the lattice's
    assert abs(sum(r["mass"] for r in red) - red1["mass"]) < 1e-6 * red1["mass"]


def test_colour_periodic_two_slabs():
    """Both neighbours of each slab are the same slab."""
    p, f = workloads.droplet(n=32, radius=8.0)
    a, _ = run_slabs(p, f, 2, 12)
    b, _ = run_single(p, f, 12)
    assert_same(a, b)


def test_phasefield_periodic_three_slabs():
    p, f = workloads.droplet(n=32, radius=8.0, mode=capi.MODE_PHASEFIELD)
    a, _ = run_slabs(p, f, 3, 10)
    b, _ = run_single(p, f, 10)
    assert_same(a, b)


def test_single_component_and_bf16_slabs():
    p, f = workloads.channel(nx=64, ny=16, nz=16, ndrops=0, gx=2.5e-5)
    p.mode = capi.MODE_SINGLE
    f["phi"][:] = 1.0
    a, _ = run_slabs(p, f, 2, 8)
    b, _ = run_single(p, f, 8)
    assert_same(a, b)
    p, f = workloads.channel(nx=64, ny=16, nz=16, ndrops=2, radius=3.0, wall_gap=1.0, gx=2.5e-5)
    p.precision = capi.PREC_BF16
    a, _ = run_slabs(p, f, 2, 8)
    b, _ = run_single(p, f, 8)
    assert_same(a, b)
