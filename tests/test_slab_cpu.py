"""z-slab decomposition on CPU: two gloo ranks, each stepping its slab (with
halo planes) on the oracle and refreshing the halos every step through
slab.exchange_halos over torch.distributed point-to-point transfers, give
the single-lattice oracle's result.

The stand-in slab follows the geometry rules of tslb_create_slab (halo
depth H = 2 in colour mode, 3 in phase-field mode; a side with a neighbour
keeps H halo planes and no boundary condition of its own) and packs the
buffer layout tslb_halo_pack documents (the 10 non-phi moments of the edge
plane, then phi of H edge planes).  The cases cover a periodic axis cut in
two (both neighbours are the same rank), walls on the lattice's own z
faces, and the phase-field mode's deeper halo.
"""
import copy
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NSTEPS = 6
HALO = {0: 3, 1: 2, 2: 1}    # by mode: phase field, colour, single component
MOMENTS = ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def workload(case):
    sys.path.insert(0, ROOT)
    from entropicthreadsafe_b200 import capi, workloads
    if case == "colour_periodic":
        return workloads.droplet(n=16, radius=4.0)
    if case == "colour_walls":
        return workloads.channel(nx=16, ny=12, nz=14, ndrops=2, radius=2.5, wall_gap=1.0, gx=2.5e-5)
    p, f = workloads.droplet(n=16, radius=4.0, mode=capi.MODE_PHASEFIELD)
    p.bc[4] = p.bc[5] = capi.BC_BOUNCEBACK
    return p, f


class OracleSlab:
    """The oracle over a slab's local planes (own planes plus halos)."""

    def __init__(self, p, nx, ny, nz, z0, z1):
        import oracle
        from entropicthreadsafe_b200 import capi
        self.H = HALO[p.mode]
        zper = p.bc[4] == capi.BC_PERIODIC
        whole = z0 == 0 and z1 == nz
        self.lo = 0 if whole else (self.H if (z0 > 0 or zper) else 0)
        self.hi = 0 if whole else (self.H if (z1 < nz or zper) else 0)
        lp = copy.deepcopy(p)
        if self.lo or self.hi:
            for face, halo in ((4, self.lo), (5, self.hi)):
                if halo or lp.bc[face] == capi.BC_PERIODIC:
                    lp.bc[face] = capi.BC_BOUNCEBACK
        self.z0, self.z1, self.nz = z0, z1, nz
        self.zt0, self.zt1 = self.lo, self.lo + (z1 - z0)
        self.o = oracle.Oracle(lp, nx, ny, self.lo + (z1 - z0) + self.hi, fp64=True)
        self.nphi = 0 if p.mode == capi.MODE_SINGLE else self.H

    def upload(self, fields):
        idx = np.arange(self.z0 - self.lo, self.z1 + self.hi) % self.nz
        self.o.set_moments({k: np.asarray(v, np.float64)[idx] for k, v in fields.items()})

    def step(self):
        self.o.step(1)

    def pack(self, side):
        m = self.o.get_moments()
        zm = self.zt0 if side == 0 else self.zt1 - 1
        zp = self.zt0 if side == 0 else self.zt1 - self.H
        parts = [m[k][zm].ravel() for k in MOMENTS] + [m["phi"][zp + i].ravel() for i in range(self.nphi)]
        return np.concatenate(parts)

    def unpack(self, side, buf):
        m = self.o.get_moments()
        zm = self.zt0 - 1 if side == 0 else self.zt1
        zp = self.zt0 - self.H if side == 0 else self.zt1
        plane = m["rho"][0].size
        for i, k in enumerate(MOMENTS):
            m[k][zm] = buf[i * plane:(i + 1) * plane].reshape(m[k][zm].shape)
        for i in range(self.nphi):
            j = len(MOMENTS) + i
            m["phi"][zp + i] = buf[j * plane:(j + 1) * plane].reshape(m["phi"][0].shape)
        self.o.set_moments(m)

    def own(self):
        m = self.o.get_moments()
        return {k: v[self.zt0:self.zt1] for k, v in m.items()}


def _rank(rank, world, port, case, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from entropicthreadsafe_b200.slab import exchange_halos, partition
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    p, f = workload(case)
    nz, ny, nx = f["rho"].shape
    s = OracleSlab(p, nx, ny, nz, *partition(nz, world, rank))
    s.upload(f)

    def sendrecv(sends, recvs):
        bufs = [torch.empty(len(s.pack(0)), dtype=torch.float64) for _ in recvs]
        ops = [dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(b)), peer, None, tag) for b, peer, tag in sends]
        ops += [dist.P2POp(dist.irecv, bufs[i], peer, None, tag) for i, (_, peer, tag) in enumerate(recvs)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        return [b.numpy() for b in bufs]

    zper = p.bc[4] == 0
    for _ in range(NSTEPS):
        s.step()
        exchange_halos(rank, world, zper, s.pack, s.unpack, sendrecv)
    out[rank] = s.own()
    dist.destroy_process_group()


@pytest.mark.parametrize("case", ["colour_periodic", "colour_walls", "phasefield_walls"])
def test_slabs_over_gloo_match_one_lattice(case):
    sys.path.insert(0, ROOT)
    import oracle
    from entropicthreadsafe_b200 import capi
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, case, out)) for r in range(world)]
        for pr in procs:
            pr.start()
        for pr in procs:
            pr.join(300)
            assert pr.exitcode == 0
        got = {k: np.concatenate([out[r][k] for r in range(world)]) for k in capi.FIELDS}
    p, f = workload(case)
    nz, ny, nx = f["rho"].shape
    o = oracle.Oracle(p, nx, ny, nz, fp64=True)
    o.set_moments({k: np.asarray(v, np.float64) for k, v in f.items()})
    o.step(NSTEPS)
    ref = o.get_moments()
    for k in capi.FIELDS:
        err = np.abs(got[k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-30)
        assert err < 1e-12, (case, k, err)
