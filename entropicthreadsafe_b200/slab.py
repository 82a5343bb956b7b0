"""One lattice cut into z slabs, one slab per GPU (include/tslb.h, "z slabs").

The reference decomposes its domain over MPI ranks and refreshes halo
planes every step (TSLB_2C-mpi/mpi_module.f90:2120-2258: pack into a send
buffer, mpi_isend/mpi_irecv with CUDA-aware MPI, wait, unpack).  Here each
rank holds a Slab (a libtslb slab context on its own GPU) and, after every
step, exchanges the edge planes with its neighbours:

    pack (device kernel) -> NCCL send/recv of one contiguous buffer per
    neighbour (torch.distributed point-to-point) -> unpack (device kernel)

all ordered on the slab's CUDA stream, so the host never waits inside a
step.  The exchange is a real data dependence of the stencil (a step reads
one moment plane and H phi planes beyond its own), the only collective on
the data path.

`exchange_halos` is written against two callables, so the same pattern
drives GPU slabs over NCCL and, in the CPU tests, slab stand-ins over gloo.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi
from .solver import Lattice, TslbError


def partition(nz: int, world: int, rank: int) -> tuple[int, int]:
    """Planes [z_begin, z_end) of rank `rank` when nz planes are cut into
    `world` slabs as evenly as possible (the first nz % world slabs one plane
    deeper)."""
    base, rem = divmod(nz, world)
    z0 = rank * base + min(rank, rem)
    return z0, z0 + base + (1 if rank < rem else 0)


def neighbours(rank: int, world: int, zper: bool) -> tuple[int | None, int | None]:
    """Ranks below (z-) and above (z+) this one; None where the lattice ends."""
    if world == 1:
        return None, None
    lo = rank - 1 if rank > 0 else (world - 1 if zper else None)
    hi = rank + 1 if rank < world - 1 else (0 if zper else None)
    return lo, hi


def exchange_halos(rank: int, world: int, zper: bool, pack, unpack, sendrecv) -> None:
    """One halo refresh.  pack(side) returns this slab's buffer for the
    neighbour on side 0 (z-) or 1 (z+); unpack(side, buf) writes a received
    buffer into the halo on that side; sendrecv(sends, recvs) runs the
    point-to-point transfers -- sends = [(buf, peer, tag)], recvs = [(side,
    peer, tag)] -- and returns the received buffers in recvs order.

    A buffer travelling down (to the z- neighbour) has tag 0 and lands in the
    receiver's top halo; one travelling up has tag 1 and lands in its bottom
    halo.  Sends go down first and receives come from above first, so that a
    transport that matches messages between two ranks in issue order (NCCL)
    pairs them right even when both neighbours are the same rank (two slabs
    of a periodic axis)."""
    lo, hi = neighbours(rank, world, zper)
    sends, recvs = [], []
    if lo is not None:
        sends.append((pack(0), lo, 0))
    if hi is not None:
        sends.append((pack(1), hi, 1))
        recvs.append((1, hi, 0))
    if lo is not None:
        recvs.append((0, lo, 1))
    if not sends:
        return
    got = sendrecv(sends, recvs)
    for (side, _, _), buf in zip(recvs, got):
        unpack(side, buf)


class Slab(Lattice):
    """Planes [z_begin, z_end) of an nx*ny*nz lattice, with halo copies of
    the neighbouring planes.  upload_moments takes the WHOLE lattice's fields
    and keeps the local planes; download returns the own planes only."""

    def __init__(self, params: capi.TslbParams, nx: int, ny: int, nz: int, z_begin: int, z_end: int):
        self.L = capi.lib()
        self.params = params
        h = ctypes.c_void_p()
        rc = self.L.tslb_create_slab(ctypes.addressof(params), nx, ny, nz, z_begin, z_end, ctypes.byref(h))
        if rc != capi.OK:
            raise TslbError(rc, self.L.tslb_last_error(None).decode())
        self.h = h
        geo = (ctypes.c_int * 6)()
        self._check(self.L.tslb_slab_geometry(self.h, geo))
        self.nz_global, self.z_begin, self.z_end, self.halo_lo, self.halo_hi, self.halo = list(geo)
        nzl = self.halo_lo + (z_end - z_begin) + self.halo_hi
        self.shape = (nzl, ny, nx)
        self.n = nx * ny * nzl
        self.halo_bytes = int(self.L.tslb_halo_bytes(self.h))

    def local_planes(self) -> np.ndarray:
        """Global plane index of every local plane (periodic wrap)."""
        return np.arange(self.z_begin - self.halo_lo, self.z_end + self.halo_hi) % self.nz_global

    def upload_moments(self, fields: dict) -> None:
        idx = self.local_planes()
        super().upload_moments({k: np.asarray(fields[k])[idx] for k in capi.FIELDS})

    def download(self, out: dict | None = None) -> dict:
        full = super().download()
        own = slice(self.halo_lo, self.halo_lo + (self.z_end - self.z_begin))
        res = {k: np.ascontiguousarray(v[own]) for k, v in full.items()}
        if out is not None:
            for k in capi.FIELDS:
                out[k][...] = res[k]
            return out
        return res

    def pack(self, side: int, d_buf: int) -> None:
        """Own edge planes for the neighbour on `side` into device memory d_buf."""
        self._check(self.L.tslb_halo_pack(self.h, side, ctypes.c_void_p(d_buf)))

    def unpack(self, side: int, d_buf: int) -> None:
        self._check(self.L.tslb_halo_unpack(self.h, side, ctypes.c_void_p(d_buf)))


class DistributedSlab:
    """A rank's slab of a lattice spread over a torch.distributed process
    group (NCCL, one GPU per rank): step() advances it and refreshes its
    halos, all on the slab's stream."""

    def __init__(self, params: capi.TslbParams, nx: int, ny: int, nz: int, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.zper = params.bc[capi.FACE_ZM] == capi.BC_PERIODIC
        z0, z1 = partition(nz, self.world, self.rank)
        self.slab = Slab(params, nx, ny, nz, z0, z1)
        self.stream = torch.cuda.ExternalStream(self.slab.stream)
        nb = max(self.slab.halo_bytes, 1)
        self.send = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self.recv = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(2)]

    def _global(self, peer: int) -> int:
        return peer if self.group is None else self.dist.get_global_rank(self.group, peer)

    def exchange(self) -> None:
        import torch

        def pack(side):
            self.slab.pack(side, self.send[side].data_ptr())
            return self.send[side]

        def unpack(side, buf):
            self.slab.unpack(side, buf.data_ptr())

        def sendrecv(sends, recvs):
            ops = [self.dist.P2POp(self.dist.isend, buf, self._global(peer), self.group, tag)
                   for buf, peer, tag in sends]
            ops += [self.dist.P2POp(self.dist.irecv, self.recv[side], self._global(peer), self.group, tag)
                    for side, peer, tag in recvs]
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
            return [self.recv[side] for side, _, _ in recvs]

        # NCCL's stream waits for the packing kernels of the slab stream, and the
        # slab stream for the transfers, through torch's current stream
        with torch.cuda.stream(self.stream):
            exchange_halos(self.rank, self.world, self.zper, pack, unpack, sendrecv)

    def upload_moments(self, fields: dict) -> None:
        self.slab.upload_moments(fields)

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            self.slab.step(1)
            self.exchange()

    def download(self) -> dict:
        return self.slab.download()

    def close(self) -> None:
        self.slab.close()
