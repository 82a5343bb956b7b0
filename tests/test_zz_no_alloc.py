"""tslb_step_noalloc: one step on device buffers the caller owns.

Some hosts cannot let a library call cudaMalloc -- a Fortran driver whose
device arrays live in an OpenACC data region, a code that hands all GPU
memory to its own pool, a time loop that must never allocate.  For them
the library offers one entry point that allocates nothing: the only
scratch the step needs, its non-finite flag, is a fixed device array inside
libtslb.so (TSLB_NOALLOC_SCRATCH_WORDS words), which tslb_noalloc_check
reads back (and clears) on the caller's stream.

These tests run that entry point twice in a row through the C-ABI and
compare each result with the context API (tslb_create/tslb_step) on the
same input, with the parity tolerance of the other GPU tests.  The device
buffers here come from torch; the entry point itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu

TARGET = 1e-5  # max relative error per field, as in test_gpu_parity


def to_device_layout(fields, stride):
    """The library's device layout: 11 fields of `stride` floats, rho - 1 first."""
    import torch
    n = fields["rho"].size
    host = np.zeros((11, stride), np.float32)
    for k, name in enumerate(capi.FIELDS):
        v = np.asarray(fields[name], np.float32).reshape(-1)
        host[k, :n] = (v - np.float32(1.0)) if name == "rho" else v
    return torch.from_numpy(host).cuda()


def from_device_layout(t, shape):
    host = t.cpu().numpy()
    n = int(np.prod(shape))
    out = {}
    for k, name in enumerate(capi.FIELDS):
        v = host[k, :n].reshape(shape)
        out[name] = (np.float32(1.0) + v) if name == "rho" else v.copy()
    return out


def context_steps(p, f, nsteps):
    nz, ny, nx = f["rho"].shape
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        outs = []
        for _ in range(nsteps):
            lat.step(1)
            outs.append(lat.download())
    return outs


def noalloc_steps(p, f, nsteps):
    import torch
    L = capi.lib()
    nz, ny, nx = f["rho"].shape
    n = nx * ny * nz
    stride = (n + 31) // 32 * 32
    bufs = [to_device_layout(f, stride), torch.empty((11, stride), dtype=torch.float32, device="cuda")]
    outs = []
    for k in range(nsteps):
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        rc = L.tslb_step_noalloc(ctypes.addressof(p), nx, ny, nz, ctypes.c_void_p(src.data_ptr()),
                                 ctypes.c_void_p(dst.data_ptr()), stride, None)
        assert rc == capi.OK, L.tslb_last_error(None).decode()
        torch.cuda.synchronize()
        outs.append(from_device_layout(dst, (nz, ny, nx)))
    return outs


def assert_close(a, b, label):
    for name in capi.FIELDS:
        ref = np.asarray(b[name], np.float64)
        err = np.abs(np.asarray(a[name], np.float64) - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err <= TARGET, f"{label} {name}: {err:.3e}"


def phasefield_walls():
    n = 24
    p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.01, sharp_c=0.9,
                         bc=[capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK] * 2, bc_phi=[0.0] * 6)
    f = workloads.empty_fields(n, n, n)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((x - 11.5) ** 2 + (y - 11.5) ** 2 + (z - 11.5) ** 2)
    f["phi"][:] = 0.5 * (1 + np.tanh((6 - r) / 1.5))
    return p, f


def test_noalloc_phasefield_matches_context_api_two_calls():
    p, f = phasefield_walls()
    ref = context_steps(p, f, 2)
    got = noalloc_steps(p, f, 2)
    for k in range(2):
        assert_close(got[k], ref[k], f"phase field, call {k + 1}")


def test_noalloc_colour_matches_context_api_two_calls():
    p, f = workloads.droplet(n=24, radius=6.0)
    ref = context_steps(p, f, 2)
    got = noalloc_steps(p, f, 2)
    for k in range(2):
        assert_close(got[k], ref[k], f"colour, call {k + 1}")


def test_noalloc_rejects_aliased_and_short_buffers():
    import torch
    L = capi.lib()
    p = capi.default_params()
    buf = torch.zeros((11, 64), dtype=torch.float32, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    # input and output must differ (and not overlap)
    rc = L.tslb_step_noalloc(ctypes.addressof(p), 4, 4, 4, ptr, ptr, 64, None)
    assert rc == capi.ERR_ARG
    assert b"overlap" in L.tslb_last_error(None)
    # a field stride below the lattice
    other = torch.zeros((11, 64), dtype=torch.float32, device="cuda")
    rc = L.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, ptr, ctypes.c_void_p(other.data_ptr()), 64, None)
    assert rc == capi.ERR_ARG
    assert b"field_stride" in L.tslb_last_error(None)


def test_noalloc_takes_a_lattice_larger_than_any_fixed_scratch():
    """The scratch does not grow with the lattice: a 128 x 96 x 96 phase-field
    box (1.2 M nodes) steps like the context API."""
    p, f = workloads.droplet(n=96, radius=20.0, mode=capi.MODE_PHASEFIELD)
    big = {k: np.concatenate([v, v[:, :, :32]], axis=2) for k, v in f.items()}   # 128 x 96 x 96
    ref = context_steps(p, big, 1)
    got = noalloc_steps(p, big, 1)
    assert_close(got[0], ref[0], "phase field, 128 x 96 x 96")


def test_noalloc_reports_a_non_finite_step_and_allocates_nothing():
    """A NaN written by the host into the caller's input buffer comes back as
    TSLB_ERR_NAN from tslb_noalloc_check (once: the check clears the flag),
    and repeated calls leave the device's free memory unchanged."""
    import torch
    L = capi.lib()
    p, f = workloads.droplet(n=24, radius=6.0)
    n = 24 ** 3
    stride = (n + 31) // 32 * 32
    src = to_device_layout(f, stride)
    dst = torch.empty_like(src)
    args = (ctypes.addressof(p), 24, 24, 24, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), stride, None)
    assert L.tslb_step_noalloc(*args) == capi.OK
    assert L.tslb_noalloc_check(None) == capi.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert L.tslb_step_noalloc(*args) == capi.OK
    assert L.tslb_noalloc_check(None) == capi.OK
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    host = src.cpu()
    host[capi.FIELDS.index("u"), 24 * 24 * 12 + 24 * 12 + 12] = float("nan")
    src.copy_(host)
    assert L.tslb_step_noalloc(*args) == capi.OK
    assert L.tslb_noalloc_check(None) == capi.ERR_NAN
    assert b"non-finite" in L.tslb_last_error(None)
    assert L.tslb_noalloc_check(None) == capi.OK
