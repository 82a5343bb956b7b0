"""GPU checks of the driver layer: checkpoints restore the state bit for
bit (every storage precision), and the C++ driver tslb_run reproduces the
Python path's frames, writes the reference's files and restarts from its
own dumps."""
import os
import subprocess

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [capi.PREC_FP32, capi.PREC_FP16S, capi.PREC_BF16])
def test_checkpoint_restart_is_bit_exact(tmp_path, prec):
    p, f = workloads.droplet(n=24, radius=6.0)
    p.precision = prec
    ck = tmp_path / "state.ckpt"
    with Lattice(p, 24, 24, 24) as a:
        a.upload_moments(f)
        a.step(10)
        a.checkpoint_save(str(ck))
        a.step(10)
        ref = a.download()
        assert a.steps_done == 20
    with Lattice(p, 24, 24, 24) as b:
        b.checkpoint_load(str(ck))
        assert b.steps_done == 10
        b.step(10)
        got = b.download()
    for k in capi.FIELDS:
        assert np.array_equal(got[k], ref[k]), k


def test_checkpoint_rejects_other_sizes(tmp_path):
    p, f = workloads.droplet(n=16, radius=4.0)
    ck = tmp_path / "s.ckpt"
    with Lattice(p, 16, 16, 16) as a:
        a.upload_moments(f)
        a.checkpoint_save(str(ck))
    with Lattice(p, 16, 16, 20) as b:
        with pytest.raises(Exception):
            b.checkpoint_load(str(ck))


def read_vti_data(path):
    b = open(path, "rb").read()
    off = b.index(b'encoding="raw">\n') + len(b'encoding="raw">\n') + 1
    nbytes = int(np.frombuffer(b[off:off + 4], np.int32)[0])
    return np.frombuffer(b[off + 4:off + 4 + nbytes], np.float32)


def run_driver(*args):
    res = subprocess.run([capi.DRIVER_PATH, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout


def test_driver_droplet_matches_python_path_and_writes_files(tmp_path):
    out = run_driver("--workload", "droplet", "--n", 32, "--steps", 40, "--stamp", 20, "--stamp2d", 20,
                     "--dump", 40, "--out", tmp_path)
    assert "glups:" in out and "step :       20" in out
    for name in ("out_phi_000001.vti", "out_phi_000002.vti", "out_phixy_000002.raw", "out_wyz_000002.raw",
                 "dump_state_000040.ckpt"):
        assert (tmp_path / name).exists(), name
    p, f = workloads.droplet(n=32, radius=8.0)
    with Lattice(p, 32, 32, 32) as lat:
        lat.upload_moments(f)
        lat.step(40)
        ref = lat.download()
    assert np.array_equal(read_vti_data(tmp_path / "out_phi_000002.vti"), ref["phi"].reshape(-1))
    xz = np.fromfile(tmp_path / "out_uxz_000002.raw", np.float32).reshape(32, 32)
    assert np.array_equal(xz, ref["u"][:, 15, :])


def test_driver_jet_restarts_from_its_dump(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    # n = 64: an inlet disc of radius 2.7 nodes (32 would give four nodes)
    run_driver("--workload", "jet", "--n", 64, "--steps", 60, "--stamp", 60, "--dump", 30, "--out", a, "--quiet")
    run_driver("--workload", "jet", "--n", 64, "--steps", 30, "--stamp", 60, "--out", b, "--quiet",
               "--load", a / "dump_state_000030.ckpt")
    full = read_vti_data(a / "out_phi_000001.vti")
    restarted = read_vti_data(b / "out_phi_000001.vti")
    assert np.array_equal(full, restarted)
    assert (full > 0).sum() > 0  # the jet has entered


def test_host_alloc_buffers_take_downloads():
    """tslb_host_alloc gives page-locked memory that downloads fill like any
    host array (the C++ driver downloads its frames into it)."""
    import ctypes
    L = capi.lib()
    p, f = workloads.droplet(n=24, radius=6.0)
    n = 24 ** 3
    assert not L.tslb_host_alloc(0)
    ptr = L.tslb_host_alloc(4 * n)
    assert ptr
    try:
        buf = np.ctypeslib.as_array((ctypes.c_float * n).from_address(ptr))
        with Lattice(p, 24, 24, 24) as lat:
            lat.upload_moments(f)
            lat.step(5)
            ref = lat.download()
            null = ctypes.POINTER(ctypes.c_float)()
            args = [null] * 10 + [ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float))]
            assert L.tslb_download_moments(lat.h, *args) == capi.OK
        assert np.array_equal(buf.reshape(24, 24, 24), ref["phi"])
    finally:
        L.tslb_host_free(ptr)
    L.tslb_host_free(None)


def test_release_memory_returns_the_cached_lattice_memory():
    """A destroyed lattice's device memory stays cached for the next lattice;
    tslb_release_memory gives it back to the device."""
    import torch
    L = capi.lib()
    p, f = workloads.droplet(n=96, radius=20.0)
    with Lattice(p, 96, 96, 96) as lat:   # two 11-field states of 96^3 nodes: 78 MB
        lat.upload_moments(f)
        lat.step(1)
    torch.cuda.synchronize()
    free_cached, _ = torch.cuda.mem_get_info()
    assert L.tslb_release_memory() == capi.OK
    free_released, _ = torch.cuda.mem_get_info()
    assert free_released - free_cached >= 60e6
    # lattices still work after the release
    with Lattice(p, 96, 96, 96) as lat:
        lat.upload_moments(f)
        lat.step(1)
        assert abs(lat.reduce()["mass"] - f["rho"].astype(np.float64).sum()) < 1e-3 * 96 ** 3
