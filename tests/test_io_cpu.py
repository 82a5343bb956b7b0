"""CPU checks of the output formats (include/tslb_io.h) against the layout of
the reference's print_module.f90: the VTK ImageData header of header_vtk /
footer_vtk (fixed-length lines: 22, 67, 70, 63, 18, 115, 19, 13, 15, 32 and
1 bytes, then an int32 byte count, the FP32 data and a 30-byte footer), raw
stream files, mid-plane slices and 6-digit frame numbers."""
import ctypes
import re

import numpy as np
import pytest

from entropicthreadsafe_b200 import capi

HEADER_LINES = (22, 67, 70, 63, 18, 115, 19, 13, 15, 32)


@pytest.fixture(scope="module")
def lib():
    from entropicthreadsafe_b200 import build
    build.build()
    return capi.lib()


def read_vti(path):
    b = open(path, "rb").read()
    i = b.index(b"_") if b"<AppendedData" in b else -1
    head = b[:b.index(b"<AppendedData")]
    start = b.index(b"\n_", 0) + 2 if b"\n_" in b else None
    off = b.index(b'encoding="raw">\n') + len(b'encoding="raw">\n') + 1
    nbytes = int(np.frombuffer(b[off:off + 4], np.int32)[0])
    data = np.frombuffer(b[off + 4:off + 4 + nbytes], np.float32)
    tail = b[off + 4 + nbytes:]
    return b, off, nbytes, data, tail


def test_vti_layout_matches_print_module(lib, tmp_path):
    nx, ny, nz = 5, 4, 3
    f = np.arange(nx * ny * nz, dtype=np.float32).reshape(nz, ny, nx) * 0.5 - 7
    path = tmp_path / "out_phi_000001.vti"
    assert lib.tslb_write_vti(str(path).encode(), b"phi", nx, ny, nz, 1, capi.fptr(f)) == capi.OK
    b, off, nbytes, data, tail = read_vti(path)
    lines = b[:off - 1].split(b"\n")
    assert [len(l) + 1 for l in lines[:-1]] == list(HEADER_LINES)
    assert lines[-1] == b"" and b[off - 1:off] == b"_"
    assert off == sum(HEADER_LINES) + 1
    assert b'<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">' in b
    assert b'WholeExtent="     1      5      1      4      1      3"' in b
    assert b'Name="phi     " NumberOfComponents="1" format="appended" offset="           0"/>' in b
    assert nbytes == 4 * nx * ny * nz and np.array_equal(data, f.reshape(-1))
    assert tail == b"\n  </AppendedData>\n</VTKFile>\n" and len(tail) == 30


def test_vti_vector_and_bad_arguments(lib, tmp_path):
    nx, ny, nz = 3, 3, 2
    v = np.random.default_rng(0).normal(size=(nz, ny, nx, 3)).astype(np.float32)
    path = tmp_path / "vel.vti"
    assert lib.tslb_write_vti(str(path).encode(), b"vel", nx, ny, nz, 3, capi.fptr(v)) == capi.OK
    b, off, nbytes, data, tail = read_vti(path)
    assert b'NumberOfComponents="3"' in b and np.array_equal(data, v.reshape(-1))
    assert lib.tslb_write_vti(str(path).encode(), b"vel", nx, ny, nz, 2, capi.fptr(v)) == capi.ERR_ARG
    assert lib.tslb_write_vti(str(path).encode(), b"toolongname", nx, ny, nz, 3, capi.fptr(v)) == capi.ERR_ARG


def test_raw_and_slices(lib, tmp_path):
    nx, ny, nz = 6, 4, 8
    f = np.random.default_rng(1).normal(size=(nz, ny, nx)).astype(np.float32)
    p = tmp_path / "f.raw"
    assert lib.tslb_write_raw(str(p).encode(), capi.fptr(f), f.size) == capi.OK
    assert np.array_equal(np.fromfile(p, np.float32), f.reshape(-1))
    assert lib.tslb_write_slices(str(tmp_path).encode(), b"phi", 7, nx, ny, nz, capi.fptr(f)) == capi.OK
    # 1-based nz/2, ny/2, nx/2 of the reference
    xy = np.fromfile(tmp_path / "out_phixy_000007.raw", np.float32).reshape(ny, nx)
    xz = np.fromfile(tmp_path / "out_phixz_000007.raw", np.float32).reshape(nz, nx)
    yz = np.fromfile(tmp_path / "out_phiyz_000007.raw", np.float32).reshape(nz, ny)
    assert np.array_equal(xy, f[nz // 2 - 1])
    assert np.array_equal(xz, f[:, ny // 2 - 1, :])
    assert np.array_equal(yz, f[:, :, nx // 2 - 1])


def test_frame_path_zero_pads_six_digits(lib):
    buf = ctypes.create_string_buffer(256)
    assert lib.tslb_frame_path(buf, 256, b"output", b"out", b"phi", 42, b"vti") == capi.OK
    assert buf.value == b"output/out_phi_000042.vti"
    assert lib.tslb_frame_path(buf, 8, b"output", b"out", b"phi", 42, b"vti") == capi.ERR_ARG
