"""CPU checks of the C-ABI library: it loads, exports every declared entry
point, and rejects bad parameters before touching the GPU."""
import ctypes
import os
import re

import pytest

from entropicthreadsafe_b200 import capi

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADERS = tuple(sorted(h for h in os.listdir(INCLUDE) if h.endswith(".h")))


def declared_symbols():
    names = set()
    for h in HEADERS:
        with open(os.path.join(INCLUDE, h)) as fh:
            text = fh.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(tslb_[a-z_0-9]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from entropicthreadsafe_b200 import build
    build.build()
    return capi.lib()


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 40
    assert "tslb_closure_train" in names and "tslb_set_tau_correction" in names
    for name in names:
        assert hasattr(lib, name), name


def test_default_params_match_python_mirror(lib):
    p = capi.TslbParams()
    lib.tslb_default_params(ctypes.addressof(p))
    q = capi.default_params()
    assert ctypes.sizeof(p) == ctypes.sizeof(q)
    assert bytes(p) == bytes(q)


@pytest.mark.parametrize("field,value,code", [
    ("tau_a", 0.5, capi.ERR_ARG),
    ("tau_a", float("nan"), capi.ERR_ARG),
    ("mode", 7, capi.ERR_ARG),
    ("precision", 7, capi.ERR_ARG),
    ("wall_phi_mode", 3, capi.ERR_ARG),
])
def test_create_rejects_bad_params(lib, field, value, code):
    p = capi.default_params()
    setattr(p, field, value)
    h = ctypes.c_void_p()
    rc = lib.tslb_create(ctypes.addressof(p), 8, 8, 8, ctypes.byref(h))
    assert rc == code
    assert not h.value
    assert lib.tslb_last_error(None)


def test_create_rejects_unpaired_periodic_faces(lib):
    p = capi.default_params()
    p.bc[4] = capi.BC_BOUNCEBACK  # z- wall, z+ periodic
    h = ctypes.c_void_p()
    assert lib.tslb_create(ctypes.addressof(p), 8, 8, 8, ctypes.byref(h)) == capi.ERR_ARG
    assert b"pairs" in lib.tslb_last_error(None)


def test_create_rejects_bad_sizes(lib):
    p = capi.default_params()
    h = ctypes.c_void_p()
    assert lib.tslb_create(ctypes.addressof(p), 0, 8, 8, ctypes.byref(h)) == capi.ERR_ARG
    assert lib.tslb_create(None, 8, 8, 8, ctypes.byref(h)) == capi.ERR_ARG


def test_null_context_calls_fail_cleanly(lib):
    assert lib.tslb_step(None, 1) == capi.ERR_ARG
    assert lib.tslb_synchronize(None) == capi.ERR_ARG
    assert lib.tslb_launch_count(None) == 0


def test_noalloc_rejects_bad_buffers_before_any_device_call(lib):
    """tslb_step_noalloc checks sizes and buffer ranges on the host before it
    touches the device, so these addresses (never dereferenced) are safe."""
    base = 1 << 32
    fbytes = 4
    p = capi.default_params()
    n = 8 * 8 * 8
    # overlapping ranges: the output starts one field after the input
    stride = 512
    for off in (0, stride * fbytes, 10 * stride * fbytes):
        rc = lib.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, ctypes.c_void_p(base),
                                   ctypes.c_void_p(base + off), stride, None)
        assert rc == capi.ERR_ARG, off
        assert b"overlap" in lib.tslb_last_error(None)
    # output before the input, ending inside it
    rc = lib.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, ctypes.c_void_p(base + 16 * fbytes),
                               ctypes.c_void_p(base + 16 * fbytes - 11 * stride * fbytes + 16), stride, None)
    assert rc == capi.ERR_ARG
    # a stride below the lattice, misalignment, an inlet face
    assert lib.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, ctypes.c_void_p(base),
                                 ctypes.c_void_p(base + (1 << 20)), n - 4, None) == capi.ERR_ARG
    assert lib.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, ctypes.c_void_p(base + 4),
                                 ctypes.c_void_p(base + (1 << 20)), n, None) == capi.ERR_ARG
    assert lib.tslb_step_noalloc(ctypes.addressof(p), 8, 8, 8, None, ctypes.c_void_p(base), n, None) == capi.ERR_ARG
    q = capi.default_params()
    q.bc[4] = q.bc[5] = capi.BC_INLET
    assert lib.tslb_step_noalloc(ctypes.addressof(q), 8, 8, 8, ctypes.c_void_p(base), ctypes.c_void_p(base + (1 << 20)),
                                 n, None) == capi.ERR_UNSUPPORTED
