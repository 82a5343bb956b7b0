"""Build libtslb.so in-tree with nvcc for sm_100a (B200).

    python -m entropicthreadsafe_b200.build [--verbose]

Each csrc/*.cu (and the host-only csrc/tslb_io.cpp) is compiled to an
object under csrc/_build (in parallel), then linked into
entropicthreadsafe_b200/libtslb.so with the static CUDA runtime; the host
driver driver/tslb_run.cpp is linked against it as entropicthreadsafe_b200/tslb_run.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
OUT = os.path.join(HERE, "libtslb.so")
DRIVER_SRC = os.path.join(HERE, "driver", "tslb_run.cpp")
DRIVER = os.path.join(HERE, "tslb_run")
SOURCES = ["tslb.cu", "k_scalar.cu", "closure.cu", "tslb_io.cpp"]
HEADERS = ["tslb_device.cuh", "tslb_step.cuh", "step_launch.h", "tslb_internal.h", "tcgen05.cuh", "closure_mlp.cuh"]
INCLUDES = ["tslb.h", "tslb_closure.h", "tslb_io.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def _deps() -> list:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(HERE, "..", "include", f) for f in INCLUDES]
    return [d for d in deps if os.path.exists(d)]


def _stale() -> bool:
    if not os.path.exists(OUT) or not os.path.exists(DRIVER):
        return True
    t = min(os.path.getmtime(OUT), os.path.getmtime(DRIVER))
    return any(os.path.getmtime(d) > t for d in _deps() + [DRIVER_SRC])


def build_driver() -> str:
    """The host driver tslb_run (C++), linked against libtslb.so next to it."""
    cxx = os.environ.get("CXX_DRIVER", "g++")
    cmd = [cxx, "-O2", "-std=c++17", "-pthread", "-o", DRIVER, DRIVER_SRC, "-L" + HERE, "-ltslb", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("driver build failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return DRIVER


def _compile(src: str):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC] + CFLAGS + ["-c", "-o", obj, os.path.join(CSRC, src)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return obj, cmd, res


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile csrc/*.cu into libtslb.so next to this file; returns its path."""
    if not force and not _stale():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(_compile, SOURCES))
    for obj, cmd, res in results:
        if res.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
        if verbose:
            print(" ".join(cmd))
            print(res.stderr)
    link = [NVCC] + ARCH + ["-shared", "-o", OUT] + [r[0] for r in results]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + " ".join(link) + "\n" + res.stdout + res.stderr)
    build_driver()
    return OUT


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
