"""The C++ driver's command line, without a GPU (CPU only)."""
import os
import subprocess

import pytest

from entropicthreadsafe_b200 import capi

pytestmark = pytest.mark.skipif(not os.path.exists(capi.DRIVER_PATH), reason="tslb_run is built by the package build")


def run(*args):
    return subprocess.run([capi.DRIVER_PATH, *map(str, args)], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args", [["--workload", "cube"], ["--n", "4"], ["--steps"], ["--frobnicate", "1"]])
def test_bad_arguments_print_usage(args):
    r = run(*args)
    assert r.returncode == 2, (r.returncode, r.stderr)
    assert "usage: tslb_run" in r.stderr


def test_without_a_gpu_the_driver_reports_the_failed_creation(tmp_path):
    r = run("--workload", "droplet", "--n", 16, "--steps", 2, "--out", tmp_path, "--quiet")
    if r.returncode == 0:   # a machine with a GPU: the run completes
        assert "glups:" in r.stdout
    else:
        assert r.returncode == 1 and "tslb_create failed" in r.stderr, (r.returncode, r.stderr)
