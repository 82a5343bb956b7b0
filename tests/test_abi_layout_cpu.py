"""The ctypes mirror of tslb_params has the C layout of include/tslb.h, field
by field (a C program compiled here prints the offsets; CPU only)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from entropicthreadsafe_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_params_field_offsets_match_the_header(tmp_path):
    names = [f[0] for f in capi.TslbParams._fields_]
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tslb.h"', "int main(void) {",
             '  printf("sizeof %zu\\n", sizeof(tslb_params));']
    lines += [f'  printf("{n} %zu\\n", offsetof(tslb_params, {n}));' for n in names]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    assert int(out["sizeof"]) == ctypes.sizeof(capi.TslbParams)
    for n in names:
        assert int(out[n]) == getattr(capi.TslbParams, n).offset, n


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_headers_compile_as_c99(tmp_path):
    """A C host includes the three public headers without a C++ compiler."""
    src = tmp_path / "hosts.c"
    src.write_text('#include "tslb.h"\n#include "tslb_io.h"\n#include "tslb_closure.h"\n'
                   "int main(void) { tslb_params p; tslb_default_params(&p); return p.mode; }\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"), "-c",
                    "-o", str(tmp_path / "hosts.o"), str(src)], check=True)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_c_host_links_and_gets_an_error_code_not_an_abort(tmp_path):
    """A C program links against libtslb.so and calls tslb_create: on a machine
    without a GPU it gets an error code and a message, the process lives on."""
    capi.lib()   # built in-tree
    lib_dir = os.path.dirname(capi.LIB_PATH)
    src = tmp_path / "host.c"
    src.write_text(
        '#include <stdio.h>\n#include "tslb.h"\n'
        "int main(void) {\n"
        "  tslb_params p; tslb_default_params(&p);\n"
        "  tslb_ctx* c = NULL;\n"
        "  int rc = tslb_create(&p, 16, 16, 16, &c);\n"
        '  if (rc == TSLB_OK) { tslb_destroy(c); printf("created\\n"); return 0; }\n'
        '  printf("error %d %s\\n", rc, tslb_last_error(NULL));\n'
        "  return c == NULL ? 0 : 1;\n"
        "}\n")
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src),
                    "-L" + lib_dir, "-ltslb", "-Wl,-rpath," + lib_dir], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout.strip()
    assert out == "created" or (out.startswith("error ") and len(out.split(" ", 2)[2]) > 0), out
