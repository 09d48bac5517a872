"""The C ABI from plain C (host only, no GPU): tests/c_abi_client.c, compiled
as pedantic C99 against include/dg_b200.h and linked against
libdg_b200.so, runs the host-side entry points and the error convention,
the way a binding from another language would call them."""
import os
import shutil
import subprocess

import pytest

import dg_b200
from conftest import ROOT


def test_plain_c_client_links_and_runs(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lib_dir = os.path.dirname(dg_b200.LIB_PATH)
    exe = tmp_path / "c_abi_client"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c_abi_client.c"),
                    "-o", str(exe), "-L" + lib_dir, "-ldg_b200", "-Wl,-rpath," + lib_dir, "-lm"],
                   check=True, capture_output=True, text=True)
    mesh = os.path.join(ROOT, "tests", "golden", "meshes", "quad_1x1.h5")
    r = subprocess.run([str(exe), mesh], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
