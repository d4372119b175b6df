"""CPU: a C host uses the drop-in boundary as the reference's binding would:
include/crimson_b200.h compiles as C99 (gcc), the program links the library
and gets a status code back without a GPU."""
import os
import shutil
import subprocess

import pytest

from crimsonflowsolver_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")
def test_c_host_links_and_gets_status(tmp_path):
    libdir = os.path.dirname(N.LIB_PATH)
    exe = tmp_path / "probe"
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                         os.path.join(ROOT, "tests", "c_abi_probe.c"), "-L", libdir, "-lcrimson_b200",
                         f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "sm_100a" in run.stdout and "rc=1" in run.stdout and "volume" in run.stdout
