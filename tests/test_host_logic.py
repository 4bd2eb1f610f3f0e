"""Host-side logic that needs no GPU: the tagged-offset encoding of the cached
operation lists (dmhm_b200/csrc/reloc.h), compiled with the host compiler."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_relocator(tmp_path):
    exe = tmp_path / "reloc_check"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "dmhm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "reloc_check.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
