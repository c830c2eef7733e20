"""Host-side check of the pair kernel's work-list split (CPU): compiles
tests/work_split/check_split.cpp against blade_b200/csrc/work_split.h with the
host C++ compiler and runs it over every tile count per item (1..32), tail
length and candidate count up to 400."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_work_split_covers_candidates_once(tmp_path):
    exe = str(tmp_path / "check_split")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "blade_b200", "csrc"),
                    os.path.join(HERE, "work_split", "check_split.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
