"""A C caller builds against include/spires.h -- and against the original
project's header when it is present -- and links against libspires.so: the
signatures the compiler checks, the enumerator values and the argument-check
paths that need no GPU (tests/c/relink_check.c)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "spires_b200", "lib")
SRC = os.path.join(ROOT, "tests", "c", "relink_check.c")
REF_INCLUDE = "/root/reference/include"

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")


def build_and_run(include_dir, tmp_path):
    exe = str(tmp_path / "relink_check")
    cmd = ["gcc", "-std=c11", "-Wall", "-Werror", "-I", include_dir, SRC, "-o", exe,
           "-L", LIB, "-lspires", "-Wl,-rpath," + LIB]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    assert "relink check ok" in run.stdout


def test_c_caller_against_this_header(tmp_path):
    build_and_run(os.path.join(ROOT, "include"), tmp_path)


@pytest.mark.skipif(not os.path.isfile(os.path.join(REF_INCLUDE, "spires.h")),
                    reason="original header absent")
def test_c_caller_against_the_original_header(tmp_path):
    build_and_run(REF_INCLUDE, tmp_path)
