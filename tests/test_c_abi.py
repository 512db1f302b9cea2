"""A C caller builds against include/spires.h -- and against the original
project's header when it is present -- and links against libspires.so, or
libspires.a with its documented extra libraries: the signatures the compiler
checks, the enumerator values and the argument-check paths that need no GPU
(tests/c/relink_check.c)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "spires_b200", "lib")
SRC = os.path.join(ROOT, "tests", "c", "relink_check.c")
# the original project's sources, when present: SPIRES_REF_DIR, else a
# checkout named `reference` beside this repository
REF_DIR = os.environ.get("SPIRES_REF_DIR",
                         os.path.abspath(os.path.join(ROOT, "..", "reference")))
REF_INCLUDE = os.path.join(REF_DIR, "include")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")


CUDA_LIB = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64")
# the static archive's extra libraries, as the integration notes give them
STATIC = [os.path.join(LIB, "libspires.a"), "-L" + CUDA_LIB, "-lcudart_static",
          "-lstdc++", "-fopenmp", "-lpthread", "-ldl", "-lrt", "-lm"]


def build_and_run(include_dir, tmp_path, static=False):
    exe = str(tmp_path / ("relink_check_static" if static else "relink_check"))
    link = STATIC if static else ["-L", LIB, "-lspires", "-Wl,-rpath," + LIB]
    cmd = ["gcc", "-std=c11", "-Wall", "-Werror", "-I", include_dir, SRC, "-o", exe] + link
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    assert "relink check ok" in run.stdout


def test_c_caller_against_this_header(tmp_path):
    build_and_run(os.path.join(ROOT, "include"), tmp_path)


@pytest.mark.skipif(not os.path.isfile(os.path.join(CUDA_LIB, "libcudart_static.a")),
                    reason="static CUDA runtime absent")
def test_c_caller_static_archive(tmp_path):
    build_and_run(os.path.join(ROOT, "include"), tmp_path, static=True)


@pytest.mark.skipif(not os.path.isfile(os.path.join(REF_INCLUDE, "spires.h")),
                    reason="original header absent")
def test_c_caller_against_the_original_header(tmp_path):
    build_and_run(REF_INCLUDE, tmp_path)


REF_EXAMPLES = os.path.join(REF_DIR, "examples")


@pytest.mark.parametrize("name", ["mackey_glass_prediction", "spoken_digit_recognition"])
def test_original_examples_link_unchanged(name, tmp_path):
    """The original project's example programs that use only the public API
    compile against this include/spires.h and link against libspires.so as
    they are (running them needs a GPU and, for the digits, a dataset). The
    third example reaches into the original's internal headers and is not a
    public-API caller."""
    src = os.path.join(REF_EXAMPLES, name, name + ".c")
    if not os.path.isfile(src):
        pytest.skip("original examples absent")
    exe = str(tmp_path / name)
    cmd = ["gcc", "-std=gnu11", "-I", os.path.join(ROOT, "include"), src, "-o", exe, "-L", LIB,
           "-lspires", "-Wl,-rpath," + LIB, "-lm"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
