"""The C ABI: libspires.so loads without a GPU and exports exactly the
functions that include/spires.h and include/spires_ext.h declare (and the
reference header's full symbol list), with nothing else leaking out."""
import ctypes as C
import os
import re
import subprocess

import pytest

import spires_b200 as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# every function of the reference include/spires.h:131-267
REFERENCE_SYMBOLS = [
    "spires_reservoir_create", "spires_reservoir_destroy", "spires_reservoir_reset",
    "spires_step", "spires_run", "spires_train_online", "spires_train_ridge",
    "spires_train_rls", "spires_coarse_grain", "spires_copy_reservoir_state",
    "spires_read_reservoir_state", "spires_read_spike_state", "spires_copy_weights",
    "spires_read_weights", "spires_compute_output", "spires_copy_readout",
    "spires_read_readout", "spires_num_neurons", "spires_num_inputs", "spires_num_outputs",
    "spires_optimize",
]


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(spires_[a-z0-9_]+)\s*\(", src)
    # drop function-pointer typedef names
    return sorted({n for n in names if not n.endswith("_fn")})


def exported():
    lib = os.path.join(ROOT, "spires_b200", "lib", "libspires.so")
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    return sorted({l.split()[-1] for l in out.splitlines() if " T " in l})


@pytest.fixture(scope="module")
def lib():
    return sp.load()


def test_library_loads_without_gpu(lib):
    assert isinstance(lib, C.CDLL)


@pytest.mark.parametrize("header", ["spires.h", "spires_ext.h"])
def test_every_declared_function_is_exported(lib, header):
    names = declared(header)
    assert names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_symbols_present(lib):
    assert not [n for n in REFERENCE_SYMBOLS if not hasattr(lib, n)]
    assert set(REFERENCE_SYMBOLS) <= set(declared("spires.h"))


def test_no_symbols_beyond_the_headers():
    decl = set(declared("spires.h")) | set(declared("spires_ext.h"))
    extra = [s for s in exported() if s not in decl]
    assert not extra, extra


def test_binding_table_covers_headers():
    decl = set(declared("spires.h")) | set(declared("spires_ext.h"))
    bound = set(sp.SIGNATURES) | set(sp.EXT_SIGNATURES)
    assert decl <= bound, sorted(decl - bound)
