"""Failure paths, made without faulting or hanging the GPU.

* A bounded wait that runs out: one CTA of the cooperative step kernel
  withholds its grid-barrier arrival once (spires_ext_test_withhold_arrival),
  so every other CTA's wait runs out after a short limit
  (spires_ext_set_wait_limit). The launch must come back with
  SPIRES_ERR_INTERNAL, the recorded error must name the micro-step whose
  barrier was withheld, and after a reset the same reservoir must again step
  bit for bit like the oracle (the context stays usable).
* Allocation failures: the library's n-th device allocation is made to fail
  on the host side (spires_ext_test_fail_device_alloc) for every n that create
  and ridge reach. Each call must return SPIRES_ERR_ALLOC, leave no device
  allocation behind (spires_ext_test_live_device_allocs), and a failed ridge
  must leave W_out as it was.

The reference has none of this: it prints or exits (src/neuron.c:6-10,
src/reservoir.c:74-77)."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def _cfg(neuron, n=2000):
    return sp.make_config(n, 2, 2, rho=1.2, ei=0.55, gamma=1.2, conn=0.01,
                          topo=sp.CONN_SCALE_FREE, neuron=neuron,
                          nparams=O.NEURON_PARAMS[neuron])


def _last_error(r):
    code, step = C.c_int(-1), C.c_longlong(-1)
    assert r.lib.spires_ext_last_device_error(r.h, C.byref(code), C.byref(step)) == sp.SPIRES_OK
    return code.value, step.value


@pytest.mark.parametrize("neuron", [sp.FLIF_GL, sp.LIF_DISCRETE])
def test_withheld_arrival_times_out_and_device_recovers(neuron):
    cfg = _cfg(neuron)
    u = np.random.default_rng(0).uniform(-1.0, 1.5, (40, 2))
    r = sp.Reservoir(cfg, seed=17)
    assert r.launch().ctas > 1, "the test needs a multi-CTA grid"
    assert _last_error(r) == (0, 0)
    assert r.lib.spires_ext_set_wait_limit(r.h, 50.0) == sp.SPIRES_OK
    # 12 steps run normally, then CTA 1 withholds its arrival at the barrier
    # that opens micro-step 5 of the next launch (absolute micro-step 17)
    r.run_record(u[:12])
    assert r.lib.spires_ext_test_withhold_arrival(r.h, 1, 5) == sp.SPIRES_OK
    T = 10
    P = np.empty((T, r.n))
    st = r.lib.spires_ext_run_record(r.h, sp.dptr(np.ascontiguousarray(u[12:12 + T])), T,
                                     sp.dptr(P), None, None)
    assert st == sp.SPIRES_ERR_INTERNAL
    assert _last_error(r) == (1, 17)
    # the hook was one-shot and the device is usable: from reset, the run is
    # bit-identical to the oracle's
    r.reset()
    phi, R, _ = r.run_record(u)
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=17))
    phi_o, ras_o, _ = orc.run(u)
    assert np.array_equal(sp.unpack_raster(R, cfg.num_neurons), ras_o)
    assert np.array_equal(phi.view(np.uint64), phi_o.view(np.uint64))


def test_wait_limit_arguments():
    r = sp.Reservoir(_cfg(sp.LIF_DISCRETE, n=100), seed=1)
    for bad in (0.0, -1.0, float("nan"), 1e9):
        assert r.lib.spires_ext_set_wait_limit(r.h, bad) == sp.SPIRES_ERR_INVALID_ARG
    assert r.lib.spires_ext_test_withhold_arrival(r.h, -1, 3) == sp.SPIRES_ERR_INVALID_ARG
    assert r.lib.spires_ext_test_withhold_arrival(r.h, 0, 0) == sp.SPIRES_ERR_INVALID_ARG
    r.close()


def _create(lib, cfg, seed):
    sp.libc.srand(seed)
    h = C.c_void_p()
    st = lib.spires_reservoir_create(C.byref(cfg), C.byref(h))
    return st, h


def test_create_allocation_failures_release_everything():
    lib = sp.load()
    cfg = _cfg(sp.FLIF_GL, n=300)
    base = lib.spires_ext_test_live_device_allocs()
    failures = 0
    try:
        for k in range(200):
            lib.spires_ext_test_fail_device_alloc(k)
            st, h = _create(lib, cfg, 5)
            lib.spires_ext_test_fail_device_alloc(-1)
            if st == sp.SPIRES_OK:
                lib.spires_reservoir_destroy(h)
                assert lib.spires_ext_test_live_device_allocs() == base
                break
            assert st == sp.SPIRES_ERR_ALLOC, (k, st)
            assert lib.spires_ext_test_live_device_allocs() == base, k
            failures += 1
        else:
            pytest.fail("create never got past the injected failures")
    finally:
        lib.spires_ext_test_fail_device_alloc(-1)
    assert failures >= 5  # every device buffer of create was reached


def test_ridge_allocation_failures_keep_the_readout():
    lib = sp.load()
    cfg = _cfg(sp.FLIF_GL, n=300)
    rng = np.random.default_rng(3)
    u = np.ascontiguousarray(rng.uniform(-1.0, 1.5, (150, 2)))
    y = np.ascontiguousarray(rng.standard_normal((150, 2)))
    r = sp.Reservoir(cfg, seed=5)
    W0 = r.readout().copy()
    base = lib.spires_ext_test_live_device_allocs()
    failures = 0
    try:
        for k in range(200):
            lib.spires_ext_test_fail_device_alloc(k)
            st = lib.spires_train_ridge(r.h, sp.dptr(u), sp.dptr(y), 150, 1e-3)
            lib.spires_ext_test_fail_device_alloc(-1)
            assert lib.spires_ext_test_live_device_allocs() == base, k
            if st == sp.SPIRES_OK:
                break
            assert st == sp.SPIRES_ERR_ALLOC, (k, st)
            assert np.array_equal(r.readout(), W0), k
            failures += 1
        else:
            pytest.fail("ridge never got past the injected failures")
    finally:
        lib.spires_ext_test_fail_device_alloc(-1)
    assert failures >= 3
    # the successful fit is the one a reservoir without failures gets
    r2 = sp.Reservoir(cfg, seed=5)
    r2.train_ridge(u, y, 1e-3)
    assert np.array_equal(r.readout(), r2.readout())
    r.close()
    r2.close()
