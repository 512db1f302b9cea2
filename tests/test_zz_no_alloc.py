"""The allocation-free ridge solve (spires_ext_ridge_solve_noalloc).

Some callers cannot allocate device memory themselves: a host framework that
hands every device buffer out from its own allocator or quota, or a control
loop that cannot pay for the device-wide synchronisation of cudaMalloc and
cudaFree. For them the library solves a ridge readout from states they already
hold on the device, working in one fixed array that the library owns.

Checked here, each time on two calls in a row (the array keeps the previous
call's contents): against the FP64 oracle ridge on the same states, with and
without washout; against the allocating entry point (spires_ext_train_ridge)
on the same reservoir; a singular system returns SPIRES_ERR_INTERNAL and leaves
the output buffer alone; sizes beyond the array are refused. No device
allocation of the library is live after the calls. This file runs last so
that a failure here leaves every other result in place.
"""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0)


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _states(n, din, dout, T, seed):
    cfg = sp.make_config(n, din, dout, rho=1.2, ei=0.55, gamma=1.2, conn=0.03,
                         topo=sp.CONN_SCALE_FREE, neuron=sp.FLIF_GL, nparams=GL)
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.5, size=(T, din))
    y = rng.standard_normal((T, dout))
    return cfg, u, y


class _Dev:
    """The caller's own device buffers (torch stands in for its allocator)."""

    def __init__(self, phi, y, dout, n):
        import torch

        self.torch = torch
        self.phi = torch.from_numpy(np.ascontiguousarray(phi)).cuda()
        self.y = torch.from_numpy(np.ascontiguousarray(y)).cuda()
        self.w = torch.empty((dout, n), dtype=torch.float64, device="cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def ptr(t):
        return C.c_void_p(t.data_ptr())

    def solve(self, lib, T, n, dout, washout, lam, fill=float("nan")):
        self.w.fill_(fill)
        self.torch.cuda.synchronize()
        st = lib.spires_ext_ridge_solve_noalloc(self.ptr(self.phi), self.ptr(self.y), T, n, dout,
                                                washout, lam, self.ptr(self.w), self.stream)
        return st, self.w.cpu().numpy()


@pytest.mark.parametrize("washout,lam", [(0, 1e-4), (150, 1e-2), (37, 1e-6)])
def test_noalloc_ridge_matches_fp64_oracle(washout, lam):
    lib = sp.load()
    n, din, dout, T = 300, 2, 3, 600
    cfg, u, y = _states(n, din, dout, T, seed=5)
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=41))
    phi, _, _ = orc.run(u)
    Wo = O.oracle_ridge(phi, y, lam, washout=washout)
    dev = _Dev(phi, y, dout, n)
    live = lib.spires_ext_test_live_device_allocs()
    for _ in range(2):
        st, W = dev.solve(lib, T, n, dout, washout, lam)
        assert st == sp.SPIRES_OK
        assert np.all(np.isfinite(W))
        # the tolerances of the allocating ridge against the same oracle
        fit = phi[washout:]
        assert rel(fit @ W.T, fit @ Wo.T) < 1e-9
        assert rel(W, Wo) < (1e-9 if lam >= 1e-2 else 1e-5)
    assert lib.spires_ext_test_live_device_allocs() == live


def test_noalloc_ridge_matches_train_ridge():
    lib = sp.load()
    n, din, dout, T, lam = 300, 2, 3, 600, 1e-4
    cfg, u, y = _states(n, din, dout, T, seed=5)
    r = sp.Reservoir(cfg, seed=41)
    opts = sp.RidgeOpts(0, 30, 1e-13, 0)
    rep = sp.RidgeReport()
    assert lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), T, lam, C.byref(opts),
                                      C.byref(rep)) == sp.SPIRES_OK
    W_ref = r.readout()
    r.reset()  # the same states, recorded from the same reset
    phi, _, _ = r.run_record(u, raster=False)
    r.close()
    dev = _Dev(phi, y, dout, n)
    for _ in range(2):
        st, W = dev.solve(lib, T, n, dout, 0, lam)
        assert st == sp.SPIRES_OK
        assert np.allclose(W, W_ref, rtol=1e-12, atol=1e-12 * np.abs(W_ref).max())


def test_noalloc_ridge_singular_and_sizes():
    lib = sp.load()
    n, dout, T = 200, 2, 300
    rng = np.random.default_rng(7)
    phi = rng.standard_normal((T, n))
    phi[:, 17] = 0.0  # a neuron that never moves: with lambda = 0, singular
    y = rng.standard_normal((T, dout))
    dev = _Dev(phi, y, dout, n)
    for _ in range(2):
        st, W = dev.solve(lib, T, n, dout, 0, 0.0, fill=123.0)
        assert st == sp.SPIRES_ERR_INTERNAL
        assert np.all(W == 123.0)  # the output buffer was not written
    # the same states with lambda > 0 solve, after the failed calls
    st, W = dev.solve(lib, T, n, dout, 10, 1e-3)
    assert st == sp.SPIRES_OK
    Wo = O.oracle_ridge(phi, y, 1e-3, washout=10)
    assert rel(W, Wo) < 1e-9
    # sizes beyond the fixed work area, and bad arguments, are refused before
    # any device work
    p, s = _Dev.ptr, dev.stream
    for args in ((T, 513, dout, 0), (16385, n, dout, 0), (T, n, 17, 0), (T, n, dout, T),
                 (0, n, dout, 0)):
        assert lib.spires_ext_ridge_solve_noalloc(p(dev.phi), p(dev.y), *args, 1e-3, p(dev.w),
                                                  s) == sp.SPIRES_ERR_INVALID_ARG
