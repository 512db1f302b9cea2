"""The allocation-free ridge solve (spires_ext_ridge_solve_noalloc).

Some callers cannot allocate device memory themselves: a host framework that
hands every device buffer out from its own allocator or quota, or a control
loop that cannot pay for the device-wide synchronisation of cudaMalloc and
cudaFree. For them the library solves a ridge readout from states they already
hold on the device, working in one fixed array that the library owns. This
file runs last so that a failure here leaves every other result in place.
"""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp

pytestmark = pytest.mark.gpu

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0)


def test_ridge_solve_without_allocation_matches_train_ridge():
    import torch

    lib = sp.load()
    n, din, dout, T, lam = 300, 2, 3, 600, 1e-4
    cfg = sp.make_config(n, din, dout, rho=1.2, ei=0.55, gamma=1.2, conn=0.03,
                         topo=sp.CONN_SCALE_FREE, neuron=sp.FLIF_GL, nparams=GL)
    rng = np.random.default_rng(5)
    u = rng.uniform(-1.0, 1.5, size=(T, din))
    y = rng.standard_normal((T, dout))

    # reference result: the allocating entry point (reset, record, FP64 ridge)
    r = sp.Reservoir(cfg, seed=41)
    opts = sp.RidgeOpts(0, 30, 1e-13, 0)
    rep = sp.RidgeReport()
    assert lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), T, lam, C.byref(opts),
                                      C.byref(rep)) == sp.SPIRES_OK
    W_ref = r.readout()
    # the same states, recorded from the same reset
    r.reset()
    phi, _, _ = r.run_record(u, raster=False)
    r.close()

    d_phi = torch.from_numpy(phi).cuda()
    d_y = torch.from_numpy(np.ascontiguousarray(y)).cuda()
    d_w = torch.empty((dout, n), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ptr = lambda t: C.c_void_p(t.data_ptr())
    for _ in range(2):  # the work area keeps the previous call's contents
        d_w.fill_(float("nan"))
        torch.cuda.synchronize()
        st = lib.spires_ext_ridge_solve_noalloc(ptr(d_phi), ptr(d_y), T, n, dout, 0, lam,
                                                ptr(d_w), C.c_void_p(stream))
        assert st == sp.SPIRES_OK
        W = d_w.cpu().numpy()
        assert np.all(np.isfinite(W))
        assert np.allclose(W, W_ref, rtol=1e-12, atol=1e-12 * np.abs(W_ref).max())

    # sizes beyond the fixed work area are refused before any device work
    assert lib.spires_ext_ridge_solve_noalloc(ptr(d_phi), ptr(d_y), T, 513, dout, 0, lam,
                                              ptr(d_w), C.c_void_p(stream)) == \
        sp.SPIRES_ERR_INVALID_ARG
    assert lib.spires_ext_ridge_solve_noalloc(ptr(d_phi), ptr(d_y), 16385, n, dout, 0, lam,
                                              ptr(d_w), C.c_void_p(stream)) == \
        sp.SPIRES_ERR_INVALID_ARG
