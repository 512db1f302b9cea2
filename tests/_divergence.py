"""First-divergence report between this library and a compiled build of the
reference (test infrastructure; the reference is the checker).

The reference's results depend on the BLAS it is linked with: its external
drive is one dgemv, ext = gamma * W_in u (src/reservoir.c:132-136), whose
summation order (and use of fused multiply-add) is the BLAS's own. This
library follows the netlib order, so it is bit-identical to the reference
built against the netlib-order shim; against the reference linked to
OpenBLAS the membrane potentials can differ in their last bit from the first
step on, and a spike raster can then differ once such a difference crosses a
threshold. `first_divergence` runs both from the same seeded creation and
reports where the trajectories first differ: the first step and neuron whose
state bits differ, the largest relative state difference before the rasters
split, and the first step and neuron whose spike differs.
"""
import numpy as np

import spires_b200 as sp
from tests import _oracle as O


def first_divergence(cfg, seed, u, ref_kind="openblas", chunk=256, stop_at_raster=True):
    n = int(cfg.num_neurons)
    T = int(u.shape[0])
    gpu = sp.Reservoir(cfg, seed=seed)
    ref = sp.Reservoir(cfg, lib=O.ref_lib(ref_kind), seed=seed)
    # dense W only where it is small; the readout (drawn after W and W_in
    # from the same rand() stream) always
    same = np.array_equal(gpu.readout().view(np.uint64), ref.readout().view(np.uint64))
    if n <= 5000:
        same = same and np.array_equal(gpu.weights().view(np.uint64),
                                       ref.weights().view(np.uint64))
    rep = {
        "reference": ref_kind, "neurons": n, "steps_compared": 0,
        "weights_identical": bool(same),
        "first_state_step": None, "first_state_neuron": None,
        "first_raster_step": None, "first_raster_neuron": None,
        "max_rel_state_diff_before_raster": 0.0, "state_rows_differing": 0,
    }
    spk = np.empty(n)
    for t0 in range(0, T, chunk):
        t1 = min(T, t0 + chunk)
        phi, R, _ = gpu.run_record(u[t0:t1])
        ras = sp.unpack_raster(R, n)
        for j in range(t1 - t0):
            t = t0 + j
            ref.step(u[t])
            v = ref.state()
            ref.lib.spires_read_spike_state(ref.h, sp.dptr(spk))
            s = spk != 0.0
            dv = phi[j].view(np.uint64) != v.view(np.uint64)
            if dv.any():
                rep["state_rows_differing"] += 1
                if rep["first_state_step"] is None:
                    rep["first_state_step"] = t
                    rep["first_state_neuron"] = int(np.flatnonzero(dv)[0])
            ds = ras[j].astype(bool) != s
            if ds.any() and rep["first_raster_step"] is None:
                rep["first_raster_step"] = t
                rep["first_raster_neuron"] = int(np.flatnonzero(ds)[0])
            if rep["first_raster_step"] is None:
                scale = np.maximum(np.abs(v), 1e-300)
                rel = float(np.max(np.abs(phi[j] - v) / scale))
                rep["max_rel_state_diff_before_raster"] = max(
                    rep["max_rel_state_diff_before_raster"], rel)
            rep["steps_compared"] = t + 1
            if stop_at_raster and rep["first_raster_step"] is not None:
                break
        if stop_at_raster and rep["first_raster_step"] is not None:
            break
    gpu.close()
    ref.close()
    return rep


# the two FP64 FLIF_GL workloads whose reports the tests produce
def flif_gl_n4000_l512_ws():
    """FLIF_GL N=4000, L=512, Watts-Strogatz k=10, rho 0.95, Mackey-Glass input."""
    from spires_b200 import datasets
    cfg = sp.make_config(4000, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10 / 3999, dt=1.0,
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0))
    u = datasets.mackey_glass(20001, seed=0)[:20000, None].copy()
    return cfg, 42, u


def flif_gl_n20000_l1024_ba():
    """FLIF_GL N=20000, L=1024, alpha 0.6, Barabasi-Albert m=5, rho 0.9,
    13-channel bursty sinusoids."""
    from spires_b200 import datasets
    cfg = sp.make_config(20000, 13, 10, rho=0.9, ei=0.5, gamma=0.5, conn=5 / 19999, dt=1.0,
                         topo=sp.CONN_SCALE_FREE, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.6, 1024.0, 0.1, 2.0))
    seqs, _ = datasets.bursty_sinusoids(num_seq=7432 // 40 + 4, seed=7)
    u = np.ascontiguousarray(np.concatenate(seqs, axis=0)[:7432])
    return cfg, 1234, u
