"""Generate the golden fixtures in this directory from the reference spires C
sources compiled unchanged (oracle/_ref/libspires_ref.so, netlib-order BLAS).

Run where the reference sources are available (builds oracle/_ref if needed):

    python tests/golden/make_golden.py

Fixtures (all small):
  small_cases.npz   -- per case: config, seed, input seed; sha256 of the dense
                       W and of W_out after create; per-step spike rasters
                       (bit-packed), final membrane potentials, sha256 of the
                       state trajectory, readouts of spires_run
  long_horizon.npz  -- FLIF_GL reservoirs run for thousands of steps: sha256
                       of the spike raster of every 500-step block, the first
                       32 bits of the sha256 of every step's raster row (so a
                       mismatch is located to its step) and the sha256 of the
                       final state (full-horizon raster parity). The N=20000,
                       L=1024 pin covers the ring fill (1032 steps) plus
                       25 launches of 256 steps: 7432 steps.
Inputs are regenerated from their seeds by spires_b200.datasets / numpy; the
sha256 of each input series is stored and checked before use.
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import spires_b200 as sp  # noqa: E402
from spires_b200 import datasets  # noqa: E402
from tests import _oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# name, n, din, dout, rho, ei, gamma, conn, dt, topo, neuron, nparams, synapse, backend, sparams
SMALL = [
    ("lif_discrete_er", 96, 2, 2, 1.3, 0.55, 1.2, 0.08, 1.0, 0, 0, (0.0, 1.0, 0.3, 0.05), 0, 0, None),
    ("lif_bio_psc_hom", 96, 2, 2, 1.3, 0.55, 1.2, 0.08, 1.0, 0, 1, (0.0, 1.0, 5.0, 0.85), 1, 0, (3.0,)),
    ("flif_caputo_frac", 96, 2, 2, 1.3, 0.55, 1.2, 0.08, 1.0, 0, 2,
     (1.0, 0.2, 0.0, 1.0, 0.0, 1.5, 0.7, 2.0, 40.0), 3, 0, (0.6, 4.0, 20.0)),
    ("flif_gl_simple_sw", 120, 2, 2, 1.3, 0.55, 1.2, 6 / 119, 1.0, 1, 3,
     (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0), 0, 0, None),
    ("flif_gl_psc_het_ba", 120, 2, 2, 1.3, 0.55, 1.2, 3 / 119, 1.0, 2, 3,
     (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0), 2, 0, (1.0, 10.0)),
    ("flif_gl_mexp_dense", 80, 2, 2, 1.3, 0.55, 1.2, 0.1, 1.0, 0, 3,
     (1.0, 0.0, 0.0, 20.0, 0.7, 32.0, 0.1, 2.0), 4, 1, (0.5, 4.0, 1.0, 40.0, 5)),
    ("flif_gl_microsteps", 64, 1, 1, 1.3, 0.55, 1.2, 0.1, 0.25, 0, 3,
     (1.0, 0.0, 0.0, 20.0, 0.7, 16.0, 0.1, 0.5), 1, 0, (2.0,)),
    ("flif_diffusive_det", 96, 2, 2, 1.3, 0.55, 1.2, 0.08, 1.0, 0, 4,
     (1.0, 0.0, 0.0, 5.0, 1.0, 3.0, 0.85), 0, 0, None),
]
SMALL_T = 80


def config(c):
    (name, n, din, dout, rho, ei, gamma, conn, dt, topo, neuron, npar, syn, be, spar) = c
    return sp.make_config(n, din, dout, rho=rho, ei=ei, gamma=gamma, conn=conn, dt=dt, topo=topo,
                          neuron=neuron, nparams=npar, synapse=syn, backend=be, sparams=spar)


def small_inputs(T, din, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.5, size=(T, din))


def make_small(ref):
    out = {}
    for k, c in enumerate(SMALL):
        name = c[0]
        cfg = config(c)
        seed, useed = 1000 + k, 2000 + k
        u = small_inputs(SMALL_T, c[2], useed)
        r = sp.Reservoir(cfg, lib=ref, seed=seed)
        W, Wout = r.weights(), r.readout()
        phi = np.empty((SMALL_T, r.n))
        ras = np.empty((SMALL_T, r.n), np.uint8)
        for t in range(SMALL_T):
            r.step(u[t])
            phi[t] = r.state()
            ras[t] = r.spikes() != 0.0
        r.reset()
        Y = r.run(u[:20])
        r.close()
        out[name + ":seeds"] = np.array([seed, useed])
        out[name + ":u_sha"] = np.array(sha(u))
        out[name + ":W_sha"] = np.array(sha(W))
        out[name + ":Wout_sha"] = np.array(sha(Wout))
        out[name + ":raster"] = np.packbits(ras, axis=1)
        out[name + ":V_final"] = phi[-1]
        out[name + ":phi_sha"] = np.array(sha(phi))
        out[name + ":run_Y"] = Y
        print(f"{name}: spike rate {ras.mean():.3f}")
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **out)


# long-horizon FLIF_GL pins: (name, n, L, topo, conn, din, rho, alpha, T, seed)
LONG = [
    ("gl_n4000_l512_ws", 4000, 512, 1, 10 / 3999, 1, 0.95, 0.7, 20000, 42),
    ("gl_n20000_l1024_ba", 20000, 1024, 2, 5 / 19999, 13, 0.9, 0.6, 1032 + 25 * 256, 1234),
]
BLOCK = 500


def long_config(c):
    name, n, L, topo, conn, din, rho, alpha, T, seed = c
    return sp.make_config(n, din, 1 if din == 1 else 10, rho=rho, ei=0.5, gamma=0.5, conn=conn,
                          dt=1.0, topo=topo, neuron=sp.FLIF_GL,
                          nparams=(1.0, 0.0, 0.0, 20.0, alpha, float(L), 0.1, 2.0))


def long_inputs(c):
    name, n, L, topo, conn, din, rho, alpha, T, seed = c
    if din == 1:
        return datasets.mackey_glass(T + 1, seed=0)[:T, None].copy()
    seqs, _ = datasets.bursty_sinusoids(num_seq=T // 40 + 4, seed=7)
    return np.ascontiguousarray(np.concatenate(seqs, axis=0)[:T])


def step_hash(packed_row):
    """First 32 bits of the sha256 of one step's bit-packed raster row."""
    return np.uint32(int(hashlib.sha256(packed_row.tobytes()).hexdigest()[:8], 16))


def make_long(ref):
    out = {}
    for c in LONG:
        name, n, L, topo, conn, din, rho, alpha, T, seed = c
        t0 = time.time()
        cfg = long_config(c)
        u = long_inputs(c)
        r = sp.Reservoir(cfg, lib=ref, seed=seed)
        spk = np.empty(n)
        ras = np.empty((BLOCK, n), np.uint8)
        hashes = []
        steps = np.empty(T, np.uint32)
        rate = 0.0
        for t in range(T):
            r.step(u[t])
            r.lib.spires_read_spike_state(r.h, sp.dptr(spk))
            ras[t % BLOCK] = spk != 0.0
            steps[t] = step_hash(np.packbits(ras[t % BLOCK]))
            if (t + 1) % BLOCK == 0 or t + 1 == T:
                m = (t % BLOCK) + 1
                blk = np.packbits(ras[:m], axis=1)
                hashes.append(sha(blk))
                rate += ras[:m].sum()
        V = r.state()
        r.close()
        out[name + ":u_sha"] = np.array(sha(u))
        out[name + ":block_sha"] = np.array(hashes)
        out[name + ":step_hash"] = steps
        out[name + ":V_final_sha"] = np.array(sha(V))
        out[name + ":V_final_head"] = V[:64]
        print(f"{name}: T={T} rate={rate / (T * n):.4f} ({time.time() - t0:.1f}s)")
    np.savez_compressed(os.path.join(HERE, "long_horizon.npz"), **out)


if __name__ == "__main__":
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    ref = O.ref_lib("netlib")
    make_small(ref)
    if "--small-only" not in sys.argv:
        make_long(ref)
