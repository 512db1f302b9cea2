"""The CUDA library against the golden fixtures generated from the reference
compiled from source: small cases bit for bit, and the FP64 FLIF_GL
configurations over their full horizon (spike-raster sha256 per 500-step block
and per step, so that a mismatch names its step, and the final state)."""
import hashlib
import os

import numpy as np
import pytest

import spires_b200 as sp
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(__file__), "golden")
SMALL = np.load(os.path.join(HERE, "small_cases.npz"))
LONG = np.load(os.path.join(HERE, "long_horizon.npz"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", G.SMALL, ids=[c[0] for c in G.SMALL])
def test_small_cases_match_golden(case):
    name = case[0]
    seed, useed = SMALL[name + ":seeds"]
    cfg = G.config(case)
    u = G.small_inputs(G.SMALL_T, case[2], int(useed))
    r = sp.Reservoir(cfg, seed=int(seed))
    assert sha(r.weights()) == str(SMALL[name + ":W_sha"])
    assert sha(r.readout()) == str(SMALL[name + ":Wout_sha"])
    phi, R, _ = r.run_record(u)
    ras = sp.unpack_raster(R, r.n)
    assert np.array_equal(np.packbits(ras, axis=1), SMALL[name + ":raster"])
    assert sha(phi) == str(SMALL[name + ":phi_sha"])
    r.reset()
    Y = r.run(u[:20])
    Yg = SMALL[name + ":run_Y"]
    assert np.all(np.abs(Y - Yg) <= 1e-12 * (np.abs(phi).sum(axis=1).max() + 1))
    r.close()


@pytest.mark.parametrize("case", G.LONG, ids=[c[0] for c in G.LONG])
def test_full_horizon_rasters_match_golden(case):
    name, n, L, topo, conn, din, rho, alpha, T, seed = case
    cfg = G.long_config(case)
    u = G.long_inputs(case)
    assert sha(u) == str(LONG[name + ":u_sha"])
    r = sp.Reservoir(cfg, seed=seed)
    hashes = []
    steps = np.empty(T, np.uint32)
    for b0 in range(0, T, G.BLOCK):
        _, R, _ = r.run_record(u[b0:b0 + G.BLOCK], phi=False)
        packed = np.packbits(sp.unpack_raster(R, n), axis=1)
        hashes.append(sha(packed))
        for j in range(packed.shape[0]):
            steps[b0 + j] = G.step_hash(packed[j])
    V = r.state()
    r.close()
    want = [str(h) for h in LONG[name + ":block_sha"]]
    assert len(want) == len(hashes)
    bad = np.flatnonzero(steps != LONG[name + ":step_hash"])
    assert bad.size == 0, f"first step whose spike raster differs: {int(bad[0])} (of {T})"
    assert hashes == want
    assert np.array_equal(V[:64], LONG[name + ":V_final_head"])
    assert sha(V) == str(LONG[name + ":V_final_sha"])
