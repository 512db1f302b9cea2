"""The oracle and the host construction against the golden fixtures generated
from the reference compiled from source (tests/golden/make_golden.py). CPU
only; runs without the reference sources present."""
import hashlib
import os

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O
from tests.golden import make_golden as G

SMALL = np.load(os.path.join(os.path.dirname(__file__), "golden", "small_cases.npz"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", G.SMALL, ids=[c[0] for c in G.SMALL])
def test_construction_and_oracle_match_golden(case):
    name = case[0]
    seed, useed = SMALL[name + ":seeds"]
    cfg = G.config(case)
    u = G.small_inputs(G.SMALL_T, case[2], int(useed))
    assert sha(u) == str(SMALL[name + ":u_sha"])
    hm = sp.HostModel(cfg, seed=int(seed))
    assert sha(hm.dense()) == str(SMALL[name + ":W_sha"])
    assert sha(hm.w_out()) == str(SMALL[name + ":Wout_sha"])
    orc = O.Oracle(cfg, hm)
    phi, ras, _ = orc.run(u)
    assert np.array_equal(np.packbits(ras, axis=1), SMALL[name + ":raster"])
    assert np.array_equal(phi[-1], SMALL[name + ":V_final"])
    assert sha(phi) == str(SMALL[name + ":phi_sha"])
    orc.reset()
    _, _, Y = orc.run(u[:20], y=True)
    assert np.array_equal(Y[:, :case[3]], SMALL[name + ":run_Y"])
