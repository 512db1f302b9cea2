"""AGILE search core against the reference's agile_optimize (src/agile.c),
step for step on a deterministic objective: same evaluations, same best point.
CPU only (the objective is a Python callback)."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="reference build absent")


def objective_factory(log):
    def f(theta, dim, ctx):
        x = np.ctypeslib.as_array(theta, shape=(dim,)).copy()
        log.append(x)
        # shifted Rosenbrock-like valley with a ridge term: several basins
        v = sum(100.0 * (x[i + 1] - x[i] ** 2) ** 2 + (1.0 - x[i]) ** 2 for i in range(dim - 1))
        return float(v + 0.3 * np.sin(3.0 * x).sum())
    return f


@pytest.mark.parametrize("reflect,seed", [(1, 0xA91E), (0, 12345), (1, 0)])
def test_agile_matches_reference(reflect, seed):
    dim = 4
    th0 = (C.c_double * dim)(0.3, -0.5, 0.8, 0.1)
    lo = (C.c_double * dim)(*([-1.5] * dim))
    hi = (C.c_double * dim)(*([1.5] * dim))
    opts = sp.AgileOpts(1.3, 1e-3, 0.3, 20.0, 0.9, 1e-3, 60, 15, 1e-3, reflect, seed, 0)

    def run(lib):
        log = []
        cb = sp.LOSS_FN(objective_factory(log))
        best = (C.c_double * dim)()
        rep = sp.AgileReport()
        if lib is None:
            st = sp.load().spires_ext_agile_minimize(th0, lo, hi, dim, cb, None, C.byref(opts),
                                                     best, C.byref(rep))
            assert st == 0
        else:
            f = lib.agile_optimize
            f.restype = C.c_int
            f.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_int, sp.LOSS_FN, C.c_void_p,
                                                          C.c_void_p, C.POINTER(sp.AgileOpts),
                                                          C.POINTER(C.c_double),
                                                          C.POINTER(sp.AgileReport)]
            assert f(th0, lo, hi, dim, cb, None, None, C.byref(opts), best, C.byref(rep)) == 0
        return np.array(best[:]), rep, np.array(log)

    b1, r1, l1 = run(None)
    b2, r2, l2 = run(O.ref_lib())
    assert l1.shape == l2.shape and np.array_equal(l1, l2), "evaluation sequences differ"
    assert np.array_equal(b1, b2)
    assert (r1.best_loss, r1.best_iter, r1.total_evals, r1.total_iters, r1.exited_refinement) == \
        (r2.best_loss, r2.best_iter, r2.total_evals, r2.total_iters, r2.exited_refinement)
