"""The seeded synthetic inputs of the workloads: determinism, shapes, value
ranges and the properties the workloads rely on. CPU only."""
import numpy as np

from spires_b200 import datasets


def test_mackey_glass_is_seeded_and_batched():
    a = datasets.mackey_glass(600, seed=3)
    assert a.shape == (600,)
    assert np.array_equal(a, datasets.mackey_glass(600, seed=3))
    assert not np.array_equal(a, datasets.mackey_glass(600, seed=4))
    b = datasets.mackey_glass(600, seed=3, batch=1)
    assert b.shape == (1, 600) and np.array_equal(b[0], a)  # same draws for one series
    c = datasets.mackey_glass(300, seed=3, batch=3)
    assert c.shape == (3, 300)
    assert not np.array_equal(c[0], c[1])


def test_mackey_glass_stays_on_its_attractor():
    x = datasets.mackey_glass(3000, seed=0)
    tail = x[500:]
    assert np.all(np.isfinite(x))
    assert 0.2 < tail.min() and tail.max() < 1.5  # tau = 17: the chaotic band
    assert tail.std() > 0.1                        # not settled on a fixed point
    # no exact period: the tail does not repeat itself at any lag up to 200
    d = [np.max(np.abs(tail[k:] - tail[:-k])) for k in range(1, 200)]
    assert min(d) > 1e-3


def test_bursty_sinusoids_shapes_and_seeding():
    seqs, labels = datasets.bursty_sinusoids(40, channels=5, classes=4, len_min=10, len_max=30,
                                             seed=2)
    assert len(seqs) == 40 and labels.shape == (40,)
    assert set(np.unique(labels)) <= set(range(4))
    for s in seqs:
        assert s.ndim == 2 and s.shape[1] == 5 and 10 <= s.shape[0] <= 30
        assert s.flags["C_CONTIGUOUS"]
    # the burst gate switches channels off: some exact zeros, not all
    flat = np.concatenate([s.ravel() for s in seqs])
    assert 0.05 < np.mean(flat == 0.0) < 0.95
    seqs2, labels2 = datasets.bursty_sinusoids(40, channels=5, classes=4, len_min=10, len_max=30,
                                               seed=2)
    assert np.array_equal(labels, labels2)
    assert all(np.array_equal(x, y) for x, y in zip(seqs, seqs2))


def test_one_step_targets_align():
    x = np.arange(10.0)
    u, y = datasets.one_step_targets(x)
    assert u.shape == (9, 1) and y.shape == (9, 1)
    assert np.array_equal(y[:, 0], u[:, 0] + 1.0)
