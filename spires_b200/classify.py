"""Sequence classification with a large reservoir.

Every sequence of multi-channel input runs through the same reservoir from
its reset state (as the reference's spoken-digit example resets between
utterances), its states are averaged over time, and a 10-way ridge
classifier is fitted on the averaged states of the training sequences
(one-hot targets, arg-max decision). With 20000 neurons and a few hundred
training sequences the ridge is solved in its dual form (a sequences x
sequences system), which the report states.
"""
from __future__ import annotations

import time

import numpy as np

from . import CONN_SCALE_FREE, FLIF_GL, Reservoir, make_config, ridge_fit
from .datasets import bursty_sinusoids

GL_C2 = (1.0, 0.0, 0.0, 20.0, 0.6, 1024.0, 0.1, 2.0)  # alpha 0.6, L = 1024 at dt = 1


def reservoir_config(n=20000, din=13, classes=10, gamma=0.5):
    return make_config(n, din, classes, rho=0.9, ei=0.5, gamma=gamma, conn=5.0 / (n - 1),
                       dt=1.0, topo=CONN_SCALE_FREE, neuron=FLIF_GL, nparams=GL_C2)


def time_averaged_states(r: Reservoir, seqs):
    feats = np.empty((len(seqs), r.n))
    steps = 0
    for k, s in enumerate(seqs):
        r.reset()
        phi, _, _ = r.run_record(s, phi=True, raster=False)
        feats[k] = phi.mean(axis=0)
        steps += s.shape[0]
    return feats, steps


def run_classification(n=20000, num_seq=500, classes=10, seed=0, res_seed=1234, lam=10.0,
                       train_frac=0.8, gram_mode=0, gamma=0.1, offset_span=0.05):
    """Class frequency offsets of +-offset_span: with the default 0.015 of the
    streaming input the classes are not separable even from per-channel
    spectral features, at 0.05 they are (about 0.4 accuracy for a linear
    classifier on power and lag-1 features)."""
    seqs, labels = bursty_sinusoids(num_seq=num_seq, classes=classes, seed=seed,
                                    offset_span=offset_span)
    cfg = reservoir_config(n=n, din=seqs[0].shape[1], classes=classes, gamma=gamma)
    r = Reservoir(cfg, seed=res_seed)
    t0 = time.perf_counter()
    feats, steps = time_averaged_states(r, seqs)
    t1 = time.perf_counter()
    r.close()
    ntr = int(train_frac * num_seq)
    Y = np.eye(classes)[labels]
    W, rep = ridge_fit(feats[:ntr], Y[:ntr], lam, gram_mode=gram_mode)
    t2 = time.perf_counter()
    pred = np.argmax(feats[ntr:] @ W.T, axis=1)
    acc = float(np.mean(pred == labels[ntr:]))
    train_acc = float(np.mean(np.argmax(feats[:ntr] @ W.T, axis=1) == labels[:ntr]))
    return {"accuracy": acc, "train_accuracy": train_acc, "chance": 1.0 / classes,
            "neuron_steps": float(n) * steps, "states_s": t1 - t0, "ridge_s": t2 - t1,
            "dual": int(rep.dual), "rel_residual": rep.rel_residual, "sequences": num_seq,
            "train_sequences": ntr}
