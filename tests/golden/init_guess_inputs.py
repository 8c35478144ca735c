"""Seeded inputs of golden_init_guess.npz, shared by make_golden.py (which feeds them to the reference) and the
tests (which regenerate them instead of storing the volumes, and check their SHA-256 against the fixture)."""

from __future__ import annotations

import hashlib

import numpy as np

from pyaldvc_b200 import synthetic as syn

PC_SHAPE = (60, 72, 84)
PC_T = (6.3, -9.6, 4.2)
PY_SHAPE = (96, 96, 96)
PY_F = np.array([[0.0, 0.01, 0.0], [0.0, 0.0, 0.0], [0.008, 0.0, 0.0]])
PY_T = np.array([5.4, -7.2, 9.7])
PY_SUBSET = (16, 16, 16)
PY_RADIUS = (12, 12, 12)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def raw_pc_pair():
    return syn.bead_pair(PC_SHAPE, density=0.03, sigma=1.5, seed=32, disp=syn.translation(PC_T), noise=0.01)


def raw_py_pair():
    return syn.bead_pair(PY_SHAPE, density=0.03, sigma=1.5, seed=33, disp=syn.affine(PY_F, PY_T, (47.5, 47.5, 47.5)), noise=0.01)


def normalised(pair):
    return syn.normalize_volume(pair.f), syn.normalize_volume(pair.g)
