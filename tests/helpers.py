"""Shared constants and fixture loaders for the test suite."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

# Parity bound: max|y - ref| / max|x| per array (2e-6, the project's stated tolerance).
TOL = 2e-6
# The reference's own normwise gate (docs/API.md:49, tests/verify_plan.py:32): Frobenius
# error relative to the input norm.
FROB = 2e-5
SIZES = (8, 16, 32, 64, 128, 256, 512, 1024)
SHAPES = [(h, w) for h in SIZES for w in SIZES]


def golden(name: str):
    return np.load(GOLDEN / name, allow_pickle=False)


def corpus_files():
    return sorted(GOLDEN.glob("corpus_*.npz"), key=lambda p: int(p.stem.split("_")[1]))


def verify_files():
    return sorted(GOLDEN.glob("verify_*.npz"))


def frob_rel(y, ref, x) -> float:
    y = np.asarray(y, np.float64)
    ref = np.asarray(ref, np.float64)
    n = float(np.linalg.norm(np.asarray(x, np.float64)))
    e = float(np.linalg.norm(y - ref))
    return e / n if n else e


def verify_families(h: int, w: int, rng) -> np.ndarray:
    """The six input families of the reference's tests/verify_plan.py:21-28."""
    random = rng.normal(size=(h, w)).astype(np.float32)
    alt = np.where(np.indices((h, w)).sum(axis=0) % 2, 1.0, -1.0).astype(np.float32)
    impulse = np.zeros((h, w), np.float32)
    impulse[h // 3, w // 2] = 1
    return np.stack([np.zeros_like(impulse), impulse, random, (1 + alt * 2 ** -23).astype(np.float32),
                     (random * 2.0 ** -70).astype(np.float32), (random * 2.0 ** 50).astype(np.float32)])
