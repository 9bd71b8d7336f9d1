"""Seeded inputs shared by the golden-fixture generator and the tests.

Every input is drawn with numpy's PCG64 (np.random.default_rng(seed)), so the
generator (run once against the reference) and the tests (run anywhere)
rebuild identical residues from the seeds recorded in the fixture.
"""

from __future__ import annotations

import hashlib

import numpy as np


def residues(seed: int, moduli, prime_ids, shape_prefix, n: int, lazy: bool = False) -> np.ndarray:
    rng = np.random.default_rng(seed)
    q = np.array([moduli[i] for i in prime_ids], dtype=np.int64)
    bound = (2 * q) if lazy else q
    x = rng.integers(0, 1 << 62, size=(*shape_prefix, len(prime_ids), n), dtype=np.int64)
    return (x % bound[:, None]).astype(np.int64)


def key_material(seed: int, moduli, num_q: int, num_p: int, n: int) -> np.ndarray:
    """[digit, 2, QP, N] uniform residues on the level-zero QP rows."""
    digits = len(range(0, num_q - 1, num_p)) + 1
    return residues(seed, moduli, list(range(num_q + num_p)), (digits, 2), n)


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<i8").tobytes()).hexdigest()


def canonical(x: np.ndarray, moduli, prime_ids) -> np.ndarray:
    q = np.array([moduli[i] for i in prime_ids], dtype=np.int64)[:, None]
    return np.mod(np.asarray(x, dtype=np.int64), q)
