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


def small_ints(seed: int, shape, bound: int) -> np.ndarray:
    """Signed integers uniform in [-bound, bound] (encryption draws, plaintexts)."""
    return np.random.default_rng(seed).integers(-bound, bound + 1, size=shape, dtype=np.int64)


def float_digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


def client_inputs(seed: int, moduli, num_q: int, num_p: int, level: int, n: int, batch: int, int32: bool):
    """Inputs of one encrypt + decrypt golden case: public key [2, Q, N] and
    secret key [QP, N] (NTT/Montgomery residues), integer plaintext
    coefficients [batch, N], draws v (ternary), e0, e1 [batch, N], and a
    ciphertext [2, batch, L, N] (coefficient/standard) to decrypt."""
    q_ids = list(range(num_q))
    bound = (1 << 20) if int32 else (1 << 40)
    return {
        "pk": residues(seed, moduli, q_ids, (2,), n),
        "sk": residues(seed + 1, moduli, list(range(num_q + num_p)), (), n),
        "m": small_ints(seed + 2, (batch, n), bound),
        "v": small_ints(seed + 3, (batch, n), 1),
        "e": small_ints(seed + 4, (2, batch, n), 20),
        "ct": residues(seed + 5, moduli, list(range(level, num_q)), (2, batch), n),
    }


def key_draws(seed: int, moduli, num_q: int, num_p: int, n: int):
    """Key-switch key draws: uniform component [D, QP, N] and error [D, N]."""
    digits = len(range(0, num_q - 1, num_p)) + 1
    return (residues(seed, moduli, list(range(num_q + num_p)), (digits,), n),
            small_ints(seed + 1, (digits, n), 20))
