"""Shared builders for the parity tests (seeded inputs, oracle contexts)."""

from __future__ import annotations

import numpy as np
import torch

from fhelium_b200.config import CkksConfig, Preset
from oracle import oracle as orc


def oracle_for(cfg: CkksConfig, log_n: int | None = None) -> orc.OracleContext:
    return orc.OracleContext(cfg.moduli, log_n or cfg.logN, cfg.num_q_primes, cfg.num_p_primes,
                             cfg.buffer_bit_length, cfg.scale_bits)


def uniform_residues(rng: np.random.Generator, moduli, rows, shape_prefix, n, lazy=False) -> np.ndarray:
    q = np.array([moduli[i] for i in rows], dtype=np.int64)
    bound = 2 * q if lazy else q
    x = rng.integers(0, 1 << 62, size=(*shape_prefix, len(rows), n), dtype=np.int64)
    return (x % bound[:, None]).astype(np.int64)


def random_key(rng, cfg: CkksConfig, n: int) -> np.ndarray:
    """[D, 2, QP, N] uniform key material (any residues are a valid input to
    the deterministic key-switch arithmetic)."""
    qp = cfg.num_q_primes + cfg.num_p_primes
    digits = len(range(0, cfg.num_q_primes - 1, cfg.num_p_primes)) + 1
    return uniform_residues(rng, cfg.moduli, range(qp), (digits, 2), n)


def to_dev(x: np.ndarray, cfg: CkksConfig) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(x)).to(cfg.torch_dtype).cuda()


def to_np(t: torch.Tensor) -> np.ndarray:
    return t.cpu().to(torch.int64).numpy()


def canon(x: np.ndarray, moduli, rows) -> np.ndarray:
    q = np.array([moduli[i] for i in rows], dtype=np.int64)
    return np.mod(x, q[:, None])


CONFIGS = {
    "int64_logn14": lambda: CkksConfig.parse(Preset.slots8192_scale40_levels7_int64),
    "int64_logn16": lambda: CkksConfig.parse(Preset.slots32768_scale40_levels34_int64),
    "int32_logn16": lambda: CkksConfig.parse(Preset.slots32768_scale25_levels24_int32),
    "int32_logn14": lambda: CkksConfig.parse(Preset.slots8192_scale25_levels14_int32),
}


def reduced_ring(cfg: CkksConfig, log_n: int) -> CkksConfig:
    """Same primes on a smaller ring (q = 1 mod 2N still holds)."""
    return _RingView(cfg, log_n)


class _RingView:
    """A CkksConfig stand-in with the same chain and a smaller logN."""

    def __init__(self, cfg: CkksConfig, log_n: int):
        self._cfg = cfg
        self.logN = log_n
        self.N = 1 << log_n

    def __getattr__(self, name):
        return getattr(self._cfg, name)
