"""CKKS parameter presets and configuration.

Mirrors the reference's ``fhelium.config.ckks`` surface (``Preset`` and
``CkksConfig``; fhelium/config/ckks.py:26-158,161-649): the same sixteen
preset names and values, the same modulus order ``[scale q..., base q, p...]``
(ckks.py:504-535), the int32 <-> 30-bit / int64 <-> 62-bit buffer rule
(ckks.py:326-328) and the Montgomery bound ``4q < 2^w`` (ckks.py:526-534).
The primes come from the reference's packaged catalog, exported verbatim to
``data/prime_catalog_v1.json``.  The exact-table security-budget assessment of
the reference (fhelium/config/security.py) is not on the evaluation path and
is not rebuilt; maintained presets carry fixed prime counts, so it does not
change any modulus.
"""

from __future__ import annotations

import json
import math
import os
from enum import Enum
from functools import cached_property, lru_cache
from typing import Any, Mapping

import torch


class Preset(Enum):
    """Maintained CKKS parameter baselines (name = slots, scale bits, levels, dtype)."""

    slots8192_scale30_levels9_int64 = "slots8192-scale30-levels9-int64"
    slots8192_scale40_levels7_int64 = "slots8192-scale40-levels7-int64"
    slots8192_scale50_levels5_int64 = "slots8192-scale50-levels5-int64"
    slots16384_scale30_levels21_int64 = "slots16384-scale30-levels21-int64"
    slots16384_scale40_levels16_int64 = "slots16384-scale40-levels16-int64"
    slots16384_scale50_levels12_int64 = "slots16384-scale50-levels12-int64"
    slots32768_scale30_levels45_int64 = "slots32768-scale30-levels45-int64"
    slots32768_scale40_levels34_int64 = "slots32768-scale40-levels34-int64"
    slots32768_scale50_levels27_int64 = "slots32768-scale50-levels27-int64"
    slots65536_scale30_levels95_int64 = "slots65536-scale30-levels95-int64"
    slots65536_scale40_levels72_int64 = "slots65536-scale40-levels72-int64"
    slots65536_scale50_levels58_int64 = "slots65536-scale50-levels58-int64"
    slots8192_scale25_levels14_int32 = "slots8192-scale25-levels14-int32"
    slots16384_scale25_levels29_int32 = "slots16384-scale25-levels29-int32"
    slots32768_scale25_levels24_int32 = "slots32768-scale25-levels24-int32"
    slots65536_scale25_levels14_int32 = "slots65536-scale25-levels14-int32"


def _preset_fields(preset: Preset) -> dict[str, int]:
    # The preset name encodes slots, scale bits, public levels and dtype; the
    # P-prime count depends on the ring only (1, 2, 4, 6 for logN 14..17).
    _, slots, scale, levels, dtype = preset.name.replace("slots", "slots_").split("_")
    log_n = int(slots).bit_length()  # slots = N/2
    fields = {
        "logN": log_n,
        "scale_bits": int(scale.removeprefix("scale")),
        "num_scale_primes": int(levels.removeprefix("levels")),
        "num_p_primes": {14: 1, 15: 2, 16: 4, 17: 6}[log_n],
    }
    if dtype == "int32":
        fields["buffer_bit_length"] = 30
    return fields


@lru_cache(maxsize=1)
def prime_catalog() -> dict[str, dict[tuple[int, int], tuple[int, ...]]]:
    path = os.path.join(os.path.dirname(__file__), "data", "prime_catalog_v1.json")
    with open(path) as fh:
        raw = json.load(fh)
    out = {}
    for kind in ("scale", "message"):
        out[kind] = {
            tuple(int(v) for v in key.split(":")): tuple(primes)
            for key, primes in raw[kind].items()
        }
    return out


def int32_ntt_primes(count: int = 36, log_n: int = 16) -> list[int]:
    """The first `count` distinct catalog primes with 4q < 2^30 and q = 1 mod 2N
    from the int32 families (25-bit scale primes, then 28-bit message primes):
    the limb set of the standalone int32 NTT workload (N = 2^16, 36 limbs)."""
    cat = prime_catalog()
    n = 1 << log_n
    out: list[int] = []
    for q in list(cat["scale"][(25, n)]) + list(cat["message"][(28, n)]):
        if q not in out and 4 * q < 2 ** 30 and (q - 1) % (2 * n) == 0:
            out.append(q)
    return out[:count]


class CkksConfig:
    r"""Immutable CKKS parameters over $\mathbb{Z}[X]/(X^N+1)$.

    ``moduli`` is ``[scale primes, structural base prime, P primes]``.  Public
    level ``l`` keeps Q rows ``[l, num_q_primes)``.
    """

    def __init__(
        self,
        *,
        buffer_bit_length: int = 62,
        scale_bits: int = 40,
        base_prime_bits: int | None = None,
        logN: int = 15,
        num_scale_primes: int = 16,
        num_p_primes: int = 2,
        sigma: float = 3.19,
        security_bits: int = 128,
        enforce_security_budget: bool = True,
    ):
        if buffer_bit_length not in (30, 62):
            raise ValueError("buffer_bit_length must be 32-2=30 or 64-2=62.")
        if type(num_scale_primes) is not int or num_scale_primes < 1:
            raise ValueError("num_scale_primes must be a positive integer")
        if num_p_primes < 1:
            raise ValueError("key switching requires at least one P prime")
        sigma = float(sigma)
        if not math.isfinite(sigma) or sigma <= 0.0:
            raise ValueError("sigma must be positive and finite")
        self.__dict__.update(
            buffer_bit_length=buffer_bit_length,
            scale_bits=scale_bits,
            base_prime_bits=base_prime_bits,
            logN=logN,
            num_scale_primes=num_scale_primes,
            num_p_primes=num_p_primes,
            sigma=sigma,
            security_bits=security_bits,
            enforce_security_budget=enforce_security_budget,
        )
        self.__dict__["_frozen"] = True
        _ = self.moduli  # validate eagerly

    def __setattr__(self, name: str, value: object) -> None:
        if self.__dict__.get("_frozen") and not name.startswith("_cache"):
            raise AttributeError("CkksConfig is immutable; construct a new config")
        object.__setattr__(self, name, value)

    @classmethod
    def parse(cls, src: Mapping[str, Any] | Preset | str, **overrides: Any) -> "CkksConfig":
        if isinstance(src, str):
            src = Preset(src) if src in {p.value for p in Preset} else Preset[src]
        base = _preset_fields(src) if isinstance(src, Preset) else dict(src)
        return cls(**{**base, **overrides})

    def dumps(self) -> dict[str, object]:
        return {k: self.__dict__[k] for k in (
            "buffer_bit_length", "scale_bits", "base_prime_bits", "logN",
            "num_scale_primes", "num_p_primes", "sigma", "security_bits",
            "enforce_security_budget")}

    # ---- derived ---------------------------------------------------------
    @cached_property
    def N(self) -> int:
        return 1 << self.logN

    @cached_property
    def num_slots(self) -> int:
        return self.N // 2

    @cached_property
    def torch_dtype(self) -> torch.dtype:
        return {30: torch.int32, 62: torch.int64}[self.buffer_bit_length]

    @cached_property
    def message_bits(self) -> int:
        return self.buffer_bit_length - 2

    @cached_property
    def int_scale(self) -> int:
        return 1 << self.scale_bits

    @cached_property
    def default_scale(self) -> float:
        return float(self.int_scale)

    @cached_property
    def _scale_primes(self) -> tuple[int, ...]:
        try:
            return prime_catalog()["scale"][(self.scale_bits, self.N)]
        except KeyError:
            raise ValueError(f"no scale primes for scale_bits={self.scale_bits}, N={self.N}")

    @cached_property
    def _message_primes(self) -> tuple[int, ...]:
        try:
            return prime_catalog()["message"][(self.message_bits, self.N)]
        except KeyError:
            raise ValueError(f"no message primes for bits={self.message_bits}, N={self.N}")

    @cached_property
    def _base_and_p_primes(self) -> tuple[int, ...]:
        # Default: first message-width prime is the structural base, the next
        # num_p ones are P.  With base_prime_bits == scale_bits the base is the
        # last scale-catalog prime and P stays message-width
        # (fhelium/config/ckks.py:_base_and_p_primes).
        if self.base_prime_bits is not None:
            if self.base_prime_bits != self.scale_bits:
                raise ValueError("base_prime_bits must equal scale_bits")
            p = self._message_primes[: self.num_p_primes]
            if len(p) != self.num_p_primes:
                raise ValueError("prime catalog has too few P primes")
            return (self._scale_primes[-1], *p)
        need = 1 + self.num_p_primes
        primes = self._message_primes[:need]
        if len(primes) != need:
            raise ValueError("prime catalog has too few base/P primes")
        return tuple(primes)

    @cached_property
    def moduli(self) -> tuple[int, ...]:
        scale = self._scale_primes[: self.num_scale_primes]
        if len(scale) != self.num_scale_primes:
            raise ValueError("prime catalog has too few scale primes")
        moduli = tuple(scale) + self._base_and_p_primes
        if len(set(moduli)) != len(moduli):
            raise ValueError("modulus chain contains duplicate primes")
        radix = 1 << self.buffer_bit_length
        for i, q in enumerate(moduli):
            if 4 * q >= radix:
                raise ValueError(
                    f"modulus at prime_id {i} violates 4 * modulus < 2**buffer_bit_length")
        return moduli

    @cached_property
    def num_q_primes(self) -> int:
        return self.num_scale_primes + 1

    @cached_property
    def q_moduli(self) -> tuple[int, ...]:
        return self.moduli[: self.num_q_primes]

    @cached_property
    def p_moduli(self) -> tuple[int, ...]:
        return self.moduli[self.num_q_primes:]

    @cached_property
    def public_level_count(self) -> int:
        return self.num_scale_primes

    @cached_property
    def inverse_ntt_scale(self) -> tuple[int, ...]:
        return tuple(pow(self.N, -1, q) for q in self.moduli)

    def __repr__(self) -> str:
        return (f"CkksConfig(logN={self.logN}, Q={self.num_q_primes}, P={self.num_p_primes}, "
                f"scale_bits={self.scale_bits}, buffer_bit_length={self.buffer_bit_length})")
