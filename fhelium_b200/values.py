"""CKKS value and key containers.

Same tensor layouts as the reference's value types (fhelium/core/
ciphertext.py:26-384, fhelium/core/keys.py:67-345):
  Ciphertext   data [component, *batch, limb, N]
  SecretKey    data [QP limb, N]            NTT/Montgomery
  PublicKey    data [2, Q limb, N]          NTT/Montgomery
  KeySwitchKey data [digit, 2, QP limb, N]  NTT/Montgomery, level-zero rows
Limb j of a level-l value holds the residue modulo prime id l + j.
"""

from __future__ import annotations

from dataclasses import dataclass, field, replace

import torch


@dataclass
class Ciphertext:
    data: torch.Tensor
    level: int
    scale: float
    polynomial_domain: str = "coefficient"  # "coefficient" | "ntt"
    residue_representation: str = "standard"  # "standard" | "montgomery"
    modulus_basis: str = "Q"

    def __post_init__(self):
        if self.data.ndim < 3 or self.data.size(0) not in (2, 3):
            raise ValueError("Ciphertext data must be [component(2|3), *batch, limb, N]")

    @property
    def component_count(self) -> int:
        return self.data.size(0)

    @property
    def batch_shape(self) -> tuple[int, ...]:
        return tuple(self.data.shape[1:-2])

    @property
    def batch_size(self) -> int:
        n = 1
        for d in self.batch_shape:
            n *= d
        return n

    @property
    def limb_count(self) -> int:
        return self.data.size(-2)

    def component(self, i: int) -> torch.Tensor:
        return self.data[i]

    @property
    def c0(self) -> torch.Tensor:
        return self.data[0]

    @property
    def c1(self) -> torch.Tensor:
        return self.data[1]

    @property
    def c2(self) -> torch.Tensor:
        if self.component_count < 3:
            raise ValueError("two-component ciphertext has no c2")
        return self.data[2]

    def clone(self) -> "Ciphertext":
        return replace(self, data=self.data.clone())

    def assert_state(self, *, polynomial_domain: str | None = None, residue_representation: str | None = None,
                     components: int | None = None) -> None:
        if polynomial_domain is not None and self.polynomial_domain != polynomial_domain:
            raise ValueError(f"expected {polynomial_domain} domain, got {self.polynomial_domain}")
        if residue_representation is not None and self.residue_representation != residue_representation:
            raise ValueError(f"expected {residue_representation} residues, got {self.residue_representation}")
        if components is not None and self.component_count != components:
            raise ValueError(f"expected {components} components, got {self.component_count}")


@dataclass(eq=False)
class Plaintext:
    """One CKKS plaintext (or dense batch) in one exact state, with the
    reference's fields (fhelium/core/plaintext.py:19-200):

      representation "slots"                    message [*batch, slot] (not encoded; data None)
                     "integer_coefficients"     data int64 [*batch, N], coefficient domain
                     "approximate_coefficients" data float64 [*batch, N] (decryption output; decode only)
                     "rns"                      data [*batch, limb, N] over prime_ids, with
                                                polynomial_domain, modulus_basis, residue_representation
    """

    message: torch.Tensor | None
    level: int
    scale: float
    data: torch.Tensor | None = None
    context_id: str | None = None
    representation: str = "slots"
    polynomial_domain: str | None = None
    modulus_basis: str | None = None
    residue_representation: str | None = None
    prime_ids: tuple = ()

    def __post_init__(self):
        if (self.message is None) == (self.data is None):
            raise ValueError("Plaintext must own exactly one representation: slots message or encoded data")
        if self.representation not in ("slots", "integer_coefficients", "approximate_coefficients", "rns"):
            raise ValueError(f"Unsupported Plaintext representation: {self.representation!r}")
        if (self.data is None) != (self.representation == "slots"):
            raise ValueError("a slots Plaintext holds a message; every other representation holds data")
        if not (self.scale > 0 and self.scale < float("inf")):
            raise ValueError("Plaintext scale must be positive and finite")
        if self.level < 0:
            raise ValueError("Plaintext level must be non-negative")
        self.prime_ids = tuple(int(i) for i in self.prime_ids)

    @property
    def is_slots(self) -> bool:
        return self.representation == "slots"

    @property
    def is_integer_coefficients(self) -> bool:
        return self.representation == "integer_coefficients"

    @property
    def is_approximate_coefficients(self) -> bool:
        return self.representation == "approximate_coefficients"

    @property
    def is_rns(self) -> bool:
        return self.representation == "rns"

    @property
    def batch_shape(self) -> tuple[int, ...]:
        if self.data is None:
            return tuple(self.message.shape[:-1]) if self.message.ndim > 0 else ()
        return tuple(self.data.shape[:-2] if self.is_rns else self.data.shape[:-1])

    def clone(self) -> "Plaintext":
        return replace(self, message=None if self.message is None else self.message.clone(),
                       data=None if self.data is None else self.data.clone())


@dataclass
class SecretKey:
    data: torch.Tensor  # [QP, N] NTT/Montgomery


@dataclass
class PublicKey:
    data: torch.Tensor  # [2, Q, N] NTT/Montgomery

    @property
    def k0(self) -> torch.Tensor:
        return self.data[0]

    @property
    def k1(self) -> torch.Tensor:
        return self.data[1]


@dataclass
class KeySwitchKey:
    data: torch.Tensor  # [D, 2, QP, N] NTT/Montgomery

    def digit(self, index: int) -> torch.Tensor:
        return self.data[index]


@dataclass
class RelinearizationKey(KeySwitchKey):
    pass


@dataclass
class RotationKey(KeySwitchKey):
    rotation_step: int = 0
    galois_element: int = 1


@dataclass
class RotationKeySet:
    keys: dict = field(default_factory=dict)

    def __contains__(self, step: int) -> bool:
        return step in self.keys

    def __getitem__(self, step: int) -> RotationKey:
        return self.keys[step]

    def __setitem__(self, step: int, key: RotationKey) -> None:
        self.keys[step] = key

    def __len__(self) -> int:
        return len(self.keys)

    def steps(self) -> list[int]:
        return sorted(self.keys)
