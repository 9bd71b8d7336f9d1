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
    """A CKKS ciphertext (or dense batch) in one state (fhelium/core/ciphertext.py:26-384).
    prime_ids default to the level's contiguous rows (level, level + 1, ...)."""

    data: torch.Tensor
    level: int
    scale: float
    polynomial_domain: str = "coefficient"  # "coefficient" | "ntt"
    residue_representation: str = "standard"  # "standard" | "montgomery"
    modulus_basis: str = "Q"
    context_id: str | None = None
    prime_ids: tuple = ()

    def __post_init__(self):
        if self.data.ndim < 3 or self.data.size(0) not in (2, 3):
            raise ValueError("Ciphertext data must be [component(2|3), *batch, limb, N]")
        if self.polynomial_domain not in ("coefficient", "ntt"):
            raise ValueError(f"unsupported polynomial_domain {self.polynomial_domain!r}")
        if self.residue_representation not in ("standard", "montgomery"):
            raise ValueError(f"unsupported residue_representation {self.residue_representation!r}")
        if self.prime_ids:
            self.prime_ids = tuple(int(i) for i in self.prime_ids)
            if len(self.prime_ids) != self.data.size(-2):
                raise ValueError("prime_ids must name every limb row")

    @property
    def limb_ids(self) -> tuple:
        return self.prime_ids or tuple(range(self.level, self.level + self.data.size(-2)))

    @property
    def ring_dimension(self) -> int:
        return self.data.size(-1)

    @property
    def is_batched(self) -> bool:
        return self.data.ndim > 3

    @property
    def is_ntt_domain(self) -> bool:
        return self.polynomial_domain == "ntt"

    @property
    def is_coefficient_domain(self) -> bool:
        return self.polynomial_domain == "coefficient"

    @property
    def includes_p(self) -> bool:
        return self.modulus_basis == "QP"

    def with_data(self, data: torch.Tensor) -> "Ciphertext":
        """The same state over another tensor of the same layout (no copy)."""
        if data.ndim != self.data.ndim or data.shape[0] != self.data.shape[0] or data.shape[-2:] != self.data.shape[-2:]:
            raise ValueError("with_data needs the same component, limb and coefficient extents")
        return replace(self, data=data)

    def slice_limbs(self, start: int, stop: int) -> "Ciphertext":
        """A view of limb rows [start, stop) (fhelium/core/ciphertext.py:252-276)."""
        ids = self.limb_ids[start:stop]
        return replace(self, data=self.data[..., start:stop, :], level=ids[0] if ids else self.level,
                       prime_ids=tuple(ids) if self.prime_ids else ())

    def select_batch(self, index: int, *, dim: int = 0) -> "Ciphertext":
        """A storage-sharing view of one batch item along batch axis `dim`."""
        if not self.is_batched:
            raise ValueError("select_batch requires a batched ciphertext")
        return replace(self, data=self.data.select(dim + 1, index))

    def unbind_batch(self, *, dim: int = 0) -> tuple:
        return tuple(self.select_batch(i, dim=dim) for i in range(self.data.size(dim + 1)))

    @classmethod
    def stack_batch(cls, values, *, dim: int = 0) -> "Ciphertext":
        """Stack ciphertexts of one state into a new batch axis `dim`."""
        values = list(values)
        if not values:
            raise ValueError("stack_batch needs at least one ciphertext")
        first = values[0]
        for v in values[1:]:
            if (v.level, v.scale, v.polynomial_domain, v.residue_representation, v.modulus_basis) != \
                    (first.level, first.scale, first.polynomial_domain, first.residue_representation,
                     first.modulus_basis):
                raise ValueError("stack_batch needs ciphertexts of one level, scale and state")
        return replace(first, data=torch.stack([v.data for v in values], dim=dim + 1))

    def replace_(self, other: "Ciphertext") -> "Ciphertext":
        """Take other's tensor and state in place (fhelium/core/ciphertext.py:358-373)."""
        self.data, self.level, self.scale = other.data, other.level, other.scale
        self.polynomial_domain, self.residue_representation = other.polynomial_domain, other.residue_representation
        self.modulus_basis, self.prime_ids = other.modulus_basis, other.prime_ids
        return self

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


COMPRESSED_PLAINTEXT_FORMAT_VERSION = 1
_COMPRESSION_LAYOUTS = ("cyclic", "contiguous", "strided_sparse")


@dataclass(eq=False)
class CompressedPlaintext:
    """An operation-ready (Montgomery) RNS plaintext stored compactly as
    [*batch, limb, unique] (fhelium/core/compressed_plaintext.py:27-560).  The
    expansion of a compact row to the ring dimension N:
      "cyclic"          [a, b] -> [a, b, a, b, ...]
      "contiguous"      [a, b] -> [a, ..., a, b, ..., b]
      "strided_sparse"  the compact values at positions k (N / unique) apart,
                        every other position implicit_data[*batch, limb].
    """

    data: torch.Tensor
    ring_dimension: int
    compression_layout: str
    level: int
    scale: float
    context_id: str
    polynomial_domain: str
    modulus_basis: str
    residue_representation: str
    prime_ids: tuple
    implicit_data: torch.Tensor | None = None
    compression_format_version: int = COMPRESSED_PLAINTEXT_FORMAT_VERSION

    def __post_init__(self):
        if self.compression_layout not in _COMPRESSION_LAYOUTS:
            raise ValueError(f"Unsupported CompressedPlaintext compression_layout: {self.compression_layout!r}")
        if self.compression_format_version != COMPRESSED_PLAINTEXT_FORMAT_VERSION:
            raise ValueError(f"Unsupported CompressedPlaintext compression format version: "
                             f"{self.compression_format_version}")
        if self.residue_representation != "montgomery":
            raise ValueError("Operation-ready CompressedPlaintext data must use Montgomery form")
        if self.polynomial_domain not in ("coefficient", "ntt") or self.modulus_basis not in ("Q", "QP"):
            raise ValueError("CompressedPlaintext has an unsupported domain or basis")
        u, n = self.data.size(-1), int(self.ring_dimension)
        if not (0 < u < n and u & (u - 1) == 0 and n % u == 0):
            raise ValueError(f"unique count {u} must be a power of two below the ring dimension {n}")
        if (self.implicit_data is None) != (self.compression_layout != "strided_sparse"):
            raise ValueError("implicit_data is required for, and only for, strided_sparse")
        self.prime_ids = tuple(int(i) for i in self.prime_ids)

    @property
    def unique_count(self) -> int:
        return self.data.size(-1)

    @property
    def repeat_count(self) -> int:
        return self.ring_dimension // self.unique_count

    @property
    def batch_shape(self) -> tuple[int, ...]:
        return tuple(self.data.shape[:-2])

    @classmethod
    def from_plaintext(cls, plaintext: Plaintext, *, unique_count: int,
                       compression_layout: str) -> "CompressedPlaintext":
        """Compress an RNS plaintext whose last axis is exactly representable
        in the layout (checked bit for bit); raises ValueError otherwise."""
        if not plaintext.is_rns:
            raise ValueError("CompressedPlaintext.from_plaintext requires a representation='rns' Plaintext")
        if compression_layout not in _COMPRESSION_LAYOUTS:
            raise ValueError(f"Unsupported compression_layout: {compression_layout!r}")
        data = plaintext.data
        n = data.size(-1)
        if not (0 < unique_count < n and unique_count & (unique_count - 1) == 0):
            raise ValueError(f"unique_count must be a power of two below {n}: {unique_count}")
        rep = n // unique_count
        implicit = None
        if compression_layout == "cyclic":
            groups = data.reshape(*data.shape[:-1], rep, unique_count)
            compact = groups[..., 0, :]
            ok = torch.equal(groups, compact.unsqueeze(-2).expand_as(groups))
        else:
            groups = data.reshape(*data.shape[:-1], unique_count, rep)
            compact = groups[..., :, 0]
            if compression_layout == "contiguous":
                ok = torch.equal(groups, compact.unsqueeze(-1).expand_as(groups))
            else:
                implicit = groups[..., 0, 1].clone()
                ok = torch.equal(groups[..., :, 1:], implicit[..., None, None].expand_as(groups[..., :, 1:]))
        if not ok:
            raise ValueError(f"Plaintext encoded data is not exactly representable by the requested "
                             f"{compression_layout!r} compression layout with unique_count={unique_count}")
        return cls(data=compact.contiguous().clone(), ring_dimension=n, compression_layout=compression_layout,
                   level=plaintext.level, scale=plaintext.scale, context_id=plaintext.context_id,
                   polynomial_domain=plaintext.polynomial_domain, modulus_basis=plaintext.modulus_basis,
                   residue_representation=plaintext.residue_representation, prime_ids=plaintext.prime_ids,
                   implicit_data=implicit)

    def decompress_data(self) -> torch.Tensor:
        u, rep = self.unique_count, self.repeat_count
        if self.compression_layout == "cyclic":
            return self.data.repeat(*([1] * (self.data.dim() - 1)), rep)
        if self.compression_layout == "contiguous":
            return self.data.repeat_interleave(rep, dim=-1)
        dense = self.implicit_data[..., None].expand(*self.data.shape[:-1], self.ring_dimension).clone()
        dense[..., ::rep] = self.data
        return dense

    def to_plaintext(self) -> Plaintext:
        return Plaintext(message=None, data=self.decompress_data(), level=self.level, scale=self.scale,
                         context_id=self.context_id, representation="rns", polynomial_domain=self.polynomial_domain,
                         modulus_basis=self.modulus_basis, residue_representation=self.residue_representation,
                         prime_ids=self.prime_ids)

    def clone(self) -> "CompressedPlaintext":
        return replace(self, data=self.data.clone(),
                       implicit_data=None if self.implicit_data is None else self.implicit_data.clone())


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
class EncryptionDraws:
    """The random draws of one public-key encryption, supplied by the caller
    instead of the engine's generator: v (ternary), e0, e1 (the error draws)
    as signed int64 [*batch, N], and, for encrypt_message, the uniforms in
    [0, 1) of encode's stochastic rounding as float64 [*batch, N] (None: the
    engine draws them).  The result is then a deterministic function of the
    message, the key and these draws, c0 = v pk0 + e0 + m, c1 = v pk1 + e1
    (fhelium/engine/ckks_encryptor.py:181-233), which is how encryption is
    compared with the reference's encryptor fed the same values.  No
    counterpart in the reference, whose draws come from its own CSPRNG."""
    v: torch.Tensor
    e0: torch.Tensor
    e1: torch.Tensor
    rounding: torch.Tensor | None = None


@dataclass
class KeySwitchKeyDraws:
    """The random draws of one key-switch key (relinearisation, rotation,
    conjugation), supplied by the caller: per level-zero key digit, the
    uniform component a [D, QP, N] (residues taken as NTT/Montgomery values,
    as the reference's uniform_component_by_key_digit) and the error e
    [D, N] (signed int64).  Digit d is then (e_d - a_d s_dst + P s_src on
    the digit's rows, a_d) (fhelium/engine/key_generator.py:197-330), which is
    how key generation is compared with the reference's key generator fed the
    same values."""
    uniform: torch.Tensor
    error: torch.Tensor


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
    """Rotation keys by canonical step (fhelium/core/keys.py:396-460)."""

    keys: dict = field(default_factory=dict)

    @staticmethod
    def canonical(step: int, ring_dimension: int) -> int:
        s = ring_dimension // 2
        return (int(step) + s // 2) % s - s // 2

    @property
    def table(self) -> dict:
        return self.keys

    def __contains__(self, step: int) -> bool:
        return step in self.keys

    def __getitem__(self, step: int) -> RotationKey:
        return self.keys[step]

    def __setitem__(self, step: int, key: RotationKey) -> None:
        if not isinstance(key, RotationKey):
            raise TypeError(f"RotationKeySet values must be RotationKey objects, got {type(key).__name__}")
        self.keys[step] = key

    def __delitem__(self, step: int) -> None:
        del self.keys[step]

    def __iter__(self):
        return iter(self.keys)

    def __len__(self) -> int:
        return len(self.keys)

    def values(self):
        return self.keys.values()

    def items(self):
        return self.keys.items()

    def add(self, key: RotationKey) -> "RotationKeySet":
        """Install a key under its own canonical rotation step."""
        self[self.canonical(key.rotation_step, key.data.size(-1))] = key
        return self

    def steps(self) -> list[int]:
        return sorted(self.keys)


@dataclass(frozen=True)
class EvaluationKeyRequirements:
    """Key roles and rotations one evaluation needs (fhelium/core/keys.py:462-495)."""

    rotation_steps: frozenset = frozenset()
    requires_relinearization: bool = False
    requires_conjugation: bool = False

    def __post_init__(self):
        steps = frozenset(int(s) for s in self.rotation_steps if int(s) != 0)
        object.__setattr__(self, "rotation_steps", steps)


@dataclass
class EvaluationKeySet:
    """The evaluator's keys: rotations, relinearisation, conjugation
    (fhelium/core/keys.py:497-640); no public or secret key."""

    rotations: RotationKeySet = field(default_factory=RotationKeySet)
    relinearization: RelinearizationKey | None = None
    conjugation: RotationKey | None = None

    def __post_init__(self):
        self.validate()

    def validate(self) -> "EvaluationKeySet":
        if not isinstance(self.rotations, RotationKeySet):
            raise TypeError("EvaluationKeySet rotations must be a RotationKeySet")
        if self.relinearization is not None and not isinstance(self.relinearization, RelinearizationKey):
            raise TypeError("EvaluationKeySet relinearization must be a RelinearizationKey or None")
        if self.conjugation is not None and not isinstance(self.conjugation, RotationKey):
            raise TypeError("EvaluationKeySet conjugation must be a conjugation (Galois 2N - 1) key or None")
        keys = list(self.rotations.values()) + [k for k in (self.relinearization, self.conjugation) if k is not None]
        for step, key in self.rotations.items():
            if RotationKeySet.canonical(key.rotation_step, key.data.size(-1)) != step:
                raise ValueError(f"EvaluationKeySet rotation mapping does not match its key: "
                                 f"mapping={step!r}, key={key.rotation_step!r}")
        if keys:
            shape = lambda k: (tuple(k.data.shape), k.data.dtype, k.data.device)
            first = shape(keys[0])
            if any(shape(k) != first for k in keys[1:]):
                raise ValueError("EvaluationKeySet members differ in layout, dtype or device")
        return self

    def require(self, requirements: EvaluationKeyRequirements) -> "EvaluationKeySet":
        """Raise ValueError naming the first capability that is missing."""
        if not isinstance(requirements, EvaluationKeyRequirements):
            raise TypeError("requirements must be an EvaluationKeyRequirements")
        self.validate()
        if requirements.rotation_steps:
            if len(self.rotations):
                n = next(iter(self.rotations.values())).data.size(-1)
                need = {RotationKeySet.canonical(s, n) for s in requirements.rotation_steps}
            else:
                need = set(requirements.rotation_steps)
            missing = sorted(need - set(self.rotations))
            if missing:
                raise ValueError(f"EvaluationKeySet is missing rotation steps: {missing}")
        if requirements.requires_relinearization and self.relinearization is None:
            raise ValueError("EvaluationKeySet is missing a relinearization key")
        if requirements.requires_conjugation and self.conjugation is None:
            raise ValueError("EvaluationKeySet is missing a conjugation key")
        return self
