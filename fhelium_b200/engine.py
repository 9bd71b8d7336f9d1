"""CkksEngine: the reference's public CKKS API on B200 kernels.

Mirrors fhelium.CkksEngine (fhelium/engine/ckks_engine.py:55-2400): the
same method names, value states and level/scale bookkeeping.  Every residue
operation runs in libfhb200.so through the C ABI (include/fhb200.h); the
engine allocates outputs with torch on the engine's CUDA device, issues the
calls on the current torch stream and never synchronises.  There is no CPU
path: constructing an engine without CUDA or without the library raises.

Randomness: the reference draws from the external `triton_csprng` package.
This engine draws from a seeded torch generator on the device instead
(uniform residues, uniform ternary secrets, rounded Gaussians with
sigma = config.sigma, and the uniforms of encode's unbiased stochastic
rounding; encode_rounding="nearest" rounds deterministically instead).  Everything after encryption is a deterministic function of
the keys and ciphertexts and matches the reference bit for bit.
"""

from __future__ import annotations

import math
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _native as nat
from .config import CkksConfig, Preset
from .encoding import decode_coefficients, encode_real_coefficients
from .values import (Ciphertext, CompressedPlaintext, EncryptionDraws, KeySwitchKey, KeySwitchKeyDraws, Plaintext,
                     PublicKey, RelinearizationKey, RotationKey, RotationKeySet, SecretKey)


def galois_element(n: int, step: int, generator: int = 3) -> int:
    """fhelium/engine/galois.py:10-26: g = gen^(+-step) mod 2N."""
    e = -int(step) if generator == 5 else int(step)
    return pow(generator, e % n, 2 * n)


class CkksEngine:
    def __init__(self, ckks_config: CkksConfig | Preset | dict | str | None = None, *,
                 device: torch.device | str | None = None, allow_sk_gen: bool = True,
                 galois_generator: int = 3, ntt_backend: str | None = None, rng_seed: int | None = None,
                 rng_nonce: int | None = None, encode_rounding: str = "stochastic",
                 basis_conversion: str = "auto"):
        if ckks_config is None:
            ckks_config = Preset.slots16384_scale40_levels16_int64
        if isinstance(ckks_config, (Preset, str, dict)):
            ckks_config = CkksConfig.parse(ckks_config)
        self.config = ckks_config
        if galois_generator not in (3, 5):
            raise ValueError("galois_generator must be 3 or 5")
        device = torch.device(device if device is not None else "cuda")
        if device.type != "cuda":
            raise ValueError("fhelium_b200 runs on CUDA devices only (no CPU path)")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available")
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.galois_generator = galois_generator
        if encode_rounding not in ("stochastic", "nearest"):
            raise ValueError("encode_rounding must be 'stochastic' or 'nearest'")
        self.encode_rounding = encode_rounding
        self.allow_sk_gen = allow_sk_gen
        self.ntt_backend = ntt_backend or "b200_cluster_radix16"
        cfg = self.config
        self.n = cfg.N
        self.log_n = cfg.logN
        self.num_q = cfg.num_q_primes
        self.num_p = cfg.num_p_primes
        self.dtype = cfg.torch_dtype
        self.moduli = cfg.moduli
        self.ctx = nat.NativeContext(64 if cfg.buffer_bit_length == 62 else 32, cfg.logN, cfg.moduli,
                                     self.num_q, self.num_p, device)
        self._gen = torch.Generator(device=device)
        # (seed, nonce) -> one 63-bit generator seed; nonce None keeps the seed as given
        seed = 0 if rng_seed is None else int(rng_seed)
        if rng_nonce is not None:
            seed = (seed * 0x9E3779B97F4A7C15 + int(rng_nonce) + 1) % (1 << 63)
        self._gen.manual_seed(seed)
        self._secret_key: SecretKey | None = None
        self._public_key: PublicKey | None = None
        self._relinearization_key: RelinearizationKey | None = None
        self._rotation_keys = RotationKeySet()
        self._scratch: torch.Tensor | None = None
        self.level_digits = self._digit_layout()
        self.basis_conversion = basis_conversion

    # ------------------------------------------------------------------
    # arithmetic form of the key switch's basis conversion
    # ------------------------------------------------------------------
    _BASIS_FORMS = {"cuda_cores": nat.BASIS_CUDA_CORES, "tensor_cores": nat.BASIS_TENSOR_CORES}

    @property
    def basis_conversion(self) -> str:
        """Where the key switch's exact basis extension runs: ``"cuda_cores"``
        (fused into the key-switch core) or ``"tensor_cores"`` (int8 tcgen05
        MMAs, int64 chains).  Results are bit-identical; no counterpart in
        the reference, whose basis conversion is CUDA-core only."""
        return "tensor_cores" if self.ctx.get_tuning(nat.TUNE_BASIS_CONVERSION) else "cuda_cores"

    @basis_conversion.setter
    def basis_conversion(self, form: str) -> None:
        """``"auto"`` (the default) picks, on int64 chains, the CUDA-core form
        when the chain's leading Q primes are below 2^42 (the key-switch core
        then computes their extensions in exact FP64 arithmetic itself, which
        measured faster than materialising them on the tensor cores) and the
        tensor-core form otherwise; int32 chains take the CUDA-core form."""
        if form == "auto":
            if self.dtype == torch.int64 and not self.ctx.get_tuning(nat.TUNE_F64_CORE):
                try:
                    self.ctx.set_tuning(nat.TUNE_BASIS_CONVERSION, nat.BASIS_TENSOR_CORES)
                    return
                except nat.NativeCallError:
                    pass
            self.ctx.set_tuning(nat.TUNE_BASIS_CONVERSION, nat.BASIS_CUDA_CORES)
            return
        if form not in self._BASIS_FORMS:
            raise ValueError("basis_conversion must be 'auto', 'cuda_cores' or 'tensor_cores'")
        self.ctx.set_tuning(nat.TUNE_BASIS_CONVERSION, self._BASIS_FORMS[form])

    # ------------------------------------------------------------------
    # layout
    # ------------------------------------------------------------------
    def _digit_layout(self) -> list[list[tuple[int, tuple[int, ...]]]]:
        """(key_digit_index, prime ids) per level (fhelium/engine/rns/decomposition.py:18-53)."""
        scale = list(range(self.num_q - 1))
        w = self.num_p
        level0 = [tuple(scale[s:s + w]) for s in range(0, len(scale), w)] + [(self.num_q - 1,)]
        out = []
        for level in range(self.num_q):
            out.append([(kd, tuple(i for i in d if i >= level)) for kd, d in enumerate(level0)
                        if any(i >= level for i in d)])
        return out

    @property
    def num_slots(self) -> int:
        return self.n // 2

    @property
    def public_level_count(self) -> int:
        return self.config.num_scale_primes

    @property
    def key_digit_count(self) -> int:
        return len(self.level_digits[0])

    def _stream(self) -> int:
        return nat.stream_of(self.device)

    def _empty(self, *shape: int) -> torch.Tensor:
        return torch.empty(shape, dtype=self.dtype, device=self.device)

    def _scratch_for(self, batch: int, level: int) -> tuple[torch.Tensor, int]:
        nbytes = int(self.ctx.lib.fhb_ckks_keyswitch_scratch_bytes(self.ctx.handle, batch, level))
        if self._scratch is None or self._scratch.numel() < nbytes:
            self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._scratch, nbytes

    def _check_ct(self, ct: Ciphertext) -> None:
        if ct.data.device != self.device or ct.data.dtype != self.dtype:
            raise ValueError("ciphertext tensor is not on this engine's device/dtype")
        if ct.data.size(-1) != self.n or ct.limb_count != self.num_q - ct.level:
            raise ValueError("ciphertext layout does not match its level")
        if not ct.data.is_contiguous():
            raise ValueError("ciphertext data must be contiguous")

    # ------------------------------------------------------------------
    # NTT domain transitions (fhelium/engine/ckks_engine.py:867-986)
    # ------------------------------------------------------------------
    def forward_ntt(self, x: torch.Tensor, row_start: int, *, montgomery_input: bool = False,
                    out: torch.Tensor | None = None) -> torch.Tensor:
        out = torch.empty_like(x) if out is None else out
        rows = x.size(-2)
        batch = x.numel() // (rows * self.n)
        self.ctx.call("fhb_forward_ntt", nat.ptr(x), nat.ptr(out), batch, rows, row_start,
                      1 if montgomery_input else 0, self._stream())
        return out

    def inverse_ntt(self, x: torch.Tensor, row_start: int, *, output: int = nat.INV_STANDARD,
                    out: torch.Tensor | None = None) -> torch.Tensor:
        out = torch.empty_like(x) if out is None else out
        rows = x.size(-2)
        batch = x.numel() // (rows * self.n)
        self.ctx.call("fhb_inverse_ntt", nat.ptr(x), nat.ptr(out), batch, rows, row_start, output,
                      self._stream())
        return out

    def coefficient_domain_to_ntt_domain(self, ct: "Ciphertext | Plaintext") -> "Ciphertext | Plaintext":
        if isinstance(ct, Plaintext):
            return self._plaintext_ntt(ct, forward=True, inplace=False)
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard")
        self._check_ct(ct)
        data = self.forward_ntt(ct.data, ct.level)
        return Ciphertext(data, ct.level, ct.scale, "ntt", "montgomery")

    def ntt_domain_to_coefficient_domain(self, ct: "Ciphertext | Plaintext") -> "Ciphertext | Plaintext":
        if isinstance(ct, Plaintext):
            return self._plaintext_ntt(ct, forward=False, inplace=False)
        ct.assert_state(polynomial_domain="ntt", residue_representation="montgomery")
        self._check_ct(ct)
        data = self.inverse_ntt(ct.data, ct.level)
        return Ciphertext(data, ct.level, ct.scale, "coefficient", "standard")

    def coefficient_domain_to_ntt_domain_(self, value: "Ciphertext | Plaintext") -> "Ciphertext | Plaintext":
        """In place (fhelium/engine/ckks_engine.py:876-938)."""
        if isinstance(value, Plaintext):
            return self._plaintext_ntt(value, forward=True, inplace=True)
        value.assert_state(polynomial_domain="coefficient", residue_representation="standard")
        self._check_ct(value)
        self.forward_ntt(value.data, value.level, out=value.data)
        value.polynomial_domain, value.residue_representation = "ntt", "montgomery"
        return value

    def ntt_domain_to_coefficient_domain_(self, value: "Ciphertext | Plaintext") -> "Ciphertext | Plaintext":
        """In place (fhelium/engine/ckks_engine.py:940-986)."""
        if isinstance(value, Plaintext):
            return self._plaintext_ntt(value, forward=False, inplace=True)
        value.assert_state(polynomial_domain="ntt", residue_representation="montgomery")
        self._check_ct(value)
        self.inverse_ntt(value.data, value.level, out=value.data)
        value.polynomial_domain, value.residue_representation = "coefficient", "standard"
        return value

    # ------------------------------------------------------------------
    # arithmetic
    # ------------------------------------------------------------------
    def _binary(self, op: int, a: torch.Tensor, b: torch.Tensor | None, row_start: int, *, b_mode: int = 0,
                out: torch.Tensor | None = None) -> torch.Tensor:
        out = torch.empty_like(a) if out is None else out
        rows = a.size(-2)
        batch = a.numel() // (rows * self.n)
        self.ctx.call("fhb_rns_binary", op, nat.ptr(a), nat.ptr(b), nat.ptr(out), batch, rows, row_start,
                      b_mode, self._stream())
        return out

    def add(self, lhs: Ciphertext, rhs: Ciphertext, *, inplace: bool = False) -> Ciphertext:
        """Componentwise modular sum (fhelium/engine/ckks_engine.py:1708-1750)."""
        if inplace:
            return self._replace(lhs, self.add(lhs, rhs))
        self._assert_same_layout(lhs, rhs)
        if lhs.scale != rhs.scale:
            raise ValueError("add requires equal scales")
        lazy = lhs.polynomial_domain == "ntt"
        out = torch.empty_like(lhs.data)
        polys = lhs.component_count * lhs.batch_size
        self.ctx.call("fhb_ckks_add", nat.ptr(lhs.data), nat.ptr(rhs.data), nat.ptr(out), polys, lhs.level,
                      1 if lazy else 0, self._stream())
        return Ciphertext(out, lhs.level, lhs.scale, lhs.polynomial_domain, lhs.residue_representation)

    def _assert_same_layout(self, a: Ciphertext, b: Ciphertext) -> None:
        self._check_ct(a)
        self._check_ct(b)
        if (a.level, a.polynomial_domain, a.residue_representation, a.component_count, a.batch_shape) != \
                (b.level, b.polynomial_domain, b.residue_representation, b.component_count, b.batch_shape):
            raise ValueError("ciphertext layouts differ")

    def multiply(self, lhs: Ciphertext, rhs: Ciphertext) -> Ciphertext:
        """NTT-domain tensor product (fhelium/engine/ckks_engine.py:1530-1606)."""
        lhs.assert_state(polynomial_domain="ntt", residue_representation="montgomery", components=2)
        self._assert_same_layout(lhs, rhs)
        out = self._empty(3, *lhs.data.shape[1:])
        self.ctx.call("fhb_ckks_multiply", nat.ptr(lhs.data), nat.ptr(rhs.data), nat.ptr(out), lhs.batch_size,
                      lhs.level, self._stream())
        return Ciphertext(out, lhs.level, lhs.scale * rhs.scale, "ntt", "montgomery")

    def relinearize(self, ct: Ciphertext, relinearization_key: RelinearizationKey | None = None) -> Ciphertext:
        """fhelium/engine/ckks_engine.py:1608-1675: returns coefficient/standard."""
        ct.assert_state(polynomial_domain="ntt", residue_representation="montgomery", components=3)
        self._check_ct(ct)
        key = relinearization_key or self.relinearization_key
        out = self._empty(2, *ct.data.shape[1:])
        scratch, nbytes = self._scratch_for(ct.batch_size, ct.level)
        self.ctx.call("fhb_ckks_relinearize", nat.ptr(ct.data), nat.ptr(key.data), nat.ptr(out), nat.ptr(scratch),
                      nbytes, ct.batch_size, ct.level, 0, self._stream())
        return Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def rescale_to_next_drop_prime(self, *, level: int) -> int:
        if level + 1 > self.public_level_count:
            raise ValueError("no further public rescale level")
        return self.moduli[level]

    def rescale_to_next_output_scale(self, input_scale: float, *, level: int) -> float:
        return float(input_scale) / float(self.rescale_to_next_drop_prime(level=level))

    def rescale_to_next_level(self, ct: Ciphertext, *, rounding: str = "nearest") -> Ciphertext:
        """fhelium/engine/ckks_rescale.py:339-377 (coefficient/standard input)."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard")
        self._check_ct(ct)
        if rounding not in ("nearest", "floor"):
            raise ValueError("rounding must be 'nearest' or 'floor'")
        scale = self.rescale_to_next_output_scale(ct.scale, level=ct.level)
        out = self._empty(ct.component_count, *ct.batch_shape, ct.limb_count - 1, self.n)
        self.ctx.call("fhb_ckks_rescale", nat.ptr(ct.data), nat.ptr(out), ct.component_count * ct.batch_size,
                      ct.level, 1 if rounding == "nearest" else 0, self._stream())
        return Ciphertext(out, ct.level + 1, scale, "coefficient", "standard")

    def multiply_relinearize_rescale(self, lhs: Ciphertext, rhs: Ciphertext,
                                     relinearization_key: RelinearizationKey | None = None,
                                     *, rescale: bool = True) -> Ciphertext:
        """multiply -> relinearize -> rescale_to_next_level in one fused
        pipeline (four kernel launches); bit-identical to the three calls."""
        lhs.assert_state(polynomial_domain="ntt", residue_representation="montgomery", components=2)
        self._assert_same_layout(lhs, rhs)
        key = relinearization_key or self.relinearization_key
        out_limbs = lhs.limb_count - (1 if rescale else 0)
        scale = lhs.scale * rhs.scale
        if rescale:
            scale = self.rescale_to_next_output_scale(scale, level=lhs.level)
        out = self._empty(2, *lhs.batch_shape, out_limbs, self.n)
        scratch, nbytes = self._scratch_for(lhs.batch_size, lhs.level)
        self.ctx.call("fhb_ckks_multiply_relinearize", nat.ptr(lhs.data), nat.ptr(rhs.data), nat.ptr(key.data),
                      nat.ptr(out), nat.ptr(scratch), nbytes, lhs.batch_size, lhs.level, 1 if rescale else 0,
                      self._stream())
        return Ciphertext(out, lhs.level + (1 if rescale else 0), scale, "coefficient", "standard")

    # ------------------------------------------------------------------
    # plaintexts, scalars, monomials, level changes
    # (fhelium/engine/ckks_engine.py:508-700, 1208-1430, 1964-2180;
    #  fhelium/experimental/bootstrap/_ops.py)
    # ------------------------------------------------------------------
    def encode_plaintext(self, slots, *, level: int, scale: float) -> torch.Tensor:
        """Slots -> NTT/Montgomery plaintext [*batch, Q_level, N] at `scale`."""
        coeffs = self.encode_coefficients(slots, scale)
        return self.forward_ntt(self._lift(coeffs, level, self.num_q - level), level)

    def multiply_plaintext(self, ct: Ciphertext, plaintext: "Plaintext | torch.Tensor",
                           plaintext_scale: float | None = None, *, inplace: bool = False) -> Ciphertext:
        """NTT-domain ct x pt, no rescale; the scale multiplies
        (fhelium/engine/ckks_engine.py:2077-2170).  `plaintext` is a Plaintext
        (slots, integer coefficients or NTT/Montgomery RNS at the ciphertext's
        level; an unbatched one is shared by every batch item), or a raw
        NTT/Montgomery tensor [Q_level, N] with its scale."""
        ct.assert_state(polynomial_domain="ntt", residue_representation="montgomery")
        self._check_ct(ct)
        if isinstance(plaintext, CompressedPlaintext) and plaintext.compression_layout != "strided_sparse":
            result = self._multiply_compressed(ct, plaintext)
            return self._replace(ct, result) if inplace else result
        if isinstance(plaintext, CompressedPlaintext):
            plaintext = plaintext.to_plaintext()
        if isinstance(plaintext, Plaintext):
            pt = self._plaintext_operand(plaintext, ct, "ntt")
            scale = ct.scale * plaintext.scale
        else:
            if plaintext_scale is None:
                raise ValueError("a raw plaintext tensor needs its scale")
            pt, scale = plaintext, ct.scale * plaintext_scale
        if pt.dim() == 2:
            out = self._binary(nat.OP_MONTGOMERY_MUL, ct.data, pt.contiguous(), ct.level, b_mode=1)
        else:
            out = torch.empty_like(ct.data)
            for c in range(ct.component_count):
                self._binary(nat.OP_MONTGOMERY_MUL, ct.data[c], pt.contiguous(), ct.level, out=out[c])
        result = Ciphertext(out, ct.level, scale, "ntt", "montgomery")
        return self._replace(ct, result) if inplace else result

    def _row_constants(self, value: int, level: int, *, montgomery: bool) -> torch.Tensor:
        R = 1 << (62 if self.dtype == torch.int64 else 30)
        vals = [(int(value) * (R if montgomery else 1)) % self.moduli[i] for i in range(level, self.num_q)]
        return torch.tensor(vals, dtype=self.dtype, device=self.device)

    def multiply_integer(self, ct: Ciphertext, value: int, *, scale_factor: float | None = None) -> Ciphertext:
        """Multiply every residue by the integer `value` (no rescale); the
        scale is multiplied by `scale_factor` (default: value)."""
        self._check_ct(ct)
        consts = self._row_constants(value, ct.level, montgomery=True)
        out = self._binary(nat.OP_MONTGOMERY_MUL, ct.data, consts, ct.level, b_mode=2)
        if ct.polynomial_domain == "coefficient":
            out = self._binary(nat.OP_ADD_CANONICAL, out, torch.zeros_like(consts), ct.level, b_mode=2)
        factor = float(value) if scale_factor is None else scale_factor
        return Ciphertext(out, ct.level, ct.scale * factor, ct.polynomial_domain, ct.residue_representation)

    def add_constant(self, ct: Ciphertext, value: float) -> Ciphertext:
        """Add `value` to every slot (round(value * scale) to the constant term)."""
        self._check_ct(ct)
        out = ct.data.clone()
        c = int(round(float(value) * ct.scale))
        ntt = ct.polynomial_domain == "ntt"
        consts = self._row_constants(c, ct.level, montgomery=ntt)
        self.ctx.call("fhb_rns_add_constant", nat.ptr(out[0]), nat.ptr(consts), ct.batch_size, ct.limb_count,
                      ct.level, 1 if ntt else 0, self._stream())
        return Ciphertext(out, ct.level, ct.scale, ct.polynomial_domain, ct.residue_representation)

    def subtract(self, lhs: Ciphertext, rhs: Ciphertext, *, inplace: bool = False) -> Ciphertext:
        if inplace:
            return self._replace(lhs, self.subtract(lhs, rhs))
        self._assert_same_layout(lhs, rhs)
        op = nat.OP_SUB_LAZY if lhs.polynomial_domain == "ntt" else nat.OP_SUB_CANONICAL
        out = self._binary(op, lhs.data, rhs.data, lhs.level)
        return Ciphertext(out, lhs.level, lhs.scale, lhs.polynomial_domain, lhs.residue_representation)

    def multiply_by_monomial(self, ct: Ciphertext, k: int) -> Ciphertext:
        """ct * X^k in Z[X]/(X^N + 1) (coefficient domain)."""
        ct.assert_state(polynomial_domain="coefficient")
        self._check_ct(ct)
        out = torch.empty_like(ct.data)
        k %= 2 * self.n
        self.ctx.call("fhb_ckks_monomial", nat.ptr(ct.data), nat.ptr(out), ct.component_count * ct.batch_size,
                      ct.limb_count, ct.level, k, self._stream())
        return Ciphertext(out, ct.level, ct.scale, ct.polynomial_domain, ct.residue_representation)

    def mod_switch_to_level(self, ct: Ciphertext, level: int) -> Ciphertext:
        """Drop leading Q rows without dividing (fhelium/engine/ckks_engine.py:1278-1345)."""
        if level < ct.level or level >= self.num_q:
            raise ValueError("target level must be at or below the ciphertext's level")
        data = ct.data[..., level - ct.level:, :].contiguous()
        return Ciphertext(data, level, ct.scale, ct.polynomial_domain, ct.residue_representation)

    def reinterpret_at_scale(self, ct: Ciphertext, scale: float) -> Ciphertext:
        return Ciphertext(ct.data, ct.level, float(scale), ct.polynomial_domain, ct.residue_representation)

    def modulus_raise(self, ct: Ciphertext, target_level: int = 0) -> Ciphertext:
        """Centred lift of a one-prime (structural base) coefficient ciphertext
        to Q_target (fhelium/experimental/bootstrap/_modraise.py:338)."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard")
        if ct.level != self.num_q - 1:
            raise ValueError("ModRaise starts from the single structural base prime")
        rows = self.num_q - target_level
        out = self._empty(*ct.data.shape[:-2], rows, self.n)
        polys = ct.component_count * ct.batch_size
        self.ctx.call("fhb_ckks_modraise", nat.ptr(ct.data), nat.ptr(out), polys, self.num_q - 1, rows,
                      target_level, self._stream())
        return Ciphertext(out, target_level, ct.scale, "coefficient", "standard")

    def create_galois_key(self, galois: int, secret_key: SecretKey | None = None, *, rotation_step: int = 0,
                          draws: KeySwitchKeyDraws | None = None) -> RotationKey:
        """Key switching sigma_g(s) -> s for any odd g (rotations, conjugation)."""
        s = secret_key or self.secret_key
        coef = self.inverse_ntt(s.data, 0, output=nat.INV_MONTGOMERY)
        rot = torch.empty_like(coef)
        self.ctx.call("fhb_ckks_automorphism", nat.ptr(coef), nat.ptr(rot), 1, self.qp_rows, 0, galois,
                      self._stream())
        rs = self.forward_ntt(rot, 0, montgomery_input=True)
        ksk = self.create_key_switch_key(SecretKey(rs), s, draws=draws)
        return RotationKey(ksk.data, rotation_step=rotation_step, galois_element=galois)

    def create_conjugation_key(self, secret_key: SecretKey | None = None) -> RotationKey:
        """sigma_{2N-1}: complex conjugation of every slot
        (fhelium/engine/key_generator.py:create_conjugation_key)."""
        return self.create_galois_key(2 * self.n - 1, secret_key)

    def conjugate(self, ct: Ciphertext, key: RotationKey) -> Ciphertext:
        """fhelium/engine/ckks_engine.py:2348-2398."""
        if key.galois_element != 2 * self.n - 1:
            raise ValueError("not a conjugation key")
        return self.rotate_with_key(ct, key)

    # ------------------------------------------------------------------
    # rotations (fhelium/engine/ckks_engine.py:2183-2300, 3726-3897)
    # ------------------------------------------------------------------
    def _canonical_step(self, step: int) -> int:
        """The reference's canonical rotation step: step mod N/2 mapped to
        [-N/4, N/4) (fhelium/core/keys.py:339-351)."""
        s = self.num_slots
        return (int(step) + s // 2) % s - s // 2

    def galois_element_for_step(self, step: int) -> int:
        return galois_element(self.n, self._canonical_step(step) % self.n, self.galois_generator)

    # --- value files (fhelium/serialization/safetensors.py:47-225) ---------
    @property
    def context_id(self) -> str:
        """SHA-256 identity of this engine's context, as the reference computes
        it (fhelium/core/context.py:72-83)."""
        from .serialization import context_id
        return context_id(self.config, self.galois_generator)

    def save_value(self, value, path, *, allow_secret: bool = False, overwrite: bool = False) -> dict:
        """Write a ciphertext or key to a value file readable by the reference's
        fh.load_value (fhelium/serialization/safetensors.py:47-131)."""
        from .serialization import save_value
        return save_value(value, path, context_id=self.context_id, allow_secret=allow_secret, overwrite=overwrite)

    def load_value(self, path, *, expected_type=None):
        """Read a value file written by this library or the reference's
        fh.save_value onto this engine's device; the file must belong to this
        engine's context.  Rotation keys get this engine's Galois element."""
        from .serialization import load_value
        value = load_value(path, device=self.device, expected_type=expected_type,
                           expected_context_id=self.context_id)
        if isinstance(value, RotationKey):
            value.galois_element = self.galois_element_for_step(value.rotation_step)
        return value

    def rotation_key(self, rotation_step: int) -> RotationKey:
        step = self._canonical_step(rotation_step)
        if step not in self._rotation_keys:
            if not self.allow_sk_gen:
                raise KeyError(f"no rotation key for step {rotation_step}")
            self._rotation_keys[step] = self.create_rotation_key(step)
        return self._rotation_keys[step]

    def rotate_by_step(self, ct: Ciphertext, rotation_step: int) -> Ciphertext:
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        step = self._canonical_step(rotation_step)
        if step == 0:
            return ct.clone()
        return self.rotate_with_key(ct, self.rotation_key(step))

    def rotate_with_key(self, ct: Ciphertext, key: RotationKey) -> Ciphertext:
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        out = torch.empty_like(ct.data)
        scratch, nbytes = self._scratch_for(ct.batch_size, ct.level)
        self.ctx.call("fhb_ckks_rotate", nat.ptr(ct.data), nat.ptr(key.data), nat.ptr(out), nat.ptr(scratch), nbytes,
                      ct.batch_size, ct.level, key.galois_element, self._stream())
        return Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def rotate_items_with_keys(self, ct: Ciphertext, keys: Sequence[RotationKey]) -> Ciphertext:
        """Rotates batch item b of `ct` with keys[b] (mixed steps, one launch
        sequence); bit-identical to rotating every item on its own."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        if len(keys) != ct.batch_size:
            raise ValueError("need one rotation key per batch item")
        galois = torch.tensor([k.galois_element for k in keys], dtype=torch.int32, device=self.device)
        for k in keys:
            if k.data.device != self.device or k.data.dtype != self.dtype or not k.data.is_contiguous():
                raise ValueError("rotation keys must be contiguous tensors on this engine's device/dtype")
        key_ptrs = torch.tensor([k.data.data_ptr() for k in keys], dtype=torch.int64, device=self.device)
        out = torch.empty_like(ct.data)
        scratch, nbytes = self._scratch_for(ct.batch_size, ct.level)
        self.ctx.call("fhb_ckks_rotate_multi", nat.ptr(ct.data), nat.ptr(key_ptrs), nat.ptr(galois), nat.ptr(out),
                      nat.ptr(scratch), nbytes, ct.batch_size, ct.level, self._stream())
        return Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def rotate_and_sum(self, cts: Sequence[Ciphertext], keys: Sequence[RotationKey]) -> Ciphertext:
        """sum_i rotate_with_key(cts[i], keys[i]) with one ModDown for the
        whole sum: ModUp of every sigma_g(c1), the key switches accumulated
        in the NTT domain (fhb_ckks_keyswitch_sum), one inverse NTT and one
        ModDown with sum_i sigma_g(c0_i) added.  The sum is rounded once
        instead of once per term, so it is within len(cts) units of the sum
        of separately rounded rotations (not bit-identical to it)."""
        if not cts or len(cts) != len(keys):
            raise ValueError("need one rotation key per ciphertext")
        first = cts[0]
        for ct in cts:
            ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
            self._check_ct(ct)
            if (ct.level, ct.data.shape, ct.scale) != (first.level, first.data.shape, first.scale):
                raise ValueError("rotate_and_sum needs ciphertexts of one level, shape and scale")
        b, level, limbs = first.batch_size, first.level, first.limb_count
        st = self._stream()
        digits = self._empty(len(cts), b, limbs, self.n)
        for i, (ct, key) in enumerate(zip(cts, keys)):
            self.ctx.call("fhb_ckks_modup_digits", nat.ptr(ct.c1), nat.ptr(digits[i]), b, level, key.galois_element, st)
        key_ptrs = torch.tensor([k.data.data_ptr() for k in keys], dtype=torch.int64, device=self.device)
        t = self._empty(2, b, limbs + self.num_p, self.n)
        if self.basis_conversion == "tensor_cores":
            # the giants' digits as one batch of len(cts) x b ciphertexts
            words = int(self.ctx.lib.fhb_tc_basis_extend_words(self.ctx.handle, len(cts) * b, level))
            ext = torch.empty(words, dtype=self.dtype, device=self.device)
            self.ctx.call("fhb_tc_basis_extend", nat.ptr(digits), nat.ptr(ext), len(cts) * b, level, st)
            self.ctx.call("fhb_ckks_keyswitch_sum_extended", nat.ptr(ext), nat.ptr(key_ptrs), nat.ptr(t[0]),
                          nat.ptr(t[1]), len(cts), b, level, st)
        else:
            self.ctx.call("fhb_ckks_keyswitch_sum", nat.ptr(digits), nat.ptr(key_ptrs), nat.ptr(t[0]),
                          nat.ptr(t[1]), len(cts), b, level, st)
        add0 = None
        for ct, key in zip(cts, keys):
            rot = self._empty(*ct.c0.shape)
            self.ctx.call("fhb_ckks_automorphism", nat.ptr(ct.c0), nat.ptr(rot), b, limbs, level, key.galois_element,
                          st)
            if add0 is None:
                add0 = rot
            else:
                self.ctx.call("fhb_ckks_add", nat.ptr(add0), nat.ptr(rot), nat.ptr(add0), b, level, 0, st)
        out = torch.empty_like(first.data)
        self.ctx.call("fhb_ckks_moddown", nat.ptr(t[0]), nat.ptr(t[1]), nat.ptr(add0), None, nat.ptr(out), b, level,
                      1, 0, st)
        return Ciphertext(out, level, first.scale, "coefficient", "standard")

    def prepare_rotation_digits(self, ct: Ciphertext) -> torch.Tensor:
        """Hoisted ModUp of c1: [digit, *batch, Q_l + P, N] NTT-domain digits."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        b, level = ct.batch_size, ct.level
        digits = self._empty(b, ct.limb_count, self.n)
        self.ctx.call("fhb_ckks_modup_digits", nat.ptr(ct.c1), nat.ptr(digits), b, level, 1, self._stream())
        nd = len(self.level_digits[level])
        prepared = self._empty(nd, b, ct.limb_count + self.num_p, self.n)
        self.ctx.call("fhb_ckks_prepare_rotation", nat.ptr(digits), nat.ptr(prepared), b, level, self._stream())
        return prepared

    def apply_prepared_rotation(self, ct: Ciphertext, prepared: torch.Tensor, key: RotationKey) -> Ciphertext:
        b, level = ct.batch_size, ct.level
        qp = ct.limb_count + self.num_p
        t = self._empty(2, b, qp, self.n)
        self.ctx.call("fhb_ckks_apply_prepared_rotation", nat.ptr(prepared), nat.ptr(key.data), nat.ptr(t[0]),
                      nat.ptr(t[1]), b, level, key.galois_element, self._stream())
        out = torch.empty_like(ct.data)
        self.ctx.call("fhb_ckks_moddown", nat.ptr(t[0]), nat.ptr(t[1]), nat.ptr(ct.c0), None, nat.ptr(out), b,
                      level, key.galois_element, 0, self._stream())
        return Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def rotate_many_by_steps(self, ct: Ciphertext, rotation_steps: Sequence[int], *,
                             use_hoisting: bool = True) -> list[Ciphertext]:
        steps = [self._canonical_step(s) for s in rotation_steps]
        nonzero = [s for s in steps if s != 0]
        if not use_hoisting or len(nonzero) < 2:
            return [self.rotate_by_step(ct, s) for s in steps]
        prepared = self.prepare_rotation_digits(ct)
        return [ct.clone() if s == 0 else self.apply_prepared_rotation(ct, prepared, self.rotation_key(s))
                for s in steps]

    # ------------------------------------------------------------------
    # keys (fhelium/engine/key_generator.py)
    # ------------------------------------------------------------------
    def _uniform_rows(self, *shape_prefix: int, rows: Iterable[int]) -> torch.Tensor:
        rows = list(rows)
        out = torch.empty((*shape_prefix, len(rows), self.n), dtype=torch.int64, device=self.device)
        for j, pid in enumerate(rows):
            out[..., j, :] = torch.randint(0, self.moduli[pid], (*shape_prefix, self.n), generator=self._gen,
                                           device=self.device, dtype=torch.int64)
        return out.to(self.dtype)

    def _ternary(self, *shape: int) -> torch.Tensor:
        return torch.randint(-1, 2, shape, generator=self._gen, device=self.device, dtype=torch.int64)

    def _gaussian(self, *shape: int) -> torch.Tensor:
        x = torch.randn(shape, generator=self._gen, device=self.device, dtype=torch.float64) * self.config.sigma
        return torch.round(x).to(torch.int64)

    def _lift(self, coeffs: torch.Tensor, row_start: int, rows: int) -> torch.Tensor:
        """Signed int64 [..., N] -> canonical residues [..., rows, N]."""
        coeffs = coeffs.contiguous()
        batch = coeffs.numel() // self.n
        out = self._empty(*coeffs.shape[:-1], rows, self.n)
        self.ctx.call("fhb_rns_lift_signed", nat.ptr(coeffs), nat.ptr(out), batch, rows, row_start, self._stream())
        return out

    @property
    def qp_rows(self) -> int:
        return self.num_q + self.num_p

    def create_secret_key(self) -> SecretKey:
        s = self._lift(self._ternary(self.n), 0, self.qp_rows)
        return SecretKey(self.forward_ntt(s, 0))

    @property
    def secret_key(self) -> SecretKey:
        if self._secret_key is None:
            if not self.allow_sk_gen:
                raise RuntimeError("secret-key generation is disabled")
            self._secret_key = self.create_secret_key()
        return self._secret_key

    def set_secret_key(self, key: SecretKey) -> None:
        self._secret_key = key

    def _encrypt_zero_qp(self, s: torch.Tensor, rows: int, uniform: torch.Tensor | None = None,
                         error: torch.Tensor | None = None):
        """(e - a s, a) over the first `rows` level-zero rows, NTT/Montgomery."""
        a = self._uniform_rows(rows=range(rows)) if uniform is None else uniform
        err = self._gaussian(self.n) if error is None else error.to(self.device, torch.int64).contiguous()
        e = self.forward_ntt(self._lift(err, 0, rows), 0)
        a_s = self._binary(nat.OP_MONTGOMERY_MUL, a, s[:rows].contiguous(), 0)
        return self._binary(nat.OP_SUB_LAZY, e, a_s, 0), a

    def create_public_key(self, secret_key: SecretKey | None = None) -> PublicKey:
        s = (secret_key or self.secret_key).data
        k0, k1 = self._encrypt_zero_qp(s, self.num_q)
        return PublicKey(torch.stack([k0, k1]))

    @property
    def public_key(self) -> PublicKey:
        if self._public_key is None:
            self._public_key = self.create_public_key()
        return self._public_key

    def create_key_switch_key(self, source: SecretKey, destination: SecretKey, *,
                              draws: KeySwitchKeyDraws | None = None) -> KeySwitchKey:
        """Digit d: (-a s_dst + e + P s_src on the digit's rows, a)
        (fhelium/engine/key_generator.py:197-262); `draws` supplies a and e
        (see KeySwitchKeyDraws)."""
        P = math.prod(self.moduli[self.num_q:])
        R = 1 << (62 if self.dtype == torch.int64 else 30)
        p_mont = torch.tensor([(P * R) % q for q in self.moduli[: self.num_q]], dtype=self.dtype,
                              device=self.device)
        src_q = source.data[: self.num_q].contiguous()
        p_src = self._binary(nat.OP_MONTGOMERY_MUL, src_q, p_mont, 0, b_mode=2)
        digits = []
        if draws is not None:
            nd, shape = len(self.level_digits[0]), (self.qp_rows, self.n)
            if tuple(draws.uniform.shape) != (nd, *shape) or tuple(draws.error.shape) != (nd, self.n):
                raise ValueError(f"key draws must be uniform [{nd}, {shape[0]}, {shape[1]}] and error [{nd}, {self.n}]")
        for kd, ids in self.level_digits[0]:
            if draws is None:
                k0, k1 = self._encrypt_zero_qp(destination.data, self.qp_rows)
            else:
                a = draws.uniform[kd].to(self.device, self.dtype).contiguous()
                k0, k1 = self._encrypt_zero_qp(destination.data, self.qp_rows, a, draws.error[kd])
            lo, hi = ids[0], ids[-1] + 1
            k0[lo:hi] = self._binary(nat.OP_ADD_LAZY, k0[lo:hi].contiguous(), p_src[lo:hi].contiguous(), lo)
            digits.append(torch.stack([k0, k1]))
        return KeySwitchKey(torch.stack(digits))

    def create_relinearization_key(self, secret_key: SecretKey | None = None, *,
                                   draws: KeySwitchKeyDraws | None = None) -> RelinearizationKey:
        s = secret_key or self.secret_key
        s2 = self._binary(nat.OP_MONTGOMERY_MUL, s.data, s.data, 0)
        return RelinearizationKey(self.create_key_switch_key(SecretKey(s2), s, draws=draws).data)

    @property
    def relinearization_key(self) -> RelinearizationKey:
        if self._relinearization_key is None:
            self._relinearization_key = self.create_relinearization_key()
        return self._relinearization_key

    def set_relinearization_key(self, key: RelinearizationKey) -> None:
        self._relinearization_key = key

    def create_rotation_key(self, rotation_step: int, secret_key: SecretKey | None = None, *,
                            draws: KeySwitchKeyDraws | None = None) -> RotationKey:
        """Key from sigma_g(s) back to s (fhelium/engine/key_generator.py:364-412)."""
        step = self._canonical_step(rotation_step)
        return self.create_galois_key(self.galois_element_for_step(step), secret_key, rotation_step=step,
                                      draws=draws)

    def generate_rotation_keys(self, steps: Iterable[int]) -> None:
        for st in steps:
            self.rotation_key(st)

    @property
    def rotation_keys(self) -> RotationKeySet:
        return self._rotation_keys

    def set_rotation_key(self, key: RotationKey) -> None:
        self._rotation_keys[self._canonical_step(key.rotation_step)] = key

    # ------------------------------------------------------------------
    # encode / encrypt / decrypt (fhelium/engine/ckks_engine.py:508-866)
    # ------------------------------------------------------------------
    def encode_coefficients(self, message, scale: float, rounding: torch.Tensor | None = None) -> torch.Tensor:
        m = torch.as_tensor(message, device=self.device)
        if m.ndim == 0:
            m = m.expand(self.num_slots)
        if m.size(-1) > self.num_slots:
            raise ValueError("message longer than the slot count")
        coeffs = encode_real_coefficients(m.to(self.device), self.n, self.galois_generator) * float(scale)
        if coeffs.abs().max().item() >= 2.0 ** 62:
            raise ValueError("encoded coefficients exceed the int64 range; lower the scale")
        if self.encode_rounding == "nearest":
            return torch.round(coeffs).to(torch.int64)
        # unbiased stochastic rounding, E[SRound(x)] = x (fhelium/engine/slot_embedding.py:100)
        low = torch.floor(coeffs)
        if rounding is not None:
            if tuple(rounding.shape) != tuple(coeffs.shape):
                raise ValueError("rounding uniforms must have the coefficients' shape [*batch, N]")
            u = rounding.to(coeffs.device, coeffs.dtype)
        else:
            u = torch.rand(coeffs.shape, generator=self._gen, device=coeffs.device, dtype=coeffs.dtype)
        return (low + (u < coeffs - low).to(coeffs.dtype)).to(torch.int64)

    def encrypt_message(self, message, public_key: PublicKey | None = None, *, level: int = 0,
                        scale: float | None = None, draws: EncryptionDraws | None = None) -> Ciphertext:
        """Encode + public-key encryption, coefficient/standard output.
        `draws` supplies the encryption's random values (see EncryptionDraws)."""
        if not 0 <= level < self.public_level_count:
            raise ValueError("level out of range")
        scale = float(self.config.default_scale if scale is None else scale)
        coeffs = self.encode_coefficients(message, scale, None if draws is None else draws.rounding)
        return self._encrypt_coefficients(coeffs, level, scale, public_key, draws)

    def _encrypt_coefficients(self, coeffs: torch.Tensor, level: int, scale: float,
                              public_key: PublicKey | None, draws: EncryptionDraws | None = None) -> Ciphertext:
        """(v pk0 + e0 + m, v pk1 + e1) of exact integer coefficients [*batch, N]
        (fhelium/engine/ckks_encryptor.py:181-233)."""
        pk = (public_key or self.public_key).data[:, level:].contiguous()
        batch_shape = tuple(coeffs.shape[:-1])
        L = self.num_q - level
        m = self.forward_ntt(self._lift(coeffs, level, L), level)
        shape = (*batch_shape, self.n)
        if draws is None:
            v_c, e0_c, e1_c = self._ternary(*shape), self._gaussian(*shape), self._gaussian(*shape)
        else:
            v_c, e0_c, e1_c = (torch.as_tensor(d).to(self.device, torch.int64) for d in (draws.v, draws.e0, draws.e1))
            if any(tuple(d.shape) != shape for d in (v_c, e0_c, e1_c)):
                raise ValueError(f"encryption draws must have shape {shape}")
        v = self.forward_ntt(self._lift(v_c, level, L), level)
        e0 = self.forward_ntt(self._lift(e0_c, level, L), level)
        e1 = self.forward_ntt(self._lift(e1_c, level, L), level)
        c0 = self._binary(nat.OP_MONTGOMERY_MUL, v, pk[0].contiguous(), level, b_mode=1)
        c0 = self._binary(nat.OP_ADD_LAZY, c0, e0, level)
        c0 = self._binary(nat.OP_ADD_LAZY, c0, m, level)
        c1 = self._binary(nat.OP_MONTGOMERY_MUL, v, pk[1].contiguous(), level, b_mode=1)
        c1 = self._binary(nat.OP_ADD_LAZY, c1, e1, level)
        data = self.inverse_ntt(torch.stack([c0, c1]), level)
        return Ciphertext(data, level, scale, "coefficient", "standard")

    def _phase(self, ct: Ciphertext, secret_key: SecretKey | None = None) -> torch.Tensor:
        """c0 + c1 s (+ c2 s^2) in coefficient/standard canonical form."""
        s = (secret_key or self.secret_key).data[ct.level: self.num_q].contiguous()
        data = ct.data if ct.polynomial_domain == "ntt" else self.forward_ntt(ct.data, ct.level)
        acc = data[0].contiguous()
        s_pow = s
        for i in range(1, ct.component_count):
            term = self._binary(nat.OP_MONTGOMERY_MUL, data[i].contiguous(), s_pow, ct.level, b_mode=1)
            acc = self._binary(nat.OP_ADD_LAZY, acc, term, ct.level)
            if i + 1 < ct.component_count:
                s_pow = self._binary(nat.OP_MONTGOMERY_MUL, s_pow, s, ct.level)
        return self.inverse_ntt(acc, ct.level)

    def decrypt_coefficients(self, ct: Ciphertext, secret_key: SecretKey | None = None) -> torch.Tensor:
        """Bounded decryption on the device: float64 [*batch, N], the centred
        class of the phase modulo the product of the trailing one or two
        active Q primes, the same doubles as the reference's decryptor
        (fhelium/engine/ckks_decryptor.py:180-272; fhb_ckks_decrypt_tail)."""
        self._check_ct(ct)
        phase = self._phase(ct, secret_key).contiguous()
        out = torch.empty((*ct.data.shape[1:-2], self.n), dtype=torch.float64, device=self.device)
        self.ctx.call("fhb_ckks_decrypt_tail", nat.ptr(phase), nat.ptr(out), ct.batch_size, ct.level, self._stream())
        return out

    def decrypt_message(self, ct: Ciphertext, secret_key: SecretKey | None = None, *,
                        is_real: bool = False) -> torch.Tensor:
        """Decrypt and decode at the ciphertext's scale; CPU [*batch, N/2]
        slots, complex unless is_real (fhelium/engine/ckks_decryptor.py:357)."""
        coeffs = self.decrypt_coefficients(ct, secret_key)
        slots = decode_coefficients(coeffs, self.n, self.galois_generator) / ct.scale
        return (slots.real if is_real else slots).cpu()

    # ------------------------------------------------------------------
    # Plaintext values (fhelium/engine/ckks_engine.py:508-760,
    # fhelium/engine/ckks_plaintext_codec.py:78-450)
    # ------------------------------------------------------------------
    def _public_level(self, level: int) -> int:
        if not 0 <= int(level) < self.public_level_count:
            raise ValueError(f"level {level} outside the public levels 0..{self.final_public_level}")
        return int(level)

    def _scale_arg(self, scale) -> float:
        scale = float(self.config.default_scale if scale is None else scale)
        if not (scale > 0 and math.isfinite(scale)):
            raise ValueError("scale must be positive and finite")
        return scale

    def _check_context(self, value) -> None:
        cid = getattr(value, "context_id", None)
        if cid not in (None, self.context_id):
            raise ValueError(f"value belongs to another CKKS context: {cid} != {self.context_id}")

    def _prime_ids(self, level: int, modulus_basis: str) -> tuple:
        if modulus_basis not in ("Q", "QP"):
            raise ValueError("modulus_basis must be 'Q' or 'QP'")
        stop = self.num_q + (self.num_p if modulus_basis == "QP" else 0)
        return tuple(range(level, stop))

    def plaintext(self, message, *, level: int = 0, scale=None) -> Plaintext:
        """An unencoded slots plaintext on this engine's device."""
        level = self._public_level(level)
        msg = torch.as_tensor(message).detach().clone().to(self.device)
        return Plaintext(message=msg, level=level, scale=self._scale_arg(scale))

    def encode(self, message, *, level: int = 0, scale=None) -> Plaintext:
        """Slots -> exact integer coefficients [*batch, N] at `scale`, rounded
        by the engine's `encode_rounding`: unbiased stochastic rounding by
        default, as the reference rounds (fhelium/engine/slot_embedding.py:100),
        or to nearest."""
        if isinstance(message, Plaintext):
            return self._integer_plaintext(message)
        level = self._public_level(level)
        scale = self._scale_arg(scale)
        coeffs = self.encode_coefficients(message, scale)
        return Plaintext(message=None, data=coeffs, level=level, scale=scale, context_id=self.context_id,
                         representation="integer_coefficients", polynomial_domain="coefficient")

    def _integer_plaintext(self, pt: Plaintext) -> Plaintext:
        self._check_context(pt)
        if pt.is_integer_coefficients:
            return pt
        if pt.is_slots:
            return self.encode(pt.message, level=pt.level, scale=pt.scale)
        raise ValueError(f"expected slots or integer_coefficients, got {pt.representation}")

    def integer_coefficients_to_rns(self, plaintext: Plaintext, *, modulus_basis: str = "Q") -> Plaintext:
        """Exact coefficients -> coefficient/standard residues over Q_level (or Q_level P)."""
        pt = self._integer_plaintext(plaintext)
        ids = self._prime_ids(pt.level, modulus_basis)
        data = self._lift(pt.data.to(device=self.device, dtype=torch.int64), pt.level, len(ids))
        return Plaintext(message=None, data=data, level=pt.level, scale=pt.scale, context_id=self.context_id,
                         representation="rns", polynomial_domain="coefficient", modulus_basis=modulus_basis,
                         residue_representation="standard", prime_ids=ids)

    def _rows_mul_const(self, data: torch.Tensor, row_start: int, value_of, *, canonical: bool) -> torch.Tensor:
        rows = data.size(-2)
        consts = torch.tensor([value_of(self.moduli[i]) for i in range(row_start, row_start + rows)],
                              dtype=self.dtype, device=self.device)
        out = self._binary(nat.OP_MONTGOMERY_MUL, data.contiguous(), consts, row_start, b_mode=2)
        if canonical:
            out = self._binary(nat.OP_ADD_CANONICAL, out, torch.zeros_like(consts), row_start, b_mode=2, out=out)
        return out

    def _rns_plaintext(self, pt: Plaintext) -> Plaintext:
        self._check_context(pt)
        if not pt.is_rns:
            raise ValueError(f"expected an RNS plaintext, got {pt.representation}")
        return pt

    def standard_residues_to_montgomery_residues(self, plaintext: Plaintext) -> Plaintext:
        return self.standard_residues_to_montgomery_residues_(plaintext.clone())

    def standard_residues_to_montgomery_residues_(self, plaintext: Plaintext) -> Plaintext:
        """x -> x R (canonical), in place (fhelium/engine/ckks_engine.py:1036-1060)."""
        pt = self._rns_plaintext(plaintext)
        if pt.residue_representation != "standard":
            raise ValueError("plaintext residues are not in standard form")
        R2 = lambda q: pow(1 << self.config.buffer_bit_length, 2, q)
        pt.data = self._rows_mul_const(pt.data, pt.prime_ids[0], R2, canonical=True)
        pt.residue_representation = "montgomery"
        return pt

    def montgomery_residues_to_standard_residues(self, plaintext: Plaintext) -> Plaintext:
        return self.montgomery_residues_to_standard_residues_(plaintext.clone())

    def montgomery_residues_to_standard_residues_(self, plaintext: Plaintext) -> Plaintext:
        """x R -> x (canonical), in place."""
        pt = self._rns_plaintext(plaintext)
        if pt.residue_representation != "montgomery" or pt.polynomial_domain != "coefficient":
            raise ValueError("expected coefficient-domain Montgomery residues")
        pt.data = self._rows_mul_const(pt.data, pt.prime_ids[0], lambda q: 1, canonical=True)
        pt.residue_representation = "standard"
        return pt

    def _plaintext_ntt(self, pt: Plaintext, *, forward: bool, inplace: bool) -> Plaintext:
        pt = self._rns_plaintext(pt)
        if not inplace:
            pt = pt.clone()
        start = pt.prime_ids[0]
        if forward:
            if pt.polynomial_domain != "coefficient":
                raise ValueError("plaintext is already in the NTT domain")
            self.forward_ntt(pt.data, start, montgomery_input=pt.residue_representation == "montgomery",
                             out=pt.data)
        else:
            if pt.polynomial_domain != "ntt":
                raise ValueError("plaintext is not in the NTT domain")
            self.inverse_ntt(pt.data, start, output=nat.INV_STANDARD, out=pt.data)
        pt.polynomial_domain = "ntt" if forward else "coefficient"
        pt.residue_representation = "montgomery" if forward else "standard"
        return pt

    def prepare_plaintext_for_addition(self, plaintext: Plaintext, *, modulus_basis: str = "Q") -> Plaintext:
        """Coefficient-domain Montgomery residues, the operand of add_plaintext."""
        return self.standard_residues_to_montgomery_residues_(
            self.integer_coefficients_to_rns(plaintext, modulus_basis=modulus_basis))

    def prepare_plaintext_for_multiplication(self, plaintext: Plaintext, *, modulus_basis: str = "Q") -> Plaintext:
        """NTT-domain Montgomery residues, the operand of multiply_plaintext."""
        return self._plaintext_ntt(self.integer_coefficients_to_rns(plaintext, modulus_basis=modulus_basis),
                                   forward=True, inplace=True)

    def decode(self, plaintext: Plaintext, *, is_real: bool = False) -> torch.Tensor:
        """Coefficients / scale -> slots [*batch, N/2] on the CPU (complex unless is_real)."""
        if not isinstance(plaintext, Plaintext):
            raise TypeError(f"decode expects Plaintext, got {type(plaintext).__name__}")
        self._check_context(plaintext)
        if plaintext.is_slots:
            plaintext = self.encode(plaintext)
        if plaintext.is_rns:
            raise ValueError("decode requires integer_coefficients or approximate_coefficients; "
                             "RNS reconstruction is not implicit")
        vals = plaintext.data.detach().to("cpu", torch.float64)
        slots = decode_coefficients(vals, self.n, self.galois_generator) / plaintext.scale
        return slots.real if is_real else slots

    def encrypt(self, plaintext: Plaintext, public_key: PublicKey | None = None, *,
                draws: EncryptionDraws | None = None) -> Ciphertext:
        """Public-key encryption of slots or exact integer coefficients;
        coefficient/standard output (fhelium/engine/ckks_engine.py:700-738).
        `draws` supplies the encryption's random values (see EncryptionDraws)."""
        if not isinstance(plaintext, Plaintext):
            raise TypeError(f"encrypt expects Plaintext, got {type(plaintext).__name__}")
        pt = self._integer_plaintext(plaintext)
        self._public_level(pt.level)
        return self._encrypt_coefficients(pt.data.to(self.device, torch.int64), pt.level, pt.scale, public_key,
                                          draws)

    def decrypt(self, ct: Ciphertext, secret_key: SecretKey | None = None) -> Plaintext:
        """Decryption to float64 coefficients [*batch, N] (approximate
        coefficients, for decode) (fhelium/engine/ckks_engine.py:740-771)."""
        if not isinstance(ct, Ciphertext):
            raise TypeError(f"decrypt expects Ciphertext, got {type(ct).__name__}")
        data = self.decrypt_coefficients(ct, secret_key)
        return Plaintext(message=None, data=data, level=ct.level, scale=ct.scale, context_id=self.context_id,
                         representation="approximate_coefficients", polynomial_domain="coefficient")

    def zero_plaintext_like(self, plaintext: Plaintext) -> Plaintext:
        """Semantic zero in the same representation and state
        (fhelium/engine/ckks_engine.py:1431-1489)."""
        self._check_context(plaintext)
        if plaintext.is_approximate_coefficients:
            out = plaintext.clone()
            out.data.zero_()
            return out
        zero = torch.zeros((*plaintext.batch_shape, self.num_slots), dtype=torch.complex128, device=self.device)
        if plaintext.is_slots:
            return Plaintext(message=zero, level=plaintext.level, scale=plaintext.scale)
        encoded = self.encode(zero, level=plaintext.level, scale=plaintext.scale)
        if plaintext.is_integer_coefficients:
            return encoded
        basis = plaintext.modulus_basis or "Q"
        if plaintext.residue_representation == "standard":
            return self.integer_coefficients_to_rns(encoded, modulus_basis=basis)
        if plaintext.polynomial_domain == "coefficient":
            return self.prepare_plaintext_for_addition(encoded, modulus_basis=basis)
        return self.prepare_plaintext_for_multiplication(encoded, modulus_basis=basis)

    def _plaintext_operand(self, pt: Plaintext, ct: Ciphertext, domain: str) -> torch.Tensor:
        """The plaintext's residues over the ciphertext's Q_level rows in the
        operation's state (coefficient/Montgomery for addition, NTT/Montgomery
        for multiplication), preparing slots or integer plaintexts first."""
        self._check_context(pt)
        if pt.level != ct.level:
            raise ValueError(f"plaintext level {pt.level} != ciphertext level {ct.level}")
        if not pt.is_rns:
            pt = (self.prepare_plaintext_for_addition(pt) if domain == "coefficient"
                  else self.prepare_plaintext_for_multiplication(pt))
        if pt.polynomial_domain != domain or pt.residue_representation != "montgomery":
            raise ValueError(f"plaintext must be {domain}-domain Montgomery residues, got "
                             f"{pt.polynomial_domain}/{pt.residue_representation}")
        data = pt.data[..., : ct.limb_count, :]     # a Q_level P plaintext contributes its Q rows
        if data.dim() > 2 and tuple(data.shape[:-2]) != ct.batch_shape:
            raise ValueError("a batched plaintext must match the ciphertext's batch shape")
        return data

    @property
    def _param_rows(self) -> torch.Tensor:
        """The reference's [8, QP] parameter rows (csrc/ops/common/rns_parameters.h:6-16)."""
        if getattr(self, "_param_rows_cache", None) is None:
            bits = self.config.buffer_bit_length
            half, R = bits // 2, 1 << bits
            cols = []
            for q in self.moduli:
                ninv = (-pow(q, -1, R)) % R
                r2 = (R * R) % q
                cols.append([2 * q, q & ((1 << half) - 1), q >> half, ninv & ((1 << half) - 1), ninv >> half, r2,
                             (r2 << self.config.scale_bits) % q, (pow(self.n, -1, q) * R) % q])
            self._param_rows_cache = torch.tensor(cols, dtype=torch.int64).T.contiguous().to(self.device, self.dtype)
        return self._param_rows_cache

    def _compressed_operand(self, pt: CompressedPlaintext, ct: Ciphertext, domain: str):
        self._check_context(pt)
        if pt.level != ct.level or pt.ring_dimension != self.n:
            raise ValueError("compressed plaintext level / ring dimension does not match the ciphertext")
        if pt.polynomial_domain != domain:
            raise ValueError(f"compressed plaintext must be {domain}-domain Montgomery residues")
        data = pt.data[..., : ct.limb_count, :].contiguous()
        if data.dim() > 2 and tuple(data.shape[:-2]) != ct.batch_shape:
            raise ValueError("a batched plaintext must match the ciphertext's batch shape")
        implicit = None
        if pt.implicit_data is not None:
            implicit = pt.implicit_data[..., : ct.limb_count].contiguous()
        return data, implicit

    def _multiply_compressed(self, ct: Ciphertext, pt: CompressedPlaintext) -> Ciphertext:
        """c_i * p with a repeated operand: one fhb_op_mul_compressed launch per component."""
        data, _ = self._compressed_operand(pt, ct, "ntt")
        rows, b = ct.limb_count, ct.batch_size
        params = self._param_rows[:, ct.level: ct.level + rows]
        layout = 1 if pt.compression_layout == "cyclic" else 2
        bits = 64 if self.dtype == torch.int64 else 32
        out = torch.empty_like(ct.data)
        for c in range(ct.component_count):
            nat.check(self.ctx.lib.fhb_op_mul_compressed(
                bits, layout, nat.ptr(ct.data[c]), rows * self.n, nat.ptr(data),
                rows * pt.unique_count if data.dim() > 2 else 0, pt.unique_count, nat.ptr(out[c]), rows * self.n, b,
                rows, self.n, nat.ptr(params), params.stride(0), self._stream()), "fhb_op_mul_compressed")
        return Ciphertext(out, ct.level, ct.scale * pt.scale, "ntt", "montgomery")

    def add_plaintext(self, ct: Ciphertext, plaintext: "Plaintext | CompressedPlaintext", *,
                      inplace: bool = False) -> Ciphertext:
        """c0 + p at exactly the ciphertext's scale, coefficient/standard
        (fhelium/engine/ckks_engine.py:1964-2066): one fhb_op_add_plaintext
        launch (dense, or a compressed plaintext expanded on the fly)."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        if plaintext.scale != ct.scale:
            raise ValueError(f"add_plaintext: ciphertext scale {ct.scale} != plaintext scale {plaintext.scale}")
        implicit, istride = None, 0
        if isinstance(plaintext, CompressedPlaintext):
            pt, implicit = self._compressed_operand(plaintext, ct, "coefficient")
            layout = {"cyclic": 1, "contiguous": 2, "strided_sparse": 3}[plaintext.compression_layout]
            if implicit is not None and implicit.dim() > 1:
                istride = ct.limb_count
        else:
            pt = self._plaintext_operand(plaintext, ct, "coefficient").contiguous()
            layout = 0
        extent = pt.size(-1)
        rows, b = ct.limb_count, ct.batch_size
        out = ct.data if inplace else ct.data.clone()
        params = self._param_rows[:, ct.level: ct.level + rows]
        bits = 64 if self.dtype == torch.int64 else 32
        nat.check(self.ctx.lib.fhb_op_add_plaintext(bits, layout, nat.ptr(ct.data[0]), rows * self.n, nat.ptr(pt),
                                                    rows * extent if pt.dim() > 2 else 0, extent,
                                                    nat.ptr(implicit), istride, nat.ptr(out[0]), rows * self.n, b,
                                                    rows, self.n, nat.ptr(params), params.stride(0), self._stream()),
                  "fhb_op_add_plaintext")
        return ct if inplace else Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def add_plaintext_(self, ct: Ciphertext, plaintext: Plaintext) -> Ciphertext:
        return self.add_plaintext(ct, plaintext, inplace=True)

    def multiply_plaintext_(self, ct: Ciphertext, plaintext: Plaintext) -> Ciphertext:
        return self.multiply_plaintext(ct, plaintext, inplace=True)

    # ------------------------------------------------------------------
    # the rest of fh.CkksEngine's public API
    # (fhelium/engine/ckks_engine.py:246-262, 455-460, 1208-1345, 1491-1530,
    #  1677-1960, 2298-2346, 2560-2620)
    # ------------------------------------------------------------------
    @property
    def final_public_level(self) -> int:
        return self.public_level_count - 1

    @property
    def rng(self) -> torch.Generator:
        """The engine's seeded device generator (keys, encryption noise)."""
        return self._gen

    def set_public_key(self, key: PublicKey) -> None:
        self.validate_public_key(key)
        self._public_key = key

    @staticmethod
    def _replace(target: Ciphertext, result: Ciphertext) -> Ciphertext:
        """Give `target` the result's tensor and state (the reference's replace_)."""
        if target.data.shape == result.data.shape and target.data.dtype == result.data.dtype:
            target.data.copy_(result.data)
        else:
            target.data = result.data
        target.level, target.scale = result.level, result.scale
        target.polynomial_domain, target.residue_representation = result.polynomial_domain, result.residue_representation
        return target

    def add_(self, lhs: Ciphertext, rhs: Ciphertext) -> Ciphertext:
        return self.add(lhs, rhs, inplace=True)

    def subtract_(self, lhs: Ciphertext, rhs: Ciphertext) -> Ciphertext:
        return self.subtract(lhs, rhs, inplace=True)

    def negate(self, ct: Ciphertext, *, inplace: bool = False) -> Ciphertext:
        """-ct, canonical residues (fhelium/engine/ckks_engine.py:1919-1957)."""
        self._check_ct(ct)
        out = ct.data if inplace else torch.empty_like(ct.data)
        rows = ct.limb_count
        self.ctx.call("fhb_rns_binary", nat.OP_NEGATE, nat.ptr(ct.data), None, nat.ptr(out),
                      ct.component_count * ct.batch_size, rows, ct.level, 0, self._stream())
        if inplace:
            return ct
        return Ciphertext(out, ct.level, ct.scale, ct.polynomial_domain, ct.residue_representation)

    def negate_(self, ct: Ciphertext) -> Ciphertext:
        return self.negate(ct, inplace=True)

    def sum_ciphertexts(self, ciphertexts: Sequence[Ciphertext]) -> Ciphertext:
        if not ciphertexts:
            raise ValueError("sum_ciphertexts requires at least one value")
        result = ciphertexts[0].clone()
        for ct in ciphertexts[1:]:
            if ct.scale != result.scale:
                raise ValueError("sum_ciphertexts needs equal scales")
            self.add_(result, ct)
        return result

    def sum_ciphertext_batch(self, batch: Ciphertext, *, dim: int = 0) -> Ciphertext:
        """Sum over one batch axis by pairwise halving (fhelium/engine/ckks_engine.py:1808-1850)."""
        shape = batch.batch_shape
        if not shape:
            raise ValueError("sum_ciphertext_batch requires a batched value")
        d = dim if dim >= 0 else dim + len(shape)
        if not 0 <= d < len(shape):
            raise IndexError(f"Batch dimension {dim} is outside shape {shape}")
        cur = batch.data
        tails = []
        while cur.size(d + 1) > 1:
            count = cur.size(d + 1)
            pairs = count // 2
            if count % 2:
                tails.append(cur.narrow(d + 1, count - 1, 1))
            lhs = Ciphertext(cur.narrow(d + 1, 0, pairs).contiguous(), batch.level, batch.scale,
                             batch.polynomial_domain, batch.residue_representation)
            rhs = Ciphertext(cur.narrow(d + 1, pairs, pairs).contiguous(), batch.level, batch.scale,
                             batch.polynomial_domain, batch.residue_representation)
            cur = self.add(lhs, rhs).data
        for tail in reversed(tails):
            cur = self.add(Ciphertext(cur.contiguous(), batch.level, batch.scale, batch.polynomial_domain,
                                      batch.residue_representation),
                           Ciphertext(tail.contiguous(), batch.level, batch.scale, batch.polynomial_domain,
                                      batch.residue_representation)).data
        return Ciphertext(cur.select(d + 1, 0).contiguous(), batch.level, batch.scale, batch.polynomial_domain,
                          batch.residue_representation)

    def switch_key(self, ct: Ciphertext, key: KeySwitchKey) -> Ciphertext:
        """(c0, c1) under s_src -> (c0 + KS(c1)) under s_dst for a key made by
        create_key_switch_key(s_src, s_dst) (fhelium/engine/ckks_engine.py:1677-1706):
        the rotation path with the identity automorphism (g = 1)."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        self.validate_key_switch_key(key)
        out = torch.empty_like(ct.data)
        scratch, nbytes = self._scratch_for(ct.batch_size, ct.level)
        self.ctx.call("fhb_ckks_rotate", nat.ptr(ct.data), nat.ptr(key.data), nat.ptr(out), nat.ptr(scratch), nbytes,
                      ct.batch_size, ct.level, 1, self._stream())
        return Ciphertext(out, ct.level, ct.scale, "coefficient", "standard")

    def mod_switch_to_next_level(self, ct: Ciphertext) -> Ciphertext:
        if ct.level >= self.final_public_level:
            raise ValueError(f"level {ct.level} is already the final public level")
        return self.mod_switch_to_level(ct, ct.level + 1)

    def mod_switch_to_next_level_(self, ct: Ciphertext) -> Ciphertext:
        return self._replace(ct, self.mod_switch_to_next_level(ct))

    def mod_switch_to_level_(self, ct: Ciphertext, target_level: int) -> Ciphertext:
        return self._replace(ct, self.mod_switch_to_level(ct, target_level))

    def rescale_to_next_level_(self, ct: Ciphertext, *, rounding: str = "nearest") -> Ciphertext:
        return self._replace(ct, self.rescale_to_next_level(ct, rounding=rounding))

    def reinterpret_at_scale_(self, ct: Ciphertext, target_scale: float, *,
                              max_relative_change: float | None = None) -> Ciphertext:
        if max_relative_change is not None and abs(target_scale / ct.scale - 1.0) > max_relative_change:
            raise ValueError("target scale changes the value by more than max_relative_change")
        ct.scale = float(target_scale)
        return ct

    def encrypt_zero_like(self, ct: Ciphertext, public_key: PublicKey | None = None) -> Ciphertext:
        """A fresh encryption of zero in ct's level, scale, batch and domain."""
        self._check_ct(ct)
        zero = torch.zeros((*ct.batch_shape, self.num_slots), dtype=torch.complex128, device=self.device)
        result = self.encrypt_message(zero, public_key, level=ct.level, scale=ct.scale)
        return self.coefficient_domain_to_ntt_domain_(result) if ct.polynomial_domain == "ntt" else result

    def rotate_by_step_(self, ct: Ciphertext, rotation_step: int) -> Ciphertext:
        return self._replace(ct, self.rotate_by_step(ct, rotation_step))

    def rotate_many_with_keys(self, ct: Ciphertext, rotation_keys: Sequence[RotationKey], *,
                              use_hoisting: bool = True) -> list[Ciphertext]:
        """One rotation per caller-owned key, sharing one ModUp when hoisting."""
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        self._check_ct(ct)
        for key in rotation_keys:
            self.validate_key_switch_key(key)
        if not use_hoisting or len(rotation_keys) < 2:
            return [self.rotate_with_key(ct, k) for k in rotation_keys]
        prepared = self.prepare_rotation_digits(ct)
        return [self.apply_prepared_rotation(ct, prepared, k) for k in rotation_keys]

    def validate_ciphertext(self, ciphertext: Ciphertext) -> None:
        if not isinstance(ciphertext, Ciphertext):
            raise TypeError(f"Expected Ciphertext, got {type(ciphertext).__name__}")
        self._check_ct(ciphertext)

    def validate_public_key(self, key: PublicKey) -> None:
        if type(key) is not PublicKey:
            raise TypeError(f"Expected PublicKey, got {type(key).__name__}")
        d = key.data
        if d.device != self.device or d.dtype != self.dtype or tuple(d.shape) != (2, self.num_q, self.n):
            raise ValueError(f"public key must be [2, {self.num_q}, {self.n}] {self.dtype} on {self.device}")

    def validate_key_switch_key(self, key: KeySwitchKey) -> None:
        if not isinstance(key, KeySwitchKey):
            raise TypeError(f"Expected KeySwitchKey, got {type(key).__name__}")
        d = key.data
        want = (self.key_digit_count, 2, self.qp_rows, self.n)
        if d.device != self.device or d.dtype != self.dtype or tuple(d.shape) != want or not d.is_contiguous():
            raise ValueError(f"key-switch key must be a contiguous {list(want)} {self.dtype} tensor on {self.device}")
        if isinstance(key, RotationKey):
            if type(key.rotation_step) is not int:
                raise TypeError("RotationKey rotation_step must be an integer")

    def __repr__(self) -> str:
        return f"CkksEngine({self.config}, device={self.device})"
