"""CPU oracle for the CKKS evaluation path (test infrastructure only).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it.
It restates the reference's (visualDust/fhelium 0.10.0) host-side table
construction and per-operation orchestration in numpy, and calls the C
restatement of the reference CPU kernels in ``fhe_oracle.c`` through ctypes.

Citations are relative to the reference project root.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from functools import cached_property

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "fhe_oracle.c")
_LIB = os.path.join(_HERE, "_build", "libfhe_oracle.so")


def build_oracle(force: bool = False) -> str:
    """Compile ``fhe_oracle.c`` with gcc into ``oracle/_build``."""
    if (
        not force
        and os.path.exists(_LIB)
        and os.path.getmtime(_LIB) >= os.path.getmtime(_SRC)
    ):
        return _LIB
    os.makedirs(os.path.dirname(_LIB), exist_ok=True)
    tmp = _LIB + f".{os.getpid()}.tmp"
    subprocess.run(
        ["gcc", "-O3", "-march=native", "-fPIC", "-shared", "-o", tmp, _SRC],
        check=True,
    )
    os.replace(tmp, _LIB)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build_oracle())
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


I64 = ctypes.c_int64
INT = ctypes.c_int


# ---------------------------------------------------------------------------
# Thin wrappers: each maps onto one C routine.  Arrays are int64 [batch, rows, n].
# ---------------------------------------------------------------------------


def montgomery_mul(a, b, params, radix_bits):
    a, b, params = _i64(a), _i64(b), _i64(params)
    out = np.empty_like(a)
    bsz, limbs, n = a.reshape(-1, a.shape[-2], a.shape[-1]).shape
    lib().orc_montgomery_mul(_p(out), _p(a), _p(b), I64(bsz), I64(limbs), I64(n),
                             _p(params), INT(radix_bits))
    return out


def add_lazy(a, b, params):
    a, b, params = _i64(a), _i64(b), _i64(params)
    out = np.empty_like(a)
    bsz, limbs, n = a.reshape(-1, a.shape[-2], a.shape[-1]).shape
    lib().orc_add_lazy(_p(out), _p(a), _p(b), I64(bsz), I64(limbs), I64(n), _p(params))
    return out


def add_canonical(a, b, moduli):
    a, b, moduli = _i64(a), _i64(b), _i64(moduli)
    out = np.empty_like(a)
    bsz, limbs, n = a.reshape(-1, a.shape[-2], a.shape[-1]).shape
    lib().orc_add_canonical(_p(out), _p(a), _p(b), I64(bsz), I64(limbs), I64(n), _p(moduli))
    return out


def forward_ntt(x, twiddles, params, radix_bits, to_montgomery=True):
    x = _i64(x).copy()
    twiddles, params = _i64(twiddles), _i64(params)
    bsz, limbs, n = x.reshape(-1, x.shape[-2], x.shape[-1]).shape
    lib().orc_forward_ntt(_p(x), I64(bsz), I64(limbs), INT(n.bit_length() - 1),
                          _p(twiddles), _p(params), INT(radix_bits), INT(1 if to_montgomery else 0))
    return x


def inverse_ntt_to_standard(x, inv_twiddles, params, radix_bits):
    x = _i64(x).copy()
    inv_twiddles, params = _i64(inv_twiddles), _i64(params)
    bsz, limbs, n = x.reshape(-1, x.shape[-2], x.shape[-1]).shape
    lib().orc_inverse_ntt_to_standard(_p(x), I64(bsz), I64(limbs), INT(n.bit_length() - 1),
                                      _p(inv_twiddles), _p(params), INT(radix_bits))
    return x


def mixed_radix_decompose(src, normalizers, propagation, params, radix_bits):
    src = _i64(src)
    out = np.empty_like(src)
    bsz, rows, n = src.reshape(-1, src.shape[-2], src.shape[-1]).shape
    norm = _i64(normalizers) if rows > 1 else np.zeros(1, np.int64)
    prop = _i64(propagation) if rows > 1 else np.zeros(1, np.int64)
    lib().orc_mixed_radix_decompose(_p(out), _p(src), I64(bsz), I64(rows), I64(n),
                                    _p(norm), _p(prop), _p(_i64(params)), INT(radix_bits))
    return out


def basis_extend_to_montgomery(digits, coeffs, params, radix_bits):
    digits = _i64(digits)
    params = _i64(params)
    dst = params.shape[1]
    lead = digits.shape[:-2]
    bsz, drows, n = digits.reshape(-1, digits.shape[-2], digits.shape[-1]).shape
    coeffs = _i64(coeffs) if drows > 1 else np.zeros((1, dst), np.int64)
    out = np.empty((*lead, dst, n), dtype=np.int64)
    lib().orc_basis_extend_to_montgomery(_p(out), _p(digits), I64(bsz), I64(drows), I64(n),
                                         _p(coeffs), I64(coeffs.shape[1]), _p(params),
                                         I64(dst), INT(radix_bits))
    return out


def keyswitch_accumulate(acc0, acc1, digit, key_digit, params, key_row_start, radix_bits):
    digit, key_digit, params = _i64(digit), _i64(key_digit), _i64(params)
    acc0 = _i64(acc0).copy()
    acc1 = _i64(acc1).copy()
    bsz, rows, n = digit.reshape(-1, digit.shape[-2], digit.shape[-1]).shape
    lib().orc_keyswitch_accumulate(_p(acc0), _p(acc1), _p(digit), _p(key_digit),
                                   I64(key_digit.shape[1]), I64(key_row_start), I64(bsz),
                                   I64(rows), I64(n), _p(params), INT(radix_bits))
    return acc0, acc1


def keyswitch_moddown(q_res, p_res, inverse, params, radix_bits):
    q_res, p_res, inverse, params = _i64(q_res), _i64(p_res), _i64(inverse), _i64(params)
    lead = q_res.shape[:-2]
    qn, n = q_res.shape[-2:]
    pn = p_res.shape[-2]
    bsz = int(np.prod(lead)) if lead else 1
    out = np.empty_like(q_res)
    lib().orc_keyswitch_moddown(_p(out), _p(q_res), _p(p_res), I64(bsz), I64(qn), I64(pn),
                                I64(n), _p(inverse), I64(inverse.shape[1]), _p(params),
                                INT(radix_bits))
    return out


def rescale_drop_leading(remaining, dropped, inverse_mont, params, half_drop, nearest, radix_bits):
    remaining, dropped = _i64(remaining), _i64(dropped)
    inverse_mont, params = _i64(inverse_mont), _i64(params)
    bsz, rows, n = remaining.reshape(-1, remaining.shape[-2], remaining.shape[-1]).shape
    out = np.empty_like(remaining)
    lib().orc_rescale_drop_leading(_p(out), _p(remaining), _p(dropped), I64(bsz), I64(rows),
                                   I64(n), _p(inverse_mont), _p(params), I64(half_drop),
                                   INT(1 if nearest else 0), INT(radix_bits))
    return out


def coefficient_automorphism(x, src, sign, twice_moduli):
    x = _i64(x)
    src = np.ascontiguousarray(src, dtype=np.int32)
    sign = np.ascontiguousarray(sign, dtype=np.int8)
    bsz, limbs, n = x.reshape(-1, x.shape[-2], x.shape[-1]).shape
    out = np.empty_like(x)
    lib().orc_coefficient_automorphism(_p(out), _p(x), I64(bsz), I64(limbs), I64(n),
                                       _p(src), _p(sign), _p(_i64(twice_moduli)))
    return out


def ntt_automorphism(x, src):
    x = _i64(x)
    src = np.ascontiguousarray(src, dtype=np.int32)
    bsz, limbs, n = x.reshape(-1, x.shape[-2], x.shape[-1]).shape
    out = np.empty_like(x)
    lib().orc_ntt_automorphism(_p(out), _p(x), I64(bsz), I64(limbs), I64(n), _p(src))
    return out


# ---------------------------------------------------------------------------
# Tables (restating the reference's Python table builders with big integers)
# ---------------------------------------------------------------------------


def primitive_2nth_root(q: int, n: int) -> int:
    """First c^((q-1)/2N), c = 2, 3, ..., whose N-th power is not 1
    (fhelium/engine/ntt/plans/twiddles.py:10-20)."""
    e = (q - 1) // (2 * n)
    for c in range(2, n):
        r = pow(c, e, q)
        if pow(r, n, q) != 1:
            return r
    raise RuntimeError("no primitive root")


def bit_reverse_table(log_n: int) -> np.ndarray:
    n = 1 << log_n
    idx = np.arange(n, dtype=np.int64)
    out = np.zeros(n, dtype=np.int64)
    for _ in range(log_n):
        out = (out << 1) | (idx & 1)
        idx >>= 1
    return out


def _powers_mod(root: int, n: int, q: int) -> np.ndarray:
    out = np.empty(n, dtype=object)
    v = 1
    for i in range(n):
        out[i] = v
        v = (v * root) % q
    return out


def galois_element(n: int, step: int, generator: int = 3) -> int:
    """fhelium/engine/galois.py:10-26."""
    e = -int(step) if generator == 5 else int(step)
    return pow(generator, e % n, 2 * n)


def coefficient_galois_tables(n: int, g: int):
    """Destination j reads source[j] with sign[j] (fhelium/engine/galois.py:49-83)."""
    m = 2 * n
    src = np.arange(n, dtype=np.int64)
    mapped = (g * src) % m
    dst = mapped % n
    sign = np.where(((mapped // n) & 1) != 0, -1, 1).astype(np.int8)
    src_idx = np.empty(n, dtype=np.int32)
    src_idx[dst] = src.astype(np.int32)
    src_sign = np.empty(n, dtype=np.int8)
    src_sign[dst] = sign
    return src_idx, src_sign


def ntt_galois_source_indices(n: int, g: int) -> np.ndarray:
    """fhelium/engine/hybrid_keyswitch.py:506-528."""
    br = bit_reverse_table(n.bit_length() - 1)
    dest_exp = 2 * br + 1
    src_br = ((dest_exp * g) % (2 * n) - 1) // 2
    return br[src_br].astype(np.int32)


@dataclass
class OracleContext:
    """Level-zero tables for one modulus chain ``[Q | P]``.

    moduli: scale primes, structural base prime, then P primes
    (fhelium/config/ckks.py:504-535).  radix_bits is 62 (int64) or 30 (int32).
    """

    moduli: tuple
    log_n: int
    num_q: int
    num_p: int
    radix_bits: int
    scale_bits: int = 40

    @property
    def n(self) -> int:
        return 1 << self.log_n

    @property
    def R(self) -> int:
        return 1 << self.radix_bits

    @cached_property
    def params(self) -> np.ndarray:
        """[8, QP] table (fhelium/engine/rns/runtime.py:136-216)."""
        half = self.radix_bits // 2
        mask = (1 << half) - 1
        R = self.R
        rows = []
        for q in self.moduli:
            neg_inv = (-pow(q, -1, R)) % R
            rows.append([
                2 * q, q & mask, q >> half, neg_inv & mask, neg_inv >> half,
                (R * R) % q, (((R * R) % q) * (1 << self.scale_bits)) % q,
                (pow(self.n, -1, q) * R) % q,
            ])
        return np.array(rows, dtype=np.int64).T.copy()

    @cached_property
    def twiddles(self) -> tuple:
        """Montgomery-form bit-reversed psi and psi^-1 powers per prime."""
        fwd = np.empty((len(self.moduli), self.n), dtype=np.int64)
        inv = np.empty_like(fwd)
        for j, q in enumerate(self.moduli):
            psi = primitive_2nth_root(q, self.n)
            lib().orc_twiddles(ctypes.c_uint64(q), ctypes.c_uint64(psi), ctypes.c_uint64(pow(psi, -1, q)),
                               INT(self.log_n), INT(self.radix_bits), _p(fwd[j]), _p(inv[j]))
        return fwd, inv

    # --- layout (fhelium/engine/rns/{chain,decomposition,layout}.py) ---------
    def q_rows(self, level: int) -> list:
        return list(range(level, self.num_q))

    def qp_rows(self, level: int) -> list:
        return list(range(level, self.num_q + self.num_p))

    @cached_property
    def level_zero_digits(self) -> list:
        scale = list(range(self.num_q - 1))
        w = self.num_p
        digits = [tuple(scale[s:s + w]) for s in range(0, len(scale), w)]
        return digits + [(self.num_q - 1,)]

    def digits_at_level(self, level: int) -> list:
        """(key_digit_index, prime_ids) of the active digits."""
        out = []
        for kd, fixed in enumerate(self.level_zero_digits):
            ids = tuple(i for i in fixed if i >= level)
            if ids:
                out.append((kd, ids))
        return out

    def digit_tables(self, prime_ids: tuple):
        """Mixed-radix normalizers/propagation and basis-extension
        coefficients (fhelium/engine/rns/parameters.py:172-259)."""
        R = self.R
        mods = [self.moduli[i] for i in prime_ids]
        w = len(mods)
        prods = [mods[0]]
        for i in range(1, w - 1):
            prods.append(prods[-1] * mods[i])
        norm = []
        prop = np.zeros((max(w - 1, 0), w), dtype=np.int64)
        for c in range(w - 1):
            inv = pow(prods[c], -1, mods[c + 1])
            norm.append((inv * R) % mods[c + 1])
            for t in range(c + 2, w):
                prop[c, t] = (prods[c] * R) % mods[t]
        dest = list(self.moduli)
        r2 = [(R * R) % m for m in dest]
        ext = np.array([[(bp * r) % m for r, m in zip(r2, dest)] for bp in prods[: w - 1]],
                       dtype=np.int64).reshape(max(w - 1, 0), len(dest))
        return np.array(norm, dtype=np.int64), prop, ext

    def moddown_inverse(self, level: int) -> np.ndarray:
        """[P, surviving] packed p_drop^{-1} R tables
        (fhelium/engine/ckks_engine.py:2991-3048)."""
        R = self.R
        pm = list(self.moduli[-self.num_p:])[::-1]
        total = len(self.moduli)
        base_rows = []
        for step, dp in enumerate(pm):
            row = [(pow(dp, -1, self.moduli[pid]) * R) % self.moduli[pid]
                   for pid in range(total - step - 1)]
            base_rows.append(row[level:])
        width = max(len(r) for r in base_rows)
        packed = np.zeros((self.num_p, width), dtype=np.int64)
        for i, r in enumerate(base_rows):
            packed[i, : len(r)] = r
        return packed

    def rescale_inverse(self, level: int) -> np.ndarray:
        """q_drop^{-1} R mod r_i over the surviving QP rows
        (fhelium/engine/ckks_engine.py:2952-2989)."""
        ids = self.qp_rows(level)
        qd = self.moduli[ids[0]]
        return np.array([(pow(qd, -1, self.moduli[i]) * self.R) % self.moduli[i]
                         for i in ids[1:]], dtype=np.int64)

    def sub_params(self, rows: list) -> np.ndarray:
        return np.ascontiguousarray(self.params[:, rows])

    # --- representation transitions -----------------------------------------
    def forward_to_montgomery(self, x: np.ndarray, rows: list) -> np.ndarray:
        fwd, _ = self.twiddles
        return forward_ntt(x, fwd[rows], self.sub_params(rows), self.radix_bits, True)

    def forward_montgomery(self, x: np.ndarray, rows: list) -> np.ndarray:
        fwd, _ = self.twiddles
        return forward_ntt(x, fwd[rows], self.sub_params(rows), self.radix_bits, False)

    def inverse_to_standard(self, x: np.ndarray, rows: list) -> np.ndarray:
        _, inv = self.twiddles
        return inverse_ntt_to_standard(x, inv[rows], self.sub_params(rows), self.radix_bits)

    def canonical(self, x: np.ndarray, rows: list) -> np.ndarray:
        q = np.array([self.moduli[i] for i in rows], dtype=np.int64)
        return np.mod(x, q[:, None])

    # --- CKKS operations ------------------------------------------------------
    def multiply(self, a: np.ndarray, b: np.ndarray, level: int) -> np.ndarray:
        """NTT-domain tensor product (fhelium/engine/ckks_engine.py:1570-1606).
        a, b: [2, *batch, L, N] -> [3, *batch, L, N]."""
        rows = self.q_rows(level)
        prm = self.sub_params(rows)
        rb = self.radix_bits
        d0 = montgomery_mul(a[0], b[0], prm, rb)
        x01 = montgomery_mul(a[0], b[1], prm, rb)
        x10 = montgomery_mul(a[1], b[0], prm, rb)
        d1 = add_lazy(x01, x10, prm)
        d2 = montgomery_mul(a[1], b[1], prm, rb)
        return np.stack([d0, d1, d2])

    def extend_digit(self, component: np.ndarray, level: int, prime_ids: tuple) -> np.ndarray:
        """Mixed-radix decompose + basis extension of one digit
        (fhelium/engine/hybrid_keyswitch.py:95-237)."""
        rows = [i - level for i in prime_ids]
        src = np.ascontiguousarray(component[..., rows[0]: rows[-1] + 1, :])
        norm, prop, ext = self.digit_tables(prime_ids)
        if len(prime_ids) > 1:
            digits = mixed_radix_decompose(src, norm, prop, self.sub_params(list(prime_ids)),
                                           self.radix_bits)
        else:
            digits = src
        dst = self.qp_rows(level)
        coeffs = ext[:, dst] if len(prime_ids) > 1 else np.zeros((0, len(dst)), np.int64)
        return basis_extend_to_montgomery(digits, coeffs, self.sub_params(dst), self.radix_bits)

    def _moddown(self, acc0, acc1, level):
        qp = self.qp_rows(level)
        acc0 = self.inverse_to_standard(acc0, qp)
        acc1 = self.inverse_to_standard(acc1, qp)
        inv = self.moddown_inverse(level)
        prm = self.sub_params(qp)
        p = self.num_p
        c0 = keyswitch_moddown(acc0[..., :-p, :], acc0[..., -p:, :], inv, prm, self.radix_bits)
        c1 = keyswitch_moddown(acc1[..., :-p, :], acc1[..., -p:, :], inv, prm, self.radix_bits)
        return c0, c1

    def keyswitch(self, component: np.ndarray, key: np.ndarray, level: int):
        """Streaming hybrid key switch of one coefficient/standard component
        (fhelium/engine/hybrid_keyswitch.py:321-371).  key: [D, 2, QP0, N]."""
        qp = self.qp_rows(level)
        prm = self.sub_params(qp)
        acc0 = acc1 = None
        for kd, ids in self.digits_at_level(level):
            y = self.extend_digit(component, level, ids)
            y = self.forward_montgomery(y, qp)
            if acc0 is None:
                acc0 = np.zeros_like(y)
                acc1 = np.zeros_like(y)
            acc0, acc1 = keyswitch_accumulate(acc0, acc1, y, key[kd], prm, level, self.radix_bits)
        return self._moddown(acc0, acc1, level)

    def relinearize(self, ct3: np.ndarray, rlk: np.ndarray, level: int) -> np.ndarray:
        """fhelium/engine/ckks_engine.py:1642-1675."""
        rows = self.q_rows(level)
        d0 = self.inverse_to_standard(ct3[0], rows)
        d1 = self.inverse_to_standard(ct3[1], rows)
        d2 = self.inverse_to_standard(ct3[2], rows)
        c0, c1 = self.keyswitch(d2, rlk, level)
        q = np.array([self.moduli[i] for i in rows], dtype=np.int64)[:, None]
        return np.stack([np.mod(d0 + c0, q), np.mod(d1 + c1, q)])

    def rescale(self, ct: np.ndarray, level: int, nearest: bool = True) -> np.ndarray:
        """fhelium/engine/ckks_rescale.py:339-377."""
        rows = self.q_rows(level)
        inv = self.rescale_inverse(level)[: len(rows) - 1]
        prm = self.sub_params(rows[1:])
        half = self.moduli[rows[0]] // 2
        return np.stack([
            rescale_drop_leading(c[..., 1:, :], c[..., 0, :], inv, prm, half, nearest,
                                 self.radix_bits)
            for c in ct
        ])

    def automorphism(self, x: np.ndarray, step: int, rows: list, generator: int = 3):
        g = galois_element(self.n, step % self.n, generator)
        src, sign = coefficient_galois_tables(self.n, g)
        tq = np.array([2 * self.moduli[i] for i in rows], dtype=np.int64)
        return coefficient_automorphism(x, src, sign, tq)

    def rotate(self, ct: np.ndarray, step: int, key: np.ndarray, level: int,
               generator: int = 3) -> np.ndarray:
        """Direct-key rotation (fhelium/engine/ckks_engine.py:3822-3897,3334-3350)."""
        rows = self.q_rows(level)
        if step % self.n == 0:
            return ct.copy()
        r0 = self.automorphism(ct[0], step, rows, generator)
        r1 = self.automorphism(ct[1], step, rows, generator)
        c0, c1 = self.keyswitch(r1, key, level)
        moduli = np.array([self.moduli[i] for i in rows], dtype=np.int64)
        return np.stack([add_canonical(r0, c0, moduli), c1])

    def prepare_rotation_digits(self, c1: np.ndarray, level: int) -> np.ndarray:
        """fhelium/engine/hybrid_keyswitch.py:373-417."""
        qp = self.qp_rows(level)
        return np.stack([
            self.forward_montgomery(self.extend_digit(c1, level, ids), qp)
            for _, ids in self.digits_at_level(level)
        ])

    def rotate_hoisted(self, ct: np.ndarray, steps: list, keys: dict, level: int,
                       generator: int = 3) -> list:
        """Hoisted rotations sharing one ModUp
        (fhelium/engine/ckks_engine.py:3787-3820, hybrid_keyswitch.py:419-595)."""
        rows = self.q_rows(level)
        qp = self.qp_rows(level)
        prm = self.sub_params(qp)
        moduli = np.array([self.moduli[i] for i in rows], dtype=np.int64)
        prepared = self.prepare_rotation_digits(ct[1], level)
        out = []
        for step in steps:
            if step % self.n == 0:
                out.append(ct.copy())
                continue
            g = galois_element(self.n, step % self.n, generator)
            src = ntt_galois_source_indices(self.n, g)
            acc0 = np.zeros_like(prepared[0])
            acc1 = np.zeros_like(prepared[0])
            for (kd, _), dig in zip(self.digits_at_level(level), prepared):
                acc0, acc1 = keyswitch_accumulate(acc0, acc1, ntt_automorphism(dig, src),
                                                  keys[step][kd], prm, level, self.radix_bits)
            c0, c1 = self._moddown(acc0, acc1, level)
            r0 = self.automorphism(ct[0], step, rows, generator)
            out.append(np.stack([add_canonical(r0, c0, moduli), c1]))
        return out
