"""Full-slot CKKS bootstrapping on the B200 engine.

Same contract as the reference's experimental FullSlotBootstrap
(fhelium/experimental/bootstrap/_full_slot.py:339-490, preset
presets/cosine.py:38-83): refresh a final-public-level, generator-5,
full-slot ciphertext by ModRaise -> CoeffsToSlots -> conjugate split ->
cosine / double-angle modular reduction -> recombination -> SlotsToCoeffs,
with BSGS diagonal linear transforms (baby step 16, hoisted baby rotations),
two collapsed radix-2 stages per transform, a degree-44 Chebyshev seed and
seven double-angle steps for an input bound of B = 1024 (|u| <= 512 in units
of the base prime, where the reference counts sin(pi r) with r = 2u).

The construction below is this library's own (derived here, not ported):

Decoding for generator 5: slot j = sum_k t_k zeta^(k 5^j), zeta = e^(i pi/N).
With n = N/2 and z_k = t_k + i t_(k+n) (zeta^(n 5^j) = i), slots s = V z with
V[j,k] = zeta^(k 5^j), and V^-1 = V^H / n.  Splitting k even/odd gives the
radix-2 recursion V x = [E + D O; E - D O], D_j = zeta^(5^j), so
V = F_n ... F_4 F_2 P, P the bit-reversal permutation and F_len the butterfly
stage with twiddles rho_len^(5^j mod 4 len), rho_len = zeta^(n/len).
  * CoeffsToSlots computes w = F_2^-1 ... F_n^-1 s = P z / n (bit-reversed),
    so no permutation is ever evaluated homomorphically;
  * SlotsToCoeffs computes F_n ... F_2 w' = V z' on the bit-reversed w'.
Each transform is split into two groups of stages whose product matrices have
at most 256 non-zero diagonals (offsets u*m, u = 1 or 128); a diagonal-form
matrix sum_d M_d * shift(v, d) is evaluated as
sum_k shift(sum_b shift(M_(g k + b), -g k) * shift(v, b), g k) (BSGS).
Diagonals are encoded at scale q_l (the prime the following rescale drops)
so every transform stage keeps the ciphertext scale exactly.

Modular reduction: x = u / B' with u = t / q_b (t the raised coefficient),
z0 ~ cos(2 pi (B' x - 1/4) / 2^R) by Chebyshev interpolation of degree 44 on
[-1, 1] (evaluated by Paterson-Stockmeyer in the Chebyshev basis), then R
double-angle steps z <- 2 z^2 - 1 give sin(2 pi u); the factor
q_b / (2 pi Delta) returning to message units is folded into SlotsToCoeffs.
All ciphertext products are relinearised and rescaled with their actual
scales tracked; terms are aligned to a common level and scale by integer
constants before every addition.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .engine import CkksEngine
from .values import Ciphertext


# ---------------------------------------------------------------------------
# Plaintext linear algebra in diagonal form
# ---------------------------------------------------------------------------

def _stage(n: int, length: int, inverse: bool) -> dict[int, np.ndarray]:
    """Butterfly stage F_len (or its inverse) as {offset: diagonal}:
    (M v)[x] = sum_d M_d[x] v[(x + d) mod n]."""
    h = length // 2
    x = np.arange(n)
    p = x % length
    top = p < h
    j = np.where(top, p, p - h)
    # rho_len = zeta^(n/len) = exp(2 pi i / (4 len)); butterfly j uses rho_len^(5^j mod 4 len)
    e = np.array([pow(5, int(jj), 4 * length) for jj in range(h)], dtype=np.int64)[j]
    omega = np.exp(2j * np.pi * e / (4 * length))
    d0 = np.zeros(n, complex)
    dp = np.zeros(n, complex)
    dm = np.zeros(n, complex)
    if not inverse:
        d0[top] = 1.0
        dp[top] = omega[top]
        dm[~top] = 1.0
        d0[~top] = -omega[~top]
    else:
        d0[top] = 0.5
        dp[top] = 0.5
        dm[~top] = np.conj(omega[~top]) * 0.5
        d0[~top] = -np.conj(omega[~top]) * 0.5
    out = {0: d0}
    for d, v in ((h % n, dp), ((-h) % n, dm)):  # +h and -h coincide when len = n
        out[d] = out[d] + v if d in out else v
    return out


def _compose(a: dict[int, np.ndarray], b: dict[int, np.ndarray], n: int) -> dict[int, np.ndarray]:
    """Diagonal form of A @ B (B applied first): C_(a+b) += A_a * shift(B_b, a)."""
    out: dict[int, np.ndarray] = {}
    for da, va in a.items():
        for db, vb in b.items():
            d = (da + db) % n
            term = va * np.roll(vb, -da)
            if d in out:
                out[d] = out[d] + term
            else:
                out[d] = term
    return {d: v for d, v in out.items() if np.max(np.abs(v)) > 1e-13}


def _group(n: int, lengths: list[int], inverse: bool) -> dict[int, np.ndarray]:
    """Product of stages, applied in the listed order."""
    m = _stage(n, lengths[0], inverse)
    for length in lengths[1:]:
        m = _compose(_stage(n, length, inverse), m, n)
    return m


def apply_diagonal_matrix(diags: dict[int, np.ndarray], v: np.ndarray) -> np.ndarray:
    """Plaintext reference of (M v)[x] = sum_d M_d[x] v[x + d]."""
    out = np.zeros_like(v, dtype=complex)
    for d, m in diags.items():
        out += m * np.roll(v, -d)
    return out


@dataclass
class _BsgsPlan:
    unit: int
    baby: int
    giants: list[int]           # k values
    entries: list[tuple[int, int, np.ndarray]]  # (k, b, pre-rotated diagonal)

    @property
    def baby_shifts(self) -> list[int]:
        return [self.unit * b for b in range(self.baby)]

    @property
    def giant_shifts(self) -> list[int]:
        return [self.unit * self.baby * k for k in self.giants]


def _bsgs_plan(diags: dict[int, np.ndarray], n: int, unit: int, baby: int, signed: bool) -> _BsgsPlan:
    entries = []
    giants = set()
    for d, m in diags.items():
        if d % unit:
            raise ValueError("diagonal offset not a multiple of the BSGS unit")
        mm = d // unit
        if signed and mm > (n // unit) // 2:
            mm -= n // unit
        k, b = divmod(mm, baby)
        giants.add(k)
        entries.append((k, b, np.roll(m, unit * baby * k)))  # shift(M, -g k)
    return _BsgsPlan(unit, baby, sorted(giants), entries)


# ---------------------------------------------------------------------------
# Chebyshev interpolation
# ---------------------------------------------------------------------------

def chebyshev_coefficients(fn, degree: int) -> np.ndarray:
    """Interpolation at the degree+1 Chebyshev nodes on [-1, 1]."""
    k = np.arange(degree + 1)
    nodes = np.cos(np.pi * (k + 0.5) / (degree + 1))
    vals = fn(nodes)
    coeffs = np.array([2.0 / (degree + 1) * np.sum(vals * np.cos(np.pi * j * (k + 0.5) / (degree + 1)))
                       for j in range(degree + 1)])
    coeffs[0] /= 2.0
    return coeffs


def chebyshev_eval(coeffs: np.ndarray, x: np.ndarray) -> np.ndarray:
    return np.polynomial.chebyshev.chebval(x, coeffs)


# ---------------------------------------------------------------------------
# The bootstrap
# ---------------------------------------------------------------------------

class FullSlotBootstrap:
    """Refresh a final-public-level full-slot ciphertext (generator 5)."""

    def __init__(self, engine: CkksEngine, *, input_bound: int = 1024, double_angle_iterations: int = 7,
                 chebyshev_degree: int = 44, baby_step: int = 16, split: int = 7,
                 modulus_raise_target_level: int = 0, ps_baby: int = 8):
        if engine.galois_generator != 5:
            raise ValueError("full-slot bootstrapping uses the generator-5 slot order")
        self.engine = engine
        self.n = engine.num_slots
        self.log_n = self.n.bit_length() - 1
        self.bound = input_bound / 2.0  # bound on |u| (units of the base prime)
        self.R = double_angle_iterations
        self.degree = chebyshev_degree
        self.baby = baby_step
        self.target = modulus_raise_target_level
        self.delta = engine.config.default_scale
        nq = engine.num_q
        self.q_base = engine.moduli[nq - 1]
        lens = [1 << i for i in range(1, self.log_n + 1)]          # 2 .. n
        low, high = lens[:split], lens[split:]
        # CoeffsToSlots: F_n^-1 first ... F_2^-1 last; SlotsToCoeffs: F_2 first ... F_n last
        self.cts_groups = [(_group(self.n, high[::-1], True), high[0] // 2),
                           (_group(self.n, low[::-1], True), 1)]
        self.stc_groups = [(_group(self.n, low, False), 1),
                           (_group(self.n, high, False), high[0] // 2)]
        # normalisations folded into the first/last transform stage
        cts_scale = self.delta / (2.0 * self.bound * self.q_base)
        self.cts_groups[1] = ({d: v * cts_scale for d, v in self.cts_groups[1][0].items()}, 1)
        stc_scale = self.q_base / (2.0 * math.pi * self.delta)
        self.stc_groups[0] = ({d: v * stc_scale for d, v in self.stc_groups[0][0].items()}, 1)
        self.cts_plans = [_bsgs_plan(m, self.n, unit, self.baby, signed=(unit == 1)) for m, unit in self.cts_groups]
        self.stc_plans = [_bsgs_plan(m, self.n, unit, self.baby, signed=(unit == 1)) for m, unit in self.stc_groups]
        phase = 2 ** self.R
        self.seed = chebyshev_coefficients(
            lambda x: np.cos(2.0 * np.pi * (self.bound * x - 0.25) / phase), self.degree)
        self.ps_baby = ps_baby
        self.cheb_depth = self._ps_depth()
        self.levels = self._level_schedule()
        self._pt_cache: dict = {}

    # -- bookkeeping ---------------------------------------------------------
    def _level_schedule(self):
        l0 = self.target
        cts = [l0, l0 + 1]
        evalmod_in = l0 + 2
        evalmod_out = evalmod_in + self.cheb_depth + self.R
        stc = [evalmod_out, evalmod_out + 1]
        return {"cts": cts, "evalmod_in": evalmod_in, "evalmod_out": evalmod_out, "stc": stc,
                "output": evalmod_out + 2}

    @property
    def output_level(self) -> int:
        return self.levels["output"]

    def rotation_steps(self) -> list[int]:
        steps = set()
        for plan in self.cts_plans + self.stc_plans:
            for s in plan.baby_shifts + plan.giant_shifts:
                if s % self.n:
                    steps.add((-s) % self.n)  # shift(v, d) = rotate(v, -d)
        return sorted(steps)

    def generate_keys(self) -> None:
        eng = self.engine
        eng.relinearization_key
        for s in self.rotation_steps():
            eng.rotation_key(s)
        if getattr(self, "_conj", None) is None:
            self._conj = eng.create_conjugation_key()

    # -- plaintext diagonals --------------------------------------------------
    def _plaintexts(self, name: str, plan: _BsgsPlan, level: int):
        key = (name, level)
        if key not in self._pt_cache:
            eng = self.engine
            q = float(eng.moduli[level])
            slots = torch.tensor(np.stack([m for _, _, m in plan.entries]), dtype=torch.complex128)
            pts = []
            chunk = 16
            for i in range(0, len(plan.entries), chunk):
                pts.append(eng.encode_plaintext(slots[i:i + chunk].to(eng.device), level=level, scale=q))
            self._pt_cache[key] = torch.cat(pts)
        return self._pt_cache[key]

    def precompute(self) -> None:
        for i, plan in enumerate(self.cts_plans):
            self._plaintexts(f"cts{i}", plan, self.levels["cts"][i])
        for i, plan in enumerate(self.stc_plans):
            self._plaintexts(f"stc{i}", plan, self.levels["stc"][i])

    # -- homomorphic pieces -----------------------------------------------------
    def _table(self, name: str, plan: _BsgsPlan) -> torch.Tensor:
        """[giants, babies] int32 device table of plaintext entry indices (-1: none)."""
        key = ("table", name)
        if key not in self._pt_cache:
            t = np.full((len(plan.giants), plan.baby), -1, dtype=np.int32)
            gidx = {k: i for i, k in enumerate(plan.giants)}
            for e, (k, b, _) in enumerate(plan.entries):
                t[gidx[k], b] = e
            self._pt_cache[key] = torch.from_numpy(t).to(self.engine.device)
        return self._pt_cache[key]

    def _linear(self, ct: Ciphertext, name: str, plan: _BsgsPlan) -> Ciphertext:
        eng = self.engine
        pts = self._plaintexts(name, plan, ct.level)
        table = self._table(name, plan)
        shifts = plan.baby_shifts
        rotated = eng.rotate_many_by_steps(ct, [(-s) % self.n for s in shifts])
        # the baby rotations in the NTT domain, stacked [babies, 2, *batch, L, N]
        rot = torch.empty((len(rotated), *ct.data.shape), dtype=ct.data.dtype, device=ct.data.device)
        for i, r in enumerate(rotated):
            eng.forward_ntt(r.data, r.level, out=rot[i])
        del rotated
        inner_all = torch.empty((len(plan.giants), *ct.data.shape), dtype=ct.data.dtype, device=ct.data.device)
        eng.ctx.call("fhb_ckks_bsgs_inner_product", rot.data_ptr(), rot[0].numel(), pts.data_ptr(), pts[0].numel(),
                     pts.size(0), table.data_ptr(), len(plan.giants), plan.baby, inner_all.data_ptr(),
                     inner_all[0].numel(),
                     2 * ct.batch_size, ct.limb_count, ct.level, eng._stream())
        del rot
        q = float(eng.moduli[ct.level])
        result = None
        rotated, keys = [], []
        for gi, k in enumerate(plan.giants):
            inner = Ciphertext(inner_all[gi], ct.level, ct.scale * q, "ntt", "montgomery")
            inner = eng.rescale_to_next_level(eng.ntt_domain_to_coefficient_domain(inner))
            inner = eng.reinterpret_at_scale(inner, ct.scale)
            shift = plan.unit * plan.baby * k
            if shift % self.n:
                rotated.append(inner)
                keys.append(eng.rotation_key((-shift) % self.n))
            else:
                result = inner if result is None else eng.add(result, inner)
        del inner_all
        if rotated:
            # the giant-step rotations summed before a single ModDown
            summed = eng.rotate_and_sum(rotated, keys)
            result = summed if result is None else eng.add(result, summed)
        return result

    # Scales are tracked exactly inside the modular reduction: the 50-bit
    # primes differ from 2^50 by up to ~6e-6 relative, and the double-angle
    # chain amplifies any unaccounted scale error by 2^R.
    def _mul(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        eng = self.engine
        level = a.level if b is None else max(a.level, b.level)
        a = eng.mod_switch_to_level(a, level)
        an = eng.coefficient_domain_to_ntt_domain(a)
        if b is None:
            bn = an
        else:
            bn = eng.coefficient_domain_to_ntt_domain(eng.mod_switch_to_level(b, level))
        return eng.multiply_relinearize_rescale(an, bn)

    def _scaled(self, ct: Ciphertext, level: int, scale: float, value: float = 1.0) -> Ciphertext:
        """value * ct moved to `level` (> ct.level) with actual scale exactly
        `scale`: mod-switch to level-1, multiply by the integer
        round(value * scale * q_(level-1) / ct.scale), rescale."""
        eng = self.engine
        if level <= ct.level:
            raise ValueError("_scaled needs a deeper target level")
        src = eng.mod_switch_to_level(ct, level - 1)
        q = eng.moduli[level - 1]
        c = int(round(value * scale * q / ct.scale))
        out = eng.multiply_integer(src, c, scale_factor=c / value if value else 1.0)
        out = eng.rescale_to_next_level(out)
        return eng.reinterpret_at_scale(out, scale)

    # -- Chebyshev series by Paterson-Stockmeyer -------------------------------
    # p = sum_k c_k T_k is split as p = q T_g + r with T_g the largest giant
    # (g = m 2^i <= deg p, baby bound m) using T_j T_g = (T_(j+g) + T_|g-j|) / 2,
    # recursively, down to leaves of degree < m evaluated from the babies
    # T_1..T_m by scalar products.  Non-scalar products: m - 1 babies, the
    # giants, and one per inner node (15 for degree 44, m = 8, against 43 for
    # the whole basis T_1..T_44); the multiplicative depth is the same.
    @staticmethod
    def _cheb_split(c: np.ndarray, g: int) -> tuple[np.ndarray, np.ndarray]:
        deg = len(c) - 1
        q = np.zeros(deg - g + 1)
        r = c[:g].astype(np.float64).copy()
        q[0] = c[g]
        for j in range(1, deg - g + 1):
            q[j] = 2.0 * c[g + j]
            r[g - j] -= c[g + j]
        return q, r

    @staticmethod
    def _trim(c: np.ndarray) -> np.ndarray:
        scale = max(float(np.max(np.abs(c))), 1e-300)
        k = len(c)
        while k > 1 and abs(c[k - 1]) < 1e-15 * scale:
            k -= 1
        return c[:k]

    def _baby_levels(self) -> dict[int, int]:
        lv = {1: 0}
        for k in range(2, self.ps_baby + 1):
            a = 1 << (math.ceil(math.log2(k)) - 1)
            lv[k] = max(lv[a], lv[k - a]) + 1
        return lv

    def _giants(self) -> list[int]:
        g, out = self.ps_baby, []
        while g <= self.degree:
            out.append(g)
            g *= 2
        return out

    def _ps_depth(self) -> int:
        """Levels consumed by the Chebyshev evaluation (symbolic dry run of
        _ps_eval's level arithmetic)."""
        lv = self._baby_levels()
        for g in self._giants():
            if g not in lv:
                lv[g] = lv[g // 2] + 1
        return self._ps_level(self._trim(np.asarray(self.seed, dtype=np.float64)), lv)

    def _ps_level(self, c: np.ndarray, lv: dict[int, int]) -> int:
        deg = len(c) - 1
        if deg < self.ps_baby:
            used = [lv[k] for k in range(1, deg + 1) if c[k] != 0.0]
            return (max(used) if used else 0) + 1
        g = max(x for x in self._giants() if x <= deg)
        q, r = self._cheb_split(c, g)
        q, r = self._trim(q), self._trim(r)
        if len(q) == 1:
            top = lv[g] + 1
        else:
            top = max(self._ps_level(q, lv), lv[g]) + 1
        if len(r) == 1:  # a constant remainder is added to the top term
            return top
        return max(top, self._ps_level(r, lv) + 1)

    def _chebyshev(self, x: Ciphertext) -> Ciphertext:
        eng = self.engine
        T = {1: x}
        for k in range(2, self.ps_baby + 1):
            a = 1 << (math.ceil(math.log2(k)) - 1)
            b = k - a
            prod = self._mul(T[a], None if a == b else T[b])
            two = eng.add(prod, prod)
            if a == b:
                T[k] = eng.add_constant(two, -1.0)
            else:
                T[k] = eng.subtract(two, self._scaled(T[a - b], two.level, two.scale))
        for g in self._giants():
            if g not in T:
                sq = self._mul(T[g // 2], None)
                T[g] = eng.add_constant(eng.add(sq, sq), -1.0)
        out = self._ps_eval(self._trim(np.asarray(self.seed, dtype=np.float64)), T)
        target = x.level + self.cheb_depth
        if out.level < target:
            out = self._scaled(out, target, self.delta)
        return out

    def _ps_eval(self, c: np.ndarray, T: dict[int, Ciphertext]) -> Ciphertext:
        eng = self.engine
        deg = len(c) - 1
        if deg < self.ps_baby:
            used = [k for k in range(1, deg + 1) if c[k] != 0.0]
            final = max(T[k].level for k in used) + 1
            acc = None
            for k in used:
                term = self._scaled(T[k], final, self.delta, float(c[k]))
                acc = term if acc is None else eng.add(acc, term)
            return eng.add_constant(acc, float(c[0]))
        g = max(x for x in self._giants() if x <= deg)
        q, r = self._cheb_split(c, g)
        q, r = self._trim(q), self._trim(r)
        if len(q) == 1:
            top = self._scaled(T[g], T[g].level + 1, self.delta, float(q[0]))
        else:
            top = self._mul(self._ps_eval(q, T), T[g])
        if len(r) == 1:
            return eng.add_constant(top, float(r[0])) if r[0] != 0.0 else top
        low = self._ps_eval(r, T)
        level = max(top.level, low.level + 1)
        if level > top.level:
            top = self._scaled(top, level, self.delta)
        return eng.add(top, self._scaled(low, level, top.scale))

    def _eval_mod(self, x: Ciphertext) -> Ciphertext:
        eng = self.engine
        z = self._chebyshev(x)
        for _ in range(self.R):
            sq = self._mul(z, None)
            z = eng.add_constant(eng.add(sq, sq), -1.0)
        return z

    def __call__(self, ct: Ciphertext) -> Ciphertext:
        eng = self.engine
        nq = eng.num_q
        if ct.level != eng.public_level_count - 1:
            raise ValueError("bootstrap input must be at the final public level")
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        # keep the message at scale ~Delta modulo the structural base prime only
        base = eng.mod_switch_to_level(ct, nq - 1)
        base = eng.reinterpret_at_scale(base, self.delta)
        raised = eng.modulus_raise(base, self.target)
        t = self._linear(raised, "cts0", self.cts_plans[0])
        t = self._linear(t, "cts1", self.cts_plans[1])
        conj = eng.conjugate(t, self._conj)
        real = eng.add(t, conj)
        imag = eng.multiply_by_monomial(eng.subtract(t, conj), 3 * self.n)
        # both halves through one modular reduction (twice the batch per launch)
        shape = real.data.shape
        rows, n = shape[-2], shape[-1]
        flat = [h.data.reshape(2, -1, rows, n) for h in (real, imag)]
        b = flat[0].size(1)
        both = self._eval_mod(Ciphertext(torch.cat(flat, dim=1), real.level, real.scale,
                                         real.polynomial_domain, real.residue_representation))
        out_shape = (2, *shape[1:-2], both.data.size(-2), n)
        real = Ciphertext(both.data[:, :b].reshape(out_shape).contiguous(), both.level, both.scale)
        imag = Ciphertext(both.data[:, b:].reshape(out_shape).contiguous(), both.level, both.scale)
        imag = eng.multiply_by_monomial(imag, self.n)
        z = eng.add(real, eng.reinterpret_at_scale(eng.mod_switch_to_level(imag, real.level), real.scale))
        z = self._linear(z, "stc0", self.stc_plans[0])
        z = self._linear(z, "stc1", self.stc_plans[1])
        return z
