"""FP64 canonical embedding (CKKS encode/decode) on the GPU.

Slot convention of the reference (fhelium/engine/slot_embedding.py,
fhelium/engine/galois.py): with zeta = exp(i pi / N), slot j of a real
polynomial a is
    generator 3:  a(zeta^(3^(-j) mod 2N))
    generator 5:  a(zeta^(5^j mod 2N))
so that the Galois element of a rotation by `step` (3^step, resp. 5^-step)
implements torch.roll(slots, shifts=step).  Decoding divides by the value's
scale.  The evaluations a(zeta^(2n+1)), n < N, are one length-N FFT of
a_k zeta^k; encoding inverts it.  FP64 is used only here, where rounding
Delta-scaled values to integers needs it.
"""

from __future__ import annotations

import math
from functools import lru_cache

import torch


@lru_cache(maxsize=32)
def slot_positions(n: int, generator: int) -> tuple[int, ...]:
    """Index n_j with zeta^(2 n_j + 1) the evaluation point of slot j."""
    m = 2 * n
    out = []
    for j in range(n // 2):
        e = pow(generator, (-j) % n, m) if generator == 3 else pow(generator, j, m)
        out.append((e - 1) // 2)
    return tuple(out)


@lru_cache(maxsize=32)
def _tables(n: int, generator: int, device: str):
    pos = torch.tensor(slot_positions(n, generator), dtype=torch.long, device=device)
    conj = (n - 1) - pos  # zeta^(2N - e) is the conjugate point
    k = torch.arange(n, dtype=torch.float64, device=device)
    twist = torch.polar(torch.ones_like(k), math.pi * k / n)
    untwist = torch.polar(torch.ones_like(k), -math.pi * k / n)
    return pos, conj, twist, untwist


def encode_real_coefficients(slots: torch.Tensor, n: int, generator: int) -> torch.Tensor:
    """[*batch, <= N/2] complex/real slots -> [*batch, N] float64 coefficients."""
    slots = slots.to(torch.complex128)
    if slots.size(-1) < n // 2:
        slots = torch.nn.functional.pad(slots, (0, n // 2 - slots.size(-1)))
    pos, conj, _, untwist = _tables(n, generator, str(slots.device))
    z = torch.zeros((*slots.shape[:-1], n), dtype=torch.complex128, device=slots.device)
    z[..., pos] = slots
    z[..., conj] = slots.conj()
    return (torch.fft.fft(z, norm="forward") * untwist).real


def decode_coefficients(coeffs: torch.Tensor, n: int, generator: int) -> torch.Tensor:
    """[*batch, N] real coefficients -> [*batch, N/2] complex slots (unscaled)."""
    pos, _, twist, _ = _tables(n, generator, str(coeffs.device))
    z = torch.fft.ifft(coeffs.to(torch.float64) * twist, norm="forward")
    return z[..., pos]
