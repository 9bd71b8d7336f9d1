"""CPU checks of the bootstrap's plaintext linear algebra and reduction."""

import math

import numpy as np
import pytest

from fhelium_b200.bootstrap import (_bsgs_plan, _group, _stage, apply_diagonal_matrix, chebyshev_coefficients,
                                    chebyshev_eval)


def _bitrev(n):
    bits = n.bit_length() - 1
    return np.array([int(format(i, f"0{bits}b")[::-1], 2) for i in range(n)])


def _V(n):
    # decoding matrix for generator 5: V[j, k] = zeta^(k 5^j), zeta = exp(i pi / (2n))
    j = np.arange(n)
    e = np.array([pow(5, int(x), 4 * n) for x in j])
    k = np.arange(n)
    return np.exp(1j * np.pi * np.outer(e, k) / (2 * n))


@pytest.mark.parametrize("log_n", [3, 5, 7])
@pytest.mark.parametrize("split", [1, 2])
def test_transforms_factor_the_decoding_matrix(log_n, split):
    n = 1 << log_n
    rng = np.random.default_rng(log_n)
    z = rng.normal(size=n) + 1j * rng.normal(size=n)
    V = _V(n)
    br = _bitrev(n)
    lens = [1 << i for i in range(1, log_n + 1)]
    low, high = lens[:split], lens[split:]
    s = V @ z
    # CoeffsToSlots: bit-reversed z
    w = apply_diagonal_matrix(_group(n, low[::-1], True), apply_diagonal_matrix(_group(n, high[::-1], True), s))
    np.testing.assert_allclose(w, z[br], atol=1e-10)
    # SlotsToCoeffs: back to V z
    back = apply_diagonal_matrix(_group(n, high, False), apply_diagonal_matrix(_group(n, low, False), z[br]))
    np.testing.assert_allclose(back, V @ z, atol=1e-9)


def test_slot_packing_identity():
    # s = V z with z_k = t_k + i t_(k+n) equals the generator-5 decoding of t
    n = 16
    rng = np.random.default_rng(1)
    t = rng.normal(size=2 * n)
    z = t[:n] + 1j * t[n:]
    s = np.array([np.sum(t * np.exp(1j * np.pi * np.arange(2 * n) * pow(5, j, 4 * n) / (2 * n))) for j in range(n)])
    np.testing.assert_allclose(_V(n) @ z, s, atol=1e-10)


def test_bsgs_reassembles_the_matrix():
    n = 64
    m = _group(n, [2, 4, 8], False)
    plan = _bsgs_plan(m, n, unit=1, baby=4, signed=True)
    rng = np.random.default_rng(3)
    v = rng.normal(size=n) + 1j * rng.normal(size=n)
    out = np.zeros(n, complex)
    for k in plan.giants:
        inner = np.zeros(n, complex)
        for kk, b, pre in plan.entries:
            if kk == k:
                inner += pre * np.roll(v, -b)
        out += np.roll(inner, -plan.unit * plan.baby * k)
    np.testing.assert_allclose(out, apply_diagonal_matrix(m, v), atol=1e-10)


def test_cosine_double_angle_reduction_accuracy():
    bound, R, degree = 512.0, 7, 44
    seed = chebyshev_coefficients(lambda x: np.cos(2 * np.pi * (bound * x - 0.25) / 2 ** R), degree)
    rng = np.random.default_rng(0)
    I = rng.integers(-500, 500, size=4000)
    f = rng.uniform(-0.01, 0.01, size=4000)
    u = I + f
    z = chebyshev_eval(seed, u / bound)
    for _ in range(R):
        z = 2 * z * z - 1
    got = z / (2 * math.pi)
    assert np.max(np.abs(got - f)) < 1e-4
