"""The exact FP64 modular product of the kernels' FP64 rows (Word<double> in
fhb_arith.cuh), restated on the host: for the chain's primes below 2^42 the
quotient estimate is within one of floor(x w / q), so
r = fma(-qt, q, h) + l = x w - qt q lies in [-q, 2q) and one correction
returns [0, 2q).

Both forms are checked: `shoup` (quotient from x times the rounded
companion w / q) and `mul_qinv` (quotient from the rounded product times the
rounded 1 / q), over the operand ranges the transforms use: twiddles w < q
times butterfly inputs x < 4q, and residues times residues below 2q.  h is
numpy's correctly rounded float64 product; the fma terms are integers below
2^53 and are formed exactly with Python integers."""

import numpy as np
import pytest

from fhelium_b200.config import CkksConfig


def _narrow_primes():
    cfg = CkksConfig.parse("slots32768_scale40_levels34_int64")
    qs = [int(q) for q in cfg.q_moduli if int(q) < (1 << 42)]
    assert len(qs) >= 30
    return qs


def _operands(rng, q, x_max, count):
    x = rng.integers(0, x_max, count, dtype=np.uint64)
    w = rng.integers(0, q, count, dtype=np.uint64)
    # edges: the largest operands and values next to multiples of q
    edge_x = np.array([x_max - 1, x_max - 2, q - 1, q, q + 1, 2 * q - 1, 0, 1], dtype=np.uint64)
    edge_w = np.array([q - 1, q - 2, 1, q - 1, q // 2, q - 1, q - 1, q - 1], dtype=np.uint64)
    return np.concatenate([x, edge_x]), np.concatenate([w, edge_w])


def _check(q, x, w, qt):
    """r = x w - qt q in [-q, 2q) for every operand pair (exact integers)."""
    for xi, wi, ti in zip(x.tolist(), w.tolist(), qt.tolist()):
        r = xi * wi - int(ti) * q
        assert -q <= r < 2 * q, (q, xi, wi, ti)


@pytest.mark.parametrize("form", ["shoup", "mul_qinv"])
def test_f64_quotient_estimate(form):
    rng = np.random.default_rng(7)
    for q in _narrow_primes()[::5]:
        x_max = 4 * q  # forward butterflies feed products with inputs below 4q
        x, w = _operands(rng, q, x_max, 4000)
        xf, wf = x.astype(np.float64), w.astype(np.float64)
        assert np.all(xf == x) and np.all(wf == w)  # exact below 2^53
        if form == "shoup":
            wc = wf / np.float64(q)
            qt = np.floor(xf * wc)
        else:
            h = xf * wf
            qt = np.floor(h * (np.float64(1.0) / np.float64(q)))
        _check(q, x, w, qt)


def test_f64_residue_products():
    """mul_qinv on two residues below 2q (the key products)."""
    rng = np.random.default_rng(8)
    for q in _narrow_primes()[1::7]:
        x = rng.integers(0, 2 * q, 4000, dtype=np.uint64)
        w = rng.integers(0, 2 * q, 4000, dtype=np.uint64)
        h = x.astype(np.float64) * w.astype(np.float64)
        qt = np.floor(h * (1.0 / np.float64(q)))
        _check(q, x, w, qt)


@pytest.mark.parametrize("form", ["shoup_bal", "mul_qinv_bal"])
def test_f64_balanced_products(form):
    """The balanced forms of the FP64 transforms: signed operands up to the
    largest an inverse pass produces (|x| < 32 q) times constants below 2q,
    quotient rounded to nearest: x w - qt q in (-0.55 q, 0.55 q)."""
    rng = np.random.default_rng(9)
    for q in _narrow_primes()[2::6]:
        x = rng.integers(-32 * q + 1, 32 * q, 4000, dtype=np.int64)
        w = rng.integers(0, 2 * q, 4000, dtype=np.int64)
        x = np.concatenate([x, np.array([32 * q - 1, -32 * q + 1, 0, q, -q], dtype=np.int64)])
        w = np.concatenate([w, np.array([2 * q - 1, 2 * q - 1, q - 1, q - 1, q // 2], dtype=np.int64)])
        xf, wf = x.astype(np.float64), w.astype(np.float64)
        if form == "shoup_bal":
            qt = np.rint(xf * (wf / np.float64(q)))
        else:
            qt = np.rint((xf * wf) * (np.float64(1.0) / np.float64(q)))
        for xi, wi, ti in zip(x.tolist(), w.tolist(), qt.tolist()):
            r = xi * wi - int(ti) * q
            assert abs(r) < 0.55 * q, (q, xi, wi, ti)
