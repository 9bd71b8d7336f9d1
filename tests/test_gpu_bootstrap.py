"""Full-slot bootstrapping on the GPU.

Bounds follow the reference's own logN=16 bootstrap test
(tests/test_ckks_bootstrap.py:482-485: max error < 7e-3, mean < 1.5e-3 for a
real linspace(-0.1, 0.1) message); the refreshed ciphertext must also
support further multiplications.
"""

import math

import pytest
import torch

from fhelium_b200.bootstrap import FullSlotBootstrap
from fhelium_b200.config import CkksConfig, Preset
from fhelium_b200.engine import CkksEngine

pytestmark = pytest.mark.gpu


def _run(cfg, message):
    eng = CkksEngine(cfg, galois_generator=5, rng_seed=3)
    bs = FullSlotBootstrap(eng)
    bs.generate_keys()
    ct = eng.encrypt_message(message, level=eng.public_level_count - 1)
    out = bs(ct)
    assert out.level == bs.output_level
    return eng, out


def test_bootstrap_small_ring_complex_slots():
    cfg = CkksConfig(logN=12, scale_bits=50, base_prime_bits=50, num_scale_primes=27, num_p_primes=4)
    g = torch.Generator().manual_seed(4)
    n = cfg.N // 2
    m = (torch.rand((2, n), dtype=torch.float64, generator=g) * 2 - 1) \
        + 1j * (torch.rand((2, n), dtype=torch.float64, generator=g) * 2 - 1)
    eng, out = _run(cfg, m)
    err = (eng.decrypt_message(out) - m).abs()
    # With scale = base prime (2^50) the coefficients of a full-range complex
    # message are ~|m|/sqrt(N) of q0, where sin(2 pi x)/(2 pi) departs from x
    # by ~x^3: about 6.8 bits at N = 2^12 (9.2e-3 max, 3.0e-3 mean), gaining
    # about one bit per doubling of N (10.1 bits at N = 2^16).  The same ring
    # with the reference test's real +-0.1 message reaches 15.9 bits.
    assert float(err.max()) < 1.5e-2 and float(err.mean()) < 4e-3
    # the refreshed ciphertext multiplies again
    sq = eng.multiply_relinearize_rescale(eng.coefficient_domain_to_ntt_domain(out),
                                          eng.coefficient_domain_to_ntt_domain(out))
    # |m| <= sqrt(2): the square's error is about 2|m| times the input's
    assert float((eng.decrypt_message(sq) - m * m).abs().max()) < 4e-2


def test_bootstrap_small_ring_reference_input():
    cfg = CkksConfig(logN=12, scale_bits=50, base_prime_bits=50, num_scale_primes=27, num_p_primes=4)
    x = torch.linspace(-0.1, 0.1, cfg.N // 2, dtype=torch.float64)
    eng, out = _run(cfg, x)
    err = (eng.decrypt_message(out, is_real=True) - x).abs()
    assert float(err.max()) < 1e-4 and float(err.mean()) < 3e-5


def test_bootstrap_reference_preset_reference_input():
    cfg = CkksConfig.parse(Preset.slots32768_scale50_levels27_int64, base_prime_bits=50)
    x = torch.linspace(-0.1, 0.1, cfg.N // 2, dtype=torch.float64)
    eng, out = _run(cfg, x)
    err = (eng.decrypt_message(out, is_real=True) - x).abs()
    assert float(err.max()) < 7e-3 and float(err.mean()) < 1.5e-3
    assert -math.log2(float(err.max())) > 8


@pytest.mark.parametrize("batch", [1, 2, 9])  # direct kernel below 8 polynomials, staged from 8
def test_bsgs_inner_product_matches_plaintext_products(batch):
    """fhb_ckks_bsgs_inner_product against the per-diagonal plaintext product
    and addition it replaces (equal modulo q)."""
    import numpy as np
    from fhelium_b200.values import Ciphertext
    cfg = CkksConfig(logN=12, scale_bits=50, base_prime_bits=50, num_scale_primes=5, num_p_primes=2)
    eng = CkksEngine(cfg, galois_generator=5, rng_seed=9)
    level, babies, giants = 1, 5, 3
    limbs = eng.num_q - level
    q = torch.tensor([eng.moduli[level + i] for i in range(limbs)], dtype=torch.int64).view(limbs, 1)
    g = torch.Generator().manual_seed(12)
    rot = torch.randint(0, 1 << 62, (babies, 2, batch, limbs, eng.n), generator=g) % (2 * q)
    pts = torch.randint(0, 1 << 62, (7, limbs, eng.n), generator=g) % q
    table = torch.tensor([[0, -1, 1, 2, -1], [3, 4, -1, -1, 5], [-1, -1, 6, -1, -1]], dtype=torch.int32)
    rot_d, pts_d, table_d = rot.cuda(), pts.cuda(), table.cuda()
    out = torch.empty((giants, 2, batch, limbs, eng.n), dtype=torch.int64, device="cuda")
    eng.ctx.call("fhb_ckks_bsgs_inner_product", rot_d.data_ptr(), rot_d[0].numel(), pts_d.data_ptr(),
                 pts_d[0].numel(), 7, table_d.data_ptr(), giants, babies, out.data_ptr(), out[0].numel(), 2 * batch,
                 limbs, level, eng._stream())
    for k in range(giants):
        want = None
        for b in range(babies):
            e = int(table[k, b])
            if e < 0:
                continue
            term = eng.multiply_plaintext(Ciphertext(rot_d[b], level, 1.0, "ntt", "montgomery"), pts_d[e], 1.0)
            want = term if want is None else eng.add(want, term)
        qd = q.cuda()
        assert torch.equal(out[k] % qd, want.data % qd)


def test_rotate_and_sum_close_to_separate_rotations():
    """One ModDown for a sum of rotations: within the number of terms of the
    separately rounded sum (exact modulo that rounding), and decrypts the same."""
    import numpy as np
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    eng = CkksEngine(cfg, rng_seed=6)
    rng = np.random.default_rng(3)
    steps = [1, 5, -7, 64]
    cts = [eng.encrypt_message(rng.uniform(-0.05, 0.05, (2, eng.num_slots)), level=1) for _ in steps]
    keys = [eng.rotation_key(s) for s in steps]
    got = eng.rotate_and_sum(cts, keys)
    want = None
    for ct, key in zip(cts, keys):
        r = eng.rotate_with_key(ct, key)
        want = r if want is None else eng.add(want, r)
    q = torch.tensor([eng.moduli[1 + i] for i in range(got.limb_count)], dtype=torch.int64,
                     device=got.data.device).view(-1, 1)
    diff = (got.data - want.data) % q
    centered = torch.where(diff > q // 2, diff - q, diff)
    # one integer k per coefficient, the same in every prime, |k| <= terms
    assert int(centered.abs().max()) <= len(steps)
    assert torch.equal(centered, centered[..., :1, :].expand_as(centered))
    assert float((eng.decrypt_message(got) - eng.decrypt_message(want)).abs().max()) < 1e-5
