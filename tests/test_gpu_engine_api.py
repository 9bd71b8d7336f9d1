"""The rest of fh.CkksEngine's public API on the GPU: Plaintext values
(plaintext / encode / integer_coefficients_to_rns / prepare_* / decode),
encrypt / decrypt, plaintext addition and multiplication, negate, sums,
switch_key, in-place variants, level switches and validation.

Decrypted results are checked against an FP64 model with the reference's
bounds (tests/test_ckks_operation_correctness.py:48-51: 2e-5 for additions
and key switching, 3e-5 for products) on slots8192_scale40_levels7_int64;
operations that must not change residues are checked bit for bit.
"""

import numpy as np
import pytest
import torch

from fhelium_b200.config import Preset
from fhelium_b200.engine import CkksEngine
from fhelium_b200.values import Ciphertext, Plaintext, PublicKey

pytestmark = pytest.mark.gpu

ATOL_ADD = 2e-5
ATOL_MUL = 3e-5


@pytest.fixture(scope="module")
def engine():
    return CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=3)


def _msg(engine, batch, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.rand((batch, engine.num_slots), dtype=torch.float64, generator=g) * 0.1 - 0.05


def _dec(engine, ct, sk=None):
    return engine.decode(engine.decrypt(ct, sk), is_real=True).numpy()


def test_plaintext_states_and_round_trip(engine):
    x = _msg(engine, 2, 0)
    slots = engine.plaintext(x, level=1)
    assert slots.is_slots and slots.level == 1 and slots.scale == engine.config.default_scale
    ints = engine.encode(x, level=1)
    assert ints.is_integer_coefficients and ints.data.shape == (2, engine.n)
    np.testing.assert_allclose(engine.decode(ints, is_real=True).numpy(), x.numpy(), atol=1e-9)
    rns = engine.integer_coefficients_to_rns(ints)
    assert rns.is_rns and rns.data.shape == (2, engine.num_q - 1, engine.n)
    assert rns.prime_ids == tuple(range(1, engine.num_q))
    qp = engine.integer_coefficients_to_rns(ints, modulus_basis="QP")
    assert qp.data.shape[-2] == engine.qp_rows - 1
    mont = engine.standard_residues_to_montgomery_residues(rns)
    assert mont.residue_representation == "montgomery" and rns.residue_representation == "standard"
    back = engine.montgomery_residues_to_standard_residues(mont)
    assert torch.equal(back.data, rns.data)
    ntt = engine.coefficient_domain_to_ntt_domain(rns)
    assert ntt.polynomial_domain == "ntt" and ntt.residue_representation == "montgomery"
    assert torch.equal(engine.ntt_domain_to_coefficient_domain(ntt).data, rns.data)
    mult = engine.prepare_plaintext_for_multiplication(ints)
    assert mult.polynomial_domain == "ntt"
    q = torch.tensor(engine.moduli[1: engine.num_q], dtype=torch.int64, device=engine.device)[:, None]
    assert torch.equal(mult.data.to(torch.int64) % q, ntt.data.to(torch.int64) % q)
    with pytest.raises(ValueError, match="RNS reconstruction is not implicit"):
        engine.decode(rns)


def test_encrypt_decrypt(engine):
    x = _msg(engine, 3, 1)
    ct = engine.encrypt(engine.encode(x))
    assert ct.polynomial_domain == "coefficient" and ct.data.shape == (2, 3, engine.num_q, engine.n)
    np.testing.assert_allclose(_dec(engine, ct), x.numpy(), atol=ATOL_ADD)
    ct1 = engine.encrypt(engine.plaintext(x, level=2, scale=2.0 ** 35))   # slots are encoded first
    assert ct1.level == 2 and ct1.scale == 2.0 ** 35
    np.testing.assert_allclose(_dec(engine, ct1), x.numpy(), atol=ATOL_ADD * 32)
    pt = engine.decrypt(ct)
    assert pt.is_approximate_coefficients and pt.data.dtype == torch.float64
    with pytest.raises(TypeError):
        engine.encrypt(x)


def test_plaintext_addition_and_product(engine):
    x, y = _msg(engine, 2, 2), _msg(engine, 2, 3)
    ct = engine.encrypt(engine.encode(x))
    for pt in (engine.prepare_plaintext_for_addition(engine.encode(y)), engine.encode(y), engine.plaintext(y)):
        s = engine.add_plaintext(ct, pt)
        np.testing.assert_allclose(_dec(engine, s), (x + y).numpy(), atol=ATOL_ADD)
    shared = engine.encode(y[0])                                    # one plaintext for the whole batch
    np.testing.assert_allclose(_dec(engine, engine.add_plaintext(ct, shared)), (x + y[0]).numpy(), atol=ATOL_ADD)
    c2 = ct.clone()
    assert engine.add_plaintext_(c2, engine.encode(y)) is c2
    np.testing.assert_allclose(_dec(engine, c2), (x + y).numpy(), atol=ATOL_ADD)
    with pytest.raises(ValueError, match="scale"):
        engine.add_plaintext(ct, engine.encode(y, scale=2.0 ** 30))
    cn = engine.coefficient_domain_to_ntt_domain(ct)
    pm = engine.prepare_plaintext_for_multiplication(engine.encode(y, scale=2.0 ** 30))
    prod = engine.multiply_plaintext(cn, pm)
    assert prod.scale == ct.scale * 2.0 ** 30
    np.testing.assert_allclose(_dec(engine, prod), (x * y).numpy(), atol=ATOL_MUL)
    prod_shared = engine.multiply_plaintext(cn, engine.encode(y[1], scale=2.0 ** 30))
    np.testing.assert_allclose(_dec(engine, prod_shared), (x * y[1]).numpy(), atol=ATOL_MUL)
    c3 = cn.clone()
    engine.multiply_plaintext_(c3, pm)
    assert torch.equal(c3.data, prod.data) and c3.scale == prod.scale


def test_negate_sums_and_in_place_arithmetic(engine):
    xs = [_msg(engine, 1, 10 + i) for i in range(5)]
    cts = [engine.encrypt(engine.encode(x)) for x in xs]
    np.testing.assert_allclose(_dec(engine, engine.negate(cts[0])), -xs[0].numpy(), atol=ATOL_ADD)
    c = cts[1].clone()
    engine.negate_(c)
    assert torch.equal(c.data, engine.negate(cts[1]).data)
    total = engine.sum_ciphertexts(cts)
    np.testing.assert_allclose(_dec(engine, total), sum(xs).numpy(), atol=ATOL_ADD)
    batch = Ciphertext(torch.cat([ct.data for ct in cts], dim=1), 0, cts[0].scale)
    summed = engine.sum_ciphertext_batch(batch)                      # 5 items: an odd tail
    assert summed.data.shape == (2, engine.num_q, engine.n)
    np.testing.assert_allclose(_dec(engine, summed), sum(xs)[0].numpy(), atol=ATOL_ADD)
    a = cts[2].clone()
    engine.add_(a, cts[3])
    assert torch.equal(a.data, engine.add(cts[2], cts[3]).data)
    engine.subtract_(a, cts[3])
    np.testing.assert_allclose(_dec(engine, a), xs[2].numpy(), atol=ATOL_ADD)


def test_switch_key(engine):
    x = _msg(engine, 2, 20)
    ct = engine.encrypt(engine.encode(x))
    dst = engine.create_secret_key()
    ksk = engine.create_key_switch_key(engine.secret_key, dst)
    switched = engine.switch_key(ct, ksk)
    np.testing.assert_allclose(_dec(engine, switched, dst), x.numpy(), atol=ATOL_ADD)
    assert np.abs(_dec(engine, switched) - x.numpy()).max() > 1.0      # no longer under the old key


def test_level_switches_rotations_and_zero_values(engine):
    x = _msg(engine, 2, 30)
    ct = engine.encrypt(engine.encode(x))
    down = engine.mod_switch_to_next_level(ct)
    assert down.level == 1
    np.testing.assert_allclose(_dec(engine, down), x.numpy(), atol=ATOL_ADD)
    c = ct.clone()
    engine.mod_switch_to_level_(c, 3)
    assert c.level == 3 and c.limb_count == engine.num_q - 3
    r = ct.clone()
    engine.rotate_by_step_(r, 1)
    assert torch.equal(r.data, engine.rotate_by_step(ct, 1).data)
    keys = [engine.rotation_key(s) for s in (1, 2, 5)]
    hoisted = engine.rotate_many_with_keys(ct, keys)
    direct = engine.rotate_many_with_keys(ct, keys, use_hoisting=False)
    # hoisting extends c1 before the automorphism, so it equals the hoisted
    # step path bit for bit and the direct path after decryption
    by_steps = engine.rotate_many_by_steps(ct, [1, 2, 5])
    for h, d, k, s, step in zip(hoisted, direct, keys, by_steps, (1, 2, 5)):
        assert torch.equal(h.data, s.data)
        assert torch.equal(d.data, engine.rotate_with_key(ct, k).data)
        np.testing.assert_allclose(_dec(engine, h), np.roll(x.numpy(), step, axis=-1), atol=ATOL_ADD)
    z = engine.encrypt_zero_like(ct)
    np.testing.assert_allclose(_dec(engine, engine.add(ct, z)), x.numpy(), atol=ATOL_ADD)
    zn = engine.encrypt_zero_like(engine.coefficient_domain_to_ntt_domain(ct))
    assert zn.polynomial_domain == "ntt"
    ints = engine.encode(x)
    for pt in (engine.plaintext(x), ints, engine.integer_coefficients_to_rns(ints),
               engine.prepare_plaintext_for_addition(ints), engine.prepare_plaintext_for_multiplication(ints)):
        zero = engine.zero_plaintext_like(pt)
        assert zero.representation == pt.representation
        assert zero.polynomial_domain == pt.polynomial_domain and zero.residue_representation == pt.residue_representation
    s = ct.clone()
    engine.reinterpret_at_scale_(s, ct.scale * 2)
    assert s.scale == ct.scale * 2 and torch.equal(s.data, ct.data)


def test_validation(engine):
    x = _msg(engine, 1, 40)
    ct = engine.encrypt(engine.encode(x))
    engine.validate_ciphertext(ct)
    engine.validate_public_key(engine.public_key)
    engine.validate_key_switch_key(engine.relinearization_key)
    with pytest.raises(ValueError):
        engine.validate_public_key(PublicKey(engine.public_key.data[:, 1:]))
    with pytest.raises(TypeError):
        engine.validate_key_switch_key(engine.public_key)
    pk = engine.create_public_key()
    engine.set_public_key(pk)
    assert engine.public_key is pk
    assert engine.final_public_level == engine.public_level_count - 1
    assert isinstance(engine.rng, torch.Generator)
    with pytest.raises(ValueError, match="exactly one"):
        Plaintext(message=None, level=0, scale=1.0)


@pytest.mark.parametrize("layout", ["cyclic", "contiguous", "strided_sparse"])
def test_compressed_plaintexts(engine, layout):
    """A compressed plaintext gives the same result as its dense expansion:
    bit for bit for additions, mod q for products."""
    from fhelium_b200.values import CompressedPlaintext
    x = _msg(engine, 2, 50)
    ct = engine.encrypt(engine.encode(x, level=1))
    rows = engine.num_q - 1
    g = torch.Generator(device=engine.device).manual_seed(7)
    q = torch.tensor(engine.moduli[1: engine.num_q], dtype=torch.int64, device=engine.device)
    u = 64
    compact = (torch.randint(0, 1 << 62, (rows, u), generator=g, device=engine.device) % q[:, None])
    implicit = torch.randint(0, 1 << 62, (rows,), generator=g, device=engine.device) % q
    for domain in ("coefficient", "ntt"):
        cp = CompressedPlaintext(data=compact.to(engine.dtype), ring_dimension=engine.n, compression_layout=layout,
                                 level=1, scale=ct.scale if domain == "coefficient" else 2.0 ** 20,
                                 context_id=engine.context_id, polynomial_domain=domain, modulus_basis="Q",
                                 residue_representation="montgomery", prime_ids=tuple(range(1, engine.num_q)),
                                 implicit_data=implicit.to(engine.dtype) if layout == "strided_sparse" else None)
        dense = cp.to_plaintext()
        again = CompressedPlaintext.from_plaintext(dense, unique_count=u, compression_layout=layout)
        assert torch.equal(again.data, cp.data)
        if domain == "coefficient":
            got = engine.add_plaintext(ct, cp)
            assert torch.equal(got.data, engine.add_plaintext(ct, dense).data)
        else:
            cn = engine.coefficient_domain_to_ntt_domain(ct)
            got = engine.multiply_plaintext(cn, cp)
            want = engine.multiply_plaintext(cn, dense)
            assert got.scale == want.scale == cn.scale * 2.0 ** 20
            qq = q[:, None]
            assert torch.equal(got.data.to(torch.int64) % qq, want.data.to(torch.int64) % qq)


def test_encode_rounding_is_unbiased_and_bounded(engine):
    """Stochastic rounding (the reference's SRound): every coefficient is the
    floor or the ceiling of the exact scaled value, and the mean error over
    many draws is near zero; "nearest" rounds deterministically."""
    x = _msg(engine, 1, 60)
    exact = engine.encode(x, scale=2.0 ** 20, level=0)   # one draw
    from fhelium_b200.encoding import encode_real_coefficients
    ref = encode_real_coefficients(x.to(engine.device), engine.n, engine.galois_generator) * 2.0 ** 20
    d = exact.data.to(torch.float64) - ref
    assert float(d.abs().max()) < 1.0 + 1e-6
    draws = torch.stack([engine.encode(x, scale=2.0 ** 20).data.to(torch.float64) - ref for _ in range(64)])
    assert abs(float(draws.mean())) < 0.01                 # unbiased
    assert float(draws.std()) > 0.2                         # genuinely random, not nearest
    nearest = CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=3, encode_rounding="nearest")
    a = nearest.encode(x, scale=2.0 ** 20).data
    assert torch.equal(a, nearest.encode(x, scale=2.0 ** 20).data)
    assert float((a.to(torch.float64) - ref).abs().max()) <= 0.5 + 1e-6


@pytest.mark.parametrize("level", [0, 2])
def test_decryption_error_distribution(engine, level):
    """The reference's statistical noise bound (tests/test_ckks_operation_correctness.py:135-169,
    349-397): RMS error < 6 N / scale and a 99th-percentile error below
    factor x N / scale (encrypt 12, rotate 12, rescale 1.25)."""
    unit = engine.n / engine.config.default_scale

    def check(ct, want, factor):
        err = (engine.decrypt_message(ct) - want.to(torch.complex128)).abs()
        assert torch.all(torch.isfinite(err))
        rms = float(err.square().mean().sqrt())
        p99 = float(torch.quantile(err.flatten(), 0.99))
        assert rms < 6.0 * unit, (rms, 6.0 * unit)
        assert p99 < factor * unit, (p99, factor * unit)

    x, y = _msg(engine, 2, 70 + level), _msg(engine, 2, 80 + level)
    cx = engine.encrypt_message(x, level=level)
    check(cx, x, 12.0)
    check(engine.rotate_by_step(cx, 1), torch.roll(x, 1, dims=-1), 12.0)
    cy = engine.encrypt_message(y, level=level)
    prod = engine.multiply_relinearize_rescale(engine.coefficient_domain_to_ntt_domain(cx),
                                               engine.coefficient_domain_to_ntt_domain(cy))
    check(prod, x * y, 1.25)
