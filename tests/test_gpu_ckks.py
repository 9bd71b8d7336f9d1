"""CKKS evaluation ops on the GPU against the oracle, bit-exact.

Inputs are seeded uniform residues (ciphertexts) and uniform key material:
the evaluation arithmetic is a deterministic function of its inputs, so the
CUDA path must reproduce the oracle (and through it the reference CPU
backend) exactly: canonical outputs integer-equal, lazy NTT-domain outputs
equal modulo q.
"""

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import Preset
from fhelium_b200.engine import CkksEngine
from fhelium_b200.values import Ciphertext, RelinearizationKey, RotationKey
from oracle import oracle as orc_mod
from tests.helpers import CONFIGS, canon, oracle_for, random_key, reduced_ring, to_dev, to_np, uniform_residues

pytestmark = pytest.mark.gpu

# (family, logN, level): every cluster size, truncated digits at higher levels
CASES = [
    ("int64_logn14", 14, 0),
    ("int64_logn14", 14, 3),
    ("int64_logn16", 13, 26),
    ("int64_logn16", 16, 30),
    ("int32_logn16", 12, 17),
    ("int32_logn14", 14, 9),
]


def _setup(family, log_n, level, seed):
    cfg = CONFIGS[family]()
    if log_n != cfg.logN:
        cfg = reduced_ring(cfg, log_n)
    eng = CkksEngine(cfg)
    orc = oracle_for(cfg, log_n)
    rng = np.random.default_rng(seed)
    return cfg, eng, orc, rng


@pytest.mark.parametrize("family,log_n,level", CASES)
def test_multiply_matches_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, level, 1)
    rows = orc.q_rows(level)
    a = uniform_residues(rng, cfg.moduli, rows, (2, 2), cfg.N, lazy=True)
    b = uniform_residues(rng, cfg.moduli, rows, (2, 2), cfg.N, lazy=True)
    ca = Ciphertext(to_dev(a, cfg), level, 2.0 ** 20, "ntt", "montgomery")
    cb = Ciphertext(to_dev(b, cfg), level, 2.0 ** 20, "ntt", "montgomery")
    got = to_np(eng.multiply(ca, cb).data)
    want = orc.multiply(a, b, level)
    np.testing.assert_array_equal(canon(got, cfg.moduli, rows), canon(want, cfg.moduli, rows))


@pytest.mark.parametrize("family,log_n,level", CASES)
def test_relinearize_matches_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, level, 2)
    rows = orc.q_rows(level)
    ct3 = uniform_residues(rng, cfg.moduli, rows, (3, 2), cfg.N, lazy=True)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    got = eng.relinearize(Ciphertext(to_dev(ct3, cfg), level, 1.0, "ntt", "montgomery"), rlk)
    want = np.stack([orc.relinearize(ct3[:, b], key, level) for b in range(2)], axis=1)
    np.testing.assert_array_equal(to_np(got.data), want)


@pytest.mark.parametrize("family,log_n,level", CASES[:2])
def test_keyswitch_work_orders_agree(family, log_n, level):
    """Every key-switch work order (rows of one ciphertext, one row across the
    batch, one row across groups of four) gives the same result; batch 6
    leaves a partial group for order 2."""
    cfg, eng, orc, rng = _setup(family, log_n, level, 4)
    rows = orc.q_rows(level)
    ct3 = uniform_residues(rng, cfg.moduli, rows, (3, 6), cfg.N, lazy=True)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    outs = []
    for order in (0, 1, 2):
        eng.ctx.set_tuning(nat.TUNE_KS_ORDER, order)
        got = eng.relinearize(Ciphertext(to_dev(ct3, cfg), level, 1.0, "ntt", "montgomery"), rlk)
        outs.append(to_np(got.data))
    eng.ctx.set_tuning(nat.TUNE_KS_ORDER, 0)
    np.testing.assert_array_equal(outs[0][:, 5], orc.relinearize(ct3[:, 5], key, level))
    np.testing.assert_array_equal(outs[1], outs[0])
    np.testing.assert_array_equal(outs[2], outs[0])


@pytest.mark.parametrize("ept", [0, 16])
@pytest.mark.parametrize("family,log_n,level", CASES)
def test_fused_multiply_relinearize_rescale_matches_oracle(family, log_n, level, ept):
    cfg, eng, orc, rng = _setup(family, log_n, level, 3)
    eng.ctx.set_tuning(nat.TUNE_NTT_INVERSE_EPT, ept)  # inverse-NTT variant of the fused HMult
    if level + 1 >= cfg.num_q_primes:
        pytest.skip("no rescale at the last level")
    rows = orc.q_rows(level)
    a = uniform_residues(rng, cfg.moduli, rows, (2, 1), cfg.N, lazy=True)
    b = uniform_residues(rng, cfg.moduli, rows, (2, 1), cfg.N, lazy=True)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    ca = Ciphertext(to_dev(a, cfg), level, 2.0 ** 30, "ntt", "montgomery")
    cb = Ciphertext(to_dev(b, cfg), level, 2.0 ** 30, "ntt", "montgomery")
    got = eng.multiply_relinearize_rescale(ca, cb, rlk)
    ct3 = orc.multiply(a[:, 0], b[:, 0], level)
    want = orc.rescale(orc.relinearize(ct3, key, level), level)
    np.testing.assert_array_equal(to_np(got.data)[:, 0], want)
    assert got.level == level + 1
    # same result through the three separate engine calls
    sep = eng.rescale_to_next_level(eng.relinearize(eng.multiply(ca, cb), rlk))
    np.testing.assert_array_equal(to_np(sep.data), to_np(got.data))


@pytest.mark.parametrize("family,log_n,level", CASES)
@pytest.mark.parametrize("nearest", [True, False])
def test_rescale_matches_oracle(family, log_n, level, nearest):
    cfg, eng, orc, rng = _setup(family, log_n, level, 4)
    if level + 1 >= cfg.num_q_primes:
        pytest.skip("no rescale at the last level")
    rows = orc.q_rows(level)
    ct = uniform_residues(rng, cfg.moduli, rows, (2, 3), cfg.N)
    c = Ciphertext(to_dev(ct, cfg), level, 2.0 ** 60, "coefficient", "standard")
    got = eng.rescale_to_next_level(c, rounding="nearest" if nearest else "floor")
    want = np.stack([orc.rescale(ct[:, b], level, nearest) for b in range(3)], axis=1)
    np.testing.assert_array_equal(to_np(got.data), want)


@pytest.mark.parametrize("family,log_n,level", CASES)
@pytest.mark.parametrize("step", [1, -1, 8])
def test_rotate_matches_oracle(family, log_n, level, step):
    cfg, eng, orc, rng = _setup(family, log_n, level, 5)
    rows = orc.q_rows(level)
    ct = uniform_residues(rng, cfg.moduli, rows, (2, 2), cfg.N)
    key = random_key(rng, cfg, cfg.N)
    g = eng.galois_element_for_step(step)
    rk = RotationKey(to_dev(key, cfg), rotation_step=step % eng.num_slots, galois_element=g)
    got = eng.rotate_with_key(Ciphertext(to_dev(ct, cfg), level, 1.0), rk)
    want = np.stack([orc.rotate(ct[:, b], step % eng.num_slots, key, level) for b in range(2)], axis=1)
    np.testing.assert_array_equal(to_np(got.data), want)


@pytest.mark.parametrize("family,log_n,level", CASES)
def test_mixed_step_rotation_matches_oracle(family, log_n, level):
    """fhb_ckks_rotate_multi: every batch item with its own step and key."""
    cfg, eng, orc, rng = _setup(family, log_n, level, 8)
    rows = orc.q_rows(level)
    steps = [1, -3, 8, 0x155 % eng.num_slots]
    ct = uniform_residues(rng, cfg.moduli, rows, (2, len(steps)), cfg.N)
    keys_np = [random_key(rng, cfg, cfg.N) for _ in steps]
    keys = [RotationKey(to_dev(k, cfg), rotation_step=s % eng.num_slots, galois_element=eng.galois_element_for_step(s))
            for k, s in zip(keys_np, steps)]
    got = eng.rotate_items_with_keys(Ciphertext(to_dev(ct, cfg), level, 1.0), keys)
    want = np.stack([orc.rotate(ct[:, b], s % eng.num_slots, k, level)
                     for b, (s, k) in enumerate(zip(steps, keys_np))], axis=1)
    np.testing.assert_array_equal(to_np(got.data), want)


@pytest.mark.parametrize("family,log_n,level", CASES[:4])
def test_hoisted_rotations_match_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, level, 6)
    rows = orc.q_rows(level)
    ct = uniform_residues(rng, cfg.moduli, rows, (2, 1), cfg.N)
    steps = [1, 2, 5]
    keys_np = {s: random_key(rng, cfg, cfg.N) for s in steps}
    for s in steps:
        eng.set_rotation_key(RotationKey(to_dev(keys_np[s], cfg), rotation_step=s,
                                         galois_element=eng.galois_element_for_step(s)))
    got = eng.rotate_many_by_steps(Ciphertext(to_dev(ct, cfg), level, 1.0), steps)
    want = orc.rotate_hoisted(ct[:, 0], steps, keys_np, level)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(to_np(g.data)[:, 0], w)


def test_automorphism_and_add_match_oracle():
    cfg, eng, orc, rng = _setup("int64_logn14", 14, 0, 7)
    rows = orc.q_rows(0)
    a = uniform_residues(rng, cfg.moduli, rows, (2, 1), cfg.N)
    b = uniform_residues(rng, cfg.moduli, rows, (2, 1), cfg.N)
    s = eng.add(Ciphertext(to_dev(a, cfg), 0, 1.0), Ciphertext(to_dev(b, cfg), 0, 1.0))
    np.testing.assert_array_equal(to_np(s.data)[0, 0], orc_mod.add_canonical(a[0, 0], b[0, 0],
                                                                            np.array(cfg.moduli[:cfg.num_q_primes])))
    import torch
    g = eng.galois_element_for_step(3)
    out = torch.empty_like(s.data)
    eng.ctx.call("fhb_ckks_automorphism", s.data.data_ptr(), out.data_ptr(), 2, len(rows), 0, g, eng._stream())
    want = orc.automorphism(to_np(s.data).reshape(2, len(rows), cfg.N), 3, rows)
    np.testing.assert_array_equal(to_np(out).reshape(2, len(rows), cfg.N), want)


@pytest.mark.parametrize("preset,batch,level", [(Preset.slots8192_scale40_levels7_int64, 26, 1),
                                                (Preset.slots32768_scale40_levels34_int64, 16, 20)])
@pytest.mark.parametrize("form", ["cuda_cores", "tensor_cores"])
def test_fused_hmult_overlapped_chunks_bit_identical(preset, batch, level, form):
    """fhb_ckks_multiply_relinearize cuts a batch of >= 16 into chunks whose
    element-wise stages run beside the other chunks' key-switch cores on
    their own streams: every chunk count gives the one-pass residues (uneven
    last chunk included)."""
    eng = CkksEngine(preset, rng_seed=5, basis_conversion=form)
    rng = np.random.default_rng(batch)
    msgs = [rng.uniform(-0.05, 0.05, (batch, eng.num_slots)) for _ in range(2)]
    ca, cb = (eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(m, level=level)) for m in msgs)
    got = {}
    try:
        for chunks in (1, 2, 3, 4):
            eng.ctx.set_tuning(nat.TUNE_OVERLAP_CHUNKS, chunks)
            got[chunks] = eng.multiply_relinearize_rescale(ca, cb).data.clone()
    finally:
        eng.ctx.set_tuning(nat.TUNE_OVERLAP_CHUNKS, 4)
    for chunks in (2, 3, 4):
        assert torch.equal(got[chunks], got[1]), chunks
    got = np.asarray(eng.decrypt_message(eng.multiply_relinearize_rescale(ca, cb)))
    assert float(np.abs(got - msgs[0] * msgs[1]).max()) < 3e-5


@pytest.mark.parametrize("preset,batch,level", [(Preset.slots8192_scale40_levels7_int64, 26, 1),
                                                (Preset.slots32768_scale40_levels34_int64, 16, 20)])
@pytest.mark.parametrize("form", ["cuda_cores", "tensor_cores"])
def test_rotation_overlapped_chunks_bit_identical(preset, batch, level, form):
    """fhb_ckks_rotate overlaps its chunks like the fused HMult: every chunk
    count gives the one-pass residues."""
    eng = CkksEngine(preset, rng_seed=6, basis_conversion=form)
    rng = np.random.default_rng(batch + 1)
    msg = rng.uniform(-0.05, 0.05, (batch, eng.num_slots))
    ct = eng.encrypt_message(msg, level=level)
    eng.generate_rotation_keys([3])
    got = {}
    try:
        for chunks in (1, 2, 3, 4):
            eng.ctx.set_tuning(nat.TUNE_OVERLAP_CHUNKS, chunks)
            got[chunks] = eng.rotate_by_step(ct, 3).data.clone()
    finally:
        eng.ctx.set_tuning(nat.TUNE_OVERLAP_CHUNKS, 4)
    for chunks in (2, 3, 4):
        assert torch.equal(got[chunks], got[1]), chunks
    dec = np.asarray(eng.decrypt_message(eng.rotate_by_step(ct, 3)))
    assert float(np.abs(dec - np.roll(msg, 3, axis=1)).max()) < 2e-5
