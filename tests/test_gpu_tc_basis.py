"""Exact int8 tensor-core basis conversion (int64 chains) on the GPU.

1. fhb_tc_basis_extend against the oracle's restatement of the reference's
   mixed-radix basis extension (fhelium/engine/hybrid_keyswitch.py:95-237,
   csrc/ops/rns/cuda/mixed_radix_cuda.cu:146-182): equal modulo every
   destination prime, for digits of 1, 2, 4 and 6 primes (one and two
   K-steps of the MMA) and truncated digits at higher levels.
2. Every key-switch path with basis_conversion="tensor_cores" gives results
   integer-equal to the CUDA-core form and to the oracle: relinearisation,
   fused HMult + relinearise + rescale, rotation, mixed-step rotation and
   hoisted rotation.
"""

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import CkksConfig, Preset
from fhelium_b200.engine import CkksEngine
from fhelium_b200.values import Ciphertext, RelinearizationKey, RotationKey
from tests.helpers import CONFIGS, oracle_for, random_key, reduced_ring, to_dev, to_np, uniform_residues

pytestmark = pytest.mark.gpu

CONFIGS = dict(CONFIGS)
CONFIGS["int64_logn17"] = lambda: CkksConfig.parse(Preset.slots65536_scale40_levels72_int64)  # P = 6

# (family, logN, level): digits of 1 (logN 14 chain), 4 and 2/1 (logN 16
# chain at levels 0 and 30), 6 primes (logN 17 chain, two K-steps)
EXT_CASES = [
    ("int64_logn14", 12, 0),
    ("int64_logn14", 13, 3),
    ("int64_logn16", 12, 0),
    ("int64_logn16", 12, 30),
    ("int64_logn16", 14, 7),
    ("int64_logn17", 12, 0),
    ("int64_logn17", 12, 65),
]


def _setup(family, log_n, seed):
    cfg = CONFIGS[family]()
    if log_n != cfg.logN:
        cfg = reduced_ring(cfg, log_n)
    eng = CkksEngine(cfg, basis_conversion="cuda_cores")  # each test switches forms itself
    return cfg, eng, oracle_for(cfg, log_n), np.random.default_rng(seed)


@pytest.mark.parametrize("family,log_n,level", EXT_CASES)
def test_tc_extension_matches_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, 11)
    rows = orc.q_rows(level)
    batch = 3
    comp = uniform_residues(rng, cfg.moduli, rows, (batch,), cfg.N)
    comp_d = to_dev(comp, cfg)
    digits = torch.empty_like(comp_d)
    eng.ctx.call("fhb_ckks_modup_digits", comp_d.data_ptr(), digits.data_ptr(), batch, level, 1, eng._stream())
    words = int(eng.ctx.lib.fhb_tc_basis_extend_words(eng.ctx.handle, batch, level))
    ext = torch.empty(words, dtype=torch.int64, device=comp_d.device)
    eng.ctx.call("fhb_tc_basis_extend", digits.data_ptr(), ext.data_ptr(), batch, level, eng._stream())
    flag = nat.ctypes.c_int(-1)
    nat.check(eng.ctx.lib.fhb_tc_basis_status(eng.ctx.handle, nat.ctypes.byref(flag)), "fhb_tc_basis_status")
    assert flag.value == 0
    qp = orc.qp_rows(level)
    got = to_np(ext).reshape(-1, batch, len(qp), cfg.N)
    layout = orc.digits_at_level(level)
    assert got.shape[0] == len(layout)
    p = np.array([cfg.moduli[i] for i in qp], dtype=object)[:, None]
    r_mod = np.array([(1 << orc.radix_bits) % int(q) for q in p[:, 0]], dtype=object)[:, None]
    bound = 2 * np.array([cfg.moduli[i] for i in qp], dtype=np.int64)[:, None]
    for a, (_, ids) in enumerate(layout):
        want = orc.extend_digit(comp, level, ids)  # Montgomery form: ext R mod p
        assert (got[a] < bound).all() and (got[a] >= 0).all()
        for b in range(batch):
            mont = (got[a, b].astype(object) * r_mod) % p
            np.testing.assert_array_equal(mont.astype(np.int64), np.mod(want[b], bound // 2))


@pytest.mark.parametrize("family,log_n,level", [("int64_logn14", 14, 0), ("int64_logn16", 13, 26),
                                                ("int64_logn16", 16, 30), ("int64_logn17", 12, 60)])
def test_tc_form_relinearize_and_hmult_match_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, 21)
    rows = orc.q_rows(level)
    ct3 = uniform_residues(rng, cfg.moduli, rows, (3, 5), cfg.N, lazy=True)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    x = Ciphertext(to_dev(ct3, cfg), level, 1.0, "ntt", "montgomery")
    plain = to_np(eng.relinearize(x, rlk).data)
    eng.basis_conversion = "tensor_cores"
    assert eng.basis_conversion == "tensor_cores"
    tc = to_np(eng.relinearize(x, rlk).data)
    np.testing.assert_array_equal(tc, plain)
    np.testing.assert_array_equal(tc[:, 4], orc.relinearize(ct3[:, 4], key, level))
    if level + 1 < cfg.num_q_primes:
        a = uniform_residues(rng, cfg.moduli, rows, (2, 5), cfg.N, lazy=True)
        b = uniform_residues(rng, cfg.moduli, rows, (2, 5), cfg.N, lazy=True)
        ca = Ciphertext(to_dev(a, cfg), level, 2.0 ** 30, "ntt", "montgomery")
        cb = Ciphertext(to_dev(b, cfg), level, 2.0 ** 30, "ntt", "montgomery")
        got_tc = to_np(eng.multiply_relinearize_rescale(ca, cb, rlk).data)
        eng.basis_conversion = "cuda_cores"
        got_plain = to_np(eng.multiply_relinearize_rescale(ca, cb, rlk).data)
        np.testing.assert_array_equal(got_tc, got_plain)
        want = orc.rescale(orc.relinearize(orc.multiply(a[:, 0], b[:, 0], level), key, level), level)
        np.testing.assert_array_equal(got_tc[:, 0], want)


@pytest.mark.parametrize("family,log_n,level", [("int64_logn14", 14, 0), ("int64_logn16", 16, 30),
                                                ("int64_logn17", 12, 60)])
def test_tc_form_rotations_match_oracle(family, log_n, level):
    cfg, eng, orc, rng = _setup(family, log_n, 22)
    rows = orc.q_rows(level)
    ct = uniform_residues(rng, cfg.moduli, rows, (2, 3), cfg.N)
    steps = [1, -3, 8]
    keys_np = {s: random_key(rng, cfg, cfg.N) for s in steps}
    keys = {s: RotationKey(to_dev(keys_np[s], cfg), rotation_step=s % eng.num_slots,
                           galois_element=eng.galois_element_for_step(s)) for s in steps}
    for s in steps:
        eng.set_rotation_key(keys[s])
    c = Ciphertext(to_dev(ct, cfg), level, 1.0)
    one = Ciphertext(to_dev(ct[:, :1], cfg), level, 1.0)
    outs = {}
    for form in ("cuda_cores", "tensor_cores"):
        eng.basis_conversion = form
        outs[form] = (to_np(eng.rotate_with_key(c, keys[1]).data),
                      to_np(eng.rotate_items_with_keys(c, [keys[s] for s in steps]).data),
                      [to_np(r.data) for r in eng.rotate_many_by_steps(one, steps)])
    p, t = outs["cuda_cores"], outs["tensor_cores"]
    np.testing.assert_array_equal(t[0], p[0])
    np.testing.assert_array_equal(t[1], p[1])
    for x, y in zip(t[2], p[2]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(t[0][:, 2], orc.rotate(ct[:, 2], 1, keys_np[1], level))
    np.testing.assert_array_equal(t[1][:, 1], orc.rotate(ct[:, 1], -3 % eng.num_slots, keys_np[-3], level))
    want = orc.rotate_hoisted(ct[:, 0], [s % eng.num_slots for s in steps],
                              {s % eng.num_slots: keys_np[s] for s in steps}, level)
    for x, w in zip(t[2], want):
        np.testing.assert_array_equal(x[:, 0], w)


def test_tc_form_rejected_on_int32_chains():
    cfg = CONFIGS["int32_logn14"]()
    eng = CkksEngine(cfg)
    with pytest.raises(nat.NativeCallError, match="int64"):
        eng.basis_conversion = "tensor_cores"
    assert eng.basis_conversion == "cuda_cores"


@pytest.mark.parametrize("family,log_n,level", [("int64_logn14", 14, 1), ("int64_logn16", 13, 20)])
def test_tc_form_rotate_and_sum_matches_cuda_core_form(family, log_n, level):
    """The giant-step sum of bootstrapping (one ModDown for a sum of key
    switches, fhb_ckks_keyswitch_sum[_extended]) is integer-equal in both forms."""
    cfg, eng, orc, rng = _setup(family, log_n, 23)
    rows = orc.q_rows(level)
    steps = [1, 5, -7, 64]
    cts = [Ciphertext(to_dev(uniform_residues(rng, cfg.moduli, rows, (2, 2), cfg.N), cfg), level, 1.0)
           for _ in steps]
    keys = [RotationKey(to_dev(random_key(rng, cfg, cfg.N), cfg), rotation_step=s % eng.num_slots,
                        galois_element=eng.galois_element_for_step(s)) for s in steps]
    outs = {}
    for form in ("cuda_cores", "tensor_cores"):
        eng.basis_conversion = form
        outs[form] = to_np(eng.rotate_and_sum(cts, keys).data)
    np.testing.assert_array_equal(outs["tensor_cores"], outs["cuda_cores"])


@pytest.mark.parametrize("tc_moddown", [0, 1])
@pytest.mark.parametrize("batch", [9, 16])
def test_tc_form_full_ring_batches_and_moddown_variants(batch, tc_moddown):
    """The tensor-core form on the full N = 2^16 ring with batches of 9 and 16
    (both work-order-2 group branches), with ModDown on the CUDA cores or the
    tensor cores: every output equals the CUDA-core form's, and one item
    equals the oracle."""
    cfg, eng, orc, rng = _setup("int64_logn16", 16, 24)
    level = 30
    rows = orc.q_rows(level)
    ct3 = uniform_residues(rng, cfg.moduli, rows, (3, batch), cfg.N, lazy=True)
    a = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N, lazy=True)
    b = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N, lazy=True)
    ct = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    steps = [1 + (i % 5) for i in range(batch)]
    rkeys = {s: RotationKey(to_dev(random_key(rng, cfg, cfg.N), cfg), rotation_step=s,
                            galois_element=eng.galois_element_for_step(s)) for s in sorted(set(steps))}
    x3 = Ciphertext(to_dev(ct3, cfg), level, 1.0, "ntt", "montgomery")
    ca = Ciphertext(to_dev(a, cfg), level, 2.0 ** 30, "ntt", "montgomery")
    cb = Ciphertext(to_dev(b, cfg), level, 2.0 ** 30, "ntt", "montgomery")
    c = Ciphertext(to_dev(ct, cfg), level, 1.0)

    def run():
        return (to_np(eng.relinearize(x3, rlk).data), to_np(eng.multiply_relinearize_rescale(ca, cb, rlk).data),
                to_np(eng.rotate_with_key(c, rkeys[1]).data),
                to_np(eng.rotate_items_with_keys(c, [rkeys[s] for s in steps]).data))

    plain = run()
    eng.basis_conversion = "tensor_cores"
    eng.ctx.set_tuning(nat.TUNE_TC_MODDOWN, tc_moddown)
    tc = run()
    for x, y in zip(tc, plain):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(tc[0][:, batch - 1], orc.relinearize(ct3[:, batch - 1], key, level))


@pytest.mark.parametrize("form", ["tensor_cores", "cuda_cores"])
@pytest.mark.parametrize("family,log_n,level,batch", [("int64_logn14", 14, 0, 3), ("int64_logn16", 16, 0, 5),
                                                      ("int64_logn16", 16, 30, 2), ("int64_logn16", 13, 12, 6)])
def test_f64_core_matches_integer_core(family, log_n, level, batch, form):
    """The key-switch core with the Q rows of primes below 2^42 in exact FP64
    arithmetic (the default), in both basis-conversion forms (the CUDA-core
    form computes the extensions in FP64 too, splitting the words of digits
    that hold the wide base prime), against the same core on the integer
    pipe: relinearisation, fused HMult, rotation, mixed-step rotation
    (per-item keys) and hoisted rotations integer-equal, and against the
    oracle."""
    cfg, eng, orc, rng = _setup(family, log_n, 31)
    eng.basis_conversion = form
    assert eng.ctx.get_tuning(nat.TUNE_F64_CORE) == 1
    rows = orc.q_rows(level)
    key = random_key(rng, cfg, cfg.N)
    rlk = RelinearizationKey(to_dev(key, cfg))
    ct3 = uniform_residues(rng, cfg.moduli, rows, (3, batch), cfg.N, lazy=True)
    x = Ciphertext(to_dev(ct3, cfg), level, 1.0, "ntt", "montgomery")
    ct = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N)
    c = Ciphertext(to_dev(ct, cfg), level, 1.0)
    keys = [RotationKey(to_dev(random_key(rng, cfg, cfg.N), cfg), rotation_step=s,
                        galois_element=eng.galois_element_for_step(s)) for s in range(1, batch + 1)]
    outs = {}
    for f64 in (1, 0):
        eng.ctx.set_tuning(nat.TUNE_F64_CORE, f64)
        res = [to_np(eng.relinearize(x, rlk).data), to_np(eng.rotate_with_key(c, keys[0]).data),
               to_np(eng.rotate_items_with_keys(c, keys).data)]
        # hoisted: the prepared digits and every per-step key switch
        res += [to_np(r.data) for r in eng.rotate_many_with_keys(c, keys[:3])]
        outs[f64] = res
    eng.ctx.set_tuning(nat.TUNE_F64_CORE, 1)
    for got, want in zip(outs[1], outs[0]):
        np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(outs[1][0][:, batch - 1], orc.relinearize(ct3[:, batch - 1], key, level))
    if level + 1 < cfg.num_q_primes:
        a = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N, lazy=True)
        b = uniform_residues(rng, cfg.moduli, rows, (2, batch), cfg.N, lazy=True)
        ca = Ciphertext(to_dev(a, cfg), level, 2.0 ** 30, "ntt", "montgomery")
        cb = Ciphertext(to_dev(b, cfg), level, 2.0 ** 30, "ntt", "montgomery")
        got = to_np(eng.multiply_relinearize_rescale(ca, cb, rlk).data)
        eng.ctx.set_tuning(nat.TUNE_F64_CORE, 0)
        want = to_np(eng.multiply_relinearize_rescale(ca, cb, rlk).data)
        eng.ctx.set_tuning(nat.TUNE_F64_CORE, 1)
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(got[:, 0], orc.rescale(orc.relinearize(orc.multiply(a[:, 0], b[:, 0], level),
                                                                             key, level), level))


def test_f64_core_unavailable_for_wide_primes():
    """50-bit Q primes: no FP64 tables, the switch reads back 0, results unchanged."""
    eng = CkksEngine(Preset.slots8192_scale50_levels5_int64)
    eng.basis_conversion = "tensor_cores"
    assert eng.ctx.get_tuning(nat.TUNE_F64_CORE) == 0
    rng = np.random.default_rng(4)
    a, b = (eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(rng.uniform(-0.05, 0.05, eng.num_slots)))
            for _ in range(2))
    got = eng.multiply_relinearize_rescale(a, b)
    eng.basis_conversion = "cuda_cores"
    assert torch.equal(got.data, eng.multiply_relinearize_rescale(a, b).data)
