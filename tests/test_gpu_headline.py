"""Parity at the benchmarked shape, bit-exact against the oracle.

Preset slots32768_scale40_levels34_int64: N = 2^16, 35 ciphertext primes
(L = 35 at level 0), 4 special primes, 10 hybrid digits (8 x 4 + 2 + 1).
Keys are the engine's own (GPU key generation), ciphertexts are the engine's
own encryptions of uniform [-0.05, 0.05] messages, and the default key-switch
work order (one destination row across groups of four ciphertexts) is used
with a batch of 5, so both its full-group and its partial-group branches run.
Every case runs with the basis conversion on the CUDA cores and on the int8
tensor cores.

Checks, as the reference checks CPU against CUDA residues
(tests/test_ckks_operation_correctness.py:256-401 of the reference):
canonical outputs integer-equal to the oracle, item by item; and the
decrypted product within the reference's multiply bound (3e-5,
tests/test_ckks_operation_correctness.py:48-51).  Where the reference's own
CPU operators were built (oracle/_ref), the first item is also compared with
the reference's operator sequence (oracle/ref_pipeline.py).
"""

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import CkksConfig, Preset
from fhelium_b200.engine import CkksEngine
from fhelium_b200.values import Ciphertext
from oracle import ref_pipeline
from tests.helpers import oracle_for, to_np

pytestmark = pytest.mark.gpu

BATCH = 5
HOISTED_STEPS = list(range(1, 17))
FORMS = ["cuda_cores", "tensor_cores"]


@pytest.fixture(scope="module")
def headline():
    cfg = CkksConfig.parse(Preset.slots32768_scale40_levels34_int64)
    eng = CkksEngine(cfg, rng_seed=2)
    assert cfg.num_q_primes == 35 and cfg.num_p_primes == 4 and eng.key_digit_count == 10
    assert eng.ctx.get_tuning(nat.TUNE_KS_ORDER) == 2
    gen = torch.Generator().manual_seed(2)
    x = torch.rand(BATCH, eng.num_slots, generator=gen, dtype=torch.float64) * 0.1 - 0.05
    y = torch.rand(BATCH, eng.num_slots, generator=gen, dtype=torch.float64) * 0.1 - 0.05
    ca = eng.encrypt_message(x)
    cb = eng.encrypt_message(y)
    assert ca.level == 0 and ca.limb_count == 35 and ca.batch_size == BATCH
    rlk = eng.relinearization_key
    eng.generate_rotation_keys(HOISTED_STEPS + [-1])
    return {"cfg": cfg, "eng": eng, "orc": oracle_for(cfg), "x": x, "y": y, "ca": ca, "cb": cb, "rlk": rlk}


@pytest.fixture(scope="module")
def hmult_oracle(headline):
    """Oracle HMult -> relinearize -> rescale of every item (NTT-domain inputs)."""
    h = headline
    eng, orc = h["eng"], h["orc"]
    a = to_np(eng.coefficient_domain_to_ntt_domain(h["ca"]).data)
    b = to_np(eng.coefficient_domain_to_ntt_domain(h["cb"]).data)
    key = to_np(h["rlk"].data)
    want = [orc.rescale(orc.relinearize(orc.multiply(a[:, i], b[:, i], 0), key, 0), 0) for i in range(BATCH)]
    return a, b, key, np.stack(want, axis=1)


@pytest.mark.parametrize("form", FORMS)
def test_headline_hmult_relin_rescale_bit_exact(headline, hmult_oracle, form):
    h = headline
    eng = h["eng"]
    eng.basis_conversion = form
    a, b, key, want = hmult_oracle
    na, nb = eng.coefficient_domain_to_ntt_domain(h["ca"]), eng.coefficient_domain_to_ntt_domain(h["cb"])
    got = eng.multiply_relinearize_rescale(na, nb, h["rlk"])
    assert got.level == 1 and got.limb_count == 34
    np.testing.assert_array_equal(to_np(got.data), want)
    # the reference engine's call order (three engine calls) gives the same residues
    sep = eng.rescale_to_next_level(eng.relinearize(eng.multiply(na, nb), h["rlk"]))
    np.testing.assert_array_equal(to_np(sep.data), want)
    # decrypted product within the reference's multiply bound
    dec = eng.decrypt_message(got).real
    err = (dec - h["x"] * h["y"]).abs().max().item()
    assert err <= 3e-5, err


def test_headline_hmult_matches_reference_operators(headline, hmult_oracle):
    if not ref_pipeline.available():
        pytest.skip("reference CPU operators were not built (oracle/build_ref.sh)")
    a, b, key, want = hmult_oracle
    pipe = ref_pipeline.ReferenceCpuPipeline(headline["orc"])
    t = lambda v: torch.from_numpy(np.ascontiguousarray(v))
    ref = pipe.multiply_relinearize_rescale(t(a[:, 0]), t(b[:, 0]), t(key), 0).numpy()
    np.testing.assert_array_equal(ref, want[:, 0])


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("step", [1, -1])
def test_headline_rotation_bit_exact(headline, step, form):
    h = headline
    eng, orc = h["eng"], h["orc"]
    eng.basis_conversion = form
    ct = h["ca"]
    got = eng.rotate_by_step(ct, step)
    key = to_np(eng.rotation_key(step).data)
    src = to_np(ct.data)
    want = np.stack([orc.rotate(src[:, i], step % eng.num_slots, key, 0) for i in range(2)], axis=1)
    np.testing.assert_array_equal(to_np(got.data)[:, :2], want)


@pytest.fixture(scope="module")
def hoisted_oracle(headline):
    h = headline
    eng, orc = h["eng"], h["orc"]
    ct = Ciphertext(h["ca"].data[:, :1].contiguous(), 0, h["ca"].scale)
    keys = {s: to_np(eng.rotation_key(s).data) for s in HOISTED_STEPS}
    return ct, orc.rotate_hoisted(to_np(ct.data)[:, 0], HOISTED_STEPS, keys, 0)


@pytest.mark.parametrize("form", FORMS)
def test_headline_hoisted_rotations_bit_exact(headline, hoisted_oracle, form):
    """Steps 1..16 sharing one ModUp, against the oracle's hoisted rotation
    (the reference's hoisting, fhelium/engine/hybrid_keyswitch.py:373-469)."""
    eng = headline["eng"]
    eng.basis_conversion = form
    ct, want = hoisted_oracle
    got = eng.rotate_many_by_steps(ct, HOISTED_STEPS)
    for s, g, w in zip(HOISTED_STEPS, got, want):
        np.testing.assert_array_equal(to_np(g.data)[:, 0], w, err_msg=f"step {s}")
