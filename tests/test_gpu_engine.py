"""End-to-end CKKS on the GPU: real keys, encrypt -> evaluate -> decrypt,
decrypted error against an FP64 plaintext model.

Bounds follow the reference's own tests
(tests/test_ckks_operation_correctness.py:48-51: arithmetic/key-switch 2e-5,
multiplication 3e-5) on slots8192_scale40_levels7_int64 with messages
uniform in [-0.05, 0.05].
"""

import numpy as np
import pytest
import torch

from fhelium_b200.config import Preset
from fhelium_b200.engine import CkksEngine

pytestmark = pytest.mark.gpu

ATOL_ADD = 2e-5
ATOL_MUL = 3e-5


@pytest.fixture(scope="module")
def engine():
    return CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=0)


def _messages(n_slots, batch, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.rand((batch, n_slots), dtype=torch.float64, generator=g) * 0.1 - 0.05


def test_encrypt_decrypt_and_add(engine):
    x = _messages(engine.num_slots, 2, 0)
    y = _messages(engine.num_slots, 2, 1)
    cx = engine.encrypt_message(x)
    cy = engine.encrypt_message(y)
    assert cx.data.shape == (2, 2, engine.num_q, engine.n)
    np.testing.assert_allclose(engine.decrypt_message(cx, is_real=True).numpy(), x.numpy(), atol=ATOL_ADD)
    s = engine.add(cx, cy)
    np.testing.assert_allclose(engine.decrypt_message(s, is_real=True).numpy(), (x + y).numpy(), atol=ATOL_ADD)


def test_multiply_relinearize_rescale(engine):
    x = _messages(engine.num_slots, 2, 2)
    y = _messages(engine.num_slots, 2, 3)
    cx = engine.coefficient_domain_to_ntt_domain(engine.encrypt_message(x))
    cy = engine.coefficient_domain_to_ntt_domain(engine.encrypt_message(y))
    prod = engine.rescale_to_next_level(engine.relinearize(engine.multiply(cx, cy)))
    assert prod.level == 1
    np.testing.assert_allclose(engine.decrypt_message(prod, is_real=True).numpy(), (x * y).numpy(), atol=ATOL_MUL)
    fused = engine.multiply_relinearize_rescale(cx, cy)
    assert torch.equal(fused.data, prod.data)
    # three-component decryption before relinearisation also works
    np.testing.assert_allclose(
        engine.decrypt_message(engine.multiply(cx, cy), is_real=True).numpy(), (x * y).numpy(), atol=ATOL_MUL)


@pytest.mark.parametrize("step", [1, -1, 8])
def test_rotation(engine, step):
    x = _messages(engine.num_slots, 1, 4)
    cx = engine.encrypt_message(x)
    r = engine.rotate_by_step(cx, step)
    np.testing.assert_allclose(engine.decrypt_message(r, is_real=True).numpy(),
                               torch.roll(x, shifts=step, dims=-1).numpy(), atol=ATOL_ADD)


def test_hoisted_rotations(engine):
    x = _messages(engine.num_slots, 1, 5)
    cx = engine.encrypt_message(x, level=2)
    steps = [1, 2, 3, 7]
    outs = engine.rotate_many_by_steps(cx, steps)
    for s, r in zip(steps, outs):
        np.testing.assert_allclose(engine.decrypt_message(r, is_real=True).numpy(),
                                   torch.roll(x, shifts=s, dims=-1).numpy(), atol=ATOL_ADD)


def test_depth_chain(engine):
    """Square repeatedly down the whole chain."""
    x = _messages(engine.num_slots, 1, 6) * 10  # [-0.5, 0.5]
    ct = engine.coefficient_domain_to_ntt_domain(engine.encrypt_message(x))
    want = x.clone()
    for _ in range(engine.public_level_count - 1):
        ct = engine.multiply_relinearize_rescale(ct, ct)
        want = want * want
        np.testing.assert_allclose(engine.decrypt_message(ct, is_real=True).numpy(), want.numpy(), atol=1e-4)
        ct = engine.coefficient_domain_to_ntt_domain(ct)
