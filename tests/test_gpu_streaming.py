"""Host-resident batches streamed through the GPU: identical to the device call."""

import numpy as np
import pytest
import torch

from fhelium_b200.config import Preset
from fhelium_b200.engine import CkksEngine
from fhelium_b200.streaming import multiply_relinearize_rescale_host, tapered
from fhelium_b200.values import Ciphertext

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chunks", [1, 3, 7])
def test_streamed_equals_device_call(chunks):
    eng = CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=4)
    rng = np.random.default_rng(2)
    x, y = (rng.uniform(-0.05, 0.05, (7, eng.num_slots)) for _ in range(2))
    a = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(x))
    b = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(y))
    want = eng.multiply_relinearize_rescale(a, b)
    ha = Ciphertext(a.data.cpu().pin_memory(), a.level, a.scale, "ntt", "montgomery")
    hb = Ciphertext(b.data.cpu().pin_memory(), b.level, b.scale, "ntt", "montgomery")
    got = multiply_relinearize_rescale_host(eng, ha, hb, chunks=chunks)
    torch.cuda.synchronize()
    assert got.data.device.type == "cpu"
    assert (got.level, got.scale) == (want.level, want.scale)
    assert torch.equal(got.data, want.data.cpu())


def test_back_to_back_calls_share_the_staging_ring():
    """Consecutive calls reuse the engine's staging slots; a call's copies
    may start under the previous call's tail.  Every result stays exact, for
    tapered schedules and a two-slot ring too."""
    eng = CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=6)
    rng = np.random.default_rng(3)
    pairs = []
    for _ in range(3):
        x, y = (rng.uniform(-0.05, 0.05, (9, eng.num_slots)) for _ in range(2))
        a = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(x))
        b = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(y))
        pairs.append((a, b, eng.multiply_relinearize_rescale(a, b).data.cpu()))
    host = [(Ciphertext(a.data.cpu().pin_memory(), a.level, a.scale, "ntt", "montgomery"),
             Ciphertext(b.data.cpu().pin_memory(), b.level, b.scale, "ntt", "montgomery")) for a, b, _ in pairs]
    for chunks, buffers in ((tapered(9, 2, 3), 3), (4, 2), ([1] * 9, 3)):
        outs = [torch.empty_like(w).pin_memory() for _, _, w in pairs]
        for (ha, hb), o in zip(host, outs):
            multiply_relinearize_rescale_host(eng, ha, hb, chunks=chunks, out=o, buffers=buffers)
        torch.cuda.synchronize()
        for o, (_, _, want) in zip(outs, pairs):
            assert torch.equal(o, want), (chunks, buffers)
