"""fhb_ckks_relinearize_noalloc: relinearisation for callers that cannot
allocate device memory (they only hold their input and output buffers, e.g. a
plugin whose host framework owns all device memory through its own pool).

The entry point takes its scratch from a fixed array inside the library, so
it must give exactly what fhb_ckks_relinearize gives with a caller-provided
scratch buffer (same exact integer tolerance as every other parity test: none),
also on a second call in a row, whose stale scratch contents from the first
call must not leak into the result.  Collected last on purpose: it runs in a
fresh process or after every other test.
"""

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import CkksConfig, Preset
from tests.helpers import random_key, to_dev, uniform_residues

pytestmark = pytest.mark.gpu


def _relin_with_buffer(ctx, ct3, key, batch, level, rescale, out_limbs, n, dtype):
    lib = ctx.lib
    nbytes = int(lib.fhb_ckks_keyswitch_scratch_bytes(ctx.handle, batch, level))
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=ct3.device)
    out = torch.empty((2, batch, out_limbs, n), dtype=dtype, device=ct3.device)
    stream = torch.cuda.current_stream().cuda_stream
    nat.check(lib.fhb_ckks_relinearize(ctx.handle, ct3.data_ptr(), key.data_ptr(), out.data_ptr(),
                                       scratch.data_ptr(), nbytes, batch, level, rescale, stream),
              "fhb_ckks_relinearize")
    return out


def _relin_noalloc(ctx, ct3, key, batch, level, rescale, out_limbs, n, dtype):
    out = torch.empty((2, batch, out_limbs, n), dtype=dtype, device=ct3.device)
    stream = torch.cuda.current_stream().cuda_stream
    nat.check(ctx.lib.fhb_ckks_relinearize_noalloc(ctx.handle, ct3.data_ptr(), key.data_ptr(), out.data_ptr(),
                                                   batch, level, rescale, stream), "fhb_ckks_relinearize_noalloc")
    return out


@pytest.mark.parametrize("rescale", [0, 1])
def test_noalloc_matches_buffered_entry_point_twice(rescale):
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    dev = torch.device("cuda", 0)
    ctx = nat.NativeContext(64, cfg.logN, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, dev)
    rng = np.random.default_rng(77 + rescale)
    key = to_dev(random_key(rng, cfg, cfg.N), cfg)
    batch = 2
    for call, level in enumerate((0, 2)):  # two calls in a row, different shapes and data
        rows = list(range(level, cfg.num_q_primes))
        ct3 = to_dev(uniform_residues(rng, cfg.moduli, rows, (3, batch), cfg.N, lazy=True), cfg)
        out_limbs = len(rows) - rescale
        want = _relin_with_buffer(ctx, ct3, key, batch, level, rescale, out_limbs, cfg.N, cfg.torch_dtype)
        got = _relin_noalloc(ctx, ct3, key, batch, level, rescale, out_limbs, cfg.N, cfg.torch_dtype)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: no-alloc result differs from the buffered entry point"
    ctx.close()


def test_noalloc_rejects_batches_beyond_its_fixed_scratch():
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    dev = torch.device("cuda", 0)
    ctx = nat.NativeContext(64, cfg.logN, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, dev)
    limit = int(ctx.lib.fhb_ckks_relinearize_noalloc_max_scratch_bytes())
    per_ct = int(ctx.lib.fhb_ckks_keyswitch_scratch_bytes(ctx.handle, 1, 0))
    too_big = limit // per_ct + 1
    dummy = torch.zeros(16, dtype=torch.int64, device=dev)
    rc = ctx.lib.fhb_ckks_relinearize_noalloc(ctx.handle, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                              too_big, 0, 0, torch.cuda.current_stream().cuda_stream)
    assert rc != 0
    assert "scratch" in nat.last_error()
    ctx.close()


def test_noalloc_rejects_invalid_level_and_negative_batch():
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    dev = torch.device("cuda", 0)
    ctx = nat.NativeContext(64, cfg.logN, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, dev)
    dummy = torch.zeros(16, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for batch, level in ((1, cfg.num_q_primes), (1, -1), (-1, 0)):
        rc = ctx.lib.fhb_ckks_relinearize_noalloc(ctx.handle, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                                  batch, level, 0, stream)
        assert rc != 0
        assert "invalid batch or level" in nat.last_error()
    ctx.close()


@pytest.mark.skipif(torch.cuda.device_count() < 2, reason="needs a second visible GPU")
def test_noalloc_on_a_device_that_is_not_current():
    """The context lives on GPU 1 while GPU 0 is current: the scratch address
    is looked up on GPU 1, the result equals the buffered entry point's, and
    GPU 0 is current again afterwards."""
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    dev = torch.device("cuda", 1)
    ctx = nat.NativeContext(64, cfg.logN, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, dev)
    rng = np.random.default_rng(91)
    key = random_key(rng, cfg, cfg.N)
    rows = list(range(cfg.num_q_primes))
    ct3_np = uniform_residues(rng, cfg.moduli, rows, (3, 1), cfg.N, lazy=True)
    k = torch.from_numpy(key).to(dev)
    c = torch.from_numpy(ct3_np).to(dev)
    torch.cuda.set_device(0)
    with torch.cuda.device(1):
        want = _relin_with_buffer(ctx, c, k, 1, 0, 0, len(rows), cfg.N, cfg.torch_dtype)
        torch.cuda.synchronize()
    out = torch.empty((2, 1, len(rows), cfg.N), dtype=cfg.torch_dtype, device=dev)
    with torch.cuda.device(1):
        stream = torch.cuda.current_stream().cuda_stream
    assert torch.cuda.current_device() == 0
    nat.check(ctx.lib.fhb_ckks_relinearize_noalloc(ctx.handle, c.data_ptr(), k.data_ptr(), out.data_ptr(), 1, 0, 0,
                                                   stream), "fhb_ckks_relinearize_noalloc")
    assert torch.cuda.current_device() == 0
    torch.cuda.synchronize(1)
    assert torch.equal(out, want)
    ctx.close()
