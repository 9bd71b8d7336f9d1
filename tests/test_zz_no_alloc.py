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
