"""Exact int8 tensor-core NTT (tcgen05) against the CUDA-core NTT.

The tensor-core forward must equal the CUDA-core forward modulo q (the
CUDA-core output is lazy in [0, 2q), the tensor-core output canonical), and
the tensor-core inverse must be bit-identical to the CUDA-core inverse with
standard canonical output, on the standalone int32 workload's limbs
(N = 2^16, 36 primes of 23-28 bits)."""

import ctypes

import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import int32_ntt_primes

pytestmark = pytest.mark.gpu

N = 1 << 16


@pytest.fixture(scope="module")
def ctx():
    primes = int32_ntt_primes()
    c = nat.NativeContext(32, 16, primes, len(primes) - 1, 1, torch.device("cuda:0"))
    nat.check(c.lib.fhb_tc_ntt_prepare(c.handle), "prepare")
    yield c, primes
    c.close()


@pytest.fixture(params=[1, 0], ids=["fused", "three_pass"])
def form(request, ctx):
    """Both launch forms: the 16-point pass fused with the adjacent 64-point
    pass (two launches per direction), and three separate passes."""
    c, _ = ctx
    c.set_tuning(nat.TUNE_TC_NTT_FUSED, request.param)
    yield request.param
    c.set_tuning(nat.TUNE_TC_NTT_FUSED, 0)


def _inputs(primes, batch, rows, row_start, seed):
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed)
    q = torch.tensor(primes[row_start:row_start + rows], dtype=torch.int64, device="cuda:0").view(1, rows, 1)
    x = torch.randint(0, 1 << 62, (batch, rows, N), generator=g, device="cuda:0", dtype=torch.int64) % q
    return x.to(torch.int32), q


def _run(c, fn, src, dst, batch, rows, row_start):
    s = torch.cuda.current_stream().cuda_stream
    nat.check(getattr(c.lib, fn)(c.handle, src.data_ptr(), dst.data_ptr(), batch, rows, row_start, s), fn)


def _status(c):
    flag = ctypes.c_int(-1)
    nat.check(c.lib.fhb_tc_ntt_status(c.handle, ctypes.byref(flag)), "status")
    return flag.value


def _plain(c, x, batch, rows, row_start):
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(c.lib.fhb_forward_ntt(c.handle, x.data_ptr(), y.data_ptr(), batch, rows, row_start, 0, s), "ntt")
    nat.check(c.lib.fhb_inverse_ntt(c.handle, y.data_ptr(), z.data_ptr(), batch, rows, row_start, 2, s), "intt")
    return y, z


@pytest.mark.parametrize("batch,rows,row_start", [(2, 36, 0), (3, 5, 3), (1, 1, 35)])
def test_tensor_core_ntt_matches_cuda_core(ctx, form, batch, rows, row_start):
    c, primes = ctx
    x, q = _inputs(primes, batch, rows, row_start, seed=1 + row_start)
    y_plain, z_plain = _plain(c, x, batch, rows, row_start)
    assert torch.equal(z_plain, x)
    y = torch.empty_like(x)
    _run(c, "fhb_tc_forward_ntt", x, y, batch, rows, row_start)
    y64 = y.to(torch.int64)
    assert bool((y64 >= 0).all()) and bool((y64 < q).all())
    assert torch.equal(y64, y_plain.to(torch.int64) % q)
    z = torch.empty_like(x)
    _run(c, "fhb_tc_inverse_ntt", y, z, batch, rows, row_start)
    assert torch.equal(z, x)
    # the CUDA-core forward's lazy output inverts bit-identically too
    _run(c, "fhb_tc_inverse_ntt", y_plain, z, batch, rows, row_start)
    assert torch.equal(z, z_plain)
    assert _status(c) == 0


def test_tensor_core_ntt_in_place_and_empty(ctx, form):
    c, primes = ctx
    x, _ = _inputs(primes, 2, 36, 0, seed=5)
    y = torch.empty_like(x)
    _run(c, "fhb_tc_forward_ntt", x, y, 2, 36, 0)
    buf = x.clone()
    _run(c, "fhb_tc_forward_ntt", buf, buf, 2, 36, 0)
    assert torch.equal(buf, y)
    _run(c, "fhb_tc_inverse_ntt", buf, buf, 2, 36, 0)
    assert torch.equal(buf, x)
    _run(c, "fhb_tc_forward_ntt", x, y, 0, 36, 0)  # empty batch: no launch
    assert _status(c) == 0


def test_tensor_core_ntt_full_workload_round_trip(ctx, form):
    """Batch 64 x 36 limbs: round trip exact and forward equal mod q to the
    CUDA-core form over the whole tensor."""
    c, primes = ctx
    x, q = _inputs(primes, 64, 36, 0, seed=1)
    y_plain, _ = _plain(c, x, 64, 36, 0)
    y = torch.empty_like(x)
    _run(c, "fhb_tc_forward_ntt", x, y, 64, 36, 0)
    assert torch.equal(y.to(torch.int64), y_plain.to(torch.int64) % q)
    z = torch.empty_like(x)
    _run(c, "fhb_tc_inverse_ntt", y, z, 64, 36, 0)
    assert torch.equal(z, x)
    assert _status(c) == 0


def test_tensor_core_ntt_rejects_other_contexts():
    from fhelium_b200.config import prime_catalog
    n = 1 << 16
    qs = list(prime_catalog()["scale"][(40, n)])[:2]
    c = nat.NativeContext(64, 16, qs, 1, 1, torch.device("cuda:0"))
    try:
        x = torch.zeros((1, 1, n), dtype=torch.int64, device="cuda:0")
        s = torch.cuda.current_stream().cuda_stream
        assert c.lib.fhb_tc_forward_ntt(c.handle, x.data_ptr(), x.data_ptr(), 1, 1, 0, s) == -7
    finally:
        c.close()
