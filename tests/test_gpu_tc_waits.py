"""The tensor-core kernels' bounded waits run out, are reported, and leave the
context usable.

Every mbarrier wait of the tcgen05 kernels (the int32 NTT and the int64
basis conversion) gives up after a time limit, raises the CTA's abort flag,
and sets a device status flag; the CTA then drains its own bulk copies and
MMAs (with the default limit) and frees its tensor memory.  No test can make
a copy or an MMA never complete without faulting the GPU, so the test mode
FHB_TUNE_TC_TEST_STALL makes every launch first wait on a barrier that
nothing completes, under a short pipeline limit (FHB_TUNE_TC_WAIT_US).  The
checks: the call returns, the CUDA context has no error, the status flag
reports the timeout (and clears), and the next call with the default limit
is exact, which also shows that tensor memory was released (a leak would
leave the next launch's allocation unsatisfied).
"""

import ctypes

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.config import CkksConfig, Preset, int32_ntt_primes
from tests.helpers import oracle_for, to_dev, to_np, uniform_residues

pytestmark = pytest.mark.gpu

N16 = 1 << 16
SHORT_US = 2000  # pipeline limit of the stalled launches


def _status(ctx, fn):
    flag = ctypes.c_int(-1)
    nat.check(getattr(ctx.lib, fn)(ctx.handle, ctypes.byref(flag)), fn)
    return flag.value


def _stalled(ctx, on: bool):
    ctx.set_tuning(nat.TUNE_TC_WAIT_US, SHORT_US if on else 0)
    ctx.set_tuning(nat.TUNE_TC_TEST_STALL, 1 if on else 0)


def test_tc_ntt_wait_runs_out_then_next_call_is_exact():
    primes = int32_ntt_primes()
    ctx = nat.NativeContext(32, 16, primes, len(primes) - 1, 1, torch.device("cuda:0"))
    nat.check(ctx.lib.fhb_tc_ntt_prepare(ctx.handle), "prepare")
    s = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda:0").manual_seed(5)
    q = torch.tensor(primes[:1], dtype=torch.int64, device="cuda:0").view(1, 1, 1)
    x = (torch.randint(0, 1 << 62, (1, 1, N16), generator=g, device="cuda:0", dtype=torch.int64) % q).to(torch.int32)
    y = torch.empty_like(x)
    assert _status(ctx, "fhb_tc_ntt_status") == 0
    _stalled(ctx, True)
    for fused in (1, 0):  # the fused-pass kernel and the separate passes
        ctx.set_tuning(nat.TUNE_TC_NTT_FUSED, fused)
        for fn in ("fhb_tc_forward_ntt", "fhb_tc_inverse_ntt"):
            nat.check(getattr(ctx.lib, fn)(ctx.handle, x.data_ptr(), y.data_ptr(), 1, 1, 0, s), "stalled " + fn)
            torch.cuda.synchronize()  # no CUDA error: the kernels returned
            assert _status(ctx, "fhb_tc_ntt_status") == 1
            assert _status(ctx, "fhb_tc_ntt_status") == 0  # read clears it
    ctx.set_tuning(nat.TUNE_TC_NTT_FUSED, 0)
    _stalled(ctx, False)
    nat.check(ctx.lib.fhb_tc_forward_ntt(ctx.handle, x.data_ptr(), y.data_ptr(), 1, 1, 0, s), "forward")
    plain = torch.empty_like(x)
    nat.check(ctx.lib.fhb_forward_ntt(ctx.handle, x.data_ptr(), plain.data_ptr(), 1, 1, 0, 0, s), "plain")
    torch.cuda.synchronize()
    assert _status(ctx, "fhb_tc_ntt_status") == 0
    assert torch.equal(y.to(torch.int64) % q, plain.to(torch.int64) % q)
    ctx.close()


def test_tc_basis_wait_runs_out_then_next_call_is_exact():
    cfg = CkksConfig.parse(Preset.slots8192_scale40_levels7_int64)
    orc = oracle_for(cfg)
    ctx = nat.NativeContext(64, cfg.logN, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, torch.device("cuda:0"))
    ctx.set_tuning(nat.TUNE_BASIS_CONVERSION, 1)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(8)
    level, batch = 0, 1
    rows = orc.q_rows(level)
    comp = uniform_residues(rng, cfg.moduli, rows, (batch,), cfg.N)
    comp_d = to_dev(comp, cfg)
    digits = torch.empty_like(comp_d)
    nat.check(ctx.lib.fhb_ckks_modup_digits(ctx.handle, comp_d.data_ptr(), digits.data_ptr(), batch, level, 1, s),
              "modup")
    words = int(ctx.lib.fhb_tc_basis_extend_words(ctx.handle, batch, level))
    ext = torch.zeros(words, dtype=torch.int64, device="cuda:0")
    _stalled(ctx, True)
    nat.check(ctx.lib.fhb_tc_basis_extend(ctx.handle, digits.data_ptr(), ext.data_ptr(), batch, level, s), "stalled")
    torch.cuda.synchronize()
    assert _status(ctx, "fhb_tc_basis_status") == 1
    assert _status(ctx, "fhb_tc_basis_status") == 0
    _stalled(ctx, False)
    nat.check(ctx.lib.fhb_tc_basis_extend(ctx.handle, digits.data_ptr(), ext.data_ptr(), batch, level, s), "extend")
    torch.cuda.synchronize()
    assert _status(ctx, "fhb_tc_basis_status") == 0
    qp = orc.qp_rows(level)
    got = to_np(ext).reshape(-1, batch, len(qp), cfg.N)
    p = np.array([cfg.moduli[i] for i in qp], dtype=object)[:, None]
    r_mod = np.array([(1 << orc.radix_bits) % int(v) for v in p[:, 0]], dtype=object)[:, None]
    for a, (_, ids) in enumerate(orc.digits_at_level(level)):
        want = orc.extend_digit(comp, level, ids)
        mont = (got[a, 0].astype(object) * r_mod) % p
        np.testing.assert_array_equal(mont.astype(np.int64), np.mod(want[0], p.astype(np.int64)))
    ctx.close()
