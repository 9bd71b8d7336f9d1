"""GPU NTT / INTT parity against the oracle (bit-exact modulo q; canonical
outputs integer-equal), every cluster size (logN 12..16) and both word sizes."""

import numpy as np
import pytest
import torch

from fhelium_b200 import _native as nat
from fhelium_b200.engine import CkksEngine
from tests.helpers import CONFIGS, canon, oracle_for, reduced_ring, to_dev, to_np, uniform_residues

pytestmark = pytest.mark.gpu

CASES = [("int64_logn16", k) for k in (12, 13, 14, 15, 16)] + [("int32_logn16", k) for k in (12, 14, 16)]


@pytest.mark.parametrize("ept", [8, 16])
@pytest.mark.parametrize("family,log_n", CASES)
def test_forward_inverse_match_oracle(family, log_n, ept):
    cfg = reduced_ring(CONFIGS[family](), log_n)
    eng = CkksEngine(cfg)
    # radix-8 (8 residues per thread) and radix-16 (16) launch variants
    eng.ctx.set_tuning(nat.TUNE_NTT_FORWARD_EPT, ept)
    eng.ctx.set_tuning(nat.TUNE_NTT_INVERSE_EPT, ept)
    orc = oracle_for(cfg, log_n)
    rng = np.random.default_rng(100 + log_n)
    rows = list(range(0, min(6, cfg.num_q_primes))) + list(range(cfg.num_q_primes, cfg.num_q_primes + cfg.num_p_primes))
    rows = rows[:6]
    start = rows[0]
    rows = list(range(start, start + len(rows)))
    x = uniform_residues(rng, cfg.moduli, rows, (3,), cfg.N)
    # standard -> NTT/Montgomery
    got = to_np(eng.forward_ntt(to_dev(x, cfg), start))
    ref = orc.forward_to_montgomery(x, rows)
    q2 = 2 * np.array([cfg.moduli[i] for i in rows])[:, None]
    assert (got >= 0).all() and (got < q2).all(), "forward output leaves the lazy range [0, 2q)"
    np.testing.assert_array_equal(canon(got, cfg.moduli, rows), canon(ref, cfg.moduli, rows))
    # Montgomery input (key-switch digit transform)
    y = uniform_residues(rng, cfg.moduli, rows, (2,), cfg.N, lazy=True)
    got = to_np(eng.forward_ntt(to_dev(y, cfg), start, montgomery_input=True))
    np.testing.assert_array_equal(canon(got, cfg.moduli, rows), canon(orc.forward_montgomery(y, rows), cfg.moduli, rows))
    # inverse to standard: canonical and integer-equal
    got_i = to_np(eng.inverse_ntt(to_dev(ref, cfg), start))
    np.testing.assert_array_equal(got_i, orc.inverse_to_standard(ref, rows))
    np.testing.assert_array_equal(got_i, x)


@pytest.mark.parametrize("kind", [nat.INV_MONTGOMERY, nat.INV_STANDARD_LAZY, nat.INV_CENTERED])
def test_inverse_output_kinds(kind):
    cfg = reduced_ring(CONFIGS["int64_logn16"](), 13)
    eng = CkksEngine(cfg)
    orc = oracle_for(cfg, 13)
    rng = np.random.default_rng(7)
    rows = [0, 1, 2]
    x = uniform_residues(rng, cfg.moduli, rows, (1,), cfg.N)
    ntt = orc.forward_to_montgomery(x, rows)
    got = to_np(eng.inverse_ntt(to_dev(ntt, cfg), 0, output=kind))
    q = np.array([cfg.moduli[i] for i in rows])[:, None]
    R = 1 << 62
    if kind == nat.INV_MONTGOMERY:
        want = np.array([[[(int(v) * R) % int(q[j, 0]) for v in x[0, j]] for j in range(3)]], dtype=object)
        np.testing.assert_array_equal(np.mod(got, q).astype(object), want)
        assert (got < 2 * q).all()
    elif kind == nat.INV_STANDARD_LAZY:
        np.testing.assert_array_equal(np.mod(got, q), x)
        assert (got < 2 * q).all()
    else:
        np.testing.assert_array_equal(np.mod(got, q), x)
        assert (np.abs(got) <= q // 2).all()


def test_ntt_in_place_and_batch_rows():
    cfg = CONFIGS["int64_logn14"]()
    eng = CkksEngine(cfg)
    orc = oracle_for(cfg)
    rng = np.random.default_rng(9)
    rows = list(range(2, 2 + 5))
    x = uniform_residues(rng, cfg.moduli, rows, (4,), cfg.N)
    t = to_dev(x, cfg)
    eng.forward_ntt(t, 2, out=t)
    np.testing.assert_array_equal(canon(to_np(t), cfg.moduli, rows), canon(orc.forward_to_montgomery(x, rows), cfg.moduli, rows))
    eng.inverse_ntt(t, 2, out=t)
    np.testing.assert_array_equal(to_np(t), x)


@pytest.mark.parametrize("log_n,rows,row_start", [(16, 35, 0), (16, 6, 31), (14, 8, 0), (13, 5, 2)])
@pytest.mark.parametrize("ept", [0, 16])
def test_f64_rows_equal_integer_rows(log_n, rows, row_start, ept):
    """Rows of primes below 2^42 in exact FP64 arithmetic (the default) against
    the integer path: forward (both input forms) and the lazy inverse kinds
    equal modulo q and in [0, 2q), the canonical inverse kinds integer-equal,
    including ranges that straddle the 60-bit rows."""
    from fhelium_b200 import _native as nat
    from fhelium_b200.config import CkksConfig, Preset
    from tests.helpers import reduced_ring
    cfg = CkksConfig.parse(Preset.slots32768_scale40_levels34_int64)
    if log_n != cfg.logN:
        cfg = reduced_ring(cfg, log_n)
    ctx = nat.NativeContext(64, log_n, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, torch.device("cuda:0"))
    assert ctx.get_tuning(nat.TUNE_F64_CORE) == 1
    ctx.set_tuning(nat.TUNE_NTT_FORWARD_EPT, ept)
    ctx.set_tuning(nat.TUNE_NTT_INVERSE_EPT, ept)
    q = torch.tensor(cfg.moduli[row_start:row_start + rows], dtype=torch.int64, device="cuda:0").view(1, rows, 1)
    g = torch.Generator(device="cuda:0").manual_seed(log_n + rows)
    x = torch.randint(0, 1 << 62, (3, rows, 1 << log_n), generator=g, device="cuda:0", dtype=torch.int64) % (2 * q)
    s = torch.cuda.current_stream().cuda_stream
    outs = {}
    for f64 in (1, 0):
        ctx.set_tuning(nat.TUNE_F64_CORE, f64)
        res = []
        for mode in (0, 1):
            y = torch.empty_like(x)
            nat.check(ctx.lib.fhb_forward_ntt(ctx.handle, x.data_ptr(), y.data_ptr(), 3, rows, row_start, mode, s), "f")
            res.append(y)
        for kind in range(4):
            z = torch.empty_like(x)
            nat.check(ctx.lib.fhb_inverse_ntt(ctx.handle, res[1].data_ptr(), z.data_ptr(), 3, rows, row_start, kind, s),
                      "i")
            res.append(z)
        outs[f64] = res
    # forward outputs and the lazy inverse kinds (0, 1) may pick another
    # representative in [0, 2q): equal modulo q; canonical kinds (2, 3) exactly
    for i, (a, b) in enumerate(zip(outs[1], outs[0])):
        if i < 4:
            assert torch.equal(a % q, b % q), i
            assert bool((a >= 0).all()) and bool((a < 2 * q).all()), i
        else:
            assert torch.equal(a, b), i
    ctx.close()
