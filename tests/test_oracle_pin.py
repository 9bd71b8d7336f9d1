"""Pin the CPU oracle against the reference's own CPU operators.

The reference's CPU kernels are compiled from its sources into
oracle/_ref (oracle/build_ref.sh) and called through their torch.ops
schemas; the oracle's C restatement must agree on the same seeded inputs:
bit-exact where the reference output is canonical, modulo q where it is lazy.
"""

import numpy as np
import pytest
import torch

from fhelium_b200.config import CkksConfig, Preset
from oracle import oracle as orc

LOG_N = 10


def _ctx(preset, log_n=LOG_N, **kw):
    cfg = CkksConfig.parse(preset, **kw)
    return orc.OracleContext(cfg.moduli, log_n, cfg.num_q_primes, cfg.num_p_primes,
                             cfg.buffer_bit_length, cfg.scale_bits)


CONTEXTS = {
    "int64": lambda: _ctx(Preset.slots8192_scale40_levels7_int64),
    "int64_p4": lambda: _ctx(Preset.slots32768_scale40_levels34_int64),
    "int32": lambda: _ctx(Preset.slots8192_scale25_levels14_int32),
}


def _uniform(rng, ctx, rows, batch=2):
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)
    return (rng.integers(0, 1 << 62, size=(batch, len(rows), ctx.n)) % q[:, None]).astype(np.int64)


def _lazy(rng, ctx, rows, batch=2):
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)
    return (rng.integers(0, 1 << 62, size=(batch, len(rows), ctx.n)) % (2 * q[:, None])).astype(np.int64)


def _t(a, ctx):
    dt = torch.int64 if ctx.radix_bits == 62 else torch.int32
    return torch.from_numpy(np.ascontiguousarray(a)).to(dt).clone()


def _np(t):
    return t.to(torch.int64).numpy()


def _indexed_schedule(log_n):
    """Forward/inverse radix-2 schedules (fhelium/engine/ntt/plans/indexed_radix2.py)."""
    n = 1 << log_n
    fe, fo, ft = [], [], []
    half = n
    for s in range(log_n):
        half //= 2
        g = np.arange(1 << s)
        e = (2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1)
        fe.append(e); fo.append(e + half); ft.append(np.repeat((1 << s) + g, half))
    ie, io, it = [], [], []
    half = 1
    for rem in range(log_n, 0, -1):
        gc = 1 << (rem - 1)
        g = np.arange(gc)
        e = (2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1)
        ie.append(e); io.append(e + half); it.append(np.repeat(gc + g, half))
        half *= 2
    as32 = lambda x: torch.tensor(np.stack(x), dtype=torch.int32)
    return as32(fe), as32(fo), np.stack(ft), as32(ie), as32(io), np.stack(it)


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_pointwise_ops_match_reference(ref_ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(11)
    rows = ctx.q_rows(0)
    a, b = _lazy(rng, ctx, rows), _lazy(rng, ctx, rows)
    prm = ctx.sub_params(rows)
    ref = _np(ref_ops.fhelium_rns_ops.montgomery_mul(_t(a, ctx), _t(b, ctx), _t(prm, ctx)))
    got = orc.montgomery_mul(a, b, prm, ctx.radix_bits)
    np.testing.assert_array_equal(got, ref)
    ref = _np(ref_ops.fhelium_rns_ops.add_lazy(_t(a, ctx), _t(b, ctx), _t(prm, ctx)))
    np.testing.assert_array_equal(orc.add_lazy(a, b, prm), ref)


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_ntt_matches_reference(ref_ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(12)
    rows = ctx.qp_rows(0)
    prm = ctx.sub_params(rows)
    fe, fo, ft, ie, io, it = _indexed_schedule(ctx.log_n)
    fwd, inv = ctx.twiddles
    fwd_stage = np.stack([fwd[j][ft] for j in range(len(rows))])
    inv_stage = np.stack([inv[j][it] for j in range(len(rows))])
    x = _uniform(rng, ctx, rows)
    ref = _np(ref_ops.fhelium_ntt_ops.forward_ntt_to_montgomery_indexed(
        _t(x, ctx), fe, fo, _t(fwd_stage, ctx), _t(prm, ctx)))
    got = ctx.forward_to_montgomery(x, rows)
    np.testing.assert_array_equal(got, ref)
    # Montgomery-input forward (the key-switch digit transform)
    y = _lazy(rng, ctx, rows)
    ref_y = _t(y, ctx).clone()
    ref_ops.fhelium_ntt_ops.forward_ntt_montgomery_indexed_(ref_y, fe, fo, _t(fwd_stage, ctx), _t(prm, ctx))
    np.testing.assert_array_equal(ctx.forward_montgomery(y, rows), _np(ref_y))
    # inverse to standard (canonical)
    ref_i = _t(ref, ctx).clone()
    ref_ops.fhelium_ntt_ops.inverse_ntt_to_standard_indexed_(ref_i, ie, io, _t(inv_stage, ctx), _t(prm, ctx))
    got_i = ctx.inverse_to_standard(ref, rows)
    np.testing.assert_array_equal(got_i, _np(ref_i))
    np.testing.assert_array_equal(got_i, x)  # round trip


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_modup_matches_reference(ref_ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(13)
    level = 0
    q_rows = ctx.q_rows(level)
    x = _lazy(rng, ctx, q_rows)
    dst = ctx.qp_rows(level)
    for kd, ids in ctx.digits_at_level(level):
        norm, prop, ext = ctx.digit_tables(ids)
        src = x[:, ids[0]:ids[-1] + 1]
        if len(ids) > 1:
            dprm = ctx.sub_params(list(ids))
            ref_d = _np(ref_ops.fhelium_rns_ops.mixed_radix_decompose(
                _t(src, ctx), _t(norm, ctx), _t(prop, ctx), _t(dprm[1], ctx), _t(dprm[2], ctx),
                _t(dprm[3], ctx), _t(dprm[4], ctx)))
            got_d = orc.mixed_radix_decompose(src, norm, prop, dprm, ctx.radix_bits)
            np.testing.assert_array_equal(got_d, ref_d)
        else:
            ref_d = src
        coeffs = ext[:, dst] if len(ids) > 1 else np.zeros((0, 0), np.int64)
        ref_e = _np(ref_ops.fhelium_rns_ops.mixed_radix_basis_extend_to_montgomery(
            _t(ref_d, ctx), _t(coeffs, ctx), _t(ctx.sub_params(dst), ctx), len(dst)))
        got_e = ctx.extend_digit(x, level, ids)
        np.testing.assert_array_equal(ctx.canonical(got_e, dst), ctx.canonical(ref_e, dst))


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("level", [0, 3])
def test_keyswitch_pieces_match_reference(ref_ops, family, level):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(14 + level)
    qp = ctx.qp_rows(level)
    prm = ctx.sub_params(qp)
    digit = _lazy(rng, ctx, qp)
    key = np.stack([_uniform(rng, ctx, ctx.qp_rows(0), batch=1)[0] for _ in range(2)])
    acc0, acc1 = _lazy(rng, ctx, qp), _lazy(rng, ctx, qp)
    r0, r1 = _t(acc0, ctx), _t(acc1, ctx)
    ref_ops.fhelium_ckks_ops.keyswitch_accumulate_digit_products_(
        r0, r1, _t(digit, ctx), _t(key, ctx), _t(prm, ctx), level)
    g0, g1 = orc.keyswitch_accumulate(acc0, acc1, digit, key, prm, level, ctx.radix_bits)
    np.testing.assert_array_equal(ctx.canonical(g0, qp), ctx.canonical(_np(r0), qp))
    np.testing.assert_array_equal(ctx.canonical(g1, qp), ctx.canonical(_np(r1), qp))
    # ModDown: canonical Q and P inputs, canonical Q output
    acc = _uniform(rng, ctx, qp)
    p = ctx.num_p
    inv = ctx.moddown_inverse(level)
    ref = _np(ref_ops.fhelium_ckks_ops.keyswitch_moddown_qp_to_q(
        _t(acc[:, :-p], ctx), _t(acc[:, -p:], ctx), _t(inv, ctx), _t(prm, ctx)))
    got = orc.keyswitch_moddown(acc[:, :-p], acc[:, -p:], inv, prm, ctx.radix_bits)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("nearest", [True, False])
def test_rescale_matches_reference(ref_ops, family, nearest):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(15)
    level = 1
    rows = ctx.q_rows(level)
    x = _uniform(rng, ctx, rows)
    inv = ctx.rescale_inverse(level)[: len(rows) - 1]
    prm = ctx.sub_params(rows[1:])
    half = ctx.moduli[rows[0]] // 2
    op = (ref_ops.fhelium_ckks_ops.rescale_drop_leading_prime_nearest if nearest
          else ref_ops.fhelium_ckks_ops.rescale_drop_leading_prime_truncate)
    args = (_t(x[:, 1:], ctx), _t(inv, ctx), _t(x[:, 0], ctx), _t(prm, ctx))
    ref = _np(op(*args, half) if nearest else op(*args))
    got = orc.rescale_drop_leading(x[:, 1:], x[:, 0], inv, prm, half, nearest, ctx.radix_bits)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("step", [1, -1, 8, 5])
def test_automorphisms_match_reference(ref_ops, family, step):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(16)
    rows = ctx.q_rows(0)
    x = _uniform(rng, ctx, rows)
    g = orc.galois_element(ctx.n, step % ctx.n)
    src, sign = orc.coefficient_galois_tables(ctx.n, g)
    tq = np.array([2 * ctx.moduli[i] for i in rows], dtype=np.int64)
    ref = _np(ref_ops.fhelium_ckks_ops.apply_coefficient_galois_automorphism(
        _t(x, ctx), torch.from_numpy(src), torch.from_numpy(sign), _t(tq, ctx)))
    np.testing.assert_array_equal(orc.coefficient_automorphism(x, src, sign, tq), ref)
    nsrc = orc.ntt_galois_source_indices(ctx.n, g)
    ref = _np(ref_ops.fhelium_ckks_ops.apply_ntt_galois_automorphism(_t(x, ctx), torch.from_numpy(nsrc)))
    np.testing.assert_array_equal(orc.ntt_automorphism(x, nsrc), ref)


@pytest.mark.parametrize("family,level", [("int64", 0), ("int64_p4", 30), ("int32", 2)])
def test_reference_pipeline_matches_oracle_engine_path(ref_ops, family, level):
    """The reference's own CPU operators, driven in the reference engine's
    order, equal the oracle's HMult -> relinearize -> rescale bit for bit."""
    from oracle.ref_pipeline import ReferenceCpuPipeline
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(21)
    rows = ctx.q_rows(level)
    a, b = _lazy(rng, ctx, rows), _lazy(rng, ctx, rows)
    key = np.stack([np.stack([_uniform(rng, ctx, ctx.qp_rows(0), batch=1)[0] for _ in range(2)])
                    for _ in ctx.digits_at_level(0)])
    pipe = ReferenceCpuPipeline(ctx)
    got = _np(pipe.multiply_relinearize_rescale(_t(a, ctx), _t(b, ctx), _t(key, ctx), level))
    want = ctx.rescale(ctx.relinearize(ctx.multiply(a, b, level), key, level), level)
    np.testing.assert_array_equal(got, want)
