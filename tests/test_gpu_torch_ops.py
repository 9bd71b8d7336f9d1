"""The reference's operator schemas served on B200 (fhelium_b200.torch_ops).

The same ``torch.ops.fhelium_*`` calls that the oracle pin tests make on CPU
tensors (where they reach the reference's own CPU kernels) are made here on CUDA
tensors, where they reach this library's kernels.  Outputs must equal the
oracle's -- integer-equal where the reference's output is canonical or lazy by
the same rule, equal modulo q for NTT-domain outputs (lazy [0, 2q) on CUDA) --
and, when the reference's CPU library is present, the reference's own CPU
kernels on the same inputs (its cross-backend rule, reference
tests/test_ckks_operation_correctness.py:276-401).  The last test drives the
reference engine's whole HMult -> relinearize -> rescale operator sequence on
CUDA tensors.
"""

import numpy as np
import pytest
import torch

from fhelium_b200.config import CkksConfig, Preset
from oracle import oracle as orc
from oracle import ref_pipeline

pytestmark = pytest.mark.gpu

LOG_N = 12


def _ctx(preset, **kw):
    cfg = CkksConfig.parse(preset, **kw)
    return orc.OracleContext(cfg.moduli, LOG_N, cfg.num_q_primes, cfg.num_p_primes, cfg.buffer_bit_length,
                             cfg.scale_bits)


CONTEXTS = {
    "int64": lambda: _ctx(Preset.slots8192_scale40_levels7_int64),
    "int64_p4": lambda: _ctx(Preset.slots32768_scale40_levels34_int64),
    "int32": lambda: _ctx(Preset.slots8192_scale25_levels14_int32),
}


@pytest.fixture(scope="module")
def ops():
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    if ref_pipeline.available():
        torch.ops.load_library(ref_pipeline.REF_LIB)   # the reference's schema definitions + CPU kernels
    from fhelium_b200 import torch_ops
    torch_ops.register()
    return torch.ops


def _uniform(rng, ctx, rows, batch=2):
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)
    return (rng.integers(0, 1 << 62, size=(batch, len(rows), ctx.n)) % q[:, None]).astype(np.int64)


def _lazy(rng, ctx, rows, batch=2):
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)
    return (rng.integers(0, 1 << 62, size=(batch, len(rows), ctx.n)) % (2 * q[:, None])).astype(np.int64)


def _dt(ctx):
    return torch.int64 if ctx.radix_bits == 62 else torch.int32


def _c(a, ctx):
    return torch.from_numpy(np.ascontiguousarray(a)).to(_dt(ctx)).cuda()


def _h(a, ctx):
    return torch.from_numpy(np.ascontiguousarray(a)).to(_dt(ctx))


def _n(t):
    return t.cpu().to(torch.int64).numpy()


def _mod(a, ctx, rows):
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)
    return a % q[:, None]


def _same_on_cpu(op, args_np, ctx, got, modq_rows=None):
    """The reference's CPU kernel on the same inputs gives the same integers."""
    if not ref_pipeline.available():
        return
    ref = op(*[_h(a, ctx) if isinstance(a, np.ndarray) else a for a in args_np])
    ref = ref.to(torch.int64).numpy()
    if modq_rows is None:
        np.testing.assert_array_equal(got, ref)
    else:
        np.testing.assert_array_equal(_mod(got, ctx, modq_rows), _mod(ref, ctx, modq_rows))


def _schedule(log_n):
    fe, fo, ft, ie, io, it = ref_pipeline._schedule(log_n)
    return fe, fo, ft, ie, io, it


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_pointwise_ops(ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(11)
    rows = ctx.q_rows(0)
    a, b = _lazy(rng, ctx, rows), _lazy(rng, ctx, rows)
    prm = ctx.sub_params(rows)
    rns = ops.fhelium_rns_ops
    got = _n(rns.montgomery_mul(_c(a, ctx), _c(b, ctx), _c(prm, ctx)))
    np.testing.assert_array_equal(got, orc.montgomery_mul(a, b, prm, ctx.radix_bits))
    _same_on_cpu(rns.montgomery_mul, (a, b, prm), ctx, got)
    got = _n(rns.add_lazy(_c(a, ctx), _c(b, ctx), _c(prm, ctx)))
    np.testing.assert_array_equal(got, orc.add_lazy(a, b, prm))
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)[:, None]
    got = _n(rns.sub_lazy(_c(a, ctx), _c(b, ctx), _c(prm, ctx)))
    np.testing.assert_array_equal(got, (a - b) % (2 * q))
    _same_on_cpu(rns.sub_lazy, (a, b, prm), ctx, got)
    # canonical add / sub, functional and in place, with a singleton rhs batch
    got = _n(rns.add_canonical(_c(a, ctx), _c(b[:1], ctx), _c(prm, ctx)))
    np.testing.assert_array_equal(got, (a + b[:1]) % q)
    _same_on_cpu(rns.add_canonical, (a, b[:1], prm), ctx, got)
    x = _c(a, ctx)
    rns.sub_canonical_(x, _c(b, ctx), _c(prm, ctx))
    np.testing.assert_array_equal(_n(x), (a - b) % q)
    # unary in-place ops
    s = _uniform(rng, ctx, rows)
    x = _c(s, ctx)
    rns.to_montgomery_(x, _c(prm, ctx))
    R = 1 << ctx.radix_bits
    want = np.stack([[np.array([(int(v) * R) % ctx.moduli[i] for v in s[bb, j]]) for j, i in enumerate(rows)]
                     for bb in range(s.shape[0])])
    np.testing.assert_array_equal(_n(x), want)
    rns.from_montgomery_(x, _c(prm, ctx))
    np.testing.assert_array_equal(_n(x), s)
    x = _c(a, ctx)
    rns.canonicalize_residues_(x, _c(prm, ctx))
    np.testing.assert_array_equal(_n(x), a % q)
    rns.center_residues_(x, _c(prm, ctx))
    centered = np.where(a % q <= q // 2, a % q, a % q - q)
    np.testing.assert_array_equal(_n(x), centered)
    rns.shift_residues_positive_(x, _c(prm, ctx))
    np.testing.assert_array_equal(_n(x), centered + q)
    # lift of signed coefficients to every row
    coeffs = rng.integers(-1000, 1000, size=(3, ctx.n)).astype(np.int64)
    tq = np.array([2 * ctx.moduli[i] for i in rows], dtype=np.int64)
    got = _n(rns.lift_centered_coefficients(_c(coeffs, ctx), _c(tq, ctx)))
    np.testing.assert_array_equal(got, coeffs[:, None, :] + q[None])
    _same_on_cpu(rns.lift_centered_coefficients, (coeffs, tq), ctx, got)


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_ntt_ops(ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(12)
    rows = ctx.qp_rows(0)
    prm = ctx.sub_params(rows)
    fe, fo, ft, ie, io, it = _schedule(ctx.log_n)
    fwd, inv = ctx.twiddles
    fwd_stage = np.stack([fwd[j][ft] for j in range(len(rows))])
    inv_stage = np.stack([inv[j][it] for j in range(len(rows))])
    ntt = ops.fhelium_ntt_ops
    x = _uniform(rng, ctx, rows)
    want = _mod(ctx.forward_to_montgomery(x, rows), ctx, rows)   # the oracle's forward output is lazy
    # indexed (the reference CPU backend's form) and compact forms
    got = _n(ntt.forward_ntt_to_montgomery_indexed(_c(x, ctx), fe.cuda(), fo.cuda(), _c(fwd_stage, ctx),
                                                   _c(prm, ctx)))
    np.testing.assert_array_equal(_mod(got, ctx, rows), want)
    _same_on_cpu(ntt.forward_ntt_to_montgomery_indexed, (x, fe, fo, fwd_stage, prm), ctx, got, modq_rows=rows)
    got = _n(ntt.forward_ntt_to_montgomery_compact_grouped_smem(_c(x, ctx), _c(fwd, ctx), _c(prm, ctx), 3))
    np.testing.assert_array_equal(_mod(got, ctx, rows), want)
    y = _lazy(rng, ctx, rows)
    t = _c(y, ctx)
    ntt.forward_ntt_montgomery_indexed_(t, fe.cuda(), fo.cuda(), _c(fwd_stage, ctx), _c(prm, ctx))
    np.testing.assert_array_equal(_mod(_n(t), ctx, rows), _mod(ctx.forward_montgomery(y, rows), ctx, rows))
    t = _c(y, ctx)
    ntt.forward_ntt_montgomery_compact_grouped_smem_(t, _c(fwd, ctx), _c(prm, ctx), 2)
    np.testing.assert_array_equal(_mod(_n(t), ctx, rows), _mod(ctx.forward_montgomery(y, rows), ctx, rows))
    # inverse: every output kind, both forms
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)[:, None]
    R = 1 << ctx.radix_bits
    xr = np.stack([[np.array([(int(v) * R) % ctx.moduli[i] for v in x[bb, j]]) for j, i in enumerate(rows)]
                   for bb in range(x.shape[0])])
    for name, want_i, exact in (("inverse_ntt_to_standard", x, True), ("inverse_ntt_to_standard_lazy", x, False),
                                ("inverse_ntt_montgomery", xr, False),
                                ("inverse_ntt_to_centered", np.where(x <= q // 2, x, x - q), True)):
        for form in ("indexed", "compact"):
            t = _c(got, ctx)
            if form == "indexed":
                getattr(ntt, name + "_indexed_")(t, ie.cuda(), io.cuda(), _c(inv_stage, ctx), _c(prm, ctx))
            else:
                getattr(ntt, name + "_compact_grouped_smem_")(t, _c(inv, ctx), _c(prm, ctx), 3)
            out = _n(t)
            if exact:
                np.testing.assert_array_equal(out, want_i, err_msg=f"{name} {form}")
            else:
                np.testing.assert_array_equal(_mod(out, ctx, rows), want_i % q, err_msg=f"{name} {form}")
    # a limb slice of a larger tensor (rows N words apart, wider batch stride), transformed in place
    big = _c(x, ctx)
    view = big[:, 2:]
    ntt.forward_ntt_to_montgomery_compact_grouped_smem_(view, _c(fwd[2:], ctx), _c(prm[:, 2:], ctx), 3)
    np.testing.assert_array_equal(_mod(_n(view), ctx, rows[2:]),
                                  _mod(ctx.forward_to_montgomery(x[:, 2:], rows[2:]), ctx, rows[2:]))
    np.testing.assert_array_equal(_n(big[:, :2]), x[:, :2])


def test_ntt_ops_reject_what_the_reference_rejects(ops):
    ctx = CONTEXTS["int64"]()
    rows = ctx.q_rows(0)
    prm = _c(ctx.sub_params(rows), ctx)
    fe, fo, ft, *_ = _schedule(ctx.log_n)
    fwd, _ = ctx.twiddles
    fwd_stage = _c(np.stack([fwd[j][ft] for j in range(len(rows))]), ctx)
    x = _c(_uniform(np.random.default_rng(3), ctx, rows), ctx)
    ntt = ops.fhelium_ntt_ops
    with pytest.raises(RuntimeError, match=r"log2\(N\) stages"):
        ntt.forward_ntt_to_montgomery_indexed(x, fe[:-1].cuda(), fo[:-1].cuda(), fwd_stage[:, :-1], prm)
    bad = fe.clone()
    bad[0, 0] = ctx.n
    with pytest.raises(RuntimeError, match="out-of-range coefficient index"):
        ntt.forward_ntt_to_montgomery_indexed(x, bad.cuda(), fo.cuda(), fwd_stage, prm)
    dup = fe.clone()
    dup[0, 1] = dup[0, 0]
    with pytest.raises(RuntimeError, match="partition every coefficient"):
        ntt.forward_ntt_to_montgomery_indexed(x, dup.cuda(), fo.cuda(), fwd_stage, prm)
    with pytest.raises(RuntimeError, match="more than one element"):
        ntt.forward_ntt_to_montgomery_indexed_(x[:1].expand(2, -1, -1), fe.cuda(), fo.cuda(), fwd_stage, prm)
    with pytest.raises(RuntimeError, match="primitive root"):
        ntt.forward_ntt_to_montgomery_compact_grouped_smem(x, torch.ones_like(_c(fwd[: len(rows)], ctx)), prm, 3)
    with pytest.raises(RuntimeError, match="dtype"):
        ops.fhelium_rns_ops.montgomery_mul(x, x.to(torch.int32), prm)


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_modup_ops(ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(13)
    level = 0
    x = _lazy(rng, ctx, ctx.q_rows(level))
    dst = ctx.qp_rows(level)
    rns = ops.fhelium_rns_ops
    for kd, ids in ctx.digits_at_level(level):
        norm, prop, ext = ctx.digit_tables(ids)
        src = x[:, ids[0]:ids[-1] + 1]
        dprm = ctx.sub_params(list(ids))
        if len(ids) > 1:
            args = (src, norm, prop, dprm[1], dprm[2], dprm[3], dprm[4])
            got_d = _n(rns.mixed_radix_decompose(*[_c(a, ctx) for a in args]))
            np.testing.assert_array_equal(got_d, orc.mixed_radix_decompose(src, norm, prop, dprm, ctx.radix_bits))
            _same_on_cpu(rns.mixed_radix_decompose, args, ctx, got_d)
        else:
            got_d = src
        coeffs = ext[:, dst] if len(ids) > 1 else np.zeros((0, 0), np.int64)
        got_e = _n(rns.mixed_radix_basis_extend_to_montgomery(_c(got_d, ctx), _c(coeffs, ctx),
                                                              _c(ctx.sub_params(dst), ctx), len(dst)))
        want = orc.basis_extend_to_montgomery(got_d, coeffs, ctx.sub_params(dst), ctx.radix_bits)
        np.testing.assert_array_equal(got_e, want)
        np.testing.assert_array_equal(ctx.canonical(got_e, dst), ctx.canonical(ctx.extend_digit(x, level, ids), dst))


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("level", [0, 3])
def test_keyswitch_ops(ops, family, level):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(14 + level)
    qp = ctx.qp_rows(level)
    prm = ctx.sub_params(qp)
    digit = _lazy(rng, ctx, qp)
    key = np.stack([_uniform(rng, ctx, ctx.qp_rows(0), batch=1)[0] for _ in range(2)])
    acc0, acc1 = _lazy(rng, ctx, qp), _lazy(rng, ctx, qp)
    r0, r1 = _c(acc0, ctx), _c(acc1, ctx)
    ops.fhelium_ckks_ops.keyswitch_accumulate_digit_products_(r0, r1, _c(digit, ctx), _c(key, ctx), _c(prm, ctx),
                                                              level)
    g0, g1 = orc.keyswitch_accumulate(acc0, acc1, digit, key, prm, level, ctx.radix_bits)
    np.testing.assert_array_equal(_n(r0), g0)
    np.testing.assert_array_equal(_n(r1), g1)
    # the fused forward-NTT + accumulate schema: NTT of the digit, then the same products
    fwd, _ = ctx.twiddles
    r0, r1, d = _c(acc0, ctx), _c(acc1, ctx), _c(digit, ctx)
    ops.fhelium_ntt_ops.forward_ntt_montgomery_compact_keyswitch_accumulate_(
        d, _c(fwd[level:], ctx), _c(prm, ctx), _c(key, ctx), r0, r1, level)
    dn = _mod(ctx.forward_montgomery(digit, qp), ctx, qp)
    np.testing.assert_array_equal(_mod(_n(d), ctx, qp), dn)
    g0, g1 = orc.keyswitch_accumulate(acc0, acc1, _n(d), key, prm, level, ctx.radix_bits)
    np.testing.assert_array_equal(_n(r0), g0)
    np.testing.assert_array_equal(_n(r1), g1)
    # ModDown of slices of one accumulator (no copies)
    acc = _uniform(rng, ctx, qp)
    p = ctx.num_p
    inv = ctx.moddown_inverse(level)
    full = _c(acc, ctx)
    got = _n(ops.fhelium_ckks_ops.keyswitch_moddown_qp_to_q(full[:, :-p], full[:, -p:], _c(inv, ctx), _c(prm, ctx)))
    want = orc.keyswitch_moddown(acc[:, :-p], acc[:, -p:], inv, prm, ctx.radix_bits)
    np.testing.assert_array_equal(got, want)
    # ModDown leaves its P rows (public values) untouched
    # (reference tests/test_native_operator_invariants.py:201-268)
    np.testing.assert_array_equal(_n(full), acc)
    # an in-place op whose read-only operand is the written tensor is rejected
    with pytest.raises(RuntimeError, match="single memory location"):
        ops.fhelium_rns_ops.add_canonical_(full, full, _c(prm, ctx))
    _same_on_cpu(ops.fhelium_ckks_ops.keyswitch_moddown_qp_to_q, (acc[:, :-p], acc[:, -p:], inv, prm), ctx, got)


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("nearest", [True, False])
def test_rescale_ops(ops, family, nearest):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(15)
    level = 1
    rows = ctx.q_rows(level)
    x = _uniform(rng, ctx, rows)
    inv = ctx.rescale_inverse(level)[: len(rows) - 1]
    prm = ctx.sub_params(rows[1:])
    half = ctx.moduli[rows[0]] // 2
    ck = ops.fhelium_ckks_ops
    want = orc.rescale_drop_leading(x[:, 1:], x[:, 0], inv, prm, half, nearest, ctx.radix_bits)
    xc = _c(x, ctx)
    if nearest:
        got = _n(ck.rescale_drop_leading_prime_nearest(xc[:, 1:], _c(inv, ctx), xc[:, 0], _c(prm, ctx), half))
    else:
        got = _n(ck.rescale_drop_leading_prime_truncate(xc[:, 1:], _c(inv, ctx), xc[:, 0], _c(prm, ctx)))
    np.testing.assert_array_equal(got, want)
    # in place on the remaining rows of the same tensor
    rem = xc[:, 1:]
    if nearest:
        ck.rescale_drop_leading_prime_nearest_(rem, _c(inv, ctx), xc[:, 0], _c(prm, ctx), half)
    else:
        ck.rescale_drop_leading_prime_truncate_(rem, _c(inv, ctx), xc[:, 0], _c(prm, ctx))
    np.testing.assert_array_equal(_n(xc[:, 1:]), want)
    np.testing.assert_array_equal(_n(xc[:, 0]), x[:, 0])


@pytest.mark.parametrize("family", list(CONTEXTS))
@pytest.mark.parametrize("step", [1, -1, 8, 5])
def test_automorphism_ops(ops, family, step):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(16)
    rows = ctx.q_rows(0)
    x = _uniform(rng, ctx, rows)
    g = orc.galois_element(ctx.n, step % ctx.n)
    src, sign = orc.coefficient_galois_tables(ctx.n, g)
    tq = np.array([2 * ctx.moduli[i] for i in rows], dtype=np.int64)
    ck = ops.fhelium_ckks_ops
    got = _n(ck.apply_coefficient_galois_automorphism(_c(x, ctx), torch.from_numpy(src).cuda(),
                                                      torch.from_numpy(sign).cuda(), _c(tq, ctx)))
    np.testing.assert_array_equal(got, orc.coefficient_automorphism(x, src, sign, tq))
    nsrc = orc.ntt_galois_source_indices(ctx.n, g)
    got = _n(ck.apply_ntt_galois_automorphism(_c(x, ctx), torch.from_numpy(nsrc).cuda()))
    np.testing.assert_array_equal(got, orc.ntt_automorphism(x, nsrc))


@pytest.mark.parametrize("family,level", [("int64", 0), ("int64_p4", 30), ("int32", 2)])
def test_reference_operator_sequence_on_cuda(ops, family, level):
    """The reference engine's HMult -> relinearize -> rescale operator sequence,
    issued on CUDA tensors, equals the oracle bit for bit."""
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(21)
    rows = ctx.q_rows(level)
    a, b = _lazy(rng, ctx, rows), _lazy(rng, ctx, rows)
    key = np.stack([np.stack([_uniform(rng, ctx, ctx.qp_rows(0), batch=1)[0] for _ in range(2)])
                    for _ in ctx.digits_at_level(0)])
    pipe = ref_pipeline.ReferenceCpuPipeline(ctx, device="cuda")
    got = _n(pipe.multiply_relinearize_rescale(_c(a, ctx), _c(b, ctx), _c(key, ctx), level))
    want = ctx.rescale(ctx.relinearize(ctx.multiply(a, b, level), key, level), level)
    np.testing.assert_array_equal(got, want)


def _expand(pt, layout, n, implicit=None):
    """Dense [*, rows, N] form of a repeated / strided plaintext (reference
    csrc/ops/common/cuda/repetition.cuh:69-86, csrc/ops/ckks/cuda/plaintext_cuda.cu:93-114)."""
    u = pt.shape[-1]
    k = np.arange(n)
    if layout == "cyclic":
        return pt[..., k % u]
    if layout == "contiguous":
        return pt[..., k // (n // u)]
    stride = n // u
    dense = np.repeat(implicit[..., None], n, axis=-1)
    dense[..., ::stride] = pt
    return dense


@pytest.mark.parametrize("family", list(CONTEXTS))
def test_plaintext_and_compressed_ops(ops, family):
    ctx = CONTEXTS[family]()
    rng = np.random.default_rng(17)
    rows = ctx.q_rows(0)
    prm = ctx.sub_params(rows)
    n = ctx.n
    q = np.array([ctx.moduli[i] for i in rows], dtype=np.int64)[:, None]
    rns, ck = ops.fhelium_rns_ops, ops.fhelium_ckks_ops
    a = _lazy(rng, ctx, rows, batch=3)
    for layout, name in (("cyclic", "montgomery_mul_cyclic_compressed"),
                         ("contiguous", "montgomery_mul_contiguous_compressed")):
        comp = _lazy(rng, ctx, rows, batch=1)[..., :64]
        got = _n(getattr(rns, name)(_c(a, ctx), _c(comp, ctx), _c(prm, ctx)))
        dense = np.broadcast_to(_expand(comp, layout, n), a.shape)
        np.testing.assert_array_equal(got, orc.montgomery_mul(a, dense, prm, ctx.radix_bits), err_msg=name)
        _same_on_cpu(getattr(rns, name), (a, comp, prm), ctx, got)
    scal = _uniform(rng, ctx, rows, batch=1)[0, :, 0].copy()
    got = _n(rns.montgomery_mul_row_scalars_canonical(_c(a, ctx), _c(scal, ctx), _c(prm, ctx)))
    want = orc.montgomery_mul(a, np.broadcast_to(scal[None, :, None], a.shape), prm, ctx.radix_bits)
    np.testing.assert_array_equal(got, want)
    x = _c(a, ctx)
    rns.montgomery_mul_row_scalars_(x, _c(scal, ctx), _c(prm, ctx))
    np.testing.assert_array_equal(_n(x), want)
    b = _lazy(rng, ctx, rows, batch=3)
    tq = (2 * q[:, 0]).copy()
    got = _n(rns.add_lazy_with_twice_modulus(_c(a, ctx), _c(b, ctx), _c(tq, ctx)))
    np.testing.assert_array_equal(got, orc.add_lazy(a, b, prm))
    # plaintext additions: c + p R^-1 mod q, canonical
    c = _uniform(rng, ctx, rows, batch=3)
    ones = np.ones_like(c)
    cases = {
        "prepared": (_lazy(rng, ctx, rows, batch=3), None),
        "cyclic_compressed": (_lazy(rng, ctx, rows, batch=1)[..., :128], None),
        "contiguous_compressed": (_lazy(rng, ctx, rows, batch=1)[..., :32], None),
        "strided": (_lazy(rng, ctx, rows, batch=3)[..., :256], _uniform(rng, ctx, rows, batch=3)[..., 0].copy()),
    }
    for kind, (pt, implicit) in cases.items():
        if kind == "prepared":
            dense = pt
        elif kind == "strided":
            dense = _expand(pt, "strided", n, implicit)
        else:
            dense = _expand(pt, kind.split("_")[0], n)
        dense = np.broadcast_to(dense, c.shape)
        want = (c + orc.montgomery_mul(dense, ones, prm, ctx.radix_bits)) % q
        op = getattr(ck, f"add_{kind}_plaintext_component")
        args = (c, pt, implicit, prm) if kind == "strided" else (c, pt, prm)
        got = _n(op(*[_c(v, ctx) for v in args]))
        np.testing.assert_array_equal(got, want, err_msg=kind)
        _same_on_cpu(op, args, ctx, got)
        t = _c(c, ctx)
        getattr(ck, f"add_{kind}_plaintext_component_")(t, *[_c(v, ctx) for v in args[1:]])
        np.testing.assert_array_equal(_n(t), want, err_msg=kind + "_")


@pytest.mark.parametrize("family,radix", [("int64", 4), ("int64_p4", 16), ("int32", 8)])
def test_power_of_two_radix_ntt_forms(ops, family, radix):
    """The reference's power-of-two-radix NTT schemas compute the same transform
    (same root, same bit-reversed order); their tables are checked for shape and
    for the radix-th root psi^(2N/radix) in Montgomery form."""
    ctx = CONTEXTS[family]()
    if ctx.log_n % {4: 2, 8: 3, 16: 4}[radix]:
        pytest.skip("radix width does not divide log N")
    rng = np.random.default_rng(18)
    rows = ctx.qp_rows(0)
    prm = ctx.sub_params(rows)
    n, R = ctx.n, 1 << ctx.radix_bits
    roots_f, roots_i = [], []
    for i in rows:
        qi = ctx.moduli[i]
        w = pow(orc.primitive_2nth_root(qi, n), 2 * n // radix, qi)
        wi = pow(w, -1, qi)
        roots_f.append([(pow(w, k, qi) * R) % qi for k in range(radix)])
        roots_i.append([(pow(wi, k, qi) * R) % qi for k in range(radix)])
    outer = np.zeros((len(rows), n - 1), np.int64)   # read for its shape only
    ntt = ops.fhelium_ntt_ops
    x = _uniform(rng, ctx, rows)
    got = _n(ntt.forward_ntt_to_montgomery_power_of_two_radix_compact(_c(x, ctx), _c(outer, ctx),
                                                                       _c(np.array(roots_f), ctx), _c(prm, ctx)))
    np.testing.assert_array_equal(_mod(got, ctx, rows), _mod(ctx.forward_to_montgomery(x, rows), ctx, rows))
    t = _c(got, ctx)
    ntt.inverse_ntt_to_standard_power_of_two_radix_compact_(t, _c(outer, ctx), _c(np.array(roots_i), ctx),
                                                            _c(prm, ctx))
    np.testing.assert_array_equal(_n(t), x)
    with pytest.raises(RuntimeError, match="primitive root"):
        ntt.forward_ntt_montgomery_power_of_two_radix_compact_(_c(x, ctx), _c(outer, ctx),
                                                               _c(np.array(roots_i), ctx), _c(prm, ctx))
