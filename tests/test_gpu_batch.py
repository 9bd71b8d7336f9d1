"""Mixed-level batches: one CUDA graph over every (kind, level) group against
one engine call sequence per ciphertext, bit for bit, and the autotuner."""

import ctypes
import json

import numpy as np
import pytest
import torch

from fhelium_b200 import autotune
from fhelium_b200.batch import (HMULT, ROTATE, MixedBatchExecutor, MixedItemsExecutor, MixedOp, run_per_ciphertext,
                                sample_mixed_workload)
from fhelium_b200.config import Preset
from fhelium_b200.engine import CkksEngine

pytestmark = pytest.mark.gpu


def _workload(eng, count, seed, max_step):
    levels, ops = sample_mixed_workload(eng.num_q, count, max_step=max_step, seed=seed)
    rng = np.random.default_rng(seed + 100)
    cts = [eng.encrypt_message(rng.uniform(-0.05, 0.05, eng.num_slots), level=lv) for lv in levels]
    return cts, ops


@pytest.fixture(scope="module")
def small():
    eng = CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=3)
    cts, ops = _workload(eng, 40, seed=11, max_step=1 << 12)
    want = run_per_ciphertext(eng, cts, ops)
    return eng, cts, ops, want


@pytest.mark.parametrize("streams,use_graph", [(1, False), (1, True), (3, True)])
def test_mixed_batch_bit_exact(small, streams, use_graph):
    eng, cts, ops, want = small
    ex = MixedBatchExecutor(eng, cts, ops, streams=streams, use_graph=use_graph)
    for _ in range(2):  # replays read the inputs afresh
        ex.run()
    torch.cuda.synchronize()
    kinds = {op.kind for op in ops}
    assert kinds == {HMULT, ROTATE}
    for i, w in enumerate(want):
        got = ex.result(i)
        assert (got.level, got.scale) == (w.level, w.scale)
        assert torch.equal(got.data, w.data), f"op {i} ({ops[i]}) differs"


@pytest.mark.parametrize("use_graph", [False, True])
def test_items_bit_exact(small, use_graph):
    """Six launches over every level: the same residues as the per-ciphertext loop."""
    eng, cts, ops, want = small
    ex = MixedItemsExecutor(eng, cts, ops, use_graph=use_graph)
    assert ex.launches_per_run == 6 and len(ex.chunks) == 1
    assert ex.chunks[0][0].max_limbs == max(c.limb_count for c in cts)
    for _ in range(2):
        ex.run()
    torch.cuda.synchronize()
    for i, w in enumerate(want):
        got = ex.result(i)
        assert (got.level, got.scale) == (w.level, w.scale)
        assert torch.equal(got.data, w.data), f"op {i} ({ops[i]}) differs"


def test_items_f64_core_matches_integer_core(small):
    """The items' rows of primes below 2^42 run the FP64 key-switch body, the
    others the integer body, in one launch.  With the FP64 core switched off
    every unit runs the integer core: the residues are the same."""
    from fhelium_b200 import _native as nat
    eng, cts, ops, want = small
    ex = MixedItemsExecutor(eng, cts, ops, use_graph=False)
    info = ex.chunks[0][0]
    assert 0 < info.core_f64_units < info.core_units
    try:
        for flag in (0, 1):
            eng.ctx.set_tuning(nat.TUNE_F64_CORE, flag)
            for i in range(len(want)):
                ex._outs[i].zero_()
            ex.run()
            torch.cuda.synchronize()
            assert ex.status() == 0
            for i, w in enumerate(want):
                assert torch.equal(ex.result(i).data, w.data), (flag, i, ops[i])
    finally:
        eng.ctx.set_tuning(nat.TUNE_F64_CORE, 1)


def test_items_work_orders_and_autotune(small, tmp_path):
    """Both key-switch work orders of the items plan give the same residues;
    the autotuner picks among (order, scratch limit) and caches the winner."""
    eng, cts, ops, want = small
    for order in (0, 2):
        ex = MixedItemsExecutor(eng, cts, ops, ks_order=order)
        ex.run()
        torch.cuda.synchronize()
        for i, w in enumerate(want):
            assert torch.equal(ex.result(i).data, w.data), (order, i)
    path = str(tmp_path / "tune.json")
    ex, first = autotune.tune_items(eng, cts, ops, limits=(1 << 28, 1 << 34), repeats=1, cache_path=path)
    assert not first["cached"] and len(first["candidates"]) == 4
    assert (ex.ks_order, ex.max_scratch_bytes) == (first["ks_order"], first["max_scratch_bytes"])
    _, second = autotune.tune_items(eng, cts, ops, cache_path=path)
    assert second["cached"] and second["ks_order"] == first["ks_order"]
    ex.run()
    torch.cuda.synchronize()
    for i, w in enumerate(want):
        assert torch.equal(ex.result(i).data, w.data)


def test_items_chunked(small):
    """A scratch limit below the batch's need splits it into chunks that
    share one scratch, in stream order; the residues do not change."""
    eng, cts, ops, want = small
    one = MixedItemsExecutor(eng, cts, ops, use_graph=False)
    total = int(one.chunks[0][0].scratch_bytes)
    del one
    ex = MixedItemsExecutor(eng, cts, ops, max_scratch_bytes=total // 3)
    assert len(ex.chunks) >= 3 and ex.scratch.numel() <= total // 3 + (64 << 20)
    assert sum(info.items for info, _ in ex.chunks) == ex.count
    ex.run()
    torch.cuda.synchronize()
    for i, w in enumerate(want):
        assert torch.equal(ex.result(i).data, w.data), f"op {i} ({ops[i]}) differs"


def test_items_detect_a_changed_descriptor(small):
    """A descriptor changed in device memory after planning no longer
    matches its check word: every kernel skips that item and the run reports
    status 2; the other items are exact, and restoring the descriptor
    restores the item."""
    eng, cts, ops, want = small
    ex = MixedItemsExecutor(eng, cts, ops, use_graph=False)
    ex.run()
    assert ex.status() == 0
    _, plan = ex.chunks[0]
    victim = ex.chunk_ops[0][0]
    # the device descriptors open the plan, 88 bytes each; bytes 4..7 of the first hold its level
    level = plan[4:8].clone()
    plan[4:8] = (level.view(torch.int32) + 1).view(torch.uint8)
    ex._outs[victim].zero_()
    ex.run()
    assert ex.status() == 2
    assert ex.status() == 0  # reading resets the word
    assert not ex._outs[victim].any()  # the changed item did no work
    for i, w in enumerate(want):
        if i != victim:
            assert torch.equal(ex.result(i).data, w.data), f"op {i} ({ops[i]}) differs"
    plan[4:8] = level
    ex.run()
    assert ex.status() == 0
    assert torch.equal(ex.result(victim).data, want[victim].data)


def test_items_inputs_updated_between_replays(small):
    eng, cts, ops, _ = small
    mine = [c.clone() for c in cts]
    ex = MixedItemsExecutor(eng, mine, ops)
    ex.run()
    first = ex.result(0).data.clone()
    i0 = ops[0].index
    other = next(j for j, c in enumerate(cts) if j != i0 and c.level == cts[i0].level)
    mine[i0].data.copy_(cts[other].data)
    ex.run()
    assert not torch.equal(ex.result(0).data, first)
    mine[i0].data.copy_(cts[i0].data)
    ex.run()
    assert torch.equal(ex.result(0).data, first)


def test_items_rotations_only_and_zero_step(small):
    eng, cts, _, _ = small
    ops = [MixedOp(ROTATE, 0, step=0), MixedOp(ROTATE, 1, step=3), MixedOp(ROTATE, 2, step=-5),
           MixedOp(ROTATE, 3, step=eng.num_slots)]
    ex = MixedItemsExecutor(eng, cts, ops)
    assert ex.launches_per_run == 3 and ex.count == 2
    ex.run()
    want = run_per_ciphertext(eng, cts, ops)
    assert torch.equal(ex.result(0).data, cts[0].data)
    assert torch.equal(ex.result(3).data, cts[3].data)
    for i in (1, 2):
        assert torch.equal(ex.result(i).data, want[i].data)


@pytest.mark.parametrize("preset", [Preset.slots32768_scale40_levels34_int64, Preset.slots16384_scale25_levels29_int32])
def test_items_large_ring_and_int32(preset):
    """logN 16 with 64-bit words, and a 32-bit-word chain (logN 15)."""
    eng = CkksEngine(preset, rng_seed=5)
    count = 10
    cts, ops = _workload(eng, count, seed=21, max_step=1 << 10)
    want = run_per_ciphertext(eng, cts, ops)
    ex = MixedItemsExecutor(eng, cts, ops)
    ex.run()
    torch.cuda.synchronize()
    for i, w in enumerate(want):
        assert torch.equal(ex.result(i).data, w.data), f"op {i} ({ops[i]}) differs"


def test_items_rejects_unaligned_and_bad_level(small):
    from fhelium_b200 import _native as nat
    eng, cts, _, _ = small
    ct = cts[0]
    out = eng._empty(2, ct.limb_count, eng.n)
    key = eng.rotation_key(1)
    good = nat.KsItem(nat.ITEM_ROTATE, ct.level, int(key.galois_element), 0, nat.ptr(ct.data), None,
                      nat.ptr(key.data), nat.ptr(out))
    info = nat.ItemsPlanInfo()
    arr = (nat.KsItem * 1)(good)
    eng.ctx.call("fhb_ckks_items_plan_info", arr, 1, ctypes.byref(info))
    assert info.items == 1 and info.hmult_items == 0 and info.core_units == ct.limb_count + eng.num_p
    for field, value in (("a", nat.ptr(ct.data) + 8), ("level", eng.num_q), ("galois", 2), ("kind", 7)):
        bad = nat.KsItem.from_buffer_copy(good)
        setattr(bad, field, value)
        with pytest.raises(nat.NativeCallError):
            eng.ctx.call("fhb_ckks_items_plan_info", (nat.KsItem * 1)(bad), 1, ctypes.byref(info))


def test_mixed_batch_decrypts(small):
    eng, cts, ops, _ = small
    ex = MixedBatchExecutor(eng, cts, ops, streams=2)
    ex.run()
    for i, op in enumerate(ops[:12]):
        x = eng.decrypt_message(cts[op.index], is_real=True)
        got = eng.decrypt_message(ex.result(i), is_real=True)
        if op.kind == HMULT:
            want = x * eng.decrypt_message(cts[op.partner], is_real=True)
        else:
            want = torch.roll(x, shifts=op.step, dims=-1)
        assert float((got - want).abs().max()) < 2e-5


def test_inputs_updated_between_replays(small):
    eng, cts, ops, _ = small
    mine = [c.clone() for c in cts]
    ex = MixedBatchExecutor(eng, mine, ops, streams=2)
    ex.run()
    first = ex.result(0).data.clone()
    i0 = ops[0].index
    other = next(j for j, c in enumerate(cts) if j != i0 and c.level == cts[i0].level)
    mine[i0].data.copy_(cts[other].data)
    ex.run()
    assert not torch.equal(ex.result(0).data, first)
    mine[i0].data.copy_(cts[i0].data)
    ex.run()
    assert torch.equal(ex.result(0).data, first)


def test_zero_step_is_a_copy(small):
    eng, cts, _, _ = small
    ops = [MixedOp(ROTATE, 0, step=0), MixedOp(ROTATE, 1, step=eng.num_slots), MixedOp(HMULT, 2, partner=2)]
    ex = MixedBatchExecutor(eng, cts, ops, streams=1)
    ex.run()
    assert torch.equal(ex.result(0).data, cts[0].data)
    assert torch.equal(ex.result(1).data, cts[1].data)


def test_rejects_cross_level_partner(small):
    eng, cts, _, _ = small
    a = next(i for i, c in enumerate(cts) if c.level != cts[0].level)
    with pytest.raises(ValueError):
        MixedBatchExecutor(eng, cts, [MixedOp(HMULT, 0, partner=a)])


def test_autotune_picks_and_caches(small, tmp_path):
    eng, cts, ops, want = small
    ex = MixedBatchExecutor(eng, cts, ops, streams=1)
    path = str(tmp_path / "tune.json")
    first = autotune.tune_mixed_batch(eng, ex, streams=(1, 2), repeats=1, cache_path=path)
    # three key-switch work orders x two branch counts
    assert not first["cached"] and len(first["candidates"]) == 6
    assert (ex.streams, ex.ks_order) == (first["streams"], first["ks_order"])
    with open(path) as f:
        assert autotune.workload_key(eng, ex) in json.load(f)
    second = autotune.tune_mixed_batch(eng, ex, streams=(1, 2), repeats=1, cache_path=path)
    assert second["cached"] and second["streams"] == first["streams"]
    ex.run()
    for i, w in enumerate(want):
        assert torch.equal(ex.result(i).data, w.data)


def test_ntt_autotune_sets_and_caches(tmp_path):
    from fhelium_b200 import _native as nat
    eng = CkksEngine(Preset.slots8192_scale40_levels7_int64, rng_seed=2)
    x = torch.randint(0, 1 << 40, (3, eng.num_q, eng.n), dtype=torch.int64, device="cuda")
    path = str(tmp_path / "ntt.json")
    first = autotune.tune_ntt(eng.ctx, x, eng.num_q, cache_path=path, repeats=1)
    assert not first["cached"] and first["forward_ept"] in (8, 16) and first["inverse_ept"] in (8, 16)
    assert eng.ctx.get_tuning(nat.TUNE_NTT_FORWARD_EPT) == first["forward_ept"]
    assert eng.ctx.get_tuning(nat.TUNE_NTT_INVERSE_EPT) == first["inverse_ept"]
    eng.ctx.set_tuning(nat.TUNE_NTT_FORWARD_EPT, 0)
    second = autotune.tune_ntt(eng.ctx, x, eng.num_q, cache_path=path)
    assert second["cached"] and eng.ctx.get_tuning(nat.TUNE_NTT_FORWARD_EPT) == first["forward_ept"]
    # results do not depend on the launch shape
    outs = []
    for ept in (8, 16):
        eng.ctx.set_tuning(nat.TUNE_NTT_FORWARD_EPT, ept)
        outs.append(eng.forward_ntt(x, 0))
    assert torch.equal(outs[0], outs[1])
