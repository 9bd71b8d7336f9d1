"""Host logic of the mixed-level batch path (no GPU): the seeded workload
sampler and the autotuner's result cache."""

import json

import pytest

from fhelium_b200 import autotune
from fhelium_b200.batch import HMULT, ROTATE, sample_mixed_workload


def test_workload_is_seeded_and_well_formed():
    levels, ops = sample_mixed_workload(35, 512, seed=7)
    again = sample_mixed_workload(35, 512, seed=7)
    assert (levels, ops) == again
    assert sample_mixed_workload(35, 512, seed=8) != (levels, ops)
    limbs = [35 - lv for lv in levels]
    assert min(limbs) >= 3 and max(limbs) <= 35
    assert len(set(limbs)) == 33  # every limb count 3..35 drawn at this size
    kinds = [op.kind for op in ops]
    assert 0.4 < kinds.count(HMULT) / len(ops) < 0.6
    for i, op in enumerate(ops):
        assert op.index == i
        if op.kind == HMULT:
            assert levels[op.partner] == levels[i]
        else:
            assert op.kind == ROTATE
            assert 1 <= abs(op.step) <= 1 << 14
    assert any(op.step < 0 for op in ops) and any(op.step > 0 for op in ops)


def test_workload_rejects_bad_ranges():
    with pytest.raises(ValueError):
        sample_mixed_workload(8, 4, min_limbs=1)
    with pytest.raises(ValueError):
        sample_mixed_workload(8, 4, max_limbs=9)


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "sub" / "tune.json")
    assert autotune._load(path) == {}
    autotune._store(path, "a", {"ks_order": 1, "streams": 2, "ms": 3.0})
    autotune._store(path, "b", {"ks_order": 0, "streams": 1, "ms": 4.0})
    data = autotune._load(path)
    assert data["a"]["streams"] == 2 and data["b"]["ks_order"] == 0
    with open(path, "w") as f:
        f.write("not json")
    assert autotune._load(path) == {}
    json.dumps(autotune.default_cache_path())


def test_streaming_chunks_cover_the_batch():
    from fhelium_b200.streaming import _chunks, tapered
    assert _chunks(7, 3) == [(0, 3), (3, 5), (5, 7)]
    assert _chunks(2, 5) == [(0, 1), (1, 2)]
    assert _chunks(32, 4) == [(0, 8), (8, 16), (16, 24), (24, 32)]
    assert _chunks(5, [2, 2, 1]) == [(0, 2), (2, 4), (4, 5)]
    for bad in ([2, 2], [3, 0, 2], []):
        with pytest.raises(ValueError):
            _chunks(5, bad)
    assert tapered(32, 2, 4) == [2] * 14 + [1] * 4
    assert tapered(7, 4, 2) == [4, 1, 1, 1]
    assert tapered(3, 2, 5) == [1, 1, 1]
    assert sum(tapered(33, 4, 3)) == 33
