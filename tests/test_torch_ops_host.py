"""Host side of the schema registrations (fhelium_b200.torch_ops), no GPU.

The schemas this library serves must be the reference's own (same names,
argument names and types, mutability annotations), every one of them must get
a CUDA kernel, the indexed-NTT schedule it accepts must be the reference's
radix-2 plan, and operands must be viewed without copies exactly when their
layout allows it."""

import numpy as np
import pytest
import torch

from oracle import ref_pipeline


@pytest.fixture(scope="module")
def torch_ops():
    if ref_pipeline.available():
        torch.ops.load_library(ref_pipeline.REF_LIB)   # schema definitions of the reference itself
    from fhelium_b200 import _native, torch_ops
    try:
        _native.load()
    except _native.NativeLibraryError:
        pytest.skip("libfhb200.so not built")
    torch_ops.register()
    return torch_ops


def test_every_served_schema_has_a_cuda_kernel(torch_ops):
    served = torch_ops.served()
    assert len(served) == 61   # 58 of fhelium_{rns,ntt,ckks}_ops + 3 of fhelium_ntt_diagnostic_ops
    for qualname in served:
        assert torch._C._dispatch_has_kernel_for_dispatch_key(qualname, "CUDA"), qualname
    torch_ops.register()   # idempotent


def test_schemas_are_the_references(torch_ops):
    if not ref_pipeline.available():
        pytest.skip("reference operator library not built")
    # the served names of each namespace are exactly the reference's: a name
    # registered under the wrong namespace would appear here as an extra one
    registered = {}
    for qualname in torch._C._dispatch_get_all_op_names():
        ns, _, name = qualname.partition("::")
        if ns in torch_ops.SCHEMAS:
            registered.setdefault(ns, set()).add(name)
    for ns, ops in torch_ops.SCHEMAS.items():
        assert registered.get(ns) == set(ops), (ns, registered.get(ns, set()) ^ set(ops))
    for ns, ops in torch_ops.SCHEMAS.items():
        for name, schema in ops.items():
            got = str(torch._C._dispatch_find_schema_or_throw(f"{ns}::{name}", "").schema())
            assert got == f"{ns}::{schema}", (got, schema)


@pytest.mark.parametrize("log_n", [4, 10, 12, 16])
def test_radix2_schedule_is_the_references_plan(torch_ops, log_n):
    fe, fo, _, ie, io, _ = ref_pipeline._schedule(log_n)
    e, o = torch_ops._radix2_schedule(log_n, False)
    assert np.array_equal(e, fe.numpy()) and np.array_equal(o, fo.numpy())
    e, o = torch_ops._radix2_schedule(log_n, True)
    assert np.array_equal(e, ie.numpy()) and np.array_equal(o, io.numpy())


def test_operand_views(torch_ops):
    bv = torch_ops._batch_view
    x = torch.zeros(3, 4, 5, 16, dtype=torch.int64)
    assert bv(x) == (12, 80)
    assert bv(x[:, :, 1:]) == (12, 80)            # limb slice: batch stride of the parent
    assert bv(x[:, 1]) == (3, 320)
    assert bv(x[0, 0]) == (1, 80)
    assert bv(x[..., ::2]) is None                 # strided coefficients
    assert bv(x[:, :, ::2]) is None                # rows not N apart
    assert bv(x.transpose(0, 1)) is None           # batch dims that do not collapse
    assert bv(x[:, :, 0], rows_dims=1) == (12, 80)
    assert bv(x[:1].expand(3, -1, -1, -1)) is None   # a broadcast batch (stride 0) is not a view


def test_operand_copy_back(torch_ops):
    x = torch.arange(2 * 3 * 8, dtype=torch.int64).reshape(2, 3, 8)
    t = x.transpose(0, 1)                          # [3, 2, 8]: batch dims do not collapse with rows
    op = torch_ops._Operand(t[:, :, ::2].transpose(0, 1), writable=True)
    assert op.copied
    op.t.zero_()
    op.finish()
    assert int(x[:, :, ::2].abs().sum()) == 0 and int(x[:, :, 1::2].abs().sum()) > 0


def test_find_run(torch_ops):
    chain = (5, 7, 11, 13, 17)
    assert torch_ops._find_run(chain, (11, 13)) == 2
    assert torch_ops._find_run(chain, chain) == 0
    assert torch_ops._find_run(chain, (7, 13)) is None
    assert torch_ops._find_run(chain, (17, 19)) is None


def test_checks_are_remembered_per_tensor_not_per_address(torch_ops):
    x = torch.zeros(8, 10, dtype=torch.int64)
    torch_ops._memo_put(x[:, 2:5], "primes", (1, 2, 3))
    assert torch_ops._memo_get(x[:, 2:5], "primes") == (1, 2, 3)     # another view of the same slice
    assert torch_ops._memo_get(x[:, 2:6], "primes") is None          # another slice
    x.add_(1)
    assert torch_ops._memo_get(x[:, 2:5], "primes") is None          # modified in place
    before = len(torch_ops._memo)
    del x
    import gc
    gc.collect()
    assert len(torch_ops._memo) == before - 1                        # forgotten with the tensor


def test_written_tensor_may_not_overlap_read_only_operands(torch_ops):
    """The reference's check_mutable_rns_output (csrc/ops/common/rns_batch.h:87-97)."""
    x = torch.zeros(2, 5, 8, dtype=torch.int64)
    with pytest.raises(RuntimeError, match="single memory location"):
        torch_ops._no_overlap(x, x)                    # lhs_ and rhs are one tensor
    with pytest.raises(RuntimeError, match="single memory location"):
        torch_ops._no_overlap(x[0], x[0, 1:3])         # dense views over shared bytes
    torch_ops._no_overlap(x[0], x[1])                  # disjoint halves
    torch_ops._no_overlap(x[:, 1:], x[:, 0])           # rows of one tensor (the rescale_ call)
    torch_ops._no_overlap(x, torch.zeros(3))


def test_schedule_checks_raise_the_references_messages(torch_ops):
    """Malformed indexed-NTT schedules fail with the reference's messages
    (tests/test_ntt_backend.py:258-297 of the reference); a valid schedule that
    is not the radix-2 plan is refused by name."""
    log_n = 6
    fe, fo, _, ie, io, _ = ref_pipeline._schedule(log_n)
    torch_ops._check_schedule(fe, fo, log_n, False)
    torch_ops._check_schedule(ie, io, log_n, True)
    with pytest.raises(RuntimeError, match=r"log2\(N\) stages"):
        torch_ops._check_schedule(fe[:-1], fo[:-1], log_n, False)
    bad = fe.clone()
    bad[0, 0] = 1 << log_n
    with pytest.raises(RuntimeError, match="out-of-range coefficient index"):
        torch_ops._check_schedule(bad, fo, log_n, False)
    dup = fe.clone()
    dup[0, 1] = dup[0, 0]
    with pytest.raises(RuntimeError, match="partition every coefficient"):
        torch_ops._check_schedule(dup, fo, log_n, False)
    with pytest.raises(RuntimeError, match="radix-2 indexed schedule only"):
        torch_ops._check_schedule(fo, fe, log_n, False)     # even/odd swapped: a partition, not the plan


def test_ops_refuse_host_tensors(torch_ops):
    x = torch.zeros(1, 2, 16, dtype=torch.int64)
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        torch_ops.montgomery_mul(x, x, torch.zeros(8, 2, dtype=torch.int64))
