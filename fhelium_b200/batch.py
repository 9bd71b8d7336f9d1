"""Mixed-level batched execution of independent CKKS operations.

A batch of ciphertexts at different levels, each with its own operation
(multiply -> relinearize -> rescale with a same-level partner, or a rotation
by its own step), runs as ONE CUDA graph launch:

* operations are grouped by (kind, level); each group runs as one fused
  launch sequence over all of its items: one forward NTT + the four-launch
  fused HMult/relinearise/rescale for multiplications, and the three-launch
  ``fhb_ckks_rotate_multi`` for rotations, where every item carries its own
  Galois element and key pointer, so mixed steps share one launch;
* groups are spread over ``streams`` capture branches (longest group first
  onto the least loaded branch), so the small levels, which fill only part
  of the 148 SMs, run side by side;
* the whole launch sequence, including the gathers of the inputs into each
  group's contiguous [2, items, limbs, N] arena, is captured once and
  replayed.

The reference runs such a batch as one engine call per ciphertext
(``CkksEngine.multiply``/``relinearize``/``rescale_to_next_level``,
fhelium/engine/ckks_engine.py:1530-1675, and ``rotate_by_step``,
fhelium/engine/ckks_engine.py:2183-2300, 3822-3897).
:func:`run_per_ciphertext` is that loop on this library; both produce the
same residues bit for bit.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _native as nat
from .values import Ciphertext

HMULT = "multiply_relinearize_rescale"
ROTATE = "rotate_by_step"


@dataclass(frozen=True)
class MixedOp:
    """One operation of a mixed batch.

    kind    HMULT or ROTATE
    index   the ciphertext operated on
    partner the same-level right-hand operand (HMULT)
    step    the rotation step (ROTATE)
    """

    kind: str
    index: int
    partner: int = -1
    step: int = 0


def sample_mixed_workload(num_q: int, count: int, *, min_limbs: int = 3, max_limbs: int | None = None,
                          max_step: int = 1 << 14, seed: int = 0) -> tuple[list[int], list[MixedOp]]:
    """Seeded mixed workload: limb counts uniform in [min_limbs, max_limbs]
    (engine level = num_q - limbs) and, per ciphertext, an operation drawn
    uniformly: HMULT with a uniformly drawn same-level partner, or ROTATE by a
    step uniform in +-[1, max_step]."""
    max_limbs = num_q if max_limbs is None else max_limbs
    if not 2 <= min_limbs <= max_limbs <= num_q:
        raise ValueError("need 2 <= min_limbs <= max_limbs <= num_q")
    rng = np.random.default_rng(seed)
    limbs = rng.integers(min_limbs, max_limbs + 1, size=count)
    levels = [int(num_q - x) for x in limbs]
    by_level: dict[int, list[int]] = {}
    for i, lv in enumerate(levels):
        by_level.setdefault(lv, []).append(i)
    ops = []
    kinds = rng.integers(0, 2, size=count)
    for i in range(count):
        if kinds[i] == 0:
            peers = by_level[levels[i]]
            ops.append(MixedOp(HMULT, i, partner=int(peers[rng.integers(0, len(peers))])))
        else:
            magnitude = int(rng.integers(1, max_step + 1))
            ops.append(MixedOp(ROTATE, i, step=magnitude if rng.integers(0, 2) else -magnitude))
    return levels, ops


@dataclass
class _Group:
    kind: str
    level: int
    ops: list[int]  # op indices, in item order
    limbs: int
    stream: int = 0
    inp: torch.Tensor | None = None   # HMULT [2(a|b), 2, B, L, N]; ROTATE [2, B, L, N]
    out: torch.Tensor | None = None   # [2, B, L', N]
    galois: torch.Tensor | None = None  # ROTATE: int32 [B] (device)
    key_ptrs: torch.Tensor | None = None  # ROTATE: int64 [B] (device)
    keys: list = field(default_factory=list)  # keeps the rotation keys alive

    @property
    def items(self) -> int:
        return len(self.ops)

    def cost(self, num_p: int) -> int:
        # key-switch work ~ items x (Q_l + P) x digits; digits grow with limbs
        return self.items * (self.limbs + num_p) * (self.limbs + num_p)


class MixedBatchExecutor:
    """Runs a fixed mixed batch (ciphertexts + ops) as one CUDA graph.

    ciphertexts: coefficient/standard two-component ciphertexts of batch
    size 1, any levels.  ops: one MixedOp per result.  The inputs are read
    in place on every run, so updating their tensors between runs is seen.
    """

    def __init__(self, engine, ciphertexts: Sequence[Ciphertext], ops: Sequence[MixedOp], *,
                 streams: int = 2, ks_order: int | None = None, use_graph: bool = True):
        self.engine = engine
        self.cts = list(ciphertexts)
        self.ops = list(ops)
        self.use_graph = use_graph
        self._validate()
        self._slot: dict[int, tuple[_Group, int]] = {}
        self._copies: set[int] = set()
        self.groups = self._plan()
        self._alloc()
        self._streams: list[torch.cuda.Stream] = []
        self._scratch: list[torch.Tensor] = []
        self._graph: torch.cuda.CUDAGraph | None = None
        self.streams = 0
        self.ks_order = None
        self.configure(streams=streams, ks_order=ks_order)

    # ---------------------------------------------------------------- plan
    def _validate(self) -> None:
        _validate(self.engine, self.cts, self.ops)

    def _plan(self) -> list[_Group]:
        eng = self.engine
        table: dict[tuple[str, int], _Group] = {}
        for i, op in enumerate(self.ops):
            ct = self.cts[op.index]
            if op.kind == ROTATE and eng._canonical_step(op.step) == 0:
                self._copies.add(i)
                continue
            key = (op.kind, ct.level)
            if key not in table:
                table[key] = _Group(op.kind, ct.level, [], ct.limb_count)
            grp = table[key]
            self._slot[i] = (grp, len(grp.ops))
            grp.ops.append(i)
        return sorted(table.values(), key=lambda g: (g.level, g.kind))

    def _alloc(self) -> None:
        eng = self.engine
        n = eng.n
        for g in self.groups:
            b, lm = g.items, g.limbs
            if g.kind == HMULT:
                g.inp = eng._empty(2, 2, b, lm, n)
                g.out = eng._empty(2, b, lm - 1, n)
            else:
                g.inp = eng._empty(2, b, lm, n)
                g.out = eng._empty(2, b, lm, n)
                g.keys = [eng.rotation_key(self.ops[i].step) for i in g.ops]
                g.galois = torch.tensor([k.galois_element for k in g.keys], dtype=torch.int32, device=eng.device)
                g.key_ptrs = torch.tensor([k.data.data_ptr() for k in g.keys], dtype=torch.int64,
                                          device=eng.device)
        self._relin = eng.relinearization_key if any(g.kind == HMULT for g in self.groups) else None

    def configure(self, *, streams: int | None = None, ks_order: int | None = None) -> None:
        """Set the branch count and key-switch work order; drops the graph."""
        eng = self.engine
        if streams is not None:
            if streams < 1:
                raise ValueError("streams must be >= 1")
            self.streams = int(streams)
        if ks_order is not None:
            self.ks_order = int(ks_order)
        self._graph = None
        loads = [0] * self.streams
        for g in sorted(self.groups, key=lambda g: -g.cost(eng.num_p)):
            s = min(range(self.streams), key=lambda i: loads[i])
            g.stream = s
            loads[s] += g.cost(eng.num_p)
        while len(self._streams) < self.streams:
            self._streams.append(torch.cuda.Stream(eng.device))
        need = [0] * self.streams
        for g in self.groups:
            nb = int(eng.ctx.lib.fhb_ckks_keyswitch_scratch_bytes(eng.ctx.handle, g.items, g.level))
            need[g.stream] = max(need[g.stream], nb)
        self._scratch = [torch.empty(max(nb, 16), dtype=torch.uint8, device=eng.device) for nb in need]

    # ---------------------------------------------------------------- run
    def _issue_group(self, g: _Group, stream: torch.cuda.Stream, scratch: torch.Tensor) -> None:
        eng = self.engine
        ctx = eng.ctx
        st = stream.cuda_stream
        with torch.cuda.stream(stream):
            if g.kind == HMULT:
                torch.stack([self.cts[self.ops[i].index].data.view(2, g.limbs, eng.n) for i in g.ops], dim=1,
                            out=g.inp[0])
                torch.stack([self.cts[self.ops[i].partner].data.view(2, g.limbs, eng.n) for i in g.ops], dim=1,
                            out=g.inp[1])
            else:
                torch.stack([self.cts[self.ops[i].index].data.view(2, g.limbs, eng.n) for i in g.ops], dim=1,
                            out=g.inp)
        if g.kind == HMULT:
            ctx.call("fhb_forward_ntt", nat.ptr(g.inp), nat.ptr(g.inp), 4 * g.items, g.limbs, g.level, 0, st)
            ctx.call("fhb_ckks_multiply_relinearize", nat.ptr(g.inp[0]), nat.ptr(g.inp[1]),
                     nat.ptr(self._relin.data), nat.ptr(g.out), nat.ptr(scratch), scratch.numel(), g.items,
                     g.level, 1, st)
        else:
            ctx.call("fhb_ckks_rotate_multi", nat.ptr(g.inp), nat.ptr(g.key_ptrs), nat.ptr(g.galois),
                     nat.ptr(g.out), nat.ptr(scratch), scratch.numel(), g.items, g.level, st)

    def _issue(self) -> None:
        eng = self.engine
        if self.ks_order is not None:
            eng.ctx.call("fhb_context_set_tuning", 0, self.ks_order)
        cur = torch.cuda.current_stream(eng.device)
        branches = self._streams[:self.streams]
        for s in branches:
            s.wait_stream(cur)
        for g in self.groups:
            self._issue_group(g, branches[g.stream], self._scratch[g.stream])
        for s in branches:
            cur.wait_stream(s)

    def capture(self) -> None:
        eng = self.engine
        self._issue()  # first run eagerly: sets kernel attributes outside the capture
        torch.cuda.synchronize(eng.device)
        graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(eng.device)
        cap.wait_stream(torch.cuda.current_stream(eng.device))
        with torch.cuda.graph(graph, stream=cap):
            self._issue()
        torch.cuda.current_stream(eng.device).wait_stream(cap)
        self._graph = graph

    def run(self) -> None:
        """One pass over the whole batch on the current stream."""
        if not self.use_graph:
            self._issue()
            return
        if self._graph is None:
            self.capture()
        self._graph.replay()

    @property
    def launches_per_run(self) -> int:
        """Library kernels one run launches (excluding the input gathers)."""
        return sum(5 if g.kind == HMULT else 3 for g in self.groups)

    # ---------------------------------------------------------------- results
    def result_view(self, op_index: int) -> torch.Tensor:
        """[2, limbs, N] view of op `op_index`'s result inside its group arena."""
        if op_index in self._copies:
            return self.cts[self.ops[op_index].index].data.view(2, -1, self.engine.n)
        g, j = self._slot[op_index]
        return g.out[:, j]

    def result(self, op_index: int) -> Ciphertext:
        return _result(self, op_index)

    def results(self) -> list[Ciphertext]:
        return [self.result(i) for i in range(len(self.ops))]


class MixedItemsExecutor:
    """A fixed mixed batch as six library launches, whatever its levels.

    Every ciphertext's operation becomes one item descriptor (level, Galois
    element, operand, key and output addresses) in a device plan, and each
    stage of the key switch (forward NTT of the HMult operands, tensor
    product, inverse NTT of d2, ModUp digits, key-switch core, ModDown) is
    ONE launch over all items, with work lists that map clusters to
    (item, row) units.  The operands are read in place (no gathers), so
    updating the ciphertexts' tensors between runs is seen.  Every item in
    flight holds its own scratch (ModUp digits, two Q_l P accumulators, and
    for HMult the operands' NTTs and ct3), so a batch whose scratch would
    pass ``max_scratch_bytes`` runs as several such six-launch chunks in
    stream order over one shared scratch.  Results are integer-equal to
    :class:`MixedBatchExecutor` and to :func:`run_per_ciphertext`.
    """

    def __init__(self, engine, ciphertexts: Sequence[Ciphertext], ops: Sequence[MixedOp], *,
                 use_graph: bool = True, max_scratch_bytes: int = 8 << 30, ks_order: int | None = None):
        self.engine = engine
        self.cts = list(ciphertexts)
        self.ops = list(ops)
        self.use_graph = use_graph
        self.max_scratch_bytes = int(max_scratch_bytes)
        self.ks_order = ks_order
        _validate(engine, self.cts, self.ops)
        eng = engine
        self._copies: set[int] = set()
        self._outs: dict[int, torch.Tensor] = {}
        self._keys = []
        items, item_ops = [], []
        relin = None
        for i, op in enumerate(self.ops):
            ct = self.cts[op.index]
            if not ct.data.is_contiguous():
                raise ValueError(f"op {op}: ciphertext storage must be contiguous")
            if op.kind == ROTATE and eng._canonical_step(op.step) == 0:
                self._copies.add(i)
                continue
            if op.kind == HMULT:
                relin = relin if relin is not None else eng.relinearization_key
                out = eng._empty(2, ct.limb_count - 1, eng.n)
                b = self.cts[op.partner].data
                if not b.is_contiguous():
                    raise ValueError(f"op {op}: partner storage must be contiguous")
                items.append(nat.KsItem(nat.ITEM_HMULT_RELIN_RESCALE, ct.level, 1, 0, nat.ptr(ct.data),
                                        nat.ptr(b), nat.ptr(relin.data), nat.ptr(out)))
                item_ops.append(i)
            else:
                key = eng.rotation_key(op.step)
                self._keys.append(key)
                out = eng._empty(2, ct.limb_count, eng.n)
                items.append(nat.KsItem(nat.ITEM_ROTATE, ct.level, int(key.galois_element), 0, nat.ptr(ct.data),
                                        None, nat.ptr(key.data), nat.ptr(out)))
                item_ops.append(i)
            self._outs[i] = out
        self._relin = relin
        self._graph: torch.cuda.CUDAGraph | None = None
        self.count = len(items)
        self.chunks: list[tuple[nat.ItemsPlanInfo, torch.Tensor]] = []
        self.chunk_ops: list[list[int]] = []  # op index of every item of each chunk, in plan order
        if self.count == 0:
            return
        ctx = eng.ctx

        def plan_info(batch):
            info = nat.ItemsPlanInfo()
            ctx.call("fhb_ckks_items_plan_info", (nat.KsItem * len(batch))(*batch), len(batch), ctypes.byref(info))
            return info

        # Items of one level (and key) side by side; chunks cut where the
        # scratch of the items in flight would pass max_scratch_bytes.
        order = sorted(range(self.count), key=lambda j: (items[j].level, items[j].kind, items[j].key or 0))
        sizes = {j: int(plan_info([items[j]]).scratch_bytes) for j in order}
        parts, cur, used = [], [], 0
        for j in order:
            if cur and used + sizes[j] > max_scratch_bytes:
                parts.append(cur)
                cur, used = [], 0
            cur.append(j)
            used += sizes[j]
        parts.append(cur)
        self.chunk_ops = [[item_ops[j] for j in part] for part in parts]
        parts = [[items[j] for j in part] for part in parts]
        infos = [plan_info(part) for part in parts]
        self.scratch = torch.empty(max(max(int(i.scratch_bytes) for i in infos), 16), dtype=torch.uint8,
                                   device=eng.device)
        # the plans' key-switch work lists follow the context's work order
        keep = ctx.get_tuning(nat.TUNE_KS_ORDER)
        if ks_order is not None:
            ctx.set_tuning(nat.TUNE_KS_ORDER, int(ks_order))
        try:
            for part, info in zip(parts, infos):
                plan = torch.empty(max(int(info.plan_bytes), 16), dtype=torch.uint8, device=eng.device)
                ctx.call("fhb_ckks_items_plan", (nat.KsItem * len(part))(*part), len(part), nat.ptr(plan),
                         nat.ptr(self.scratch), ctypes.byref(info))
                self.chunks.append((info, plan))
        finally:
            ctx.set_tuning(nat.TUNE_KS_ORDER, keep)

    def _issue(self) -> None:
        eng = self.engine
        st = torch.cuda.current_stream(eng.device).cuda_stream
        for info, plan in self.chunks:  # in stream order: the chunks share one scratch
            eng.ctx.call("fhb_ckks_items_run", nat.ptr(plan), ctypes.byref(info), st)

    def capture(self) -> None:
        eng = self.engine
        self._issue()  # first run eagerly: sets kernel attributes outside the capture
        torch.cuda.synchronize(eng.device)
        graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(eng.device)
        cap.wait_stream(torch.cuda.current_stream(eng.device))
        with torch.cuda.graph(graph, stream=cap):
            self._issue()
        torch.cuda.current_stream(eng.device).wait_stream(cap)
        self._graph = graph

    def run(self) -> None:
        """One pass over the whole batch on the current stream."""
        if not self.use_graph:
            self._issue()
            return
        if self._graph is None:
            self.capture()
        self._graph.replay()

    @property
    def launches_per_run(self) -> int:
        """Library kernels one run launches."""
        return sum(6 if info.hmult_items else 3 for info, _ in self.chunks)

    def status(self) -> int:
        """First error the kernels raised since the last call (0: none), after
        waiting for the device; see fhb_ckks_items_status for the codes."""
        torch.cuda.synchronize(self.engine.device)
        worst = 0
        for info, plan in self.chunks:
            word = ctypes.c_int(0)
            self.engine.ctx.call("fhb_ckks_items_status", nat.ptr(plan), ctypes.byref(info), ctypes.byref(word))
            worst = worst or int(word.value)
        return worst

    def result_view(self, op_index: int) -> torch.Tensor:
        """[2, limbs, N] view of op `op_index`'s result."""
        if op_index in self._copies:
            return self.cts[self.ops[op_index].index].data.view(2, -1, self.engine.n)
        return self._outs[op_index]

    def result(self, op_index: int) -> Ciphertext:
        return _result(self, op_index)

    def results(self) -> list[Ciphertext]:
        return [self.result(i) for i in range(len(self.ops))]


def _validate(eng, cts: Sequence[Ciphertext], ops: Sequence[MixedOp]) -> None:
    for ct in cts:
        ct.assert_state(polynomial_domain="coefficient", residue_representation="standard", components=2)
        eng._check_ct(ct)
        if ct.batch_size != 1:
            raise ValueError("mixed batches take ciphertexts of batch size 1")
    for op in ops:
        if not 0 <= op.index < len(cts):
            raise ValueError(f"op {op} refers to a missing ciphertext")
        if op.kind == HMULT:
            if not 0 <= op.partner < len(cts):
                raise ValueError(f"op {op} has no partner")
            a, b = cts[op.index], cts[op.partner]
            if a.level != b.level:
                raise ValueError(f"op {op}: partner is at another level")
            if a.limb_count < 2:
                raise ValueError(f"op {op}: no level left to rescale into")
        elif op.kind != ROTATE:
            raise ValueError(f"unknown op kind {op.kind!r}")


def _result(ex, op_index: int) -> Ciphertext:
    eng = ex.engine
    op = ex.ops[op_index]
    ct = ex.cts[op.index]
    data = ex.result_view(op_index).contiguous().view(2, *ct.batch_shape, -1, eng.n)
    if op_index in ex._copies:
        return Ciphertext(data, ct.level, ct.scale, "coefficient", "standard")
    if op.kind == HMULT:
        scale = eng.rescale_to_next_output_scale(ct.scale * ex.cts[op.partner].scale, level=ct.level)
        return Ciphertext(data, ct.level + 1, scale, "coefficient", "standard")
    return Ciphertext(data, ct.level, ct.scale, "coefficient", "standard")


def run_per_ciphertext(engine, ciphertexts: Sequence[Ciphertext], ops: Sequence[MixedOp]) -> list[Ciphertext]:
    """The unbatched form: one engine call sequence per operation, exactly as
    a caller of the reference engine issues them."""
    out = []
    for op in ops:
        a = ciphertexts[op.index]
        if op.kind == HMULT:
            b = ciphertexts[op.partner]
            out.append(engine.multiply_relinearize_rescale(engine.coefficient_domain_to_ntt_domain(a),
                                                           engine.coefficient_domain_to_ntt_domain(b)))
        else:
            out.append(engine.rotate_by_step(a, op.step))
    return out
