"""Host-resident batches streamed through the GPU with copy/compute overlap.

A serving loop whose ciphertexts live in (pinned) host memory pays two PCIe
transfers per operation.  Running the batch as a single device call makes
the three phases strictly sequential: host->device copies, the fused
kernels, device->host copy.  Here the batch is cut into chunks along the
batch axis and the phases of different chunks overlap on three streams:

    copy-in stream   H2D(chunk i+1)      | waits until its staging slot is free
    compute stream   kernels(chunk i)    | waits for H2D(chunk i)
    copy-out stream  D2H(chunk i-1)      | waits for kernels(chunk i-1)

The device input slots are kept on the engine between calls (a ring of
`buffers` slots per chunk shape, each with the event of its last use), and
the copy-in of a chunk waits only for the slot it reuses.  So the copies of
one call also run under the tail of the previous call (its last kernels and
copy-out), and back-to-back calls keep the PCIe link busy.  Outputs are
allocated on the compute stream and handed to the copy-out stream with
record_stream, so the caching allocator never reuses them before their copy
has finished.  Every chunk runs the same engine call (same kernels, same
keys) as the unchunked batch, so the results are identical bit for bit.  The
call returns once the work is queued; the caller's current stream waits for
the last copy-out.

The chunk schedule is a count of equal chunks or an explicit list of chunk
sizes: a few small chunks at the end (see :func:`tapered`) shorten the tail
after the last copy-in, during which only the last chunk's kernels and
copy-out run.
"""

from __future__ import annotations

from typing import Sequence

import torch

from .values import Ciphertext


def _chunks(batch: int, chunks: int | Sequence[int]) -> list[tuple[int, int]]:
    """[start, end) of every chunk: `chunks` equal parts (the first ones one
    longer when they do not divide the batch), or the given sizes in order."""
    if not isinstance(chunks, int):
        sizes = [int(c) for c in chunks]
        if not sizes or min(sizes) < 1 or sum(sizes) != batch:
            raise ValueError(f"chunk sizes {sizes} must be positive and sum to the batch {batch}")
        out, start = [], 0
        for size in sizes:
            out.append((start, start + size))
            start += size
        return out
    chunks = max(1, min(int(chunks), batch))
    base, extra = divmod(batch, chunks)
    out, start = [], 0
    for i in range(chunks):
        size = base + (1 if i < extra else 0)
        out.append((start, start + size))
        start += size
    return out


def tapered(batch: int, width: int, tail: int) -> list[int]:
    """Chunk sizes: `width`-ciphertext chunks, then `tail` chunks of one
    ciphertext (fewer when the batch is smaller)."""
    if width < 1 or tail < 0:
        raise ValueError("need width >= 1 and tail >= 0")
    tail = min(tail, batch)
    head = batch - tail
    sizes = [width] * (head // width)
    if head % width:
        sizes.append(head % width)
    return sizes + [1] * tail


class _Staging:
    """A ring of device input slots (both operands of one chunk) with the
    event of each slot's last use on the compute stream."""

    def __init__(self, shape, dtype, device, buffers: int):
        self.slots = [(torch.empty(shape, dtype=dtype, device=device), torch.empty(shape, dtype=dtype, device=device),
                       torch.cuda.Event()) for _ in range(buffers)]
        self.next = 0

    def take(self):
        slot = self.slots[self.next]
        self.next = (self.next + 1) % len(self.slots)
        return slot


def _staging(engine, shape, dtype, buffers: int) -> _Staging:
    cache = getattr(engine, "_stream_staging", None)
    if cache is None:
        cache = engine._stream_staging = {}
    key = (tuple(shape), dtype, buffers)
    if key not in cache:
        cache.clear()  # one chunk shape at a time: release the slots of another
        cache[key] = _Staging(shape, dtype, engine.device, buffers)
    return cache[key]


def multiply_relinearize_rescale_host(engine, lhs: Ciphertext, rhs: Ciphertext, relinearization_key=None, *,
                                      chunks: int | Sequence[int] = 4, out: torch.Tensor | None = None,
                                      buffers: int = 3) -> Ciphertext:
    """engine.multiply_relinearize_rescale over host-resident operands.

    lhs, rhs: NTT/Montgomery ciphertexts [2, B, L, N] in host memory (pinned
    for asynchronous copies).  chunks: a chunk count or a list of chunk
    sizes; buffers: device input slots in the ring (>= 2).  Returns the
    result as a host ciphertext ([2, B, L - 1, N] coefficient/standard,
    written into `out` when given).
    """
    lhs.assert_state(polynomial_domain="ntt", residue_representation="montgomery", components=2)
    if lhs.data.device.type != "cpu" or rhs.data.device.type != "cpu":
        raise ValueError("operands must be host tensors")
    if lhs.data.shape != rhs.data.shape or lhs.level != rhs.level or lhs.data.dim() != 4:
        raise ValueError("operands must be [2, B, L, N] host ciphertexts of the same shape and level")
    if buffers < 2:
        raise ValueError("need at least two staging buffers")
    dev = engine.device
    key = relinearization_key or engine.relinearization_key
    _, batch, limbs, n = lhs.data.shape
    if out is None:
        out = torch.empty((2, batch, limbs - 1, n), dtype=lhs.data.dtype, pin_memory=True)
    elif out.shape != (2, batch, limbs - 1, n) or out.device.type != "cpu":
        raise ValueError("out must be a host tensor [2, B, L - 1, N]")
    compute = torch.cuda.current_stream(dev)
    streams = getattr(engine, "_copy_streams", None)
    if streams is None:
        streams = engine._copy_streams = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
    copy_in, copy_out = streams
    parts = _chunks(batch, chunks)
    width = max(e - s for s, e in parts)
    staging = _staging(engine, (2, width, limbs, n), lhs.data.dtype, buffers)
    scale = None
    level = lhs.level
    for s, e in parts:
        w = e - s
        buf_a, buf_b, free = staging.take()
        da, db = buf_a[:, :w], buf_b[:, :w]
        copy_in.wait_event(free)  # the slot's last chunk (of this call or an earlier one) is computed
        with torch.cuda.stream(copy_in):
            for c in range(2):
                da[c].copy_(lhs.data[c, s:e], non_blocking=True)
                db[c].copy_(rhs.data[c, s:e], non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(copy_in)
        compute.wait_event(loaded)
        res = engine.multiply_relinearize_rescale(
            Ciphertext(da.contiguous() if w != width else buf_a, level, lhs.scale, "ntt", "montgomery"),
            Ciphertext(db.contiguous() if w != width else buf_b, level, rhs.scale, "ntt", "montgomery"),
            key)
        free.record(compute)
        done = torch.cuda.Event()
        done.record(compute)
        res.data.record_stream(copy_out)
        copy_out.wait_event(done)
        with torch.cuda.stream(copy_out):
            for c in range(2):
                out[c, s:e].copy_(res.data[c], non_blocking=True)
        scale, level_out = res.scale, res.level
    finished = torch.cuda.Event()
    finished.record(copy_out)
    compute.wait_event(finished)
    return Ciphertext(out, level_out, scale, "coefficient", "standard")
