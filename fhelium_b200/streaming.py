"""Host-resident batches streamed through the GPU with copy/compute overlap.

A serving loop whose ciphertexts live in (pinned) host memory pays two PCIe
transfers per operation.  Running the batch as a single device call makes
the three phases strictly sequential: host->device copies, the fused
kernels, device->host copy.  Here the batch is cut into chunks along the
batch axis and the phases of different chunks overlap on three streams:

    copy-in stream   H2D(chunk i+1)      | waits until its device buffer is free
    compute stream   kernels(chunk i)    | waits for H2D(chunk i)
    copy-out stream  D2H(chunk i-1)      | waits for kernels(chunk i-1)

Device input buffers are double-buffered; outputs are allocated on the
compute stream and handed to the copy-out stream with record_stream, so the
caching allocator never reuses them before their copy has finished.  Every
chunk runs the same engine call (same kernels, same keys) as the unchunked
batch, so the results are identical bit for bit.  The call returns once the
work is queued; the caller's current stream waits for the last copy-out.
"""

from __future__ import annotations

import torch

from .values import Ciphertext


def _chunks(batch: int, chunks: int) -> list[tuple[int, int]]:
    chunks = max(1, min(int(chunks), batch))
    base, extra = divmod(batch, chunks)
    out, start = [], 0
    for i in range(chunks):
        size = base + (1 if i < extra else 0)
        out.append((start, start + size))
        start += size
    return out


def multiply_relinearize_rescale_host(engine, lhs: Ciphertext, rhs: Ciphertext, relinearization_key=None, *,
                                      chunks: int = 4, out: torch.Tensor | None = None) -> Ciphertext:
    """engine.multiply_relinearize_rescale over host-resident operands.

    lhs, rhs: NTT/Montgomery ciphertexts [2, B, L, N] in host memory (pinned
    for asynchronous copies).  Returns the result as a host ciphertext
    ([2, B, L - 1, N] coefficient/standard, written into `out` when given).
    """
    lhs.assert_state(polynomial_domain="ntt", residue_representation="montgomery", components=2)
    if lhs.data.device.type != "cpu" or rhs.data.device.type != "cpu":
        raise ValueError("operands must be host tensors")
    if lhs.data.shape != rhs.data.shape or lhs.level != rhs.level or lhs.data.dim() != 4:
        raise ValueError("operands must be [2, B, L, N] host ciphertexts of the same shape and level")
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
    bufs = [(torch.empty((2, width, limbs, n), dtype=lhs.data.dtype, device=dev),
             torch.empty((2, width, limbs, n), dtype=lhs.data.dtype, device=dev)) for _ in range(2)]
    free = [torch.cuda.Event(), torch.cuda.Event()]
    start = torch.cuda.Event()
    start.record(compute)
    for ev in free:
        ev.record(compute)
    scale = None
    level = lhs.level
    for i, (s, e) in enumerate(parts):
        w = e - s
        da, db = (t[:, :w] for t in bufs[i % 2])
        copy_in.wait_event(start)
        copy_in.wait_event(free[i % 2])
        with torch.cuda.stream(copy_in):
            for c in range(2):
                da[c].copy_(lhs.data[c, s:e], non_blocking=True)
                db[c].copy_(rhs.data[c, s:e], non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(copy_in)
        compute.wait_event(loaded)
        res = engine.multiply_relinearize_rescale(
            Ciphertext(da.contiguous() if w != width else bufs[i % 2][0], level, lhs.scale, "ntt", "montgomery"),
            Ciphertext(db.contiguous() if w != width else bufs[i % 2][1], level, rhs.scale, "ntt", "montgomery"),
            key)
        free[i % 2].record(compute)
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
