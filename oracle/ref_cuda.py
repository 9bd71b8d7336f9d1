"""The reference's own CUDA kernels on this GPU, beside this library.

Test/baseline infrastructure only.  Loads the reference's operator library
built with its CUDA kernels (build_ref_cuda.sh; never together with
libfhelium_ref_cpu_ops.so, which defines the same schemas, and never
together with fhelium_b200.torch_ops, which would register this library's
kernels for them), runs the reference engine's HMult -> relinearize ->
rescale operator sequence (ref_pipeline.ReferenceCpuPipeline, with the
reference's default CUDA NTT policy) on CUDA tensors, and compares it bit
for bit with fhelium_b200's fused HMult + relinearise + rescale on the same
inputs.  Both are timed with CUDA events on the same stream.  Where the two
differ, the reference's own CPU kernels (the same library) are run on the
differing ciphertexts to tell which side left the reference's arithmetic.

    python -m oracle.ref_cuda --batch 32 --steps 3

prints one JSON line.  Inputs: seeded uniform NTT/Montgomery residues for
both ciphertexts (lazy, [0, 2q)) and the relinearisation key at
slots32768_scale40_levels34_int64, level 0.
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from oracle.ref_pipeline import ReferenceCpuPipeline, available  # noqa: E402


def _time(fn, steps: int, stream) -> float:
    for _ in range(2):  # warm-up: kernel attributes, allocator pools
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def run(preset: str, batch: int, steps: int, level: int = 0, seed: int = 7, arbiter: int = 3) -> dict:
    from fhelium_b200.config import CkksConfig
    from fhelium_b200.engine import CkksEngine
    from fhelium_b200.values import Ciphertext, RelinearizationKey

    if not available("cuda"):
        raise FileNotFoundError("oracle/_ref/libfhelium_ref_ops_cuda.so (run oracle/build_ref_cuda.sh)")
    cfg = CkksConfig.parse(preset)
    dev = torch.device("cuda:0")
    ctx = orc.OracleContext(cfg.moduli, cfg.logN, cfg.num_q_primes, cfg.num_p_primes, 62, cfg.scale_bits)
    pipe = ReferenceCpuPipeline(ctx, device=dev, library="cuda", ntt="compact")
    rng = np.random.default_rng(seed)
    q = np.array(cfg.moduli, dtype=np.int64)
    rows = ctx.q_rows(level)

    def uni(shape, rws, bound):
        return torch.from_numpy((rng.integers(0, 1 << 62, size=(*shape, len(rws), cfg.N)) %
                                 (bound * q[rws][:, None])).astype(np.int64)).to(dev)

    a, b = uni((2, batch), rows, 2), uni((2, batch), rows, 2)
    key = uni((len(ctx.digits_at_level(0)), 2), list(range(len(cfg.moduli))), 1)
    stream = torch.cuda.current_stream(dev)
    out = {}

    def ref_step():
        out["ref"] = pipe.multiply_relinearize_rescale(a, b, key, level)

    eng = CkksEngine(cfg, device=dev)
    rlk = RelinearizationKey(key)
    ca = Ciphertext(a, level, 2.0 ** cfg.scale_bits, "ntt", "montgomery")
    cb = Ciphertext(b, level, 2.0 ** cfg.scale_bits, "ntt", "montgomery")
    res = {"preset": preset, "batch": batch, "level": level, "steps": steps,
           "reference_ntt_policy": "radix2_compact_group8_smem8"}
    for form in ("cuda_cores", "tensor_cores"):
        eng.basis_conversion = form

        def ours_step():
            out["ours"] = eng.multiply_relinearize_rescale(ca, cb, rlk)

        ms = _time(ours_step, steps, stream)
        res[f"ours_{form}_ms"] = ms
        res[f"ours_{form}_ops_per_s"] = batch / (ms / 1e3)
        res[f"ours_{form}_bit_exact_vs_reference_cuda"] = None  # filled below
        out[f"ours_{form}"] = out["ours"].data.clone()
    ref_ms = _time(ref_step, steps, stream)
    res["reference_cuda_ms"] = ref_ms
    res["reference_cuda_ops_per_s"] = batch / (ref_ms / 1e3)
    want = out["ref"]
    for form in ("cuda_cores", "tensor_cores"):
        res[f"ours_{form}_bit_exact_vs_reference_cuda"] = bool(torch.equal(out[f"ours_{form}"], want))
        res[f"speedup_{form}"] = ref_ms / res[f"ours_{form}_ms"]
    ours = out["ours_cuda_cores"]
    bad = [i for i in range(batch) if not torch.equal(ours[:, i], want[:, i])]
    res["mismatching_ciphertexts"] = bad
    res["forms_bit_identical"] = bool(torch.equal(out["ours_cuda_cores"], out["ours_tensor_cores"]))
    if bad and arbiter:
        # the reference's own CPU kernels (in the same library) decide, on up
        # to `arbiter` mismatching ciphertexts, which side is off
        cpu = ReferenceCpuPipeline(ctx, device="cpu", library="cuda", ntt="indexed", threads=os.cpu_count())
        verdicts = {}
        for i in bad[:arbiter]:
            ref_cpu = cpu.multiply_relinearize_rescale(a[:, i].cpu(), b[:, i].cpu(), key.cpu(), level)
            diff = ours[:, i] != want[:, i]
            verdicts[str(i)] = {"reference_cpu_equals_ours": bool(torch.equal(ref_cpu, ours[:, i].cpu())),
                                "reference_cpu_equals_reference_cuda": bool(torch.equal(ref_cpu, want[:, i].cpu())),
                                "differing_words": int(diff.sum()),
                                "differing_positions": [[int(c), int(r), int(k)] for c, r, k in
                                                        diff.nonzero().tolist()[:8]]}
        res["arbitrated"] = verdicts
    return res


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--preset", default="slots32768_scale40_levels34_int64")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--arbiter", type=int, default=3, help="mismatching ciphertexts to re-run on the CPU kernels")
    args = ap.parse_args()
    print(json.dumps(run(args.preset, args.batch, args.steps, args.level, arbiter=args.arbiter)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
