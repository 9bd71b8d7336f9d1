"""Benchmark: CKKS HMult + relinearize + rescale throughput at logN=16, L=35.

Workload (one step): 32 top-level ciphertext pairs of preset
slots32768_scale40_levels34_int64 (N = 2^16, 35 Q primes + 4 P primes,
dnum = 10 hybrid digits), each encrypting float64 messages uniform in
[-0.05, 0.05] (seed 2 + rank), multiplied, relinearised with the
relinearisation key and rescaled - the whole batch per step.

  value       ops/s with the inputs resident in HBM (device time, CUDA events,
              max over ranks); the batch (2.35 GB of inputs) is larger than
              L2 (126 MB), so every step streams from HBM.
  e2e         the same metric through the public API with the inputs in pinned
              host memory: per step the host->device copy of both input
              ciphertext batches and the device->host copy of the result are
              inside the timed region.
  roofline    the dominant kernel (fused key-switch core) timed alone with
              CUDA events on its launch stream: algorithmic bytes per launch /
              duration against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own CPU operators (compiled from its sources
              into oracle/_ref) driven in the reference engine's order, on a
              bounded sample (a few ciphertexts) with all host threads.
  gpu_baseline  the reference's own CUDA kernels (compiled from its sources
              for sm_100a into oracle/_ref) driven in the same order on this
              GPU, on the whole batch, in a child process.

Multi-GPU (torchrun): every rank runs the same per-GPU batch on its own
ciphertexts (independent objects, no collective on the data path);
`value` = all ranks' ops / max-over-ranks time ("scaling": "weak").

`--impl reference` times the reference CPU implementation (the same
operators) on this workload's config and prints its own JSON line.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PRESET = "slots32768_scale40_levels34_int64"
KS_TRAFFIC_BYTES_BATCH32 = 12741399552 + 2934590720  # ncu dram read + write, k_keyswitch_core, batch 32 (profiles/)
# same for the key-switch core of the tensor-core form: captured at batch 8 (3094038784 + 705889536 bytes,
# 2.01x the batch-4 capture) and scaled by the ciphertexts processed
KS_EXT_TRAFFIC_BYTES_BATCH32 = 4 * (3094038784 + 705889536)
# the CUDA-core form's core with its FP64 rows (k_keyswitch_core_split<false>, the extension computed in FP64 in
# the core, the default for this chain): captured at batch 8 (3810678272 + 360568320 bytes; every destination row
# re-reads its group's digit rows and the group's key rows, so the traffic grows with the batch) and scaled by the
# ciphertexts processed
KS_SPLIT_TRAFFIC_BYTES_BATCH32 = 4 * (3810678272 + 360568320)
# the tensor-core form's core with its FP64 rows (k_keyswitch_core_split<PRE>): captured at batch 8 (3085136640 + 355092224
# bytes; the key and digit rows are re-read per group of four ciphertexts, so the traffic grows with the batch)
# and scaled by the ciphertexts processed
KS_F64_TRAFFIC_BYTES_BATCH32 = 4 * (3085136640 + 355092224)
METRIC = "hmult_relin_rescale_ops_per_s_logN16_L35"
UNIT = "ops/s"
CONFIG = {
    "workload": "HMult+relinearize+rescale, preset slots32768_scale40_levels34_int64 "
                "(logN=16, L=35 Q + 4 P primes, dnum=10), batch of top-level ciphertext pairs",
    "logN": 16, "limbs": 35, "special_primes": 4, "dnum": 10,
    "l2_policy": "inputs larger than L2 (2.35 GB per step at batch 32)",
}


def _dist():
    from fhelium_b200 import ranks
    return ranks.init()


def _barrier(ws):
    from fhelium_b200 import ranks
    ranks.barrier(ws)


def _max_over_ranks(x: float, ws: int, device) -> float:
    from fhelium_b200 import ranks
    return ranks.max_over_ranks(x, ws, device)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _messages(batch, slots, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.rand((batch, slots), dtype=torch.float64, generator=g) * 0.1 - 0.05


def _time_events(fn, steps, stream):
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end) / steps


def _int8_peak_tops() -> tuple[float, str]:
    """Dense int8 tensor peak: twice the measured dense bf16 GEMM rate (the
    B200's dense int8 rate is twice its bf16 rate), else twice the bf16
    fallback."""
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return 2.0 * float(peaks["bf16_tflops"]), "2 x measured bf16 burst"
    except Exception:
        return 2.0 * 1590.0, "2 x fallback bf16"


def ntt_int32_primes(count: int = 36, log_n: int = 16) -> list[int]:
    from fhelium_b200.config import int32_ntt_primes
    return int32_ntt_primes(count, log_n)


def ntt_leg(dev, stream, steps):
    """Standalone forward + inverse NTT: N = 2^16, 36 int32 limbs, batch 64,
    residues uniform in [0, q_i) (seed 1).  Timed with the default launch
    shape (8 residues per thread) and with the autotuner's pick; the round
    trip is checked bit-exact under both."""
    from fhelium_b200 import _native as nat
    from fhelium_b200 import autotune
    primes = ntt_int32_primes()
    ctx = nat.NativeContext(32, 16, primes, len(primes) - 1, 1, dev)
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    B, L, N = 64, len(primes), 1 << 16
    q = torch.tensor(primes, dtype=torch.int64, device=dev).view(1, L, 1)
    x = (torch.randint(0, 1 << 62, (B, L, N), generator=g, device=dev, dtype=torch.int64) % q).to(torch.int32)
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    s = stream.cuda_stream
    fwd = lambda: nat.check(ctx.lib.fhb_forward_ntt(ctx.handle, x.data_ptr(), y.data_ptr(), B, L, 0, 0, s), "ntt")
    inv = lambda: nat.check(ctx.lib.fhb_inverse_ntt(ctx.handle, y.data_ptr(), z.data_ptr(), B, L, 0, 2, s), "intt")
    nbytes = 2 * B * L * N * 4  # read + write per direction
    for _ in range(3):  # warm-up (clocks, caches, kernel attributes)
        fwd()
        inv()
    torch.cuda.synchronize(dev)
    out = {}
    for tag in ("plain", "tuned"):
        if tag == "tuned":
            tune = autotune.tune_ntt(ctx, x, L, use_cache=False)
            out["autotune"] = {k: tune[k] for k in ("forward_ept", "inverse_ept", "candidates")}
        fwd_ms = _time_events(fwd, max(3, steps), stream)
        inv_ms = _time_events(inv, max(3, steps), stream)
        out[tag] = {"forward_ms": fwd_ms, "inverse_ms": inv_ms, "roundtrip_bit_exact": bool(torch.equal(x, z)),
                    "forward_gbs": nbytes / (fwd_ms / 1e3) / 1e9, "inverse_gbs": nbytes / (inv_ms / 1e3) / 1e9,
                    "limb_ntts_per_s": 2 * B * L / ((fwd_ms + inv_ms) / 1e3)}
        z.zero_()
        fwd()
        inv()
        out[tag]["roundtrip_bit_exact"] = bool(torch.equal(x, z))
    # exact int8 tensor-core form: passes of 64 x 64 x 16 points per
    # direction over 4 x 4 byte-digit products; 2 N (n1 + n2 + n3) d_a d_b
    # int8 operations per limb-polynomial and direction.  Default launch form:
    # three passes, each reading and writing every residue once (3 HBM round
    # trips per direction); the form with the 16-point pass fused into the
    # adjacent 64-point pass (2 round trips) is timed beside it
    tc = {}
    nat.check(ctx.lib.fhb_tc_ntt_prepare(ctx.handle), "tc prepare")
    tfwd = lambda: nat.check(ctx.lib.fhb_tc_forward_ntt(ctx.handle, x.data_ptr(), y.data_ptr(), B, L, 0, s), "tc ntt")
    tinv = lambda: nat.check(ctx.lib.fhb_tc_inverse_ntt(ctx.handle, y.data_ptr(), z.data_ptr(), B, L, 0, s), "tc intt")
    ctx.set_tuning(nat.TUNE_TC_NTT_FUSED, 1)
    for _ in range(3):
        tfwd()
        tinv()
    fused = {"forward_ms": _time_events(tfwd, max(3, steps), stream),
             "inverse_ms": _time_events(tinv, max(3, steps), stream)}
    z.zero_()
    tfwd()
    tinv()
    fused["roundtrip_bit_exact"] = bool(torch.equal(x, z))
    y_fused = y.clone()
    ctx.set_tuning(nat.TUNE_TC_NTT_FUSED, 0)
    for _ in range(3):
        tfwd()
        tinv()
    tc["forward_ms"] = _time_events(tfwd, max(3, steps), stream)
    tc["inverse_ms"] = _time_events(tinv, max(3, steps), stream)
    tfwd()
    fused["forward_equals_three_pass"] = bool(torch.equal(y, y_fused))
    tc["fused_passes"] = fused
    del y_fused
    y_tc = torch.empty_like(x)
    nat.check(ctx.lib.fhb_tc_forward_ntt(ctx.handle, x.data_ptr(), y_tc.data_ptr(), B, L, 0, s), "tc ntt")
    fwd()  # CUDA-core forward into y
    tc["forward_equals_plain_mod_q"] = bool(torch.equal(y_tc.to(torch.int64), y.to(torch.int64) % q))
    z.zero_()
    nat.check(ctx.lib.fhb_tc_inverse_ntt(ctx.handle, y.data_ptr(), z.data_ptr(), B, L, 0, s), "tc intt")
    tc["inverse_of_plain_bit_exact"] = bool(torch.equal(x, z))
    z.zero_()
    nat.check(ctx.lib.fhb_tc_inverse_ntt(ctx.handle, y_tc.data_ptr(), z.data_ptr(), B, L, 0, s), "tc intt")
    tc["roundtrip_bit_exact"] = bool(torch.equal(x, z))
    flag = ctypes.c_int(-1)
    nat.check(ctx.lib.fhb_tc_ntt_status(ctx.handle, ctypes.byref(flag)), "tc status")
    tc["wait_timeouts"] = flag.value
    int8_ops = B * L * 2 * N * (64 + 64 + 16) * 4 * 4
    int8_peak, src = _int8_peak_tops()
    tc["int8_tops_forward"] = int8_ops / (tc["forward_ms"] / 1e3) / 1e12
    tc["int8_tops_inverse"] = int8_ops / (tc["inverse_ms"] / 1e3) / 1e12
    tc["int8_peak_tops"] = int8_peak
    tc["int8_peak_source"] = src
    tc["tensor_frac_forward"] = tc["int8_tops_forward"] / int8_peak
    tc["tensor_frac_inverse"] = tc["int8_tops_inverse"] / int8_peak
    tc["forward_gbs"] = nbytes / (tc["forward_ms"] / 1e3) / 1e9
    tc["inverse_gbs"] = nbytes / (tc["inverse_ms"] / 1e3) / 1e9
    # the passes' own HBM traffic (3 x read + write of every residue) against
    # the measured copy bandwidth
    try:
        hbm = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        hbm = 6650.0
    tc["pass_traffic_gbs_forward"] = 3 * nbytes / (tc["forward_ms"] / 1e3) / 1e9
    tc["pass_traffic_gbs_inverse"] = 3 * nbytes / (tc["inverse_ms"] / 1e3) / 1e9
    tc["hbm_frac_forward"] = tc["pass_traffic_gbs_forward"] / hbm
    tc["hbm_frac_inverse"] = tc["pass_traffic_gbs_inverse"] / hbm
    out["tensor_core"] = tc
    # integer-pipe roof: Shoup products per transform (N/2 log N butterflies
    # + the N x R or x N^-1 pass) against the int32 probe's rate
    probe_out = torch.empty(148 * 8 * 256, dtype=torch.int32, device=dev)
    probe = lambda: nat.check(ctx.lib.fhb_modmul_probe(ctx.handle, probe_out.data_ptr(), 148 * 8, 2048, s), "probe")
    probe()
    torch.cuda.synchronize(dev)
    peak = 148 * 8 * 256 * 8 * 2048 / (min(_time_events(probe, 3, stream) for _ in range(3)) / 1e3)
    per_dir = B * L * (N // 2 * 16 + N)
    out["alu_roofline"] = {"unit": "modular products/s", "peak": peak,
                           "forward_frac": per_dir / (out["tuned"]["forward_ms"] / 1e3) / peak,
                           "inverse_frac": per_dir / (out["tuned"]["inverse_ms"] / 1e3) / peak}
    ctx.close()
    return out


def bootstrap_leg(dev, stream, batch=8, steps=2):
    """Full-slot bootstrap of `batch` ciphertexts, preset
    slots32768_scale50_levels27_int64 + base_prime_bits=50, generator 5,
    slots with real and imaginary parts uniform in [-1, 1] (seed 4)."""
    import math
    from fhelium_b200.bootstrap import FullSlotBootstrap
    from fhelium_b200.config import CkksConfig
    from fhelium_b200.engine import CkksEngine
    cfg = CkksConfig.parse("slots32768_scale50_levels27_int64", base_prime_bits=50)
    eng = CkksEngine(cfg, device=dev, galois_generator=5, rng_seed=5)
    bs = FullSlotBootstrap(eng)
    t0 = time.perf_counter()
    bs.generate_keys()
    bs.precompute()
    torch.cuda.synchronize(dev)
    setup_s = time.perf_counter() - t0
    g = torch.Generator().manual_seed(4)
    n = eng.num_slots
    m = (torch.rand((batch, n), dtype=torch.float64, generator=g) * 2 - 1) \
        + 1j * (torch.rand((batch, n), dtype=torch.float64, generator=g) * 2 - 1)
    ct = eng.encrypt_message(m, level=eng.public_level_count - 1)
    state = {}

    def step():
        state["out"] = bs(ct)

    out = {"batch": batch, "setup_s": setup_s, "rotation_keys": len(bs.rotation_steps())}
    # the key switches' basis conversion on the CUDA cores, then on the int8
    # tensor cores (the default reported above the per-form figures)
    results = {}
    for form in ("cuda_cores", "tensor_cores"):
        eng.basis_conversion = form
        step()
        torch.cuda.synchronize(dev)
        ms = _time_events(step, steps, stream)
        err = (eng.decrypt_message(state["out"]) - m).abs()
        results[form] = state["out"].data.clone()
        out[form] = {"ms_per_call": ms, "ms_per_bootstrap": ms / batch, "bootstraps_per_s": batch / (ms / 1e3),
                     "output_level": state["out"].level, "max_abs_err": float(err.max()),
                     "mean_abs_err": float(err.mean()), "precision_bits": -math.log2(float(err.max()))}
    out.update(out["tensor_cores"])
    out["forms_bit_identical"] = bool(torch.equal(results["cuda_cores"], results["tensor_cores"]))
    out["tensor_cores_over_cuda_cores_latency"] = out["cuda_cores"]["ms_per_call"] / out["tensor_cores"]["ms_per_call"]
    del bs, eng, ct, state
    torch.cuda.empty_cache()
    return out


def ops_leg(dev, stream, batch=2, steps=3):
    """Every evaluation op of the path once per step at logN=16, L=35 on
    `batch` ciphertexts (a small case for per-kernel profiles): fused
    HMult+relin+rescale, relinearize of an NTT-domain product, rescale,
    rotation by one step, 4 hoisted rotations, forward and inverse NTT of a
    ciphertext.  Returns per-op CUDA-event milliseconds."""
    from fhelium_b200.engine import CkksEngine
    eng = CkksEngine(PRESET, device=dev, rng_seed=11)
    x = _messages(batch, eng.num_slots, 5)
    ct = eng.encrypt_message(x)
    ca = eng.coefficient_domain_to_ntt_domain(ct)
    steps4 = [1, 2, 3, 4]
    eng.generate_rotation_keys(steps4)
    ct3 = eng.multiply(ca, ca)
    # BSGS inner products as in a bootstrap transform group: 16 baby
    # rotations x 4 giant steps over 64 diagonal plaintexts
    g16 = torch.Generator(device=dev)
    g16.manual_seed(7)
    qcol = torch.tensor(eng.moduli[:eng.num_q], dtype=torch.int64, device=dev).view(-1, 1)
    rot = torch.randint(0, 1 << 62, (16, *ca.data.shape), generator=g16, device=dev) % qcol
    pts = torch.randint(0, 1 << 62, (64, eng.num_q, eng.n), generator=g16, device=dev) % qcol
    table = torch.arange(64, dtype=torch.int32, device=dev).view(4, 16)
    inner = torch.empty((4, *ca.data.shape), dtype=torch.int64, device=dev)

    def bsgs():
        eng.ctx.call("fhb_ckks_bsgs_inner_product", rot.data_ptr(), rot[0].numel(), pts.data_ptr(), pts[0].numel(),
                     64, table.data_ptr(), 4, 16, inner.data_ptr(), inner[0].numel(), 2 * batch, eng.num_q, 0,
                     stream.cuda_stream)

    ops = {
        "bsgs_inner_product_16x4": bsgs,
        "multiply_relinearize_rescale": lambda: eng.multiply_relinearize_rescale(ca, ca),
        "relinearize": lambda: eng.relinearize(ct3),
        "rescale": lambda: eng.rescale_to_next_level(ct),
        "rotate": lambda: eng.rotate_by_step(ct, 1),
        "hoisted_rotations_4": lambda: eng.rotate_many_by_steps(ct, steps4),
        "forward_ntt": lambda: eng.coefficient_domain_to_ntt_domain(ct),
        "inverse_ntt": lambda: eng.ntt_domain_to_coefficient_domain(ca),
    }
    out = {}
    for name, fn in ops.items():
        fn()
        torch.cuda.synchronize(dev)
        out[name + "_ms"] = _time_events(fn, max(1, steps), stream)
    return {"batch": batch, **out}


def schema_ops_leg(eng, x, y, kd, stream, steps=5):
    """The operator-level kernels behind the reference's custom-op schemas
    (fhb_op_*, served to torch.ops.fhelium_* by fhelium_b200.torch_ops), timed
    through the C ABI at the headline shape: 32 ciphertexts at L = 35, N = 2^16,
    int64, P = 4.  x, y: [B, L, N] residues; kd: one key digit [2, QP, N].
    Algorithmic bytes = every operand read once and every output written once;
    reported against the measured HBM copy bandwidth."""
    from fhelium_b200 import _native as nat
    lib, s = eng.ctx.lib, stream.cuda_stream
    n, L, P = eng.n, eng.num_q, eng.num_p
    QP = L + P
    B = x.size(0)
    word = 8 if eng.dtype == torch.int64 else 4
    prm = eng._param_rows
    try:
        hbm = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        hbm = 6650.0
    g = torch.Generator(device=x.device).manual_seed(5)
    rnd = lambda *shape: torch.randint(0, 1 << 40, shape, generator=g, device=x.device, dtype=eng.dtype)
    out = torch.empty_like(x)
    acc0, acc1, digit = torch.zeros(B, QP, n, dtype=eng.dtype, device=x.device), \
        torch.zeros(B, QP, n, dtype=eng.dtype, device=x.device), rnd(B, QP, n)
    inv_md, inv_rs = rnd(P, QP), rnd(L - 1)
    md_out = torch.empty(B, L, n, dtype=eng.dtype, device=x.device)
    ext_out, ext_coef = torch.empty(B, QP, n, dtype=eng.dtype, device=x.device), rnd(3, QP)
    rs_out = torch.empty(B, L - 1, n, dtype=eng.dtype, device=x.device)
    bits = 64 if eng.dtype == torch.int64 else 32
    P_ = nat.ptr
    cases = {
        "montgomery_mul": (lambda: lib.fhb_op_rns_binary(bits, 0, P_(x), L * n, P_(y), L * n, P_(out), L * n, B, L, n,
                                                           P_(prm), prm.stride(0), s),
                           3 * B * L * n * word),
        "keyswitch_accumulate_digit_products_": (
            lambda: lib.fhb_op_keyswitch_accumulate(bits, P_(acc0), QP * n, P_(acc1), QP * n, P_(digit), QP * n,
                                                    P_(kd), QP * n, 0, B, QP, n, P_(prm), prm.stride(0), s),
            (5 * B * QP + 2 * QP) * n * word),
        "keyswitch_moddown_qp_to_q": (
            lambda: lib.fhb_op_moddown(bits, P_(digit), QP * n, P_(digit[:, L:]), QP * n, P_(md_out), L * n, B, L, P,
                                       n, P_(inv_md), QP, P_(prm), prm.stride(0), s),
            (B * QP + B * L) * n * word),
        "mixed_radix_basis_extend_to_montgomery": (
            lambda: lib.fhb_op_basis_extend(bits, P_(x), L * n, 4, P_(ext_out), QP * n, B, QP, n, P_(ext_coef), QP,
                                            P_(prm), prm.stride(0), s),
            (B * 4 + B * QP) * n * word),
        "rescale_drop_leading_prime_nearest": (
            lambda: lib.fhb_op_rescale(bits, P_(x[:, 1:]), L * n, P_(x[:, 0]), L * n, P_(rs_out), (L - 1) * n, B,
                                       L - 1, n, P_(inv_rs), P_(prm[:, 1:]), prm.stride(0), eng.moduli[0] // 2, 1, s),
            (B * L + B * (L - 1)) * n * word),
    }
    res = {"shape": f"batch {B}, L = {L}, P = {P}, N = {n}, {bits}-bit words", "hbm_peak_gbs": hbm}
    for name, (fn, nbytes) in cases.items():
        nat.check(fn(), name)
        torch.cuda.synchronize(x.device)
        ms = _time_events(lambda: nat.check(fn(), name), steps, stream)
        res[name] = {"ms": ms, "gbs": nbytes / ms / 1e6, "hbm_frac": nbytes / ms / 1e6 / hbm,
                     "algorithmic_bytes": nbytes}
    return res


def forms_leg(eng, ca, cb, rlk, stream, steps=5):
    """The key switch with its basis conversion on the CUDA cores and on the
    int8 tensor cores, same inputs: HMult+relin+rescale, single rotation and
    16 hoisted rotations (ops/s), and the bit identity of their outputs."""
    out, results = {}, {}
    keep = eng.basis_conversion
    eng.generate_rotation_keys(list(range(1, 17)))
    # warm both forms up first (kernel loading, scratch, clocks), then time each
    for form in ("cuda_cores", "tensor_cores"):
        eng.basis_conversion = form
        for _ in range(2):
            eng.rotate_by_step(eng.multiply_relinearize_rescale(ca, cb, rlk), 1)
    torch.cuda.synchronize()
    # three interleaved rounds (the forms alternate which goes first), the
    # best time of each form and operation, so that drift over the leg does
    # not favour one form
    best: dict = {}
    for rnd in range(3):
        for form in (("cuda_cores", "tensor_cores") if rnd % 2 == 0 else ("tensor_cores", "cuda_cores")):
            eng.basis_conversion = form
            r = eng.multiply_relinearize_rescale(ca, cb, rlk)
            torch.cuda.synchronize()
            ms = _time_events(lambda: eng.multiply_relinearize_rescale(ca, cb, rlk), steps, stream)
            rot = eng.rotate_by_step(r, 1)
            torch.cuda.synchronize()
            rms = _time_events(lambda: eng.rotate_by_step(r, 1), steps, stream)
            hoisted = eng.rotate_many_by_steps(r, list(range(1, 17)))
            torch.cuda.synchronize()
            hms = _time_events(lambda: eng.rotate_many_by_steps(r, list(range(1, 17))), max(2, steps // 2), stream)
            if rnd == 0:
                results[form] = (r.data.clone(), rot.data.clone(), torch.stack([h.data for h in hoisted]))
            b = best.setdefault(form, [ms, rms, hms])
            best[form] = [min(x, y) for x, y in zip(b, (ms, rms, hms))]
    for form, (ms, rms, hms) in best.items():
        out[form] = {"hmult_relin_rescale_ops_per_s": ca.batch_size / (ms / 1000.0), "hmult_relin_rescale_ms": ms,
                     "rotate_ops_per_s": ca.batch_size / (rms / 1000.0),
                     "hoisted_rotations_16_ops_per_s": 16 * ca.batch_size / (hms / 1000.0)}
    a, b = results["cuda_cores"], results["tensor_cores"]
    out["bit_identical"] = all(bool(torch.equal(x, y)) for x, y in zip(a, b))
    # variant of the tensor-core form, HMult+relin+rescale only: ModDown on
    # the tensor cores too
    import fhelium_b200._native as nat
    eng.basis_conversion = "tensor_cores"
    variants = {}
    # and the key-switch core's Q rows on the integer pipe instead of FP64
    for name, param, value in (("tc_moddown", nat.TUNE_TC_MODDOWN, 1), ("integer_core", nat.TUNE_F64_CORE, 0)):
        keep_v = eng.ctx.get_tuning(param)
        eng.ctx.set_tuning(param, value)
        r = eng.multiply_relinearize_rescale(ca, cb, rlk)
        torch.cuda.synchronize()
        ms = _time_events(lambda: eng.multiply_relinearize_rescale(ca, cb, rlk), steps, stream)
        variants[name] = {"hmult_relin_rescale_ops_per_s": ca.batch_size / (ms / 1000.0),
                          "bit_identical": bool(torch.equal(r.data, a[0]))}
        eng.ctx.set_tuning(param, keep_v)
    out["tensor_cores_variants"] = variants
    out["tensor_cores_over_cuda_cores"] = {
        k: out["tensor_cores"][k] / out["cuda_cores"][k]
        for k in ("hmult_relin_rescale_ops_per_s", "rotate_ops_per_s", "hoisted_rotations_16_ops_per_s")}
    eng.basis_conversion = keep
    return out


def mixed_batch_leg(dev, stream, count=512, steps=3):
    """Mixed-level batch at slots32768_scale40_levels34_int64: `count`
    ciphertexts with limb counts uniform in 3..35 (uniform [-0.05, 0.05]
    messages), each with a seeded op (HMult+relin+rescale with a same-level
    partner, or a rotation by a step uniform in +-[1, 2^14]).  Three forms,
    every result compared bit for bit with one engine call sequence per
    ciphertext: the descriptor-driven items path (six launches per chunk of
    items, whatever their levels), the per-(kind, level) group graph (knobs
    from the autotuner), and the per-ciphertext loop itself.  The rotation
    keys (one per distinct step, about 0.4 GB each) dominate the memory."""
    from fhelium_b200 import autotune
    from fhelium_b200.batch import HMULT, MixedBatchExecutor, run_per_ciphertext, sample_mixed_workload
    from fhelium_b200.engine import CkksEngine
    # the CUDA-core form, as the items path's own key switch: the group
    # executor's scratch then holds no extensions (the keys leave little room)
    eng = CkksEngine(PRESET, device=dev, rng_seed=9, basis_conversion="cuda_cores")
    levels, ops = sample_mixed_workload(eng.num_q, count, seed=0)
    msgs = _messages(count, eng.num_slots, 3)
    cts = [eng.encrypt_message(msgs[i], level=lv) for i, lv in enumerate(levels)]
    t0 = time.perf_counter()
    for op in ops:
        if op.kind != HMULT:
            eng.rotation_key(op.step)
    torch.cuda.synchronize(dev)
    keygen_s = time.perf_counter() - t0
    def mismatches(ex):
        bad = 0
        for i, op in enumerate(ops):
            want = run_per_ciphertext(eng, cts, [op])[0].data.view(2, -1, eng.n)
            bad += int(not torch.equal(ex.result_view(i), want))
        return bad

    # one executor alive at a time: the keys leave little room for two
    items, items_tune = autotune.tune_items(eng, cts, ops, limits=(4 << 30, 8 << 30))
    items.run()
    torch.cuda.synchronize(dev)
    items_ms = _time_events(items.run, max(3, steps), stream)
    bad = {"items": mismatches(items)}
    item_chunks, item_launches = len(items.chunks), items.launches_per_run
    peak_gb = {"items": torch.cuda.max_memory_allocated(dev) / 1e9}
    del items
    torch.cuda.empty_cache()
    ex = MixedBatchExecutor(eng, cts, ops)
    tune = autotune.tune_mixed_batch(eng, ex, ks_orders=(0, 1), streams=(1, 2, 4), repeats=2)
    torch.cuda.empty_cache()
    ex.run()
    torch.cuda.synchronize(dev)
    batched_ms = _time_events(ex.run, max(3, steps), stream)
    bad["groups"] = mismatches(ex)
    groups, group_launches = len(ex.groups), ex.launches_per_run
    peak_gb["groups"] = torch.cuda.max_memory_allocated(dev) / 1e9
    del ex
    torch.cuda.empty_cache()

    def per_ct():
        run_per_ciphertext(eng, cts, ops)

    per_ct()
    torch.cuda.synchronize(dev)
    loop_ms = _time_events(per_ct, 2, stream)
    n_rot = sum(1 for op in ops if op.kind != HMULT)
    best = min(items_ms, batched_ms)
    out = {"ciphertexts": count, "hmult_ops": count - n_rot, "rotate_ops": n_rot,
           "distinct_rotation_keys": len({eng._canonical_step(op.step) for op in ops if op.kind != HMULT}),
           "basis_conversion": eng.basis_conversion,
           "items_ms": items_ms, "items_ops_per_s": count / (items_ms / 1e3), "items_chunks": item_chunks,
           "items_library_launches_per_pass": item_launches,
           "items_autotune": {"ks_order": items_tune["ks_order"], "max_scratch_bytes": items_tune["max_scratch_bytes"],
                              "cached": items_tune["cached"], "candidates": items_tune.get("candidates")},
           "groups": groups, "library_launches_per_pass": group_launches,
           "batched_graph_ms": batched_ms, "batched_ops_per_s": count / (batched_ms / 1e3),
           "per_ciphertext_ms": loop_ms, "per_ciphertext_ops_per_s": count / (loop_ms / 1e3),
           "speedup": loop_ms / best, "items_over_groups": batched_ms / items_ms,
           "bit_exact_mismatches": bad, "peak_allocated_gb": peak_gb,
           "autotune": {"ks_order": tune["ks_order"], "streams": tune["streams"], "cached": tune["cached"],
                        "candidates": tune.get("candidates")},
           "keygen_s": keygen_s}
    del cts, eng
    torch.cuda.empty_cache()
    return out


def gpu_reference_sample(batch: int, steps: int = 5):
    """The reference's own CUDA kernels (oracle/_ref, built from its sources
    for sm_100a) running its engine's HMult -> relinearize -> rescale
    operator sequence on the same GPU, batch `batch` at level 0 of the
    headline preset, timed with CUDA events.  A child process: that library
    defines the reference's operator schemas itself."""
    import subprocess
    from oracle.ref_pipeline import available
    if not available("cuda"):
        return None
    cmd = [sys.executable, "-m", "oracle.ref_cuda", "--batch", str(batch), "--steps", str(steps), "--arbiter", "0"]
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    if res.returncode != 0:
        return {"error": res.stderr.strip().splitlines()[-1][:300] if res.stderr.strip() else "failed"}
    line = json.loads(res.stdout.strip().splitlines()[-1])
    return {"value": line["reference_cuda_ops_per_s"], "unit": UNIT, "kind": "reference",
            "ms_per_step": line["reference_cuda_ms"],
            "sample": f"its engine's operator sequence through its CUDA kernels ({line['reference_ntt_policy']} NTT), "
                      f"batch {batch}, level 0, same GPU; this library in the same process: "
                      f"{line['ours_tensor_cores_ops_per_s']:.1f} ops/s",
            "ciphertexts_equal": batch - len(line["mismatching_ciphertexts"]), "batch": batch}


def cpu_reference_sample(n_ops: int, threads: int, level: int = 0):
    """Time the reference CPU operators on `n_ops` HMult+relin+rescale ops
    (one ciphertext pair each).  Returns (ops/s, kind, sample text)."""
    from fhelium_b200.config import CkksConfig
    from oracle import oracle as orc
    from oracle.ref_pipeline import ReferenceCpuPipeline, available
    cfg = CkksConfig.parse(PRESET)
    ctx = orc.OracleContext(cfg.moduli, cfg.logN, cfg.num_q_primes, cfg.num_p_primes, 62, cfg.scale_bits)
    rng = np.random.default_rng(5)
    rows = ctx.q_rows(level)
    q = np.array(cfg.moduli, dtype=np.int64)

    def uni(shape, rws, bound=1):
        return (rng.integers(0, 1 << 62, size=(*shape, len(rws), cfg.N)) % (bound * q[rws][:, None])).astype(np.int64)

    key = uni((len(ctx.digits_at_level(0)), 2), list(range(len(cfg.moduli))))
    a, b = uni((2,), rows, 2), uni((2,), rows, 2)
    if available():
        pipe = ReferenceCpuPipeline(ctx, threads=threads)
        ta, tb, tk = (torch.from_numpy(x) for x in (a, b, key))
        pipe.multiply_relinearize_rescale(ta, tb, tk, level)  # warm-up
        t0 = time.perf_counter()
        for _ in range(n_ops):
            pipe.multiply_relinearize_rescale(ta, tb, tk, level)
        dt = time.perf_counter() - t0
        return n_ops / dt, "reference", threads, f"{n_ops} ops of one ciphertext pair at L=35 (reference CPU operators)"
    # the oracle port (single thread C restatement)
    t0 = time.perf_counter()
    ctx.rescale(ctx.relinearize(ctx.multiply(a, b, level), key, level), level)
    dt = time.perf_counter() - t0
    return 1 / dt, "port", 1, "1 op of one ciphertext pair at L=35 (oracle C restatement)"


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    per_step = []
    for _ in range(args.warmup):
        cpu_reference_sample(1, threads)
    for _ in range(args.steps):
        v, kind, cores, sample = cpu_reference_sample(2, threads)
        per_step.append(v)
    value = statistics.median(per_step)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": dict(CONFIG, batch=1, parallelism="host threads"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-extras", action="store_true", help="skip rotation/parity/CPU legs")
    ap.add_argument("--mixed-count", type=int, default=512, help="ciphertexts of the mixed-level leg (0: skip)")
    ap.add_argument("--basis", choices=["auto", "cuda_cores", "tensor_cores"], default="auto",
                    help="where the key switch's basis conversion runs in the headline step (auto: the "
                         "engine's default for the chain)")
    ap.add_argument("--leg", choices=["ntt_int32", "bootstrap", "mixed", "ops", "schema", "forms"], default=None,
                    help="run only this side leg on one GPU and print its result (profiling aid)")
    args = ap.parse_args()
    ws, rank, local = _dist()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.leg is not None:
        dev = torch.device("cuda", local)
        torch.cuda.set_device(dev)
        stream = torch.cuda.current_stream(dev)
        if args.leg == "ntt_int32":
            res = ntt_leg(dev, stream, args.steps)
        elif args.leg == "bootstrap":
            res = bootstrap_leg(dev, stream, steps=max(1, args.steps))
        elif args.leg == "ops":
            res = ops_leg(dev, stream, batch=args.batch, steps=args.steps)
        elif args.leg == "schema":
            from fhelium_b200.config import Preset
            from fhelium_b200.engine import CkksEngine
            eng = CkksEngine(Preset.slots32768_scale40_levels34_int64, device=dev)
            q = torch.tensor(eng.moduli, dtype=torch.int64, device=dev)[:, None]
            g = torch.Generator(device=dev).manual_seed(9)
            rows = lambda b, r: (torch.randint(0, 1 << 62, (b, r, eng.n), generator=g, device=dev) % q[:r])
            x, y = rows(args.batch, eng.num_q), rows(args.batch, eng.num_q)
            kd = rows(2, eng.num_q + eng.num_p)
            res = schema_ops_leg(eng, x, y, kd, stream, steps=max(1, args.steps))
        elif args.leg == "forms":
            from fhelium_b200.engine import CkksEngine
            eng = CkksEngine(PRESET, device=dev, rng_seed=7)
            ca = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(_messages(args.batch, eng.num_slots, 2)))
            cb = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(_messages(args.batch, eng.num_slots, 3)))
            res = forms_leg(eng, ca, cb, eng.relinearization_key, stream, steps=max(2, args.steps))
        else:
            res = mixed_batch_leg(dev, stream, args.mixed_count, args.steps)
        print(json.dumps({"leg": args.leg, **res}), flush=True)
        return 0

    from fhelium_b200 import _native as nat
    from fhelium_b200.config import CkksConfig
    from fhelium_b200.engine import CkksEngine

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg = CkksConfig.parse(PRESET)
    eng = CkksEngine(cfg, device=dev, rng_seed=1234 + rank, basis_conversion=args.basis)
    form = eng.basis_conversion  # the resolved form
    B = args.batch
    x = _messages(B, eng.num_slots, 2 + 2 * rank)
    y = _messages(B, eng.num_slots, 3 + 2 * rank)
    ca = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(x))
    cb = eng.coefficient_domain_to_ntt_domain(eng.encrypt_message(y))
    rlk = eng.relinearization_key
    stream = torch.cuda.current_stream(dev)

    state = {}

    def step():
        state["out"] = eng.multiply_relinearize_rescale(ca, cb, rlk)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        _barrier(ws)
        torch.cuda.synchronize(dev)
        ms = _time_events(step, args.steps, stream)
        torch.cuda.synchronize(dev)
        _barrier(ws)
    ms = _max_over_ranks(ms, ws, dev)
    from fhelium_b200 import ranks
    value = ranks.job_rate(B, ws, ms)
    # tensor product, INTT of c2, ModUp digits, (tensor-core basis extension,) key-switch core, ModDown+rescale
    # (the tensor-core form's core is two launches when its Q rows run in FP64:
    # the P rows stay on the integer kernel)
    f64_core = bool(eng.ctx.get_tuning(nat.TUNE_F64_CORE))
    # tensor product, inverse NTT of d2, ModUp digits, (tensor-core extension,) core, ModDown; the FP64 rows of
    # the NTT and of the core share their launches with the integer rows
    # per chunk of the overlapped call (batches of 16 or more run in up to FHB_TUNE_OVERLAP_CHUNKS chunks)
    chunks_per_step = max(1, min(int(eng.ctx.get_tuning(nat.TUNE_OVERLAP_CHUNKS)), B // 8))
    launches_per_step = (6 if form == "tensor_cores" else 5) * (chunks_per_step if chunks_per_step > 1 else 1)

    # ---- end to end through the public API with host buffers -------------
    host_a = ca.data.cpu().pin_memory()
    host_b = cb.data.cpu().pin_memory()
    out_host = torch.empty((2, B, cfg.num_q_primes - 1, cfg.N), dtype=torch.int64).pin_memory()
    from fhelium_b200.values import Ciphertext

    from fhelium_b200.streaming import multiply_relinearize_rescale_host, tapered
    ha = Ciphertext(host_a, 0, ca.scale, "ntt", "montgomery")
    hb = Ciphertext(host_b, 0, cb.scale, "ntt", "montgomery")
    e2e_chunks = {"chunks": 1, "buffers": 3}

    def e2e_step():
        # host batch streamed through the GPU: copy-in, kernels and copy-out
        # of successive chunks overlap on three streams, and the copy-in of a
        # step runs under the previous step's last kernels and copy-out
        multiply_relinearize_rescale_host(eng, ha, hb, rlk, chunks=e2e_chunks["chunks"], out=out_host,
                                          buffers=e2e_chunks["buffers"])

    # as many steps as the device-timed value, so the pipeline's fill and
    # drain are spread the same way
    e2e_steps = max(3, args.steps)
    # chunk schedules x staging slots, picked on untimed passes: equal
    # chunks, or chunks of 2-3 ciphertexts ending in single-ciphertext chunks
    schedules = {str(c): min(c, B) for c in (1, 4, 8, 16, 32)}
    for width, tail in ((2, 2), (3, 2), (4, 2), (8, 4)):
        schedules[f"{width}x..+1x{tail}"] = tapered(B, width, tail)
    trial = {}
    for name, chunks in schedules.items():
        for buffers in (3, 4):
            e2e_chunks.update(chunks=chunks, buffers=buffers)
            e2e_step()
            torch.cuda.synchronize(dev)
            trial[f"{name}/{buffers}"] = _time_events(e2e_step, 2, stream)
    best = min(trial, key=trial.get)
    e2e_chunks.update(chunks=schedules[best.split("/")[0]], buffers=int(best.split("/")[1]))
    torch.cuda.synchronize(dev)
    _barrier(ws)
    e2e_ms = _time_events(e2e_step, e2e_steps, stream)
    e2e_ms = _max_over_ranks(e2e_ms, ws, dev)
    h2d = host_a.numel() * 8 + host_b.numel() * 8
    d2h = out_host.numel() * 8

    # ---- dominant kernel alone: fused key-switch core --------------------
    lib, h = eng.ctx.lib, eng.ctx.handle
    L = cfg.num_q_primes
    coef = torch.empty((3, B, L, cfg.N), dtype=torch.int64, device=dev)
    digits = torch.empty((B, L, cfg.N), dtype=torch.int64, device=dev)
    t = torch.empty((2, B, L + cfg.num_p_primes, cfg.N), dtype=torch.int64, device=dev)
    s = stream.cuda_stream
    kernels = {
        "mul_to_coefficient": lambda: lib.fhb_ckks_multiply_to_coefficient(h, nat.ptr(ca.data), nat.ptr(cb.data),
                                                                             nat.ptr(coef), B, 0, s),
        "modup_digits": lambda: lib.fhb_ckks_modup_digits(h, nat.ptr(coef[2]), nat.ptr(digits), B, 0, 1, s),
        "keyswitch_core": lambda: lib.fhb_ckks_keyswitch_core(h, nat.ptr(digits), nat.ptr(rlk.data), nat.ptr(t[0]),
                                                              nat.ptr(t[1]), B, 0, s),
        "moddown_rescale": lambda: lib.fhb_ckks_moddown(h, nat.ptr(t[0]), nat.ptr(t[1]), nat.ptr(coef[0]),
                                                        nat.ptr(coef[1]), nat.ptr(state["out"].data), B, 0, 1, 1, s),
        # the two launches the fused step uses before ModUp: NTT-domain tensor
        # product, then d2 alone to the coefficient domain
        "tensor_product": lambda: lib.fhb_ckks_multiply(h, nat.ptr(ca.data), nat.ptr(cb.data), nat.ptr(coef), B, 0, s),
        "inverse_ntt_d2": lambda: lib.fhb_inverse_ntt(h, nat.ptr(coef[2]), nat.ptr(digits), B, L, 0, 2, s),
    }
    ext = None
    if form == "tensor_cores":
        # the tensor-core form's two key-switch kernels
        ext = torch.empty(int(lib.fhb_tc_basis_extend_words(h, B, 0)), dtype=torch.int64, device=dev)
        kernels["tc_basis_extend"] = lambda: lib.fhb_tc_basis_extend(h, nat.ptr(digits), nat.ptr(ext), B, 0, s)
        kernels["keyswitch_core_extended"] = lambda: lib.fhb_ckks_keyswitch_core_extended(
            h, nat.ptr(ext), nat.ptr(rlk.data), nat.ptr(t[0]), nat.ptr(t[1]), B, 0, s)
    per_kernel = {}
    for name, fn in kernels.items():
        fn()
        torch.cuda.synchronize(dev)
        per_kernel[name] = _time_events(fn, max(2, min(args.steps, 5)), stream)
    mib = 1 << 20
    limb = cfg.N * 8
    ks_bytes = B * (L + 2 * (L + cfg.num_p_primes)) * limb + 10 * 2 * (L + cfg.num_p_primes) * limb
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = ks_bytes / (per_kernel["keyswitch_core"] / 1000.0) / 1e9
    # The key-switch core is bound by 64-bit modular products on the integer
    # pipes, so it is also measured against their attainable rate: modular
    # products per launch (Shoup butterflies of 10 forward and 2 inverse
    # transforms per row, the basis extension's sum_r alpha_r = L Shoup
    # products per digit row, 2 Montgomery key products per digit, the N^-1
    # epilogue) over the probe's rate of independent Shoup chains.
    n_, logn_ = cfg.N, cfg.logN
    dnum_ = len(eng.level_digits[0])
    bfly_ = n_ // 2 * logn_
    qp_ = L + cfg.num_p_primes
    ks_modmul = B * qp_ * (dnum_ * bfly_ + L * n_ + 2 * dnum_ * n_ + 2 * (bfly_ + n_))
    probe_out = torch.empty(148 * 8 * 256, dtype=torch.int64, device=dev)
    probe_iters = 2048
    probe = lambda: nat.check(lib.fhb_modmul_probe(h, probe_out.data_ptr(), 148 * 8, probe_iters, s), "probe")
    probe()
    torch.cuda.synchronize(dev)
    # a peak: the best of three timings (each of three launches)
    probe_ms = min(_time_events(probe, 3, stream) for _ in range(3))
    modmul_peak = 148 * 8 * 256 * 8 * probe_iters / (probe_ms / 1000.0)
    # the FP64 rows' balanced product, probed the same way; the key-switch
    # core's attainable rate is the row-weighted mix of the two
    f64_rows = 0
    probe_f64_ms = None
    if f64_core:
        probe_f64 = torch.empty(148 * 8 * 256, dtype=torch.float64, device=dev)
        probe64 = lambda: nat.check(lib.fhb_modmul_probe_f64(h, probe_f64.data_ptr(), 148 * 8, probe_iters, s),
                                    "probe f64")
        probe64()
        torch.cuda.synchronize(dev)
        probe_f64_ms = min(_time_events(probe64, 3, stream) for _ in range(3))
        modmul_peak_f64 = 148 * 8 * 256 * 8 * probe_iters / (probe_f64_ms / 1000.0)
        f64_rows = sum(1 for q in cfg.q_moduli if int(q) < (1 << 42))
    else:
        modmul_peak_f64 = None

    def mixed_peak(share):
        """attainable modular-product rate of a kernel running `share` of its rows in FP64"""
        return 1.0 / (share / modmul_peak_f64 + (1.0 - share) / modmul_peak) if modmul_peak_f64 else modmul_peak

    ks_peak = mixed_peak(f64_rows / (L + cfg.num_p_primes))
    # kernels whose rows of primes below 2^42 run in FP64, and their FP64 share
    f64_share = {"inverse_ntt_d2": f64_rows / L, "keyswitch_core": f64_rows / (L + cfg.num_p_primes),
                 "keyswitch_core_extended": f64_rows / (L + cfg.num_p_primes)}
    modmul_achieved = ks_modmul / (per_kernel["keyswitch_core"] / 1000.0)
    step_bytes = B * (4 * L + 2 * (L - 1)) * limb + 10 * 2 * (L + cfg.num_p_primes) * limb
    # every step kernel against its roofs: algorithmic bytes (each operand row
    # read once, each output row written once, keys once per launch) over the
    # measured copy bandwidth, and for the transform / basis-conversion
    # kernels the modular products per launch over the probe's rate
    P_ = cfg.num_p_primes
    rows = lambda r: B * r * limb
    kroof = {
        "tensor_product": (rows(7 * L), 0),
        "inverse_ntt_d2": (rows(2 * L), B * L * (bfly_ + n_)),
        "mul_to_coefficient": (rows(7 * L), B * L * (4 * n_ + 3 * (bfly_ + n_))),
        "modup_digits": (rows(2 * L), B * n_ * sum(len(d) * (len(d) + 1) // 2 for _, d in eng.level_digits[0])),
        "keyswitch_core": (ks_bytes, ks_modmul),
        "moddown_rescale": (rows(2 * (L + P_) + 2 * L + 2 * (L - 1)),
                            2 * B * n_ * (P_ * (P_ + 1) // 2 + L * (P_ + 2))),
    }
    int8_ops = {}
    if ext is not None:
        nd_ = len(eng.level_digits[0])
        ext_rows = nd_ * (L + P_)
        # basis extension: digit rows read once, every extension row written once;
        # int8 MMA work: per 128 coefficients and 16-row chunk 2 x 128 x N x 32
        chunk_n = [min(16, L + P_ - 16 * c) * 8 for c in range((L + P_ + 15) // 16)]
        int8_ops["tc_basis_extend"] = nd_ * B * (n_ // 128) * sum(2 * 128 * ((c + 15) // 16 * 16) * 32
                                                                  for c in chunk_n)
        kroof["tc_basis_extend"] = (rows(L) + rows(ext_rows), 0)
        kroof["keyswitch_core_extended"] = (rows(ext_rows) + rows(2 * (L + P_)) + 2 * dnum_ * (L + P_) * limb,
                                            ks_modmul - B * qp_ * L * n_)
    int8_peak, int8_src = _int8_peak_tops()
    kernel_roofline = {}
    for name, (nbytes, nmul) in kroof.items():
        sec = per_kernel[name] / 1000.0
        entry = {"ms": per_kernel[name], "algorithmic_bytes": nbytes, "hbm_gbs": nbytes / sec / 1e9,
                 "hbm_frac": nbytes / sec / 1e9 / peak}
        if nmul:
            kpeak = mixed_peak(f64_share.get(name, 0.0))
            entry.update({"modmul": nmul, "modmul_per_s": nmul / sec, "modmul_frac": nmul / sec / kpeak})
        entry["bound"] = "hbm" if not nmul or entry["hbm_frac"] > entry["modmul_frac"] else "integer"
        if name in int8_ops:
            entry.update({"int8_ops": int8_ops[name], "int8_tops": int8_ops[name] / sec / 1e12,
                          "int8_frac": int8_ops[name] / sec / 1e12 / int8_peak, "int8_peak_source": int8_src})
        kernel_roofline[name] = entry
    # DRAM bytes of one k_keyswitch_core launch: 15.7 GB measured by ncu
    # (dram__bytes_read.sum + dram__bytes_write.sum) on the batch-32 launch of
    # this command, work order 2 (groups of four ciphertexts share the key
    # rows); every destination row re-reads the digit rows of its group, so
    # the traffic grows with the batch and is scaled by the units processed.
    traffic = KS_TRAFFIC_BYTES_BATCH32 * B / 32 if cfg.logN == 16 and L == 35 else None
    # the dominant kernel of the headline form
    dom = "keyswitch_core_extended" if ext is not None else "keyswitch_core"
    dom_kernel = {"keyswitch_core": ("k_keyswitch_core_split<false> (FP64 rows for the primes below 2^42 with the "
                                     "extension computed in FP64, int64 rows for the base prime and P)"
                                     if f64_core else "k_keyswitch_core"),
                  "keyswitch_core_extended": ("k_keyswitch_core_split<PRE> (FP64 rows for the primes below 2^42, "
                                              "int64 rows for the base prime and P)"
                                              if f64_core else "k_keyswitch_core<PRE>")}[dom]
    if dom == "keyswitch_core_extended":
        ext_traffic = KS_F64_TRAFFIC_BYTES_BATCH32 if f64_core else KS_EXT_TRAFFIC_BYTES_BATCH32
        traffic = ext_traffic * B / 32 if ext_traffic and cfg.logN == 16 and L == 35 else None
    elif f64_core:
        traffic = (KS_SPLIT_TRAFFIC_BYTES_BATCH32 * B / 32
                   if KS_SPLIT_TRAFFIC_BYTES_BATCH32 and cfg.logN == 16 and L == 35 else None)
    dom_bytes, dom_modmul = kroof[dom]
    achieved = dom_bytes / (per_kernel[dom] / 1000.0) / 1e9
    modmul_achieved = dom_modmul / (per_kernel[dom] / 1000.0)

    extras = {}
    if not args.no_extras:
        # unfused reference-order path: multiply, relinearize, rescale separately
        def plain_step():
            state["plain"] = eng.rescale_to_next_level(eng.relinearize(eng.multiply(ca, cb), rlk))
        plain_step()
        torch.cuda.synchronize(dev)
        plain_ms = _time_events(plain_step, max(2, min(args.steps, 5)), stream)
        extras["plain_path_ops_per_s"] = B / (plain_ms / 1000.0)
        extras["fused_equals_plain"] = bool(torch.equal(state["plain"].data, state["out"].data))
        # rotation throughput (coefficient-domain ciphertexts at level 1)
        rot_in = state["out"]
        eng.rotation_key(1)
        rot_ms = _time_events(lambda: eng.rotate_by_step(rot_in, 1), max(2, min(args.steps, 5)), stream)
        extras["rotate_ops_per_s"] = B / (rot_ms / 1000.0)
        steps16 = list(range(1, 17))
        eng.generate_rotation_keys(steps16)
        h_ms = _time_events(lambda: eng.rotate_many_by_steps(rot_in, steps16), 2, stream)
        extras["hoisted_rotations_16_ops_per_s"] = 16 * B / (h_ms / 1000.0)

        def leg(name, fn):
            # a secondary leg that fails (e.g. out of memory) is reported, and
            # the headline line is still printed
            try:
                extras[name] = fn()
            except Exception as exc:  # report, never hide
                extras[name] = f"error: {type(exc).__name__}: {str(exc)[:300]}"
            eng._scratch = None  # the headline engine's key-switch scratch is re-made on demand
            torch.cuda.empty_cache()

        leg("reference_schema_kernels", lambda: schema_ops_leg(eng, ca.data[0], ca.data[1], rlk.data[0], stream))
        leg("basis_conversion_forms", lambda: forms_leg(eng, ca, cb, rlk, stream, steps=max(2, min(args.steps, 5))))
        leg("ntt_int32_logN16_36limbs_batch64", lambda: ntt_leg(dev, stream, args.steps))
        leg("bootstrap_logN16_batch8", lambda: bootstrap_leg(dev, stream))
        if args.mixed_count > 0:
            # the mixed leg holds ~95 GB of rotation keys of its own: the
            # headline engine's rotation keys (earlier legs only) go first
            for step in list(eng.rotation_keys):
                del eng.rotation_keys[step]
            torch.cuda.empty_cache()
            leg("mixed_level_batch", lambda: mixed_batch_leg(dev, stream, args.mixed_count, args.steps))
        # decrypted error of the product (first ciphertext)
        dec = eng.decrypt_message(Ciphertext(state["out"].data[:, :1].contiguous(), 1, state["out"].scale),
                                  is_real=True)
        extras["decrypt_max_abs_err"] = float((dec[0] - (x[0] * y[0])).abs().max())
        # bit-exact vs the reference's own CPU operators on ciphertext 0
        try:
            from oracle import oracle as orc
            from oracle.ref_pipeline import ReferenceCpuPipeline, available
            if available() and rank == 0:
                ctx = orc.OracleContext(cfg.moduli, cfg.logN, cfg.num_q_primes, cfg.num_p_primes, 62, cfg.scale_bits)
                pipe = ReferenceCpuPipeline(ctx, threads=os.cpu_count())
                ref = pipe.multiply_relinearize_rescale(ca.data[:, 0].cpu(), cb.data[:, 0].cpu(), rlk.data.cpu(), 0)
                extras["bit_exact_vs_reference_cpu"] = bool(torch.equal(ref, state["out"].data[:, 0].cpu()))
        except Exception as exc:  # report, never hide
            extras["bit_exact_vs_reference_cpu"] = f"error: {exc}"

    cpu = gpu_base = None
    if rank == 0 and ws == 1 and not args.no_extras:
        threads = os.cpu_count() or 1
        v, kind, cores, sample = cpu_reference_sample(2, threads)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        eng._scratch = None
        torch.cuda.empty_cache()
        try:
            gpu_base = gpu_reference_sample(B)
        except Exception as exc:  # report, never hide
            gpu_base = {"error": f"{type(exc).__name__}: {str(exc)[:300]}"}

    csum = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded uniform messages, engine-generated keys)",
        "config": dict(CONFIG, batch_per_gpu=B, global_batch=B * ws, parallelism=f"independent ciphertexts x{ws}",
                       basis_conversion=form),
        "e2e": {"value": ws * B / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "chunks": e2e_chunks["chunks"], "staging_buffers": e2e_chunks["buffers"],
                "chunk_trials_ms": trial},
        "gpu_launches": launches_per_step * args.steps,
        "alu_roofline": {"kernel": dom_kernel, "unit": "modular products/s",
                         "modmul_per_launch": dom_modmul, "achieved": modmul_achieved, "peak": ks_peak,
                         "frac": modmul_achieved / ks_peak, "probe_ms": probe_ms,
                         "int64_peak": modmul_peak, "f64_peak": modmul_peak_f64, "f64_probe_ms": probe_f64_ms,
                         "f64_rows": f64_rows,
                         "peak_source": "fhb_modmul_probe (int64 Shoup) and fhb_modmul_probe_f64 (balanced FP64): "
                                        "148x8 CTAs x 256 threads x 8 independent chains, timed in this run; the "
                                        "peak is their mix weighted by the rows each form runs"},
        "roofline": {"kernel": dom_kernel, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": per_kernel[dom],
                     "note": ("Q rows: exact FP64 arithmetic on the FP64 pipe, P rows: int64 Shoup/Montgomery; "
                              "bound by arithmetic issue, not HBM") if f64_core else
                             ("int64 Montgomery/Shoup arithmetic (NTT butterflies, key products) on CUDA cores: "
                              "the kernel is integer-ALU bound")},
        "kernel_ms": per_kernel,
        "kernel_roofline": kernel_roofline,
        "kernel_ms_note": "each public entry point timed alone on the same inputs; the fused step runs the "
                          "HMult->INTT for d2 only and folds d0, d1 into the key-switch accumulators",
        "step_algorithmic_gbs": step_bytes / (ms / 1000.0) / 1e9,
        "clocks": csum,
        "cpu_baseline": cpu,
        "gpu_baseline": gpu_base,
        "extras": extras,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    from fhelium_b200 import ranks
    ranks.finish(ws)
    return 0


if __name__ == "__main__":
    sys.exit(main())
