"""The reference's CPU implementation of HMult -> relinearize -> rescale.

Test/baseline infrastructure only (used by tests/ and bench.py's CPU
baseline and `--impl reference` arm).  It drives the reference's own CPU
operators - compiled from its sources into oracle/_ref by build_ref.sh and
loaded through their torch.ops schemas - in the order the reference's Python
engine issues them:

  CkksEngine.multiply            fhelium/engine/ckks_engine.py:1570-1606
  CkksEngine.relinearize         fhelium/engine/ckks_engine.py:1642-1675
  HybridKeySwitcher (streaming)  fhelium/engine/hybrid_keyswitch.py:321-371,530-568
  StandardDirectKeySwitchDigitConsumer  fhelium/engine/direct_keyswitch_consumer.py:53-82
  CkksRescaler._drop_leading_scale_prime  fhelium/engine/ckks_rescale.py:339-377

The CPU backend of the reference only implements the indexed radix-2 NTT
(fhelium/config/ntt.py:87-126), so that is the transform used here.  The
tables come from the oracle's restatement of the reference's table builders
(oracle.OracleContext), which tests pin against the reference.
"""

from __future__ import annotations

import os

import numpy as np
import torch

from .oracle import OracleContext

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libfhelium_ref_cpu_ops.so")
# the same schemas with the reference's CUDA kernels too (build_ref_cuda.sh)
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libfhelium_ref_ops_cuda.so")
_loaded: list[str] = []


def available(library: str = "cpu") -> bool:
    return os.path.exists(REF_CUDA_LIB if library == "cuda" else REF_LIB)


def _load(library: str) -> None:
    """Loads one of the two reference libraries once per process; they define
    the same schemas, so a process holds only one."""
    path = REF_CUDA_LIB if library == "cuda" else REF_LIB
    if _loaded and _loaded[0] != path:
        raise RuntimeError(f"{os.path.basename(_loaded[0])} is already loaded in this process")
    if not _loaded:
        torch.ops.load_library(path)
        _loaded.append(path)


def _schedule(log_n: int):
    """Indexed radix-2 schedules (fhelium/engine/ntt/plans/indexed_radix2.py:55-110)."""
    n = 1 << log_n
    fe, fo, ft, ie, io, it = [], [], [], [], [], []
    half = n
    for s in range(log_n):
        half //= 2
        g = np.arange(1 << s)
        e = (2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1)
        fe.append(e), fo.append(e + half), ft.append(np.repeat((1 << s) + g, half))
    half = 1
    for rem in range(log_n, 0, -1):
        gc = 1 << (rem - 1)
        g = np.arange(gc)
        e = (2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1)
        ie.append(e), io.append(e + half), it.append(np.repeat(gc + g, half))
        half *= 2
    i32 = lambda x: torch.tensor(np.stack(x), dtype=torch.int32)
    return i32(fe), i32(fo), np.stack(ft), i32(ie), i32(io), np.stack(it)


class ReferenceCpuPipeline:
    """The reference engine's operator sequence.  On "cpu" it runs the
    reference's own CPU operators (oracle/_ref, required).  With a CUDA
    `device` the same calls dispatch to whatever CUDA kernels are registered
    for the reference's schemas: with library="cpu" the reference's CPU
    library is loaded first when present (its schema definitions are the ones
    in use, another library registers the CUDA kernels), with
    library="cuda" the reference's own CUDA kernels (build_ref_cuda.sh).
    ntt="compact" uses the reference's default CUDA transform policy
    (radix2_compact_group8_smem8: grouped radix-2 stages, three per launch,
    fhelium/config/ntt.py:87-126) instead of the indexed radix-2 form its
    CPU backend implements."""

    def __init__(self, ctx: OracleContext, threads: int | None = None, device: str | torch.device = "cpu",
                 library: str = "cpu", ntt: str = "indexed"):
        device = torch.device(device)
        if (device.type == "cpu" or library == "cuda") and not available(library):
            raise FileNotFoundError(REF_CUDA_LIB if library == "cuda" else REF_LIB)
        if available(library):
            _load(library)
        if ntt not in ("indexed", "compact"):
            raise ValueError("ntt must be 'indexed' or 'compact'")
        self.compact = ntt == "compact"
        if threads:
            torch.set_num_threads(threads)
        self.ctx = ctx
        self.device = device
        self.dtype = torch.int64 if ctx.radix_bits == 62 else torch.int32
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.dtype).to(device)
        self.params = t(ctx.params)
        fe, fo, ft, ie, io, it = _schedule(ctx.log_n)
        fwd, inv = ctx.twiddles
        self.fe, self.fo, self.ie, self.io = (x.to(device) for x in (fe, fo, ie, io))
        self.fwd_stage = t(np.stack([fwd[j][ft] for j in range(len(ctx.moduli))]))
        self.inv_stage = t(np.stack([inv[j][it] for j in range(len(ctx.moduli))]))
        self.fwd_compact, self.inv_compact = t(fwd), t(inv)
        self._t = t
        self.rns = torch.ops.fhelium_rns_ops
        self.ntt = torch.ops.fhelium_ntt_ops
        self.ckks = torch.ops.fhelium_ckks_ops
        self._digit_cache = {}

    def _p(self, start, stop):
        return self.params[:, start:stop]

    def _inverse_to_standard_(self, x, start, stop):
        if self.compact:
            self.ntt.inverse_ntt_to_standard_compact_grouped_smem_(x, self.inv_compact[start:stop],
                                                                   self._p(start, stop), 3)
        else:
            self.ntt.inverse_ntt_to_standard_indexed_(x, self.ie, self.io, self.inv_stage[start:stop],
                                                      self._p(start, stop))

    def _forward_montgomery_(self, x, start, stop):
        if self.compact:
            self.ntt.forward_ntt_montgomery_compact_grouped_smem_(x, self.fwd_compact[start:stop],
                                                                  self._p(start, stop), 3)
        else:
            self.ntt.forward_ntt_montgomery_indexed_(x, self.fe, self.fo, self.fwd_stage[start:stop],
                                                     self._p(start, stop))

    def _digit_args(self, level, ids):
        key = (level, ids)
        if key not in self._digit_cache:
            norm, prop, ext = self.ctx.digit_tables(ids)
            dst = self.ctx.qp_rows(level)
            dp = self.ctx.sub_params(list(ids))
            self._digit_cache[key] = (self._t(norm), self._t(prop), self._t(dp[1]), self._t(dp[2]), self._t(dp[3]),
                                      self._t(dp[4]), self._t(ext[:, dst] if len(ids) > 1 else np.zeros((0, 0))))
        return self._digit_cache[key]

    def keyswitch(self, comp: torch.Tensor, key: torch.Tensor, level: int):
        qp0 = len(self.ctx.moduli)
        acc0 = acc1 = None
        for kd, ids in self.ctx.digits_at_level(level):
            norm, prop, lo, hi, nlo, nhi, ext = self._digit_args(level, ids)
            src = comp[..., ids[0] - level: ids[-1] - level + 1, :].clone()
            if len(ids) > 1:
                src = self.rns.mixed_radix_decompose(src, norm, prop, lo, hi, nlo, nhi)
            y = self.rns.mixed_radix_basis_extend_to_montgomery(src, ext, self._p(level, qp0), qp0 - level)
            self._forward_montgomery_(y, level, qp0)
            if acc0 is None:
                acc0, acc1 = torch.zeros_like(y), torch.zeros_like(y)
            self.ckks.keyswitch_accumulate_digit_products_(acc0, acc1, y, key[kd], self._p(level, qp0), level)
        self._inverse_to_standard_(acc0, level, qp0)
        self._inverse_to_standard_(acc1, level, qp0)
        p = self.ctx.num_p
        inv = self._t(self.ctx.moddown_inverse(level))
        c0 = self.ckks.keyswitch_moddown_qp_to_q(acc0[..., :-p, :], acc0[..., -p:, :], inv, self._p(level, qp0))
        c1 = self.ckks.keyswitch_moddown_qp_to_q(acc1[..., :-p, :], acc1[..., -p:, :], inv, self._p(level, qp0))
        return c0, c1

    def multiply_relinearize_rescale(self, a: torch.Tensor, b: torch.Tensor, key: torch.Tensor, level: int):
        """a, b: [2, L, N] NTT/Montgomery -> [2, L-1, N] coefficient/standard."""
        nq = self.ctx.num_q
        prm = self._p(level, nq)
        d0 = self.rns.montgomery_mul(a[0], b[0], prm)
        x01 = self.rns.montgomery_mul(a[0], b[1], prm)
        x10 = self.rns.montgomery_mul(a[1], b[0], prm)
        d1 = self.rns.add_lazy(x01, x10, prm)
        d2 = self.rns.montgomery_mul(a[1], b[1], prm)
        for d in (d0, d1, d2):
            self._inverse_to_standard_(d, level, nq)
        c0, c1 = self.keyswitch(d2, key, level)
        d0 = d0 + c0
        d1 = d1 + c1
        self.rns.canonicalize_residues_(d0, prm)
        self.rns.canonicalize_residues_(d1, prm)
        inv = self._t(self.ctx.rescale_inverse(level)[: nq - level - 1])
        rp = self._p(level + 1, nq)
        half = self.ctx.moduli[level] // 2
        return torch.stack([self.ckks.rescale_drop_leading_prime_nearest(d[..., 1:, :], inv, d[..., 0, :], rp, half)
                            for d in (d0, d1)])
