"""CUDA implementations of the reference's custom-op schemas, served by libfhb200.

The reference reaches its kernels through PyTorch custom ops
(``torch.ops.fhelium_rns_ops``, ``fhelium_ntt_ops``, ``fhelium_ckks_ops``, and the tuning
overrides of ``fhelium_ntt_diagnostic_ops``; schemas
in csrc/ops/rns/rns_arithmetic.cpp:30-72, rns_canonical_arithmetic.cpp:15-23,
csrc/ops/ntt/forward_ntt.cpp:25-67, inverse_ntt.cpp:23-73, csrc/ops/ckks/ckks.cpp:29-90)
with one CPU and one CUDA kernel registered per schema
(``TORCH_LIBRARY_IMPL(<ns>, CUDA, m)``, csrc/ops/ntt/cuda/forward_ntt_cuda.cpp:218-245).
:func:`register` installs this library's kernels as the CUDA implementations of
the evaluation-path schemas, so code that calls those ops on CUDA tensors -- the
reference's ``RnsRuntime``, ``HybridKeySwitcher`` and ``CkksRescaler`` -- runs on
B200 unchanged.

* If the reference's native operator library is loaded first, its schema
  definitions (and CPU kernels) stay and only the CUDA kernels are added.  If it
  is not loaded, :func:`register` defines the schemas itself from the
  reference's own schema strings; loading the reference's library afterwards
  would then define them twice, so load it first.
* Element-wise, mixed-radix, key-switch, ModDown, rescale and automorphism ops
  go to the operator-level entry points ``fhb_op_*`` (one kernel per op, the
  reference's operand tables used as given).  The NTT ops go to the library's
  cluster NTT through a transform context per distinct prime set
  (``fhb_context_create_transform``), built on first use and cached.  The NTT
  uses the reference's root choice; the twiddle tensor passed in is checked once
  (its psi entry) and the indexed forms' schedules once (against the reference's
  radix-2 schedule) -- once per table tensor and version, remembered through a
  weak reference, so a new table at a reused address is checked again;
  grouped_stage_count and shared_memory_log_n only pick launch shapes in the
  reference and are ignored here.
* Outputs carry the integers of the reference's CPU kernels, except the NTT
  outputs, which are lazy [0, 2q) like the reference's CUDA kernels (equal mod q).
* Errors are ``RuntimeError`` (bad dtype, device, shape, overlapping in-place
  operand, unsupported table), as the reference's ``TORCH_CHECK`` raises.
* Operands are viewed as [batch, rows, N] without copying when their rows are N
  words apart with contiguous coefficients (so limb slices of a larger tensor
  are used in place); other layouts are copied in and, for in-place ops,
  copied back.
"""

from __future__ import annotations

import threading
import weakref

import numpy as np
import torch

from . import _native

# The reference's schema strings for the ops served here.
SCHEMAS: dict[str, dict[str, str]] = {
    "fhelium_rns_ops": {
        "montgomery_mul": "montgomery_mul(Tensor lhs, Tensor rhs, Tensor rns_params) -> Tensor",
        "add_lazy": "add_lazy(Tensor lhs, Tensor rhs, Tensor rns_params) -> Tensor",
        "sub_lazy": "sub_lazy(Tensor lhs, Tensor rhs, Tensor rns_params) -> Tensor",
        "add_canonical": "add_canonical(Tensor lhs, Tensor rhs, Tensor rns_params) -> Tensor",
        "add_canonical_": "add_canonical_(Tensor(a!) lhs, Tensor rhs, Tensor rns_params) -> ()",
        "sub_canonical": "sub_canonical(Tensor lhs, Tensor rhs, Tensor rns_params) -> Tensor",
        "sub_canonical_": "sub_canonical_(Tensor(a!) lhs, Tensor rhs, Tensor rns_params) -> ()",
        "to_montgomery_": "to_montgomery_(Tensor(a!) standard_residues, Tensor rns_params) -> ()",
        "from_montgomery_": "from_montgomery_(Tensor(a!) montgomery_residues, Tensor rns_params) -> ()",
        "canonicalize_residues_": "canonicalize_residues_(Tensor(a!) lazy_residues, Tensor rns_params) -> ()",
        "center_residues_": "center_residues_(Tensor(a!) canonical_residues, Tensor rns_params) -> ()",
        "shift_residues_positive_": "shift_residues_positive_(Tensor(a!) centered_residues, Tensor rns_params) -> ()",
        "lift_centered_coefficients": "lift_centered_coefficients(Tensor centered_coefficients, "
                                      "Tensor twice_modulus) -> Tensor",
        "montgomery_mul_cyclic_compressed": "montgomery_mul_cyclic_compressed(Tensor lhs, Tensor compressed_rhs, "
                                            "Tensor rns_params) -> Tensor",
        "montgomery_mul_contiguous_compressed": "montgomery_mul_contiguous_compressed(Tensor lhs, "
                                                "Tensor compressed_rhs, Tensor rns_params) -> Tensor",
        "montgomery_mul_row_scalars_": "montgomery_mul_row_scalars_(Tensor(a!) residues, Tensor row_scalars, "
                                       "Tensor rns_params) -> ()",
        "montgomery_mul_row_scalars_canonical": "montgomery_mul_row_scalars_canonical(Tensor residues, "
                                                "Tensor row_scalars, Tensor rns_params) -> Tensor",
        "add_lazy_with_twice_modulus": "add_lazy_with_twice_modulus(Tensor lhs, Tensor rhs, "
                                       "Tensor twice_modulus) -> Tensor",
        "mixed_radix_decompose": "mixed_radix_decompose(Tensor source_residues, Tensor mixed_radix_normalizers, "
                                 "Tensor mixed_radix_propagation_coefficients, Tensor modulus_lo, "
                                 "Tensor modulus_hi, Tensor neg_inv_modulus_lo, Tensor neg_inv_modulus_hi) -> Tensor",
        "mixed_radix_basis_extend_to_montgomery": "mixed_radix_basis_extend_to_montgomery(Tensor "
                                                  "mixed_radix_components, Tensor basis_extension_coefficients, "
                                                  "Tensor rns_params, int destination_row_count) -> Tensor",
    },
    "fhelium_ntt_ops": {
        "forward_ntt_montgomery_indexed_": "forward_ntt_montgomery_indexed_(Tensor(a!) montgomery_residues, "
                                           "Tensor even_indices, Tensor odd_indices, Tensor forward_twiddles, "
                                           "Tensor rns_params) -> ()",
        "forward_ntt_to_montgomery_indexed_": "forward_ntt_to_montgomery_indexed_(Tensor(a!) standard_residues, "
                                              "Tensor even_indices, Tensor odd_indices, Tensor forward_twiddles, "
                                              "Tensor rns_params) -> ()",
        "forward_ntt_to_montgomery_indexed": "forward_ntt_to_montgomery_indexed(Tensor standard_residues, "
                                             "Tensor even_indices, Tensor odd_indices, Tensor forward_twiddles, "
                                             "Tensor rns_params) -> Tensor",
        "forward_ntt_montgomery_compact_grouped_smem_": "forward_ntt_montgomery_compact_grouped_smem_(Tensor(a!) "
                                                        "montgomery_residues, Tensor forward_twiddles, "
                                                        "Tensor rns_params, int grouped_stage_count) -> ()",
        "forward_ntt_to_montgomery_compact_grouped_smem_": "forward_ntt_to_montgomery_compact_grouped_smem_(Tensor(a!) "
                                                           "standard_residues, Tensor forward_twiddles, "
                                                           "Tensor rns_params, int grouped_stage_count) -> ()",
        "forward_ntt_to_montgomery_compact_grouped_smem": "forward_ntt_to_montgomery_compact_grouped_smem(Tensor "
                                                          "standard_residues, Tensor forward_twiddles, "
                                                          "Tensor rns_params, int grouped_stage_count) -> Tensor",
        "forward_ntt_montgomery_compact_keyswitch_accumulate_": "forward_ntt_montgomery_compact_keyswitch_accumulate_("
                                                                "Tensor(a!) coefficient_digit_qp, Tensor "
                                                                "forward_twiddles, Tensor rns_params, Tensor "
                                                                "key_digit_qp, Tensor(b!) accumulator0_qp, "
                                                                "Tensor(c!) accumulator1_qp, int key_row_start) -> ()",
        "forward_ntt_montgomery_power_of_two_radix_compact_": "forward_ntt_montgomery_power_of_two_radix_compact_("
                                                              "Tensor(a!) montgomery_residues, Tensor outer_twiddles, "
                                                              "Tensor radix_root_powers, Tensor rns_params) -> ()",
        "forward_ntt_to_montgomery_power_of_two_radix_compact_": "forward_ntt_to_montgomery_power_of_two_radix_"
                                                                 "compact_(Tensor(a!) standard_residues, Tensor "
                                                                 "outer_twiddles, Tensor radix_root_powers, "
                                                                 "Tensor rns_params) -> ()",
        "forward_ntt_to_montgomery_power_of_two_radix_compact": "forward_ntt_to_montgomery_power_of_two_radix_"
                                                                "compact(Tensor standard_residues, Tensor "
                                                                "outer_twiddles, Tensor radix_root_powers, "
                                                                "Tensor rns_params) -> Tensor",
        "inverse_ntt_montgomery_power_of_two_radix_compact_": "inverse_ntt_montgomery_power_of_two_radix_compact_("
                                                              "Tensor(a!) montgomery_residues, Tensor outer_twiddles, "
                                                              "Tensor radix_root_powers, Tensor rns_params) -> ()",
        "inverse_ntt_to_standard_lazy_power_of_two_radix_compact_": "inverse_ntt_to_standard_lazy_power_of_two_"
                                                                    "radix_compact_(Tensor(a!) montgomery_residues, "
                                                                    "Tensor outer_twiddles, Tensor radix_root_powers, "
                                                                    "Tensor rns_params) -> ()",
        "inverse_ntt_to_standard_power_of_two_radix_compact_": "inverse_ntt_to_standard_power_of_two_radix_compact_("
                                                               "Tensor(a!) montgomery_residues, Tensor "
                                                               "outer_twiddles, Tensor radix_root_powers, "
                                                               "Tensor rns_params) -> ()",
        "inverse_ntt_to_centered_power_of_two_radix_compact_": "inverse_ntt_to_centered_power_of_two_radix_compact_("
                                                               "Tensor(a!) montgomery_residues, Tensor "
                                                               "outer_twiddles, Tensor radix_root_powers, "
                                                               "Tensor rns_params) -> ()",
        "inverse_ntt_montgomery_indexed_": "inverse_ntt_montgomery_indexed_(Tensor(a!) montgomery_residues, "
                                           "Tensor even_indices, Tensor odd_indices, Tensor inverse_twiddles, "
                                           "Tensor rns_params) -> ()",
        "inverse_ntt_to_standard_lazy_indexed_": "inverse_ntt_to_standard_lazy_indexed_(Tensor(a!) "
                                                 "montgomery_residues, Tensor even_indices, Tensor odd_indices, "
                                                 "Tensor inverse_twiddles, Tensor rns_params) -> ()",
        "inverse_ntt_to_standard_indexed_": "inverse_ntt_to_standard_indexed_(Tensor(a!) montgomery_residues, "
                                            "Tensor even_indices, Tensor odd_indices, Tensor inverse_twiddles, "
                                            "Tensor rns_params) -> ()",
        "inverse_ntt_to_centered_indexed_": "inverse_ntt_to_centered_indexed_(Tensor(a!) montgomery_residues, "
                                            "Tensor even_indices, Tensor odd_indices, Tensor inverse_twiddles, "
                                            "Tensor rns_params) -> ()",
        "inverse_ntt_montgomery_compact_grouped_smem_": "inverse_ntt_montgomery_compact_grouped_smem_(Tensor(a!) "
                                                        "montgomery_residues, Tensor inverse_twiddles, "
                                                        "Tensor rns_params, int grouped_stage_count) -> ()",
        "inverse_ntt_to_standard_lazy_compact_grouped_smem_": "inverse_ntt_to_standard_lazy_compact_grouped_smem_("
                                                              "Tensor(a!) montgomery_residues, Tensor "
                                                              "inverse_twiddles, Tensor rns_params, "
                                                              "int grouped_stage_count) -> ()",
        "inverse_ntt_to_standard_compact_grouped_smem_": "inverse_ntt_to_standard_compact_grouped_smem_(Tensor(a!) "
                                                         "montgomery_residues, Tensor inverse_twiddles, "
                                                         "Tensor rns_params, int grouped_stage_count) -> ()",
        "inverse_ntt_to_centered_compact_grouped_smem_": "inverse_ntt_to_centered_compact_grouped_smem_(Tensor(a!) "
                                                         "montgomery_residues, Tensor inverse_twiddles, "
                                                         "Tensor rns_params, int grouped_stage_count) -> ()",
    },
    # tuning-override forms the reference keeps outside its production ABI
    # (csrc/ops/ntt/forward_ntt.cpp:68-80, inverse_ntt.cpp)
    "fhelium_ntt_diagnostic_ops": {
        "forward_ntt_montgomery_compact_grouped_smem_override_": "forward_ntt_montgomery_compact_grouped_smem_"
                                                                 "override_(Tensor(a!) montgomery_residues, Tensor "
                                                                 "forward_twiddles, Tensor rns_params, int "
                                                                 "grouped_stage_count, int shared_memory_log_n) -> ()",
        "forward_ntt_montgomery_power_of_two_radix_compact_override_": "forward_ntt_montgomery_power_of_two_radix_"
                                                                       "compact_override_(Tensor(a!) "
                                                                       "montgomery_residues, Tensor outer_twiddles, "
                                                                       "Tensor radix_root_powers, Tensor rns_params, "
                                                                       "int shared_memory_log_n) -> ()",
        "inverse_ntt_montgomery_power_of_two_radix_compact_override_": "inverse_ntt_montgomery_power_of_two_radix_"
                                                                       "compact_override_(Tensor(a!) "
                                                                       "montgomery_residues, Tensor outer_twiddles, "
                                                                       "Tensor radix_root_powers, Tensor rns_params, "
                                                                       "int shared_memory_log_n) -> ()",
    },
    "fhelium_ckks_ops": {
        "add_prepared_plaintext_component": "add_prepared_plaintext_component(Tensor ciphertext_component, "
                                            "Tensor prepared_plaintext, Tensor rns_params) -> Tensor",
        "add_prepared_plaintext_component_": "add_prepared_plaintext_component_(Tensor(a!) ciphertext_component, "
                                             "Tensor prepared_plaintext, Tensor rns_params) -> ()",
        "add_cyclic_compressed_plaintext_component": "add_cyclic_compressed_plaintext_component(Tensor "
                                                     "ciphertext_component, Tensor compressed_plaintext, "
                                                     "Tensor rns_params) -> Tensor",
        "add_cyclic_compressed_plaintext_component_": "add_cyclic_compressed_plaintext_component_(Tensor(a!) "
                                                      "ciphertext_component, Tensor compressed_plaintext, "
                                                      "Tensor rns_params) -> ()",
        "add_contiguous_compressed_plaintext_component": "add_contiguous_compressed_plaintext_component(Tensor "
                                                         "ciphertext_component, Tensor compressed_plaintext, "
                                                         "Tensor rns_params) -> Tensor",
        "add_contiguous_compressed_plaintext_component_": "add_contiguous_compressed_plaintext_component_(Tensor(a!) "
                                                          "ciphertext_component, Tensor compressed_plaintext, "
                                                          "Tensor rns_params) -> ()",
        "add_strided_plaintext_component": "add_strided_plaintext_component(Tensor ciphertext_component, "
                                           "Tensor strided_plaintext, Tensor implicit_plaintext, "
                                           "Tensor rns_params) -> Tensor",
        "add_strided_plaintext_component_": "add_strided_plaintext_component_(Tensor(a!) ciphertext_component, "
                                            "Tensor strided_plaintext, Tensor implicit_plaintext, "
                                            "Tensor rns_params) -> ()",
        "rescale_drop_leading_prime_nearest": "rescale_drop_leading_prime_nearest(Tensor remaining_residues, "
                                              "Tensor drop_prime_inverse_mont, Tensor dropped_residue, "
                                              "Tensor rns_params, int half_drop_prime) -> Tensor",
        "rescale_drop_leading_prime_nearest_": "rescale_drop_leading_prime_nearest_(Tensor(a!) remaining_residues, "
                                               "Tensor drop_prime_inverse_mont, Tensor dropped_residue, "
                                               "Tensor rns_params, int half_drop_prime) -> ()",
        "rescale_drop_leading_prime_truncate": "rescale_drop_leading_prime_truncate(Tensor remaining_residues, "
                                               "Tensor drop_prime_inverse_mont, Tensor dropped_residue, "
                                               "Tensor rns_params) -> Tensor",
        "rescale_drop_leading_prime_truncate_": "rescale_drop_leading_prime_truncate_(Tensor(a!) remaining_residues, "
                                                "Tensor drop_prime_inverse_mont, Tensor dropped_residue, "
                                                "Tensor rns_params) -> ()",
        "apply_coefficient_galois_automorphism": "apply_coefficient_galois_automorphism(Tensor residues, "
                                                 "Tensor source_indices, Tensor source_sign, "
                                                 "Tensor twice_modulus) -> Tensor",
        "apply_ntt_galois_automorphism": "apply_ntt_galois_automorphism(Tensor residues_ntt, "
                                         "Tensor source_indices) -> Tensor",
        "keyswitch_moddown_qp_to_q": "keyswitch_moddown_qp_to_q(Tensor q_residues, Tensor p_residues, "
                                     "Tensor moddown_p_drop_inverses_montgomery, Tensor rns_params) -> Tensor",
        "keyswitch_accumulate_digit_products_": "keyswitch_accumulate_digit_products_(Tensor(a!) accumulator0_qp, "
                                                "Tensor(b!) accumulator1_qp, Tensor extended_digit_ntt_qp, "
                                                "Tensor key_switch_key_digit, Tensor rns_params, "
                                                "int key_digit_row_start) -> ()",
    },
}

_lock = threading.Lock()
_libraries: list = []          # keeps the torch.library registrations alive
_registered = False
_contexts: dict = {}           # (bits, log_n, primes, device) -> NativeContext
_slices: dict = {}             # (bits, log_n, primes, device) -> (NativeContext, first prime id)
# Verification results and prime lists, remembered per tensor: keyed weakly by the tensor that
# owns the storage (a view's base), then by the view's offset, shape, strides and version, so a
# freed table whose address is reused is never mistaken for a checked one.
_memo: dict = {}               # id(owning tensor) -> {key: value}; dropped when that tensor dies


def _memo_key(t: torch.Tensor, tag):
    return (tag, t.storage_offset(), tuple(t.shape), tuple(t.stride()), t._version)


def _anchor(t: torch.Tensor) -> torch.Tensor:
    return t._base if t._base is not None else t


def _memo_get(t: torch.Tensor, tag):
    entries = _memo.get(id(_anchor(t)))
    return None if entries is None else entries.get(_memo_key(t, tag))


def _memo_put(t: torch.Tensor, tag, value) -> None:
    anchor = _anchor(t)
    entries = _memo.get(id(anchor))
    if entries is None:
        entries = _memo[id(anchor)] = {}
        weakref.finalize(anchor, _memo.pop, id(anchor), None)
    entries[_memo_key(t, tag)] = value


# --------------------------------------------------------------------------- helpers
def _fail(msg: str):
    raise RuntimeError(msg)


def _bits(t: torch.Tensor, name: str) -> int:
    if t.dtype == torch.int64:
        return 64
    if t.dtype == torch.int32:
        return 32
    _fail(f"{name} must be int64 or int32, got {t.dtype}")


def _same(t: torch.Tensor, ref: torch.Tensor, name: str) -> None:
    if t.dtype != ref.dtype:
        _fail(f"{name} must have dtype {ref.dtype}, got {t.dtype}")
    if t.device != ref.device:
        _fail(f"{name} must be on {ref.device}, got {t.device}")


def _batch_view(t: torch.Tensor, rows_dims: int = 2):
    """(batch, batch_stride) if t's leading dims collapse into one stride and its
    trailing [rows, N] (rows_dims = 2) or [N] (rows_dims = 1) is dense, else None."""
    shape, stride = t.shape, t.stride()
    if t.dim() < rows_dims:
        return None
    n = shape[-1]
    if n > 1 and stride[-1] != 1:
        return None
    if rows_dims == 2 and shape[-2] > 1 and stride[-2] != n:
        return None
    lead = t.dim() - rows_dims
    batch = 1
    for s in shape[:lead]:
        batch *= s
    inner = n * (shape[-2] if rows_dims == 2 else 1)
    if lead == 0:
        return 1, inner
    dims = [(s, st) for s, st in zip(shape[:lead], stride[:lead]) if s != 1]
    if not dims:
        return batch, inner
    for (s0, st0), (s1, st1) in zip(dims, dims[1:]):
        if st0 != st1 * s1:
            return None
    return batch, dims[-1][1]


class _Operand:
    """A [batch, rows, N] view of a tensor for the C ABI (copied when not viewable)."""

    def __init__(self, t: torch.Tensor, writable: bool = False, rows_dims: int = 2):
        self.orig = t
        v = _batch_view(t, rows_dims)
        if v is None:
            t = t.contiguous()
            v = _batch_view(t, rows_dims)
            self.copied = True
        else:
            self.copied = False
        self.t = t
        self.batch, self.stride = v
        self.writable = writable

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()

    def finish(self) -> None:
        if self.writable and self.copied:
            self.orig.copy_(self.t)


def _params(p: torch.Tensor, ref: torch.Tensor, rows: int, name: str = "rns_params"):
    _same(p, ref, name)
    if p.dim() != 2 or p.shape[0] < 8:
        _fail(f"{name} must be [8, limb], got {tuple(p.shape)}")
    if p.shape[1] != rows:
        _fail(f"{name} has {p.shape[1]} limb columns for {rows} residue rows")
    if p.shape[1] > 1 and p.stride(1) != 1:
        p = p.contiguous()
    return p, p.stride(0)


def _check_writable(t: torch.Tensor, name: str) -> None:
    if torch._debug_has_internal_overlap(t) == 1:
        _fail(f"{name}: unsupported operation: more than one element of the written-to tensor "
              "refers to a single memory location")


def _no_overlap(out: torch.Tensor, *others) -> None:
    """The reference's check_mutable_rns_output (csrc/ops/common/rns_batch.h:87-97,
    at::assert_no_overlap): a written tensor may not share elements with a
    read-only operand or table.  Like ATen, the same tensor or two dense tensors
    with intersecting byte ranges are rejected; other layouts are not examined."""
    from torch._prims_common import is_non_overlapping_and_dense_or_false as is_non_overlapping_and_dense
    for other in others:
        if other is None or other.numel() == 0 or out.numel() == 0:
            continue
        if other is out:
            overlap = True
        elif out.untyped_storage().data_ptr() != other.untyped_storage().data_ptr():
            continue
        elif not (is_non_overlapping_and_dense(out) and is_non_overlapping_and_dense(other)):
            continue
        else:
            a0, b0 = out.data_ptr(), other.data_ptr()
            overlap = a0 < b0 + other.numel() * other.element_size() and b0 < a0 + out.numel() * out.element_size()
        if overlap:
            _fail("unsupported operation: some elements of the input tensor and the written-to tensor refer to "
                  "a single memory location.")


def _cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        _fail(f"{name} must be a CUDA tensor")


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _call(name: str, *args) -> None:
    _native.check(getattr(_native.load(), name)(*args), name)


def _rows_n(t: torch.Tensor, name: str):
    if t.dim() < 2:
        _fail(f"{name} must be [*batch, limb, N]")
    return t.shape[-2], t.shape[-1]


# --------------------------------------------------------------------------- rns ops
def _binary(op: int, lhs: torch.Tensor, rhs: torch.Tensor, params: torch.Tensor, out=None):
    _cuda(lhs, "lhs")
    bits = _bits(lhs, "lhs")
    _same(rhs, lhs, "rhs")
    rows, n = _rows_n(lhs, "lhs")
    if tuple(rhs.shape[-2:]) != (rows, n):
        _fail(f"rhs limb/coefficient shape {tuple(rhs.shape[-2:])} does not match lhs {(rows, n)}")
    a = _Operand(lhs)
    b = _Operand(rhs)
    if b.batch not in (1, a.batch):
        _fail(f"rhs batch {b.batch} must equal lhs batch {a.batch} or be 1")
    p, ps = _params(params, lhs, rows)
    writable = out is not None
    if out is None:
        out = torch.empty_like(lhs, memory_format=torch.contiguous_format)
    o = _Operand(out, writable=writable)
    with torch.cuda.device(lhs.device):
        _call("fhb_op_rns_binary", bits, op, a.ptr, a.stride, b.ptr, b.stride if b.batch > 1 else 0, o.ptr,
              o.stride, a.batch, rows, n, p.data_ptr(), ps, _stream(lhs))
    o.finish()
    return out


def _unary_(op: int, x: torch.Tensor, params: torch.Tensor) -> None:
    _cuda(x, "residues")
    _check_writable(x, "residues")
    _no_overlap(x, params)
    bits = _bits(x, "residues")
    rows, n = _rows_n(x, "residues")
    p, ps = _params(params, x, rows)
    o = _Operand(x, writable=True)
    with torch.cuda.device(x.device):
        _call("fhb_op_rns_unary", bits, op, o.ptr, o.stride, o.batch, rows, n, p.data_ptr(), ps, _stream(x))
    o.finish()


def montgomery_mul(lhs, rhs, rns_params):
    return _binary(0, lhs, rhs, rns_params)


def add_lazy(lhs, rhs, rns_params):
    return _binary(1, lhs, rhs, rns_params)


def sub_lazy(lhs, rhs, rns_params):
    return _binary(2, lhs, rhs, rns_params)


def add_canonical(lhs, rhs, rns_params):
    return _binary(3, lhs, rhs, rns_params)


def add_canonical_(lhs, rhs, rns_params):
    _check_writable(lhs, "lhs")
    _no_overlap(lhs, rhs, rns_params)
    _binary(3, lhs, rhs, rns_params, out=lhs)


def sub_canonical(lhs, rhs, rns_params):
    return _binary(4, lhs, rhs, rns_params)


def sub_canonical_(lhs, rhs, rns_params):
    _check_writable(lhs, "lhs")
    _no_overlap(lhs, rhs, rns_params)
    _binary(4, lhs, rhs, rns_params, out=lhs)


def to_montgomery_(x, rns_params):
    _unary_(0, x, rns_params)


def from_montgomery_(x, rns_params):
    _unary_(1, x, rns_params)


def canonicalize_residues_(x, rns_params):
    _unary_(2, x, rns_params)


def center_residues_(x, rns_params):
    _unary_(3, x, rns_params)


def shift_residues_positive_(x, rns_params):
    _unary_(4, x, rns_params)


def _mul_compressed(layout: int, lhs, rhs, params):
    _cuda(lhs, "lhs")
    bits = _bits(lhs, "lhs")
    _same(rhs, lhs, "compressed_rhs")
    rows, n = _rows_n(lhs, "lhs")
    if rhs.dim() < 2 or rhs.shape[-2] != rows:
        _fail(f"compressed_rhs must be [*batch, {rows}, unique], got {tuple(rhs.shape)}")
    unique = rhs.shape[-1]
    if not (0 < unique < n and unique & (unique - 1) == 0 and n % unique == 0):
        _fail(f"compressed unique count must be a power of two smaller than the ring dimension: {unique} vs {n}")
    a, b = _Operand(lhs), _Operand(rhs)
    if b.batch not in (1, a.batch):
        _fail(f"operand batch counts differ: {a.batch} vs {b.batch}")
    p, ps = _params(params, lhs, rows)
    out = torch.empty_like(lhs, memory_format=torch.contiguous_format)
    with torch.cuda.device(lhs.device):
        _call("fhb_op_mul_compressed", bits, layout, a.ptr, a.stride, b.ptr, b.stride if b.batch > 1 else 0, unique,
              out.data_ptr(), rows * n, a.batch, rows, n, p.data_ptr(), ps, _stream(lhs))
    return out


def montgomery_mul_cyclic_compressed(lhs, compressed_rhs, rns_params):
    return _mul_compressed(1, lhs, compressed_rhs, rns_params)


def montgomery_mul_contiguous_compressed(lhs, compressed_rhs, rns_params):
    return _mul_compressed(2, lhs, compressed_rhs, rns_params)


def _row_scalars(x, scalars, params, out=None):
    _cuda(x, "residues")
    bits = _bits(x, "residues")
    rows, n = _rows_n(x, "residues")
    _same(scalars, x, "row_scalars")
    if scalars.numel() != rows:
        _fail(f"row_scalars must have {rows} entries, got {scalars.numel()}")
    p, ps = _params(params, x, rows)
    a = _Operand(x)
    writable = out is not None
    if out is None:
        out = torch.empty_like(x, memory_format=torch.contiguous_format)
    o = _Operand(out, writable=writable)
    sc = scalars.contiguous()
    with torch.cuda.device(x.device):
        _call("fhb_op_mul_row_scalars", bits, a.ptr, a.stride, o.ptr, o.stride, a.batch, rows, n, sc.data_ptr(),
              p.data_ptr(), ps, _stream(x))
    o.finish()
    return out


def montgomery_mul_row_scalars_(residues, row_scalars, rns_params):
    _check_writable(residues, "residues")
    _no_overlap(residues, row_scalars, rns_params)
    _row_scalars(residues, row_scalars, rns_params, out=residues)


def montgomery_mul_row_scalars_canonical(residues, row_scalars, rns_params):
    return _row_scalars(residues, row_scalars, rns_params)


def add_lazy_with_twice_modulus(lhs, rhs, twice_modulus):
    _cuda(lhs, "lhs")
    bits = _bits(lhs, "lhs")
    _same(rhs, lhs, "rhs")
    _same(twice_modulus, lhs, "twice_modulus")
    rows, n = _rows_n(lhs, "lhs")
    if twice_modulus.numel() != rows or tuple(rhs.shape[-2:]) != (rows, n):
        _fail("twice_modulus / rhs do not match lhs's limbs")
    a, b = _Operand(lhs), _Operand(rhs)
    if b.batch not in (1, a.batch):
        _fail(f"rhs batch {b.batch} must equal lhs batch {a.batch} or be 1")
    tm = twice_modulus.contiguous()
    out = torch.empty_like(lhs, memory_format=torch.contiguous_format)
    with torch.cuda.device(lhs.device):
        # ops 1 (add_lazy) reads only parameter row 0: a 2q vector with row stride 0
        _call("fhb_op_rns_binary", bits, 1, a.ptr, a.stride, b.ptr, b.stride if b.batch > 1 else 0, out.data_ptr(),
              rows * n, a.batch, rows, n, tm.data_ptr(), 0, _stream(lhs))
    return out


def lift_centered_coefficients(coefficients, twice_modulus):
    _cuda(coefficients, "centered_coefficients")
    bits = _bits(coefficients, "centered_coefficients")
    _same(twice_modulus, coefficients, "twice_modulus")
    if twice_modulus.dim() != 1:
        _fail("twice_modulus must be one-dimensional")
    rows, n = twice_modulus.shape[0], coefficients.shape[-1]
    c = _Operand(coefficients, rows_dims=1)
    out = coefficients.new_empty(tuple(coefficients.shape[:-1]) + (rows, n))
    tm = twice_modulus.contiguous()
    with torch.cuda.device(coefficients.device):
        _call("fhb_op_lift_centered", bits, c.ptr, c.stride, out.data_ptr(), rows * n, c.batch, rows, n,
              tm.data_ptr(), _stream(coefficients))
    return out


def mixed_radix_decompose(source, normalizers, propagation, modulus_lo, modulus_hi, neg_lo, neg_hi):
    _cuda(source, "source_residues")
    bits = _bits(source, "source_residues")
    rows, n = _rows_n(source, "source_residues")
    if rows > 8:
        _fail(f"mixed_radix_decompose supports at most 8 rows per digit, got {rows}")
    vecs = []
    for t, name in ((modulus_lo, "modulus_lo"), (modulus_hi, "modulus_hi"), (neg_lo, "neg_inv_modulus_lo"),
                    (neg_hi, "neg_inv_modulus_hi")):
        _same(t, source, name)
        if t.numel() != rows:
            _fail(f"{name} must have {rows} entries, got {t.numel()}")
        vecs.append(t.contiguous())
    for t, name in ((normalizers, "mixed_radix_normalizers"), (propagation, "mixed_radix_propagation_coefficients")):
        _same(t, source, name)
    if rows > 1 and normalizers.numel() < rows - 1:
        _fail("mixed_radix_normalizers needs one entry per row after the first")
    if rows > 1 and (propagation.dim() != 2 or propagation.shape[0] < rows - 1 or propagation.shape[1] < rows):
        _fail("mixed_radix_propagation_coefficients must be [rows - 1, rows]")
    norm = normalizers.contiguous()
    prop = propagation.contiguous() if propagation.dim() == 2 else propagation
    s = _Operand(source)
    out = torch.empty_like(source, memory_format=torch.contiguous_format)
    with torch.cuda.device(source.device):
        _call("fhb_op_mixed_radix_decompose", bits, s.ptr, s.stride, out.data_ptr(), rows * n, s.batch, rows, n,
              norm.data_ptr() if rows > 1 else None, prop.data_ptr() if rows > 1 else None,
              prop.shape[1] if rows > 1 else 0, *[v.data_ptr() for v in vecs], _stream(source))
    return out


def mixed_radix_basis_extend_to_montgomery(components, coefficients, rns_params, destination_row_count):
    _cuda(components, "mixed_radix_components")
    bits = _bits(components, "mixed_radix_components")
    digits, n = _rows_n(components, "mixed_radix_components")
    dst = int(destination_row_count)
    if dst < 0:
        _fail("destination_row_count must be non-negative")
    p, ps = _params(rns_params, components, dst)
    coeff_ptr, coeff_stride = None, 0
    if digits > 1:
        _same(coefficients, components, "basis_extension_coefficients")
        if coefficients.dim() != 2 or coefficients.shape[0] < digits - 1 or coefficients.shape[1] < dst:
            _fail(f"basis_extension_coefficients must be [{digits - 1}, {dst}], got {tuple(coefficients.shape)}")
        if coefficients.stride(1) != 1:
            coefficients = coefficients.contiguous()
        coeff_ptr, coeff_stride = coefficients.data_ptr(), coefficients.stride(0)
    d = _Operand(components)
    out = components.new_empty(tuple(components.shape[:-2]) + (dst, n))
    with torch.cuda.device(components.device):
        _call("fhb_op_basis_extend", bits, d.ptr, d.stride, digits, out.data_ptr(), dst * n, d.batch, dst, n,
              coeff_ptr, coeff_stride, p.data_ptr(), ps, _stream(components))
    return out


# --------------------------------------------------------------------------- ntt ops
def _primes(params: torch.Tensor) -> tuple:
    primes = _memo_get(params, "primes")
    if primes is None:
        primes = tuple(int(v) // 2 for v in params[0].cpu().tolist())
        _memo_put(params, "primes", primes)
    return primes


def _transform_context(x: torch.Tensor, params: torch.Tensor):
    bits = _bits(x, "residues")
    rows, n = _rows_n(x, "residues")
    if n < 2 or n & (n - 1):
        _fail(f"ring dimension {n} is not a power of two")
    log_n = n.bit_length() - 1
    _params(params, x, rows)
    primes = _primes(params)
    key = (bits, log_n, primes, x.device.index)
    with _lock:
        hit = _slices.get(key)
        if hit is None:
            # a slice of a chain already served reuses its context at an offset
            for (cb, cl, cprimes, cdev), ctx in _contexts.items():
                if (cb, cl, cdev) == (bits, log_n, x.device.index):
                    off = _find_run(cprimes, primes)
                    if off is not None:
                        hit = (ctx, off)
                        break
            if hit is None:
                ctx = _native.NativeContext.transform(bits, log_n, primes, x.device)
                _contexts[key] = ctx
                hit = (ctx, 0)
            _slices[key] = hit
    return hit[0], hit[1], primes, bits, log_n


def _find_run(chain: tuple, run: tuple):
    """Offset of `run` as a contiguous run of `chain`, or None."""
    if not run or len(run) > len(chain):
        return None
    first = run[0]
    for off, q in enumerate(chain[: len(chain) - len(run) + 1]):
        if q == first and chain[off: off + len(run)] == run:
            return off
    return None


def _check_twiddles(tw: torch.Tensor, ctx, offset: int, primes: tuple, bits: int, log_n: int, inverse: bool,
                    indexed: bool, radix_roots: torch.Tensor | None = None):
    n, rows = 1 << log_n, len(primes)
    exponent = 1
    if radix_roots is not None:
        # power-of-two radix tables (fhelium/engine/ntt/plans/twiddles.py:152-230): outer twists
        # [prime, N - 1] and the powers of the radix-th root psi^(2N/radix) [prime, radix]
        radix = radix_roots.shape[-1] if radix_roots.dim() == 2 else 0
        if radix not in (4, 8, 16) or radix_roots.shape[0] != rows:
            _fail(f"radix_root_powers must be [{rows}, 4 | 8 | 16], got {tuple(radix_roots.shape)}")
        if log_n % {4: 2, 8: 3, 16: 4}[radix]:
            _fail("Strict radix width must divide log_ring_dimension")
        if tw.dim() != 2 or tuple(tw.shape) != (rows, n - 1):
            _fail(f"outer_twiddles must be [{rows}, {n - 1}], got {tuple(tw.shape)}")
        _same(radix_roots, tw, "radix_root_powers")
        probe = radix_roots[:, 1]
        exponent = 2 * n // radix
    elif indexed:
        if tw.dim() != 3 or tw.shape[0] != rows or tw.shape[2] != n // 2:
            _fail(f"twiddles must be [{rows}, log2(N) stages, {n // 2}], got {tuple(tw.shape)}")
        if tw.shape[1] != log_n:
            _fail(f"twiddles must hold log2(N) stages ({log_n}), got {tw.shape[1]}")
        probe = tw[:, 0, 0] if inverse else tw[:, log_n - 1, 0]
    else:
        if tw.dim() != 2 or tuple(tw.shape) != (rows, n):
            _fail(f"twiddles must be [{rows}, {n}], got {tuple(tw.shape)}")
        probe = tw[:, n // 2]
    probed = radix_roots if radix_roots is not None else tw
    tag = ("twiddles", inverse, indexed, radix_roots is not None, primes)
    if _memo_get(probed, tag):
        return
    got = [int(v) for v in probe.cpu().tolist()]
    radix = 62 if bits == 64 else 30
    for j, q in enumerate(primes):
        psi = pow(ctx.root(offset + j), exponent, q)
        w = pow(psi, -1, q) if inverse else psi
        if got[j] % q != (w << radix) % q:
            _fail(f"twiddle row {j} does not hold the reference's primitive root (Montgomery form) "
                  f"for modulus {q}")
    _memo_put(probed, tag, True)


def _radix2_schedule(log_n: int, inverse: bool):
    """The reference's indexed radix-2 schedule (fhelium/engine/ntt/plans/indexed_radix2.py:55-110)."""
    even = []
    if not inverse:
        half = 1 << log_n
        for s in range(log_n):
            half //= 2
            g = np.arange(1 << s)
            even.append((2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1))
            # odd = even + half
    else:
        half = 1
        for rem in range(log_n, 0, -1):
            g = np.arange(1 << (rem - 1))
            even.append((2 * g[:, None] * half + np.arange(half)[None, :]).reshape(-1))
            half *= 2
    even = np.stack(even)
    halves = np.array([(1 << log_n) >> (s + 1) for s in range(log_n)]) if not inverse else \
        np.array([1 << s for s in range(log_n)])
    return even, even + halves[:, None]


def _check_schedule(even: torch.Tensor, odd: torch.Tensor, log_n: int, inverse: bool):
    tag = ("schedule", log_n, inverse)
    if _memo_get(even, tag + ("even",)) and _memo_get(odd, tag + ("odd",)):
        return
    n = 1 << log_n
    for t, name in ((even, "even_indices"), (odd, "odd_indices")):
        if t.dim() != 2 or t.shape[0] != log_n or t.shape[1] != n // 2:
            _fail(f"{name} must be [log2(N) stages, N/2] = [{log_n}, {n // 2}], got {tuple(t.shape)}")
    e = even.cpu().numpy().astype(np.int64)
    o = odd.cpu().numpy().astype(np.int64)
    if e.min() < 0 or o.min() < 0 or e.max() >= n or o.max() >= n:
        _fail("NTT schedule holds an out-of-range coefficient index")
    both = np.concatenate([e, o], axis=1)
    both.sort(axis=1)
    if not np.array_equal(both, np.broadcast_to(np.arange(n), both.shape)):
        _fail("NTT schedule stages must partition every coefficient exactly once")
    want_e, want_o = _radix2_schedule(log_n, inverse)
    if not (np.array_equal(e, want_e) and np.array_equal(o, want_o)):
        _fail("fhelium_b200 serves the reference's radix-2 indexed schedule only")
    _memo_put(even, tag + ("even",), True)
    _memo_put(odd, tag + ("odd",), True)


def _ntt_(x: torch.Tensor, tw: torch.Tensor, params: torch.Tensor, *, inverse: bool, mode: int,
          schedule=None, radix_roots=None) -> None:
    """mode: forward 0 = standard input, 1 = Montgomery input; inverse = fhb_inverse_output."""
    _cuda(x, "residues")
    _check_writable(x, "residues")
    _no_overlap(x, tw, params, radix_roots, *(schedule or ()))
    ctx, offset, primes, bits, log_n = _transform_context(x, params)
    _same(tw, x, "twiddles")
    if schedule is not None:
        _check_schedule(schedule[0], schedule[1], log_n, inverse)
    _check_twiddles(tw, ctx, offset, primes, bits, log_n, inverse, schedule is not None, radix_roots)
    rows = len(primes)
    o = _Operand(x, writable=True)
    if o.stride != rows * x.shape[-1] and o.batch > 1:
        o = _Operand(x.contiguous(), writable=False)
        o.orig, o.writable, o.copied = x, True, True
    with torch.cuda.device(x.device):
        name = "fhb_inverse_ntt" if inverse else "fhb_forward_ntt"
        ctx.call(name, o.ptr, o.ptr, o.batch, rows, offset, mode, _stream(x))
    o.finish()


def _fwd_indexed_(montgomery: int):
    def f(x, even, odd, tw, params):
        _ntt_(x, tw, params, inverse=False, mode=montgomery, schedule=(even, odd))
    return f


def _fwd_compact_(montgomery: int):
    def f(x, tw, params, grouped_stage_count):
        _ntt_(x, tw, params, inverse=False, mode=montgomery)
    return f


def _inv_indexed_(kind: int):
    def f(x, even, odd, tw, params):
        _ntt_(x, tw, params, inverse=True, mode=kind, schedule=(even, odd))
    return f


def _inv_compact_(kind: int):
    def f(x, tw, params, grouped_stage_count):
        _ntt_(x, tw, params, inverse=True, mode=kind)
    return f


def _fwd_radix_(montgomery: int):
    def f(x, outer, roots, params, shared_memory_log_n=None):
        _ntt_(x, outer, params, inverse=False, mode=montgomery, radix_roots=roots)
    return f


def _inv_radix_(kind: int):
    def f(x, outer, roots, params, shared_memory_log_n=None):
        _ntt_(x, outer, params, inverse=True, mode=kind, radix_roots=roots)
    return f


def forward_ntt_to_montgomery_power_of_two_radix_compact(x, outer, roots, params):
    y = x.clone(memory_format=torch.contiguous_format)
    _ntt_(y, outer, params, inverse=False, mode=0, radix_roots=roots)
    return y


def forward_ntt_montgomery_compact_grouped_smem_override_(x, tw, params, grouped_stage_count, shared_memory_log_n):
    _ntt_(x, tw, params, inverse=False, mode=1)


def forward_ntt_to_montgomery_indexed(x, even, odd, tw, params):
    y = x.clone(memory_format=torch.contiguous_format)
    _ntt_(y, tw, params, inverse=False, mode=0, schedule=(even, odd))
    return y


def forward_ntt_to_montgomery_compact_grouped_smem(x, tw, params, grouped_stage_count):
    y = x.clone(memory_format=torch.contiguous_format)
    _ntt_(y, tw, params, inverse=False, mode=0)
    return y


def forward_ntt_montgomery_compact_keyswitch_accumulate_(digit, tw, params, key_digit, acc0, acc1, key_row_start):
    _ntt_(digit, tw, params, inverse=False, mode=1)
    keyswitch_accumulate_digit_products_(acc0, acc1, digit, key_digit, params, key_row_start)


# --------------------------------------------------------------------------- ckks ops
def _add_plaintext(layout: int, ct, pt, params, implicit=None, out=None):
    _cuda(ct, "ciphertext_component")
    bits = _bits(ct, "ciphertext_component")
    _same(pt, ct, "plaintext")
    rows, n = _rows_n(ct, "ciphertext_component")
    if pt.dim() < 2 or pt.shape[-2] != rows:
        _fail(f"plaintext must be [*batch, {rows}, extent], got {tuple(pt.shape)}")
    extent = pt.shape[-1]
    if layout == 0 and extent != n:
        _fail(f"prepared plaintext must have {n} coefficients, got {extent}")
    if layout in (1, 2) and not (0 < extent < n and extent & (extent - 1) == 0):
        _fail(f"compressed unique count must be a power of two smaller than the ring dimension: {extent} vs {n}")
    if layout == 3 and not (0 < extent <= n and extent & (extent - 1) == 0):
        _fail(f"strided plaintext extent must be a power of two dividing the ring dimension: {extent} vs {n}")
    c, pl = _Operand(ct), _Operand(pt)
    if pl.batch not in (1, c.batch):
        _fail(f"plaintext batch {pl.batch} must equal the ciphertext batch {c.batch} or be 1")
    imp_ptr, imp_stride = None, 0
    if layout == 3:
        _same(implicit, ct, "implicit_plaintext")
        if implicit.shape[-1] != rows:
            _fail(f"implicit_plaintext must be [*batch, {rows}], got {tuple(implicit.shape)}")
        im = _Operand(implicit, rows_dims=1)
        if im.batch != pl.batch:
            _fail("implicit_plaintext and strided_plaintext batches differ")
        imp_ptr, imp_stride = im.ptr, (im.stride if im.batch > 1 else 0)
    p, ps = _params(params, ct, rows)
    writable = out is not None
    if out is None:
        out = torch.empty_like(ct, memory_format=torch.contiguous_format)
    o = _Operand(out, writable=writable)
    with torch.cuda.device(ct.device):
        _call("fhb_op_add_plaintext", bits, layout, c.ptr, c.stride, pl.ptr, pl.stride if pl.batch > 1 else 0,
              extent, imp_ptr, imp_stride, o.ptr, o.stride, c.batch, rows, n, p.data_ptr(), ps, _stream(ct))
    o.finish()
    return out


def _plaintext_op(layout: int, inplace: bool):
    if layout == 3:
        def f(ct, strided, implicit, params):
            if inplace:
                _check_writable(ct, "ciphertext_component")
                _no_overlap(ct, strided, implicit, params)
                _add_plaintext(3, ct, strided, params, implicit, out=ct)
                return None
            return _add_plaintext(3, ct, strided, params, implicit)
    else:
        def f(ct, pt, params):
            if inplace:
                _check_writable(ct, "ciphertext_component")
                _no_overlap(ct, pt, params)
                _add_plaintext(layout, ct, pt, params, out=ct)
                return None
            return _add_plaintext(layout, ct, pt, params)
    return f


def _rescale(remaining, inverse_mont, dropped, params, half, nearest, out=None):
    _cuda(remaining, "remaining_residues")
    bits = _bits(remaining, "remaining_residues")
    rows, n = _rows_n(remaining, "remaining_residues")
    _same(dropped, remaining, "dropped_residue")
    _same(inverse_mont, remaining, "drop_prime_inverse_mont")
    if dropped.shape[-1] != n or tuple(dropped.shape[:-1]) != tuple(remaining.shape[:-2]):
        _fail(f"dropped_residue must be [*batch, N] matching remaining_residues, got {tuple(dropped.shape)}")
    if inverse_mont.numel() < rows:
        _fail(f"drop_prime_inverse_mont needs {rows} entries, got {inverse_mont.numel()}")
    p, ps = _params(params, remaining, rows)
    r = _Operand(remaining)
    d = _Operand(dropped, rows_dims=1)
    writable = out is not None
    if out is None:
        out = torch.empty_like(remaining, memory_format=torch.contiguous_format)
    o = _Operand(out, writable=writable)
    inv = inverse_mont.contiguous()
    with torch.cuda.device(remaining.device):
        _call("fhb_op_rescale", bits, r.ptr, r.stride, d.ptr, d.stride, o.ptr, o.stride, r.batch, rows, n,
              inv.data_ptr(), p.data_ptr(), ps, int(half), int(nearest), _stream(remaining))
    o.finish()
    return out


def rescale_drop_leading_prime_nearest(remaining, inverse_mont, dropped, params, half_drop_prime):
    return _rescale(remaining, inverse_mont, dropped, params, half_drop_prime, True)


def rescale_drop_leading_prime_nearest_(remaining, inverse_mont, dropped, params, half_drop_prime):
    _check_writable(remaining, "remaining_residues")
    _no_overlap(remaining, inverse_mont, dropped, params)
    _rescale(remaining, inverse_mont, dropped, params, half_drop_prime, True, out=remaining)


def rescale_drop_leading_prime_truncate(remaining, inverse_mont, dropped, params):
    return _rescale(remaining, inverse_mont, dropped, params, 0, False)


def rescale_drop_leading_prime_truncate_(remaining, inverse_mont, dropped, params):
    _check_writable(remaining, "remaining_residues")
    _no_overlap(remaining, inverse_mont, dropped, params)
    _rescale(remaining, inverse_mont, dropped, params, 0, False, out=remaining)


def _index_map(t: torch.Tensor, n: int, dtype, name: str, ref: torch.Tensor) -> torch.Tensor:
    if t.dtype != dtype:
        _fail(f"{name} must be {dtype}, got {t.dtype}")
    if t.device != ref.device:
        _fail(f"{name} must be on {ref.device}")
    if t.numel() != n:
        _fail(f"{name} must have N = {n} entries, got {t.numel()}")
    return t.contiguous()


def apply_coefficient_galois_automorphism(residues, source_indices, source_sign, twice_modulus):
    _cuda(residues, "residues")
    bits = _bits(residues, "residues")
    rows, n = _rows_n(residues, "residues")
    src = _index_map(source_indices, n, torch.int32, "source_indices", residues)
    sign = _index_map(source_sign, n, torch.int8, "source_sign", residues)
    _same(twice_modulus, residues, "twice_modulus")
    if twice_modulus.numel() != rows:
        _fail(f"twice_modulus must have {rows} entries, got {twice_modulus.numel()}")
    a = _Operand(residues)
    out = torch.empty_like(residues, memory_format=torch.contiguous_format)
    tm = twice_modulus.contiguous()
    with torch.cuda.device(residues.device):
        _call("fhb_op_coefficient_automorphism", bits, a.ptr, a.stride, out.data_ptr(), rows * n, a.batch, rows, n,
              src.data_ptr(), sign.data_ptr(), tm.data_ptr(), _stream(residues))
    return out


def apply_ntt_galois_automorphism(residues, source_indices):
    _cuda(residues, "residues_ntt")
    bits = _bits(residues, "residues_ntt")
    rows, n = _rows_n(residues, "residues_ntt")
    src = _index_map(source_indices, n, torch.int32, "source_indices", residues)
    a = _Operand(residues)
    out = torch.empty_like(residues, memory_format=torch.contiguous_format)
    with torch.cuda.device(residues.device):
        _call("fhb_op_ntt_automorphism", bits, a.ptr, a.stride, out.data_ptr(), rows * n, a.batch, rows, n,
              src.data_ptr(), _stream(residues))
    return out


def keyswitch_moddown_qp_to_q(q_residues, p_residues, inverses, params):
    _cuda(q_residues, "q_residues")
    bits = _bits(q_residues, "q_residues")
    qn, n = _rows_n(q_residues, "q_residues")
    _same(p_residues, q_residues, "p_residues")
    pn, pn_n = _rows_n(p_residues, "p_residues")
    if pn_n != n or tuple(p_residues.shape[:-2]) != tuple(q_residues.shape[:-2]):
        _fail("p_residues must match q_residues in batch and N")
    if not 1 <= pn <= 16:
        _fail(f"ModDown supports 1..16 special primes, got {pn}")
    _same(inverses, q_residues, "moddown_p_drop_inverses_montgomery")
    if inverses.dim() != 2 or inverses.shape[0] < pn or inverses.shape[1] < qn + pn - 1:
        _fail(f"moddown_p_drop_inverses_montgomery must be [{pn}, >= {qn + pn - 1}], got {tuple(inverses.shape)}")
    inv = inverses if inverses.stride(1) == 1 else inverses.contiguous()
    p, ps = _params(params, q_residues, qn + pn)
    qo, po = _Operand(q_residues), _Operand(p_residues)
    out = torch.empty_like(q_residues, memory_format=torch.contiguous_format)
    with torch.cuda.device(q_residues.device):
        _call("fhb_op_moddown", bits, qo.ptr, qo.stride, po.ptr, po.stride, out.data_ptr(), qn * n, qo.batch, qn, pn,
              n, inv.data_ptr(), inv.stride(0), p.data_ptr(), ps, _stream(q_residues))
    return out


def keyswitch_accumulate_digit_products_(acc0, acc1, digit, key_digit, params, key_digit_row_start):
    _cuda(acc0, "accumulator0_qp")
    bits = _bits(acc0, "accumulator0_qp")
    rows, n = _rows_n(acc0, "accumulator0_qp")
    for t, name in ((acc1, "accumulator1_qp"), (digit, "extended_digit_ntt_qp"), (key_digit, "key_switch_key_digit")):
        _same(t, acc0, name)
    if acc1.shape != acc0.shape or digit.shape != acc0.shape:
        _fail("accumulators and digit must have the same shape")
    _check_writable(acc0, "accumulator0_qp")
    _check_writable(acc1, "accumulator1_qp")
    _no_overlap(acc0, acc1, digit, key_digit, params)
    _no_overlap(acc1, digit, key_digit, params)
    start = int(key_digit_row_start)
    if key_digit.dim() != 3 or key_digit.shape[0] != 2 or key_digit.shape[2] != n:
        _fail(f"key_switch_key_digit must be [2, key_rows, N], got {tuple(key_digit.shape)}")
    if start < 0 or start + rows > key_digit.shape[1]:
        _fail(f"key rows [{start}, {start + rows}) exceed the key's {key_digit.shape[1]} rows")
    key = key_digit.contiguous()
    p, ps = _params(params, acc0, rows)
    a0, a1 = _Operand(acc0, writable=True), _Operand(acc1, writable=True)
    d = _Operand(digit)
    with torch.cuda.device(acc0.device):
        _call("fhb_op_keyswitch_accumulate", bits, a0.ptr, a0.stride, a1.ptr, a1.stride, d.ptr, d.stride,
              key.data_ptr(), key.stride(0), start, a0.batch, rows, n, p.data_ptr(), ps, _stream(acc0))
    a0.finish()
    a1.finish()


# --------------------------------------------------------------------------- registration
IMPLS = {
    "fhelium_rns_ops": {
        "montgomery_mul": montgomery_mul, "add_lazy": add_lazy, "sub_lazy": sub_lazy,
        "add_canonical": add_canonical, "add_canonical_": add_canonical_, "sub_canonical": sub_canonical,
        "sub_canonical_": sub_canonical_, "to_montgomery_": to_montgomery_, "from_montgomery_": from_montgomery_,
        "canonicalize_residues_": canonicalize_residues_, "center_residues_": center_residues_,
        "shift_residues_positive_": shift_residues_positive_,
        "lift_centered_coefficients": lift_centered_coefficients,
        "mixed_radix_decompose": mixed_radix_decompose,
        "mixed_radix_basis_extend_to_montgomery": mixed_radix_basis_extend_to_montgomery,
        "montgomery_mul_cyclic_compressed": montgomery_mul_cyclic_compressed,
        "montgomery_mul_contiguous_compressed": montgomery_mul_contiguous_compressed,
        "montgomery_mul_row_scalars_": montgomery_mul_row_scalars_,
        "montgomery_mul_row_scalars_canonical": montgomery_mul_row_scalars_canonical,
        "add_lazy_with_twice_modulus": add_lazy_with_twice_modulus,
    },
    "fhelium_ntt_ops": {
        "forward_ntt_montgomery_indexed_": _fwd_indexed_(1),
        "forward_ntt_to_montgomery_indexed_": _fwd_indexed_(0),
        "forward_ntt_to_montgomery_indexed": forward_ntt_to_montgomery_indexed,
        "forward_ntt_montgomery_compact_grouped_smem_": _fwd_compact_(1),
        "forward_ntt_to_montgomery_compact_grouped_smem_": _fwd_compact_(0),
        "forward_ntt_to_montgomery_compact_grouped_smem": forward_ntt_to_montgomery_compact_grouped_smem,
        "forward_ntt_montgomery_compact_keyswitch_accumulate_": forward_ntt_montgomery_compact_keyswitch_accumulate_,
        "forward_ntt_montgomery_power_of_two_radix_compact_": _fwd_radix_(1),
        "forward_ntt_to_montgomery_power_of_two_radix_compact_": _fwd_radix_(0),
        "forward_ntt_to_montgomery_power_of_two_radix_compact": forward_ntt_to_montgomery_power_of_two_radix_compact,
        "inverse_ntt_montgomery_power_of_two_radix_compact_": _inv_radix_(_native.INV_MONTGOMERY),
        "inverse_ntt_to_standard_lazy_power_of_two_radix_compact_": _inv_radix_(_native.INV_STANDARD_LAZY),
        "inverse_ntt_to_standard_power_of_two_radix_compact_": _inv_radix_(_native.INV_STANDARD),
        "inverse_ntt_to_centered_power_of_two_radix_compact_": _inv_radix_(_native.INV_CENTERED),
        "inverse_ntt_montgomery_indexed_": _inv_indexed_(_native.INV_MONTGOMERY),
        "inverse_ntt_to_standard_lazy_indexed_": _inv_indexed_(_native.INV_STANDARD_LAZY),
        "inverse_ntt_to_standard_indexed_": _inv_indexed_(_native.INV_STANDARD),
        "inverse_ntt_to_centered_indexed_": _inv_indexed_(_native.INV_CENTERED),
        "inverse_ntt_montgomery_compact_grouped_smem_": _inv_compact_(_native.INV_MONTGOMERY),
        "inverse_ntt_to_standard_lazy_compact_grouped_smem_": _inv_compact_(_native.INV_STANDARD_LAZY),
        "inverse_ntt_to_standard_compact_grouped_smem_": _inv_compact_(_native.INV_STANDARD),
        "inverse_ntt_to_centered_compact_grouped_smem_": _inv_compact_(_native.INV_CENTERED),
    },
    "fhelium_ntt_diagnostic_ops": {
        "forward_ntt_montgomery_compact_grouped_smem_override_": forward_ntt_montgomery_compact_grouped_smem_override_,
        "forward_ntt_montgomery_power_of_two_radix_compact_override_": _fwd_radix_(1),
        "inverse_ntt_montgomery_power_of_two_radix_compact_override_": _inv_radix_(_native.INV_MONTGOMERY),
    },
    "fhelium_ckks_ops": {
        "add_prepared_plaintext_component": _plaintext_op(0, False),
        "add_prepared_plaintext_component_": _plaintext_op(0, True),
        "add_cyclic_compressed_plaintext_component": _plaintext_op(1, False),
        "add_cyclic_compressed_plaintext_component_": _plaintext_op(1, True),
        "add_contiguous_compressed_plaintext_component": _plaintext_op(2, False),
        "add_contiguous_compressed_plaintext_component_": _plaintext_op(2, True),
        "add_strided_plaintext_component": _plaintext_op(3, False),
        "add_strided_plaintext_component_": _plaintext_op(3, True),
        "rescale_drop_leading_prime_nearest": rescale_drop_leading_prime_nearest,
        "rescale_drop_leading_prime_nearest_": rescale_drop_leading_prime_nearest_,
        "rescale_drop_leading_prime_truncate": rescale_drop_leading_prime_truncate,
        "rescale_drop_leading_prime_truncate_": rescale_drop_leading_prime_truncate_,
        "apply_coefficient_galois_automorphism": apply_coefficient_galois_automorphism,
        "apply_ntt_galois_automorphism": apply_ntt_galois_automorphism,
        "keyswitch_moddown_qp_to_q": keyswitch_moddown_qp_to_q,
        "keyswitch_accumulate_digit_products_": keyswitch_accumulate_digit_products_,
    },
}


def _defined(ns: str, name: str) -> bool:
    try:
        torch._C._dispatch_find_schema_or_throw(f"{ns}::{name}", "")
        return True
    except RuntimeError:
        return False


def register() -> None:
    """Install the CUDA kernels of every schema in SCHEMAS (idempotent).  Loads
    libfhb200 first, so a missing library fails here, not at the first op."""
    global _registered
    with _lock:
        if _registered:
            return
        _native.load()
        for ns, ops in SCHEMAS.items():
            missing = [name for name in ops if not _defined(ns, name)]
            if missing:
                frag = torch.library.Library(ns, "FRAGMENT")
                for name in missing:
                    frag.define(ops[name])
                _libraries.append(frag)
            lib = torch.library.Library(ns, "IMPL")
            for name in ops:
                lib.impl(name, IMPLS[ns][name], "CUDA")
            _libraries.append(lib)
        _registered = True


def served() -> list[str]:
    """Qualified names of the schemas whose CUDA kernel this module provides."""
    return [f"{ns}::{name}" for ns, ops in SCHEMAS.items() for name in ops]
