"""ctypes binding of libfhb200.so (the C ABI declared in include/fhb200.h).

The library is built in-tree (``python -m fhelium_b200.csrc.build``) and is
the only compute path of the package: there is no CPU or PyTorch fallback.
Loading fails loudly when the library is missing.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libfhb200.so")

# Every exported symbol with (restype, argtypes).
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_U32 = ctypes.c_uint32
class KsItem(ctypes.Structure):
    """fhb_ks_item: one ciphertext's operation in a mixed-level batch."""
    _fields_ = [("kind", ctypes.c_int32), ("level", ctypes.c_int32), ("galois", ctypes.c_uint32),
                ("reserved", ctypes.c_int32), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("key", ctypes.c_void_p), ("out", ctypes.c_void_p)]


class ItemsPlanInfo(ctypes.Structure):
    """fhb_items_plan_info: sizes and counts of a mixed-level batch plan."""
    _fields_ = [("plan_bytes", ctypes.c_int64), ("scratch_bytes", ctypes.c_int64), ("items", ctypes.c_int32),
                ("hmult_items", ctypes.c_int32), ("forward_units", ctypes.c_int32),
                ("inverse_units", ctypes.c_int32), ("core_units", ctypes.c_int32), ("max_limbs", ctypes.c_int32),
                ("max_digits", ctypes.c_int32), ("core_f64_units", ctypes.c_int32)]


ITEM_HMULT_RELIN_RESCALE, ITEM_ROTATE = 0, 1

SIGNATURES: dict[str, tuple] = {
    "fhb_version": (_I, []),
    "fhb_modmul_probe": (_I, [_P, _P, _I, _I, _P]),
    "fhb_modmul_probe_f64": (_I, [_P, _P, _I, _I, _P]),
    "fhb_tc_ntt_prepare": (_I, [_P]),
    "fhb_tc_forward_ntt": (_I, [_P, _P, _P, _I64, _I, _I, _P]),
    "fhb_tc_inverse_ntt": (_I, [_P, _P, _P, _I64, _I, _I, _P]),
    "fhb_tc_ntt_status": (_I, [_P, ctypes.POINTER(_I)]),
    "fhb_tc_basis_extend": (_I, [_P, _P, _P, _I64, _I, _P]),
    "fhb_tc_basis_extend_words": (_I64, [_P, _I64, _I]),
    "fhb_tc_basis_status": (_I, [_P, ctypes.POINTER(_I)]),
    "fhb_tc_ntt_tables_host": (_I, [ctypes.c_uint64, ctypes.c_uint64, _I, _P, _P]),
    "fhb_last_error": (ctypes.c_char_p, []),
    "fhb_context_create": (_I, [_I, _I, ctypes.POINTER(ctypes.c_uint64), _I, _I, _I, ctypes.POINTER(_P)]),
    "fhb_context_destroy": (_I, [_P]),
    "fhb_context_root": (_I, [_P, _I, ctypes.POINTER(ctypes.c_uint64)]),
    "fhb_context_set_tuning": (_I, [_P, _I, _I]),
    "fhb_context_get_tuning": (_I, [_P, _I, ctypes.POINTER(_I)]),
    "fhb_forward_ntt": (_I, [_P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_inverse_ntt": (_I, [_P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_ckks_multiply": (_I, [_P, _P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_multiply_to_coefficient": (_I, [_P, _P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_modup_digits": (_I, [_P, _P, _P, _I64, _I, _U32, _P]),
    "fhb_ckks_keyswitch_core": (_I, [_P, _P, _P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_keyswitch_core_extended": (_I, [_P, _P, _P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_moddown": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I, _U32, _I, _P]),
    "fhb_ckks_prepare_rotation": (_I, [_P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_apply_prepared_rotation": (_I, [_P, _P, _P, _P, _P, _I64, _I, _U32, _P]),
    "fhb_ckks_rescale": (_I, [_P, _P, _P, _I64, _I, _I, _P]),
    "fhb_ckks_automorphism": (_I, [_P, _P, _P, _I64, _I, _I, _U32, _P]),
    "fhb_ckks_add": (_I, [_P, _P, _P, _P, _I64, _I, _I, _P]),
    "fhb_rns_binary": (_I, [_P, _I, _P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_rns_lift_signed": (_I, [_P, _P, _P, _I64, _I, _I, _P]),
    "fhb_ckks_keyswitch_scratch_bytes": (_I64, [_P, _I64, _I]),
    "fhb_ckks_relinearize": (_I, [_P, _P, _P, _P, _P, _I64, _I64, _I, _I, _P]),
    "fhb_ckks_multiply_relinearize": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I, _I, _P]),
    "fhb_ckks_rotate": (_I, [_P, _P, _P, _P, _P, _I64, _I64, _I, _U32, _P]),
    "fhb_ckks_rotate_multi": (_I, [_P, _P, _P, _P, _P, _P, _I64, _I64, _I, _P]),
    "fhb_ckks_keyswitch_sum": (_I, [_P, _P, _P, _P, _P, _I, _I64, _I, _P]),
    "fhb_ckks_keyswitch_sum_extended": (_I, [_P, _P, _P, _P, _P, _I, _I64, _I, _P]),
    "fhb_ckks_decrypt_tail": (_I, [_P, _P, _P, _I64, _I, _P]),
    "fhb_ckks_items_plan_info": (_I, [_P, ctypes.POINTER(KsItem), _I, ctypes.POINTER(ItemsPlanInfo)]),
    "fhb_ckks_items_plan": (_I, [_P, ctypes.POINTER(KsItem), _I, _P, _P, ctypes.POINTER(ItemsPlanInfo)]),
    "fhb_ckks_items_run": (_I, [_P, _P, ctypes.POINTER(ItemsPlanInfo), _P]),
    "fhb_ckks_items_status": (_I, [_P, _P, ctypes.POINTER(ItemsPlanInfo), ctypes.POINTER(ctypes.c_int)]),
    "fhb_ckks_bsgs_inner_product": (_I, [_P, _P, _I64, _P, _I64, _I, _P, _I, _I, _P, _I64, _I64, _I, _I, _P]),
    "fhb_ckks_monomial": (_I, [_P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_ckks_modraise": (_I, [_P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_rns_add_constant": (_I, [_P, _P, _P, _I64, _I, _I, _I, _P]),
    "fhb_ckks_relinearize_noalloc": (_I, [_P, _P, _P, _P, _I64, _I, _I, _P]),
    "fhb_ckks_relinearize_noalloc_max_scratch_bytes": (_I64, []),
    # operator-level entry points (the reference's custom-op schemas)
    "fhb_op_rns_binary": (_I, [_I, _I, _P, _I64, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _I64, _P]),
    "fhb_op_rns_unary": (_I, [_I, _I, _P, _I64, _I64, _I, _I64, _P, _I64, _P]),
    "fhb_op_lift_centered": (_I, [_I, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P]),
    "fhb_op_mixed_radix_decompose": (_I, [_I, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P, _I64, _P, _P, _P, _P,
                                          _P]),
    "fhb_op_basis_extend": (_I, [_I, _P, _I64, _I, _P, _I64, _I64, _I, _I64, _P, _I64, _P, _I64, _P]),
    "fhb_op_keyswitch_accumulate": (_I, [_I, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _I64, _I64, _I, _I64, _P,
                                         _I64, _P]),
    "fhb_op_moddown": (_I, [_I, _P, _I64, _P, _I64, _P, _I64, _I64, _I, _I, _I64, _P, _I64, _P, _I64, _P]),
    "fhb_op_rescale": (_I, [_I, _P, _I64, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P, _I64, _I64, _I, _P]),
    "fhb_op_coefficient_automorphism": (_I, [_I, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P, _P, _P]),
    "fhb_op_ntt_automorphism": (_I, [_I, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P]),
    "fhb_op_mul_compressed": (_I, [_I, _I, _P, _I64, _P, _I64, _I64, _P, _I64, _I64, _I, _I64, _P, _I64, _P]),
    "fhb_op_add_plaintext": (_I, [_I, _I, _P, _I64, _P, _I64, _I64, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _I64,
                                  _P]),
    "fhb_op_mul_row_scalars": (_I, [_I, _P, _I64, _P, _I64, _I64, _I, _I64, _P, _P, _I64, _P]),
    "fhb_context_create_transform": (_I, [_I, _I, ctypes.POINTER(ctypes.c_uint64), _I, _I, ctypes.POINTER(_P)]),
}

(TUNE_KS_ORDER, TUNE_NTT_FORWARD_EPT, TUNE_NTT_INVERSE_EPT, TUNE_BASIS_CONVERSION, TUNE_TC_WAIT_US,
 TUNE_TC_TEST_STALL, TUNE_TC_MODDOWN, TUNE_TC_NTT_FUSED, TUNE_F64_CORE, TUNE_OVERLAP_CHUNKS) = range(10)
BASIS_CUDA_CORES, BASIS_TENSOR_CORES = 0, 1
OP_MONTGOMERY_MUL, OP_ADD_LAZY, OP_SUB_LAZY, OP_ADD_CANONICAL, OP_SUB_CANONICAL, OP_NEGATE = range(6)
INV_MONTGOMERY, INV_STANDARD_LAZY, INV_STANDARD, INV_CENTERED = range(4)


class NativeLibraryError(RuntimeError):
    """libfhb200.so is missing or failed to load."""


class NativeCallError(RuntimeError):
    """A C-ABI call returned a non-zero status."""


_lib = None
_lock = threading.Lock()


def load(path: str | None = None) -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = path or os.environ.get("FHB200_LIB", LIB_PATH)
        if not os.path.exists(path):
            raise NativeLibraryError(
                f"{path} not found: build it with `python -m fhelium_b200.csrc.build` "
                "(fhelium_b200 has no fallback path)")
        try:
            lib = ctypes.CDLL(path)
        except OSError as exc:
            raise NativeLibraryError(f"cannot load {path}: {exc}") from exc
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().fhb_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise NativeCallError(f"{what} failed ({rc}): {last_error()}")


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_of(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class NativeContext:
    """Owns one fhb_context (device tables of a modulus chain)."""

    def __init__(self, residue_bits: int, log_n: int, moduli, num_q: int, num_p: int, device: torch.device):
        lib = load()
        arr = (ctypes.c_uint64 * len(moduli))(*[int(m) for m in moduli])
        handle = _P()
        check(lib.fhb_context_create(residue_bits, log_n, arr, num_q, num_p, device.index or 0,
                                     ctypes.byref(handle)), "fhb_context_create")
        self.handle = handle
        self.lib = lib
        self.device = device

    @classmethod
    def transform(cls, residue_bits: int, log_n: int, moduli, device: torch.device) -> "NativeContext":
        """A context whose prime ids 0..len(moduli)-1 are exactly `moduli`, for
        the transforms and element-wise entry points (fhb_context_create_transform)."""
        self = cls.__new__(cls)
        lib = load()
        arr = (ctypes.c_uint64 * len(moduli))(*[int(m) for m in moduli])
        handle = _P()
        check(lib.fhb_context_create_transform(residue_bits, log_n, arr, len(moduli), device.index or 0,
                                               ctypes.byref(handle)), "fhb_context_create_transform")
        self.handle, self.lib, self.device = handle, lib, device
        return self

    def root(self, prime_id: int) -> int:
        out = ctypes.c_uint64()
        check(self.lib.fhb_context_root(self.handle, prime_id, ctypes.byref(out)), "fhb_context_root")
        return int(out.value)

    def set_tuning(self, param: int, value: int) -> None:
        check(self.lib.fhb_context_set_tuning(self.handle, param, value), "fhb_context_set_tuning")

    def get_tuning(self, param: int) -> int:
        out = ctypes.c_int()
        check(self.lib.fhb_context_get_tuning(self.handle, param, ctypes.byref(out)), "fhb_context_get_tuning")
        return int(out.value)

    def call(self, name: str, *args) -> None:
        check(getattr(self.lib, name)(self.handle, *args), name)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.fhb_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
