"""Value files interchangeable with the reference's (safetensors + manifest).

A value file is one safetensors file whose header metadata carries three
strings: the format tag "fhelium-value", the file schema version "1", and a
JSON manifest (sorted keys, compact separators) describing the value:

    {"context_id": ..., "file_schema_version": 1, "nbytes": ...,
     "tensor_metadata": {name: {"dtype": "torch.int64", "encoding": "direct",
                                "payloads": [name], "shape": [...]}},
     "value_metadata": {...}, "value_schema_version": 2, "value_type": ...}

This is the layout of the reference's fhelium.serialization.save_value /
load_value (fhelium/serialization/safetensors.py:22-131, value.py:33-183),
so files move between the two libraries: a ciphertext or key written by one
loads in the other with the same residues and metadata, and writing a value
back gives the same header metadata (manifest text included) and payload.
The context id is the reference's SHA-256 of the context parameters
(fhelium/core/context.py:72-83); values record it so that a file cannot be
applied under different moduli.

Supported value types: Ciphertext, PublicKey, SecretKey, RelinearizationKey,
RotationKey.  Residue tensors keep the layouts of fhelium_b200.values (limb j
of a level-l ciphertext is prime id l + j; keys hold the level-zero rows), so
prime ids are implied on save and checked on load.
"""

from __future__ import annotations

import json
import math
import os
import tempfile
from hashlib import sha256
from pathlib import Path
from typing import Any

import torch

from .values import Ciphertext, KeySwitchKey, PublicKey, RelinearizationKey, RotationKey, SecretKey

FILE_FORMAT = "fhelium-value"
FILE_SCHEMA_VERSION = 1
VALUE_SCHEMA_VERSION = 2
_FORMAT_KEY = "fhelium.format"
_SCHEMA_KEY = "fhelium.schema_version"
_MANIFEST_KEY = "fhelium.manifest"
_MANIFEST_FIELDS = {"file_schema_version", "value_schema_version", "value_type", "context_id", "nbytes",
                    "tensor_metadata", "value_metadata"}
_SAFETENSORS_DTYPE = {"torch.int64": "I64", "torch.int32": "I32", "torch.uint64": "U64", "torch.uint32": "U32",
                      "torch.float64": "F64", "torch.float32": "F32", "torch.complex128": "F64",
                      "torch.complex64": "F32"}
_TYPES = {"Ciphertext": Ciphertext, "PublicKey": PublicKey, "SecretKey": SecretKey,
          "RelinearizationKey": RelinearizationKey, "RotationKey": RotationKey}


def context_id(config, galois_generator: int = 3) -> str:
    """The reference's identity of a CKKS context: SHA-256 over its
    representation tag, ring degree, default scale, Q and P moduli and Galois
    generator."""
    q = ",".join(str(int(m)) for m in config.moduli[:config.num_q_primes])
    p = ",".join(str(int(m)) for m in config.moduli[config.num_q_primes:])
    payload = (f"representation=direct_per_value_scale_v1;logN={config.logN};"
               f"default_scale={float(config.default_scale)!r};Q={q};P={p};galois_generator={galois_generator}")
    return sha256(payload.encode("utf-8")).hexdigest()


# --------------------------------------------------------------- describe ---
def _describe(value) -> tuple[str, dict[str, Any], torch.Tensor]:
    if isinstance(value, Ciphertext):
        limbs = value.data.size(-2)
        return "Ciphertext", {
            "level": int(value.level), "scale": float(value.scale),
            "prime_ids": list(range(value.level, value.level + limbs)),
            "polynomial_domain": value.polynomial_domain, "modulus_basis": value.modulus_basis,
            "residue_representation": value.residue_representation}, value.data
    if isinstance(value, (RelinearizationKey, RotationKey)) or type(value) is KeySwitchKey:
        if type(value) is KeySwitchKey:
            raise TypeError("save a RelinearizationKey or RotationKey, not a bare KeySwitchKey")
        meta = {"prime_ids": list(range(value.data.size(-2))), "polynomial_domain": "ntt", "modulus_basis": "QP",
                "residue_representation": "montgomery"}
        if isinstance(value, RotationKey):
            meta["rotation_step"] = int(value.rotation_step)
        return type(value).__name__, meta, value.data
    if isinstance(value, PublicKey):
        return "PublicKey", {"prime_ids": list(range(value.data.size(-2))), "polynomial_domain": "ntt",
                             "modulus_basis": "Q", "residue_representation": "montgomery"}, value.data
    if isinstance(value, SecretKey):
        return "SecretKey", {"prime_ids": list(range(value.data.size(-2))), "polynomial_domain": "ntt",
                             "modulus_basis": "QP", "residue_representation": "montgomery"}, value.data
    raise TypeError(f"value files hold {sorted(_TYPES)}; got {type(value).__name__}")


def save_value(value, path: str | os.PathLike, *, context_id: str, allow_secret: bool = False,
               overwrite: bool = False) -> dict:
    """Write `value` to `path` atomically (temporary file + rename, mode 0600)
    and return its manifest.  A SecretKey needs allow_secret=True (the file is
    not encrypted); an existing file needs overwrite=True."""
    from safetensors.torch import save_file

    value_type, meta, data = _describe(value)
    if value_type == "SecretKey" and not allow_secret:
        raise PermissionError("SecretKey files are refused unless allow_secret=True (the file is not encrypted)")
    if not isinstance(context_id, str) or not context_id:
        raise ValueError("context_id must be a non-empty string")
    dest = Path(path).expanduser()
    if not dest.parent.is_dir():
        raise FileNotFoundError(f"no directory {dest.parent}")
    if dest.exists() and (dest.is_dir() or not overwrite):
        raise FileExistsError(dest)
    tensor = data.detach().to("cpu").contiguous()
    manifest = {
        "file_schema_version": FILE_SCHEMA_VERSION, "value_schema_version": VALUE_SCHEMA_VERSION,
        "value_type": value_type, "context_id": context_id, "nbytes": tensor.numel() * tensor.element_size(),
        "tensor_metadata": {"data": {"shape": list(tensor.shape), "dtype": str(tensor.dtype), "encoding": "direct",
                                     "payloads": ["data"]}},
        "value_metadata": meta,
    }
    _check_manifest(manifest)
    header = {_FORMAT_KEY: FILE_FORMAT, _SCHEMA_KEY: str(FILE_SCHEMA_VERSION),
              _MANIFEST_KEY: json.dumps(manifest, sort_keys=True, separators=(",", ":"))}
    fd, tmp = tempfile.mkstemp(prefix=f".{dest.name}.", suffix=".tmp", dir=dest.parent)
    os.close(fd)
    try:
        save_file({"data": tensor}, tmp, metadata=header)
        os.chmod(tmp, 0o600)
        if dest.exists() and not overwrite:
            raise FileExistsError(dest)
        os.replace(tmp, dest)
    except BaseException:
        Path(tmp).unlink(missing_ok=True)
        raise
    return manifest


# --------------------------------------------------------------- validate ---
def _check_manifest(m: dict) -> None:
    if not isinstance(m, dict):
        raise ValueError("value file manifest must be a JSON object")
    if set(m) != _MANIFEST_FIELDS:
        raise ValueError(f"value file manifest fields differ: missing {sorted(_MANIFEST_FIELDS - set(m))}, "
                         f"unexpected {sorted(set(m) - _MANIFEST_FIELDS)}")
    if m["file_schema_version"] != FILE_SCHEMA_VERSION or type(m["file_schema_version"]) is not int:
        raise ValueError(f"unsupported value file schema version {m['file_schema_version']!r}")
    if m["value_schema_version"] != VALUE_SCHEMA_VERSION or type(m["value_schema_version"]) is not int:
        raise ValueError(f"unsupported value schema version {m['value_schema_version']!r}")
    if m["value_type"] not in _TYPES:
        raise ValueError(f"unsupported value type {m['value_type']!r}")
    if not isinstance(m["context_id"], str):
        raise ValueError("value file context_id must be a string")
    if type(m["nbytes"]) is not int or m["nbytes"] < 0:
        raise ValueError("value file nbytes must be a non-negative integer")
    tmeta, vmeta = m["tensor_metadata"], m["value_metadata"]
    if not isinstance(tmeta, dict) or not isinstance(vmeta, dict):
        raise ValueError("value file metadata fields must be JSON objects")
    if set(tmeta) != {"data"}:
        raise ValueError(f"{m['value_type']} holds exactly one tensor 'data'")
    item = tmeta["data"]
    if set(item) != {"shape", "dtype", "encoding", "payloads"} or item["encoding"] not in ("direct",) or \
            item["payloads"] != ["data"] or item["dtype"] not in _SAFETENSORS_DTYPE or \
            not isinstance(item["shape"], list) or any(type(d) is not int or d < 0 for d in item["shape"]):
        raise ValueError(f"invalid tensor metadata {item!r}")
    if "int" not in item["dtype"]:
        raise ValueError("residue tensors must be integral")
    _check_value_metadata(m["value_type"], vmeta, item["shape"])


def _check_value_metadata(value_type: str, vm: dict, shape: list) -> None:
    fields = {"prime_ids", "polynomial_domain", "modulus_basis", "residue_representation"}
    if value_type == "Ciphertext":
        fields |= {"level", "scale"}
    if value_type == "RotationKey":
        fields |= {"rotation_step"}
    if set(vm) != fields:
        raise ValueError(f"{value_type} metadata fields differ from {sorted(fields)}")
    dom, basis, rep = vm["polynomial_domain"], vm["modulus_basis"], vm["residue_representation"]
    if dom not in ("coefficient", "ntt") or basis not in ("Q", "QP") or rep not in ("standard", "montgomery"):
        raise ValueError(f"unsupported {value_type} representation {dom}/{basis}/{rep}")
    if dom == "ntt" and rep != "montgomery":
        raise ValueError(f"NTT-domain {value_type} requires Montgomery residues")
    ids = vm["prime_ids"]
    if not isinstance(ids, list) or not ids or any(type(i) is not int or i < 0 for i in ids) or \
            any(a >= b for a, b in zip(ids, ids[1:])):
        raise ValueError(f"{value_type} prime_ids must be a non-empty strictly increasing list")
    if value_type == "Ciphertext":
        if type(vm["level"]) is not int or vm["level"] < 0:
            raise ValueError("Ciphertext level must be a non-negative integer")
        s = vm["scale"]
        if isinstance(s, bool) or not isinstance(s, (int, float)) or not math.isfinite(float(s)) or float(s) <= 0:
            raise ValueError("Ciphertext scale must be finite and positive")
        if dom == "coefficient" and rep != "standard":
            raise ValueError("coefficient-domain Ciphertext requires standard residues")
        if len(shape) < 3 or shape[0] not in (2, 3):
            raise ValueError("Ciphertext data must be [component(2|3), *batch, limb, N]")
    if value_type == "RotationKey" and type(vm["rotation_step"]) is not int:
        raise ValueError("RotationKey rotation_step must be an integer")
    ndim = {"Ciphertext": None, "PublicKey": 3, "SecretKey": 2, "RelinearizationKey": 4, "RotationKey": 4}[value_type]
    if ndim is not None and len(shape) != ndim:
        raise ValueError(f"{value_type} data must have {ndim} dimensions")
    if len(shape) < 2 or shape[-2] != len(ids):
        raise ValueError(f"{value_type} limb count does not match prime_ids")


def _read_manifest(handle) -> dict:
    raw = handle.metadata()
    if raw is None:
        raise ValueError("value file has no safetensors metadata")
    if raw.get(_FORMAT_KEY) != FILE_FORMAT:
        raise ValueError(f"unsupported value file format {raw.get(_FORMAT_KEY)!r}")
    if raw.get(_SCHEMA_KEY) != str(FILE_SCHEMA_VERSION):
        raise ValueError(f"unsupported value file schema version {raw.get(_SCHEMA_KEY)!r}")
    if _MANIFEST_KEY not in raw:
        raise ValueError("value file has no manifest")
    try:
        manifest = json.loads(raw[_MANIFEST_KEY])
    except json.JSONDecodeError as exc:
        raise ValueError("value file manifest is not valid JSON") from exc
    _check_manifest(manifest)
    if set(handle.keys()) != {"data"}:
        raise ValueError(f"value file payloads {sorted(handle.keys())} differ from its manifest")
    item = manifest["tensor_metadata"]["data"]
    sl = handle.get_slice("data")
    if list(sl.get_shape()) != item["shape"] or sl.get_dtype() != _SAFETENSORS_DTYPE[item["dtype"]]:
        raise ValueError("value file payload header does not match its manifest")
    return manifest


def inspect_value(path: str | os.PathLike) -> dict:
    """The validated manifest of a value file, without reading its payload."""
    from safetensors import safe_open

    src = Path(path).expanduser()
    if not src.is_file():
        raise FileNotFoundError(f"no value file at {src}")
    with safe_open(str(src), framework="pt", device="cpu") as handle:
        return _read_manifest(handle)


def load_value(path: str | os.PathLike, *, device: torch.device | str = "cpu", expected_type: type | None = None,
               expected_context_id: str | None = None):
    """Read a value file into the matching fhelium_b200.values type on
    `device`.  Prime ids must be the ones this library's layouts imply
    (contiguous from the ciphertext's level; all level-zero rows for keys)."""
    from safetensors import safe_open

    src = Path(path).expanduser()
    if not src.is_file():
        raise FileNotFoundError(f"no value file at {src}")
    with safe_open(str(src), framework="pt", device="cpu") as handle:
        m = _read_manifest(handle)
        data = handle.get_tensor("data")
    if expected_context_id is not None and m["context_id"] != expected_context_id:
        raise ValueError(f"value file context {m['context_id']!r} differs from {expected_context_id!r}")
    vtype = m["value_type"]
    if expected_type is not None and vtype != expected_type.__name__:
        raise TypeError(f"value file holds a {vtype}, expected {expected_type.__name__}")
    if data.numel() * data.element_size() != m["nbytes"]:
        raise ValueError("value file byte count differs from its manifest")
    vm = m["value_metadata"]
    ids = vm["prime_ids"]
    data = data.to(device)
    if vtype == "Ciphertext":
        if ids != list(range(vm["level"], vm["level"] + len(ids))):
            raise ValueError("Ciphertext prime_ids must run contiguously from its level")
        return Ciphertext(data, vm["level"], float(vm["scale"]), vm["polynomial_domain"],
                          vm["residue_representation"], vm["modulus_basis"], context_id=m.get("context_id"),
                          prime_ids=tuple(ids))
    if ids != list(range(len(ids))):
        raise ValueError(f"{vtype} prime_ids must be the level-zero rows 0..{len(ids) - 1}")
    if vm["polynomial_domain"] != "ntt" or vm["residue_representation"] != "montgomery":
        raise ValueError(f"{vtype} must be NTT-domain Montgomery residues")
    if vtype == "RotationKey":
        return RotationKey(data, rotation_step=vm["rotation_step"])
    return _TYPES[vtype](data)
