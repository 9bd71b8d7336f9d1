"""Value files interchangeable with the reference's (no GPU).

tests/golden/values/*.safetensors were written by the reference's own
fhelium.serialization.save_value (tests/golden/make_value_files.py).  Each
must load with fhelium_b200.serialization with the same residues and
metadata, and writing the loaded value back must reproduce the file's header
metadata (the manifest text included) and payload exactly; the context id
must match the reference's hash of the preset."""

import os
import shutil

import pytest
import torch
from safetensors import safe_open

from fhelium_b200 import serialization as ser
from fhelium_b200.config import CkksConfig
from fhelium_b200.values import Ciphertext, PublicKey, RelinearizationKey, RotationKey, SecretKey

HERE = os.path.dirname(os.path.abspath(__file__))
VALUES = os.path.join(HERE, "golden", "values")
FILES = {"ciphertext": Ciphertext, "public_key": PublicKey, "secret_key": SecretKey,
         "relinearization_key": RelinearizationKey, "rotation_key": RotationKey}
CID = ser.context_id(CkksConfig.parse("slots8192_scale40_levels7_int64"))


def _payload(path):
    with safe_open(path, framework="pt", device="cpu") as h:
        return h.get_tensor("data")


@pytest.mark.parametrize("name", sorted(FILES))
def test_reference_files_load_and_round_trip(name, tmp_path):
    path = os.path.join(VALUES, name + ".safetensors")
    manifest = ser.inspect_value(path)
    assert manifest["context_id"] == CID  # the reference's context hash, reproduced
    value = ser.load_value(path, expected_type=FILES[name], expected_context_id=CID)
    assert type(value) is FILES[name]
    assert torch.equal(value.data, _payload(path))
    if name == "ciphertext":
        assert (value.level, value.scale) == (5, 2.0 ** 40)
        assert (value.polynomial_domain, value.residue_representation, value.modulus_basis) == ("ntt", "montgomery",
                                                                                               "Q")
    if name == "rotation_key":
        assert value.rotation_step == 3
    out = tmp_path / (name + ".safetensors")
    written = ser.save_value(value, out, context_id=CID, allow_secret=True)
    assert written == manifest
    # same header metadata strings (manifest text included) and payload; the
    # safetensors writer orders header keys differently from run to run, so
    # the files are compared entry by entry rather than byte by byte
    with safe_open(str(out), framework="pt", device="cpu") as a, safe_open(path, framework="pt", device="cpu") as b:
        assert a.metadata() == b.metadata()
        assert list(a.keys()) == list(b.keys()) == ["data"]
        assert torch.equal(a.get_tensor("data"), b.get_tensor("data"))


def test_save_refuses_secret_keys_and_existing_files(tmp_path):
    sk = ser.load_value(os.path.join(VALUES, "secret_key.safetensors"))
    with pytest.raises(PermissionError):
        ser.save_value(sk, tmp_path / "sk.safetensors", context_id=CID)
    ct = ser.load_value(os.path.join(VALUES, "ciphertext.safetensors"))
    ser.save_value(ct, tmp_path / "ct.safetensors", context_id=CID)
    with pytest.raises(FileExistsError):
        ser.save_value(ct, tmp_path / "ct.safetensors", context_id=CID)
    ser.save_value(ct, tmp_path / "ct.safetensors", context_id=CID, overwrite=True)


def test_load_rejects_mismatches(tmp_path):
    path = os.path.join(VALUES, "ciphertext.safetensors")
    with pytest.raises(ValueError):
        ser.load_value(path, expected_context_id="0" * 64)
    with pytest.raises(TypeError):
        ser.load_value(path, expected_type=RotationKey)
    # a manifest that lies about the shape is refused before the payload is used
    from safetensors.torch import save_file
    import json
    with safe_open(path, framework="pt", device="cpu") as h:
        meta = dict(h.metadata())
        data = h.get_tensor("data")
    manifest = json.loads(meta["fhelium.manifest"])
    manifest["tensor_metadata"]["data"]["shape"][-1] = 8
    bad = dict(meta, **{"fhelium.manifest": json.dumps(manifest, sort_keys=True, separators=(",", ":"))})
    save_file({"data": data}, str(tmp_path / "bad.safetensors"), metadata=bad)
    with pytest.raises(ValueError):
        ser.load_value(tmp_path / "bad.safetensors")
    wrong = dict(meta, **{"fhelium.format": "something-else"})
    save_file({"data": data}, str(tmp_path / "wrong.safetensors"), metadata=wrong)
    with pytest.raises(ValueError):
        ser.inspect_value(tmp_path / "wrong.safetensors")
    shutil.copy(path, tmp_path / "ok.safetensors")
    assert ser.load_value(tmp_path / "ok.safetensors").level == 5


def test_engine_context_id_matches_the_files():
    from fhelium_b200.engine import CkksEngine
    eng = CkksEngine.__new__(CkksEngine)  # context id needs only the parameters
    eng.config = CkksConfig.parse("slots8192_scale40_levels7_int64")
    eng.galois_generator = 3
    assert eng.context_id == CID


def test_top_level_names_match_the_reference_namespace():
    """fh.<name> for the evaluation path (fhelium/__init__.py __all__)."""
    import fhelium_b200 as fh
    for name in ("CkksConfig", "Preset", "Ciphertext", "Plaintext", "SecretKey", "PublicKey", "KeySwitchKey",
                 "RelinearizationKey", "RotationKey", "ConjugationKey", "RotationKeySet", "ModulusBasis",
                 "PolynomialDomain", "ResidueRepresentation", "PlaintextRepresentation", "save_value", "load_value",
                 "inspect_value"):
        assert getattr(fh, name) is not None, name


@pytest.mark.parametrize("layout", ["cyclic", "contiguous", "strided_sparse"])
def test_compressed_plaintext_round_trip(layout):
    """CompressedPlaintext.from_plaintext / decompress_data are exact inverses
    on representable data and reject the rest (fhelium/core/compressed_plaintext.py:244-366)."""
    from fhelium_b200.values import CompressedPlaintext, Plaintext
    g = torch.Generator().manual_seed(1)
    compact = torch.randint(0, 1000, (2, 3, 8), generator=g)
    implicit = torch.randint(0, 1000, (2, 3), generator=g) if layout == "strided_sparse" else None
    cp = CompressedPlaintext(data=compact, ring_dimension=64, compression_layout=layout, level=0, scale=2.0,
                             context_id="c", polynomial_domain="ntt", modulus_basis="Q",
                             residue_representation="montgomery", prime_ids=(0, 1, 2), implicit_data=implicit)
    dense = cp.to_plaintext()
    assert dense.data.shape == (2, 3, 64)
    back = CompressedPlaintext.from_plaintext(dense, unique_count=8, compression_layout=layout)
    assert torch.equal(back.data, compact)
    if implicit is not None:
        assert torch.equal(back.implicit_data, implicit)
    broken = dense.clone()
    broken.data[0, 0, 5] += 1
    with pytest.raises(ValueError, match="not exactly representable"):
        CompressedPlaintext.from_plaintext(broken, unique_count=8, compression_layout=layout)


def test_ciphertext_batch_and_limb_helpers():
    """Ciphertext.select_batch / unbind_batch / stack_batch / slice_limbs /
    with_data / replace_ (fhelium/core/ciphertext.py:221-373)."""
    data = torch.arange(2 * 3 * 4 * 8, dtype=torch.int64).reshape(2, 3, 4, 8)
    ct = Ciphertext(data, 2, 4.0, "ntt", "montgomery")
    assert ct.is_batched and ct.is_ntt_domain and not ct.includes_p and ct.ring_dimension == 8
    assert ct.limb_ids == (2, 3, 4, 5)
    items = ct.unbind_batch()
    assert len(items) == 3 and torch.equal(items[1].data, data[:, 1])
    again = Ciphertext.stack_batch(items)
    assert torch.equal(again.data, data) and again.level == 2
    part = ct.slice_limbs(1, 3)
    assert part.level == 3 and torch.equal(part.data, data[..., 1:3, :])
    other = ct.with_data(data + 1)
    assert torch.equal(other.data, data + 1) and other.scale == 4.0
    target = Ciphertext(torch.zeros(2, 4, 8, dtype=torch.int64), 0, 1.0)
    assert target.replace_(items[0]) is target and target.level == 2 and target.is_ntt_domain
    with pytest.raises(ValueError):
        Ciphertext(data, 0, 1.0, "frequency")


def test_rotation_steps_and_evaluation_key_sets():
    """Signed canonical rotation steps and key inventories as the reference
    defines them (fhelium/core/keys.py:339-351, 396-640)."""
    from fhelium_b200.values import EvaluationKeyRequirements, EvaluationKeySet, RelinearizationKey, RotationKeySet
    n = 64                                          # 32 slots: canonical steps in [-16, 16)
    assert [RotationKeySet.canonical(s, n) for s in (1, -1, 31, 16, -16, 32, 17)] == [1, -1, -1, -16, -16, 0, -15]
    key = lambda step: RotationKey(torch.zeros(2, 2, 3, n, dtype=torch.int64), rotation_step=step, galois_element=3)
    rs = RotationKeySet().add(key(1)).add(key(-1))
    assert sorted(rs) == [-1, 1] and len(rs) == 2
    with pytest.raises(TypeError):
        rs[2] = "not a key"
    ks = EvaluationKeySet(rotations=rs, relinearization=RelinearizationKey(torch.zeros(2, 2, 3, n, dtype=torch.int64)))
    ks.require(EvaluationKeyRequirements(rotation_steps={1, 31, 0}, requires_relinearization=True))
    with pytest.raises(ValueError, match="missing rotation steps: \\[2\\]"):
        ks.require(EvaluationKeyRequirements(rotation_steps={2}))
    with pytest.raises(ValueError, match="conjugation"):
        ks.require(EvaluationKeyRequirements(requires_conjugation=True))
    bad = RotationKeySet()
    bad.keys[5] = key(1)                            # mapping and key disagree
    with pytest.raises(ValueError, match="does not match"):
        EvaluationKeySet(rotations=bad)
