"""B200-native (sm_100a) CKKS evaluation path with the fhelium CkksEngine API.

The names a user of the reference reaches as ``fh.<name>`` (fhelium/__init__.py)
for the evaluation path: the engine, configuration, value and key types, the
state literals and the value-file functions."""

from typing import Literal

from .config import CkksConfig, Preset
from .values import (COMPRESSED_PLAINTEXT_FORMAT_VERSION, Ciphertext, CompressedPlaintext, EncryptionDraws,
                     EvaluationKeyRequirements, EvaluationKeySet, KeySwitchKey, KeySwitchKeyDraws, Plaintext, PublicKey, RelinearizationKey, RotationKey,
                     RotationKeySet, SecretKey)

# state literals (fhelium/core/state.py:10-21)
PlaintextRepresentation = Literal["slots", "integer_coefficients", "approximate_coefficients", "rns"]
PolynomialDomain = Literal["coefficient", "ntt"]
ModulusBasis = Literal["Q", "QP"]
ResidueRepresentation = Literal["standard", "montgomery"]
CompressedPlaintextLayout = Literal["cyclic", "contiguous", "strided_sparse"]

# A conjugation key is the Galois key of g = 2N - 1 (CkksEngine.create_conjugation_key).
ConjugationKey = RotationKey

__all__ = ["CkksConfig", "Preset", "CkksEngine", "Ciphertext", "Plaintext", "CompressedPlaintext",
           "CompressedPlaintextLayout", "COMPRESSED_PLAINTEXT_FORMAT_VERSION", "SecretKey", "PublicKey",
           "KeySwitchKey", "RelinearizationKey", "RotationKey", "ConjugationKey", "RotationKeySet",
           "EvaluationKeySet", "EvaluationKeyRequirements", "EncryptionDraws",
           "KeySwitchKeyDraws",
           "PlaintextRepresentation", "PolynomialDomain", "ModulusBasis", "ResidueRepresentation",
           "save_value", "load_value", "inspect_value"]


def __getattr__(name):
    if name == "CkksEngine":
        from .engine import CkksEngine
        return CkksEngine
    if name in ("save_value", "load_value", "inspect_value"):
        from . import serialization
        return getattr(serialization, name)
    raise AttributeError(name)
