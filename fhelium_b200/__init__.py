"""B200-native (sm_100a) CKKS evaluation path with the fhelium CkksEngine API."""

from .config import CkksConfig, Preset
from .values import (Ciphertext, KeySwitchKey, PublicKey, RelinearizationKey, RotationKey, RotationKeySet,
                     SecretKey)

__all__ = ["CkksConfig", "Preset", "CkksEngine", "Ciphertext", "SecretKey", "PublicKey", "KeySwitchKey",
           "RelinearizationKey", "RotationKey", "RotationKeySet"]


def __getattr__(name):
    if name == "CkksEngine":
        from .engine import CkksEngine
        return CkksEngine
    raise AttributeError(name)
