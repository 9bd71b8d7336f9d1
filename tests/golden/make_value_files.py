"""Write value files with the reference's own serializer (fixtures).

Run in a checkout where the reference sources exist (FHELIUM_REFERENCE,
default /root/reference):

    python tests/golden/make_value_files.py

Each file is one small value (ring dimension 16, seeded residues) saved by the
reference's fhelium.serialization.save_value: a ciphertext, a public key, a
secret key, a relinearization key and a rotation key, all under the context
id of preset slots8192_scale40_levels7_int64.  tests/test_serialization.py
reads them with fhelium_b200.serialization and checks that writing the same
values back produces identical files.
"""

from __future__ import annotations

import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("FHELIUM_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "values")


def main() -> None:
    sys.path.insert(0, REFERENCE)
    from fhelium.core import Ciphertext, PublicKey, RelinearizationKey, RotationKey, SecretKey
    from fhelium.core.context import CkksContextSpec
    from fhelium.serialization import save_value

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from fhelium_b200.config import CkksConfig

    cfg = CkksConfig.parse("slots8192_scale40_levels7_int64")
    spec = CkksContextSpec(logN=cfg.logN, default_scale=float(cfg.default_scale),
                           q_moduli=tuple(cfg.moduli[:cfg.num_q_primes]),
                           p_moduli=tuple(cfg.moduli[cfg.num_q_primes:]), galois_generator=3)
    cid = spec.context_id
    g = torch.Generator().manual_seed(7)
    res = lambda *shape: torch.randint(0, 1 << 59, shape, generator=g, dtype=torch.int64)
    qp = cfg.num_q_primes + cfg.num_p_primes
    values = {
        "ciphertext": Ciphertext(res(2, 1, 3, 16), 5, 2.0 ** 40, cid, (5, 6, 7), "ntt", "Q", "montgomery"),
        "public_key": PublicKey(res(2, cfg.num_q_primes, 16), cid, tuple(range(cfg.num_q_primes)), "ntt", "Q",
                                "montgomery"),
        "secret_key": SecretKey(res(qp, 16), cid, tuple(range(qp)), "ntt", "QP", "montgomery"),
        "relinearization_key": RelinearizationKey(res(2, 2, qp, 16), cid, tuple(range(qp)), "ntt", "QP",
                                                  "montgomery"),
        "rotation_key": RotationKey(res(2, 2, qp, 16), cid, tuple(range(qp)), "ntt", "QP", "montgomery",
                                    rotation_step=3),
    }
    os.makedirs(OUT, exist_ok=True)
    for name, value in values.items():
        save_value(value, os.path.join(OUT, name + ".safetensors"), allow_secret=True, overwrite=True)
    print("wrote", sorted(values), "context", cid)


if __name__ == "__main__":
    main()
