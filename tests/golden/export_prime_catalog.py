"""Export the reference's packaged prime catalog to ``prime_catalog_v1.json``.

The CKKS preset moduli must be the very same primes the reference selects, so
the catalog is data shared with the reference, not something re-derived here.
This script reads the reference's two safetensors resources
(``fhelium/config/resources/{scale,message}_primes_v1.safetensors``) and
writes them as plain JSON keyed ``"<bits>:<ring_dimension>"`` into the
package's data folder (``fhelium_b200/data/prime_catalog_v1.json``).  It is
run once, in a checkout that has the reference sources; the package only
reads the JSON and does not ship this script.
"""

from __future__ import annotations

import json
import os
import sys

from safetensors import safe_open

REFERENCE = os.environ.get("FHELIUM_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(os.path.dirname(HERE)), "fhelium_b200", "data")


def _table(name: str) -> dict:
    path = os.path.join(REFERENCE, "fhelium", "config", "resources", name)
    out = {}
    with safe_open(path, framework="pt", device="cpu") as handle:
        for key in handle.keys():
            fields = dict(part.split("=", 1) for part in key.split(";"))
            out[f"{int(fields['sb'])}:{int(fields['N'])}"] = [
                int(v) for v in handle.get_tensor(key).tolist()
            ]
    return dict(sorted(out.items(), key=lambda kv: tuple(map(int, kv[0].split(":")))))


def main() -> int:
    catalog = {
        "version": 1,
        "scale": _table("scale_primes_v1.safetensors"),
        "message": _table("message_primes_v1.safetensors"),
    }
    with open(os.path.join(DATA, "prime_catalog_v1.json"), "w") as fh:
        json.dump(catalog, fh, separators=(",", ":"))
        fh.write("\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
