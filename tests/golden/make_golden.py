"""Generate engine-level golden digests by running the reference itself.

Run in a checkout where the reference sources exist (FHELIUM_REFERENCE,
default /root/reference) after `bash oracle/build_ref.sh`:

    python tests/golden/make_golden.py [names of the fixtures to regenerate]

It copies the reference's Python package to a scratch directory, installs the
reference's CPU operators compiled from its own sources (oracle/_ref) as the
package's native extension, and drives the reference's public CkksEngine on
CPU.  The reference needs the external `triton_csprng` package only to
construct its random-number adapter; a stand-in module that refuses to
sample is provided, because every input here (ciphertexts and key material)
is injected from the seeded generator in inputs.py.  Outputs are recorded
as SHA-256 digests of their canonical residues (plus a few leading values),
so the fixture stays small; tests rebuild the same inputs and compare.
"""

from __future__ import annotations

import json
import os
import shutil
import sys
import sysconfig
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from inputs import (canonical, client_inputs, digest, float_digest, key_draws, key_material,  # noqa: E402
                    residues)

REFERENCE = os.environ.get("FHELIUM_REFERENCE", "/root/reference")
REF_OPS = os.path.join(ROOT, "oracle", "_ref", "libfhelium_ref_cpu_ops.so")

STUB = '''
class _Refuse:
    def __getattr__(self, name):
        raise RuntimeError("golden generation must not sample randomness")

class RnsRandomStreams:
    def __init__(self, **kw):
        self.key_words = [0] * 8
        self.nonce_words = [0, 0]
        self._device_streams = [_Refuse()]
        self._repeat_streams = [_Refuse()]
    def randint_channels(self, *a, **k):
        raise RuntimeError("golden generation must not sample randomness")
    def discrete_gaussian_channels(self, *a, **k):
        raise RuntimeError("golden generation must not sample randomness")

class ChaCha20Rng:
    def __init__(self, **kw):
        pass
    def stochastic_round(self, *a, **k):
        raise RuntimeError("golden generation must not sample randomness")
'''

CASES = [
    # (name, preset, overrides, generator, levels)
    ("logn14_int64", "slots8192_scale40_levels7_int64", {}, 3, (0, 3)),
    ("logn14_int32", "slots8192_scale25_levels14_int32", {}, 3, (0, 3)),
    ("logn14_int64_gen5", "slots8192_scale40_levels7_int64", {}, 5, (0, 3)),
    # the benchmarked preset: N = 2^16, L = 35 at level 0, 10 hybrid digits
    ("logn16_int64", "slots32768_scale40_levels34_int64", {}, 3, (0, 30)),
]


def _install_reference(tmp: str):
    pkg = os.path.join(tmp, "fhelium")
    shutil.copytree(os.path.join(REFERENCE, "fhelium"), pkg)
    torchops = os.path.join(pkg, "native", "torchops")
    os.makedirs(torchops, exist_ok=True)
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    soabi = sysconfig.get_config_var("SOABI")
    shutil.copy(REF_OPS, os.path.join(torchops, f"_ops{ext}"))
    sys.path.insert(0, tmp)
    # load the reference's ABI helper by path (importing the package would
    # already require the manifest being written here)
    import importlib.util
    spec = importlib.util.spec_from_file_location("_fh_abi", os.path.join(pkg, "native", "_abi.py"))
    abi = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(abi)
    manifest = {"manifest_schema_version": abi.MANIFEST_SCHEMA_VERSION, "native_backends": ["cpu"],
                "project_version": "0.10.0", **abi.runtime_identity(torch)}
    # the package reads its own version from installed metadata
    dist = os.path.join(tmp, "fhelium-0.10.0.dist-info")
    os.makedirs(dist, exist_ok=True)
    with open(os.path.join(dist, "METADATA"), "w") as fh:
        fh.write("Metadata-Version: 2.1\nName: fhelium\nVersion: 0.10.0\n")
    with open(os.path.join(torchops, f"_build_manifest.{soabi}.json"), "w") as fh:
        json.dump(manifest, fh)
    os.makedirs(os.path.join(tmp, "triton_csprng"), exist_ok=True)
    with open(os.path.join(tmp, "triton_csprng", "__init__.py"), "w") as fh:
        fh.write(STUB)


def _record(out, moduli, prime_ids):
    c = canonical(out, moduli, prime_ids)
    return {"digest": digest(c), "shape": list(c.shape), "head": c.reshape(-1, c.shape[-1])[:4, :2].tolist()}


def generate_case(fh, name, preset, overrides, generator, levels):
    from fhelium.config import CkksConfig, Preset
    from fhelium.core import Ciphertext, RelinearizationKey, RotationKey

    cfg = CkksConfig.parse(Preset[preset], **overrides)
    eng = fh.CkksEngine(cfg, device="cpu", galois_generator=generator, allow_sk_gen=False)
    dt = cfg.torch_dtype
    mod, nq, npr, n = cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, cfg.N
    ctx_id = eng.context.context_id
    qp_ids = tuple(range(nq + npr))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dt)
    out = {"preset": preset, "overrides": overrides, "generator": generator, "cases": []}

    def ct(data, level, scale, domain, rep):
        return Ciphertext(data=t(data), level=level, scale=scale, context_id=ctx_id,
                          prime_ids=tuple(range(level, nq)), polynomial_domain=domain,
                          residue_representation=rep, modulus_basis="Q")

    def key(seed, cls, **kw):
        return cls(data=t(key_material(seed, mod, nq, npr, n)), context_id=ctx_id, prime_ids=qp_ids,
                   polynomial_domain="ntt", modulus_basis="QP", residue_representation="montgomery", **kw)

    rlk = key(900, RelinearizationKey)
    eng.set_relinearization_key(rlk)
    rot_steps = [1, -1, 8, 2, 5]
    for i, s in enumerate(rot_steps):
        eng.set_rotation_key(key(910 + i, RotationKey, rotation_step=s))
    for level in levels:
        ids = list(range(level, nq))
        # forward NTT of a coefficient ciphertext
        seed = 100 + level
        x = residues(seed, mod, ids, (2, 2), n)
        r = eng.coefficient_domain_to_ntt_domain(ct(x, level, 2.0 ** 30, "coefficient", "standard"))
        out["cases"].append({"op": "coefficient_domain_to_ntt_domain", "level": level, "seed": seed,
                             **_record(r.data.numpy(), mod, ids)})
        # multiply (NTT domain)
        sa, sb = 200 + level, 300 + level
        a = residues(sa, mod, ids, (2, 2), n, lazy=True)
        b = residues(sb, mod, ids, (2, 2), n, lazy=True)
        r = eng.multiply(ct(a, level, 2.0 ** 20, "ntt", "montgomery"), ct(b, level, 2.0 ** 20, "ntt", "montgomery"))
        out["cases"].append({"op": "multiply", "level": level, "seed": [sa, sb], **_record(r.data.numpy(), mod, ids)})
        # relinearize
        seed = 400 + level
        c3 = residues(seed, mod, ids, (3, 2), n, lazy=True)
        r = eng.relinearize(ct(c3, level, 2.0 ** 40, "ntt", "montgomery"))
        out["cases"].append({"op": "relinearize", "level": level, "seed": seed, "key_seed": 900,
                             **_record(r.data.numpy(), mod, ids)})
        # rescale (nearest)
        seed = 500 + level
        x = residues(seed, mod, ids, (2, 2), n)
        r = eng.rescale_to_next_level(ct(x, level, 2.0 ** 80, "coefficient", "standard"))
        out["cases"].append({"op": "rescale_to_next_level", "level": level, "seed": seed,
                             **_record(r.data.numpy(), mod, ids[1:])})
        # rotations with direct keys
        seed = 600 + level
        x = residues(seed, mod, ids, (2, 1), n)
        for i, s in enumerate(rot_steps[:3]):
            r = eng.rotate_by_step(ct(x, level, 2.0 ** 40, "coefficient", "standard"), s)
            out["cases"].append({"op": "rotate_by_step", "level": level, "seed": seed, "step": s,
                                 "key_seed": 910 + i, **_record(r.data.numpy(), mod, ids)})
        # hoisted rotations sharing one ModUp
        seed = 700 + level
        x = residues(seed, mod, ids, (2, 1), n)
        steps = [1, 2, 5]
        rs = eng.rotate_many_by_steps(ct(x, level, 2.0 ** 40, "coefficient", "standard"), steps)
        for s, r in zip(steps, rs):
            out["cases"].append({"op": "rotate_many_by_steps", "level": level, "seed": seed, "step": s,
                                 "steps": steps, "key_seed": 910 + rot_steps.index(s),
                                 **_record(r.data.numpy(), mod, ids)})
    out["client"] = client_cases(fh, eng, cfg, levels)
    return out


def client_cases(fh, eng, cfg, levels):
    """Encryption with injected draws and public key, and decryption with an
    injected secret key, through the reference's CkksEngine.encrypt /
    decrypt: the reference's random source is replaced by functions that
    return the recorded draws (e0 and e1 as its discrete_gaussian rows, v as
    its randint), so the ciphertext is a deterministic function of inputs."""
    from fhelium.core import Ciphertext, Plaintext, PublicKey, SecretKey

    dt = cfg.torch_dtype
    mod, nq, npr, n = cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, cfg.N
    ctx_id = eng.context.context_id
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dt)
    out = []
    batch = 2
    for level in levels:
        seed = 1000 + level
        x = client_inputs(seed, mod, nq, npr, level, n, batch, dt == torch.int32)
        draws = {"gauss": torch.from_numpy(x["e"].reshape(2 * batch, n)).to(dt),
                 "v": torch.from_numpy(x["v"]).to(dt)}
        eng._rng.discrete_gaussian = lambda non_repeats=0, repeats=1: [draws["gauss"]]
        eng._rng.randint = lambda amax, shift=0, repeats=0: [draws["v"]]
        pk = PublicKey(t(x["pk"]), ctx_id, tuple(range(nq)))
        pt = Plaintext(message=None, level=level, scale=2.0 ** 40, data=t(x["m"]), context_id=ctx_id,
                       representation="integer_coefficients", polynomial_domain="coefficient")
        r = eng.encrypt(pt, pk)
        ids = list(range(level, nq))
        out.append({"op": "encrypt", "level": level, "seed": seed, "batch": batch,
                    **_record(r.data.numpy(), mod, ids)})
        sk = SecretKey(t(x["sk"]), ctx_id, tuple(range(nq + npr)))
        c = Ciphertext(data=t(x["ct"]), level=level, scale=2.0 ** 40, context_id=ctx_id, prime_ids=tuple(ids),
                       polynomial_domain="coefficient", residue_representation="standard", modulus_basis="Q")
        d = eng.decrypt(c, sk).data.numpy().astype(np.float64)
        out.append({"op": "decrypt", "level": level, "seed": seed, "batch": batch, "digest": float_digest(d),
                    "shape": list(d.shape), "head": d.reshape(-1, d.shape[-1])[:2, :2].tolist()})
    # key generation: relinearisation key and one rotation key from an
    # injected secret key, with the per-digit uniform components and errors
    # returned in digit order by the replaced random source
    qp_ids = list(range(nq + npr))
    for op, seed in (("relinearization_key", 1200), ("rotation_key", 1300)):
        x = client_inputs(seed, mod, nq, npr, 0, n, 1, dt == torch.int32)
        uni, err = key_draws(seed + 10, mod, nq, npr, n)
        queue = {"u": [t(u) for u in uni], "e": [torch.from_numpy(e).to(dt) for e in err]}
        eng._rng.discrete_gaussian = lambda non_repeats=0, repeats=1: [queue["e"].pop(0).view(1, n)]
        eng._rng.randint = lambda amax, shift=0, repeats=0: [queue["u"].pop(0)]
        sk = SecretKey(t(x["sk"]), ctx_id, tuple(qp_ids))
        kg = eng._key_generator
        if op == "relinearization_key":
            k = kg.create_relinearization_key(sk)
            extra = {}
        else:
            k = kg.create_rotation_key(3, secret_key=sk)
            extra = {"step": 3}
        assert not queue["u"] and not queue["e"], "every draw consumed once"
        out.append({"op": op, "level": 0, "seed": seed, **extra, **_record(k.data.numpy(), mod, qp_ids)})
    return out


def main() -> int:
    if not os.path.exists(REF_OPS):
        print("build the reference CPU operators first: bash oracle/build_ref.sh", file=sys.stderr)
        return 1
    tmp = tempfile.mkdtemp(prefix="fhb_golden_ref_")
    try:
        _install_reference(tmp)
        import fhelium as fh
        torch.set_num_threads(os.cpu_count() or 1)
        fixtures = {}
        only = set(sys.argv[1:])
        path = os.path.join(HERE, "engine_golden.json")
        if only and os.path.exists(path):  # regenerate the named fixtures, keep the others
            fixtures.update(json.load(open(path))["fixtures"])
        for name, preset, overrides, gen, levels in CASES:
            if only and name not in only:
                continue
            fixtures[name] = generate_case(fh, name, preset, overrides, gen, levels)
            print(name, len(fixtures[name]["cases"]), "cases")
        meta = {"generator": "tests/golden/make_golden.py", "reference": "visualDust/fhelium 0.10.0",
                "key_seeds": {"relinearization": 900, "rotation": {"1": 910, "-1": 911, "8": 912, "2": 913, "5": 914}}}
        with open(os.path.join(HERE, "engine_golden.json"), "w") as fh_out:
            json.dump({"meta": meta, "fixtures": fixtures}, fh_out, indent=1)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
