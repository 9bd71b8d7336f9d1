"""Encryption and decryption against the reference's own CkksEngine.

tests/golden/engine_golden.json holds, per fixture, "client" cases written
by tests/golden/make_golden.py: the reference's CkksEngine.encrypt of an
integer-coefficient plaintext under an injected public key, with its random
source replaced by the recorded draws (v, e0, e1), and CkksEngine.decrypt of
a ciphertext under an injected secret key (the reference's bounded float64
reconstruction from the trailing Q primes, fhelium/engine/ckks_decryptor.py:
180-272), and the reference key generator's relinearisation and rotation
keys from an injected secret key with recorded per-digit draws
(fhelium/engine/key_generator.py:197-412).  Encryption outputs are compared
as canonical residues (integer equal, by digest); key material modulo q (its
state is lazy); decryption outputs as the exact float64 values (by digest of
their bytes).

The CPU test checks the oracle's restatement of both; the GPU test checks
the engine (encryption with EncryptionDraws, decryption by the
fhb_ckks_decrypt_tail kernel).
"""

import json
import os

import numpy as np
import pytest

from fhelium_b200.config import CkksConfig
from oracle import oracle as orc
from tests.golden.inputs import canonical, client_inputs, digest, float_digest, key_draws

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "engine_golden.json")))


def _cases():
    for name, fx in GOLDEN["fixtures"].items():
        for i, case in enumerate(fx.get("client", [])):
            yield pytest.param(name, i, id=f"{name}-{case['op']}-L{case['level']}")


def _setup(name, index):
    fx = GOLDEN["fixtures"][name]
    cfg = CkksConfig.parse(fx["preset"], **fx["overrides"])
    case = fx["client"][index]
    x = client_inputs(case["seed"], cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, case["level"], cfg.N,
                      case.get("batch", 1), cfg.buffer_bit_length == 30)
    return cfg, case, x


def _check_encrypt(case, out, cfg, ids=None):
    ids = list(range(case["level"], cfg.num_q_primes)) if ids is None else ids
    c = canonical(out, cfg.moduli, ids)
    assert list(c.shape) == case["shape"]
    assert c.reshape(-1, c.shape[-1])[:4, :2].tolist() == case["head"]
    assert digest(c) == case["digest"]


def _check_decrypt(case, out):
    out = np.asarray(out, dtype=np.float64)
    assert list(out.shape) == case["shape"]
    assert out.reshape(-1, out.shape[-1])[:2, :2].tolist() == case["head"]
    assert float_digest(out) == case["digest"]


def _tail_float64(phase: np.ndarray, moduli, level: int, num_q: int) -> np.ndarray:
    """The reference's trailing-pair float64 reconstruction, restated in numpy
    (fhelium/engine/ckks_decryptor.py:180-272): mixed-radix digits of the
    trailing two Q rows, above-half test on the digits, negation, then
    float64(d1) * float64(q_a) + float64(d0) with separately rounded operations."""
    qa, qb = int(moduli[num_q - 2]), int(moduli[num_q - 1])
    xa = phase[..., -2, :].astype(object)
    xb = phase[..., -1, :].astype(object)
    inv = pow(qa, -1, qb)
    half = qa * qb // 2
    h0, h1 = half % qa, half // qa

    def digits(a, b):
        return a, ((b - a) % qb) * inv % qb

    d0, d1 = digits(xa, xb)
    above = (d1 > h1) | ((d1 == h1) & (d0 > h0))
    na = np.where(xa == 0, 0, qa - xa)
    nb = np.where(xb == 0, 0, qb - xb)
    n0, n1 = digits(na, nb)
    d0 = np.where(above, n0, d0).astype(np.int64)
    d1 = np.where(above, n1, d1).astype(np.int64)
    v = d1.astype(np.float64) * np.float64(qa) + d0.astype(np.float64)
    return np.where(above, -v, v)


def _oracle_key(case, cfg, oc, x, generator):
    """Key-switch key of fhelium/engine/key_generator.py:197-330, restated:
    digit d = (NTT(e_d) R - a_d s + [P s_src on the digit's rows], a_d)."""
    nq, npr = cfg.num_q_primes, cfg.num_p_primes
    qp = list(range(nq + npr))
    prm = oc.sub_params(qp)
    rb = oc.radix_bits
    s = x["sk"]
    if case["op"] == "relinearization_key":
        src = orc.montgomery_mul(s, s, prm, rb)
    else:
        std = oc.inverse_to_standard(s, qp)
        src = oc.forward_to_montgomery(oc.automorphism(std, case["step"], qp, generator), qp)
    p_mont = np.array([(int(np.prod([int(v) for v in cfg.moduli[nq:]], dtype=object)) << rb) % cfg.moduli[i]
                       for i in qp], dtype=np.int64)
    psrc = orc.montgomery_mul(src, np.broadcast_to(p_mont[:, None], src.shape), prm, rb)
    uni, err = key_draws(case["seed"] + 10, cfg.moduli, nq, npr, cfg.N)
    q = np.array(cfg.moduli, dtype=np.int64)[:, None]
    digits = []
    for kd, ids in enumerate(oc.level_zero_digits):
        e = oc.forward_to_montgomery(np.mod(err[kd][None, :], q), qp)
        k0 = np.mod(e - orc.montgomery_mul(uni[kd], s, prm, rb), q)
        lo, hi = ids[0], ids[-1] + 1
        k0[lo:hi] = np.mod(k0[lo:hi] + psrc[lo:hi], q[lo:hi])
        digits.append(np.stack([k0, uni[kd]]))
    return np.stack(digits)


@pytest.mark.parametrize("name,index", list(_cases()))
def test_oracle_reproduces_reference_client(name, index):
    cfg, case, x = _setup(name, index)
    oc = orc.OracleContext(cfg.moduli, cfg.logN, cfg.num_q_primes, cfg.num_p_primes, cfg.buffer_bit_length,
                           cfg.scale_bits)
    level = case["level"]
    if case["op"].endswith("_key"):
        _check_encrypt(case, _oracle_key(case, cfg, oc, x, GOLDEN["fixtures"][name]["generator"]), cfg,
                       list(range(cfg.num_q_primes + cfg.num_p_primes)))
        return
    rows = oc.q_rows(level)
    q = np.array([cfg.moduli[i] for i in rows], dtype=np.int64)[:, None]
    lift = lambda c: np.mod(c[..., None, :], q)  # signed [*, N] -> canonical [*, L, N]
    prm = oc.sub_params(rows)
    if case["op"] == "encrypt":
        pk = x["pk"][:, level:]
        v = oc.forward_to_montgomery(lift(x["v"]), rows)
        comps = []
        for k, extra in ((0, lift(x["e"][0]) + lift(x["m"])), (1, lift(x["e"][1]))):
            prod = orc.montgomery_mul(v, np.broadcast_to(pk[k], v.shape), prm, oc.radix_bits)
            comps.append(np.mod(oc.inverse_to_standard(prod, rows) + extra, q))
        _check_encrypt(case, np.stack(comps), cfg)
    else:
        ct = x["ct"]
        s = x["sk"][level: cfg.num_q_primes]
        c1 = oc.forward_to_montgomery(ct[1], rows)
        prod = orc.montgomery_mul(c1, np.broadcast_to(s, c1.shape), prm, oc.radix_bits)
        phase = np.mod(ct[0] + oc.inverse_to_standard(prod, rows), q)
        _check_decrypt(case, _tail_float64(phase, cfg.moduli, level, cfg.num_q_primes))


@pytest.mark.gpu
@pytest.mark.parametrize("name,index", list(_cases()))
def test_gpu_engine_reproduces_reference_client(name, index):
    import torch

    from fhelium_b200.engine import CkksEngine
    from fhelium_b200.values import Ciphertext, EncryptionDraws, KeySwitchKeyDraws, Plaintext, PublicKey, SecretKey

    cfg, case, x = _setup(name, index)
    fx = GOLDEN["fixtures"][name]
    eng = CkksEngine(cfg, galois_generator=fx["generator"], allow_sk_gen=False)
    dev = lambda a, dt=cfg.torch_dtype: torch.from_numpy(np.ascontiguousarray(a)).to(dt).cuda()
    level = case["level"]
    if case["op"].endswith("_key"):
        uni, err = key_draws(case["seed"] + 10, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, cfg.N)
        draws = KeySwitchKeyDraws(uniform=dev(uni), error=dev(err, torch.int64))
        sk = SecretKey(dev(x["sk"]))
        if case["op"] == "relinearization_key":
            k = eng.create_relinearization_key(sk, draws=draws)
        else:
            k = eng.create_rotation_key(case["step"], sk, draws=draws)
        _check_encrypt(case, k.data.cpu().to(torch.int64).numpy(), cfg,
                       list(range(cfg.num_q_primes + cfg.num_p_primes)))
    elif case["op"] == "encrypt":
        pt = Plaintext(message=None, data=dev(x["m"], torch.int64), level=level, scale=2.0 ** 40,
                       context_id=eng.context_id, representation="integer_coefficients",
                       polynomial_domain="coefficient")
        draws = EncryptionDraws(v=dev(x["v"], torch.int64), e0=dev(x["e"][0], torch.int64),
                                e1=dev(x["e"][1], torch.int64))
        out = eng.encrypt(pt, PublicKey(dev(x["pk"])), draws=draws)
        _check_encrypt(case, out.data.cpu().to(torch.int64).numpy(), cfg)
    else:
        ct = Ciphertext(dev(x["ct"]), level, 2.0 ** 40)
        pt = eng.decrypt(ct, SecretKey(dev(x["sk"])))
        assert pt.data.device.type == "cuda" and pt.data.dtype == torch.float64
        _check_decrypt(case, pt.data.cpu().numpy())
