"""Engine-level golden digests produced by the reference's own CkksEngine.

tests/golden/engine_golden.json was written by tests/golden/make_golden.py,
which drives the reference's Python engine (with its CPU operators compiled
from the reference sources) on inputs rebuilt here from the recorded seeds.
The CPU oracle must reproduce every digest (this pins the oracle's
orchestration of multiply, relinearize, rescale, direct and hoisted
rotations, for generators 3 and 5 and both word sizes against the reference
itself); the GPU engine must reproduce them too.
"""

import json
import os

import numpy as np
import pytest

from fhelium_b200.config import CkksConfig
from oracle import oracle as orc
from tests.golden.inputs import canonical, digest, key_material, residues

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "engine_golden.json")))
KEY_SEEDS = GOLDEN["meta"]["key_seeds"]


def _cases():
    for name, fx in GOLDEN["fixtures"].items():
        for i, case in enumerate(fx["cases"]):
            yield pytest.param(name, i, id=f"{name}-{case['op']}-L{case['level']}-{case.get('step', '')}-{i}")


def _setup(name):
    fx = GOLDEN["fixtures"][name]
    cfg = CkksConfig.parse(fx["preset"], **fx["overrides"])
    return fx, cfg


def _inputs(case, cfg):
    mod, nq, npr, n = cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, cfg.N
    level = case["level"]
    ids = list(range(level, nq))
    op = case["op"]
    if op == "coefficient_domain_to_ntt_domain":
        return ids, residues(case["seed"], mod, ids, (2, 2), n)
    if op == "multiply":
        sa, sb = case["seed"]
        return ids, (residues(sa, mod, ids, (2, 2), n, lazy=True), residues(sb, mod, ids, (2, 2), n, lazy=True))
    if op == "relinearize":
        return ids, residues(case["seed"], mod, ids, (3, 2), n, lazy=True)
    if op == "rescale_to_next_level":
        return ids, residues(case["seed"], mod, ids, (2, 2), n)
    return ids, residues(case["seed"], mod, ids, (2, 1), n)


def _key(cfg, seed):
    return key_material(seed, cfg.moduli, cfg.num_q_primes, cfg.num_p_primes, cfg.N)


def _check(case, out, cfg, ids):
    rows = ids[1:] if case["op"] == "rescale_to_next_level" else ids
    c = canonical(out, cfg.moduli, rows)
    assert list(c.shape) == case["shape"]
    assert c.reshape(-1, c.shape[-1])[:4, :2].tolist() == case["head"]
    assert digest(c) == case["digest"]


@pytest.mark.parametrize("name,index", list(_cases()))
def test_oracle_reproduces_reference_engine(name, index):
    fx, cfg = _setup(name)
    case = fx["cases"][index]
    gen = fx["generator"]
    oc = orc.OracleContext(cfg.moduli, cfg.logN, cfg.num_q_primes, cfg.num_p_primes, cfg.buffer_bit_length,
                           cfg.scale_bits)
    ids, x = _inputs(case, cfg)
    level, op = case["level"], case["op"]
    if op == "coefficient_domain_to_ntt_domain":
        out = oc.forward_to_montgomery(x, ids)
    elif op == "multiply":
        out = oc.multiply(x[0], x[1], level)
    elif op == "relinearize":
        out = oc.relinearize(x, _key(cfg, KEY_SEEDS["relinearization"]), level)
    elif op == "rescale_to_next_level":
        out = oc.rescale(x, level)
    elif op == "rotate_by_step":
        out = oc.rotate(x, case["step"], _key(cfg, case["key_seed"]), level, gen)
    else:
        keys = {s: _key(cfg, KEY_SEEDS["rotation"][str(s)]) for s in case["steps"]}
        outs = oc.rotate_hoisted(x, case["steps"], keys, level, gen)
        out = outs[case["steps"].index(case["step"])]
    _check(case, out, cfg, ids)


@pytest.mark.gpu
@pytest.mark.parametrize("name,index", list(_cases()))
def test_gpu_engine_reproduces_reference_engine(name, index):
    import torch

    from fhelium_b200.engine import CkksEngine
    from fhelium_b200.values import Ciphertext, RelinearizationKey, RotationKey

    fx, cfg = _setup(name)
    case = fx["cases"][index]
    eng = _engine(name, cfg, fx["generator"])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cfg.torch_dtype).cuda()
    ids, x = _inputs(case, cfg)
    level, op = case["level"], case["op"]
    if op == "coefficient_domain_to_ntt_domain":
        out = eng.coefficient_domain_to_ntt_domain(Ciphertext(dev(x), level, 1.0)).data
    elif op == "multiply":
        out = eng.multiply(Ciphertext(dev(x[0]), level, 1.0, "ntt", "montgomery"),
                           Ciphertext(dev(x[1]), level, 1.0, "ntt", "montgomery")).data
    elif op == "relinearize":
        rlk = RelinearizationKey(dev(_key(cfg, KEY_SEEDS["relinearization"])))
        out = eng.relinearize(Ciphertext(dev(x), level, 1.0, "ntt", "montgomery"), rlk).data
    elif op == "rescale_to_next_level":
        out = eng.rescale_to_next_level(Ciphertext(dev(x), level, 2.0 ** 80)).data
    else:
        steps = case["steps"] if op == "rotate_many_by_steps" else [case["step"]]
        for s in steps:
            seed = KEY_SEEDS["rotation"][str(s)]
            eng.set_rotation_key(RotationKey(dev(_key(cfg, seed)), rotation_step=s,
                                             galois_element=eng.galois_element_for_step(s)))
        c = Ciphertext(dev(x), level, 1.0)
        if op == "rotate_by_step":
            out = eng.rotate_by_step(c, case["step"]).data
        else:
            out = eng.rotate_many_by_steps(c, steps)[steps.index(case["step"])].data
    _check(case, out.cpu().to(torch.int64).numpy(), cfg, ids)


_ENGINES = {}


def _engine(name, cfg, generator):
    from fhelium_b200.engine import CkksEngine
    if name not in _ENGINES:
        _ENGINES[name] = CkksEngine(cfg, galois_generator=generator, allow_sk_gen=False)
    return _ENGINES[name]
