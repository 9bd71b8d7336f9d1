"""Host side of the exact int8 tensor-core NTT (no GPU).

The library's host table builder writes, per pass and prime, the byte-split
constant matrix in the tensor cores' shared-memory layout and the
elementwise twiddles (as t 2^32 mod q) in output order.  Here the six passes (three forward,
three inverse) are emulated in numpy from those very bytes -- unsigned 8-bit
digit products with exact accumulation, the epilogue's Montgomery reduction
by 2^32, the twiddle's second reduction, the instance maps of the kernels -- and checked
against the oracle's negacyclic NTT: forward equal mod q, inverse
bit-identical, with the accumulator and range bounds the kernels rely on."""

import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as orc

N = 1 << 16
NK = [64, 64, 16, 16, 64, 64]          # outputs per instance of each pass
KIND = [1, 2, 3, 3, 2, 1]              # instance map of each pass
POST = [True, True, False, True, True, False]


def _lib():
    from fhelium_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libfhb200.so not built")
    return _native.load()


def _prime():
    # smallest prime q = 1 mod 2^17 above 2^27 (a 28-bit NTT prime, 4q < 2^30)
    q = (1 << 27) + 1
    while not all(q % p for p in range(3, int(q ** 0.5) + 1, 2)):
        q += 2 * N
    return q


def _offsets(kind, nk):
    """[instances, nk] word offsets of an instance's inputs (= its outputs)."""
    m = np.arange(N // nk)[:, None]
    k = np.arange(nk)[None, :]
    if kind == 1:
        return m + 1024 * k
    if kind == 2:
        return (m // 16) * 1024 + m % 16 + 16 * k
    return 16 * m + k


def _tables(lib, q, psi, p):
    nk = NK[p]
    bmat = np.zeros(16 * nk * nk, dtype=np.uint8)
    post = np.zeros(N, dtype=np.uint32)
    rc = lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(psi), p, bmat.ctypes.data,
                                    post.ctypes.data)
    assert rc == 0
    # decode: row r = e * nk + n, byte kappa = d * nk + k of a K-major tile
    # with 8-row groups nk * 32 bytes apart
    r = np.arange(4 * nk)[:, None]
    kap = np.arange(4 * nk)[None, :]
    off = (r % 8) * 16 + (r // 8) * (nk * 32) + (kap // 16) * 128 + kap % 16
    full = bmat[off].astype(np.float64)            # [e * nk + n][d * nk + k]
    planes = full.reshape(4, nk, 4, nk).transpose(2, 3, 0, 1)   # [d][k][e][n]
    return planes, post


def _pass(x, p, planes, post, q):
    nk, kind = NK[p], KIND[p]
    offs = _offsets(kind, nk)
    a = x[offs].astype(np.uint64)                  # [instances][k]
    acc = np.zeros((offs.shape[0], 4, nk))
    for d in range(4):
        digit = ((a >> np.uint64(8 * d)) & np.uint64(255)).astype(np.float64)
        acc += np.einsum("mk,ken->men", digit, planes[d])
    assert acc.max() < 2 ** 24
    acc = acc.astype(np.uint64)
    s = sum(acc[:, e] << np.uint64(8 * e) for e in range(4))
    qneg = (-pow(q, -1, 1 << 32)) % (1 << 32)
    mm = ((s & np.uint64(0xFFFFFFFF)) * np.uint64(qneg)) & np.uint64(0xFFFFFFFF)
    r = (s + mm * np.uint64(q)) >> np.uint64(32)
    assert r.max() < 2 * q
    if POST[p]:
        pr = r * post[offs].astype(np.uint64)        # twiddle stored as t 2^32 mod q
        assert pr.max() < q * 2 ** 32
        m2 = ((pr & np.uint64(0xFFFFFFFF)) * np.uint64(qneg)) & np.uint64(0xFFFFFFFF)
        r = (pr + m2 * np.uint64(q)) >> np.uint64(32)
        assert r.max() < 2 * q
    out = np.empty(N, dtype=np.int64)
    out[offs] = np.where(r >= q, r - np.uint64(q), r).astype(np.int64)
    return out


def test_three_pass_matches_oracle_ntt():
    lib = _lib()
    q = _prime()
    psi = orc.primitive_2nth_root(q, N)
    tabs = [_tables(lib, q, psi, p) for p in range(6)]
    oc = orc.OracleContext((q, q), 16, 1, 1, 30)
    rng = np.random.default_rng(11)
    x = rng.integers(0, q, N, dtype=np.int64)
    ref = oc.forward_to_montgomery(x.reshape(1, 1, N), [0]).reshape(-1)
    fwd = x
    for p in (0, 1, 2):
        fwd = _pass(fwd, p, *tabs[p], q)
    assert fwd.max() < q
    assert np.array_equal(fwd, ref % q)
    inv = fwd
    for p in (3, 4, 5):
        inv = _pass(inv, p, *tabs[p], q)
    assert np.array_equal(inv, x)
    # lazy [0, 2q) input (the CUDA-core forward's output range) inverts exactly
    inv = fwd + q * rng.integers(0, 2, N, dtype=np.int64)
    for p in (3, 4, 5):
        inv = _pass(inv, p, *tabs[p], q)
    assert np.array_equal(inv, x)


def test_tables_reject_bad_arguments():
    lib = _lib()
    buf = np.zeros(1 << 16, dtype=np.uint8)
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(97), ctypes.c_uint64(3), 0, buf.ctypes.data, None) != 0
    q = _prime()
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(5), 6, buf.ctypes.data, None) != 0
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(0), 0, buf.ctypes.data, None) != 0
