"""Host side of the exact int8 tensor-core NTT (no GPU).

The library's host table builder writes, per pass and prime, the byte-split
constant matrices in the tensor cores' shared-memory layout and the
elementwise twiddles.  Here the four passes are emulated in numpy from those
very bytes (unsigned 8-bit digit products with exact accumulation, the
epilogue's Montgomery reduction by 2^32 and Shoup twiddle) and checked
against the oracle's negacyclic NTT: forward equal mod q, inverse
bit-identical, with the accumulator and range bounds the kernels rely on."""

import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

N, SIDE, TILE = 1 << 16, 256, 64


def _lib():
    from fhelium_b200 import _native
    import os
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libfhb200.so not built")
    return _native.load()


def _prime():
    # smallest prime q = 1 mod 2^17 above 2^27 (a 28-bit NTT prime, 4q < 2^30)
    q = (1 << 27) + 1
    while True:
        if q % (2 * N) == 1 and all(q % p for p in range(3, int(q ** 0.5) + 1, 2)):
            return q
        q += 2 * N - (q % (2 * N)) + 1 if q % (2 * N) != 1 else 2 * N


def _tables(lib, q, psi, p):
    bmat = np.zeros(1 << 20, dtype=np.uint8)
    post = np.zeros(2 * N, dtype=np.uint32)
    rc = lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(psi), p, bmat.ctypes.data,
                                    post.ctypes.data)
    assert rc == 0
    # decode the chunk layout: chunk (tile j, kc * 4 + d) holds rows e * 64 + col
    # and K bytes kk at (row % 8) * 16 + (row // 8) * 256 + (kk // 16) * 128 + kk % 16
    row = np.arange(256)[:, None]
    kk = np.arange(32)[None, :]
    off = (row % 8) * 16 + (row // 8) * 256 + (kk // 16) * 128 + kk % 16  # [256 rows, 32]
    chunks = bmat.reshape(4, 8, 4, 8192)  # [j][kc][d][bytes]
    planes = np.zeros((4, 4, SIDE, SIDE), dtype=np.float64)  # [d][e][k][n]
    for j in range(4):
        for kc in range(8):
            for d in range(4):
                blk = chunks[j, kc, d][off]  # [256 rows, 32 k]
                for e in range(4):
                    planes[d, e, kc * 32:(kc + 1) * 32, j * TILE:(j + 1) * TILE] = blk[e * TILE:(e + 1) * TILE].T
    return planes, post.reshape(N, 2)


def _pass(a_mat, planes, post, q, column, post_on):
    """One kernel pass on a [256, 256] data matrix A[m][k]; returns D[m][n]."""
    a = a_mat.astype(np.uint64)
    digits = [((a >> np.uint64(8 * d)) & np.uint64(255)).astype(np.float64) for d in range(4)]
    acc = [sum(digits[d] @ planes[d, e] for d in range(4)) for e in range(4)]
    for x in acc:
        assert x.max() < 2 ** 26
    s = sum(np.asarray(acc[e], dtype=np.uint64) << np.uint64(8 * e) for e in range(4))
    qneg = (-pow(q, -1, 1 << 32)) % (1 << 32)
    mm = ((s & np.uint64(0xFFFFFFFF)) * np.uint64(qneg)) & np.uint64(0xFFFFFFFF)
    r = (s + mm * np.uint64(q)) >> np.uint64(32)
    assert r.max() < 2 * q
    if post_on:
        idx = np.arange(SIDE)
        m, n = np.meshgrid(idx, idx, indexing="ij")
        flat = n * SIDE + m if column else m * SIDE + n
        w = post[flat, 0].astype(np.uint64)
        wp = post[flat, 1].astype(np.uint64)
        qh = (r * wp) >> np.uint64(32)
        r = (r * w - qh * np.uint64(q)) & np.uint64(0xFFFFFFFF)
        assert r.max() < 2 * q
    return np.where(r >= q, r - np.uint64(q), r).astype(np.int64)


def _forward(x, tabs, q):
    d1 = _pass(x.reshape(SIDE, SIDE).T, *tabs[0], q, True, True)      # D[m = i2][n = r]
    y = d1.T                                                            # Y[r][i2]
    return _pass(y, *tabs[1], q, False, False).reshape(-1)             # O[r][c]


def _inverse(o, tabs, q):
    e = _pass(o.reshape(SIDE, SIDE), *tabs[2], q, False, True)        # E[r][i2]
    d2 = _pass(e.T, *tabs[3], q, True, False)                          # D[m = i2][n = i1]
    return d2.T.reshape(-1)


def test_four_step_matches_oracle_ntt():
    lib = _lib()
    q = _prime()
    psi = orc.primitive_2nth_root(q, N)
    tabs = [_tables(lib, q, psi, p) for p in range(4)]
    oc = orc.OracleContext((q, q), 16, 1, 1, 30)
    rng = np.random.default_rng(11)
    x = rng.integers(0, q, N, dtype=np.int64)
    ref = oc.forward_to_montgomery(x.reshape(1, 1, N), [0]).reshape(-1)
    fwd = _forward(x, tabs, q)
    assert fwd.max() < q
    assert np.array_equal(fwd, ref % q)
    assert np.array_equal(_inverse(fwd, tabs, q), x)
    # lazy [0, 2q) input (the CUDA-core forward's output range) inverts exactly
    lazy = fwd + q * rng.integers(0, 2, N, dtype=np.int64)
    assert np.array_equal(_inverse(lazy, tabs, q), x)
    assert np.array_equal(oc.inverse_to_standard(ref.reshape(1, 1, N), [0]).reshape(-1), x)


def test_tables_reject_bad_arguments():
    lib = _lib()
    buf = np.zeros(1 << 20, dtype=np.uint8)
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(97), ctypes.c_uint64(3), 0, buf.ctypes.data, None) != 0
    q = _prime()
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(5), 4, buf.ctypes.data, None) != 0
    assert lib.fhb_tc_ntt_tables_host(ctypes.c_uint64(q), ctypes.c_uint64(0), 0, buf.ctypes.data, None) != 0
