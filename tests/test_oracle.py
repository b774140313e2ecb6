"""CPU tests: the oracle restatement is pinned to the XPIR reference.

Two pins: the committed golden fixtures (produced by the reference's own libpir code,
tests/golden/make_golden.py), and, where the reference checker binary is built, direct
comparisons against it on randomized inputs.  Bit-exact everywhere: this is integer work.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from helpers import golden_cases, load_golden, random_db


@pytest.mark.parametrize("name", golden_cases())
def test_golden_import_and_reply(oracle, name):
    g = load_golden(name)
    mt = g["meta"]
    N, m, n, alpha = mt["N"], mt["m"], mt["n"], mt["alpha"]
    F, L, b, P = mt["nb_elements"], mt["element_bytes"], mt["bits_per_coeff"], mt["polys_per_element"]
    assert oracle.bits_per_coeff(N, m, n[0]) == b
    assert oracle.polys_for_bits(8 * alpha * L, b, N) == P
    imp = oracle.import_db(g["db"], F, L, alpha, b, N, m)
    assert hashlib.sha256(imp.tobytes()).hexdigest() == mt["imported_sha256"]
    rep = oracle.reply(imp, mt["nb_aggregated"], P, n, g["query"], b, N, m)
    assert rep.size == g["reply"].size
    assert np.array_equal(rep, g["reply"])
    assert oracle.reply_count(L, alpha, len(n), b, N, m) == mt["n_replies"]


def test_golden_fixtures_present():
    assert len(golden_cases()) >= 3


@pytest.mark.parametrize("N", [512, 1024, 2048, 4096, 8192])
@pytest.mark.parametrize("m", [1, 2, 3])
def test_tables_match_reference(ref, N, m):
    a = ref.tables(N, m)
    r = ref.ref_tables(N, m)
    blk = 1 + 8 * N
    for c in range(m):
        x = a[c * blk:(c + 1) * blk]
        y = r[c * blk:(c + 1) * blk]
        assert x[0] == y[0]
        for t in range(8):
            sl = slice(1 + t * N, 1 + (t + 1) * N)
            xs, ys = x[sl], y[sl]
            if t in (2, 3, 6, 7):  # twiddle layers fill N-1 words; the N-th is never read
                xs, ys = xs[:N - 1], ys[:N - 1]
            assert np.array_equal(xs, ys), (c, t)
    assert np.array_equal(a[m * blk:], r[m * blk:])


@pytest.mark.parametrize("N,m,n0", [(1024, 1, 1000), (2048, 2, 100000), (4096, 3, 1024), (2048, 2, 256),
                                     (2048, 2, 65536), (1024, 4, 100), (512, 1, 7), (8192, 4, 3)])
def test_bits_per_coeff_match_reference(ref, N, m, n0):
    assert ref.bits_per_coeff(N, m, n0) == ref.ref_info(N, m, n0)["bits_per_coeff"]


@pytest.mark.parametrize("N", [512, 2048, 8192])
@pytest.mark.parametrize("m", [1, 3])
def test_ntt_matches_reference(ref, N, m):
    rng = np.random.default_rng(N + m)
    x = rng.integers(0, 2**63, size=2 * m * N, dtype=np.uint64)
    x[:6] = [0, 1, ref.modulus(0) - 1, 2 * ref.modulus(0) - 1, 2**56 - 1, 2**63 - 1]
    assert np.array_equal(ref.ntt_phi(x, N, m), ref.ref_ntt(N, m, x))


def test_bitsplit_matches_reference(ref):
    """The reference's byte-unaligned multi-buffer bit walk equals a plain LSB-first
    stream over the concatenated buffers (b <= 56 replicated per modulus, b > 56 CRT)."""
    rng = np.random.default_rng(7)
    for trial in range(80):
        N = int(rng.choice([512, 1024]))
        m = int(rng.integers(1, 5))
        b = int(rng.integers(1, min(60 * m // 2, 119) + 1))
        nbufs = int(rng.integers(1, 5))
        nbytes = int(rng.integers(1, 3000))
        stride = nbytes + int(rng.integers(0, 9))
        bufs = rng.integers(0, 256, size=nbufs * stride, dtype=np.uint8)
        a = ref.bitsplit(bufs, nbufs, stride, 8 * nbytes, b, N, m)
        r = ref.ref_bitsplit(N, m, bufs, nbufs, 8 * nbytes, b, stride)
        assert np.array_equal(a, r), dict(N=N, m=m, b=b, nbufs=nbufs, nbytes=nbytes)


@pytest.mark.parametrize("N,m,n,alpha,F,L", [
    (1024, 1, [20], 1, 20, 1000),
    (1024, 1, [7], 3, 20, 1000),       # short last group
    (2048, 2, [10, 5], 2, 100, 3000),  # d = 2
    (4096, 3, [8, 5], 3, 100, 3000),   # d = 2, short group, grid padding, b > 56
    (1024, 2, [5, 5, 4], 1, 100, 3000),  # d = 3
    (1024, 4, [30], 1, 25, 3000),      # four moduli, b > 56, padded grid
    (512, 1, [4, 4], 5, 50, 700),      # P > 1 at level 0
])
def test_import_and_reply_match_reference(ref, N, m, n, alpha, F, L):
    db = random_db(F * 31 + L, F, L)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=5, chosen=0, want_imported=True, extract=False)
    b, P = r["bits_per_coeff"], r["polys_per_element"]
    imp = ref.import_db(db, F, L, alpha, b, N, m)
    assert np.array_equal(imp, r["imported"])
    rep = ref.reply(imp, -(-F // alpha), P, n, r["query"], b, N, m)
    assert np.array_equal(rep, r["reply"])


def test_short_group_aggregation_quirk(oracle):
    """DBHandler::readAggregatedStream on a short last group: the last real element's
    slot and the following slots up to alpha-2 read as zeros, slot alpha-1 keeps the
    previous group's last element."""
    L, alpha, nb = 4, 4, 10  # groups: [0..3], [4..7], [8, 9, -, -]
    elems = np.arange(nb * L, dtype=np.uint8)
    g2 = oracle.aggregate(elems, nb, L, L, alpha, 2)
    assert np.array_equal(g2[0:L], elems[8 * L:9 * L])          # slot 0: element 8
    assert np.all(g2[L:3 * L] == 0)                               # slots 1-2: zero (element 9 lost)
    assert np.array_equal(g2[3 * L:4 * L], elems[7 * L:8 * L])  # slot 3: element 7 (stale)
    g0 = oracle.aggregate(elems[:2 * L], 2, L, L, alpha, 0)      # short first group: stale slot is zero
    assert np.array_equal(g0[0:L], elems[0:L]) and np.all(g0[L:] == 0)


@pytest.mark.parametrize("N,m,b", [(1024, 2, 40), (4096, 3, 74)])
def test_zero_elements_import_to_one_constant_poly(oracle, N, m, b):
    """The import of an all-zero element is one fixed poly per modulus, the same for every
    element and poly, and not zero: the lazy butterfly maps 0 - 0 to 2p, whose Shoup
    product is p. The recursion relies on this to broadcast the import of the idle groups'
    (exactly zero) level replies instead of transforming each."""
    L = 3 * N * b // 8  # three polys per element
    imp = oracle.import_db(np.zeros(5 * L, dtype=np.uint8), 5, L, 1, b, N, m).reshape(-1, m, N)
    assert imp.shape[0] == 5 * oracle.polys_for_bits(8 * L, b, N)
    assert np.all(imp == imp[0])
    p = np.array(oracle.moduli(m), dtype=np.uint64)[:, None]
    assert np.all((imp[0] == 0) | (imp[0] == p)) and np.any(imp[0] != 0)


def test_reference_extraction_recovers_element(ref):
    db = random_db(3, 12, 2000)
    r = ref.ref_run(1024, 1, [12], 1, db, 12, 2000, keyseed=9, chosen=7)
    assert r["extract_ok"] == 1
    assert np.array_equal(r["plain"], db[7 * 2000:8 * 2000])


@pytest.mark.parametrize("N,m,n,alpha,L,reduced", [
    (1024, 1, [20], 1, 900, True), (2048, 3, [8], 2, 700, True), (1024, 2, [6, 5], 1, 400, True),
    (512, 1, [4, 4, 3], 1, 300, True), (1024, 2, [12], 1, 600, False)])
def test_extraction_matches_reference(ref, N, m, n, alpha, L, reduced):
    """Decryption and multi-level extraction of arbitrary ciphertexts (words below 2p as
    replies have them, or any 64-bit words) equal the reference's PIRReplyExtraction with
    the same seeded key, byte for byte."""
    rng = np.random.default_rng(N + m + L)
    d, b = len(n), ref.bits_per_coeff(N, m, n[0])
    key = ref.ref_key(N, m, 9)
    nct = ref.extract_count(L * alpha, d, b, N, m)
    ct = rng.integers(0, 2**64, size=(nct, 2, m, N), dtype=np.uint64)
    if reduced:
        for c, p in enumerate(ref.moduli(m)):
            ct[:, :, c, :] %= np.uint64(2 * p)
    ct = ct.reshape(-1)
    assert np.array_equal(ref.extract(ct, key, d, b, N, m, L * alpha), ref.ref_extract(N, m, n, alpha, L, 9, ct))


def test_extraction_round_trip_with_reference_key(ref):
    """The reference answers its own query; the restatement, given the reference's secret
    key, recovers the chosen aggregated element from that reply."""
    N, m, n, alpha, F, L, chosen = 1024, 2, [5, 4], 2, 37, 600, 13
    db = np.random.default_rng(12).integers(0, 256, size=F * L, dtype=np.uint8)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=21, chosen=chosen)
    key = ref.ref_key(N, m, 21)
    b = ref.bits_per_coeff(N, m, n[0])
    got = ref.extract(r["reply"], key, len(n), b, N, m, L * alpha)
    assert np.array_equal(got, db[chosen * alpha * L:(chosen + 1) * alpha * L])
    assert np.array_equal(got, r["plain"])


@pytest.mark.parametrize("N,m", [(1024, 1), (2048, 2), (4096, 3)])
def test_keygen_matches_reference(ref, N, m):
    """The Salsa20 keystream restatement keyed like the reference's fastrandombytes gives
    the reference's secret key (the first PRNG call of a fresh crypto object)."""
    key = ref.seeded_prng_key(9)
    assert np.array_equal(ref.keygen(key, 0, N, m), ref.ref_key(N, m, 9))


@pytest.mark.parametrize("N,m,n,alpha,F,L,chosen,seed", [
    (1024, 2, [5, 4], 1, 20, 300, 13, 21), (2048, 3, [7], 2, 13, 900, 5, 4), (512, 1, [3, 3, 2], 1, 18, 200, 11, 8)])
def test_query_generation_matches_reference(ref, N, m, n, alpha, F, L, chosen, seed):
    """Query ciphertexts from the restatement (noise, amplification, NTT, uniform a, a*s,
    full reduction) equal the reference's PIRQueryGenerator output word for word."""
    db = np.random.default_rng(1).integers(0, 256, size=F * L, dtype=np.uint8)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=seed, chosen=chosen, extract=False)
    key = ref.seeded_prng_key(seed)
    sk = ref.keygen(key, 0, N, m)
    b = ref.bits_per_coeff(N, m, n[0])
    assert np.array_equal(ref.query(key, 1, sk, n, chosen, b, N, m), r["query"])
