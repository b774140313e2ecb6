"""GPU tests of client-side extraction (xpir_b200_extract): decrypting replies and
recursing back to the element must give the same bytes as the oracle restatement (and
so as the reference's PIRReplyExtraction, which the restatement is pinned to), and a
full round trip through the GPU must recover the chosen element."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,m,n,alpha,L,reduced", [
    (1024, 1, [20], 1, 900, True), (2048, 3, [8], 2, 700, True), (1024, 2, [6, 5], 1, 400, True),
    (512, 1, [4, 4, 3], 1, 300, True), (1024, 2, [12], 1, 600, False), (4096, 3, [5, 4], 3, 500, True),
    (8192, 2, [50], 1, 5000, True), (2048, 4, [9], 1, 2000, True)])
def test_extract_matches_oracle(engine, oracle, N, m, n, alpha, L, reduced):
    rng = np.random.default_rng(N * 7 + m + L)
    d, b = len(n), oracle.bits_per_coeff(N, m, n[0])
    key = np.empty((m, N), dtype=np.uint64)
    for c, p in enumerate(oracle.moduli(m)):
        key[c] = rng.integers(0, p, size=N, dtype=np.uint64)
    key = key.reshape(-1)
    nct = oracle.extract_count(L * alpha, d, b, N, m)
    assert engine.extract_count(L * alpha, d, b, N, m) == nct
    ct = rng.integers(0, 2**64, size=(nct, 2, m, N), dtype=np.uint64)
    if reduced:
        for c, p in enumerate(oracle.moduli(m)):
            ct[:, :, c, :] %= np.uint64(2 * p)
    ct = ct.reshape(-1)
    want = oracle.extract(ct, key, d, b, N, m, L * alpha)
    with engine.Context(N, m) as ctx:
        got = ctx.extract(key, d, b, L * alpha, ct)
        assert np.array_equal(got, want)
        # device-resident replies and output
        torch = pytest.importorskip("torch")
        dct = torch.from_numpy(ct.view(np.int64)).cuda()
        dout = torch.zeros(L * alpha, dtype=torch.uint8, device="cuda")
        ctx.extract(key, d, b, L * alpha, dct, dout)
        assert np.array_equal(dout.cpu().numpy(), want)


def test_gpu_round_trip_recovers_element(engine, ref):
    """The reference generates the query (seeded key); the GPU imports, replies and
    extracts with that key; the chosen aggregated element comes back."""
    N, m, n, alpha, F, L, chosen = 2048, 2, [6, 5], 2, 57, 1500, 17
    db = np.random.default_rng(3).integers(0, 256, size=F * L, dtype=np.uint8)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=33, chosen=chosen, extract=False)
    key = ref.ref_key(N, m, 33)
    b = ref.bits_per_coeff(N, m, n[0])
    with engine.Context(N, m) as ctx:
        dbh = ctx.import_db(db, F, L, alpha, b)
        reply = ctx.reply(dbh, n, r["query"])
        assert np.array_equal(reply, r["reply"])
        got = ctx.extract(key, len(n), b, L * alpha, reply)
    assert np.array_equal(got, db[chosen * alpha * L:(chosen + 1) * alpha * L])
