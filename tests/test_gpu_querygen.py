"""GPU tests of client-side query generation (xpir_b200_generate_query): the ciphertexts
must equal the oracle restatement's (and so the reference PIRQueryGenerator's, which the
restatement is pinned to) word for word, and a query generated, answered and extracted
entirely on the GPU must bring back the chosen element."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,m,n,chosen,seed", [
    (1024, 2, [5, 4], 13, 21), (2048, 3, [7], 5, 4), (512, 1, [3, 3, 2], 11, 8), (8192, 2, [6], 2, 3),
    (4096, 4, [3, 2], 4, 5)])
def test_query_matches_oracle(engine, oracle, N, m, n, chosen, seed):
    key = oracle.seeded_prng_key(seed)
    sk = oracle.keygen(key, 0, N, m)
    b = oracle.bits_per_coeff(N, m, n[0])
    want = oracle.query(key, 1, sk, n, chosen, b, N, m)
    with engine.Context(N, m) as ctx:
        assert np.array_equal(ctx.generate_query(key, 1, sk, n, chosen, b), want)
        torch = pytest.importorskip("torch")
        dq = torch.zeros(want.size, dtype=torch.int64, device="cuda")
        ctx.generate_query(key, 1, sk, n, chosen, b, out=dq)
        assert np.array_equal(dq.cpu().numpy().view(np.uint64), want)


def test_query_matches_reference(engine, ref):
    N, m, n, alpha, F, L, chosen, seed = 1024, 2, [6, 5], 2, 60, 700, 19, 31
    db = np.random.default_rng(2).integers(0, 256, size=F * L, dtype=np.uint8)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=seed, chosen=chosen, extract=False)
    key = ref.seeded_prng_key(seed)
    b = ref.bits_per_coeff(N, m, n[0])
    with engine.Context(N, m) as ctx:
        assert np.array_equal(ctx.generate_query(key, 1, ref.ref_key(N, m, seed), n, chosen, b), r["query"])


@pytest.mark.parametrize("N,m", [(1024, 1), (2048, 2), (4096, 3)])
def test_secret_key_matches_oracle(engine, oracle, N, m):
    key = oracle.seeded_prng_key(12)
    with engine.Context(N, m) as ctx:
        assert np.array_equal(ctx.generate_secret_key(key, 0), oracle.keygen(key, 0, N, m))


def test_gpu_only_round_trip(engine, oracle):
    """Key, query, import, reply and extraction all on the GPU: the chosen aggregated
    element comes back."""
    N, m, n, alpha, F, L, chosen = 2048, 2, [9, 8], 3, 200, 1000, 41
    db = np.random.default_rng(4).integers(0, 256, size=F * L, dtype=np.uint8)
    key = oracle.seeded_prng_key(77)
    b = engine.bits_per_coeff(N, m, n[0])
    with engine.Context(N, m) as ctx:
        sk = ctx.generate_secret_key(key, 0)
        q = ctx.generate_query(key, 1, sk, n, chosen, b)
        dbh = ctx.import_db(db, F, L, alpha, b)
        reply = ctx.reply(dbh, n, q)
        got = ctx.extract(sk, len(n), b, L * alpha, reply)
    assert np.array_equal(got, db[chosen * alpha * L:(chosen + 1) * alpha * L])
