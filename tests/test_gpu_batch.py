"""GPU tests of batched replies, captured batches and the autotuner: every reply must be
bit-identical to the single-query reply of the same query (integer work, no tolerance)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def mixed_batch(engine, ctx, torch):
    """Three databases of one parameter set queried with uneven shapes, as in the batched
    configuration: d=1/alpha=1, d=1/alpha=4 (3 polys per element), d=2, and d=2 with 9 of
    24 level-0 groups idle in every query's row (their re-import is the constant fill)."""
    N, m, F, L = 2048, 2, 600, 3000  # alpha=4 gives 2 polys per element
    elems = random_db(77, F, L)
    shapes = [([600], 1), ([150], 4), ([25, 24], 1), ([40, 24], 1)]
    dbs = []
    for n, alpha in shapes:
        b = engine.bits_per_coeff(N, m, n[0])
        dbs.append(ctx.import_db(elems, F, L, alpha, b))
    items, expect = [], []
    seed = 0
    for (n, alpha), db in zip(shapes, dbs):
        for _ in range(3):
            seed += 1
            q = random_query(1000 + seed, n, N, m, engine.moduli(m))
            want = ctx.reply(db, n, q)
            out = torch.full((want.size,), -1, dtype=torch.int64, device="cuda")
            items.append((db, n, to_dev(torch, q), out))
            expect.append(want)
    return items, expect, dbs


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_single_replies(engine, use_graph):
    torch = pytest.importorskip("torch")
    with engine.Context(2048, 2) as ctx:
        items, expect, _ = mixed_batch(engine, ctx, torch)
        counts = ctx.reply_batch(items, use_graph=use_graph)
        for (db, n, q, out), want, cnt in zip(items, expect, counts):
            assert cnt * 2 * 2 * 2048 == want.size
            assert np.array_equal(out.cpu().numpy().view(np.uint64), want)


def test_graph_replay_with_new_query_contents(engine):
    """A captured batch replayed after the queries' contents change in place gives the
    replies of the new queries."""
    torch = pytest.importorskip("torch")
    with engine.Context(2048, 2) as ctx:
        items, expect, _ = mixed_batch(engine, ctx, torch)
        ctx.reply_batch(items, use_graph=True)  # capture
        for i, (db, n, q, out) in enumerate(items):
            newq = random_query(5000 + i, n, 2048, 2, engine.moduli(2))
            q.copy_(to_dev(torch, newq))
            expect[i] = ctx.reply(db, n, newq)
        ctx.reply_batch(items, use_graph=True)  # replay
        for (db, n, q, out), want in zip(items, expect):
            assert np.array_equal(out.cpu().numpy().view(np.uint64), want)


def test_autotune_keeps_replies_identical(engine, oracle):
    torch = pytest.importorskip("torch")
    N, m, n, F, L = 2048, 2, [3000], 3000, 4096
    b = engine.bits_per_coeff(N, m, n[0])
    db_bytes = random_db(8, F, L)
    q = random_query(9, n, N, m, engine.moduli(m))
    with engine.Context(N, m) as ctx:
        db = ctx.import_db(db_bytes, F, L, 1, b)
        before = ctx.reply(db, n, q)
        tile = ctx.autotune(db, n, to_dev(torch, q))
        assert tile >= 0
        after = ctx.reply(db, n, q)
        assert np.array_equal(before, after)
        assert np.array_equal(after, oracle.reply(db.export(), F, 1, n, q, b, N, m))


def test_graph_of_a_freed_database_is_not_replayed(engine):
    """Captured batches are keyed by database identity, not by handle address: after the
    database a graph read is freed, a new database -- here of the same device size but a
    different shape (200 elements of 2 polys instead of 400 of 1), whose handle the heap
    is likely to place at the freed one's address -- submitted with the same query and
    reply buffers gets its own replies, not a replay of the old graph."""
    torch = pytest.importorskip("torch")
    N, m, n = 2048, 2, [400]
    b = engine.bits_per_coeff(N, m, n[0])
    assert engine.polys_per_element(3000, 1, b, N) == 1 and engine.polys_per_element(12000, 1, b, N) == 2
    with engine.Context(N, m) as ctx:
        q = random_query(41, n, N, m, engine.moduli(m))
        qd = to_dev(torch, q)
        out = torch.full((2 * 2 * m * N,), -1, dtype=torch.int64, device="cuda")
        db1 = ctx.import_db(random_db(42, 400, 3000), 400, 3000, 1, b)
        want1 = ctx.reply(db1, n, q)
        assert ctx.reply_batch([(db1, n, qd, out)], use_graph=True) == [1]  # captured
        assert np.array_equal(out[: want1.size].cpu().numpy().view(np.uint64), want1)
        db1.free()
        db2 = ctx.import_db(random_db(43, 200, 12000), 200, 12000, 1, b)
        want2 = ctx.reply(db2, n, q)
        out.fill_(-1)
        assert ctx.reply_batch([(db2, n, qd, out)], use_graph=True) == [2]
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want2)
        db2.free()
