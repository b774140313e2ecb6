"""GPU tests of the serving loop (xpir_b200_server_*): queries from several clients on
databases of two parameter sets, admitted by a device-memory budget and batched as they
arrive.  Every served reply must be bit-identical to the single-query reply of the same
query computed alone, and that reply to the oracle restatement's (integer work, no
tolerance)."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu


def make_load(engine, ctxs, oracle=None):
    """Databases on two parameter sets with d in {1, 2} and alpha in {1, 4}, and a list of
    (db, n, host query, expected reply) of 4 queries per database.  With the oracle, each
    expected reply is first checked against the restatement's."""
    (ctx_a, (Na, ma)), (ctx_b, (Nb, mb)) = ctxs
    specs = [(ctx_a, Na, ma, 900, 2000, [900], 1), (ctx_a, Na, ma, 900, 2000, [30, 30], 1),
             (ctx_b, Nb, mb, 1200, 700, [300], 4), (ctx_b, Nb, mb, 1200, 700, [20, 15], 4)]
    load, dbs = [], []
    for k, (ctx, N, m, F, L, n, alpha) in enumerate(specs):
        elems = random_db(300 + k, F, L)
        b = engine.bits_per_coeff(N, m, n[0])
        db = ctx.import_db(elems, F, L, alpha, b)
        dbs.append(db)
        imported = oracle.import_db(elems, F, L, alpha, b, N, m) if oracle else None
        for j in range(4):
            q = random_query(7000 + 10 * k + j, n, N, m, engine.moduli(m))
            want = ctx.reply(db, n, q)
            if oracle:
                P = oracle.polys_for_bits(8 * alpha * L, b, N)
                assert np.array_equal(want, oracle.reply(imported, -(-F // alpha), P, n, q, b, N, m))
            load.append((db, n, q, want))
    return load, dbs


def serve_all(engine, server, load, clients=4):
    """Submits the load from `clients` threads at once; returns the replies by index."""
    outs = [np.full(want.size, 0xDEAD, dtype=np.uint64) for (_, _, _, want) in load]
    counts = [None] * len(load)
    errors = []

    def client(idx):
        try:
            tickets = [(i, server.submit(load[i][0], load[i][1], load[i][2], outs[i])) for i in idx]
            for i, t in tickets:
                counts[i] = server.wait(t, timeout_ms=60000)[0]
        except Exception as e:  # reported below, in the test's thread
            errors.append(e)

    threads = [threading.Thread(target=client, args=(list(range(c, len(load), clients)),)) for c in range(clients)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    return outs, counts


def test_served_replies_equal_replies_alone(engine, oracle):
    with engine.Context(1024, 1) as ca, engine.Context(2048, 2) as cb:
        load, _ = make_load(engine, [(ca, (1024, 1)), (cb, (2048, 2))], oracle)
        with engine.Server([ca, cb], device_budget_bytes=1 << 30, max_batch=16) as srv:
            outs, counts = serve_all(engine, srv, load)
            st = srv.stats()
        for (db, n, q, want), got, cnt in zip(load, outs, counts):
            assert cnt * engine.ciphertext_bytes(db.ctx.N, db.ctx.m) == want.size * 8
            assert np.array_equal(got, want)
        assert st["completed"] == len(load)
        assert st["max_batch"] >= 1


def test_small_budget_queues_but_stays_exact(engine):
    """A budget that admits about one query at a time: queries wait for memory, results
    are unchanged, and the admitted bytes never exceed the budget."""
    with engine.Context(1024, 1) as ca, engine.Context(2048, 2) as cb:
        load, _ = make_load(engine, [(ca, (1024, 1)), (cb, (2048, 2))])
        fp = [engine.Server.footprint(db, n) for (db, n, _, _) in load]
        budget = max(fp) + min(fp) // 2  # the largest query fits, two large ones do not
        with engine.Server([ca, cb], device_budget_bytes=budget, max_batch=8) as srv:
            outs, _ = serve_all(engine, srv, load)
            st = srv.stats()
        for (_, _, _, want), got in zip(load, outs):
            assert np.array_equal(got, want)
        assert st["peak_device_bytes"] <= budget
        assert st["completed"] == len(load)


def test_oversize_query_refused(engine):
    with engine.Context(1024, 1) as ca:
        F, L = 500, 1000
        db = ca.import_db(random_db(5, F, L), F, L, 1, engine.bits_per_coeff(1024, 1, F))
        q = random_query(6, [F], 1024, 1, engine.moduli(1))
        out = np.zeros(ca.reply(db, [F], q).size, dtype=np.uint64)
        with engine.Server([ca], device_budget_bytes=4096) as srv:
            with pytest.raises(engine.XpirError) as ei:
                srv.submit(db, [F], q, out)
            assert ei.value.status == engine.ERR_NOMEM


def test_large_pinned_query_is_pulled_and_exact(engine):
    """A query of 256 MB or more in pinned host memory is pulled over PCIe by the server's
    copy kernel instead of the copy engine; pageable queries of the same size take the copy
    engine.  Both replies equal the reply computed alone, and small queries served beside
    them too."""
    import torch

    N, m, F, L = 2048, 2, 4500, 4096
    n = [F]  # 4,500 ciphertexts of 64 KB: 295 MB of query
    b = engine.bits_per_coeff(N, m, n[0])
    with engine.Context(1024, 1) as ca, engine.Context(N, m) as cb:
        db = cb.import_db(random_db(91, F, L), F, L, 1, b)
        q = random_query(92, n, N, m, engine.moduli(m))
        want = cb.reply(db, n, q)
        pinned = torch.from_numpy(q.view(np.int64)).pin_memory()
        small, _ = make_load(engine, [(ca, (1024, 1)), (cb, (2048, 2))])
        with engine.Server([ca, cb], device_budget_bytes=4 << 30, max_batch=16) as srv:
            # alone, each: the pinned query costs one launch more (the pull kernel)
            deltas = []
            for buf in (pinned.numpy().view(np.uint64), q):
                before = cb.launch_count
                outs, _ = serve_all(engine, srv, [(db, n, buf, want)], clients=1)
                assert np.array_equal(outs[0], want)
                deltas.append(cb.launch_count - before)
            assert deltas[0] == deltas[1] + 1, deltas
            big = [(db, n, pinned.numpy().view(np.uint64), want), (db, n, q, want)]
            outs, _ = serve_all(engine, srv, big + small, clients=3)
        for (_, _, _, w), got in zip(big + small, outs):
            assert np.array_equal(got, w)


def test_context_outlives_its_server(engine):
    """A context cannot be destroyed while a server has a lane on it (the C call refuses
    with XPIR_B200_ERR_STATE and destroys nothing); Context.close() closes the server first."""
    lib = engine._load()
    ctx = engine.Context(1024, 1)
    srv = engine.Server([ctx], device_budget_bytes=1 << 28, max_batch=4)
    assert lib.xpir_b200_ctx_destroy(ctx.handle) == engine.ERR_STATE
    assert ctx.launch_count >= 0  # still alive
    ctx.close()
    assert srv.handle is None and ctx.handle is None


def test_parameter_sets_launch_concurrently(engine):
    """Contexts of different parameter sets running recursive replies (import and re-import
    kernels whose shared memory depends on N) from several threads at once: every call
    succeeds and equals its single-threaded result (a per-launch shared-memory attribute
    set by one thread between another's setting and launch once made such launches fail)."""
    specs = [(1024, 1, [12, 8], 900), (4096, 3, [10, 6], 700), (2048, 2, [14, 5], 800)]
    work = []
    for k, (N, m, n, L) in enumerate(specs):
        ctx = engine.Context(N, m)
        F = n[0] * n[1]
        b = engine.bits_per_coeff(N, m, n[0])
        db = ctx.import_db(random_db(500 + k, F, L), F, L, 1, b)
        q = random_query(600 + k, n, N, m, engine.moduli(m))
        work.append((ctx, db, n, q, ctx.reply(db, n, q)))
    errors = []

    def run(ctx, db, n, q, want):
        try:
            for _ in range(25):
                assert np.array_equal(ctx.reply(db, n, q), want)
        except Exception as e:  # reported in the test's thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=w) for w in work for _ in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for ctx, *_ in work:
        ctx.close()
    assert not errors, errors[:3]
