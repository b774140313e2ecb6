"""Full-size workloads pinned to the reference itself (oracle/_ref, XPIR compiled unchanged)
and to the oracle restatement, on the GPU.  Integer work: every comparison is bit for bit.

* Memory-bound workload, exactly: 100,000 elements x 4 KB, LWE:80:2048:120, d = 1, the
  query for element 54,321 generated by XPIR's own PIRQueryGenerator with a seeded key.
  The GPU reply must equal XPIR's reply, and XPIR's PIRReplyExtraction must recover
  element 54,321 from the GPU reply.
* Recursive workload: 1,048,576 elements x 256 B, LWE:80:4096:180, alpha = 16, d = 2,
  n = [1024, n1] with n1 = 1024 when the host has the memory for the reference's
  zero-padding slots (one 96 KiB poly each, all touched: about 103 GB for the full grid)
  and otherwise the largest n1 that fits (at least 64, which holds the 65,536 aggregated
  elements exactly).  The grid used is printed.
* Batched workload's three full shapes on one 65,536 x 8 KB database (d=1/alpha=1,
  d=1/alpha=4, d=2 on a 256 x 256 grid), two queries each in one xpir_b200_reply_batch
  submission, uncaptured and captured in a graph: every reply equals the restatement's
  (oracle/xpir_oracle.c) reply for the same database and query.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu


def mem_available_bytes() -> int:
    with open("/proc/meminfo") as f:
        for line in f:
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    return 0


def test_memory_bound_config_pinned_to_reference(engine, ref):
    N, m, F, L, chosen, keyseed = 2048, 2, 100000, 4096, 54321, 31
    db = random_db(2, F, L)
    r = ref.ref_run(N, m, [F], 1, db, F, L, keyseed=keyseed, chosen=chosen, extract=True)
    assert r["extract_ok"] == 1 and r["polys_per_element"] == 1 and r["nb_elements"] == F
    b = engine.bits_per_coeff(N, m, F)
    assert b == r["bits_per_coeff"]
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, 1, b)
        got = ctx.reply(d, [F], r["query"])
        d.free()
    assert np.array_equal(got, r["reply"]), "GPU reply differs from XPIR's reply"
    plain = ref.ref_extract(N, m, [F], 1, L, keyseed, got)
    assert np.array_equal(plain[:L], db[chosen * L:(chosen + 1) * L]), "XPIR's extraction of the GPU reply"


def recursive_grid() -> list[int]:
    real = (1 << 20) // 16                   # aggregated elements
    per_slot = 4096 * 3 * 8 + 256            # the reference's zero-padding poly per slot, + malloc overhead
    fixed = 40 << 30                         # reference import (6.4 GB) + queries + this process's arrays
    n1 = (mem_available_bytes() - fixed) // (1024 * per_slot)
    return [1024, int(max(real // 1024, min(1024, n1)))]


def test_recursive_config_pinned_to_reference(engine, ref):
    N, m, F, L, alpha, chosen, keyseed = 4096, 3, 1 << 20, 256, 16, 12345, 32
    n = recursive_grid()
    print(f"recursive workload grid: n = {n} (MemAvailable {mem_available_bytes() / 2**30:.0f} GiB)")
    db = random_db(3, F, L)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=keyseed, chosen=chosen, extract=True)
    assert r["extract_ok"] == 1 and r["bits_per_coeff"] == 74
    b = engine.bits_per_coeff(N, m, n[0])
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, alpha, b)
        got = ctx.reply(d, n, r["query"])
        d.free()
    assert got.size == r["reply"].size
    assert np.array_equal(got, r["reply"]), "GPU reply differs from XPIR's reply"


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_config_full_shapes_match_oracle(engine, oracle, use_graph):
    torch = pytest.importorskip("torch")
    N, m, F, L = 2048, 2, 65536, 8192
    elems = random_db(4, F, L)
    classes = [([65536], 1), ([16384], 4), ([256, 256], 1)]
    want, items, dbs = [], [], []
    with engine.Context(N, m) as ctx:
        for k, (n, alpha) in enumerate(classes):
            b = engine.bits_per_coeff(N, m, n[0])
            P = oracle.polys_for_bits(8 * alpha * L, b, N)
            imported = oracle.import_db(elems, F, L, alpha, b, N, m)
            db = ctx.import_db(elems, F, L, alpha, b)
            dbs.append(db)
            for j in range(2):
                q = random_query(100 * k + j, n, N, m, engine.moduli(m))
                want.append(oracle.reply(imported, -(-F // alpha), P, n, q, b, N, m))
                qd = torch.from_numpy(q.view(np.int64)).cuda()
                out = torch.full((want[-1].size,), -1, dtype=torch.int64, device="cuda")
                items.append((db, n, qd, out))
                del q
            del imported
        for _ in range(2 if use_graph else 1):  # captured: capture, then a replay
            for _, _, _, out in items:
                out.fill_(-1)
            counts = ctx.reply_batch(items, use_graph=use_graph)
            for (db, n, qd, out), w, cnt in zip(items, want, counts):
                assert cnt * 2 * m * N == w.size
                assert np.array_equal(out.cpu().numpy().view(np.uint64), w)
        for db in dbs:
            db.free()
