"""GPU parity tests: the CUDA engine, called through its C ABI, against the reference.

Bit-exact comparisons (integer work, no tolerance) of the imported database and of the
reply ciphertexts with (1) the golden fixtures produced by the XPIR reference, (2) the
reference binary itself where it is built, and (3) the oracle restatement (which the CPU
tests pin to the reference) on randomized shapes, edge inputs and full BASELINE sizes.
Round trips end with the reference's PIRReplyExtraction recovering the chosen element
from the GPU's reply.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from helpers import golden_cases, load_golden, random_db, random_query, shapes

pytestmark = pytest.mark.gpu


def gpu_reply(engine, N, m, n, alpha, db, F, L, b, query, stride=None):
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, alpha, b, element_stride=stride)
        imp = d.export()
        rep = ctx.reply(d, n, query)
        d.free()
    return imp, rep


@pytest.mark.parametrize("name", golden_cases())
def test_golden(engine, name):
    g = load_golden(name)
    mt = g["meta"]
    imp, rep = gpu_reply(engine, mt["N"], mt["m"], mt["n"], mt["alpha"], g["db"], mt["nb_elements"],
                         mt["element_bytes"], mt["bits_per_coeff"], g["query"])
    assert hashlib.sha256(imp.tobytes()).hexdigest() == mt["imported_sha256"]
    assert np.array_equal(rep, g["reply"])


SHAPES = [
    # N, m, n levels, alpha, nb elements, element bytes
    (1024, 1, [40], 1, 40, 12288),        # P = 7 polys per element
    (2048, 2, [300], 1, 300, 4096),       # P = 1, d = 1
    (512, 1, [70], 1, 70, 777),           # odd element size: unaligned bit streams
    (512, 2, [9, 4], 3, 100, 333),        # d = 2, short last group, grid padding
    (4096, 3, [16, 8], 16, 2000, 256),    # the recursive config's shape, smaller grid
    (1024, 2, [5, 5, 4], 1, 100, 3000),   # d = 3
    (1024, 4, [33], 1, 25, 3000),         # four moduli, b > 56, padded grid
    (8192, 1, [6], 1, 6, 20000),          # largest degree
    (2048, 3, [64], 2, 100, 1500),        # alpha = 2, n0 not a multiple of the slot tile
    (512, 1, [1], 1, 1, 100),             # a single slot
    (1024, 2, [4, 8, 3], 1, 9, 700),      # d = 3, 21 of 24 level-0 groups idle: constant re-import
    (512, 3, [8, 5], 1, 3, 5000),         # P > 1, 4 of 5 level-0 groups idle
]


@pytest.mark.parametrize("N,m,n,alpha,F,L", SHAPES)
def test_random_shapes_vs_oracle(engine, oracle, N, m, n, alpha, F, L):
    b, P = shapes(N, m, n, alpha, L, oracle)
    db = random_db(N + F + L, F, L)
    q = random_query(N * 7 + F, n, N, m, oracle.moduli(m))
    imp, rep = gpu_reply(engine, N, m, n, alpha, db, F, L, b, q)
    want_imp = oracle.import_db(db, F, L, alpha, b, N, m)
    assert np.array_equal(imp, want_imp)
    want = oracle.reply(want_imp, -(-F // alpha), P, n, q, b, N, m)
    assert np.array_equal(rep, want)


def test_unreduced_query_words(engine, oracle):
    """Query words of any 64 bits (not reduced mod p): the Shoup factors must still be
    the reference's floor(y*2^64/p) truncated to 64 bits."""
    N, m, n, F, L = 2048, 2, [50], 50, 2000
    b, P = shapes(N, m, n, 1, L, oracle)
    db = random_db(11, F, L)
    q = random_query(12, n, N, m, oracle.moduli(m), reduced=False)
    imp, rep = gpu_reply(engine, N, m, n, 1, db, F, L, b, q)
    assert np.array_equal(rep, oracle.reply(imp, F, P, n, q, b, N, m))


def test_extreme_bytes(engine, oracle):
    """All-ones and all-zero elements, strided element storage."""
    N, m, n, F, L, stride = 1024, 3, [16], 16, 1000, 1024
    b, P = shapes(N, m, n, 1, L, oracle)
    db = np.zeros(F * stride, dtype=np.uint8)
    for i in range(0, F, 2):
        db[i * stride:i * stride + L] = 0xFF
    q = random_query(13, n, N, m, oracle.moduli(m))
    imp, rep = gpu_reply(engine, N, m, n, 1, db, F, L, b, q, stride=stride)
    want_imp = oracle.import_db(db, F, L, 1, b, N, m, stride=stride)
    assert np.array_equal(imp, want_imp)
    assert np.array_equal(rep, oracle.reply(want_imp, F, P, n, q, b, N, m))


@pytest.mark.parametrize("N,m,n,alpha,F,L,chosen", [
    (1024, 1, [1000], 1, 1000, 12288, 137),  # plain single-query config, full size
    (2048, 2, [20, 10], 2, 400, 4096, 77),   # d = 2 round trip
    (4096, 3, [32, 32], 16, 16384, 256, 5),  # recursive config's shape (32x32 grid)
])
def test_round_trip_with_reference(engine, ref, N, m, n, alpha, F, L, chosen):
    """Reference query in, GPU reply out, bit-identical to the reference's reply, and the
    reference's PIRReplyExtraction recovers the chosen element from the GPU reply."""
    db = random_db(chosen + F, F, L)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=77, chosen=chosen, extract=True)
    assert r["extract_ok"] == 1
    b = r["bits_per_coeff"]
    _, rep = gpu_reply(engine, N, m, n, alpha, db, F, L, b, r["query"])
    assert np.array_equal(rep, r["reply"])
    plain = ref.ref_extract(N, m, n, alpha, L, 77, rep)
    assert np.array_equal(plain, db[chosen * alpha * L:(chosen + 1) * alpha * L])


def test_device_resident_inputs_and_outputs(engine, oracle):
    """Query and replies in device memory (torch CUDA tensors): same bits."""
    torch = pytest.importorskip("torch")
    N, m, n, F, L = 2048, 2, [64], 64, 4096
    b, P = shapes(N, m, n, 1, L, oracle)
    db = random_db(21, F, L)
    q = random_query(22, n, N, m, oracle.moduli(m))
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(torch.from_numpy(db).cuda(), F, L, 1, b)
        qd = torch.from_numpy(q.view(np.int64)).cuda()
        out = torch.empty(P * 2 * m * N, dtype=torch.int64, device="cuda")
        ctx.reply(d, n, qd, out)
        rep = out.cpu().numpy().view(np.uint64)
        imp = d.export()
    assert np.array_equal(rep, oracle.reply(imp, F, P, n, q, b, N, m))


def test_full_size_memory_bound_config(engine, oracle):
    """N=2048, 2 moduli, 100,000 elements x 4 KB, d=1: the full benchmark workload,
    checked bit for bit against the oracle restatement."""
    N, m, n, F, L = 2048, 2, [100000], 100000, 4096
    b, P = shapes(N, m, n, 1, L, oracle)
    assert (b, P) == (41, 1)
    db = random_db(2, F, L)
    q = random_query(54321, n, N, m, oracle.moduli(m))
    imp, rep = gpu_reply(engine, N, m, n, 1, db, F, L, b, q)
    want_imp = oracle.import_db(db, F, L, 1, b, N, m)
    assert np.array_equal(imp, want_imp)
    assert np.array_equal(rep, oracle.reply(want_imp, F, P, n, q, b, N, m))


def test_launch_count_and_reuse(engine, oracle):
    """One context, one database, several queries: every reply independent of the
    previous ones (no state leaks through the workspaces)."""
    N, m, n, F, L = 1024, 2, [8, 4], 30, 900
    b, P = shapes(N, m, n, 1, L, oracle)
    db = random_db(31, F, L)
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, 1, b)
        imp = d.export()
        before = ctx.launch_count
        for s in range(3):
            q = random_query(100 + s, n, N, m, oracle.moduli(m))
            rep = ctx.reply(d, n, q)
            assert np.array_equal(rep, oracle.reply(imp, F, P, n, q, b, N, m))
        # per reply: 2 level kernels and 1 re-import (every level-0 group holds data)
        assert ctx.launch_count - before == 3 * 3


def test_context_close_releases_databases(engine, oracle):
    """Closing a context frees the databases imported through it; freeing such a
    database afterwards (explicitly or by garbage collection) is harmless."""
    ctx = engine.Context(1024, 1)
    d = ctx.import_db(random_db(41, 10, 500), 10, 500, 1, oracle.bits_per_coeff(1024, 1, 10))
    ctx.close()
    d.free()
    del d
    with engine.Context(1024, 1) as ctx2:
        d2 = ctx2.import_db(random_db(42, 10, 500), 10, 500, 1, oracle.bits_per_coeff(1024, 1, 10))
    del d2


def test_full_size_recursive_config(engine, oracle):
    """N=4096, 3 moduli, d=2 on a 1024x1024 grid, alpha=16, 1,048,576 elements x 256 B:
    the full recursive configuration (65,536 aggregated elements, 983,040 zero-padding
    slots never materialised), bit for bit against the oracle restatement."""
    N, m, n, alpha, F, L = 4096, 3, [1024, 1024], 16, 1048576, 256
    b, P = shapes(N, m, n, alpha, L, oracle)
    assert (b, P) == (74, 1)
    db = random_db(3, F, L)
    q = random_query(5, n, N, m, oracle.moduli(m))
    imp, rep = gpu_reply(engine, N, m, n, alpha, db, F, L, b, q)
    want_imp = oracle.import_db(db, F, L, alpha, b, N, m)
    assert np.array_equal(imp, want_imp)
    want = oracle.reply(want_imp, F // alpha, P, n, q, b, N, m)
    assert rep.size == want.size == 6 * 2 * m * N
    assert np.array_equal(rep, want)
