"""GPU test of xpir_b200_reply_noalloc, the reply entry point that allocates nothing.

It serves callers that cannot allocate device memory while they answer a query (for
example code that set up all its memory in advance under a fixed budget, or that runs
inside an allocator hook of its own).  Such a caller passes the query and the reply
buffer in device memory, and the recursion's intermediate data goes to a fixed scratch
area the library keeps in each GPU's global memory.

The test calls the entry point through the C ABI and requires its replies to be
bit-identical (integer data: no tolerance) to those of the allocating entry point,
xpir_b200_reply, on two calls in a row (the scratch keeps the first call's contents),
that the first recursive call on a new context changes neither the device's free memory
nor torch's allocator, and that a query whose intermediate data exceeds the scratch is
rejected.
This file is named to be collected last, so that a run stopping at its first failure
has run every other test before it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 64 << 20  # XPIR_B200_NOALLOC_SCRATCH_BYTES


def noalloc_fn(engine):
    fn = engine.lib().xpir_b200_reply_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    return fn


def reply_noalloc(engine, ctx, db, n, q_dev, out_dev):
    narr = (ctypes.c_uint32 * len(n))(*n)
    count = ctypes.c_uint64(0)
    status = noalloc_fn(engine)(ctx.handle, db.handle, len(n), narr, q_dev.data_ptr(), out_dev.data_ptr(),
                                out_dev.numel() * 8, ctypes.byref(count))
    return status, count.value


@pytest.mark.parametrize("N,m,n,alpha,F,L", [
    (1024, 2, [16, 12], 1, 150, 2000),   # d = 2: level replies and the level-1 database in scratch
    (2048, 2, [10, 6, 4], 2, 400, 1500),  # d = 3: the scratch is reused level after level
    (2048, 2, [300], 1, 300, 4096),      # d = 1: no scratch needed
])
def test_noalloc_matches_allocating_reply(engine, oracle, N, m, n, alpha, F, L):
    torch = pytest.importorskip("torch")
    b = oracle.bits_per_coeff(N, m, n[0])
    db_bytes = random_db(N + F, F, L)
    with engine.Context(N, m) as ctx:
        db = ctx.import_db(db_bytes, F, L, alpha, b)
        for call in range(2):
            q = random_query(900 + call, n, N, m, engine.moduli(m))
            want = ctx.reply(db, n, q)  # allocating entry point, host buffers
            q_dev = torch.from_numpy(q.view(np.int64)).cuda()
            out_dev = torch.full((want.size,), -1, dtype=torch.int64, device="cuda")
            status, count = reply_noalloc(engine, ctx, db, n, q_dev, out_dev)
            assert status == engine.OK, engine.lib().xpir_b200_strerror(status)
            assert count * 2 * m * N == want.size
            got = out_dev.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, want), f"call {call}"
        db.free()


def test_noalloc_first_call_allocates_nothing(engine, oracle):
    """The first d = 2 call on a fresh context: the context's creation has already loaded
    the engine's kernels and the scratch area onto the device, so the call leaves the
    device's free memory (cudaMemGetInfo) and torch's allocator statistics unchanged."""
    torch = pytest.importorskip("torch")
    N, m, n, F, L = 1024, 2, [16, 12], 150, 2000
    b = oracle.bits_per_coeff(N, m, n[0])
    q = random_query(77, n, N, m, engine.moduli(m))
    with engine.Context(N, m) as ctx:
        db = ctx.import_db(random_db(76, F, L), F, L, 1, b)
        q_dev = torch.from_numpy(q.view(np.int64)).cuda()
        count_want = engine.reply_count(L, 1, len(n), b, N, m)
        out_dev = torch.full((count_want * 2 * m * N,), -1, dtype=torch.int64, device="cuda")
        ctx.synchronize()
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        stats_before = torch.cuda.memory_stats()
        status, count = reply_noalloc(engine, ctx, db, n, q_dev, out_dev)
        assert status == engine.OK, engine.lib().xpir_b200_strerror(status)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        stats_after = torch.cuda.memory_stats()
        assert free_after == free_before
        for key in ("allocation.all.allocated", "reserved_bytes.all.current", "allocated_bytes.all.current"):
            assert stats_after.get(key) == stats_before.get(key), key
        want = ctx.reply(db, n, q)
        assert count * 2 * m * N == want.size
        assert np.array_equal(out_dev.cpu().numpy().view(np.uint64), want)
        db.free()


def test_noalloc_rejects_queries_larger_than_scratch(engine, oracle):
    torch = pytest.importorskip("torch")
    # d = 2 with 1024 level-0 groups of N=4096, 3 moduli: 1024 level replies of 192 KiB
    # alone exceed the scratch.
    N, m, n, F, L = 4096, 3, [2, 1024], 8, 100
    b = oracle.bits_per_coeff(N, m, n[0])
    with engine.Context(N, m) as ctx:
        db = ctx.import_db(random_db(5, F, L), F, L, 1, b)
        assert 1024 * 2 * m * N * 8 > SCRATCH_BYTES
        q_dev = torch.zeros(sum(n) * 2 * m * N, dtype=torch.int64, device="cuda")
        out_dev = torch.zeros(16 * 2 * m * N, dtype=torch.int64, device="cuda")
        status, _ = reply_noalloc(engine, ctx, db, n, q_dev, out_dev)
        assert status == engine.ERR_ARG
        db.free()
