"""Kernel timing of xpir_b200_reply (xpir_b200_ctx_set_kernel_timing / _kernel_time): the
engine records a CUDA event pair on its stream around each level's reply launch and each
re-import, and sums the elapsed times after the call's synchronisation.  The replies stay
bit-identical, the counts follow the launches, and the times are positive and within the
calls' wall time."""
from __future__ import annotations

import time

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu


def test_kernel_timing_counts_and_bounds(engine):
    N, m, n, alpha, L = 2048, 2, [40, 24], 2, 3000
    F = n[0] * alpha * (n[1] // 2)
    b = engine.bits_per_coeff(N, m, n[0])
    q = random_query(72, n, N, m, engine.moduli(m))
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(random_db(71, F, L), F, L, alpha, b)
        want = ctx.reply(d, n, q)
        ctx.set_kernel_timing(True)
        t0 = time.perf_counter()
        for _ in range(3):
            assert np.array_equal(ctx.reply(d, n, q), want)
        wall_ms = (time.perf_counter() - t0) * 1e3
        kt = ctx.kernel_time()
        assert kt["reply_launches"][:3] == [3, 3, 0] and kt["import_launches"] == 3
        assert all(t > 0 for t in kt["reply_ms"][:2]) and kt["import_ms"] > 0
        assert sum(kt["reply_ms"]) + kt["import_ms"] < wall_ms
        ctx.set_kernel_timing(False)
        ctx.reply(d, n, q)
        assert ctx.kernel_time() == kt  # sums kept, nothing added while off
        ctx.set_kernel_timing(True)
        assert ctx.kernel_time()["reply_launches"][0] == 0  # switching on restarts the sums
        d.free()
