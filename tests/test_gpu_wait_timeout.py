"""The reply kernel's bounded waits, made to run out on purpose (xpir_b200_ctx_set_wait_test).

Every mbarrier wait in the reply kernel gives up after a bounded number of polls,
records kStatusWaitTimeout in the context's status word and lets the CTA return once its
own copies in flight have landed; the C ABI then reports XPIR_B200_ERR_TIMEOUT.  Here
the copy producer of every CTA stops before one tile's copies, so that the consumers'
waits for that tile run out (a short limit keeps the test fast).  Nothing faults or
spins without a bound: the producer issues no copy it does not wait for, and every
consumer wait is bounded.  The same context must then answer the next query bit-exactly.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu

SHORT_LIMIT = 16384  # polls per wait; each poll suspends for at most 20 us


@pytest.mark.parametrize("n,alpha,L", [([3000], 1, 4096), ([40, 24], 2, 3000)])
def test_withheld_tile_times_out_and_context_recovers(engine, oracle, n, alpha, L):
    N, m = 2048, 2
    F = n[0] * alpha * (n[1] // 2 if len(n) > 1 else 1)
    b = engine.bits_per_coeff(N, m, n[0])
    db_bytes = random_db(61, F, L)
    q = random_query(62, n, N, m, engine.moduli(m))
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db_bytes, F, L, alpha, b)
        want = ctx.reply(d, n, q)
        assert np.array_equal(want, oracle.reply(d.export(), -(-F // alpha), d.polys_per_element, n, q, b, N, m))

        ctx.set_wait_test(SHORT_LIMIT, 1)
        t0 = time.perf_counter()
        with pytest.raises(engine.XpirError) as err:
            ctx.reply(d, n, q)
        took = time.perf_counter() - t0
        assert err.value.status == engine.ERR_TIMEOUT
        assert took < 30, f"the timed-out reply took {took:.1f} s"

        ctx.set_wait_test(0, -1)
        again = ctx.reply(d, n, q)
        assert np.array_equal(again, want), "reply after a timed-out one differs"
        d.free()


def test_short_wait_limit_alone_changes_nothing(engine):
    """A short limit without a withheld tile still lets every wait complete."""
    N, m, n, F, L = 2048, 2, [3000], 3000, 4096
    b = engine.bits_per_coeff(N, m, n[0])
    q = random_query(64, n, N, m, engine.moduli(m))
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(random_db(63, F, L), F, L, 1, b)
        want = ctx.reply(d, n, q)
        ctx.set_wait_test(SHORT_LIMIT, -1)
        assert np.array_equal(ctx.reply(d, n, q), want)
        ctx.set_wait_test(0, -1)
        d.free()
