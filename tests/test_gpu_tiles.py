"""Every compiled reply tile shape, pinned one at a time on the level shapes it can run
(Context.set_level_tile), against the oracle: poly columns, group columns (one-poly
levels whose groups share each query tile), partial last groups, idle groups, and the
batched (descriptor-table) form.  Integer work: bit-exact, no tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_db, random_query

pytestmark = pytest.mark.gpu

# N, m, n levels, alpha, nb elements, element bytes
SHAPES = [
    (1024, 2, [16, 7], 1, 100, 500),   # 7 one-poly groups, the last one partial (4 real slots)
    (1024, 2, [16, 8], 1, 40, 500),    # 3 of 8 groups with data, 5 idle
    (2048, 1, [9, 12], 1, 100, 1000),  # n_i not a multiple of any slot tile
]


def level_shapes(engine, N, m, n, alpha, L, P0):
    """(P, n_i, groups) of every level, as the engine keys its tile choices."""
    out, P = [], P0
    ct_bits = 2 * m * N * 64
    b = engine.bits_per_coeff(N, m, n[0])
    for lvl in range(len(n)):
        groups = int(np.prod(n[lvl + 1:])) if lvl + 1 < len(n) else 1
        out.append((P, n[lvl], groups))
        P = engine.polys_per_element(P * ct_bits // 8, 1, b, N)
    return out


def fitting_tiles(engine, ctx, key):
    tiles = []
    for t in range(engine.tile_count()):
        try:
            ctx.set_level_tile(*key, t)
        except Exception:
            continue
        tiles.append(t)
    ctx.set_level_tile(*key, -1)
    return tiles


@pytest.mark.parametrize("N,m,n,alpha,F,L", SHAPES)
def test_every_tile_equals_oracle(engine, oracle, N, m, n, alpha, F, L):
    b = engine.bits_per_coeff(N, m, n[0])
    db = random_db(61, F, L)
    q = random_query(62, n, N, m, oracle.moduli(m))
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, alpha, b)
        P0 = d.polys_per_element
        imp = d.export()
        want = oracle.reply(imp, -(-F // alpha), P0, n, q, b, N, m)
        keys = level_shapes(engine, N, m, n, alpha, L, P0)
        assert keys[0][0] == 1  # a one-poly first level: group tiles apply
        tried = 0
        for lvl, key in enumerate(keys):
            tiles = fitting_tiles(engine, ctx, key)
            if key[0] == 1:
                assert len(tiles) >= 8  # one-column and group-column shapes
            for t in tiles:
                ctx.set_level_tile(*key, t)
                rep = ctx.reply(d, n, q)
                assert np.array_equal(rep, want), f"level {lvl} tile {t}"
                tried += 1
            ctx.set_level_tile(*key, -1)
        assert tried > 0


def test_group_tiles_in_batches(engine, oracle):
    """The descriptor-table kernel with group columns: a batch of queries on a pinned
    group tile gives each query's oracle reply."""
    torch = pytest.importorskip("torch")
    N, m, n, F, L = 1024, 2, [16, 7], 100, 500
    b = engine.bits_per_coeff(N, m, n[0])
    db = random_db(71, F, L)
    with engine.Context(N, m) as ctx:
        d = ctx.import_db(db, F, L, 1, b)
        imp = d.export()
        key = level_shapes(engine, N, m, n, 1, L, d.polys_per_element)[0]
        # group-column tiles: those that run one-poly levels but not two-poly ones
        two_poly = set(fitting_tiles(engine, ctx, (2,) + key[1:]))
        group_tiles = [t for t in fitting_tiles(engine, ctx, key) if t not in two_poly]
        assert group_tiles
        for t in group_tiles:
            ctx.set_level_tile(*key, t)
            items, want = [], []
            for s in range(3):
                q = random_query(80 + s, n, N, m, oracle.moduli(m))
                w = oracle.reply(imp, F, 1, n, q, b, N, m)
                out = torch.full((w.size,), -1, dtype=torch.int64, device="cuda")
                items.append((d, n, torch.from_numpy(q.view(np.int64)).cuda(), out))
                want.append(w)
            ctx.reply_batch(items)
            for (_, _, _, out), w in zip(items, want):
                assert np.array_equal(out.cpu().numpy().view(np.uint64), w), f"tile {t}"


def test_set_level_tile_rejects_unfit_tiles(engine):
    with engine.Context(1024, 1) as ctx:
        count = engine.tile_count()
        for bad in (count, -2):
            with pytest.raises(Exception):
                ctx.set_level_tile(1, 16, 4, bad)
        # group columns need one poly per element
        with pytest.raises(Exception):
            ctx.set_level_tile(3, 16, 4, count - 1)
