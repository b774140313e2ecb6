"""GPU test of the optimizer cost measurement and the cache writer (xpir_b200.optim_cache):
positive per-plaintext costs, and a cache file in the format XPIR's OptimService reads
(parameter string, then the reply and import seconds per plaintext)."""
from __future__ import annotations

import math

import pytest

pytestmark = pytest.mark.gpu


def test_measure_costs_and_cache_file(engine, tmp_path):
    from xpir_b200 import optim_cache

    with engine.Context(2048, 2) as ctx:
        reply, imp = ctx.measure_costs(80, 0.01)
    assert 0 < reply < 1e-2 and 0 < imp < 1e-2 and math.isfinite(reply) and math.isfinite(imp)
    params = ["LWE:80:2048:120", "LWE:97:1024:60"]
    lines = optim_cache.cache_lines(params, target_s=0.01)
    for param, line in zip(params, lines):
        f = line.split(" ")
        assert f[0] == param and len(f) == 3 and float(f[1]) > 0 and float(f[2]) > 0

