"""CPU tests of the engine library: it loads, exports exactly the ABI its header
declares, its host-side sizing matches the reference's formulas, and its calls fail
cleanly (status codes, no abort) where no GPU is present.  No compute calls here."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "xpir_b200.h"


def declared_symbols() -> list[str]:
    return re.findall(r"XPIR_B200_API[^;]*?\b(xpir_b200_\w+)\s*\(", HEADER.read_text())


def test_library_exports_every_declared_symbol():
    import xpir_b200

    L = xpir_b200.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(xpir_b200.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported == set(names)


@pytest.mark.parametrize("N,m,n0", [(1024, 1, 1000), (2048, 2, 100000), (4096, 3, 1024), (2048, 2, 256),
                                     (512, 1, 7), (8192, 4, 3), (2048, 2, 65536), (1024, 2, 200000)])
def test_sizing_matches_oracle(oracle, N, m, n0):
    import xpir_b200

    b = xpir_b200.bits_per_coeff(N, m, n0)
    assert b == oracle.bits_per_coeff(N, m, n0)
    for L, alpha in [(12288, 1), (4096, 1), (256, 16), (8192, 4), (1, 1), (12345, 3)]:
        assert xpir_b200.polys_per_element(L, alpha, b, N) == oracle.polys_for_bits(8 * alpha * L, b, N)
        for d in (1, 2, 3):
            assert xpir_b200.reply_count(L, alpha, d, b, N, m) == oracle.reply_count(L, alpha, d, b, N, m)
    assert xpir_b200.ciphertext_bytes(N, m) == 16 * m * N


def test_baseline_config_sizes():
    """Sizes of the benchmark configurations, from the reference's formulas."""
    import xpir_b200 as x

    assert x.bits_per_coeff(1024, 1, 1000) == 15 and x.polys_per_element(12288, 1, 15, 1024) == 7
    assert x.bits_per_coeff(2048, 2, 100000) == 41 and x.polys_per_element(4096, 1, 41, 2048) == 1
    assert x.bits_per_coeff(4096, 3, 1024) == 74 and x.polys_per_element(256, 16, 74, 4096) == 1
    assert x.reply_count(256, 16, 2, 74, 4096, 3) == 6


def test_invalid_shapes_rejected_without_gpu():
    import xpir_b200

    for N, m in [(1000, 1), (256, 1), (16384, 1), (1024, 0), (1024, 18)]:
        with pytest.raises(xpir_b200.XpirError) as ei:
            xpir_b200.Context(N, m)
        assert ei.value.status == xpir_b200.ERR_ARG
    assert xpir_b200.bits_per_coeff(1000, 1, 10) == 0


def test_tile_table_and_pinning_arguments_without_gpu():
    """The tile table is compiled in (one-column, poly-column and group-column shapes);
    pinning a tile needs a context and a real level shape."""
    import ctypes

    import xpir_b200

    assert xpir_b200.tile_count() >= 20
    L = xpir_b200.lib()
    assert L.xpir_b200_set_level_tile(None, 1, 16, 4, 0) == xpir_b200.ERR_ARG
    assert L.xpir_b200_set_level_tile(None, 0, 16, 4, -1) == xpir_b200.ERR_ARG
    assert L.xpir_b200_set_level_tile(ctypes.c_void_p(0), 1, 0, 4, 0) == xpir_b200.ERR_ARG


def test_no_device_is_an_error_not_a_fallback():
    import xpir_b200

    if xpir_b200.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(xpir_b200.XpirError) as ei:
        xpir_b200.Context(1024, 1)
    assert ei.value.status == xpir_b200.ERR_NODEV


def test_shoup_factor_formula_host(tmp_path):
    exe = tmp_path / "test_modarith"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), str(ROOT / "tests" / "cpp" / "test_modarith.cpp"),
                    str(ROOT / "xpir_b200" / "csrc" / "params.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")


def test_admission_and_continuous_batching_host(tmp_path):
    """The serving loop's queueing rules (xpir_b200/csrc/admission.h) under a fake executor:
    FIFO per lane, budget never exceeded, oversize refused, batches formed from arrivals,
    lanes concurrent, head-of-line job waits for memory."""
    exe = tmp_path / "test_admission"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "test_admission.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")


def test_optimizer_cache_parameter_parsing():
    from xpir_b200 import optim_cache

    assert optim_cache.parse_params("LWE:80:2048:120") == (80, 2048, 2)
    with pytest.raises(ValueError):
        optim_cache.parse_params("LWE:80:2048:100")
