"""XPIR itself, with the B200 reply engine plugged in: the nine cases of XPIR's
apps/simplepir/simplePIR.cpp (seeded data) run through XPIR's own classes, once with the
stock libpir and reply-generator factory (oracle/_ref/xpir_simplepir) and once with the B200
ones (tests/cpp/_build/xpir_simplepir_b200, linked against xpir_b200/xpir/_build/libpir_b200.a
and libxpir_b200.so).  Keys and queries come from XPIR's PIRQueryGenerator with the same
seeded PRNG on both sides; every reply ciphertext must be byte-identical, and XPIR's
PIRReplyExtraction must recover the chosen element from the B200 replies.

Two flows per case:
  libpir  PIRReplyGenerator::pushQuery / importData / generateReply / popReply, as
          simplePIR drives libpir (apps/simplepir/simplePIR.cpp:3-182);
  server  the GenericPIRReplyGenerator virtuals the way XPIR's server drives them
          (apps/server/PIRSession.cpp:215-240, 383-565): a generator from
          PIRReplyGeneratorFactory("LWE"), pushQuery(buf, size, dim, nbr) from a download
          thread, replies taken from repliesArray by an upload thread, a first session
          that keeps the imported database (driven mode, PIRServer.cpp:71-104) and a second
          session replying from it with generateReplyGenericFromData.
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
B200_EXE = ROOT / "tests" / "cpp" / "_build" / "xpir_simplepir_b200"
STOCK_EXE = ROOT / "oracle" / "_ref" / "xpir_simplepir"
ARCHIVE = ROOT / "xpir_b200" / "xpir" / "_build" / "libpir_b200.a"


def need(path: Path):
    if not path.exists():
        pytest.skip(f"{path.relative_to(ROOT)} is not built (built by __graft_entry__.build() from the XPIR sources)")


def test_archive_replaces_libpir_and_factory():
    """The pir library built for XPIR holds the B200 libpir and factory, not the stock ones."""
    need(ARCHIVE)
    members = subprocess.run(["ar", "t", str(ARCHIVE)], capture_output=True, text=True, check=True).stdout.split()
    for m in ("libpir_b200.o", "PIRReplyGeneratorFactory_b200.o", "PIRReplyGeneratorB200.o", "b200_engine.o"):
        assert m in members, m
    assert "libpir.o" not in members and "PIRReplyGeneratorFactory.o" not in members
    syms = subprocess.run(["nm", "-C", "--defined-only", str(ARCHIVE)], capture_output=True, text=True,
                          check=True).stdout
    for s in ("PIRReplyGenerator::generateReply(imported_database const*)",
              "PIRReplyGeneratorFactory::getPIRReplyGenerator(", "PIRReplyGeneratorB200::generateReplyGeneric(bool)",
              "imported_database::~imported_database()"):
        assert s in syms, s


def run(exe: Path, mode: str, case: int, workdir: Path) -> dict:
    workdir.mkdir(parents=True, exist_ok=True)
    out = subprocess.run([str(exe), mode, str(case), str(workdir)], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, f"{exe.name} {mode} {case}: rc {out.returncode}\n{out.stdout}\n{out.stderr[-3000:]}"
    return json.loads(out.stdout.strip().splitlines()[-1])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["libpir", "server"])
@pytest.mark.parametrize("case", range(1, 10))
def test_simplepir_case_bit_identical(tmp_path, case, mode):
    need(B200_EXE)
    need(STOCK_EXE)
    got = run(B200_EXE, mode, case, tmp_path / "b200")
    want = run(STOCK_EXE, mode, case, tmp_path / "stock")
    assert got["extract_ok"] == 1, got
    assert got["replies"] == want["replies"] > 0
    files = ["replies.bin", "replies2.bin"] if mode == "server" else ["replies.bin"]
    for name in files:
        a = (tmp_path / "b200" / name).read_bytes()
        b = (tmp_path / "stock" / name).read_bytes()
        assert len(a) == len(b) > 0, name
        assert a == b, f"{name}: replies differ from the stock XPIR build"
    if mode == "server":
        assert got["kept_database"] == 1 and got["extract2_ok"] == 1 and got["replies2"] == want["replies2"]
