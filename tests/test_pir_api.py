"""The libpir-shaped C++ API (include/xpir_b200_pir.hpp, xpir_b200/libxpir_b200_pir.so),
driven by tests/cpp/test_pir_api.cpp the way a libpir server drives PIRReplyGenerator.
Host-only checks run everywhere; the reply runs (gpu) compare the popped replies, from
generateReply and from the memory-chunked generateReplyGeneric, bit for bit with the
oracle restatement of the reference."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import random_query

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def pir_exe(tmp_path_factory):
    from xpir_b200 import build as engine_build

    engine_build.build()
    lib = engine_build.build_pir()
    exe = tmp_path_factory.mktemp("pir") / "test_pir_api"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "test_pir_api.cpp"), "-L", str(lib.parent), "-l:libxpir_b200_pir.so",
                    "-l:libxpir_b200.so", f"-Wl,-rpath,{lib.parent}"], check=True)
    return exe


def test_pir_api_parameters_host(pir_exe, oracle):
    b = oracle.bits_per_coeff(2048, 2, 100000)
    out = subprocess.run([str(pir_exe), "params", "LWE:80:2048:120", "100000", str(b), str(2 * 2 * 2048 * 8)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok params")


def run_case(pir_exe, oracle, tmp_path, N, m, alpha, n, sizes, seed, budget):
    """Elements of the given byte sizes (short ones read as zero-padded to the longest,
    as DBVectorProcessor does); returns (reply, generic reply, expected, output line)."""
    rng = np.random.default_rng(seed)
    elems = [rng.integers(0, 256, size=s, dtype=np.uint8) for s in sizes]
    L = max(sizes)
    padded = np.zeros((len(sizes), L), dtype=np.uint8)
    for i, e in enumerate(elems):
        padded[i, :len(e)] = e
    q = random_query(seed + 1, n, N, m, oracle.moduli(m))
    (tmp_path / "params.txt").write_text(f"LWE:80:{N}:{60 * m} {alpha} {len(n)} {' '.join(map(str, n))} {budget}\n")
    (tmp_path / "sizes.bin").write_bytes(np.array(sizes, dtype=np.uint64).tobytes())
    (tmp_path / "db.bin").write_bytes(b"".join(e.tobytes() for e in elems))
    (tmp_path / "query.bin").write_bytes(q.tobytes())
    out = subprocess.run([str(pir_exe), "run", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    b = oracle.bits_per_coeff(N, m, n[0])
    P = oracle.polys_for_bits(8 * alpha * L, b, N)
    db = oracle.import_db(padded.reshape(-1), len(sizes), L, alpha, b, N, m)
    want = oracle.reply(db, -(-len(sizes) // alpha), P, n, q, b, N, m)
    rep = np.frombuffer((tmp_path / "reply.bin").read_bytes(), dtype=np.uint64)
    gen = np.frombuffer((tmp_path / "reply_generic.bin").read_bytes(), dtype=np.uint64)
    return rep, gen, want, out.stdout


@pytest.mark.gpu
def test_pir_api_chunked_reply_equals_oracle(pir_exe, oracle, engine, tmp_path):
    """d=1, alpha=1, ragged elements; a device budget of one poly per element, so that
    generateReplyGeneric imports and answers the database in two chunks."""
    N, m, F, L = 1024, 1, 300, 3000
    sizes = [L if i % 7 else L - 37 * (i % 5 + 1) for i in range(F)]
    budget = F * m * N * 8  # one poly per element per chunk
    rep, gen, want, line = run_case(pir_exe, oracle, tmp_path, N, m, 1, [F], sizes, 41, budget)
    assert np.array_equal(rep, want)
    assert np.array_equal(gen, want)
    assert "kept=0" in line  # several chunks: nothing kept


@pytest.mark.gpu
def test_pir_api_recursive_aggregated_equals_oracle(pir_exe, oracle, engine, tmp_path):
    """d=2 with alpha=2 and a short last group: generateReplyGeneric runs as one chunk and
    hands back the imported database."""
    N, m = 1024, 2
    sizes = [1500 - (i % 3) * 100 for i in range(101)]
    rep, gen, want, line = run_case(pir_exe, oracle, tmp_path, N, m, 2, [8, 7], sizes, 43, 1 << 30)
    assert np.array_equal(rep, want)
    assert np.array_equal(gen, want)
    assert "kept=1" in line


@pytest.mark.gpu
def test_pir_api_server_and_client_round_trip(pir_exe, ref, engine, tmp_path):
    """The reference's client builds the query (seeded key); the C++ API answers it
    (PIRReplyGenerator) and decrypts the answer with the same key (PIRReplyExtraction):
    the chosen element comes back, and the reply equals the reference's own."""
    N, m, n, alpha, F, L, chosen = 1024, 2, [7, 6], 2, 80, 900, 23
    db = np.random.default_rng(51).integers(0, 256, size=F * L, dtype=np.uint8)
    r = ref.ref_run(N, m, n, alpha, db, F, L, keyseed=77, chosen=chosen, extract=False)
    (tmp_path / "params.txt").write_text(f"LWE:80:{N}:{60 * m} {alpha} {len(n)} {' '.join(map(str, n))} {1 << 30}\n")
    (tmp_path / "sizes.bin").write_bytes(np.full(F, L, dtype=np.uint64).tobytes())
    (tmp_path / "db.bin").write_bytes(db.tobytes())
    (tmp_path / "query.bin").write_bytes(r["query"].tobytes())
    (tmp_path / "key.bin").write_bytes(ref.ref_key(N, m, 77).tobytes())
    out = subprocess.run([str(pir_exe), "run", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert np.array_equal(np.frombuffer((tmp_path / "reply.bin").read_bytes(), dtype=np.uint64), r["reply"])
    plain = np.frombuffer((tmp_path / "plain.bin").read_bytes(), dtype=np.uint8)
    assert np.array_equal(plain[:alpha * L], db[chosen * alpha * L:(chosen + 1) * alpha * L])
