"""Python access to the two CPU checkers (test infrastructure only).

* ``liboracle.so`` -- the plain-C restatement of XPIR's NFLLWE reply path
  (``oracle/xpir_oracle.c``).
* ``_ref/xpir_ref`` -- the XPIR reference sources compiled unchanged, driven through
  the reference's own libpir API (``oracle/ref/xpir_ref.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU arms import this
module.  The product library (``xpir_b200``) never does.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "xpir_ref"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_lib = None


def build(reference_root: str | None = None) -> None:
    """Compile liboracle.so, and the reference checker when the XPIR source tree is given
    (``reference_root`` or the XPIR_REF environment variable) and present."""
    env = dict(os.environ, CC="gcc", CXX="g++")
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True, env=env)
    ref = reference_root or os.environ.get("XPIR_REF", "")
    if ref and Path(ref, "crypto", "NFLlib.cpp").exists():
        subprocess.run(["make", "-s", "-j8", "-C", str(HERE), "ref", "simplepir", "apps", f"XPIR_REF={ref}"], check=True,
                       env=env)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.xo_modulus.restype = ctypes.c_uint64
        L.xo_modulus.argtypes = [ctypes.c_uint32]
        L.xo_tables.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_tables_words.restype = ctypes.c_uint64
        L.xo_tables_words.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.xo_bits_per_coeff.restype = ctypes.c_uint32
        L.xo_bits_per_coeff.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
        L.xo_polys_for_bits.restype = ctypes.c_uint64
        L.xo_polys_for_bits.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.xo_bitsplit.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_ntt_phi.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.xo_intt_phi.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.xo_aggregate.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                   ctypes.c_uint64, _u8p]
        L.xo_import.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_query_primes.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_reply_level.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                     _u64p, ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_reimport.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, _u64p]
        L.xo_reply.restype = ctypes.c_uint64
        L.xo_reply.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                               ctypes.POINTER(ctypes.c_uint32), _u64p, ctypes.c_uint32, ctypes.c_uint32,
                               ctypes.c_uint32, _u64p]
        L.xo_decrypt.argtypes = [_u64p, _u64p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u8p]
        L.xo_extract_count.restype = ctypes.c_uint64
        L.xo_extract_count.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32]
        L.xo_extract.argtypes = [_u64p, ctypes.c_uint64, _u64p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint64, _u8p]
        L.xo_salsa20_stream.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint64, _u8p]
        L.xo_keygen.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_encrypt.argtypes = [_u8p, ctypes.c_uint64, _u64p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, _u64p]
        L.xo_query.argtypes = [_u8p, ctypes.c_uint64, _u64p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                               ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                               _u64p]
        L.xo_reply_count.restype = ctypes.c_uint64
        L.xo_reply_count.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.c_uint32]
        _lib = L
    return _lib


def _p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(_u64p)


def _p8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_u8p)


# ----------------------------------------------------------------------------------
# Restatement (liboracle.so)
# ----------------------------------------------------------------------------------

def modulus(i: int) -> int:
    return int(lib().xo_modulus(i))


def moduli(m: int) -> list[int]:
    return [modulus(i) for i in range(m)]


def tables(N: int, m: int) -> np.ndarray:
    out = np.zeros(int(lib().xo_tables_words(N, m)), dtype=np.uint64)
    assert lib().xo_tables(N, m, _p64(out)) == 0
    return out


def bits_per_coeff(N: int, m: int, n0: int, k: int = 80) -> int:
    return int(lib().xo_bits_per_coeff(N, m, k, n0))


def polys_for_bits(total_bits: int, b: int, N: int) -> int:
    return int(lib().xo_polys_for_bits(total_bits, b, N))


def bitsplit(bufs: np.ndarray, nbufs: int, stride: int, bits: int, b: int, N: int, m: int) -> np.ndarray:
    P = polys_for_bits(nbufs * bits, b, N)
    out = np.zeros(P * m * N, dtype=np.uint64)
    bufs = np.ascontiguousarray(bufs, dtype=np.uint8)
    assert lib().xo_bitsplit(_p8(bufs), nbufs, stride, bits, b, N, m, _p64(out)) == 0
    return out


def ntt_phi(polys: np.ndarray, N: int, m: int) -> np.ndarray:
    x = np.ascontiguousarray(polys, dtype=np.uint64).copy()
    assert lib().xo_ntt_phi(_p64(x), x.size // (m * N), N, m) == 0
    return x


def intt_phi(polys: np.ndarray, N: int, m: int) -> np.ndarray:
    x = np.ascontiguousarray(polys, dtype=np.uint64).copy()
    assert lib().xo_intt_phi(_p64(x), x.size // (m * N), N, m) == 0
    return x


def aggregate(elements: np.ndarray, nb: int, L: int, stride: int, alpha: int, s: int) -> np.ndarray:
    out = np.zeros(alpha * L, dtype=np.uint8)
    elements = np.ascontiguousarray(elements, dtype=np.uint8)
    lib().xo_aggregate(_p8(elements), nb, L, stride, alpha, s, _p8(out))
    return out


def import_db(elements: np.ndarray, nb: int, L: int, alpha: int, b: int, N: int, m: int,
              stride: int | None = None) -> np.ndarray:
    stride = L if stride is None else stride
    groups = -(-nb // alpha)
    P = polys_for_bits(8 * alpha * L, b, N)
    out = np.zeros(groups * P * m * N, dtype=np.uint64)
    elements = np.ascontiguousarray(elements, dtype=np.uint8)
    assert lib().xo_import(_p8(elements), nb, L, stride, alpha, b, N, m, _p64(out)) == 0
    return out


def query_primes(query: np.ndarray, N: int, m: int) -> np.ndarray:
    q = np.ascontiguousarray(query, dtype=np.uint64)
    out = np.zeros_like(q)
    lib().xo_query_primes(_p64(q), q.size // (2 * m * N), N, m, _p64(out))
    return out


def reply_level(db: np.ndarray, n_real: int, P: int, n_groups: int, n_i: int, query: np.ndarray,
                N: int, m: int) -> np.ndarray:
    out = np.zeros(n_groups * P * 2 * m * N, dtype=np.uint64)
    db = np.ascontiguousarray(db, dtype=np.uint64)
    q = np.ascontiguousarray(query, dtype=np.uint64)
    assert lib().xo_reply_level(_p64(db), n_real, P, n_groups, n_i, _p64(q), N, m, _p64(out)) == 0
    return out


def reimport(replies: np.ndarray, n_elts: int, P: int, b: int, N: int, m: int) -> np.ndarray:
    P2 = polys_for_bits(P * 128 * m * N, b, N)
    out = np.zeros(n_elts * P2 * m * N, dtype=np.uint64)
    r = np.ascontiguousarray(replies, dtype=np.uint64)
    assert lib().xo_reimport(_p64(r), n_elts, P, b, N, m, _p64(out)) == 0
    return out


def reply(db: np.ndarray, n_real: int, P: int, n: list[int], query: np.ndarray, b: int, N: int,
          m: int) -> np.ndarray:
    d = len(n)
    Pl = P
    for _ in range(d - 1):
        Pl = polys_for_bits(Pl * 128 * m * N, b, N)
    out = np.zeros(Pl * 2 * m * N, dtype=np.uint64)
    narr = (ctypes.c_uint32 * d)(*n)
    db = np.ascontiguousarray(db, dtype=np.uint64)
    q = np.ascontiguousarray(query, dtype=np.uint64)
    got = lib().xo_reply(_p64(db), n_real, P, d, narr, _p64(q), b, N, m, _p64(out))
    assert got == Pl, (got, Pl)
    return out


def decrypt(ct: np.ndarray, sk: np.ndarray, b: int, N: int, m: int) -> np.ndarray:
    """b*N/8 plaintext bytes of one ciphertext (NFLLWE::dec + decrypt)."""
    out = np.zeros(b * N // 8, dtype=np.uint8)
    c = np.ascontiguousarray(ct, dtype=np.uint64)
    k = np.ascontiguousarray(sk, dtype=np.uint64)
    assert lib().xo_decrypt(_p64(c), _p64(k), b, N, m, _p8(out)) == 0
    return out


def extract_count(agg_bytes: int, lvl: int, b: int, N: int, m: int) -> int:
    return int(lib().xo_extract_count(agg_bytes, lvl, b, N, m))


def extract(replies: np.ndarray, sk: np.ndarray, d: int, b: int, N: int, m: int, agg_bytes: int) -> np.ndarray:
    """The aggregated element (agg_bytes) recovered from d-level replies."""
    out = np.zeros(agg_bytes, dtype=np.uint8)
    r = np.ascontiguousarray(replies, dtype=np.uint64)
    k = np.ascontiguousarray(sk, dtype=np.uint64)
    assert lib().xo_extract(_p64(r), r.size // (2 * m * N), _p64(k), d, b, N, m, agg_bytes, _p8(out)) == 0
    return out


def seeded_prng_key(seed: int) -> np.ndarray:
    """The 32-byte Salsa20 key the reference's fastrandombytes draws from randombytes on its
    first call, when randombytes is the seeded one linked into oracle/_ref
    (oracle/ref/seeded_randombytes.cpp: splitmix64 from seed*0x2545F4914F6CDD1D + golden)."""
    mask = (1 << 64) - 1
    state = (seed * 0x2545F4914F6CDD1D + 0x9E3779B97F4A7C15) & mask
    out = bytearray()
    for _ in range(4):
        state = (state + 0x9E3779B97F4A7C15) & mask
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        out += z.to_bytes(8, "little")
    return np.frombuffer(bytes(out), dtype=np.uint8).copy()


def salsa20_stream(key: np.ndarray, nonce: int, nbytes: int) -> np.ndarray:
    out = np.zeros(nbytes, dtype=np.uint8)
    k = np.ascontiguousarray(key, dtype=np.uint8)
    lib().xo_salsa20_stream(_p8(out), nbytes, nonce, _p8(k))
    return out


def keygen(key: np.ndarray, nonce: int, N: int, m: int) -> np.ndarray:
    out = np.zeros(m * N, dtype=np.uint64)
    k = np.ascontiguousarray(key, dtype=np.uint8)
    assert lib().xo_keygen(_p8(k), nonce, N, m, _p64(out)) == 0
    return out


def query(key: np.ndarray, first_nonce: int, sk: np.ndarray, n: list[int], chosen: int, b: int, N: int, m: int,
          k: int = 80) -> np.ndarray:
    """The sum(n) query ciphertexts for `chosen` (PIRQueryGenerator)."""
    out = np.zeros(sum(n) * 2 * m * N, dtype=np.uint64)
    kk = np.ascontiguousarray(key, dtype=np.uint8)
    s = np.ascontiguousarray(sk, dtype=np.uint64)
    narr = (ctypes.c_uint32 * len(n))(*n)
    assert lib().xo_query(_p8(kk), first_nonce, _p64(s), len(n), narr, chosen, b, k, N, m, _p64(out)) == 0
    return out


def reply_count(L: int, alpha: int, d: int, b: int, N: int, m: int) -> int:
    return int(lib().xo_reply_count(L, alpha, d, b, N, m))


# ----------------------------------------------------------------------------------
# The reference itself (_ref/xpir_ref)
# ----------------------------------------------------------------------------------

def ref_available() -> bool:
    return REF_BIN.exists() and os.access(REF_BIN, os.X_OK)


def _ref(cmd: str, args: dict, threads: int | None = None) -> dict:
    argv = [str(REF_BIN), cmd]
    for k, v in args.items():
        if v is None or v is False:
            continue
        argv.append("--" + k)
        if v is not True:
            argv.append(str(v))
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    res = subprocess.run(argv, capture_output=True, text=True, env=env)
    line = res.stdout.strip().splitlines()[-1] if res.stdout.strip() else "{}"
    out = json.loads(line) if line.startswith("{") else {}
    out["returncode"] = res.returncode
    if res.returncode not in (0, 1):
        raise RuntimeError(f"xpir_ref {cmd} failed ({res.returncode}): {res.stderr[-2000:]}")
    return out


def params_str(N: int, m: int, k: int = 80) -> str:
    return f"LWE:{k}:{N}:{60 * m}"


def ref_run(N: int, m: int, n: list[int], alpha: int, db: np.ndarray, nfiles: int, L: int, keyseed: int,
            chosen: int, query: np.ndarray | None = None, want_imported: bool = False,
            extract: bool = True, threads: int | None = None) -> dict:
    """Full reference round trip.  Returns the JSON summary plus 'query', 'reply',
    optionally 'imported' and 'plain' as arrays."""
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(db, dtype=np.uint8).tofile(t / "db.bin")
        args = {"params": params_str(N, m), "alpha": alpha, "d": len(n), "n": ",".join(map(str, n)),
                "nfiles": nfiles, "eltbytes": L, "db": t / "db.bin", "keyseed": keyseed, "chosen": chosen,
                "reply-out": t / "r.bin", "skip-extract": not extract}
        if query is not None:
            np.ascontiguousarray(query, dtype=np.uint64).tofile(t / "qin.bin")
            args["query-in"] = t / "qin.bin"
        else:
            args["query-out"] = t / "q.bin"
        if want_imported:
            args["imported-out"] = t / "imp.bin"
        if extract:
            args["plain-out"] = t / "plain.bin"
        out = _ref("run", args, threads)
        out["reply"] = np.fromfile(t / "r.bin", dtype=np.uint64)
        out["query"] = query if query is not None else np.fromfile(t / "q.bin", dtype=np.uint64)
        if want_imported:
            out["imported"] = np.fromfile(t / "imp.bin", dtype=np.uint64)
        if extract and (t / "plain.bin").exists():
            out["plain"] = np.fromfile(t / "plain.bin", dtype=np.uint8)
        return out


def ref_bench(N: int, m: int, n: list[int], alpha: int, db: np.ndarray, nfiles: int, L: int, keyseed: int,
              chosen: int, reps: int, warmup: int = 0, threads: int | None = None) -> dict:
    """The reference answering repeated queries on one imported database (xpir_ref bench):
    the JSON summary with the per-repetition reply times in 'reply_s'."""
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(db, dtype=np.uint8).tofile(t / "db.bin")
        args = {"params": params_str(N, m), "alpha": alpha, "d": len(n), "n": ",".join(map(str, n)),
                "nfiles": nfiles, "eltbytes": L, "db": t / "db.bin", "keyseed": keyseed, "chosen": chosen,
                "reps": reps, "warmup": warmup}
        return _ref("bench", args, threads)


def ref_querygen(N: int, m: int, n: list[int], chosen: int, keyseed: int, threads: int | None = None) -> dict:
    """The reference's client-side query generation alone (xpir_ref querygen)."""
    args = {"params": params_str(N, m), "alpha": 1, "d": len(n), "n": ",".join(map(str, n)), "keyseed": keyseed,
            "chosen": chosen}
    return _ref("querygen", args, threads)


def host_cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the record of a CPU timing."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_extract(N: int, m: int, n: list[int], alpha: int, L: int, keyseed: int, reply: np.ndarray) -> np.ndarray:
    """Decrypt replies with the reference's PIRReplyExtraction and the seeded key."""
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(reply, dtype=np.uint64).tofile(t / "r.bin")
        _ref("extract", {"params": params_str(N, m), "alpha": alpha, "d": len(n), "n": ",".join(map(str, n)),
                         "eltbytes": L, "keyseed": keyseed, "reply-in": t / "r.bin", "plain-out": t / "p.bin"})
        return np.fromfile(t / "p.bin", dtype=np.uint8)


def ref_extract_bench(N: int, m: int, n: list[int], alpha: int, L: int, keyseed: int, reply: np.ndarray,
                      threads: int | None = None) -> dict:
    """The reference's PIRReplyExtraction::extractReply alone, timed with omp_get_wtime."""
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(reply, dtype=np.uint64).tofile(t / "r.bin")
        return _ref("extract", {"params": params_str(N, m), "alpha": alpha, "d": len(n), "n": ",".join(map(str, n)),
                                "eltbytes": L, "keyseed": keyseed, "reply-in": t / "r.bin", "plain-out": t / "p.bin"},
                    threads)


def ref_key(N: int, m: int, keyseed: int) -> np.ndarray:
    """The reference's seeded secret key, [m][N] in the NTT domain."""
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        _ref("key", {"params": params_str(N, m), "keyseed": keyseed, "key-out": t / "k.bin"})
        return np.fromfile(t / "k.bin", dtype=np.uint64)


def ref_info(N: int, m: int, n0: int) -> dict:
    return _ref("info", {"params": params_str(N, m), "n": n0})


def ref_tables(N: int, m: int) -> np.ndarray:
    with tempfile.TemporaryDirectory() as td:
        _ref("tables", {"params": params_str(N, m), "n": 1, "out": Path(td) / "t.bin"})
        return np.fromfile(Path(td) / "t.bin", dtype=np.uint64)


def ref_bitsplit(N: int, m: int, bufs: np.ndarray, nbufs: int, bits: int, b: int, stride: int,
                 ntt: bool = False) -> np.ndarray:
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(bufs, dtype=np.uint8).tofile(t / "in.bin")
        _ref("deser" if ntt else "bitsplit",
             {"params": params_str(N, m), "n": 1, "in": t / "in.bin", "nbufs": nbufs, "bufbits": bits,
              "bufstride": stride, "bits": b, "out": t / "o.bin"})
        return np.fromfile(t / "o.bin", dtype=np.uint64)


def ref_ntt(N: int, m: int, polys: np.ndarray) -> np.ndarray:
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        np.ascontiguousarray(polys, dtype=np.uint64).tofile(t / "in.bin")
        _ref("ntt", {"params": params_str(N, m), "n": 1, "in": t / "in.bin", "out": t / "o.bin"})
        return np.fromfile(t / "o.bin", dtype=np.uint64)
