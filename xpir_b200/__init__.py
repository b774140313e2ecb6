"""Python binding of the B200 reply engine's C ABI (include/xpir_b200.h).

This is plumbing for tests and benchmarks: every computation happens in the CUDA
library ``libxpir_b200.so`` built in-tree by ``xpir_b200.build``.  There is no CPU
compute path; if the library is missing or no GPU is usable, calls raise.

The class names follow XPIR's vocabulary: a :class:`Context` is one NFLLWE parameter
set ("LWE:k:N:60m") on one GPU, a :class:`Database` is an imported database resident in
HBM (XPIR's ``imported_database``), and :meth:`Context.reply` is
``PIRReplyGenerator::generateReply`` for one query.
"""
from __future__ import annotations

import ctypes
import weakref
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libxpir_b200.so"

OK = 0
ERR_ARG = -1
ERR_NOMEM = -2
ERR_CUDA = -3
ERR_NODEV = -4
ERR_STATE = -5
ERR_TIMEOUT = -6

MAX_LEVELS = 10
_lib = None


class Request(ctypes.Structure):
    """xpir_b200_request: one query of a batch (device buffers)."""

    _fields_ = [("db", ctypes.c_void_p), ("d", ctypes.c_uint32), ("n", ctypes.c_uint32 * MAX_LEVELS),
                ("query", ctypes.c_void_p), ("replies", ctypes.c_void_p), ("capacity_bytes", ctypes.c_uint64),
                ("status", ctypes.c_int), ("nb_replies", ctypes.c_uint64)]


class XpirError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = _load().xpir_b200_strerror(status).decode()
        cuda = _load().xpir_b200_last_cuda_error().decode()
        super().__init__(f"{where}: {msg} (status {status}, last CUDA error {cuda})")
        self.status = status


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m xpir_b200.build` "
                               "(the engine has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        c_u32, c_u64, c_i32, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p
        L.xpir_b200_version.restype = ctypes.c_char_p
        L.xpir_b200_strerror.restype = ctypes.c_char_p
        L.xpir_b200_strerror.argtypes = [ctypes.c_int]
        L.xpir_b200_last_cuda_error.restype = ctypes.c_char_p
        L.xpir_b200_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.xpir_b200_bits_per_coeff.restype = c_i32
        L.xpir_b200_bits_per_coeff.argtypes = [c_u32, c_u32, c_u32, c_u64]
        L.xpir_b200_polys_per_element.restype = c_u64
        L.xpir_b200_polys_per_element.argtypes = [c_u64, c_u32, c_u32, c_u32]
        L.xpir_b200_reply_count.restype = c_u64
        L.xpir_b200_reply_count.argtypes = [c_u64, c_u32, c_u32, c_u32, c_u32, c_u32]
        L.xpir_b200_ciphertext_bytes.restype = c_u64
        L.xpir_b200_ciphertext_bytes.argtypes = [c_u32, c_u32]
        L.xpir_b200_modulus.restype = c_u64
        L.xpir_b200_modulus.argtypes = [c_u32]
        L.xpir_b200_ctx_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, c_u32, c_u32]
        L.xpir_b200_ctx_destroy.argtypes = [vp]
        L.xpir_b200_ctx_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.xpir_b200_ctx_synchronize.argtypes = [vp]
        L.xpir_b200_ctx_launch_count.argtypes = [vp, ctypes.POINTER(c_u64)]
        L.xpir_b200_ctx_set_wait_test.argtypes = [vp, c_u32, ctypes.c_int32]
        L.xpir_b200_ctx_set_kernel_timing.argtypes = [vp, ctypes.c_int]
        L.xpir_b200_ctx_kernel_time.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_u64),
                                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_u64)]
        L.xpir_b200_db_import.argtypes = [vp, vp, c_u64, c_u64, c_u64, c_u32, c_u32, ctypes.c_int,
                                          ctypes.POINTER(vp)]
        L.xpir_b200_db_free.argtypes = [vp]
        L.xpir_b200_db_info.argtypes = [vp, ctypes.POINTER(c_u64), ctypes.POINTER(c_u64),
                                        ctypes.POINTER(c_u32), ctypes.POINTER(c_u64)]
        L.xpir_b200_db_export.argtypes = [vp, vp, c_u64]
        L.xpir_b200_reply.argtypes = [vp, vp, c_u32, ctypes.POINTER(c_u32), vp, ctypes.c_int, vp, c_u64,
                                      ctypes.c_int, ctypes.POINTER(c_u64)]
        L.xpir_b200_reply_batch.argtypes = [vp, ctypes.POINTER(Request), c_u32, ctypes.c_int]
        L.xpir_b200_autotune.argtypes = [vp, vp, c_u32, ctypes.POINTER(c_u32), vp, ctypes.POINTER(ctypes.c_int)]
        L.xpir_b200_set_level_tile.argtypes = [vp, c_u64, c_u32, c_u64, ctypes.c_int]
        L.xpir_b200_tile_count.argtypes = []
        L.xpir_b200_extract_count.restype = c_u64
        L.xpir_b200_extract_count.argtypes = [c_u64, c_u32, c_u32, c_u32, c_u32]
        L.xpir_b200_extract.argtypes = [vp, vp, c_u32, c_u32, c_u64, vp, c_u64, ctypes.c_int, vp, c_u64,
                                        ctypes.c_int]
        L.xpir_b200_generate_query.argtypes = [vp, vp, c_u64, vp, c_u32, ctypes.POINTER(c_u32), c_u64, c_u32,
                                                c_u32, vp, c_u64, ctypes.c_int]
        L.xpir_b200_generate_secret_key.argtypes = [vp, vp, c_u64, vp]
        L.xpir_b200_measure_costs.argtypes = [vp, c_u32, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_double)]
        L.xpir_b200_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), c_u32, c_u64, c_u32]
        L.xpir_b200_server_submit.argtypes = [vp, vp, c_u32, ctypes.POINTER(c_u32), vp, vp, c_u64,
                                              ctypes.POINTER(c_u64)]
        L.xpir_b200_server_wait.argtypes = [vp, c_u64, ctypes.c_int, ctypes.POINTER(c_u64),
                                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.xpir_b200_server_stats.argtypes = [vp, ctypes.POINTER(c_u64), ctypes.POINTER(c_u64),
                                             ctypes.POINTER(c_u64), ctypes.POINTER(c_u64)]
        L.xpir_b200_server_destroy.argtypes = [vp]
        L.xpir_b200_server_footprint.argtypes = [vp, c_u32, ctypes.POINTER(c_u32), ctypes.POINTER(c_u64)]
        _lib = L
    return _lib


def lib():
    return _load()


def _check(status: int, where: str) -> None:
    if status != OK:
        raise XpirError(status, where)


def version() -> str:
    return _load().xpir_b200_version().decode()


def device_count() -> int:
    n = ctypes.c_int(0)
    _load().xpir_b200_device_count(ctypes.byref(n))
    return n.value


def bits_per_coeff(N: int, m: int, n0: int, security_bits: int = 80) -> int:
    return int(_load().xpir_b200_bits_per_coeff(N, m, security_bits, n0))


def polys_per_element(element_bytes: int, alpha: int, b: int, N: int) -> int:
    return int(_load().xpir_b200_polys_per_element(element_bytes, alpha, b, N))


def reply_count(element_bytes: int, alpha: int, d: int, b: int, N: int, m: int) -> int:
    return int(_load().xpir_b200_reply_count(element_bytes, alpha, d, b, N, m))


def ciphertext_bytes(N: int, m: int) -> int:
    return int(_load().xpir_b200_ciphertext_bytes(N, m))


def extract_count(aggregated_bytes: int, level: int, b: int, N: int, m: int) -> int:
    """Ciphertexts decrypted at recursion level `level` (the reply count at level d)."""
    return int(_load().xpir_b200_extract_count(aggregated_bytes, level, b, N, m))


def tile_count() -> int:
    """Number of compiled reply tile shapes (indices for Context.set_level_tile)."""
    return _load().xpir_b200_tile_count()


def modulus(i: int) -> int:
    return int(_load().xpir_b200_modulus(i))


def moduli(m: int) -> list[int]:
    return [modulus(i) for i in range(m)]


def _ptr(x) -> int:
    """Address of a numpy array (host) or of anything exposing data_ptr() (device)."""
    if isinstance(x, np.ndarray):
        assert x.flags.c_contiguous
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    return int(x)


def _on_device(x) -> int:
    return 0 if isinstance(x, np.ndarray) else int(getattr(x, "is_cuda", True))


class Database:
    """An imported database resident in HBM (XPIR's imported_database)."""

    def __init__(self, ctx: "Context", handle: int):
        self.ctx = ctx
        self.handle = ctypes.c_void_p(handle)
        n = ctypes.c_uint64()
        P = ctypes.c_uint64()
        b = ctypes.c_uint32()
        nbytes = ctypes.c_uint64()
        _check(_load().xpir_b200_db_info(self.handle, ctypes.byref(n), ctypes.byref(P), ctypes.byref(b),
                                         ctypes.byref(nbytes)), "db_info")
        self.nb_aggregated, self.polys_per_element = n.value, P.value
        self.bits_per_coeff, self.device_bytes = b.value, nbytes.value

    def export(self) -> np.ndarray:
        words = self.nb_aggregated * self.polys_per_element * self.ctx.m * self.ctx.N
        out = np.empty(words, dtype=np.uint64)
        _check(_load().xpir_b200_db_export(self.handle, out.ctypes.data, words), "db_export")
        return out

    def free(self) -> None:
        # A closed context has already released its databases.
        if self.handle and self.ctx.handle:
            _check(_load().xpir_b200_db_free(self.handle), "db_free")
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """One NFLLWE parameter set (poly degree N, m 60-bit moduli) on one GPU."""

    def __init__(self, N: int, m: int, device: int = 0):
        self.N, self.m, self.device = N, m, device
        h = ctypes.c_void_p()
        _check(_load().xpir_b200_ctx_create(ctypes.byref(h), device, N, m), "ctx_create")
        self.handle = h
        self.ct_words = 2 * m * N
        self._dbs: "weakref.WeakSet[Database]" = weakref.WeakSet()
        self._servers: "weakref.WeakSet[Server]" = weakref.WeakSet()

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(_load().xpir_b200_ctx_stream(self.handle, ctypes.byref(s)), "ctx_stream")
        return s.value or 0

    def synchronize(self) -> None:
        _check(_load().xpir_b200_ctx_synchronize(self.handle), "ctx_synchronize")

    @property
    def launch_count(self) -> int:
        c = ctypes.c_uint64()
        _check(_load().xpir_b200_ctx_launch_count(self.handle, ctypes.byref(c)), "ctx_launch_count")
        return c.value

    def import_db(self, elements, nb_elements: int, element_bytes: int, alpha: int, bits_per_coeff: int,
                  element_stride: int | None = None) -> Database:
        stride = element_bytes if element_stride is None else element_stride
        h = ctypes.c_void_p()
        _check(_load().xpir_b200_db_import(self.handle, _ptr(elements), nb_elements, element_bytes, stride, alpha,
                                           bits_per_coeff, _on_device(elements), ctypes.byref(h)), "db_import")
        db = Database(self, h.value)
        self._dbs.add(db)
        return db

    def reply(self, db: Database, n: list[int], query, out=None) -> np.ndarray:
        """Reply of one query; `query` and `out` may be numpy (host) or torch CUDA tensors."""
        d = len(n)
        narr = (ctypes.c_uint32 * d)(*n)
        Pl = db.polys_per_element
        for _ in range(d - 1):
            Pl = polys_per_element(Pl * self.ct_words * 8, 1, db.bits_per_coeff, self.N)
        if out is None:
            out = np.empty(Pl * self.ct_words, dtype=np.uint64)
        cap = out.nbytes if isinstance(out, np.ndarray) else out.numel() * out.element_size()
        cnt = ctypes.c_uint64()
        _check(_load().xpir_b200_reply(self.handle, db.handle, d, narr, _ptr(query), _on_device(query), _ptr(out),
                                       cap, _on_device(out), ctypes.byref(cnt)), "reply")
        assert cnt.value == Pl
        return out

    def reply_batch(self, items, use_graph: bool = False) -> list[int]:
        """Replies to several queries in one submission.  `items` are tuples
        (database, n, query, replies) with query and replies in device memory (torch
        CUDA tensors or raw device addresses).  Returns the per-query reply counts."""
        reqs = (Request * len(items))()
        for r, (db, n, q, out) in zip(reqs, items):
            r.db = db.handle
            r.d = len(n)
            for j, v in enumerate(n):
                r.n[j] = v
            r.query = _ptr(q)
            r.replies = _ptr(out)
            r.capacity_bytes = out.numel() * out.element_size() if hasattr(out, "numel") else 2**63
        status = _load().xpir_b200_reply_batch(self.handle, reqs, len(items), int(use_graph))
        _check(status, "reply_batch")
        return [r.nb_replies for r in reqs]

    def extract(self, secret_key: np.ndarray, d: int, b: int, aggregated_bytes: int, replies, out=None):
        """Client-side extraction on the GPU: the aggregated element (aggregated_bytes) from
        d-level replies, with the secret key ([m][N] u64, NTT domain).  `replies` and `out`
        may be numpy (host) or torch CUDA tensors; returns `out` (a new uint8 array if None)."""
        sk = np.ascontiguousarray(secret_key, dtype=np.uint64)
        if out is None:
            out = np.zeros(aggregated_bytes, dtype=np.uint8)
        cap = out.nbytes if isinstance(out, np.ndarray) else out.numel() * out.element_size()
        nrep = (replies.nbytes if isinstance(replies, np.ndarray) else replies.numel() * replies.element_size())
        nrep //= 16 * self.m * self.N
        _check(_load().xpir_b200_extract(self.handle, sk.ctypes.data, d, b, aggregated_bytes, _ptr(replies), nrep,
                                         _on_device(replies), _ptr(out), cap, _on_device(out)), "extract")
        return out

    def measure_costs(self, security_bits: int = 80, target_s: float = 0.05) -> tuple[float, float]:
        """(reply, import) seconds per absorbed plaintext on this GPU, the two figures XPIR's
        optimizer caches per parameter set."""
        r, i = ctypes.c_double(), ctypes.c_double()
        _check(_load().xpir_b200_measure_costs(self.handle, security_bits, target_s, ctypes.byref(r),
                                               ctypes.byref(i)), "measure_costs")
        return r.value, i.value

    def generate_secret_key(self, prng_key: np.ndarray, nonce: int = 0) -> np.ndarray:
        """NFLLWE key generation on the GPU from the PRNG call with `nonce`."""
        key = np.ascontiguousarray(prng_key, dtype=np.uint8)
        out = np.zeros(self.m * self.N, dtype=np.uint64)
        _check(_load().xpir_b200_generate_secret_key(self.handle, key.ctypes.data, nonce, out.ctypes.data),
               "generate_secret_key")
        return out

    def generate_query(self, prng_key: np.ndarray, first_nonce: int, secret_key: np.ndarray, n: list[int],
                       chosen: int, b: int, security_bits: int = 80, out=None):
        """Client-side query generation on the GPU (PIRQueryGenerator with the reference's
        Salsa20 PRNG stream): sum(n) ciphertexts for element `chosen`."""
        key = np.ascontiguousarray(prng_key, dtype=np.uint8)
        sk = np.ascontiguousarray(secret_key, dtype=np.uint64)
        if out is None:
            out = np.zeros(sum(n) * self.ct_words, dtype=np.uint64)
        cap = out.nbytes if isinstance(out, np.ndarray) else out.numel() * out.element_size()
        narr = (ctypes.c_uint32 * len(n))(*n)
        _check(_load().xpir_b200_generate_query(self.handle, key.ctypes.data, first_nonce, sk.ctypes.data, len(n),
                                                narr, chosen, b, security_bits, _ptr(out), cap, _on_device(out)),
               "generate_query")
        return out

    def autotune(self, db: Database, n: list[int], query) -> int:
        """Times the compiled tile shapes on this query's shape and keeps the fastest."""
        narr = (ctypes.c_uint32 * len(n))(*n)
        tile = ctypes.c_int(-1)
        _check(_load().xpir_b200_autotune(self.handle, db.handle, len(n), narr, _ptr(query), ctypes.byref(tile)),
               "autotune")
        return tile.value

    def set_wait_test(self, spin_limit: int = 0, withhold_tile: int = -1) -> None:
        """Test support of the reply kernel's bounded waits (xpir_b200_ctx_set_wait_test)."""
        _check(_load().xpir_b200_ctx_set_wait_test(self.handle, spin_limit, withhold_tile), "set_wait_test")

    def set_kernel_timing(self, on: bool = True) -> None:
        """Event-timed reply and re-import launches of the following replies
        (xpir_b200_ctx_set_kernel_timing); switching on restarts the sums."""
        _check(_load().xpir_b200_ctx_set_kernel_timing(self.handle, int(on)), "set_kernel_timing")

    def kernel_time(self) -> dict:
        """The sums since set_kernel_timing(True): per recursion level the reply launches'
        milliseconds and count, and the re-imports' milliseconds and count."""
        ms = (ctypes.c_double * MAX_LEVELS)()
        cnt = (ctypes.c_uint64 * MAX_LEVELS)()
        ims, icnt = ctypes.c_double(), ctypes.c_uint64()
        _check(_load().xpir_b200_ctx_kernel_time(self.handle, ms, cnt, ctypes.byref(ims), ctypes.byref(icnt)),
               "kernel_time")
        return {"reply_ms": list(ms), "reply_launches": [int(c) for c in cnt], "import_ms": ims.value,
                "import_launches": int(icnt.value)}

    def set_level_tile(self, P: int, n_i: int, groups: int, tile: int) -> None:
        """Pins the reply kernel's tile shape for one level shape (-1: default choice)."""
        _check(_load().xpir_b200_set_level_tile(self.handle, P, n_i, groups, tile), "set_level_tile")

    def close(self) -> None:
        if self.handle:
            for srv in list(self._servers):  # a server's lanes run on the context
                srv.close()
            for db in list(self._dbs):
                db.free()
            _check(_load().xpir_b200_ctx_destroy(self.handle), "ctx_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop over one or more contexts (xpir_b200_server_*): admission by a device
    memory budget and continuous batching.  Query and reply buffers are host memory
    (numpy arrays or pinned torch tensors) that must stay alive until wait() returns."""

    def __init__(self, contexts: list[Context], device_budget_bytes: int, max_batch: int = 64):
        arr = (ctypes.c_void_p * len(contexts))(*[c.handle.value for c in contexts])
        h = ctypes.c_void_p()
        _check(_load().xpir_b200_server_create(ctypes.byref(h), arr, len(contexts), device_budget_bytes, max_batch),
               "server_create")
        self.handle = h
        self.contexts = contexts  # kept alive while the server is
        for c in contexts:
            c._servers.add(self)

    def submit(self, db: Database, n: list[int], query, replies) -> int:
        narr = (ctypes.c_uint32 * len(n))(*n)
        cap = replies.nbytes if isinstance(replies, np.ndarray) else replies.numel() * replies.element_size()
        t = ctypes.c_uint64()
        _check(_load().xpir_b200_server_submit(self.handle, db.handle, len(n), narr, _ptr(query), _ptr(replies), cap,
                                               ctypes.byref(t)), "server_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> tuple[int, float, float]:
        """Returns (reply count, latency seconds, queued seconds)."""
        cnt = ctypes.c_uint64()
        lat = ctypes.c_double()
        qd = ctypes.c_double()
        _check(_load().xpir_b200_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(cnt), ctypes.byref(lat),
                                             ctypes.byref(qd)), "server_wait")
        return cnt.value, lat.value, qd.value

    @staticmethod
    def footprint(db: Database, n: list[int]) -> int:
        """Device bytes reserved while one query of this shape is admitted."""
        narr = (ctypes.c_uint32 * len(n))(*n)
        v = ctypes.c_uint64()
        _check(_load().xpir_b200_server_footprint(db.handle, len(n), narr, ctypes.byref(v)), "server_footprint")
        return v.value

    def stats(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(4)]
        _check(_load().xpir_b200_server_stats(self.handle, *[ctypes.byref(x) for x in v]), "server_stats")
        return dict(zip(["completed", "batches", "max_batch", "peak_device_bytes"], [x.value for x in v]))

    def close(self) -> None:
        if self.handle:
            _check(_load().xpir_b200_server_destroy(self.handle), "server_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
