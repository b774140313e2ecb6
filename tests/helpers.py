"""Shared helpers for the parity tests: seeded inputs and the two ways to compute a reply."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_cases() -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz")
    out = {k: z[k] for k in z.files if k != "meta"}
    out["meta"] = json.loads(str(z["meta"]))
    return out


def random_db(seed: int, nb: int, L: int) -> np.ndarray:
    return np.random.default_rng(seed).integers(0, 256, size=nb * L, dtype=np.uint8)


def random_query(seed: int, n: list[int], N: int, m: int, moduli: list[int], reduced: bool = True) -> np.ndarray:
    """sum(n) ciphertexts of uniform words, reduced mod p per modulus (as XPIR's enc
    leaves them) or, with reduced=False, arbitrary 64-bit words."""
    rng = np.random.default_rng(seed)
    q = rng.integers(0, 2**64, size=(sum(n), 2, m, N), dtype=np.uint64)
    if reduced:
        for c in range(m):
            q[:, :, c, :] %= np.uint64(moduli[c])
    return q.reshape(-1)


def shapes(N: int, m: int, n: list[int], alpha: int, L: int, oracle) -> tuple[int, int]:
    """(bits per coefficient, polys per element) as the reference sizes them."""
    b = oracle.bits_per_coeff(N, m, n[0])
    P = oracle.polys_for_bits(8 * alpha * L, b, N)
    return b, P
