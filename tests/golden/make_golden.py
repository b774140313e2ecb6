"""Regenerates the golden fixtures in this directory from the XPIR reference itself.

Each fixture is one complete PIR round trip run by the reference's own libpir code
(compiled unchanged by ``make -C oracle ref``): a seeded random database, the query
produced by the reference's PIRQueryGenerator with a seeded key, the imported database
(as a SHA-256 digest of its words) and the reply ciphertexts.  The reference has no
known-answer tests of its own, so these fixtures pin the CPU restatement and the GPU
path to the reference's outputs wherever the reference binary is not available.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import pyoracle as po  # noqa: E402

# name: (N, m, n levels, alpha, nb elements, element bytes, key seed, db seed, chosen)
CASES = {
    # d=1, P=6 polys per element (a small version of the 12 KB-element plain config)
    "d1_n1024_m1_p6": (1024, 1, [8], 1, 8, 12288, 101, 1, 5),
    # d=2 with alpha=3: a short last group (reference zero-fill behaviour) and grid padding
    "d2_n512_m2_a3": (512, 2, [4, 3], 3, 31, 200, 102, 2, 2),
    # b > 56: the CRT sub-chunk path, three moduli
    "d1_n512_m3_crt": (512, 3, [4], 1, 4, 300, 103, 3, 1),
}


def make(name: str) -> dict:
    N, m, n, alpha, F, L, keyseed, dbseed, chosen = CASES[name]
    rng = np.random.default_rng(dbseed)
    db = rng.integers(0, 256, size=F * L, dtype=np.uint8)
    r = po.ref_run(N, m, n, alpha, db, F, L, keyseed=keyseed, chosen=chosen, want_imported=True)
    meta = {
        "N": N, "m": m, "n": n, "alpha": alpha, "nb_elements": F, "element_bytes": L, "keyseed": keyseed,
        "chosen": chosen, "bits_per_coeff": r["bits_per_coeff"], "polys_per_element": r["polys_per_element"],
        "nb_aggregated": r["nb_elements"], "n_replies": r["n_replies"], "extract_ok": r["extract_ok"],
        "imported_sha256": hashlib.sha256(r["imported"].tobytes()).hexdigest(),
    }
    np.savez_compressed(HERE / f"{name}.npz", db=db, query=r["query"], reply=r["reply"],
                        plain=r.get("plain", np.zeros(0, np.uint8)), meta=json.dumps(meta))
    return meta


if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("build the reference checker first: make -C oracle ref")
    for name in CASES:
        print(name, make(name))
