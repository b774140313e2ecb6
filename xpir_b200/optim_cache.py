"""Writes XPIR's optimizer performance cache (exp/preCompute<crypto>.abs) with costs
measured on a B200 instead of the CPU, so that XPIR's client optimizer chooses the
recursion depth and aggregation for a GPU server.

    python -m xpir_b200.optim_cache --params LWE:80:2048:120,LWE:97:1024:60 --out exp/preComputeLWE.abs
    python -m xpir_b200.optim_cache --params-from exp/preComputeLWE.abs --out exp/preComputeLWE.abs

One line per parameter set, as PIROptimizer::computeOptimData writes it
(pir/replyGenerator/PIROptimizer.cpp:119-151): the parameter string, the reply seconds per
absorbed plaintext and the import seconds per plaintext, 5 significant digits.  The
parameter list comes from the command line or from the first column of an existing cache
(XPIR's own enumeration of parameter sets, which depends on its security estimator).
"""
from __future__ import annotations

import argparse
from pathlib import Path

import xpir_b200


def parse_params(param: str) -> tuple[int, int, int]:
    f = param.split(":")
    if len(f) < 4 or f[0] != "LWE" or int(f[3]) % 60:
        raise ValueError(f"not an LWE parameter set: {param}")
    return int(f[1]), int(f[2]), int(f[3]) // 60


def cache_lines(params: list[str], device: int = 0, target_s: float = 0.05) -> list[str]:
    lines = []
    for param in params:
        k, N, m = parse_params(param)
        with xpir_b200.Context(N, m, device=device) as ctx:
            reply, imp = ctx.measure_costs(k, target_s)
        lines.append(f"{param} {reply:.5g} {imp:.5g}")
    return lines


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--params", default="")
    ap.add_argument("--params-from", default="")
    ap.add_argument("--out", required=True)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--target-s", type=float, default=0.05)
    args = ap.parse_args()
    params = [p for p in args.params.split(",") if p]
    if args.params_from:
        params += [ln.split(" ")[0] for ln in Path(args.params_from).read_text().splitlines()
                   if ln.strip() and not ln.startswith("#")]
    Path(args.out).write_text("\n".join(cache_lines(params, args.device, args.target_s)) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
