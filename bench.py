#!/usr/bin/env python
"""Benchmark of the B200 reply engine on XPIR's NFLLWE reply path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one reply generation for one query against a database already imported into
HBM.  The default workload is the memory-bound single-query configuration: N=2048, two
60-bit moduli ("LWE:80:2048:120"), d=1, alpha=1, 100,000 elements of 4 KB (imported:
3.28 GB; one query: 100,000 ciphertexts = 6.55 GB).

Reported (one JSON line on rank 0):
  value      DB GB/s = imported-DB bytes streamed per step / reply time, with the query
             resident in HBM; whole job = sum over ranks / max time over ranks.
  e2e        the same metric through the C ABI with host buffers: the query copied from
             pinned host memory and the reply copied back inside every timed step.
  roofline   the reply kernel's algorithmic bytes (DB + query + reply) per launch over
             its CUDA-event duration, against the measured HBM copy bandwidth.
  cpu_baseline  the XPIR reference itself (oracle/_ref, compiled unchanged) on a bounded
             sample of the same workload on this host's cores.
Inputs are larger than L2 (9.8 GB per step vs 126 MB), so no L2 flush is needed.
With --gpus N every rank runs an independent replica (its own database and query):
the reply of one query has no cross-GPU exchange.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "reply-gen DB GB/s vs HBM peak; batched vs plain queries/s; p50/p99 latency"

# dram__bytes_read.sum + dram__bytes_write.sum over the algorithmic bytes (DB + query +
# replies) of one first-level reply_tma_kernel launch, per workload, each from one
# `ncu --set full` capture of a smaller case of the same kernel and tile (traffic grows
# with the elements: each is one DB row and its share of the query):
#   memory_bound: 10,000 elements, (995.5 + 3.7) MB / 983.1 MB;
#   recursive:    262,144 elements (16 groups), (1,823 + 6.7) MB / (1,811.9 + 3.1) MB;
#   plain:        the full workload (L2 flushed before the launch), (73.8 + 1.7) MB / 73.8 MB.
REPLY_TRAFFIC_PER_ALGORITHMIC_BYTE = {"memory_bound": 1.0164, "recursive": 1.0081, "plain": 1.0219}

WORKLOADS = {
    # name: N, m, n levels, alpha, elements, element bytes, chosen index, cpu-sample elements
    "memory_bound": dict(N=2048, m=2, n=[100000], alpha=1, F=100000, L=4096, chosen=54321, sample=100000,
                         desc="memory-bound single query: LWE:80:2048:120, d=1, alpha=1, 100000 x 4 KB"),
    "plain": dict(N=1024, m=1, n=[1000], alpha=1, F=1000, L=12288, chosen=137, sample=1000,
                  desc="plain single query: LWE:80:1024:60, d=1, alpha=1, 1000 x 12 KB"),
    "recursive": dict(N=4096, m=3, n=[1024, 1024], alpha=16, F=1048576, L=256, chosen=5, sample=262144,
                      desc="recursive: LWE:80:4096:180, d=2, 1024x1024 grid, alpha=16, 1048576 x 256 B"),
    # 64 queries of uneven form against one 65,536 x 8 KB database (three imports, one per
    # query shape): 32 d=1/alpha=1, 16 d=1/alpha=4, 16 d=2 on a 256x256 grid.
    "batched": dict(N=2048, m=2, F=65536, L=8192, sample=8192,
                    classes=[(32, [65536], 1), (16, [16384], 4), (16, [256, 256], 1)],
                    desc="batched: LWE:80:2048:120, 65536 x 8 KB, 64 queries (32 d1/a1, 16 d1/a4, 16 d2 256x256)"),
    # Client-side query generation on the GPU: the memory-bound workload's query (100,000
    # ciphertexts, 6.55 GB) for element 54,321, PIRQueryGenerator with the reference's PRNG.
    "querygen": dict(N=2048, m=2, n=[100000], chosen=54321, sample=100000,
                     desc="query generation: LWE:80:2048:120, d=1, 100000 ciphertexts (6.55 GB) for element 54321"),
    # Client-side extraction on the GPU: the replies to a d=1 query for one 50 MB element
    # on the memory-bound parameter set (4,763 reply ciphertexts, 312 MB).
    "extract": dict(N=2048, m=2, n=[100000], L=50_000_000,
                    desc="extraction: LWE:80:2048:120, d=1, one 50 MB element (n0=100000)"),
    # Serving loop over three resident databases, one lane (context) each.  mix: (database,
    # d, alpha, weight) of the admitted shapes; grids from the client optimizer's rule.
    "serving": dict(dbs=[("DB1", 1024, 1, 200000, 2048), ("DB2", 2048, 2, 100000, 8192),
                         ("DB3", 4096, 3, 1 << 20, 256)],
                    mix=[(0, 2, 1, 20), (0, 2, 4, 20), (0, 2, 16, 20), (0, 1, 16, 4),
                         (1, 2, 1, 20), (1, 2, 4, 20), (1, 2, 16, 20), (1, 1, 16, 4),
                         (2, 2, 16, 20), (2, 2, 4, 8), (2, 1, 16, 1)],
                    not_admitted="not in the mix: DB3 alpha=1 (103 GB imported: beyond HBM beside the other "
                                 "databases; a d=1 query is 206 GB) and d=1 at alpha<16 (3.3-51.5 GB queries, "
                                 "0.06-0.94 s of PCIe each)",
                    rates=[10, 100, 500, 2000], seconds=4.0, min_queries=40, max_queries=600,
                    budget=96 << 30, max_batch=16, sample_div=20,
                    desc="serving: DB1 LWE:80:1024:60 200000 x 2 KB, DB2 LWE:80:2048:120 100000 x 8 KB, "
                         "DB3 LWE:80:4096:180 1048576 x 256 B; Poisson arrivals; mixed d in {1,2}, "
                         "alpha in {1,4,16}"),
}


for _name, _w in WORKLOADS.items():
    _w["name"] = _name


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every 20 ms through NVML during
    the timed region (read-only queries; no GPU setting is changed)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device: int, interval_s: float = 0.02):
        self.device, self.interval = device, interval_s
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def _run(self, nvml, handle):
        while not self._stop.is_set():
            try:
                mhz = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                reasons = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                self.samples.append((float(mhz), int(reasons)))
            except Exception:
                pass
            self._stop.wait(self.interval)

    def __enter__(self):
        import threading

        try:
            import pynvml as nvml

            nvml.nvmlInit()
            # NVML enumerates all GPUs; map the CUDA ordinal through the visible-device list.
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.device]) if vis and vis.split(",")[0].isdigit() else self.device
            handle = nvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = float(nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM))
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._run, args=(nvml, handle), daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"], "samples": 0}
        mhz = [s[0] for s in self.samples]
        seen = 0
        for _, r in self.samples:
            seen |= r
        reasons = sorted(name for name, bit in self.REASONS.items() if seen & bit)
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(dist, values: list[float], device: str) -> list[float]:
    """The slowest rank's times: every rank passes its own and gets the maxima (one
    collective, taken by every rank in the same order). Without a process group, the
    values themselves."""
    if dist is None:
        return list(values)
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def synthetic_db(seed: int, F: int, L: int) -> np.ndarray:
    return np.random.default_rng(seed).integers(0, 256, size=F * L, dtype=np.uint8)


def synthetic_query(seed: int, n: list[int], N: int, m: int, moduli: list[int], out: np.ndarray) -> None:
    """Uniform words reduced mod p per modulus, the shape and value range of a query
    produced by XPIR's PIRQueryGenerator (crypto/NFLLWE.cpp:354-357)."""
    rng = np.random.default_rng(seed)
    q = out.reshape(sum(n), 2, m, N)
    for c in range(m):
        q[:, :, c, :] = rng.integers(0, moduli[c], size=(sum(n), 2, N), dtype=np.uint64)


def run_reference(w: dict, steps: int, warmup: int, threads: int) -> dict:
    """The XPIR reference (oracle/_ref) answering `steps` queries after `warmup` untimed
    ones, on one import of the workload: the full workload, except where the reference's
    host memory for the index grid rules it out (the recursive workload: its zero-padding
    slots take about 103 GB), where it takes `sample` elements on the same grid.  The
    reference pads the grid with zero polys (PIRReplyGeneratorNFL_internal.cpp:146-154) and
    its reply loop multiplies every slot, padding included (:540-560), so on the same grid
    its reply does the same work whatever the share of real elements: the sample's reply
    time stands for the full workload's, unscaled.  (Zero slots may run a little faster
    than real ones, which makes this estimate of the reference's time a lower bound.)"""
    from oracle import pyoracle as po

    if not po.ref_available():
        return {"unavailable": "reference checker oracle/_ref/xpir_ref was not built"}
    S = min(w["sample"], w["F"])
    n = list(w["n"])
    if len(n) == 1:
        n = [-(-S // w["alpha"])]
    db = synthetic_db(1, S, w["L"])
    chosen = w["chosen"] // w["alpha"] if w["chosen"] < S else 0
    r = po.ref_bench(w["N"], w["m"], n, w["alpha"], db, S, w["L"], keyseed=1000, chosen=chosen, reps=steps,
                     warmup=warmup, threads=threads)
    imported = r["nb_elements"] * r["polys_per_element"] * w["m"] * w["N"] * 8
    reply_s = statistics.mean(r["reply_s"])
    full_imported = imported * w["F"] / S
    # d = 1: the sample's grid is the sample (time scales with it); d > 1: the same grid.
    full_reply_s = reply_s * w["F"] / S if len(n) == 1 else reply_s
    return {"value": full_imported / full_reply_s / 1e9, "reply_s": reply_s, "full_reply_s": full_reply_s,
            "reply_s_all": r["reply_s"], "import_s": r["import_s"], "import_gbs": imported / r["import_s"] / 1e9,
            "imported_bytes": imported, "elements": S, "same_config": S == w["F"], "n": n,
            "threads": r["omp_threads"], "bits_per_coeff": r["bits_per_coeff"],
            "polys_per_element": r["polys_per_element"], "cpu_model": po.host_cpu_model()}


def sample_words(r: dict, w: dict) -> str:
    if len(w["n"]) > 1:
        return (f"{r['elements']} of {w['F']} elements on the full {'x'.join(map(str, w['n']))} grid (reply time "
                f"unscaled: the reference multiplies every grid slot, zero padding included)")
    return f"{r['elements']} of {w['F']} elements (reply time scaled by {w['F']}/{r['elements']})"


def reference_arm(args, w: dict, world: int, rank: int) -> int:
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    r = run_reference(w, args.steps, args.warmup, threads)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return 0
    sample = (f"{'the full workload' if r['same_config'] else sample_words(r, w)} "
              f"(n={r['n']}, bits/coeff {r['bits_per_coeff']}): one import, {args.steps} timed replies after "
              f"{args.warmup} untimed, each timed with omp_get_wtime at the reference's own boundaries")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(r["value"], 4), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["full_reply_s"] * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: seeded uniform DB bytes; query from the reference's own PIRQueryGenerator",
        "config": {"workload": w["desc"], "elements_timed": r["elements"], "same_config": r["same_config"]},
        "cpu_baseline": {"value": round(r["value"], 4), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "cpu_model": r["cpu_model"], "sample": sample},
        "e2e": {"value": round(r["value"], 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "import": {"seconds": round(r["import_s"], 4), "gbs": round(r["import_gbs"], 4)},
        "reply_s": [round(x, 4) for x in r["reply_s_all"]],
        "note": "the reference reply loop is OpenMP-parallel only over the polys of an element "
                "(PIRReplyGeneratorNFL_internal.cpp:531-534); with 1 poly per element it runs on one thread",
    }
    print(json.dumps(line))
    return 0


def ours_arm(args, w: dict, world: int, rank: int, local: int) -> int:
    import torch

    dist = init_dist(world, local)
    line = measure_single(args, w, world, rank, local, dist)
    torch.cuda.empty_cache()
    # The rest of the metric, on the same GPU after the single query's buffers are freed:
    # batched vs plain queries/s (every rank, as replicas), the serving loop's p50/p99
    # latency (one GPU: a server answers on the GPU it runs on), and the reference's other
    # two single-query configurations (plain and recursive) as replicas.
    if args.extras and args.workload == "memory_bound" and not args.elements:
        b = measure_batched(args, WORKLOADS["batched"], world, rank, local, dist)
        if rank == 0:
            line["batched"] = sub_object(b)
        if world == 1:
            # One GPU, no collective: a failure here is reported in the line, beside the
            # measurements already taken, instead of ending the run.
            try:
                line["serving"] = sub_object(measure_serving(args, WORKLOADS["serving"], local))
            except Exception as exc:  # noqa: BLE001 - recorded, not hidden
                line["serving"] = {"error": f"{type(exc).__name__}: {exc}"}
                log(f"serving failed: {exc}")
        elif rank == 0:
            line["serving"] = {"skipped": "the serving loop runs on one GPU; it is measured in the N=1 run"}
        for name in ("plain", "recursive"):
            sub = measure_single(args, dict(WORKLOADS[name]), world, rank, local, dist)
            torch.cuda.empty_cache()
            if rank == 0:
                line[name] = sub_object(sub)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def measure_single(args, w: dict, world: int, rank: int, local: int, dist) -> dict | None:
    """One single-query workload: device-resident `value`, kernel roofline, e2e through the
    C ABI with host buffers, and (N = 1) the reference's CPU reply beside it.  Returns the
    result line on rank 0 (None elsewhere)."""
    import torch

    import xpir_b200

    device = local
    torch.cuda.set_device(device)
    N, m, n, alpha, F, L = w["N"], w["m"], w["n"], w["alpha"], w["F"], w["L"]
    b = xpir_b200.bits_per_coeff(N, m, n[0])
    ct_words = 2 * m * N
    nq = sum(n)

    log(f"[rank {rank}] generating {F * L / 1e9:.2f} GB database and {nq * ct_words * 8 / 1e9:.2f} GB query")
    db = synthetic_db(1 + rank, F, L)
    q_host = torch.empty(nq * ct_words, dtype=torch.int64, pin_memory=True)
    moduli = xpir_b200.moduli(m)
    synthetic_query(54321 + rank, n, N, m, moduli, q_host.numpy().view(np.uint64))

    ctx = xpir_b200.Context(N, m, device=device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    # Import (not part of a step): timed separately, from host bytes.
    t0 = time.perf_counter()
    dbh = ctx.import_db(db, F, L, alpha, b)
    import_s = time.perf_counter() - t0
    del db
    P = dbh.polys_per_element
    Pl = P
    for _ in range(len(n) - 1):
        Pl = xpir_b200.polys_per_element(Pl * ct_words * 8, 1, b, N)
    db_bytes = dbh.device_bytes
    q_dev = q_host.to(f"cuda:{device}")
    out_dev = torch.empty(Pl * ct_words, dtype=torch.int64, device=f"cuda:{device}")
    out_host = torch.empty(Pl * ct_words, dtype=torch.int64, pin_memory=True)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- value: query resident in HBM -------------------------------------------------
    # Workloads whose inputs fit in L2 (126 MB) get an L2 flush (a 512 MB write) before
    # every step, outside the step's event pair; larger ones stream past L2 anyway.
    input_bytes = db_bytes + nq * ct_words * 8
    l2_flush = input_bytes < 2 * 126 * 2**20
    flush_buf = torch.empty(512 * 2**20 // 8, dtype=torch.int64, device=f"cuda:{device}") if l2_flush else None
    for _ in range(args.warmup):
        ctx.reply(dbh, n, q_dev, out_dev)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    # The reply kernels' own CUDA-event times, recorded by the engine around each launch on
    # its stream (the roofline's kernel time; the step also holds the synchronous call's
    # host path).
    ctx.set_kernel_timing(True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for k in range(args.steps):
            if l2_flush:
                with torch.cuda.stream(stream):
                    flush_buf.fill_(k)
            evs[k][0].record(stream)
            ctx.reply(dbh, n, q_dev, out_dev)
            evs[k][1].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count - launches0
    kt = ctx.kernel_time()
    ctx.set_kernel_timing(False)
    step_ms = [a.elapsed_time(b_) for a, b_ in evs]
    # With flushes in the loop the timed work is the sum of the steps' own intervals.
    elapsed_ms = sum(step_ms) if l2_flush else t_start.elapsed_time(t_end)
    clocks = clk.summary()

    # ---- e2e: host query in, host reply out, through the C ABI -------------------------
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    ctx.reply(dbh, n, q_host, out_host)  # warm the host path once
    barrier()
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(e2e_steps):
        ctx.reply(dbh, n, q_host, out_host)
    e_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e_start.elapsed_time(e_end) / e2e_steps

    # ---- aggregate over ranks ---------------------------------------------------------
    elapsed_ms, e2e_ms = max_over_ranks(dist, [elapsed_ms, e2e_ms], f"cuda:{device}")
    total_db = db_bytes * world
    value = total_db * args.steps / (elapsed_ms / 1e3) / 1e9
    e2e_value = total_db / (e2e_ms / 1e3) / 1e9

    line = None
    if rank == 0:
        pcie = h2d_gbs(device)
        peaks = measured_peaks()
        query_bytes = nq * ct_words * 8
        reply_bytes = Pl * ct_words * 8
        # The dominant kernel is the first level's reply: it reads the whole imported
        # database and the first dimension's query once and writes one reply per group
        # that holds data (groups past the last element are not launched).
        aggregated = math.ceil(F / alpha)
        active0 = min(math.prod(n[1:]), math.ceil(aggregated / n[0]))
        algo_bytes = db_bytes + n[0] * ct_words * 8 + active0 * P * ct_words * 8
        kern_ms = kt["reply_ms"][0] / max(1, kt["reply_launches"][0])
        roofline = None
        if kt["reply_launches"][0]:
            achieved = algo_bytes / (kern_ms / 1e3) / 1e9
            # DRAM traffic cannot be read without a profiler: it is the ncu capture's
            # measured bytes per algorithmic byte of this kernel on this workload, applied
            # to this launch's algorithmic bytes.
            ratio = REPLY_TRAFFIC_PER_ALGORITHMIC_BYTE.get(w["name"])
            traffic = round(algo_bytes * ratio) if ratio else None
            roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                        "kernel": "reply_tma_kernel" + (" (level 1)" if len(n) > 1 else ""),
                        "peak_source": peaks["source"], "algorithmic_bytes_per_launch": algo_bytes,
                        "kernel_ms": round(kern_ms, 4), "kernel_launches_timed": kt["reply_launches"][0]}
            if len(n) > 1:
                roofline["later_levels_ms"] = [round(t / max(1, c), 4) for t, c in
                                               zip(kt["reply_ms"][1:len(n)], kt["reply_launches"][1:len(n)])]
                roofline["reimport_ms"] = round(kt["import_ms"] / max(1, kt["import_launches"]), 4)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            r = run_reference(w, steps=1, warmup=0, threads=os.cpu_count() or 1)
            if "unavailable" not in r:
                what = "the full workload" if r["same_config"] else sample_words(r, w)
                cpu = {"value": round(r["value"], 4), "unit": "GB/s", "cores": r["threads"], "kind": "reference",
                       "cpu_model": r["cpu_model"],
                       "sample": (f"{what} (n={r['n']}); one reference reply {r['reply_s']:.3f} s, import "
                                  f"{r['import_s']:.3f} s"),
                       "import_gbs": round(r["import_gbs"], 4)}
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform DB bytes; query words uniform mod p (PIRQueryGenerator shape)",
            "config": {"workload": w["desc"], "N": N, "moduli": m, "d": len(n), "n": n, "alpha": alpha,
                       "elements": F, "element_bytes": L, "bits_per_coeff": b, "polys_per_element": P,
                       "imported_db_bytes": db_bytes, "query_bytes": query_bytes,
                       "l2": ("L2 flushed before every step (512 MB write, outside the step timing)" if l2_flush
                              else "inputs larger than L2 (no flush needed)"),
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 3), "unit": "GB/s", "h2d_bytes_per_step": query_bytes,
                    "d2h_bytes_per_step": reply_bytes, "ms_per_step": round(e2e_ms, 3),
                    "pcie_h2d_gbs_measured": round(pcie, 2),
                    "frac_of_pcie": round((query_bytes + reply_bytes) / (e2e_ms / 1e3) / 1e9 / pcie, 4)},
            "gpu_launches": launches,
            "clocks": clocks,
            "import": {"seconds_wall": round(import_s, 4), "input_bytes": F * L, "imported_bytes": db_bytes},
            "total_gbs": round((db_bytes + nq * ct_words * 8) * world * args.steps / (elapsed_ms / 1e3) / 1e9, 2),
        }
    dbh.free()
    ctx.close()
    del q_dev, q_host, out_dev, out_host, flush_buf
    return line


def h2d_gbs(device: int, nbytes: int = 1 << 30, reps: int = 3) -> float:
    """Pinned host-to-device copy rate of this GPU's PCIe link (best of `reps` copies of
    `nbytes`, CUDA events): the bound of the end-to-end steps, which move each step's query
    across it."""
    import torch

    src = torch.empty(nbytes // 8, dtype=torch.int64, pin_memory=True)
    dst = torch.empty(nbytes // 8, dtype=torch.int64, device=f"cuda:{device}")
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return nbytes / (best / 1e3) / 1e9


def sub_object(line: dict) -> dict:
    """A workload's result line as a sub-object of the default line: without the keys
    that repeat the enclosing line's."""
    drop = {"metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype"}
    return {k: v for k, v in line.items() if k not in drop}


def init_dist(world: int, local: int):
    """The process group of a multi-GPU run (NCCL; used for barriers and the max over
    ranks only), or None on one GPU."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist


def batched_arm(args, w: dict, world: int, rank: int, local: int) -> int:
    dist = init_dist(world, local)
    line = measure_batched(args, w, world, rank, local, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def measure_batched(args, w: dict, world: int, rank: int, local: int, dist) -> dict | None:
    """64 concurrent queries of uneven shape: one batched submission (captured in a CUDA
    graph) against 64 sequential single-query replies, both with queries resident in HBM.
    value = queries/s of the batched form.  Returns the result line on rank 0."""
    import torch

    import xpir_b200

    device = local
    torch.cuda.set_device(device)
    N, m, F, L = w["N"], w["m"], w["F"], w["L"]
    ct_words = 2 * m * N
    moduli = xpir_b200.moduli(m)
    elems = synthetic_db(4 + rank, F, L)
    ctx = xpir_b200.Context(N, m, device=device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    gen = torch.Generator(device=f"cuda:{device}")
    gen.manual_seed(4000 + rank)
    items, dbs, db_bytes_read = [], {}, 0
    query_bytes = 0
    for count, n, alpha in w["classes"]:
        b = xpir_b200.bits_per_coeff(N, m, n[0])
        key = (alpha, b)
        if key not in dbs:
            dbs[key] = ctx.import_db(elems, F, L, alpha, b)
        db = dbs[key]
        Pl = db.polys_per_element
        for _ in range(len(n) - 1):
            Pl = xpir_b200.polys_per_element(Pl * ct_words * 8, 1, b, N)
        for _ in range(count):
            q = torch.empty((sum(n), 2, m, N), dtype=torch.int64, device=f"cuda:{device}")
            for c in range(m):  # uniform words mod p, the range of XPIR's PIRQueryGenerator output
                q[:, :, c, :].random_(0, moduli[c], generator=gen)
            out = torch.empty(Pl * ct_words, dtype=torch.int64, device=f"cuda:{device}")
            items.append((db, n, q.view(-1), out))
            query_bytes += q.numel() * 8
            db_bytes_read += db.device_bytes
    del elems
    nq = len(items)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # batched: first call captures the graph, then replays
    for _ in range(max(1, args.warmup)):
        ctx.reply_batch(items, use_graph=True)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    barrier()
    with ClockSampler(device) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.reply_batch(items, use_graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    batched_ms = e0.elapsed_time(e1) / args.steps
    launches = ctx.launch_count - launches0
    clocks = clk.summary()
    # plain: the same 64 queries one after another through the single-query call
    # warm-up: one query of every shape (workspaces, first kernel loads)
    seen = set()
    for db, n, q, out in items:
        if (id(db), tuple(n)) not in seen:
            seen.add((id(db), tuple(n)))
            ctx.reply(db, n, q, out)
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for db, n, q, out in items:
        ctx.reply(db, n, q, out)
    p1.record(stream)
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    batched_ms, plain_ms = max_over_ranks(dist, [batched_ms, plain_ms], f"cuda:{device}")
    value = world * nq / (batched_ms / 1e3)
    plain_qps = world * nq / (plain_ms / 1e3)
    if rank == 0:
        peaks = measured_peaks()
        # Bytes a batch must move at least: every query once, every database once.
        batch_bytes = query_bytes + sum(d.device_bytes for d in dbs.values())
        achieved = batch_bytes / (batched_ms / 1e3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            r = reference_batch_rate(w, os.cpu_count() or 1)
            if "unavailable" not in r:
                cpu = {"value": round(r["qps"], 4), "unit": "queries/s", "cores": r["threads"], "kind": "reference",
                       "cpu_model": r["cpu_model"],
                       "sample": "one query of each class on the full database, the batch's time = the classes' "
                                 "counts x their reply times (the reference answers one query at a time)",
                       "per_class": r["per_class"]}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(batched_ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform DB bytes; query words uniform mod p generated on the device",
            "config": {"workload": w["desc"], "N": N, "moduli": m, "elements": F, "element_bytes": L,
                       "queries": nq, "query_bytes": query_bytes,
                       "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
            "plain_queries_per_s": round(plain_qps, 2), "plain_ms_for_batch": round(plain_ms, 3),
            "batched_over_plain": round(value / plain_qps, 3),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                         "kernel": "reply_tma_tasks_kernel (whole batch)", "peak_source": peaks["source"],
                         "algorithmic_bytes_per_launch": batch_bytes, "kernel_ms": round(batched_ms, 4)},
            "cpu_baseline": cpu,
            "e2e": None,
            "e2e_note": "queries are generated in HBM for this workload (155 GB); the end-to-end host path is "
                        "measured on the single-query workloads",
            "gpu_launches": launches, "clocks": clocks,
        }
    else:
        line = None
    items.clear()
    for d in dbs.values():
        d.free()
    ctx.close()
    torch.cuda.empty_cache()
    return line


def querygen_arm(args, w: dict, world: int, rank: int, local: int) -> int:
    """Client-side query generation (xpir_b200_generate_query) into HBM, one query of
    sum(n) ciphertexts per step; value = ciphertexts/s.  Replicas on N GPUs."""
    import torch

    import xpir_b200
    from oracle import pyoracle as po

    dist = init_dist(world, local)
    torch.cuda.set_device(local)
    N, m, n = w["N"], w["m"], w["n"]
    b = xpir_b200.bits_per_coeff(N, m, n[0])
    ctx = xpir_b200.Context(N, m, device=local)
    key = po.seeded_prng_key(7 + rank)
    sk = ctx.generate_secret_key(key, 0)
    out = torch.empty(sum(n) * 2 * m * N, dtype=torch.int64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    for _ in range(args.warmup):
        ctx.generate_query(key, 1, sk, n, w["chosen"], b, out=out)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.generate_query(key, 1, sk, n, w["chosen"], b, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    (ms,) = max_over_ranks(dist, [ms], f"cuda:{local}")
    count = sum(n)
    if rank == 0:
        peaks = measured_peaks()
        out_bytes = count * 2 * m * N * 8
        achieved = out_bytes / (ms / 1e3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu_baseline and po.ref_available():
            r = po.ref_querygen(N, m, n, w["chosen"], keyseed=7, threads=os.cpu_count() or 1)
            cpu = {"value": round(count / r["query_s"], 2), "unit": "ciphertexts/s", "cores": r["omp_threads"],
                   "kind": "reference", "cpu_model": po.host_cpu_model(),
                   "sample": f"the full query ({count} ciphertexts) by the reference's PIRQueryGenerator, "
                             f"{r['query_s']:.2f} s"}
        line = {
            "metric": METRIC, "value": round(world * count / (ms / 1e3), 1), "unit": "ciphertexts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded PRNG key; the secret key and noise from the reference's Salsa20 stream",
            "config": {"workload": w["desc"], "N": N, "moduli": m, "n": n, "bits_per_coeff": b,
                       "l2": "output larger than L2 (no flush needed)",
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                         "kernel": "encrypt_kernel (query written once)", "peak_source": peaks["source"],
                         "algorithmic_bytes_per_launch": out_bytes, "kernel_ms": round(ms, 4)},
            "cpu_baseline": cpu, "e2e": None,
            "gpu_launches": ctx.launch_count - launches0, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def extract_replies(w: dict, moduli: list[int], seed: int):
    """Synthetic replies of the extraction workload on the device: words in [0, 2p) per
    modulus (the range of the reply chain's lazily reduced output)."""
    import torch

    from xpir_b200 import extract_count, bits_per_coeff

    N, m = w["N"], w["m"]
    b = bits_per_coeff(N, m, w["n"][0])
    nct = extract_count(w["L"], len(w["n"]), b, N, m)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    r = torch.empty((nct, 2, m, N), dtype=torch.int64, device="cuda")
    for c in range(m):
        r[:, :, c, :].random_(0, 2 * moduli[c], generator=gen)
    return r, b, nct


def extract_arm(args, w: dict, world: int, rank: int, local: int) -> int:
    """Client-side extraction (xpir_b200_extract) of one element's d=1 replies, device
    resident (value) and from pinned host memory to host memory (e2e); ciphertexts/s."""
    import torch

    import xpir_b200
    from oracle import pyoracle as po

    dist = init_dist(world, local)
    torch.cuda.set_device(local)
    N, m, L = w["N"], w["m"], w["L"]
    moduli = xpir_b200.moduli(m)
    ctx = xpir_b200.Context(N, m, device=local)
    sk = ctx.generate_secret_key(po.seeded_prng_key(11 + rank), 0)
    dct, b, nct = extract_replies(w, moduli, 77 + rank)
    dout = torch.empty(L, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    for _ in range(args.warmup):
        ctx.extract(sk, 1, b, L, dct, dout)
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.extract(sk, 1, b, L, dct, dout)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = ctx.launch_count - launches0
    # e2e: replies from pinned host memory, the element back to host memory
    host_ct = torch.empty(dct.numel(), dtype=torch.int64, pin_memory=True)
    host_ct.copy_(dct.view(-1))
    host_out = torch.empty(L, dtype=torch.uint8, pin_memory=True)
    hct, hout = host_ct.numpy().view(np.uint64), host_out.numpy()
    ctx.extract(sk, 1, b, L, hct, hout)
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    e0.record(stream)
    for _ in range(e2e_steps):
        ctx.extract(sk, 1, b, L, hct, hout)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms], f"cuda:{local}")
    if rank == 0:
        peaks = measured_peaks()
        ct_bytes = 2 * m * N * 8
        algo = nct * ct_bytes + L
        achieved = algo / (ms / 1e3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu_baseline and po.ref_available():
            r = po.ref_extract_bench(N, m, w["n"], 1, L, 1000, host_ct.numpy().view(np.uint64),
                                     threads=os.cpu_count() or 1)
            cpu = {"value": round(nct / r["extract_s"], 2), "unit": "ciphertexts/s", "cores": r["omp_threads"],
                   "kind": "reference", "cpu_model": po.host_cpu_model(),
                   "sample": f"the same {nct} replies through the reference's PIRReplyExtraction::extractReply "
                             f"(its own seeded key), {r['extract_s']:.3f} s"}
        line = {
            "metric": METRIC, "value": round(world * nct / (ms / 1e3), 1), "unit": "ciphertexts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded reply words in [0, 2p); the secret key from the reference's Salsa20 stream",
            "config": {"workload": w["desc"], "N": N, "moduli": m, "n": w["n"], "bits_per_coeff": b,
                       "element_bytes": L, "reply_ciphertexts": nct,
                       "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                         "kernel": "decrypt_poly_kernel + lift_pack_kernel (replies read once, element written once)",
                         "peak_source": peaks["source"], "algorithmic_bytes_per_launch": algo,
                         "kernel_ms": round(ms, 4)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(world * nct / (e2e_ms / 1e3), 1), "unit": "ciphertexts/s",
                    "h2d_bytes_per_step": nct * ct_bytes, "d2h_bytes_per_step": L, "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def reference_batch_rate(w: dict, threads: int) -> dict:
    """The reference answering the batch's queries one at a time on the full database: one
    query of each class timed (xpir_ref bench, one repetition); the batch takes the sum of
    the classes' counts times their reply times."""
    from oracle import pyoracle as po

    if not po.ref_available():
        return {"unavailable": "reference checker oracle/_ref/xpir_ref was not built"}
    db = synthetic_db(4, w["F"], w["L"])
    per, total, nq, threads_used = [], 0.0, 0, threads
    for k, (count, n, alpha) in enumerate(w["classes"]):
        r = po.ref_bench(w["N"], w["m"], n, alpha, db, w["F"], w["L"], keyseed=3000 + k, chosen=0, reps=1,
                         threads=threads)
        t = r["reply_s"][0]
        per.append({"class": f"{count} x d={len(n)} alpha={alpha} n={n}", "reply_s": round(t, 4),
                    "import_s": round(r["import_s"], 3)})
        total += count * t
        nq += count
        threads_used = r["omp_threads"]
    return {"qps": nq / total, "batch_s": total, "per_class": per, "threads": threads_used,
            "cpu_model": po.host_cpu_model()}


def reference_batched_arm(args, w: dict, world: int, rank: int) -> int:
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    r = reference_batch_rate(w, threads)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return 0
    qps = r["qps"]
    line = {"impl": "reference", "metric": METRIC, "value": round(qps, 4), "unit": "queries/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": round(r["batch_s"] * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform DB bytes; query from the reference's own PIRQueryGenerator",
            "config": {"workload": w["desc"]},
            "cpu_baseline": {"value": round(qps, 4), "unit": "queries/s", "cores": r["threads"], "kind": "reference",
                             "cpu_model": r["cpu_model"],
                             "sample": "one query of each class on the full database, scaled by the class counts",
                             "per_class": r["per_class"]},
            "e2e": {"value": round(qps, 4), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def dim_sizes(n: int, alpha: int, d: int) -> list[int]:
    """Grid of a d-dimensional query over n elements aggregated by alpha: the client
    optimizer's rule (apps/optim/PIROptimizer.cpp:338-365), d equal sides of
    floor((n/alpha)^(1/d)), incremented one by one until their product covers n/alpha."""
    new_n = -(-n // alpha)
    f = [math.floor(new_n ** (1.0 / d))] * d
    if f[0] != new_n ** (1.0 / d):
        prod, j = 1, 0
        while prod < new_n and j < d:
            f[j] += 1
            j += 1
            prod = math.prod(f)
    return f


def serving_shapes(w: dict) -> list[dict]:
    import xpir_b200

    shapes = []
    for k, (db, d, alpha, weight) in enumerate(w["mix"]):
        name, N, m, F, L = w["dbs"][db]
        n = dim_sizes(F, alpha, d)
        b = xpir_b200.bits_per_coeff(N, m, n[0])
        ct = xpir_b200.ciphertext_bytes(N, m)
        shapes.append(dict(id=k, db=db, name=f"{name} d{d} a{alpha}", N=N, m=m, F=F, L=L, d=d, alpha=alpha, n=n,
                           b=b, weight=weight, query_bytes=sum(n) * ct,
                           reply_bytes=xpir_b200.reply_count(L, alpha, d, b, N, m) * ct))
    return shapes


def reference_mix(w: dict, threads: int) -> dict:
    """The reference, one query at a time, on a 1/sample_div sample of every admitted
    shape (the grid recomputed for the sample), each reply time scaled to the full
    database; the mix's queries/s weights the shapes as the arrivals do."""
    from oracle import pyoracle as po

    if not po.ref_available():
        return {"unavailable": "reference checker oracle/_ref/xpir_ref was not built"}
    per, tot_w, tot_s = [], 0.0, 0.0
    for sh in serving_shapes(w):
        S = max(sh["alpha"] * 64, sh["F"] // w["sample_div"])
        n = dim_sizes(S, sh["alpha"], sh["d"])
        db = synthetic_db(11 + sh["db"], S, sh["L"])
        r = po.ref_run(sh["N"], sh["m"], n, sh["alpha"], db, S, sh["L"], keyseed=2000 + sh["id"], chosen=0,
                       extract=False, threads=threads)
        full_s = r["reply_s"] * sh["F"] / S
        per.append({"shape": sh["name"], "elements": S, "n": n, "reply_s": round(r["reply_s"], 4),
                    "scaled_s": round(full_s, 3)})
        tot_w += sh["weight"]
        tot_s += sh["weight"] * full_s
    return {"qps": tot_w / tot_s, "per_shape": per, "threads": threads}


def serving_arm(args, w: dict, world: int, rank: int, local: int) -> int:
    if world > 1 and rank != 0:
        # Replicas only: every rank would run the same independent server; the serving
        # measurement is taken on rank 0's GPU.
        return 0
    line = measure_serving(args, w, local)
    print(json.dumps(line), flush=True)
    if not line["bit_exact"]:
        log("some served replies differ from the replies computed alone")
        return 1
    return 0


def measure_serving(args, w: dict, local: int) -> dict:
    """Poisson arrivals of mixed queries through the serving loop (xpir_b200.Server): host
    queries in, host replies out, admission by a device budget, continuous batching per
    lane.  value = completed queries/s at the highest offered rate; every reply is checked
    against the same query's reply computed alone.  Returns the result line."""
    import queue
    import threading

    import torch

    import xpir_b200

    device = local
    torch.cuda.set_device(device)
    dev = f"cuda:{device}"
    free, total = torch.cuda.mem_get_info(device)
    log(f"serving: {free / 1e9:.1f} of {total / 1e9:.1f} GB free on the device")
    shapes = serving_shapes(w)
    ctxs = [xpir_b200.Context(N, m, device=device) for (_, N, m, _, _) in w["dbs"]]
    # Imports: one per (database, alpha, bits per coefficient), from device-resident bytes.
    t0 = time.perf_counter()
    imported = {}
    for i, (name, N, m, F, L) in enumerate(w["dbs"]):
        raw = torch.from_numpy(synthetic_db(11 + i, F, L)).to(dev)
        for sh in shapes:
            key = (i, sh["alpha"], sh["b"])
            if sh["db"] == i and key not in imported:
                imported[key] = ctxs[i].import_db(raw, F, L, sh["alpha"], sh["b"])
        del raw
    torch.cuda.synchronize()
    import_s = time.perf_counter() - t0
    resident = sum(d.device_bytes for d in imported.values())
    log(f"imported {len(imported)} shapes, {resident / 1e9:.1f} GB resident, {import_s:.1f} s")
    # Query pools (pinned host memory) and each query's reply computed alone.
    gen = torch.Generator(device=dev)
    gen.manual_seed(5000)
    pools, expect = {}, {}
    for sh in shapes:
        sh["dbh"] = imported[(sh["db"], sh["alpha"], sh["b"])]
        k = max(1, min(3, int(1.5e9 // sh["query_bytes"])))
        moduli = xpir_b200.moduli(sh["m"])
        pools[sh["id"]] = []
        for j in range(k):
            q = torch.empty((sum(sh["n"]), 2, sh["m"], sh["N"]), dtype=torch.int64, device=dev)
            for c in range(sh["m"]):  # uniform words mod p, the range of XPIR's query ciphertexts
                q[:, :, c, :].random_(0, moduli[c], generator=gen)
            qh = torch.empty(q.numel(), dtype=torch.int64, pin_memory=True)
            qh.copy_(q.view(-1))
            del q
            pools[sh["id"]].append(qh)
            expect[(sh["id"], j)] = ctxs[sh["db"]].reply(sh["dbh"], sh["n"], qh)
        torch.cuda.synchronize()
    log(f"query pools: {sum(q.numel() * 8 for v in pools.values() for q in v) / 1e9:.1f} GB pinned")
    footprints = {sh["id"]: xpir_b200.Server.footprint(sh["dbh"], sh["n"]) for sh in shapes}
    srv = xpir_b200.Server(ctxs, device_budget_bytes=w["budget"], max_batch=w["max_batch"])
    weights = np.array([sh["weight"] for sh in shapes], dtype=np.float64)
    weights /= weights.sum()

    def run_rate(rate: float, count: int, seed: int) -> dict:
        rng = np.random.default_rng(seed)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
        picks = rng.choice(len(shapes), size=count, p=weights)
        which = [int(rng.integers(0, len(pools[int(s)]))) for s in picks]
        rbytes = [shapes[int(s)]["reply_bytes"] for s in picks]
        arena = torch.empty(sum(rbytes) // 8, dtype=torch.int64, pin_memory=True)
        offs = np.concatenate([[0], np.cumsum(rbytes) // 8])
        outs = [arena[offs[i]:offs[i + 1]] for i in range(count)]
        pending: "queue.Queue" = queue.Queue()
        sub_t = [0.0] * count
        err: list = []

        def submitter():
            try:
                start = time.perf_counter()
                for i in range(count):
                    delay = start + arrivals[i] - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    sh = shapes[int(picks[i])]
                    sub_t[i] = time.perf_counter()
                    pending.put((i, srv.submit(sh["dbh"], sh["n"], pools[sh["id"]][which[i]], outs[i])))
            except Exception as e:
                err.append(e)
                pending.put(None)

        l0 = sum(c.launch_count for c in ctxs)
        st0 = srv.stats()
        th = threading.Thread(target=submitter)
        th.start()
        lat, qd, done_t = [0.0] * count, [0.0] * count, [0.0] * count
        for _ in range(count):
            item = pending.get()
            if item is None:
                break
            i, t = item
            try:
                _, lat[i], qd[i] = srv.wait(t)
            except Exception as e:  # every ticket is still waited for before raising
                err.append(e)
            done_t[i] = sub_t[i] + lat[i]
        th.join()
        if err:
            raise err[0]
        st1 = srv.stats()
        bad = sum(not np.array_equal(outs[i].numpy().view(np.uint64), expect[(int(picks[i]), which[i])])
                  for i in range(count))
        span = max(done_t) - min(sub_t)
        lat_ms = np.array(lat) * 1e3
        qbytes = sum(shapes[int(s)]["query_bytes"] for s in picks)
        algo = sum(shapes[int(s)]["dbh"].device_bytes + shapes[int(s)]["query_bytes"] + shapes[int(s)]["reply_bytes"]
                   for s in picks)
        return {"offered_qps": rate, "queries": count, "achieved_qps": round(count / span, 2),
                "p50_ms": round(float(np.percentile(lat_ms, 50)), 3),
                "p99_ms": round(float(np.percentile(lat_ms, 99)), 3),
                "queued_p50_ms": round(float(np.percentile(np.array(qd) * 1e3, 50)), 3),
                "mean_batch": round((st1["completed"] - st0["completed"]) / max(1, st1["batches"] - st0["batches"]), 2),
                "mismatches": int(bad), "span_s": round(span, 3), "launches": sum(c.launch_count for c in ctxs) - l0,
                "h2d_bytes": qbytes, "d2h_bytes": sum(rbytes), "algorithmic_bytes": algo}

    # Warm-up: every shape once per pool entry (pools, kernels, workspaces).
    for _ in range(max(1, args.warmup)):
        bufs = [(sh, j, np.empty(sh["reply_bytes"] // 8, dtype=np.uint64))
                for sh in shapes for j in range(len(pools[sh["id"]]))]
        ts = [srv.submit(sh["dbh"], sh["n"], pools[sh["id"]][j], out) for sh, j, out in bufs]
        for t in ts:
            srv.wait(t)
        for sh, j, out in bufs:
            if not np.array_equal(out, expect[(sh["id"], j)]):
                raise RuntimeError(f"served reply of {sh['name']} differs from the reply computed alone")
    results = []
    # Clocks every 200 ms here (the recipe's nvidia-smi interval): polling NVML every 20 ms
    # beside the lanes' host threads cost throughput at saturation (three runs each: 2000 q/s
    # offered gave 266-364 q/s with it against 360-382 without).
    with ClockSampler(device, interval_s=0.2) as clk:
        for k, rate in enumerate(w["rates"]):
            count = int(min(w["max_queries"], max(w["min_queries"], rate * w["seconds"])))
            results.append(run_rate(rate, count, 9000 + k))
            log(f"rate {rate}: {results[-1]}")
    clocks = clk.summary()
    st = srv.stats()
    srv.close()
    mism = sum(r["mismatches"] for r in results)
    top = results[-1]
    peaks = measured_peaks()
    achieved = top["algorithmic_bytes"] / top["span_s"] / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        r = reference_mix(w, os.cpu_count() or 1)
        if "unavailable" not in r:
            cpu = {"value": round(r["qps"], 4), "unit": "queries/s", "cores": r["threads"], "kind": "reference",
                   "sample": f"one query per admitted shape on 1/{w['sample_div']} of its database, reply time "
                             f"scaled to the full database, weighted as the arrivals",
                   "per_shape": r["per_shape"]}
    line = {
        "metric": METRIC, "value": top["achieved_qps"], "unit": "queries/s", "n_gpus": 1, "steps": top["queries"],
        "warmup": args.warmup, "ms_per_step": round(1e3 / top["achieved_qps"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: seeded uniform DB bytes; query words uniform mod p, generated on the device and "
                "held in pinned host memory",
        "config": {"workload": w["desc"], "admitted_mix": [f"{sh['name']} n={sh['n']} w={sh['weight']}" for sh in shapes],
                   "not_admitted": w["not_admitted"], "device_budget_bytes": w["budget"],
                   "max_batch": w["max_batch"], "resident_db_bytes": resident, "import_s": round(import_s, 2),
                   "lanes": len(ctxs), "footprints": {sh["name"]: footprints[sh["id"]] for sh in shapes},
                   "l2": "inputs larger than L2 (no flush needed)", "parallelism": "single GPU"},
        "rates": results,
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
        "bit_exact": mism == 0,
        "server": st,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                     "kernel": "whole serving run at the highest offered rate (all lanes)",
                     "peak_source": peaks["source"],
                     "algorithmic_bytes": "per query: its imported database + query + reply"},
        "cpu_baseline": cpu,
        "e2e": {"value": top["achieved_qps"], "unit": "queries/s",
                "h2d_bytes_per_step": top["h2d_bytes"] // top["queries"],
                "d2h_bytes_per_step": top["d2h_bytes"] // top["queries"]},
        "gpu_launches": sum(r["launches"] for r in results), "clocks": clocks,
        "replies_checked": sum(r["queries"] for r in results), "mismatches": mism,
    }
    pools.clear()
    expect.clear()
    for d in imported.values():
        d.free()
    for c in ctxs:
        c.close()
    torch.cuda.empty_cache()
    return line


def reference_serving_arm(args, w: dict, world: int, rank: int) -> int:
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    r = reference_mix(w, threads)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return 0
    qps = r["qps"]
    line = {"impl": "reference", "metric": METRIC, "value": round(qps, 4), "unit": "queries/s",
            "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(1e3 / qps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform DB bytes; query from the reference's own PIRQueryGenerator",
            "config": {"workload": w["desc"]},
            "cpu_baseline": {"value": round(qps, 4), "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"one query per admitted shape on 1/{w['sample_div']} of its database, "
                                       f"scaled, weighted as the arrivals; one query at a time",
                             "per_shape": r["per_shape"]},
            "e2e": {"value": round(qps, 4), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--workload", default="memory_bound", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="default workload only: leave out the batched and serving sub-objects")
    ap.add_argument("--batch-div", type=int, default=1,
                    help="batched workload: divide the query count of every class (profiling runs)")
    ap.add_argument("--elements", type=int, default=0,
                    help="override the element count (profiling runs on a smaller case): a d=1 workload's "
                         "grid follows it, a d>1 workload keeps its grid")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    w = dict(WORKLOADS[args.workload])
    if args.workload == "serving":
        if args.impl == "reference":
            return reference_serving_arm(args, w, world, rank)
        return serving_arm(args, w, world, rank, local)
    if args.workload == "extract":
        if args.elements:
            w.update(L=args.elements, desc=w["desc"].replace("one 50 MB element", f"one {args.elements}-byte element"))
        if args.impl == "reference":
            if rank != 0:
                return 0
            from oracle import pyoracle as po
            import xpir_b200

            if not po.ref_available():
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/xpir_ref is not built "
                                  "(extraction has no port timed in the oracle)"}))
                return 0
            b = xpir_b200.bits_per_coeff(w["N"], w["m"], w["n"][0])
            nct = xpir_b200.extract_count(w["L"], 1, b, w["N"], w["m"])
            rng = np.random.default_rng(77)
            ct = np.empty((nct, 2, w["m"], w["N"]), dtype=np.uint64)
            for c, p in enumerate(xpir_b200.moduli(w["m"])):
                ct[:, :, c, :] = rng.integers(0, 2 * p, size=(nct, 2, w["N"]), dtype=np.uint64)
            r = po.ref_extract_bench(w["N"], w["m"], w["n"], 1, w["L"], 1000, ct, threads=os.cpu_count() or 1)
            v = round(nct / r["extract_s"], 2)
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "ciphertexts/s",
                              "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                              "ms_per_step": round(r["extract_s"] * 1e3, 3), "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                              "data": "seeded reply words in [0, 2p); the reference's PIRReplyExtraction",
                              "config": {"workload": w["desc"], "reply_ciphertexts": nct},
                              "cpu_baseline": {"value": v, "unit": "ciphertexts/s", "cores": r["omp_threads"],
                                               "kind": "reference", "cpu_model": po.host_cpu_model(),
                                               "sample": "the whole reply set"},
                              "e2e": {"value": v, "unit": "ciphertexts/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
            return 0
        return extract_arm(args, w, world, rank, local)
    if args.workload == "querygen":
        if args.elements:
            w.update(n=[args.elements], chosen=min(w["chosen"], args.elements - 1),
                     desc=w["desc"].replace("100000 ciphertexts (6.55 GB)", f"{args.elements} ciphertexts"))
        if args.impl == "reference":
            if rank != 0:
                return 0
            from oracle import pyoracle as po

            if not po.ref_available():
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/xpir_ref is not built "
                                  "(query generation has no port in the oracle)"}))
                return 0
            r = po.ref_querygen(w["N"], w["m"], w["n"], w["chosen"], keyseed=7, threads=os.cpu_count() or 1)
            v = round(sum(w["n"]) / r["query_s"], 2)
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "ciphertexts/s",
                              "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(r["query_s"] * 1e3, 3),
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                              "data": "seeded key; the reference's PIRQueryGenerator", "config": {"workload": w["desc"]},
                              "cpu_baseline": {"value": v, "unit": "ciphertexts/s", "cores": r["omp_threads"],
                                               "kind": "reference", "cpu_model": po.host_cpu_model(),
                                               "sample": "the full query"},
                              "e2e": {"value": v, "unit": "ciphertexts/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
            return 0
        return querygen_arm(args, w, world, rank, local)
    if args.workload == "batched":
        if args.elements or args.batch_div > 1:
            # A smaller batch of the same three classes (profiling): E elements, class
            # counts divided by batch_div, the d = 2 grid [E / 256, 256].
            E = args.elements or w["F"]
            if E % 1024:
                ap.error("--elements: the batched workload needs a multiple of 1024")
            w.update(F=E, classes=[(max(1, c // args.batch_div), n, a) for c, n, a in
                                   [(w["classes"][0][0], [E], 1), (w["classes"][1][0], [E // 4], 4),
                                    (w["classes"][2][0], [E // 256, 256], 1)]],
                     desc=f"batched (reduced): LWE:80:2048:120, {E} x 8 KB, classes d1/a1, d1/a4, d2 "
                          f"[{E // 256}, 256], counts divided by {args.batch_div}")
        if args.impl == "reference":
            return reference_batched_arm(args, w, world, rank)
        return batched_arm(args, w, world, rank, local)
    if args.elements:
        if len(w["n"]) == 1:
            w.update(n=[args.elements])
        elif args.elements > math.prod(w["n"]) * w["alpha"]:
            ap.error("--elements: more elements than the workload's grid holds")
        w.update(F=args.elements, sample=min(w["sample"], args.elements),
                 desc=w["desc"].replace(f"{WORKLOADS[args.workload]['F']} x", f"{args.elements} x"))
    if args.impl == "reference":
        return reference_arm(args, w, world, rank)
    return ours_arm(args, w, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
