"""Benchmark of the curvelet path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the whole path (spatial hash -> neighbour CSR -> pairwise
curve bundles -> chain growth, dedup, record -> compacted chains + info) over
one batch of seeded synthetic edges. Workloads:

  mixed64     64 maps of uneven size (640x480 .. 3840x2160, 8k .. 3.8M edges,
              33.7M in all) in one ragged batch (default). The same line reports
              the plain form (the 64 maps one per launch, same GPU), and a served
              run: an open-loop Poisson stream of maps drawn from the same 64
              through cvl_server_* (continuous batching, 40 GB admission budget),
              with p50/p95/p99 latency.
  plain_hd    one 1920x1080 map, ~242k edges, one map per launch
  plain_small one 480x320 map (~4.5k edges)
  served      only the served stream, at each rate of --rates
  stress      16 dense 3840x2160 maps interleaved with 1,024 small 640x480 maps,
              Poisson at 150 maps/s; small-map p99 apart
  contours    the downstream stage fused behind the path: one 1920x1080 map,
              edges -> curvelets -> edgel link graph -> contour fragments
              (cvl_run_contours), the stage's own time and roofline apart; the
              CPU baseline adds the reference's original_code link graph and
              one-chain extraction to its cpu_curvelet time

value: edges/s with the edges already in HBM (CUDA events on the engine's
stream around each step, L2 flushed between steps). e2e: the same metric
through the C ABI call a user makes (cvl_run for one map, cvl_run_maps for many:
pinned host edges in, chains and info out, copies inside the timed region). With N GPUs (torchrun) every rank
processes its own instance of the workload (replicas, weak scaling) and the
step time is the max over ranks; there is no data-path collective.

--impl reference times the reference's own cpu_curvelet code (compiled from
its sources into oracle/_ref/libcvlref.so) on this host's cores, on the same
workload, metric and unit.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges/s"
# per computed (non-close) pair: 63 cells x 20 FP64 flops, divisions counted as 1
FLOPS_PER_PAIR_CELL = 20
# DRAM bytes of k_bundles per computed pair, from one ncu capture of the kernel
# (--set full, profiles/k_bundles_k_growth_persistent_hd.md) on the 242k-edge
# 1920x1080 map: dram__bytes_read.sum 0.153864 GB + dram__bytes_write.sum 1.430769 GB
# over 2,176,780 non-close pairs. The traffic is the valid pairs' bundle writes
# (1,008 B each, about half of the computed pairs) plus the pair/anchor reads, so it
# scales with the pairs a launch processes.
BUNDLE_DRAM_BYTES_PER_PAIR = (0.153864e9 + 1.430769e9) / 2_176_780
# FP64-pipe instructions of k_bundles per cell, from the same capture: the pipe was
# active 51.553% of 1,750,328 active cycles per SM on 148 SMs (each issues 2 FP64
# warp-instructions a cycle), 30.73 active lanes per warp-instruction, 2,176,780 x 63
# cells. A division costs about 10 of them, which the algorithmic count takes as 1 flop.
BUNDLE_FP64_INSTR_PER_CELL = 0.51553 * 1_750_328 * 148 * 2 * 30.73 / (2_176_780 * 63)


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="mixed64",
                    choices=["mixed64", "plain_hd", "plain_small", "served", "stress", "contours"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the one-map-per-launch comparison")
    ap.add_argument("--no-sweep", action="store_true", help="skip the served rate sweep (20 to 400 maps/s)")
    ap.add_argument("--no-stress", action="store_true", help="skip the stress stream (dense 4K maps among small ones)")
    ap.add_argument("--no-small", action="store_true", help="skip batched vs plain on the 1,024 small maps")
    ap.add_argument("--rate", type=float, default=50.0, help="served stream: offered maps/s")
    ap.add_argument("--rates", default="20,50,100,200,400", help="served workload: rates to sweep")
    ap.add_argument("--requests", type=int, default=400, help="served stream: requests per rate")
    ap.add_argument("--workers", type=int, default=4, help="served stream: server workers")
    ap.add_argument("--large-yield-ms", type=int, default=10,
                    help="served stream: longest hold-back of a large launch between chunks (0: none)")
    ap.add_argument("--large-workers", type=int, default=0,
                    help="served stream: workers on the large-map lane (0: half of them)")
    args = ap.parse_args()
    args.rate_given = any(a == "--rate" or a.startswith("--rate=") for a in sys.argv[1:])
    return args


def _workload(name: str, rank: int):
    from curvelet_construction_on_gpu_b200 import synth
    if name == "plain_hd":
        return [synth.plain_hd(1000 + rank)], {"image": "1920x1080", "curves": 1500, "clutter": 0.2}
    if name == "contours":
        return [synth.plain_hd(1000 + rank)], {"image": "1920x1080", "curves": 1500, "clutter": 0.2,
                                               "min_group_size": 4, "gap": 1.5, "polyarcs": True}
    if name == "plain_small":
        return [synth.plain_small(0 + rank)], {"image": "480x320", "curves": 50, "clutter": 0.1}
    if name == "stress":
        maps, kinds = synth.stress_mix(5000 + 10_000 * rank)
        return maps, {"maps": len(maps), "dense": "16 x 3840x2160 (6,000 curves, half radius 3-15 px, 40% clutter)",
                      "small": "1024 x 640x480 (config-0 generator)", "_labels": kinds}
    # mixed64 and served share the pool of 64 seeded maps
    maps = synth.mixed64(2000 + 64 * rank, 64)
    images = ["%dx%d" % synth.mixed_map_image(2000 + 64 * rank + i) for i in range(64)]
    return maps, {"maps": 64, "images": "640x480..3840x2160", "clutter": 0.2, "_labels": images}


class _Clocks:
    """Samples SM clocks and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        # the nvidia-smi samples go to $CVL_BENCH_OUT (default bench_out/ beside this file)
        self.path = os.path.join(os.environ.get("CVL_BENCH_OUT", os.path.join(ROOT, "bench_out")),
                                 f"clocks_rank{index}.csv")
        self.proc = None
        self.index = index

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # a timed region shorter than the sampling interval would otherwise end before
        # the sampler's first row: wait (at most 3 s) until it has written one
        t0 = time.perf_counter()
        while self.proc is not None and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


_PINNED_KEEP = []  # the torch tensors behind the page-locked arrays handed out


def _pinned(a: np.ndarray) -> np.ndarray:
    """A page-locked copy of a (torch's pinned allocator), for the e2e copies."""
    import torch
    t = torch.empty(a.size, dtype=torch.float64).pin_memory()
    _PINNED_KEEP.append(t)
    out = t.numpy().reshape(a.shape)
    out[...] = a
    return out


def _progress(msg: str) -> None:
    print(f"[bench] {time.strftime('%H:%M:%S')} {msg}", file=sys.stderr, flush=True)


# The reference sizes its outputs as num_edges * (max_degree + 1) * 2 * 10 in
# 32-bit unsigned arithmetic (cpu_curvelet.hpp:64-67). That product wraps, and
# the info array is under-allocated, once a map is large enough: above 2^32 /
# (2 * 10 * (max_candidates + 1)) = 1,664,804 edges it can wrap at any degree.
# The CPU timings therefore run on whole maps below that size.
REF_SAFE_EDGES = (1 << 32) // (2 * 10 * (128 + 1))


def _physical_cores() -> int:
    """Physical cores of this host (distinct (package, core) pairs), not hardware threads."""
    try:
        seen, phys, core = set(), None, None
        for line in open("/proc/cpuinfo"):
            if line.startswith("physical id"):
                phys = line.split(":", 1)[1].strip()
            elif line.startswith("core id"):
                core = line.split(":", 1)[1].strip()
            elif not line.strip():
                if core is not None:
                    seen.add((phys, core))
                phys = core = None
        if core is not None:
            seen.add((phys, core))
        if seen:
            return len(seen)
    except Exception:
        pass
    return os.cpu_count() or 1


def _by_class(maps, labels):
    """Map indices per image class, each class in workload order."""
    out = {}
    for i, lab in enumerate(labels or ["all"] * len(maps)):
        out.setdefault(lab, []).append(i)
    return out


def _ref_sample(maps, max_edges: int, labels=None, max_map_edges: int | None = None):
    """Whole maps the reference can hold (below REF_SAFE_EDGES, and max_map_edges when
    given), stratified across the image classes: round robin over the classes, each in
    workload order, until max_edges."""
    classes = _by_class(maps, labels)
    queues = {k: [i for i in v if maps[i].shape[0] < REF_SAFE_EDGES and
                  (max_map_edges is None or maps[i].shape[0] <= max_map_edges)] for k, v in classes.items()}
    out, tot = [], 0
    while any(queues.values()) and tot < max_edges:
        for k in sorted(queues):
            if queues[k] and tot < max_edges:
                i = queues[k].pop(0)
                out.append(maps[i])
                tot += maps[i].shape[0]
    return out, tot


def _ref_step_sample(maps, labels):
    """The reference arm's per-step sample: the smallest map of each image class (the
    lowest densities, where the reference's cost per edge is lowest)."""
    out = []
    for k, idx in sorted(_by_class(maps, labels).items()):
        ok = [i for i in idx if maps[i].shape[0] < REF_SAFE_EDGES]
        if ok:
            out.append(maps[min(ok, key=lambda i: maps[i].shape[0])])
    return out, int(sum(m.shape[0] for m in out))


def _dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def _max_over_ranks(pg, v: float) -> float:
    from curvelet_construction_on_gpu_b200.replicas import reduce_max
    return reduce_max(pg, v)


def _sum_over_ranks(pg, v: float) -> float:
    from curvelet_construction_on_gpu_b200.replicas import reduce_sum
    return reduce_sum(pg, v)


def _barrier(pg):
    if pg is not None:
        pg.barrier()


def _cpu_baseline(maps, budget_s: float = 20.0, labels=None) -> dict:
    """The reference's own code (oracle/_ref) on this host's physical cores, on a
    bounded sample of the workload: whole maps, stratified across the image classes
    (round robin, each class in workload order), until ~budget_s of CPU work."""
    from oracle import oracle as O
    threads = _physical_cores()
    kind = "reference" if O.ref_available() else "port"
    edges = 0
    secs = 0.0
    used = 0
    phases = {"csr": 0.0, "pairwise": 0.0, "greedy": 0.0}
    cand, _ = _ref_sample(maps, 1 << 62, labels, max_map_edges=600_000)  # 600k: within the time budget
    for m in cand:
        t0 = time.perf_counter()
        if kind == "reference":
            r = O.ref_run(m, nthreads=threads, want_outputs=False)
            dt = (r.ms["csr"] + r.ms["pairwise"] + r.ms["greedy"]) / 1e3
            for k in phases:
                phases[k] += r.ms[k]
        else:
            O.run(m, nthreads=threads)
            dt = time.perf_counter() - t0
        edges += m.shape[0]
        secs += dt
        used += 1
        if secs > budget_s:
            break
    out = {"value": edges / secs, "unit": METRIC, "cores": threads, "logical_cpus": os.cpu_count(), "kind": kind,
           "cpu_model": _cpu_model(),
           "sample": f"{used} of {len(maps)} map(s) (whole maps of at most 600k edges, round robin over the "
                     f"image classes), "
                     f"{edges} edges, timed as the reference's own CSR + form_pairwise_bundles + "
                     f"build_curvelets_greedy phases (file I/O excluded)"}
    if kind == "reference":
        # the reference's three timed phases over the sample (main.cpp:43-66), and the
        # CSR + greedy subtotal
        out["phases_ms"] = dict(phases, csr_plus_greedy=phases["csr"] + phases["greedy"])
    # the same on one thread (--nthreads 1), on the first map of the sample
    if kind == "reference" and cand:
        m = min(cand, key=lambda x: abs(x.shape[0] - 60_000))
        r = O.ref_run(m, nthreads=1, want_outputs=False)
        dt = (r.ms["csr"] + r.ms["pairwise"] + r.ms["greedy"]) / 1e3
        out["single_thread"] = {"value": m.shape[0] / dt, "unit": METRIC, "cores": 1,
                                "sample": f"one map of {m.shape[0]} edges"}
    return out


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def _config(args, n_edges: int, world: int, cfg: dict) -> dict:
    """The workload's description, the same in both arms' lines."""
    return dict(workload=args.workload, edges_per_gpu=int(n_edges), parallelism=f"replicas x{world}",
                l2="inputs larger than L2 (32 B per edge); the GPU arm also flushes L2 between steps",
                **{k: v for k, v in cfg.items() if not k.startswith("_")})


# The reference arm times a bounded sample of the workload per step: the reference's
# output sizing (num_edges * (max_degree + 1) * 2 rows, 32-bit, cpu_curvelet.hpp:59-67)
# wraps above 1,664,804 edges, and its CPU time per step must stay within minutes.
SAMPLE_NOTE = ("the reference arm times a sample of the workload's maps per step (the smallest map of each image "
               "class it can hold: its 32-bit output sizing, cpu_curvelet.hpp:59-67, wraps above 1,664,804 edges); "
               "both arms report edges/s, a per-edge rate")


def run_reference(args, maps, cfg, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcvlref.so was not built "
                          "(the reference sources were absent at build time)"}))
        return
    threads = _physical_cores()
    # each step: the whole workload when it is one map, else the smallest map of each
    # image class that the reference can hold (REF_SAFE_EDGES)
    if len(maps) == 1:
        sample, tot = maps, int(maps[0].shape[0])
    else:
        sample, tot = _ref_step_sample(maps, cfg.get("_labels"))
    for _ in range(args.warmup):
        O.ref_run(sample[0], nthreads=threads, want_outputs=False)
    step_s = []
    for _ in range(args.steps):
        s = 0.0
        for m in sample:
            r = O.ref_run(m, nthreads=threads, want_outputs=False)
            s += (r.ms["csr"] + r.ms["pairwise"] + r.ms["greedy"]) / 1e3
        step_s.append(s)
    ms = 1e3 * float(np.mean(step_s))
    value = tot / (ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": _config(args, int(sum(m.shape[0] for m in maps)), world, cfg),
            "sample": {"maps": len(sample), "edges": tot, "note": SAMPLE_NOTE if len(maps) > 1 else "the whole workload"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "logical_cpus": os.cpu_count(),
                             "kind": "reference", "cpu_model": _cpu_model(),
                             "sample": f"{len(sample)} of {len(maps)} map(s), {tot} edges per step"
                                       + ("" if len(maps) == 1 else
                                          ": the smallest map of each image class the reference can hold")},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _stage_sums(times) -> dict:
    """Per-stage device ms of one run, summed over chunks."""
    out = {}
    for name, ms in times:
        out[name] = out.get(name, 0.0) + ms
    return out


def _plain_wall_ms(eng, maps, steps: int) -> float:
    """Mean wall ms per step of the plain form: one map per launch (cvl_batch_run on
    single-map batches resident in HBM), one after another, host syncs and launch
    gaps included, as a caller that runs maps one at a time sees it."""
    singles = [eng.upload_batch([m]) for m in maps]
    for b in singles[:2]:
        eng.run_batch(b).close()
    total = 0.0
    for _ in range(steps):
        eng.flush_l2()
        t0 = time.perf_counter()
        for b in singles:
            eng.run_batch(b).close()
        total += time.perf_counter() - t0
    for b in singles:
        b.close()
    return 1e3 * total / steps


def _small_maps(eng, maps, steps: int, pg) -> dict:
    """Batched against plain on a stream of small maps: the 1,024 small 640x480 maps
    of the stress mix (the config-0 generator), where the per-launch cost of the
    plain form is not hidden by the work. Resident: one ragged launch against 1,024
    sequential single-map launches, both by wall clock. e2e: cvl_run_maps against
    1,024 sequential cvl_run calls, pinned host edges in, results out."""
    n_edges = int(sum(m.shape[0] for m in maps))
    batch = eng.upload_batch(maps)
    for _ in range(2):
        eng.run_batch(batch).close()
    dev, wall = [], []
    for _ in range(steps):
        eng.flush_l2()
        t0 = time.perf_counter()
        r = eng.run_batch(batch)
        wall.append(time.perf_counter() - t0)
        dev.append(r.stats()["device_ms"])
        launches = int(r.stats()["launches"])
        r.close()
    batch.close()
    b_wall = _max_over_ranks(pg, float(np.mean(wall)))
    p_ms = _max_over_ranks(pg, _plain_wall_ms(eng, maps, steps))
    pinned = _pinned(np.concatenate(maps, axis=0))
    counts = np.array([m.shape[0] for m in maps], np.int32)
    singles = [pinned[o - c:o] for o, c in zip(np.cumsum(counts), counts)]
    held = eng.run_maps(pinned, counts=counts)
    del held
    t0 = time.perf_counter()
    for _ in range(steps):
        for res in eng.run_maps(pinned, counts=counts):
            del res
    be2e = _max_over_ranks(pg, (time.perf_counter() - t0) / steps)
    for m in singles[:4]:
        eng.run(m)
    t0 = time.perf_counter()
    for _ in range(steps):
        for m in singles:
            res = eng.run(m)
            del res
    pe2e = _max_over_ranks(pg, (time.perf_counter() - t0) / steps)
    return {"maps": len(maps), "edges": n_edges, "steps": steps,
            "batched": {"wall_ms": 1e3 * b_wall, "device_ms": float(np.mean(dev)), "launches": launches,
                        "edges_per_s": n_edges / b_wall},
            "plain": {"wall_ms": p_ms, "edges_per_s": n_edges / (p_ms / 1e3),
                      "form": "1,024 sequential cvl_batch_run calls on resident single-map batches"},
            "batched_vs_plain": p_ms / (1e3 * b_wall),
            "e2e": {"batched_ms": 1e3 * be2e, "plain_ms": 1e3 * pe2e, "batched_vs_plain": pe2e / be2e,
                    "batched_edges_per_s": n_edges / be2e, "plain_edges_per_s": n_edges / pe2e,
                    "form": "cvl_run_maps against sequential cvl_run, pinned host edges, results to host"}}


def _distinct_pool(maps, labels, copies: int, rank: int):
    """The served streams' pool: the workload's maps and copies-1 more copies of
    each, translated by whole pixels (a seeded offset per copy), so that a stream
    of a few hundred requests meets few repeated inputs. A whole-pixel translation
    moves every pixel cell with its edges, so each copy is a valid map of the
    same size class."""
    pool, labs = list(maps), list(labels)
    rng = np.random.default_rng(77 + rank)
    for _ in range(copies - 1):
        for m, lab in zip(maps, labels):
            t = m.copy()
            t[:, 0] += float(rng.integers(1, 64))
            t[:, 1] += float(rng.integers(1, 64))
            pool.append(t)
            labs.append(lab)
    return pool, labs


def _served(maps, labels, rate: float, n_req: int, workers: int, device: int, seed: int = 7,
            sequence=None, warm_all: bool = True, n_warm: int | None = None) -> dict:
    """Open-loop Poisson stream through cvl_server_*: arrivals at `rate` maps/s,
    submitted on schedule by one thread while another takes the results in
    completion order. The maps are `sequence` (indices into maps) when given,
    else n_req draws with replacement. Latency is the server's own clock from the
    submit call to the result being ready in host memory; labels[i] names map
    i's class, and each class gets its own percentiles."""
    import threading

    import curvelet_construction_on_gpu_b200 as cvl
    from curvelet_construction_on_gpu_b200 import _abi
    rng = np.random.default_rng(seed)
    picks = np.asarray(sequence) if sequence is not None else rng.integers(0, len(maps), n_req)
    n_req = len(picks)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    srv = cvl.Server(device=device, workers=workers, large_workers=_LARGE_WORKERS, large_yield_ms=_LARGE_YIELD_MS)
    try:
        # warm-up (workspace and page-locked arena growth): the largest map once per
        # worker, then every map of the pool once (or a few of each class)
        order = np.argsort([m.shape[0] for m in maps])
        warm = [srv.submit(maps[int(order[-1])]) for _ in range(workers)]
        if warm_all:
            warm += [srv.submit(m) for m in maps[:n_warm]]
        else:
            seen = {}
            for i, lab in enumerate(labels):
                if seen.get(lab, 0) < 4:
                    seen[lab] = seen.get(lab, 0) + 1
                    warm.append(srv.submit(maps[i]))
        for _ in warm:
            srv.next()
        warm_stats = srv.stats()
        ids = [None] * n_req
        t0 = time.perf_counter()

        def submitter():
            for k in range(n_req):
                dt = t0 + arrivals[k] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[k] = srv.submit(maps[int(picks[k])])

        th = threading.Thread(target=submitter)
        th.start()
        # results are taken in completion order (as each client would take its own)
        got = 0
        while got < n_req:
            try:
                r = srv.next(timeout_s=0.5)
            except cvl.CvlError as e:
                if e.code == _abi.CVL_ETIMEDOUT:
                    continue
                raise
            if r is None:  # nothing submitted yet
                time.sleep(0.0002)
                continue
            got += 1
            del r
        th.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
        ms, ed, rid = srv.latencies(with_ids=True)
        rt = srv.request_times()
        st0 = warm_stats
    finally:
        srv.close()
    label_of = {int(ids[k]): labels[int(picks[k])] for k in range(n_req)}
    keep = np.array([int(r) in label_of for r in rid], bool)
    ms, ed, rid = ms[keep], ed[keep], rid[keep]

    def pct(a, q):
        return float(np.percentile(a, q, method="inverted_cdf")) if len(a) else None

    rt = rt[np.array([int(r) in label_of for r in rt["id"]], bool)] if len(rt) else rt
    classes = {}
    for lab in sorted(set(label_of.values())):
        sel = np.array([label_of[int(r)] == lab for r in rid], bool)
        classes[lab] = {"requests": int(sel.sum()), "p50_ms": pct(ms[sel], 50), "p99_ms": pct(ms[sel], 99)}
        # where the slowest 5% of the class spent their time (means, ms)
        rsel = rt[np.array([label_of[int(r)] == lab for r in rt["id"]], bool)] if len(rt) else rt
        if len(rsel):
            cut = np.percentile(rsel["total_ms"], 95)
            tail = rsel[rsel["total_ms"] >= cut]
            classes[lab]["tail5"] = {k: float(np.mean(tail[k])) for k in
                                     ("total_ms", "queue_ms", "upload_ms", "run_ms", "result_ms", "launch_maps")}
    edges = float(np.sum(ed))
    return {"rate_maps_per_s": rate, "requests": n_req, "workers": workers,
            "large_workers": _LARGE_WORKERS or max(1, workers // 2), "large_yield_ms": _LARGE_YIELD_MS,
            "wall_s": wall,
            "edges_per_s": edges / wall, "maps_per_s": len(ms) / wall,
            "p50_ms": pct(ms, 50), "p95_ms": pct(ms, 95), "p99_ms": pct(ms, 99), "max_ms": float(np.max(ms)),
            "by_class": classes,
            "launches": int(st["launches"] - st0["launches"]), "failed": int(st["failed"]),
            "worker_ms": {k: float(st[k] - st0[k]) for k in ("upload_ms", "run_ms", "device_ms", "result_ms")},
            "queue_ms_mean": float(st["queue_ms"] - st0["queue_ms"]) / max(1, len(ms)),
            "growth_during_stream": {k: float(st[k] - st0[k]) for k in ("device_grows", "device_grow_ms",
                                                                        "host_grows", "host_grow_ms")},
            "reserved_gib": float(st["reserved_bytes"]) / 2 ** 30,
            "admission": "40 GiB budget; each request charged its workspace footprint (40 pairs, 8 curvelets "
                         "per edge), each worker's workspace reserved at creation",
            "pool": f"{len(maps)} seeded maps" + (f" (the workload's {n_warm} and translated copies)"
                                                  if n_warm and n_warm < len(maps) else "")}


def _measured_peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def path_hbm(n_edges: int, n_curv: int, ms_per_step: float, peaks: dict, edge_bytes: int = 32) -> dict:
    """The whole path against the HBM roofline, per GPU: the algorithmic bytes of a
    step are the edges in (4 FP64 values, 32 B per edge) and the curvelets out (a
    5-column uint32 chain row and 10 FP64 info values, 100 B per curvelet)."""
    hbm = peaks.get("hbm_gbs") or 6650.0
    b = float(edge_bytes) * n_edges + 100.0 * n_curv
    achieved = b / (ms_per_step / 1e3) / 1e9 if ms_per_step > 0 else 0.0
    return {"bound": "hbm", "scope": "whole path, per GPU", "bytes_per_step": b, "achieved": achieved,
            "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
            "work": f"{edge_bytes} B per edge in + 100 B per curvelet out",
            "note": "the path is bound by its FP64 bundle transport and by latency, not by HBM"}


def run_ours(args, maps, cfg, world, rank, local, pg):
    import curvelet_construction_on_gpu_b200 as cvl
    eng = cvl.Engine(device=local)
    n_edges = int(sum(m.shape[0] for m in maps))
    _progress(f"{len(maps)} map(s), {n_edges} edges: upload")
    batch = eng.upload_batch(maps)
    fp64_peak = eng.fp64_peak_tflops() if rank == 0 else None

    for _ in range(args.warmup):
        r = eng.run_batch(batch)
        r.close()
    _barrier(pg)
    _progress("timed steps")
    step_ms, kern, launches, bundle_launches = [], [], 0, 1
    with _Clocks(local) as clk:
        for _ in range(args.steps):
            eng.flush_l2()
            r = eng.run_batch(batch)
            st = r.stats()
            step_ms.append(st["device_ms"])
            launches = int(st["launches"])
            kt = eng.kernel_times()
            bundle_launches = sum(1 for name, _ in kt if name == "bundles")
            kern.append(_stage_sums(kt))
            r.close()
    _barrier(pg)
    sum_ms = _max_over_ranks(pg, float(np.sum(step_ms)))
    total_edges = _sum_over_ranks(pg, float(n_edges)) * args.steps
    value = total_edges / (sum_ms / 1e3)
    last = eng.run_batch(batch)
    stats = last.stats()
    n_curv = int(stats["num_curvelets"])
    nonclose = int(stats["total_pairs"]) - int(stats["close_pairs"])
    valid_nonclose = int(stats["valid_pairs"]) - int(stats["close_pairs"])
    last.close()

    plain = None
    if len(maps) > 1 and not args.no_plain:
        _progress("plain form (one map per launch)")
        pms = _plain_wall_ms(eng, maps, max(1, min(args.steps, 3)))
        pms = _max_over_ranks(pg, pms)
        plain = {"value": _sum_over_ranks(pg, float(n_edges)) / (pms / 1e3), "unit": METRIC, "ms_per_step": pms,
                 "form": "one map per launch (cvl_batch_run), maps resident, same engine, wall clock with the "
                         "host syncs between launches"}

    # e2e through the public C ABI with host buffers: the one-shot call for a
    # single map, the batch calls (upload, run, download every map) for a batch
    e2e = None
    if not args.no_e2e:
        _progress("e2e through the C ABI")
        if len(maps) == 1:
            pinned = _pinned(maps[0])
            # untimed: the engine's page-locked result pool grows to the two results
            # the timed loop holds at once (the previous step's and the current one)
            held = [eng.run(pinned), eng.run(pinned)]
            del held
        else:
            pinned = _pinned(np.concatenate(maps, axis=0))
            counts = np.array([m.shape[0] for m in maps], np.int32)
            # untimed pass: the result pool's page-locked blocks are allocated once
            held = eng.run_maps(pinned, counts=counts)
            del held
        _barrier(pg)
        t0 = time.perf_counter()
        bo = 0
        for _ in range(args.steps):
            if len(maps) == 1:
                res = eng.run(pinned)
                bo += res.chains.nbytes + res.info.nbytes
            else:
                for res in eng.run_maps(pinned, counts=counts):
                    bo += res.chains.nbytes + res.info.nbytes
                    del res
        wall = time.perf_counter() - t0
        wall = _max_over_ranks(pg, wall)
        e2e = {"value": _sum_over_ranks(pg, float(n_edges)) * args.steps / wall, "unit": METRIC,
               "h2d_bytes_per_step": int(sum(m.nbytes for m in maps)), "d2h_bytes_per_step": int(bo // args.steps),
               "path": ("cvl_run (C ABI), pinned host edges" if len(maps) == 1 else
                        "cvl_run_maps (C ABI): pinned host edges in, one result per map out; groups of maps "
                        "pipelined, result copies overlapping the next group's compute")}

    small = stress = None
    sweep = []
    stress_maps = None
    if len(maps) > 1 and (not args.no_small or not args.no_stress):
        from curvelet_construction_on_gpu_b200 import synth
        _progress("stress mix maps")
        stress_maps, stress_kinds = synth.stress_mix(5000 + 10_000 * rank)
    if stress_maps is not None and not args.no_small:
        _progress("small maps: batched vs plain")
        small = _small_maps(eng, [m for m, k in zip(stress_maps, stress_kinds) if k == "small"],
                            max(1, min(args.steps, 3)), pg)

    served = None
    if len(maps) > 1 and not args.no_served and cfg.get("_labels"):
        batch.close()
        eng.close()
        rates = [args.rate] if args.no_sweep else sorted({float(r) for r in args.rates.split(",") if r} | {args.rate})
        pool, labels = _distinct_pool(maps, cfg["_labels"], 1 if args.no_sweep else 4, rank)
        for rate in rates:
            _progress(f"served stream at {rate:g} maps/s")
            sv = _served(pool, labels, rate, args.requests, args.workers, local, n_warm=len(maps))
            sweep.append(sv)
            if rate == args.rate:
                served = sv
        del pool
    if stress_maps is not None and not args.no_stress:
        _progress("stress stream at 150 maps/s")
        stress = _served(stress_maps, stress_kinds, 150.0, len(stress_maps), args.workers, local,
                         sequence=list(range(len(stress_maps))), warm_all=False)

    if rank != 0:
        return
    curv_ms = float(np.mean([k.get("bundles", 0.0) for k in kern]))
    flops = FLOPS_PER_PAIR_CELL * 63 * nonclose
    achieved = flops / (curv_ms / 1e3) / 1e12 if curv_ms > 0 else 0.0
    launches_b = max(1, int(bundle_launches))
    clocks = clk.summary()
    stage_ms = {k: float(np.mean([d.get(k, 0.0) for d in kern])) for k in kern[0]} if kern else {}
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators, curvelet_construction_on_gpu_b200/synth.py)",
        "config": _config(args, n_edges, world, cfg),
        "workload_stats": {"curvelets_per_gpu": n_curv, "pairs_per_gpu": int(stats["total_pairs"]),
                           "valid_pairs_per_gpu": int(stats["valid_pairs"])},
        "curvelets_per_s": n_curv * world * args.steps / (sum_ms / 1e3),
        "stage_ms": stage_ms,
        "roofline": {"bound": "fp64", "kernel": "k_bundles", "achieved": achieved, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if fp64_peak else None,
                     "peak_source": "measured DFMA loop (cvl_measure_fp64_peak), 2 flops per FMA",
                     "work": f"{FLOPS_PER_PAIR_CELL} flops x 63 cells x {nonclose} non-close pairs, "
                             f"{launches_b} launch(es) per step",
                     "traffic": BUNDLE_DRAM_BYTES_PER_PAIR * nonclose / launches_b,
                     "traffic_unit": "bytes per launch",
                     "traffic_source": "ncu dram bytes of k_bundles on the 242k-edge map, per non-close pair, "
                                       "times this workload's pairs per launch",
                     "algorithmic_bytes": (1008.0 * valid_nonclose + 10.0 * nonclose) / launches_b,
                     "algorithmic_bytes_note": "1,008 B of bundle per valid non-close pair written, 10 B per "
                                               "computed pair of ids and flags",
                     "fp64_pipe": {
                         "instr_per_cell": BUNDLE_FP64_INSTR_PER_CELL,
                         "frac": (BUNDLE_FP64_INSTR_PER_CELL * 63 * nonclose / (curv_ms / 1e3)
                                  / (fp64_peak * 1e12 / 2.0)) if (fp64_peak and curv_ms > 0) else None,
                         "note": "FP64-pipe instructions per cell from ncu, scaled to this run's k_bundles time, "
                                 "against the DFMA issue peak (measured TFLOP/s / 2)"}},
        "path_hbm": path_hbm(n_edges, n_curv, sum_ms / args.steps, _measured_peaks(),
                             edge_bytes=8 * int(maps[0].shape[1])),
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": e2e,
    }
    if plain is not None:
        line["plain"] = plain
        line["batched_vs_plain"] = value / plain["value"]
    if served is not None:
        line["served"] = served
    if len(sweep) > 1:
        line["served_sweep"] = sweep
    if stress is not None:
        line["stress"] = stress
    if small is not None:
        line["small_maps"] = small
    if world == 1 and not args.no_cpu_baseline:
        _progress("cpu baseline")
        line["cpu_baseline"] = _cpu_baseline(maps, labels=cfg.get("_labels"))
    if len(maps) > 1:
        line["reference_sample_note"] = SAMPLE_NOTE
    print(json.dumps(line))
    eng.close()


def _contour_algorithmic_bytes(n_curv: int, width: int, c) -> int:
    """The stage's minimal DRAM traffic: the chains read once (4 B per entry),
    the links written (3 x 4 B), the fragments written (4 B per id, 8 B per
    offset), and two edge positions (2 x 16 B) read per fragment step."""
    return int(4 * n_curv * width + 12 * c.links.shape[0] + 4 * c.frag_ids.shape[0]
               + 8 * (c.num_frags + 1) + 32 * c.frag_ids.shape[0])


def run_contours(args, maps, cfg, world, rank, local, pg):
    import curvelet_construction_on_gpu_b200 as cvl
    eng = cvl.Engine(device=local)
    e = maps[0]
    cp = cvl.ContourParams(cfg["min_group_size"], cfg["gap"], fit_polyarcs=cfg["polyarcs"])
    n_edges = int(e.shape[0])
    pinned = _pinned(e)
    for _ in range(args.warmup):
        eng.run_contours(pinned, contour_params=cp, want_curvelets=False)
    _barrier(pg)
    step_ms, stage_ms, launches = [], [], 0
    with _Clocks(local) as clk:
        for _ in range(args.steps):
            eng.flush_l2()
            _, c = eng.run_contours(pinned, contour_params=cp, want_curvelets=False)
            step_ms.append(c.device_ms)
            kt = _stage_sums(eng.kernel_times())
            stage_ms.append(kt)
            launches = eng.launch_count()
    _barrier(pg)
    sum_ms = _max_over_ranks(pg, float(np.sum(step_ms)))
    value = _sum_over_ranks(pg, float(n_edges)) * args.steps / (sum_ms / 1e3)
    res, c = eng.run_contours(pinned, contour_params=cp)
    n_curv, width = res.num_curvelets, res.chains.shape[1]
    e2e = None
    if not args.no_e2e:
        _barrier(pg)
        t0 = time.perf_counter()
        bo = 0
        for _ in range(args.steps):
            r2, c2 = eng.run_contours(pinned, contour_params=cp)
            bo += r2.chains.nbytes + r2.info.nbytes + c2.links.nbytes + c2.frag_offsets.nbytes + c2.frag_ids.nbytes
            if c2.poly_offsets is not None:
                bo += c2.poly_offsets.nbytes + c2.poly_ids.nbytes + c2.poly_info.nbytes
            del r2, c2
        wall = _max_over_ranks(pg, time.perf_counter() - t0)
        e2e = {"value": _sum_over_ranks(pg, float(n_edges)) * args.steps / wall, "unit": METRIC,
               "h2d_bytes_per_step": int(e.nbytes), "d2h_bytes_per_step": int(bo // args.steps),
               "path": "cvl_run_contours (C ABI): pinned host edges in; curvelets, links, fragments and "
                       "polyarcs out"}
    if rank != 0:
        eng.close()
        return
    peaks = _measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    cms = float(np.mean([k.get("contours", 0.0) for k in stage_ms]))
    alg = _contour_algorithmic_bytes(n_curv, width, c)
    achieved = alg / (cms / 1e3) / 1e9 if cms > 0 else 0.0
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators, curvelet_construction_on_gpu_b200/synth.py)",
        "config": dict(workload="contours", edges_per_gpu=n_edges, curvelets_per_gpu=n_curv,
                       links=int(c.links.shape[0]), fragments=int(c.num_frags), fragment_ids=int(c.frag_ids.shape[0]),
                       l2="flushed between steps", parallelism=f"replicas x{world}", **cfg),
        "stage_ms": {k: float(np.mean([d.get(k, 0.0) for d in stage_ms])) for k in stage_ms[0]},
        "contour_stage": {"ms": cms, "edges_per_s": n_edges / (cms / 1e3) if cms > 0 else None,
                          "links_per_s": c.links.shape[0] / (cms / 1e3) if cms > 0 else None},
        "polyarc_stage": {"ms": float(np.mean([k.get("polyarcs", 0.0) for k in stage_ms])),
                          "polyarcs": c.num_polyarcs},
        "roofline": {"bound": "hbm", "kernel": "contour stage (k_link_* + k_trace_* + k_frag_*)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                     "algorithmic_bytes": alg, "traffic": None,
                     "note": "the stage walks contours edge by edge (one thread per component): latency-bound, "
                             "so the HBM fraction is low by nature"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        threads = _physical_cores()
        if O.ref_available() and O.orig_available():
            r = O.ref_run(e, nthreads=threads)
            ref_s = (r.ms["csr"] + r.ms["pairwise"] + r.ms["greedy"]) / 1e3
            fw = (r.info[:, 0] > 0).astype(np.uint8)
            rc = O.ref_link_contours(e, r.chains, fw, cp.min_group_size, cp.gap)
            line["cpu_baseline"] = {
                "value": n_edges / (ref_s + rc.seconds), "unit": METRIC, "cores": threads, "kind": "reference",
                "cpu_model": _cpu_model(),
                "sample": f"the whole map ({n_edges} edges): cpu_curvelet CSR + pairwise + greedy on {threads} "
                          f"threads ({ref_s * 1e3:.1f} ms) + original_code construct_the_link_graph + "
                          f"extract_regular_contours_from_the_link_graph, single-threaded as written "
                          f"({rc.seconds * 1e3:.1f} ms)",
                "contour_stage_ms": rc.seconds * 1e3,
                "same_result": bool(np.array_equal(rc.links, c.links) and np.array_equal(rc.frag_ids, c.frag_ids)
                                    and np.array_equal(rc.frag_offsets, c.frag_offsets))}
            # the polyarc fit on the CPU: the C restatement (linear). The reference's own
            # fit refits every earlier polyarc at the end of each fragment (quadratic) and
            # is not timed here.
            t0 = time.perf_counter()
            pc = O.polyarcs(e, rc.frag_offsets, rc.frag_ids)
            line["cpu_baseline"]["polyarc_stage"] = {
                "ms": 1e3 * (time.perf_counter() - t0), "kind": "port", "cores": 1, "polyarcs": pc.num,
                "same_chains": bool(np.array_equal(pc.ids, c.poly_ids) and np.array_equal(pc.offsets, c.poly_offsets))}
        else:
            t0 = time.perf_counter()
            r = O.run(e, nthreads=threads)
            oc = O.link_contours(e, r.chains, cp.min_group_size, cp.gap)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": n_edges / dt, "unit": METRIC, "cores": threads, "kind": "port",
                                    "sample": f"the whole map ({n_edges} edges), oracle restatement"}
    print(json.dumps(line))
    eng.close()


def run_reference_contours(args, maps, cfg, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    if not (O.ref_available() and O.orig_available()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref harnesses were not built "
                          "(the reference sources were absent at build time)"}))
        return
    threads = _physical_cores()
    e = maps[0]
    r = O.ref_run(e, nthreads=threads)
    fw = (r.info[:, 0] > 0).astype(np.uint8)
    for _ in range(max(1, args.warmup)):
        O.ref_link_contours(e, r.chains, fw, cfg["min_group_size"], cfg["gap"])
    step_s = []
    for _ in range(args.steps):
        r = O.ref_run(e, nthreads=threads)
        rc = O.ref_link_contours(e, r.chains, fw, cfg["min_group_size"], cfg["gap"])
        step_s.append((r.ms["csr"] + r.ms["pairwise"] + r.ms["greedy"]) / 1e3 + rc.seconds)
    ms = 1e3 * float(np.mean(step_s))
    value = e.shape[0] / (ms / 1e3)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": dict(workload="contours", edges=int(e.shape[0]), **cfg),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": "the whole map per step: cpu_curvelet phases + original_code link graph "
                                   "and one-chain extraction"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_served(args, maps, cfg, world, rank, local, pg):
    """The served stream alone, swept over --rates (one JSON line)."""
    rates = [float(r) for r in args.rates.split(",") if r]
    sweep = [_served(maps, cfg["_labels"], r, args.requests, args.workers, local) for r in rates]
    if rank != 0:
        return
    best = max(sweep, key=lambda d: d["edges_per_s"])
    cfg = {k: v for k, v in cfg.items() if not k.startswith("_")}
    print(json.dumps({
        "metric": METRIC, "value": best["edges_per_s"], "unit": METRIC, "n_gpus": world, "steps": len(rates),
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generators, curvelet_construction_on_gpu_b200/synth.py)",
        "config": dict(workload="served", requests_per_rate=args.requests, rates=rates, **cfg),
        "served": sweep}))


def run_stress(args, maps, cfg, world, rank, local, pg):
    """The stress stream (16 dense 3840x2160 maps among 1,024 small 640x480 maps): every map once, in its seeded
    interleaved order, Poisson at --rate (150 maps/s unless given); small-map
    latency reported apart from the dense maps'."""
    rate = args.rate if args.rate_given else 150.0
    sv = _served(maps, cfg["_labels"], rate, len(maps), args.workers, local, sequence=list(range(len(maps))),
                 warm_all=False)
    if rank != 0:
        return
    cfg = {k: v for k, v in cfg.items() if not k.startswith("_")}
    print(json.dumps({
        "metric": METRIC, "value": sv["edges_per_s"], "unit": METRIC, "n_gpus": world, "steps": 1, "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators, curvelet_construction_on_gpu_b200/synth.py)",
        "config": dict(workload="stress", rate_maps_per_s=rate, **cfg), "served": sv}))


_LARGE_WORKERS = 0  # the served stream's large-lane workers (--large-workers; 0: half of them)
_LARGE_YIELD_MS = 10  # --large-yield-ms


def main():
    global _LARGE_WORKERS, _LARGE_YIELD_MS
    args = _args()
    _LARGE_WORKERS = args.large_workers
    _LARGE_YIELD_MS = args.large_yield_ms
    world, rank, local, pg = _dist_init(args)
    maps, cfg = _workload(args.workload, rank)
    try:
        if args.impl == "reference" and args.workload == "contours":
            run_reference_contours(args, maps, cfg, world, rank)
        elif args.impl == "reference":
            run_reference(args, maps, cfg, world, rank)
        elif args.workload == "contours":
            run_contours(args, maps, cfg, world, rank, local, pg)
        elif args.workload == "served":
            run_served(args, maps, cfg, world, rank, local, pg)
        elif args.workload == "stress":
            run_stress(args, maps, cfg, world, rank, local, pg)
        else:
            run_ours(args, maps, cfg, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
