#!/usr/bin/env python
"""Mixed-batch throughput of the B200 masstree on the 16M variable-length-key
workload (one step = one mixed_batch call of 1M requests: 50% find, 30% insert
of fresh keys, 10% update, 10% erase, Zipf(0.99) key choice, after a 16M-key
preload; keys 2-16 slices sharing 4096 four-slice prefixes, values 1-8 slices).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl ours (default) prints one JSON line with the device-resident throughput
(`value`), the end-to-end throughput through the C ABI with pinned host buffers
(`e2e`: mt_mixed_batch_host uploads every step's requests and downloads its
results, overlapped with the work), the roofline of the batch kernel, the CPU
baseline and the SM clocks seen during the timed region.
--impl reference times the CPU restatement of the path (the reference's own CPU
counterpart, masstree-beta, is not available) with every host thread, on the
same workload.  Under torchrun each rank runs an independent replica (the index
is not partitioned across GPUs), so `value` is the sum over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from indexingpu_b200 import workload as wl  # noqa: E402

MAXK, MAXV = 16, 8
METRIC = "mixed-batch Mops/s @16M var-len keys"
UNIT = "Mops/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--preload", type=int, default=1 << 24)
    ap.add_argument("--batch", type=int, default=1 << 20)
    ap.add_argument("--tile", type=int, default=8, help="lanes per find")
    ap.add_argument("--write-tile", type=int, default=32, help="lanes per insert/update/erase")
    ap.add_argument("--upderase-tile", type=int, default=0,
                    help="lanes per update/erase of a mixed batch (0: the write width)")
    ap.add_argument("--scan-tile", type=int, default=4, help="lanes per scan query (c3 section)")
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--bucket", type=int, default=0, help="1: mixed_batch serves short keys before long keys")
    ap.add_argument("--host-chunk", type=int, default=0,
                    help="requests per chunk of mt_mixed_batch_host in the e2e leg (0: the library's default)")
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-batches", type=int, default=4, help="timed 1M-request batches in the CPU sample")
    ap.add_argument("--pool-gb", type=float, default=0.0,
                    help="slab pool size in GB (default: 60%% of the free device memory)")
    ap.add_argument("--grouped-max-ops", type=int, default=1 << 20,
                    help="largest sub-batch of the opt-in grouped section")
    ap.add_argument("--sections", default="batched,served,c1,c3",
                    help="extra measurements at N=1: batched (256 sub-batches, tuned form replayed from a "
                         "CUDA graph, against one call per sub-batch), served (request loop over 64M keys, "
                         "latency against offered load, against one call per request), c1 (plain insert and "
                         "find, 1M keys), c3 (range scan, 32M keys); 'none' to skip; also space (slabs "
                         "held after erase rounds without merges, with merges, and with merges and emptied-"
                         "layer removal; not in the default list), grouped (one grouped mixed_batches call on "
                         "--subbatches sub-batches of up to --grouped-max-ops requests: the profiling case of "
                         "that form; not in the default list)")
    ap.add_argument("--space-keys", type=int, default=1 << 21, help="tree size for the space section")
    ap.add_argument("--subbatches", type=int, default=256)
    ap.add_argument("--tune-subbatches", type=int, default=16, help="sub-batches per autotuner trial")
    ap.add_argument("--serve-keys", type=int, default=1 << 26, help="tree size for the served section")
    ap.add_argument("--serve-requests", type=int, default=8000, help="requests per offered-load point")
    ap.add_argument("--serve-chunk", type=int, default=0,
                    help="ops per work item of the request loop (0: chosen per request from the backlog)")
    return ap.parse_args()


# ---- data --------------------------------------------------------------------------

def gen_keys(c2, ids, threads=16):
    chunks = np.array_split(ids, max(1, min(threads, len(ids) // 65536)))
    with ThreadPoolExecutor(len(chunks)) as ex:
        parts = list(ex.map(c2.keys, chunks))
    return tuple(np.concatenate([p[i] for p in parts]) for i in range(4))


def gen_batches(c2, first, count, n, threads=16):
    with ThreadPoolExecutor(min(threads, count)) as ex:
        return list(ex.map(lambda b: c2.batch(b, n), range(first, first + count)))


def alg_bytes(bt, vlen_out, results):
    """Compulsory-traffic model per request (bytes): request I/O plus one
    128-byte border line and, for a hit on a chained entry, one 128-byte suffix
    line; successful insert/update/erase count their lines twice (read and
    write back).  Interior levels are assumed L2-resident."""
    t = bt["types"]
    L = bt["lens"].astype(np.int64)
    vin = bt["vlens"].astype(np.int64)
    req = 4 * L + 4 + 1
    find = t == wl.REQ_FIND
    io = np.where(find, 4 * np.minimum(vlen_out.astype(np.int64), MAXV) + 4, 1)
    io = io + np.where((t == wl.REQ_INSERT) | (t == wl.REQ_UPDATE), 4 * vin + 4, 0)
    hit = np.where(find, vlen_out > 0, results.astype(bool))
    vl = np.where(find, vlen_out.astype(np.int64), vin)
    chained = hit & ((vl > 1) | (L >= 6))
    lines = 128 * (1 + chained.astype(np.int64))
    mut_ok = (~find) & results.astype(bool)
    lines = np.where(mut_ok, 2 * lines, lines)
    return int((req + io + lines).sum())


# ---- clocks ------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_profile():
    """Per-launch DRAM bytes of the batch kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "mixed_batch_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_request")
    return None


# ---- CPU leg (oracle port) -----------------------------------------------------------

def cpu_run(preload_data, batches, threads):
    """Times the range-partitioned multi-threaded CPU restatement (the oracle
    port) on mixed batches after the same preload; returns Mops/s per batch."""
    from oracle.pyoracle import CpuOracle
    keys, lens, vals, vlens = preload_data
    o = CpuOracle(shards=threads, threads=threads)
    o.insert(keys, MAXK, lens, vals, MAXV, vlens, len(keys))
    rates = []
    for bt in batches:
        v = bt["vals"].copy()
        vl = bt["vlens"].copy()
        res = np.zeros(len(bt["types"]), np.uint8)
        t0 = time.perf_counter()
        o.mixed(bt["types"], bt["keys"], MAXK, bt["lens"], v, MAXV, vl, res, len(bt["types"]))
        dt = time.perf_counter() - t0
        rates.append(len(bt["types"]) / dt / 1e6)
    del o
    return rates


# ---- GPU leg -------------------------------------------------------------------------

def max_over_ranks(dist, values, device):
    """Element-wise maximum of per-rank times over all ranks (every rank gets it)."""
    import torch
    t = torch.tensor(values, device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(requests_per_rank, world, ms):
    """Mops/s of the whole job: every rank's requests over the slowest rank's time
    (replicas: each rank serves its own index, weak scaling)."""
    return requests_per_rank * world / (ms / 1e3) / 1e6


def run_ours(args, rank, world, dist):
    import torch
    from indexingpu_b200 import GpuMasstree

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    c2 = wl.C2(n_preload=args.preload, seed=0xC2 + rank)
    pre = gen_keys(c2, np.arange(args.preload))
    nb = args.warmup + args.steps
    batches = gen_batches(c2, 0, nb, args.batch)
    e2e_w, e2e_k = 2, max(1, min(args.e2e_steps, args.steps))
    e2e_batches = gen_batches(c2, nb, e2e_w + e2e_k, args.batch)

    if args.pool_gb > 0:
        tree = GpuMasstree(pool_bytes=int(args.pool_gb * (1 << 30)), tile_size=args.tile)
    else:
        tree = GpuMasstree(pool_ratio=0.6, tile_size=args.tile)
    tree.set_write_tile_size(args.write_tile)
    tree.set_upderase_tile_size(args.upderase_tile)
    if args.blocks_per_sm:
        tree.set_blocks_per_sm(args.blocks_per_sm)
    stream = torch.cuda.current_stream()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    # Preload in 1M chunks.
    pk = d(pre[0]); pl = d(pre[1]); pv = d(pre[2]); pvl = d(pre[3])
    for s in range(0, args.preload, 1 << 20):
        e = min(args.preload, s + (1 << 20))
        tree.insert(pk[s:e], MAXK, pl[s:e], pv[s:e], MAXV, pvl[s:e], e - s, stream=stream)
    tree.sync(stream)
    del pk, pl, pv, pvl

    # Device-resident batches.
    dev_b = []
    for bt in batches:
        dev_b.append(dict(types=d(bt["types"]), keys=d(bt["keys"]), lens=d(bt["lens"]), vals=d(bt["vals"]),
                          vlens=d(bt["vlens"]), res=torch.zeros(args.batch, dtype=torch.bool, device="cuda")))
    torch.cuda.synchronize()

    def step(b):
        tree.mixed_batch(b["types"], b["keys"], MAXK, b["lens"], b["vals"], MAXV, b["vlens"], b["res"], args.batch,
                         stream=stream, bucket_keys=bool(args.bucket))

    for i in range(args.warmup):
        step(dev_b[i])
    tree.sync(stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(dev)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step(dev_b[args.warmup + i])
        ev[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    tree.sync(stream)
    total_ms = t0.elapsed_time(t1)
    per_step = [a.elapsed_time(b) for a, b in ev]

    # Algorithmic bytes from the timed batches' own outcomes.
    abytes = 0
    for i in range(args.steps):
        b = dev_b[args.warmup + i]
        bt = batches[args.warmup + i]
        abytes += alg_bytes(bt, b["vlens"].cpu().numpy(), b["res"].cpu().numpy())
    del dev_b

    # End to end: pinned host buffers in, results out, every step, through
    # mt_mixed_batch_host (uploads, work and downloads of consecutive chunks
    # overlap, also across steps).
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    host = [dict(types=pin(bt["types"]), keys=pin(bt["keys"]), lens=pin(bt["lens"]), vals=pin(bt["vals"]),
                 vlens=pin(bt["vlens"]), res=torch.zeros(args.batch, dtype=torch.bool).pin_memory())
            for bt in e2e_batches]
    h2d = sum(host[0][k].numel() * host[0][k].element_size() for k in ("types", "keys", "lens", "vals", "vlens"))
    d2h = sum(host[0][k].numel() * host[0][k].element_size() for k in ("vals", "vlens", "res"))

    def e2e_step(h):
        tree.mixed_batch_host(h["types"], h["keys"], MAXK, h["lens"], h["vals"], MAXV, h["vlens"], h["res"],
                              args.batch, stream=stream, chunk=args.host_chunk, bucket_keys=bool(args.bucket))

    for i in range(e2e_w):
        e2e_step(host[i])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h0 = time.perf_counter()
    for i in range(e2e_k):
        e2e_step(host[e2e_w + i])
    host_ms = (time.perf_counter() - h0) * 1e3  # the calls' own host time (enqueueing), for comparison
    e1.record(stream)
    torch.cuda.synchronize()
    tree.sync(stream)
    e2e_ms = e0.elapsed_time(e1)
    stats = tree.stats()
    extra = {}
    wanted = set() if args.sections == "none" else set(args.sections.split(","))
    if world == 1:
        del host
        if "batched" in wanted:
            extra["batched"] = run_batched(args, tree, c2, stream)
        if "served" in wanted:
            extra["served"] = run_served(args, tree, c2, stream)
        if "grouped" in wanted:
            extra["grouped"] = run_grouped(args, tree, c2, stream)
    tree.close()
    if world == 1 and ("c1" in wanted or "c3" in wanted):
        del tree
        peak_c, _ = measured_peak()
        if "c1" in wanted:
            extra["c1"] = run_c1(args, stream, peak_c)
        if "c3" in wanted:
            extra["c3"] = run_c3(args, stream, peak_c)
    if world == 1 and "space" in wanted:
        extra["space"] = run_space(args, stream)

    # Reduce over ranks: max time.
    if dist:
        total_ms, e2e_ms = max_over_ranks(dist, [total_ms, e2e_ms], "cuda")
    value = whole_job_rate(args.steps * args.batch, world, total_ms)
    e2e_value = whole_job_rate(e2e_k * args.batch, world, e2e_ms)

    res = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        kern_s = statistics.mean(per_step) / 1e3
        achieved = abytes / args.steps / kern_s / 1e9
        tr = traffic_profile()
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            cpu_b = gen_batches(c2, 0, args.cpu_batches, args.batch)
            rates = cpu_run(pre, cpu_b, threads)
            cpu = {"value": round(statistics.mean(rates), 3), "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_batches} mixed batches of {args.batch} requests after the "
                             f"{args.preload}-key preload, range-partitioned std::map restatement, "
                             f"{threads} threads"}
        sorted_steps = sorted(per_step)
        res = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded, counter-based)",
            "config": {"workload": "mixed_batch 1M requests (50/30/10/10 find/insert/update/erase, Zipf 0.99) "
                                   "after a 16M-key preload; keys 2-16 slices, 4096 shared prefixes; values 1-8 slices",
                       "preload_keys": args.preload, "batch_requests": args.batch, "max_key_length": MAXK,
                       "max_value_length": MAXV, "tile_size": args.tile, "write_tile_size": args.write_tile,
                       "upderase_tile_size": args.upderase_tile or args.write_tile,
                       "form": "plain per-call mixed_batch (reclaim, three-way partition, find / insert / "
                               "update+erase class kernels on forked streams, updates of one key combined)",
                       "l2": "no flush: the index (>2 GB of slabs) and each batch's inputs exceed the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "batch_latency_ms": {"p50": round(sorted_steps[len(sorted_steps) // 2], 4),
                                 "p99": round(sorted_steps[min(len(sorted_steps) - 1,
                                                               int(0.99 * len(sorted_steps)))], 4)},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_k,
                    "host_call_ms_per_step": round(host_ms / e2e_k, 4),
                    "call": "mt_mixed_batch_host (pinned host buffers; chunked uploads, work and downloads "
                            "overlapped)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": None if tr is None else int(tr * args.batch),
                         "algorithmic_bytes_per_step": abytes // args.steps,
                         "kernel": "mixed_batch call: reclaim + partition + three class kernels"},
            "cpu_baseline": cpu,
            "clocks": clk,
            # reclaim, partition, find class, insert class, update combining,
            # update/erase class, combined results: 7 kernels per step
            "gpu_launches": 7 * args.steps,
            "pool": {"used_slabs": stats["used_slabs"], "total_slabs": stats["total_slabs"]},
        }
        res.update(extra)
        if "served" in res:
            # Served peaks against this run's plain 1M-request mixed batches.
            for k in ("served_peak", "online_peak"):
                res["served"][k + "_over_plain_1M_batch"] = round(res["served"][k]["mops"] / value, 3)
    return res


# ---- batched and served forms ------------------------------------------------------

def _dev_ops(torch, st):
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return dict(types=d(st["types"]), keys=d(st["keys"]), lens=d(st["lens"]), vals=d(st["vals"]),
                vlens=d(st["vlens"]), res=torch.zeros(len(st["types"]), dtype=torch.bool, device="cuda"))


def _subbatches(dev, st):
    subs = []
    for f, n in zip(st["first"].tolist(), st["nops"].tolist()):
        subs.append(dict(types=dev["types"][f:f + n], keys=dev["keys"][f:f + n], lens=dev["lens"][f:f + n],
                         vals=dev["vals"][f:f + n], vlens=dev["vlens"][f:f + n], results=dev["res"][f:f + n],
                         n=n))
    return subs


def run_batched(args, tree, c2, stream):
    """256 mixed sub-batches of log-uniform sizes in [1K, 1M] (sizes from seed
    0xC4, C2 op mix and key choice): one mixed_batch call per sub-batch against
    the autotuned persistent launch (mt_mixed_batches) replayed from a CUDA
    graph, each on its own draw of the ops (same sizes)."""
    import torch
    from indexingpu_b200 import autotune
    from indexingpu_b200.masstree import pack_subbatches

    base = args.preload + (1 << 30)  # fresh-key ids of this section, above every c2.batch id
    shape = dict(min_ops=1024, max_ops=1 << 20, seed=0xC4)
    # One call per sub-batch.
    st = wl.serve_stream(c2, args.subbatches, op_seed=0xC4, first_fresh=base, **shape)
    dev = _dev_ops(torch, st)
    total = int(st["nops"].sum())
    # Size the per-call scratch for the largest sub-batch outside the timed
    # region (an untimed call of finds that miss: the tree does not change).
    n_max = int(st["nops"].max())
    tree.mixed_batch(torch.full((n_max,), wl.REQ_FIND, dtype=torch.uint8, device="cuda"),
                     torch.zeros((n_max, MAXK), dtype=torch.uint32, device="cuda"), MAXK,
                     torch.full((n_max,), MAXK, dtype=torch.uint32, device="cuda"),
                     torch.zeros((n_max, MAXV), dtype=torch.uint32, device="cuda"), MAXV,
                     torch.zeros(n_max, dtype=torch.uint32, device="cuda"), None, n_max, stream=stream)
    tree.sync(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sb in _subbatches(dev, st):
        tree.mixed_batch(sb["types"], sb["keys"], MAXK, sb["lens"], sb["vals"], MAXV, sb["vlens"], sb["results"],
                         sb["n"], stream=stream, bucket_keys=bool(args.bucket))
    e1.record(stream)
    tree.sync(stream)
    per_call = total / (e0.elapsed_time(e1) / 1e3) / 1e6
    del dev

    # Autotune on smaller cases of the same size distribution, fresh ops each.
    def make_case(i):
        cst = wl.serve_stream(c2, args.tune_subbatches, min_ops=1024, max_ops=1 << 20, seed=0xC4 + 7,
                              op_seed=0xC4 + 100 + i, first_fresh=base + (1 << 27) + i * (1 << 23))
        cdev = _dev_ops(torch, cst)
        desc = torch.from_numpy(pack_subbatches(_subbatches(cdev, cst))).cuda()
        return dict(descriptors=desc, num_subbatches=len(cst["nops"]), total=int(cst["nops"].sum()),
                    max_key_length=MAXK, max_value_length=MAXV, keep=cdev)

    best, trials = autotune.tune(tree, make_case, stream=stream)

    # The tuned form: one persistent launch for all sub-batches, from a graph.
    st = wl.serve_stream(c2, args.subbatches, op_seed=0xC4 + 1, first_fresh=base + (1 << 26), **shape)
    dev = _dev_ops(torch, st)
    desc = torch.from_numpy(pack_subbatches(_subbatches(dev, st))).cuda()
    total_b = int(st["nops"].sum())
    autotune.apply(tree, best)
    tree.reserve_batches(args.subbatches, total_b)
    side = torch.cuda.Stream()
    grouped = best["form"] == "grouped"
    if grouped:
        # The grouped form sizes its scratch on its first call after the
        # reserve: one untimed call of a single find that misses (the tree
        # does not change), outside the capture.
        one = dict(types=torch.full((1,), wl.REQ_FIND, dtype=torch.uint8, device="cuda"),
                   keys=torch.zeros((1, MAXK), dtype=torch.uint32, device="cuda"),
                   lens=torch.full((1,), MAXK, dtype=torch.uint32, device="cuda"),
                   vals=torch.zeros((1, MAXV), dtype=torch.uint32, device="cuda"),
                   vlens=torch.zeros(1, dtype=torch.uint32, device="cuda"), results=None, n=1)
        one_desc = torch.from_numpy(pack_subbatches([one])).cuda()
        tree.mixed_batches(one_desc, 1, MAXK, MAXV, stream=side, group_by_key=True)
        tree.sync(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        tree.mixed_batches(desc, args.subbatches, MAXK, MAXV, stream=side, bucket_keys=best["bucketing"],
                           persistent=best["form"] == "persistent", group_by_key=grouped)
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        e0.record(side)
        g.replay()
        e1.record(side)
    tree.sync(side)
    batched = total_b / (e0.elapsed_time(e1) / 1e3) / 1e6
    del g, dev
    autotune.apply(tree, dict(find_tile=args.tile, write_tile=args.write_tile, blocks_per_sm=args.blocks_per_sm))
    return {"workload": f"{args.subbatches} mixed sub-batches, sizes log-uniform in [1K, 1M] (seed 0xC4), "
                        "C2 mix and Zipf(0.99) key choice over the preloaded keys",
            "requests": [total, total_b],
            "per_call_mops": round(per_call, 2), "batched_graph_mops": round(batched, 2),
            "batched_over_per_call": round(batched / per_call, 3),
            "tuned": best, "trials": trials,
            "note": "each form runs its own draw of the ops (same sizes) on the live tree"}


def run_grouped(args, tree, c2, stream):
    """One grouped mt_mixed_batches call (MT_FLAG_GROUP_BY_KEY) on --subbatches
    sub-batches of log-uniform sizes in [1K, --grouped-max-ops], after one untimed
    call of a single find that sizes its scratch (opt-in section, the profiling
    case of the grouped form)."""
    import torch
    from indexingpu_b200.masstree import pack_subbatches
    st = wl.serve_stream(c2, args.subbatches, min_ops=1024, max_ops=args.grouped_max_ops, seed=0xC4, op_seed=0xC4,
                         first_fresh=args.preload + (1 << 30))
    dev = _dev_ops(torch, st)
    desc = torch.from_numpy(pack_subbatches(_subbatches(dev, st))).cuda()
    total = int(st["nops"].sum())
    tree.set_tile_size(32)
    tree.reserve_batches(args.subbatches, total)
    one = dict(types=torch.full((1,), wl.REQ_FIND, dtype=torch.uint8, device="cuda"),
               keys=torch.zeros((1, MAXK), dtype=torch.uint32, device="cuda"),
               lens=torch.full((1,), MAXK, dtype=torch.uint32, device="cuda"),
               vals=torch.zeros((1, MAXV), dtype=torch.uint32, device="cuda"),
               vlens=torch.zeros(1, dtype=torch.uint32, device="cuda"), results=None, n=1)
    tree.mixed_batches(torch.from_numpy(pack_subbatches([one])).cuda(), 1, MAXK, MAXV, stream=stream,
                       group_by_key=True)
    tree.sync(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tree.mixed_batches(desc, args.subbatches, MAXK, MAXV, stream=stream, group_by_key=True)
    e1.record(stream)
    tree.sync(stream)
    ms = e0.elapsed_time(e1)
    tree.set_tile_size(args.tile)
    return {"workload": f"{args.subbatches} sub-batches of log-uniform sizes in [1K, {args.grouped_max_ops}], C2 mix",
            "requests": total, "ms": round(ms, 3), "mops": round(total / ms / 1e3, 2),
            "tiles": {"find": 32, "write": args.write_tile}}


def run_served(args, tree, c2, stream):
    """Open-loop request streams over the tree grown to --serve-keys keys:
    requests of 1-4096 ops (log-uniform, C2 mix), Poisson arrivals at 10..100%
    of the loop's measured peak, latency from arrival to the host seeing the
    completion; beside it one synchronous mixed_batch call per request."""
    import torch
    t_grow = time.time()
    step = 1 << 20
    for s0 in range(args.preload, args.serve_keys, step):
        ids = np.arange(s0, min(args.serve_keys, s0 + step))
        k, l, v, vl = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in gen_keys(c2, ids))
        tree.insert(k, MAXK, l, v, MAXV, vl, len(ids), stream=stream)
    tree.sync(stream)
    t_grow = time.time() - t_grow
    c5 = wl.C2(n_preload=args.serve_keys, seed=c2.seed)
    fresh0 = args.serve_keys + (1 << 31)
    n = args.serve_requests

    def once(i, rate, plain=False, n_req=n, online=False):
        st = wl.serve_stream(c5, n_req, rate_per_s=rate, min_ops=1, max_ops=4096, seed=0xC5 + i,
                             first_fresh=fresh0 + i * (1 << 24))
        if online:
            # Host (pinned) buffers: each request is uploaded when it is
            # submitted and its results downloaded when it completes.
            dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).pin_memory()
                   for k in ("types", "keys", "lens", "vals", "vlens")}
            dev["res"] = torch.zeros(len(st["types"]), dtype=torch.bool).pin_memory()
        else:
            dev = _dev_ops(torch, st)
        lat, stats = tree.serve(dev["types"], dev["keys"], MAXK, dev["lens"], dev["vals"], MAXV, dev["vlens"],
                                dev["res"], st["first"], st["nops"], st["arrival_ns"], plain=plain,
                                chunk_ops=args.serve_chunk, online=online)
        tree.sync(stream)
        ops = int(st["nops"].sum())
        p = np.percentile(lat / 1e3, [50, 99, 99.9])
        r = {"offered_req_s": None if rate is None else round(rate, 1), "requests": n_req, "ops": ops,
             "req_s": round(n_req / (stats["wall_ns"] / 1e9), 1), "mops": round(ops / stats["wall_ns"] * 1e3, 3),
             "p50_us": round(float(p[0]), 1), "p99_us": round(float(p[1]), 1), "p999_us": round(float(p[2]), 1),
             "admission_waits": stats["admission_waits"]}
        if online:
            # Mean time per stage of the server (submit -> admitted -> uploaded
            # and published -> completion flag seen -> results delivered).
            r["stage_mean_us"] = {k: round(v / 1e3 / max(1, stats["requests_done"]), 1)
                                  for k, v in stats["stage_ns"].items()}
        return r

    peak = once(0, None)
    curve = []
    for j, frac in enumerate((0.1, 0.25, 0.5, 0.75, 0.9, 1.0)):
        r = once(1 + j, frac * peak["req_s"])
        r["load"] = frac
        curve.append(r)
    # The same through the online server API from host buffers (uploads and
    # downloads inside every request's latency).
    online_peak = once(20, None, online=True)
    online_curve = []
    for j, frac in enumerate((0.1, 0.25, 0.5, 0.75, 0.9, 1.0)):
        r = once(21 + j, frac * online_peak["req_s"], online=True)
        r["load"] = frac
        online_curve.append(r)
    n_plain = max(200, n // 4)
    plain_peak = once(10, None, plain=True, n_req=n_plain)
    rate_eq = 0.5 * plain_peak["req_s"]
    plain_half = once(11, rate_eq, plain=True, n_req=n_plain)
    served_half = once(12, rate_eq, n_req=n_plain)
    return {"workload": f"requests of 1-4096 ops (log-uniform, C2 mix, Zipf(0.99) over {args.serve_keys} keys), "
                        "Poisson arrivals (seed 0xC5+i); latency = arrival to completion seen by the host",
            "tree_keys": args.serve_keys, "grow_s": round(t_grow, 1), "chunk_ops": args.serve_chunk,
            "served_peak": peak, "served_curve": curve,
            "online_note": "mt_server_* from pinned host buffers: upload, device work and download of each "
                           "request inside its latency",
            "online_peak": online_peak, "online_curve": online_curve,
            "plain_per_request_peak": plain_peak, "plain_at_half_its_peak": plain_half,
            "served_at_same_load": served_half,
            "served_over_plain_mops": round(peak["mops"] / plain_peak["mops"], 2)}


def _timed(stream, fn, reps=1):
    """Device time of reps calls of fn on stream (ms per call)."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_c1(args, stream, peak):
    """1M distinct keys of 1-8 random slices, 2-slice values: bulk insert, then
    1M finds (half hits, half absent keys), each timed on the device."""
    import torch
    from indexingpu_b200 import GpuMasstree
    torch.cuda.empty_cache()  # blocks cached by earlier sections would crowd the bulk build's scratch
    d = wl.c1()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    k, l, v, vl = dev(d["keys"]), dev(d["lens"]), dev(d["vals"]), dev(d["vlens"])
    fk, fl = dev(d["find_keys"]), dev(d["find_lens"])
    n, nf, mk, mv = len(d["keys"]), len(d["find_keys"]), d["maxK"], d["maxV"]
    out_v = torch.zeros((nf, mv), dtype=torch.uint32, device="cuda")
    out_l = torch.zeros(nf, dtype=torch.uint32, device="cuda")
    # The insert into an empty tree is one call (the bulk build): untimed once on
    # a small sample (kernels loaded on first use), then the median of three
    # fresh trees.
    with GpuMasstree(pool_bytes=256 << 20, tile_size=args.tile) as w:
        w.set_write_tile_size(args.write_tile)
        w.insert(k[:65536], mk, l[:65536], v[:65536], mv, vl[:65536], 65536, stream=stream)
        w.sync(stream)
    ins = []
    for rep in range(3):
        t = GpuMasstree(pool_bytes=2 << 30, tile_size=args.tile)
        t.set_write_tile_size(args.write_tile)
        ins.append(_timed(stream, lambda: t.insert(k, mk, l, v, mv, vl, n, stream=stream)))
        t.sync(stream)
        if rep < 2:
            t.close()
    ins_ms = sorted(ins)[1]
    with t:
        find = lambda: t.find(fk, mk, fl, out_v, mv, out_l, nf, stream=stream)  # noqa: E731
        for _ in range(3):
            find()
        find_ms = _timed(stream, find, reps=10)
        t.sync(stream)
    got = out_l.cpu().numpy()
    hits = int((got > 0).sum())
    assert hits == int(d["find_hit"].sum()), "C1 find hits differ from the generator's"
    # Compulsory bytes per find: request I/O + border line + value chain line on
    # a hit (2-slice values of 1-slice keys and the key rests of longer keys
    # live in chains).
    L = d["find_lens"].astype(np.int64)
    fb = int((4 * L + 4 + np.where(d["find_hit"], 4 * mv + 4 + 256, 4 + 128)).sum())
    ach = fb / (find_ms / 1e3) / 1e9
    return {"workload": "1M distinct keys of 1-8 random slices, 2-slice values; 1M finds, 50% hits",
            "insert_mops": round(n / ins_ms / 1e3, 2), "insert_ms_3_trees": [round(x, 3) for x in ins],
            "find_mops": round(nf / find_ms / 1e3, 2),
            "find_hits": hits,
            "find_roofline": {"achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                              "frac": round(ach / peak, 4), "algorithmic_bytes": fb,
                              "note": "the 1M-key index (~150 MB of slabs) is mostly L2-resident"}}


def run_space(args, stream):
    """Space held after erases: a tree of C2 keys erased in four rounds of a
    quarter of its keys each (random order), once per erase mode (no merges,
    MT_FLAG_MERGE, MT_FLAG_MERGE | MT_FLAG_REMOVE_EMPTY_LAYERS).  Reports used
    slabs after the preload and after every round, and each round's erase rate."""
    import torch
    from indexingpu_b200 import GpuMasstree
    n = args.space_keys
    c2 = wl.C2(n_preload=n)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    hk, hl, hv, hvl = wl.keys_threaded(c2, np.arange(n))
    k, l, v, vl = dev(hk), dev(hl), dev(hv), dev(hvl)
    order = np.random.default_rng(0x5BACE).permutation(n)
    rounds = [order[i * n // 4:(i + 1) * n // 4] for i in range(4)]
    rk = [(dev(hk[r]), dev(hl[r])) for r in rounds]
    res = torch.zeros(n // 4 + 1, dtype=torch.bool, device="cuda")
    modes = {"none": {}, "merge": {"merge": True}, "merge_remove_layers": {"merge": True, "remove_empty_layers": True}}
    out = {"workload": f"{n} C2 keys (2-16 slices, 4096 shared 4-slice prefixes), erased in 4 rounds of {n // 4}",
           "modes": {}}
    for name, flags in modes.items():
        with GpuMasstree(pool_bytes=2 << 30, tile_size=args.tile) as t:
            t.set_write_tile_size(args.write_tile)
            t.insert(k, c2.maxK, l, v, c2.maxV, vl, n, stream=stream)
            t.sync(stream)
            used = [t.stats()["used_slabs"]]
            rates = []
            for rkeys, rlens in rk:
                m = len(rlens)
                ms = _timed(stream, lambda: t.erase(rkeys, c2.maxK, rlens, m, stream=stream, results=res, **flags))
                t.sync(stream)
                assert int(res[:m].sum()) == m, "an erase round missed keys it had inserted"
                rates.append(round(m / ms / 1e3, 2))
                used.append(t.stats()["used_slabs"])
            out["modes"][name] = {"used_slabs": used, "erase_mops": rates}
    base = out["modes"]["none"]["used_slabs"][0]
    for m in out["modes"].values():
        m["used_pct_of_preload"] = [round(100.0 * u / base, 2) for u in m["used_slabs"]]
    return out


def run_c3(args, stream, peak):
    """32M fixed 2-slice keys (big-endian halves of random u64s), 1-slice
    values; 1M scans from random lower bounds, up to 100 results each, keys,
    values and lengths returned."""
    import torch
    from indexingpu_b200 import GpuMasstree
    torch.cuda.empty_cache()
    n, nq, mc = 1 << 25, 1 << 20, 100
    d = wl.c3(n, nq)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    lo, lol = dev(d["lower"]), dev(d["lower_lens"])
    counts = torch.zeros(nq, dtype=torch.uint32, device="cuda")
    vals = torch.zeros((nq, mc, 1), dtype=torch.uint32, device="cuda")
    vlens = torch.zeros((nq, mc), dtype=torch.uint32, device="cuda")
    okeys = torch.zeros((nq, mc, 2), dtype=torch.uint32, device="cuda")
    oklens = torch.zeros((nq, mc), dtype=torch.uint32, device="cuda")
    with GpuMasstree(pool_bytes=8 << 30, tile_size=args.tile) as t:
        t.set_write_tile_size(args.write_tile)
        t.set_scan_tile_size(args.scan_tile)
        step = 1 << 20
        for s0 in range(0, n, step):
            sl = slice(s0, s0 + step)
            t.insert(dev(d["keys"][sl]), 2, dev(d["lens"][sl]), dev(d["vals"][sl]), 1, dev(d["vlens"][sl]),
                     min(step, n - s0), stream=stream)
        t.sync(stream)
        scan = lambda: t.scan(lo, lol, 2, mc, nq, counts=counts, values=vals, max_value_length=1,  # noqa: E731
                              value_lengths=vlens, out_keys=okeys, out_key_lengths=oklens, stream=stream)
        scan()
        scan_ms = _timed(stream, scan, reps=3)
        t.sync(stream)
    c = counts.cpu().numpy().astype(np.int64)
    results = int(c.sum())
    # Sortedness of every query's output keys (as u64), checked on a sample.
    ok = okeys[:1024].cpu().numpy().astype(np.uint64)
    kk = (ok[:, :, 0] << np.uint64(32)) | ok[:, :, 1]
    for q in range(1024):
        assert np.all(kk[q, 1:c[q]] > kk[q, :c[q] - 1]), q
    # Compulsory bytes per query: lower key, the border lines the results span
    # (13 entries per node at most), one suffix line per result (key rest and
    # value), and the output rows.
    fb = int((8 + 128 * (np.ceil(c / 13.0) + 1) + 128 * c + c * (8 + 4 + 4 + 4) + 4).sum())
    ach = fb / (scan_ms / 1e3) / 1e9
    return {"workload": "32M keys of 2 slices, 1-slice values; 1M scans of up to 100 results from random lower "
                        "bounds (keys, values, lengths returned)",
            "scan_queries_per_s_M": round(nq / scan_ms / 1e3, 3), "results_per_s_M": round(results / scan_ms / 1e3, 2),
            "mean_results": round(results / nq, 2),
            "scan_roofline": {"achieved": round(ach, 2), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                              "algorithmic_bytes": fb}}


def run_reference(args, rank):
    """CPU restatement timed with every host thread (bounded per-step sample)."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    c2 = wl.C2(n_preload=args.preload, seed=0xC2)
    pre = gen_keys(c2, np.arange(args.preload))
    batches = gen_batches(c2, 0, args.warmup + args.steps, args.batch)
    from oracle.pyoracle import CpuOracle
    o = CpuOracle(shards=threads, threads=threads)
    o.insert(pre[0], MAXK, pre[1], pre[2], MAXV, pre[3], args.preload)
    times = []
    for i, bt in enumerate(batches):
        v, vl = bt["vals"].copy(), bt["vlens"].copy()
        res = np.zeros(args.batch, np.uint8)
        t0 = time.perf_counter()
        o.mixed(bt["types"], bt["keys"], MAXK, bt["lens"], v, MAXV, vl, res, args.batch)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps * args.batch / total / 1e6
    return {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded, counter-based)",
            "config": {"workload": "mixed_batch 1M requests (50/30/10/10 find/insert/update/erase, Zipf 0.99) "
                                   "after a 16M-key preload; keys 2-16 slices, 4096 shared prefixes; values 1-8 slices",
                       "preload_keys": args.preload, "batch_requests": args.batch},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} timed mixed batches of {args.batch} requests; CPU restatement "
                                       "(range-partitioned std::map, one thread per shard); the reference's own "
                                       "CPU path (masstree-beta) is absent and its GPU gpu_masstree hung on B200"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        if args.impl == "reference":
            res = run_reference(args, rank)
        else:
            res = run_ours(args, rank, world, dist)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
