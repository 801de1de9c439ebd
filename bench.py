#!/usr/bin/env python
"""Batched RAPTOR throughput of the B200 engine on the 40k-stop regional
timetable (workload 2: 10,000-query class, intermodal one-to-one, batches of
1024 resident queries per device pass).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
    python bench.py --impl reference ...   # the CPU raptor (oracle) arm

A step is one batch of B seeded queries through b2r_search_batch.  `value`
is queries / device time of the batch (timetable resident, queries
prepared); `e2e` is queries / wall time of the C-ABI call from host query
structs to host results (host preparation, admission copies, result copies
included).  Under torchrun every rank runs its own engine on its own query
shard (replicas; no collective on the data path) and the max over ranks is
reported.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = 2
METRIC = "queries/sec & p99 latency, batched/served vs 1-query GPU RAPTOR, bit-exact"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--batch", type=int, default=1024)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--cpu-sample", type=int, default=0, help="queries in the CPU baseline sample")
    p.add_argument("--no-extras", action="store_true", help="skip plain / roofline / CPU legs")
    p.add_argument("--no-national", action="store_true", help="skip the national-scale leg")
    p.add_argument("--ncu-case", action="store_true",
                   help="one batch without CUDA graphs (the case profiled with ncu)")
    p.add_argument("--ncu-counters", action="store_true",
                   help="with --ncu-case: count route-scan work (stop visits, events)")
    p.add_argument("--ncu-workload", type=int, default=2, choices=[1, 2, 3, 4, 5],
                   help="with --ncu-case: the workload's timetable and queries")
    p.add_argument("--shape", metavar="B,T,P,R,S,O",
                   help="with --ncu-case: launch shape (route-scan blocks per SM, threads, pair "
                        "blocks per SM, reconstruction blocks per SM, super-steps per sync, "
                        "route-scan occupancy build)")
    p.add_argument("--ncu-summary", metavar="CSV",
                   help="summarise an ncu --csv log (launches, time, share and any other metric "
                        "per kernel) and exit; runs on a machine without a GPU")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def percentile(xs, q):
    if not xs:
        return None
    xs = sorted(xs)
    k = (len(xs) - 1) * q
    f = int(k)
    c = min(f + 1, len(xs) - 1)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_unit():
    """The route scan's DRAM bytes per launch from the committed ncu capture
    of the bench's batch and launch shape (profiles/route_scan_traffic.json),
    with a few counters of the same kernel's detailed capture."""
    try:
        with open(os.path.join(ROOT, "profiles", "route_scan_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# --------------------------------------------------------------- CPU arms
def cpu_run(desc, qarr, n, threads):
    import oracle_lib  # tests/ is on the path only for the CPU arms
    lat = (C.c_double * max(1, n))()
    nj = C.c_uint64()
    wall = C.c_double()
    oracle_lib.lib().or_run_many(C.byref(desc), qarr, n, threads, lat, C.byref(nj), C.byref(wall))
    return wall.value, [lat[i] / 1e3 for i in range(n)], nj.value


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args, rank, world):
    """The reference's CPU raptor (oracle restatement) on all host threads."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from nigiri_b200.timetable import HostTimetable, QuerySet
    h = HostTimetable.generate(WORKLOAD)
    sample = args.cpu_sample or args.batch  # the GPU arm's batch: the same queries, step by step
    threads = host_threads()
    qs = QuerySet(h, WORKLOAD, sample * (args.steps + args.warmup), seed=1000 + WORKLOAD)
    for w in range(args.warmup):
        cpu_run(h.desc, qs.subset(range(w * sample, (w + 1) * sample)), sample, threads)
    total, lats = 0.0, []
    for k in range(args.steps):
        off = (args.warmup + k) * sample
        wall, lat, _ = cpu_run(h.desc, qs.subset(range(off, off + sample)), sample, threads)
        total += wall
        lats += lat
    qps = sample * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded generator)",
        "config": config_block(args, sample),
        "p50_ms": percentile(lats, 0.5), "p99_ms": percentile(lats, 0.99),
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} workload-2 queries per step, one query per thread"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args, batch):
    return {"workload": "regional-40k-stops batched one-to-one (intermodal offset sets)",
            "timetable": "40,009 locations, 4,000 base routes, ~436k transports, 365 days",
            "global_batch": batch, "queries_per_step": batch, "max_transfers": 14,
            "parallelism": f"replicas x{args.gpus}"}


METHOD = {"lower_bounds": "all-pairs tables on the device (built once per timetable, before timing)",
          "l2": "round state of a step (>2.5 GB) exceeds L2; 512 MB written between steps",
          "admission": "continuous: queries enter free slots between super-steps"}


# --------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, local):
    import torch
    from nigiri_b200 import _abi as A
    from nigiri_b200 import replicas
    from nigiri_b200 import routing as R
    from nigiri_b200.timetable import HostTimetable, QuerySet

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        pg = dist
    h = HostTimetable.generate(WORKLOAD)
    dtt = R.Timetable(h.desc, device=local, owner=h)
    B = args.batch
    eng = R.Engine(dtt, max_slots=B)
    n_total = B * (args.warmup + args.steps)
    qs = QuerySet(h, WORKLOAD, n_total, seed=replicas.query_seed(1000 + WORKLOAD, rank))
    lib = A.lib()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def one_batch(off, engine=eng):
        arr = qs.subset(range(off, off + B))
        out = (A.Result * B)()
        t0 = time.perf_counter()
        rc = lib.b2r_search_batch(engine.handle, arr, B, out)
        t1 = time.perf_counter()
        if rc != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        st = engine.stats()
        return t1 - t0, st, out

    # launch shape picked by the autotuner on a separate sample of the
    # workload, on rank 0; every rank then runs rank 0's shape
    fields = [f for f, _ in A.LaunchShape._fields_]
    tune = None
    picked = [0] * len(fields)
    if rank == 0:
        tune_qs = QuerySet(h, WORKLOAD, B, seed=9000 + WORKLOAD)
        tune = eng.autotune(tune_qs.arr, tune_qs.n)
        picked = [getattr(tune.best, f) for f in fields]
    picked = replicas.from_rank0(picked, pg, f"cuda:{local}")
    eng.shape = A.LaunchShape(*picked)
    shape = dict(zip(fields, picked))
    for w in range(args.warmup):
        one_batch(w * B)
    clocks = ClockSampler(local)
    clocks.start()
    walls, devs, lats, launches, h2d, d2h = [], [], [], 0, 0, 0
    kept = {}  # query index -> engine records, checked against the oracle after timing
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
        wall, st, out = one_batch((args.warmup + k) * B)
        torch.cuda.synchronize()
        walls.append(wall)
        devs.append(st.device_ms / 1e3)
        launches += st.kernel_launches
        h2d += st.h2d_bytes
        d2h += st.d2h_bytes
        for i in range(B):
            lats.append(out[i].latency_ms)
        if rank == 0:  # outside the batch's own timing: step 0 whole, 1% of the others
            for i in (range(B) if k == 0 else range(0, B, 100)):
                kept[(args.warmup + k) * B + i] = journey_records(out[i])
    ck = clocks.stop()
    tot_wall, tot_dev = sum(walls), sum(devs)
    tot_wall, tot_dev = replicas.max_over_ranks([tot_wall, tot_dev], pg, f"cuda:{local}")
    n_q = B * args.steps * world
    value = replicas.whole_job_throughput(B * args.steps, world, tot_dev)
    e2e = replicas.whole_job_throughput(B * args.steps, world, tot_wall)
    # bytes the engine copied between host and device (its own count)
    h2d_step = h2d // max(1, args.steps)

    extras = {}
    if rank == 0:
        extras["checked_against_cpu"] = oracle_check(h.desc, qs.arr, kept, host_threads())
        extras["checked_against_cpu"]["sample"] = (
            f"every query of timed step 0 ({B}) and every 100th of the other {args.steps - 1} steps")
    if rank == 0 and not args.no_extras:
        extras.update(extras_legs(args, h, dtt, qs, B, local, shape))
        extras["served"] = served_leg(eng, qs, [5000.0, 15000.0, 25000.0, None], 4096)
        extras["range"] = range_leg(eng, h, 1024, seed=1003)
        del eng
        extras["batch_sweep"] = batch_sweep_leg(dtt, h, shape, (64, 256), local)
        extras["batch_sweep"]["1024"] = {"value": value, "e2e": e2e, "p99_ms": percentile(lats, 0.99),
                                         "unit": "queries/s", "note": "the headline steps"}
        extras["small_city"] = small_city_leg(local)
        if not args.no_national:
            extras["national"] = national_leg(local)
    if rank == 0:
        peak, peak_kind = measured_peak()
        rl = extras.get("roofline")
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_dev / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16",
            "data": "synthetic (seeded generator: timetable seed 2, query seed 1002 + 7919 x rank)",
            "config": config_block(args, B),
            "method": dict(METHOD, launch_shape=shape,
                           autotune={"tried": tune.n_tried, "start_ms": tune.start_ms,
                                     "best_ms": tune.best_ms}),
            "p50_ms": percentile(lats, 0.5), "p99_ms": percentile(lats, 0.99),
            "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": h2d_step,
                    "d2h_bytes_per_step": d2h // max(1, args.steps)},
            "gpu_launches": launches,
            "clocks": ck,
        }
        line.update({k: v for k, v in extras.items()})
        if rl is not None:
            rl["peak"] = peak
            rl["peak_kind"] = peak_kind
            rl["frac"] = rl["achieved"] / peak
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def served_leg(eng, qs, rates, n_per_rate, seed=17, keep_every=0, kept=None, warm=0):
    """Continuous batching: queries arrive as a Poisson stream at each
    offered rate (and all at once for the saturation point) and are
    submitted to the request loop as they arrive; latency is submit ->
    result, measured by the engine.  With keep_every = m, every m-th
    answer is kept in `kept` (query index -> result key) for checking.
    With warm = n, n queries are first run all at once, unmeasured, as a
    server that has been running would have: its pool of page-locked
    one-to-all result buffers is then filled."""
    import random
    from nigiri_b200 import routing as R
    srv = R.Server(eng)
    out = []
    try:
        warm_tickets = [srv.submit_raw(qs.arr[i]) for i in range(min(warm, qs.n))]
        for tk in warm_tickets:
            srv.wait(tk)
        for tk in warm_tickets:
            srv.release(tk)
        for rate in rates:
            rnd = random.Random(seed)
            n = min(n_per_rate(rate) if callable(n_per_rate) else n_per_rate, qs.n)
            gaps = [0.0] * n if rate is None else [rnd.expovariate(rate) for _ in range(n)]
            tickets, t_sub = [], []
            t0 = time.perf_counter()
            due = t0
            for i in range(n):
                due += gaps[i]
                while True:
                    now = time.perf_counter()
                    if now >= due:
                        break
                    if due - now > 2e-4:
                        time.sleep(due - now - 1e-4)
                t_sub.append(time.perf_counter())
                tickets.append(srv.submit_raw(qs.arr[i]))
            lat, t_end = [], t0
            for i, tk in enumerate(tickets):
                r = srv.wait(tk)
                if keep_every and i % keep_every == 0 and kept is not None:
                    kept[i] = result_key(r, eng.tt.n_locations)
                lat.append(r.latency_ms)
                t_end = max(t_end, t_sub[i] + r.latency_ms / 1e3)
                srv.release(tk)
            out.append({"offered_qps": rate if rate is not None else "all at once",
                        "achieved_qps": n / (t_end - t0), "queries": n,
                        "p50_ms": percentile(lat, 0.5), "p95_ms": percentile(lat, 0.95),
                        "p99_ms": percentile(lat, 0.99)})
    finally:
        srv.stop()
    return out


def journey_records(r):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from journeys import records
    return (r.status, records(r))


def oracle_check(desc, qarr, kept, threads):
    """The engine's answers (query index -> (status, journey records)) against
    the CPU oracle's on the same queries: departure, arrival, transfers and
    every leg must be identical.  The oracle runs on host threads (its calls
    release the interpreter lock)."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    oracle_lib.lib()

    def one(i):
        return i, (0, oracle_lib.OracleResult(desc, qarr[i]).records())

    mismatches, first = 0, []
    with ThreadPoolExecutor(max(1, threads)) as ex:
        for i, want in ex.map(one, sorted(kept)):
            if kept[i] != want:
                mismatches += 1
                if len(first) < 5:
                    first.append(i)
    return {"queries": len(kept), "mismatches": mismatches, "first_mismatches": first}


def result_key(r, n_loc):
    """A query's complete answer: journeys with every leg, or one-to-all rows."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from journeys import records
    if r.round_times:
        rows = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n_loc,))
        return ("rows", r.status, r.base_day, rows.tobytes())
    return ("journeys", r.status, records(r))


def range_leg(eng, h, n, seed, reps=2):
    """Range queries (generated range mix: 30..240 min windows, both
    directions, station to station, walking allowed at both ends) run as
    range RAPTOR and as pong on the same engine; queries/s on the device and
    end to end, and the agreement nigiri's benchmark checks between the two
    (the Pareto sets on the intersection of their final search intervals)."""
    from nigiri_b200 import _abi as A
    from nigiri_b200.timetable import QuerySet
    lib = A.lib()
    qs = QuerySet(h, 3, n, seed=seed)
    arrs = {}
    for algo, code in (("range_raptor", A.B2R_ALGO_RAPTOR), ("pong", A.B2R_ALGO_PONG)):
        arr = (A.Query * qs.n)()
        for i in range(qs.n):
            arr[i] = qs.arr[i]
            arr[i].use_start_footpaths = 1
            arr[i].algorithm = code
        arrs[algo] = arr
    out = {"queries": qs.n, "unit": "queries/s"}
    keys, ivs = {}, {}
    for algo, arr in arrs.items():
        res = (A.Result * qs.n)()
        devs, walls = [], []
        for rep in range(reps + 1):
            t0 = time.perf_counter()
            if lib.b2r_search_batch(eng.handle, arr, qs.n, res) != 0:
                raise RuntimeError(lib.b2r_last_error().decode())
            if rep > 0:  # the first run warms up
                walls.append(time.perf_counter() - t0)
                devs.append(eng.stats().device_ms / 1e3)
        st = eng.stats()
        out[algo] = {"value": qs.n * reps / sum(devs), "e2e": qs.n * reps / sum(walls),
                     "super_steps": st.super_steps,
                     "failed": sum(1 for i in range(qs.n) if res[i].status != 0)}
        keys[algo] = [[(r.journeys[j].start_time, r.journeys[j].dest_time, r.journeys[j].transfers)
                       for j in range(r.n_journeys)] for r in res[:qs.n]]
        ivs[algo] = [(r.interval_from, r.interval_to) for r in res[:qs.n]]
    agree = 0
    for i in range(qs.n):
        lo = max(ivs["range_raptor"][i][0], ivs["pong"][i][0])
        hi = min(ivs["range_raptor"][i][1], ivs["pong"][i][1])
        fwd = arrs["pong"][i].direction == A.B2R_FORWARD
        inside = [sorted(t for t in keys[a][i] if lo <= (min(t[0], t[1]) if fwd else max(t[0], t[1])) < hi)
                  for a in ("range_raptor", "pong")]
        agree += 1 if inside[0] == inside[1] else 0
    out["pareto_sets_agree"] = agree
    out["pong_speedup"] = out["pong"]["value"] / out["range_raptor"]["value"]
    return out


def batch_sweep_leg(dtt, h, shape, sizes, local, reps=3):
    """The regional workload in batches of 64 and 256 resident queries (the
    batch sizes the configuration names beside 1,024), each on an engine of
    that many slots with the launch shape tuned at 1,024: device and
    end-to-end queries/s and the per-query latency percentiles."""
    from nigiri_b200 import _abi as A
    from nigiri_b200 import routing as R
    from nigiri_b200.timetable import QuerySet
    lib = A.lib()
    out = {}
    for B in sizes:
        eng = R.Engine(dtt, max_slots=B)
        sh = A.LaunchShape()
        for f, v in shape.items():
            setattr(sh, f, v)
        eng.shape = sh
        qs = QuerySet(h, WORKLOAD, B * (reps + 1), seed=5000 + B)
        res = (A.Result * B)()
        devs, walls, lat = [], [], []
        for k in range(reps + 1):
            arr = qs.subset(range(k * B, (k + 1) * B))
            t0 = time.perf_counter()
            if lib.b2r_search_batch(eng.handle, arr, B, res) != 0:
                raise RuntimeError(lib.b2r_last_error().decode())
            if k > 0:  # the first batch warms up
                walls.append(time.perf_counter() - t0)
                devs.append(eng.stats().device_ms / 1e3)
                lat += [res[i].latency_ms for i in range(B)]
        out[str(B)] = {"value": B * reps / sum(devs), "e2e": B * reps / sum(walls), "unit": "queries/s",
                       "p50_ms": percentile(lat, 0.5), "p99_ms": percentile(lat, 0.99),
                       "queries": B * reps}
        del eng
    return out


def small_city_leg(local):
    """The 1,000-stop city: its 1,000 one-to-one queries batched (one batch),
    one query per launch sequence (plain), and on the CPU oracle (all host
    threads), with every batched answer compared with the oracle's."""
    from nigiri_b200 import _abi as A
    from nigiri_b200 import routing as R
    from nigiri_b200.timetable import HostTimetable, QuerySet
    lib = A.lib()
    h = HostTimetable.generate(1)
    dtt = R.Timetable(h.desc, device=local, owner=h)
    n = 1000
    qs = QuerySet(h, 1, n, seed=1001)
    eng = R.Engine(dtt, max_slots=1024)
    res = (A.Result * n)()
    walls, devs = [], []
    for rep in range(3):
        t0 = time.perf_counter()
        if lib.b2r_search_batch(eng.handle, qs.arr, n, res) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        if rep > 0:
            walls.append(time.perf_counter() - t0)
            devs.append(eng.stats().device_ms / 1e3)
    kept = {i: journey_records(res[i]) for i in range(n)}
    out = {"timetable": f"{h.desc.n_locations:,} locations, {h.desc.n_routes:,} routes",
           "queries": n,
           "batched": {"value": 2 * n / sum(devs), "e2e": 2 * n / sum(walls), "unit": "queries/s"}}
    del eng
    plain = R.Engine(dtt, max_slots=32, use_graphs=False)
    one = A.Result()
    lat = []
    t0 = time.perf_counter()
    for i in range(n):
        a = time.perf_counter()
        if lib.b2r_search_plain(plain.handle, C.byref(qs.arr[i]), C.byref(one)) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        lat.append((time.perf_counter() - a) * 1e3)
    out["plain_gpu"] = {"value": n / (time.perf_counter() - t0), "unit": "queries/s",
                        "p50_ms": percentile(lat, 0.5), "p99_ms": percentile(lat, 0.99)}
    del plain
    threads = host_threads()
    wall, lat, _ = cpu_run(h.desc, qs.arr, n, threads)
    out["cpu_baseline"] = {"value": n / wall, "unit": "queries/s", "cores": threads, "kind": "port",
                           "p99_ms": percentile(lat, 0.99)}
    out["checked_against_cpu"] = oracle_check(h.desc, qs.arr, kept, threads)
    return out


def national_leg(local):
    """National-scale timetable (300k stops, 25k base routes, 2.7M transports,
    stay-seated chain routes).  Batched: batches of 256 mixing one-to-one, 1 h
    range and one-to-all queries, on an engine of 256 slots.  Served: the
    request loop (1,024 slots) fed by Poisson streams of the 70% one-to-one /
    20% 2 h range / 10% one-to-all mix at 100 .. 20,000 q/s.  Plain: one query per launch sequence.  CPU: the
    oracle on all host threads, on the served answers kept for checking (1%),
    which are compared with its results."""
    from nigiri_b200 import _abi as A
    from nigiri_b200 import routing as R
    from nigiri_b200.timetable import HostTimetable, QuerySet
    lib = A.lib()
    h = HostTimetable.generate(4)
    dtt = R.Timetable(h.desc, device=local, owner=h)
    n_loc = h.desc.n_locations
    out = {"timetable": f"{n_loc:,} locations, {h.desc.n_routes:,} routes, "
                        f"{h.desc.n_transports:,} transports, 365 days"}
    # batches of 256 on an engine of 256 slots (the per-location mark words
    # then cover 8 slot groups, not 32)
    B = 256
    eng = R.Engine(dtt, max_slots=B)
    # launch shape picked by the autotuner on a separate sample of the mix
    tune_qs = QuerySet(h, 4, B, seed=9004)
    tune = eng.autotune(tune_qs.arr, tune_qs.n)
    out["launch_shape"] = {f: getattr(tune.best, f) for f, _ in A.LaunchShape._fields_}
    qs = QuerySet(h, 4, B * 4, seed=1004)
    res = (A.Result * B)()
    devs, walls = [], []
    for k in range(4):
        arr = qs.subset(range(k * B, (k + 1) * B))
        t0 = time.perf_counter()
        if lib.b2r_search_batch(eng.handle, arr, B, res) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        if k > 0:  # the first batch warms up
            walls.append(time.perf_counter() - t0)
            devs.append(eng.stats().device_ms / 1e3)
    out["batched"] = {"batch": B, "slots": B, "queries": B * 3, "value": B * 3 / sum(devs),
                      "e2e": B * 3 / sum(walls), "unit": "queries/s",
                      "ms_per_batch": sum(walls) / 3 * 1e3}
    del eng
    # plain: one query per launch sequence (same engine design, per-round launches)
    n_plain = 64
    plain = R.Engine(dtt, max_slots=32, use_graphs=False)
    arr = qs.subset(range(n_plain))
    one = A.Result()
    t0 = time.perf_counter()
    for i in range(n_plain):
        if lib.b2r_search_plain(plain.handle, C.byref(arr[i]), C.byref(one)) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
    out["plain_gpu"] = {"value": n_plain / (time.perf_counter() - t0), "unit": "queries/s", "queries": n_plain}
    del plain
    eng = R.Engine(dtt, max_slots=1024)
    eng.shape = tune.best  # the shape tuned on the mix above
    # served (continuous batching), 1% of the answers kept for the check
    sq = QuerySet(h, 5, 4096, seed=1005)
    kept = {}
    out["served"] = served_leg(eng, sq, [100.0, 1000.0, 5000.0, 20000.0, None],
                               lambda r: 4096 if r is None else max(256, min(4096, int(r))),
                               keep_every=100, kept=kept, warm=4096)
    out["range"] = range_leg(eng, h, 256, seed=1006, reps=1)
    del eng
    # CPU baseline on the kept queries, which also checks their answers
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    idx = sorted(kept)
    threads = host_threads()
    wall, lat, _ = cpu_run(h.desc, sq.subset(idx), len(idx), threads)
    out["cpu_baseline"] = {"value": len(idx) / wall, "unit": "queries/s", "cores": threads,
                           "kind": "port", "sample": f"{len(idx)} served queries (1%)"}
    mismatches = 0
    for i in idx:
        q = sq.arr[i]
        o = oracle_lib.OracleResult(h.desc, q)
        if q.kind == A.B2R_ONE_TO_ALL:
            rows, _, base_day = o.state()
            n_rows = len(kept[i][3]) // (2 * n_loc)
            want = ("rows", 0, base_day, rows[:n_rows].tobytes())
        else:
            want = ("journeys", 0, o.records())
        mismatches += 0 if kept[i] == want else 1
    out["checked_against_cpu"] = {"queries": len(idx), "mismatches": mismatches}
    return out


def extras_legs(args, h, dtt, qs, B, local, shape):
    """Plain one-query-per-launch baseline, route-scan roofline and the CPU
    baseline (rank 0, outside the timed region)."""
    import torch
    from nigiri_b200 import _abi as A
    from nigiri_b200 import routing as R
    lib = A.lib()
    out = {}
    # plain engine: one query per pass, per-round launches, sync per round
    plain = R.Engine(dtt, max_slots=32, use_graphs=False)
    n_plain = 64
    arr = qs.subset(range(n_plain))
    res = A.Result()
    lat = []
    t0 = time.perf_counter()
    for i in range(n_plain):
        a = time.perf_counter()
        if lib.b2r_search_plain(plain.handle, C.byref(arr[i]), C.byref(res)) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        lat.append((time.perf_counter() - a) * 1e3)
    t1 = time.perf_counter()
    out["plain_gpu"] = {"value": n_plain / (t1 - t0), "unit": "queries/s",
                        "p50_ms": percentile(lat, 0.5), "p99_ms": percentile(lat, 0.99),
                        "queries": n_plain}
    del plain
    # roofline of the route scan: the algorithmic bytes come from a counting
    # build (profile = 1), the launch times from CUDA events around every
    # launch of the build the bench runs (profile = 2, the tuned shape); both
    # run the step-0 batch without graphs
    sh = A.LaunchShape()
    for f, v in shape.items():
        setattr(sh, f, v)
    arr = qs.subset(range(B))
    o = (A.Result * B)()
    runs = {}
    for mode in (1, 2):
        prof = R.Engine(dtt, max_slots=B, profile=mode)
        prof.shape = sh
        if lib.b2r_search_batch(prof.handle, arr, B, o) != 0:
            raise RuntimeError(lib.b2r_last_error().decode())
        runs[mode] = prof.stats()
        del prof
    st, tm = runs[1], runs[2]
    per_launch_bytes = st.route_scan_bytes / max(1, st.route_scan_launches)
    per_launch_s = tm.route_scan_ms / 1e3 / max(1, tm.route_scan_launches)
    traffic, cap = None, ncu_traffic_per_unit()
    # the capture's batch and route-scan build (the grid shape changes no
    # DRAM traffic of the work, the build's spills could)
    if cap is not None and cap.get("batch") == B and cap.get("shape", [None] * 6)[5] == sh.scan_occupancy:
        traffic = cap["dram_bytes_per_launch"]
    out["roofline"] = {
        "bound": "hbm", "achieved": per_launch_bytes / per_launch_s / 1e9, "peak": None,
        "unit": "GB/s", "frac": None, "traffic": traffic,
        "traffic_source": None if traffic is None else cap.get("command"),
        "limiter": "instruction issue and dependent L2 loads, not DRAM (ncu at batch 256: issue "
                   "active 60%, SM throughput 55%, L2 hit 80%, DRAM throughput 5%, 19 of 32 "
                   "threads per instruction)",
        "kernel": "k_route_scan", "launches": tm.route_scan_launches,
        "avg_launch_ms": per_launch_s * 1e3, "algorithmic_bytes_per_launch": per_launch_bytes,
        "route_stop_visits": st.route_stop_visits, "et_events": st.et_events, "et_days": st.et_days,
        "label_writes": st.label_writes,
        "lane_utilisation": st.route_stop_visits / max(1, 32 * st.route_warp_steps),
        "route_scan_share_of_device_time": tm.route_scan_ms / max(1e-9, tm.device_ms),
        "ncu": None if cap is None else cap.get("ncu"),
        # L2 throughput of the same kernel as a fraction of its peak (ncu,
        # detailed capture at batch 256): the level that serves its loads
        "l2_frac": (None if cap is None or not cap.get("ncu")
                    else cap["ncu"]["l2_throughput_pct"] / 100.0),
    }
    # CPU baseline: the oracle on a bounded sample, all host threads
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    threads = host_threads()
    sample = args.cpu_sample or min(B, 512)
    wall, lat, _ = cpu_run(h.desc, qs.subset(range(sample)), sample, threads)
    out["cpu_baseline"] = {"value": sample / wall, "unit": "queries/s", "cores": threads,
                           "kind": "port", "sample": f"{sample} queries of the step-0 batch",
                           "p99_ms": percentile(lat, 0.99)}
    wall1, lat1, _ = cpu_run(h.desc, qs.subset(range(64)), 64, 1)
    out["cpu_baseline_1thread"] = {"value": 64 / wall1, "unit": "queries/s", "cores": 1,
                                   "kind": "port", "sample": "64 queries of the step-0 batch",
                                   "p50_ms": percentile(lat1, 0.5), "p99_ms": percentile(lat1, 0.99)}
    return out


def ncu_case(args, local):
    """One batch of `--batch` queries of workload `--ncu-workload` (2: the
    regional one-to-one batch, 4: the national mix) on an engine of that many
    slots, kernels launched one by one (no graph) so that a profiler sees
    every launch."""
    from nigiri_b200 import _abi as A
    from nigiri_b200 import routing as R
    from nigiri_b200.timetable import HostTimetable, QuerySet
    h = HostTimetable.generate(args.ncu_workload)
    dtt = R.Timetable(h.desc, device=local, owner=h)
    eng = R.Engine(dtt, max_slots=args.batch, use_graphs=False, profile=args.ncu_counters)
    if args.shape:
        eng.shape = A.LaunchShape(*[int(x) for x in args.shape.split(",")])
    qs = QuerySet(h, args.ncu_workload, args.batch, seed=1000 + args.ncu_workload)
    out = (A.Result * args.batch)()
    rc = A.lib().b2r_search_batch(eng.handle, qs.arr, args.batch, out)
    if rc != 0:
        raise RuntimeError(A.lib().b2r_last_error().decode())
    st = eng.stats()
    sh = eng.shape
    print(json.dumps({"ncu_case": True, "batch": args.batch, "super_steps": st.super_steps,
                      "shape": [sh.scan_blocks_per_sm, sh.scan_threads, sh.pair_blocks_per_sm,
                                sh.recon_blocks_per_sm, sh.steps_per_sync, sh.scan_occupancy],
                      "kernel_launches": st.kernel_launches, "device_ms": st.device_ms,
                      "route_scan_launches": st.route_scan_launches,
                      "route_stop_visits": st.route_stop_visits,
                      "route_warp_steps": st.route_warp_steps,
                      "route_scan_ms": st.route_scan_ms, "recon_ms": st.recon_ms,
                      "recon_max_journey_us": st.recon_max_journey_us,
                      "recon_journeys": st.recon_journeys,
                      "route_scan_bytes": st.route_scan_bytes}))


def ncu_summary(path):
    """Per-kernel table of an ncu --csv log: launches, total and mean
    gpu__time_duration, share of the total, and the per-launch mean of every
    other metric captured (DRAM bytes and the like)."""
    import csv
    scale = {"ns": 1e-6, "nsecond": 1e-6, "us": 1e-3, "usecond": 1e-3, "ms": 1.0, "msecond": 1.0,
             "s": 1e3, "second": 1e3}
    bytes_scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}
    with open(path, newline="") as f:
        lines = [ln for ln in f if ln.startswith('"')]  # ncu's own log lines are not quoted
    per = {}
    for row in csv.DictReader(lines):
        name = row["Kernel Name"].split("(")[0]
        k = per.setdefault(name, {"launches": set(), "ms": 0.0, "other": {}})
        k["launches"].add(row["ID"])
        metric, unit = row["Metric Name"], row["Metric Unit"]
        val = float(row["Metric Value"].replace(",", ""))
        if metric == "gpu__time_duration.sum":
            k["ms"] += val * scale.get(unit, 1e-6)
        else:
            k["other"].setdefault(metric, 0.0)
            k["other"][metric] += val * bytes_scale.get(unit, 1)
    total = sum(k["ms"] for k in per.values())
    n_launch = sum(len(k["launches"]) for k in per.values())
    print(f"total {total:.3f} ms over {n_launch} launches")
    metrics = sorted({m for k in per.values() for m in k["other"]})
    head = f"{'kernel':<24} {'launches':>8} {'total ms':>9} {'share':>7} {'mean us':>9}"
    print(head + "".join(f" {m + ' / launch':>34}" for m in metrics))
    for name, k in sorted(per.items(), key=lambda x: -x[1]["ms"]):
        n = len(k["launches"])
        line = (f"{name:<24} {n:>8} {k['ms']:>9.3f} {100 * k['ms'] / max(total, 1e-12):>6.2f}% "
                f"{1e3 * k['ms'] / max(n, 1):>9.1f}")
        print(line + "".join(f" {k['other'].get(m, 0.0) / max(n, 1):>34,.0f}" for m in metrics))


def main():
    args = parse()
    if args.ncu_summary:
        ncu_summary(args.ncu_summary)
        return
    rank, world, local = dist_env()
    if args.ncu_case:
        ncu_case(args, local)
        return
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        gpu_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
