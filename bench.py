#!/usr/bin/env python3
"""Benchmark of the plain BN254 G1 MSM at N = 2^22 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload uniform|skewed] [--log-n 22]

A step is one msm_execute_async over 2^22 points: uniform Montgomery-form
scalars (seed 1) against resident bases k_i * G (k_i from seed 1, generated on
the device).  `value` times K steps with device-resident inputs (bases
256 MiB + scalars 128 MiB, larger than the 126 MB L2, so no flush is needed);
`e2e` times K steps through the same C ABI with the scalars in pinned host
memory and the 254 results written to pinned host memory, copies included.

Two more objects on the same line (rank 0, one GPU):
  "batched"  the uneven 64-instance batch (lengths log-uniform in [2^10, 2^22],
             seed 3, over one resident 2^22-point table): one execution of the
             batched graph against 64 sequential plain calls; for the reference,
             64 zero-padded msm_execute_async calls (--no-batched skips it);
  "serving"  Poisson arrivals of requests with sizes log-uniform in [2^12, 2^23]
             over a resident 2^23-point table and a 16 GiB scratch budget: the
             request server (continuous batching) against a plain loop running
             one request per call, p50/p99 latency and Mpoints/s at rates of 0.6,
             0.9 and 1.2 times the plain loop's capacity (--serving-requests sets
             the requests per rate, 200 by default, 10000 for the full config;
             --no-serving skips it).

--impl reference runs the reference era-bellman-cuda msm_execute_async built
for sm_100a from its own sources (oracle/_ref/libbellman-cuda-ref.so) on the
same inputs; that is the reference implementation of this path (a CUDA
library: it has no CPU implementation of the MSM).

Multi-GPU: one process per GPU (torchrun); the MSM does not shard in the
reference's API, so every rank runs an independent replica (weak scaling) and
the job value is N * 2^22 points over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "era-bellman-cuda_b200"))

METRIC = "BN254 MSM Mpoints/s at 2^22 and batched p50/p99 vs plain per-call; bit-exact"
REF_LIB = os.path.join(REPO, "oracle", "_ref", "libbellman-cuda-ref.so")
MEASURED_PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
MADD_MULOPS = 2392  # 6 mul (264) + 2 sqr (208) + one a*b - c*d (392) per XYZZ += affine
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one accumulate_kernel launch per
# nonzero entry it processes, from the ncu --set full capture of the 2^21 uniform case at
# c = 17 (2.678 GB over 31.46 M entries); a launch's traffic grows with the entries it gathers.
ACC_DRAM_BYTES_PER_ENTRY = 85.1


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["uniform", "skewed"], default="uniform")
    ap.add_argument("--log-n", type=int, default=22)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-instance batch")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving run")
    ap.add_argument("--serving-requests", type=int, default=200, help="requests per rate (the full config: 10000)")
    ap.add_argument("--batched-only", action="store_true",
                    help="profiling aid: run only the batched section (--steps executions) and print its object")
    ap.add_argument("--batched-scale", type=int, default=1, help="with --batched-only: divide every instance length by this")
    return ap.parse_args()


class Dist:
    """Rank bookkeeping; a gloo group only for the barrier and the max of times."""

    def __init__(self, n):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
            self.pg = dist
        if n != self.world and self.world > 1:
            print(f"warning: --gpus {n} but WORLD_SIZE {self.world}", file=sys.stderr)

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"bench_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        return float(json.load(open(MEASURED_PEAKS))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def make_inputs(bc, workload: str, n: int, stream):
    """Scalars (host, Montgomery form) and device-resident bases k_i * G."""
    import synth
    seed = 1 if workload == "uniform" else 2
    scalars, k = synth.workload(workload, n, seed)
    kd = bc.to_device(k)
    bd = bc.malloc(n * 64)
    bc.generator_multiples(kd, bd, n, stream)
    bc.stream_synchronize(stream)
    bc.free(kd)
    return scalars, bd, seed


def time_steps(bc, stream, k: int, enqueue) -> float:
    """ms per step of k enqueued steps, CUDA events on the launching stream."""
    e0, e1 = bc.event_create(), bc.event_create()
    bc.stream_synchronize(stream)
    bc.event_record(e0, stream)
    for _ in range(k):
        enqueue()
    bc.event_record(e1, stream)
    bc.event_synchronize(e1)
    ms = bc.elapsed_ms(e0, e1) / k
    bc.event_destroy(e0)
    bc.event_destroy(e1)
    return ms


def cpu_baseline(bc, scalars_all: np.ndarray, bases_dev: int, results_dev: int, target_s: float = 6.0):
    """Multithreaded host Pippenger (the CPU oracle) on a bounded prefix of the
    workload; also the caller-side Horner pass over this run's 254 results on
    one host core, the CPU counterpart of msm_b200_final_sum_async."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    o = orc.Oracle()
    results = bc.from_device(results_dev, (254, 24))
    horner_s = []
    for _ in range(5):
        t0 = time.perf_counter()
        o.horner(results)
        horner_s.append(time.perf_counter() - t0)
    cores = os.cpu_count() or 1
    n = 1 << 14
    best = None
    while True:
        bases = bc.from_device(bases_dev, (n, 16))
        secs, _ = orc.time_cpu_pippenger(o, bases, np.ascontiguousarray(scalars_all[:n]), cores)
        best = (n, secs)
        if secs * 2.5 > target_s or n >= len(scalars_all):
            break
        n <<= 1
    n, secs = best
    return {"value": n / secs / 1e6, "unit": "Mpoints/s", "cores": cores, "kind": "port",
            "sample": f"host Pippenger (oracle/bn254_oracle.c, {cores} threads) over the first 2^{n.bit_length() - 1} points of the same "
                      f"workload, {secs:.2f} s wall",
            "host_horner_ms": round(1e3 * statistics.median(horner_s), 4)}


def generated_table(bc, seed: int, n: int, stream) -> int:
    """n bases k_i * G (k_i from `seed`) generated on the device; returns the device pointer."""
    import synth
    kd = bc.to_device(synth.base_multipliers(seed, n))
    bd = bc.malloc(n * 64)
    bc.generator_multiples(kd, bd, n, stream)
    bc.stream_synchronize(stream)
    bc.free(kd)
    return bd


def batched_section(ours, bc, pool, stream, steps: int, warmup: int, scale: int = 1) -> dict:
    """The uneven 64-instance batch (lengths log-uniform in [2^10, 2^22], seed 3;
    even instances uniform, odd ones skewed; prefixes of one resident 2^22-point
    table): one execution of the batched graph against 64 sequential plain calls
    (for the reference: 64 calls padded with zero scalars to powers of two)."""
    import synth
    lengths = [max(1, int(x) // scale) for x in synth.batch_lengths(3, 64)]
    n_table = (1 << 22) // scale
    table_dev = generated_table(ours, 3, n_table, stream)
    work = [s for _, s in synth.batch_workload(3, lengths)]
    points = sum(lengths)
    out = {"workload": "64 MSMs, lengths log-uniform in [2^10, 2^22] (seed 3), even instances uniform scalars, odd ones the skewed mix, "
                       "prefixes of one resident 2^22-point base table", "instances": 64, "points": points}
    if bc is ours:
        table = bc.base_table_create(table_dev, n_table, stream)
        sd = [bc.to_device(w) for w in work]
        rd = [bc.malloc(254 * 96) for _ in lengths]
        batch = bc.batch_create(table, lengths)
        scratch, kernels, entries = bc.batch_info(batch)
        for _ in range(warmup):
            bc.batch_execute(batch, sd, rd, stream)
        ms = time_steps(bc, stream, steps, lambda: bc.batch_execute(batch, sd, rd, stream))

        def plain():
            for n, s_, r in zip(lengths, sd, rd):
                bc.check(bc.msm_any(pool, stream, table_dev, s_, r, n), "msm_b200_execute_async")

        for _ in range(warmup):
            plain()
        ms_plain = time_steps(bc, stream, steps, plain)
        out.update({"value": round(points / ms / 1e3, 2), "unit": "Mpoints/s", "ms": round(ms, 3),
                    "plain_per_call": {"value": round(points / ms_plain / 1e3, 2), "ms": round(ms_plain, 3)},
                    "speedup_vs_plain_per_call": round(ms_plain / ms, 3), "graph_kernels": kernels, "entries": entries,
                    "scratch_gib": round(scratch / 2**30, 2), "table_gib": round(bc.base_table_bytes(table) / 2**30, 2)})
        bc.batch_destroy(batch)
        bc.base_table_destroy(table)
        for p_ in sd + rd:
            bc.free(p_)
    else:  # the reference: one call per instance, zero-padded to the next power of two
        bases = bc.to_device(ours.from_device(table_dev, (n_table, 16)))
        padded = []
        for w in work:
            logn = max(0, (len(w) - 1).bit_length())
            full = np.zeros((1 << logn, 8), np.uint32)
            full[: len(w)] = w
            padded.append((logn, bc.to_device(full)))
        rd = bc.malloc(254 * 96)

        def plain():
            for logn, s_ in padded:
                bc.msm(pool, stream, bases, s_, rd, logn)

        for _ in range(warmup):
            plain()
        ms_plain = time_steps(bc, stream, steps, plain)
        out.update({"plain_per_call": {"value": round(points / ms_plain / 1e3, 2), "ms": round(ms_plain, 3),
                                       "note": "64 reference msm_execute_async calls, each zero-padded to a power of two"}})
        for _, p_ in padded:
            bc.free(p_)
        bc.free(rd)
        bc.free(bases)
    ours.free(table_dev)
    return out


def serving_section(bc, pool, stream, requests: int, rates_rel=(0.6, 0.9, 1.2)) -> dict:
    """Config 4 (reduced to `requests` requests unless asked for 10,000): Poisson
    arrivals (seed 4), sizes log-uniform in [2^12, 2^23], scalars half uniform and
    half skewed (device-resident slices of two 2^23-point pools), over a resident
    2^23-point table with a 16 GiB scratch budget.  The server (continuous
    batching) against a plain loop that runs one request per call in arrival
    order; rates are multiples of the plain loop's measured capacity."""
    import threading
    import synth
    n_table = 1 << 23
    table_dev = generated_table(bc, 4, n_table, stream)
    table = bc.base_table_create(table_dev, n_table, stream)
    pools = {"uniform": bc.to_device(synth.uniform_scalars(40, n_table)), "skewed": bc.to_device(synth.skewed_scalars(41, n_table))}
    rng = np.random.Generator(np.random.PCG64(np.random.SeedSequence([4, 5])))
    sizes = np.rint(np.exp2(rng.uniform(12, 23, requests))).astype(np.int64)
    offsets = [int(rng.integers(0, n_table - n + 1)) for n in sizes]
    dists = ["uniform" if j % 2 == 0 else "skewed" for j in range(requests)]
    src = [pools[d] + 32 * off for d, off in zip(dists, offsets)]
    results = [bc.malloc(254 * 96) for _ in range(requests)]
    points = int(sizes.sum())

    # plain capacity: back-to-back calls, no arrivals
    for j in range(min(8, requests)):
        bc.msm_any(pool, stream, table_dev, src[j], results[j], int(sizes[j]))
    bc.stream_synchronize(stream)
    t0 = time.perf_counter()
    for j in range(requests):
        bc.msm_any(pool, stream, table_dev, src[j], results[j], int(sizes[j]))
    bc.stream_synchronize(stream)
    capacity = requests / (time.perf_counter() - t0)

    def pct(lat):
        return {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3)}

    out = {"workload": f"{requests} requests, Poisson arrivals (seed 4), sizes log-uniform in [2^12, 2^23], half uniform / half skewed "
                       "scalars, resident 2^23-point table, 16 GiB scratch budget",
           "requests": requests, "points": points, "plain_capacity_rps": round(capacity, 1), "rates": []}
    server = bc.server_create(table, 16 << 30, streams=4, max_group=16)
    for rel in rates_rel:
        rate = rel * capacity
        gaps = np.random.Generator(np.random.PCG64(np.random.SeedSequence([4, int(rel * 1000)]))).exponential(1.0 / rate, requests)
        # plain loop: one call per request, in arrival order
        lat = np.zeros(requests)
        start = time.perf_counter() + 0.01
        arrival = start + np.cumsum(gaps)
        for j in range(requests):
            while time.perf_counter() < arrival[j]:
                pass
            bc.msm_any(pool, stream, table_dev, src[j], results[j], int(sizes[j]))
            bc.stream_synchronize(stream)
            lat[j] = (time.perf_counter() - arrival[j]) * 1e3
        plain_span = time.perf_counter() - start
        # server: a producer submits at the arrival times, this thread waits in order
        tickets = [None] * requests
        start = time.perf_counter() + 0.01
        arrival = start + np.cumsum(gaps)

        def producer():
            for j in range(requests):
                while time.perf_counter() < arrival[j]:
                    pass
                tickets[j] = bc.server_submit(server, src[j], int(sizes[j]), results[j])

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        slat, first, last = np.zeros(requests), None, 0.0
        groups = []
        for j in range(requests):
            rc, times = bc.server_wait(server, tickets[j])
            bc.check(rc, "msm_b200_server_wait")
            slat[j] = (times.done_us - times.submit_us) / 1e3
            first = times.submit_us if first is None else min(first, times.submit_us)
            last = max(last, times.done_us)
            groups.append(times.group_size)
        server_span = (last - first) / 1e6
        out["rates"].append({"rate_rps": round(rate, 1), "rate_vs_plain_capacity": rel,
                             "server": {"mpoints_s": round(points / server_span / 1e6, 2), **pct(slat), "mean_group": round(float(np.mean(groups)), 2)},
                             "plain": {"mpoints_s": round(points / plain_span / 1e6, 2), **pct(lat)}})
    stats = bc.server_stats(server)
    out["server_groups"] = stats.groups
    out["max_inflight_groups"] = stats.max_inflight_groups
    bc.server_destroy(server)
    for p_ in results + list(pools.values()):
        bc.free(p_)
    bc.base_table_destroy(table)
    bc.free(table_dev)
    return out


def main():
    args = parse()
    dist = Dist(args.gpus)
    import bellman_cuda as bcm

    n = 1 << args.log_n
    if args.impl == "reference" and not os.path.exists(REF_LIB):
        if dist.rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "reference sm_100a build oracle/_ref/libbellman-cuda-ref.so absent "
                                                                  "(build it with `make -C oracle ref` where the reference tree exists)"}))
        dist.close()
        return
    ours = bcm.BellmanCuda()  # generates the inputs in both arms
    ours.set_device(dist.local)
    if args.batched_only:
        ours.msm_set_up()
        pool, stream = ours.mem_pool_create(dist.local), ours.stream_create(True)
        print(json.dumps(batched_section(ours, ours, pool, stream, args.steps, max(args.warmup, 3), args.batched_scale)))
        dist.close()
        return
    bc = ours if args.impl == "b200" else bcm.BellmanCuda(REF_LIB)
    bc.set_device(dist.local)
    bc.ff_set_up(25, 14)
    bc.msm_set_up()
    pool = bc.mem_pool_create(dist.local)
    stream = bc.stream_create(True)
    gen_stream = ours.stream_create(True)
    scalars, bases_dev_ours, seed = make_inputs(ours, args.workload, n, gen_stream)
    if bc is ours:
        bases_dev = bases_dev_ours
    else:  # hand the reference its own copy, through its own allocator
        host_bases = ours.from_device(bases_dev_ours, (n, 16))
        bases_dev = bc.to_device(host_bases)
    scalars_dev = bc.to_device(scalars)
    results_dev = bc.malloc(254 * 96)

    def step_device():
        bc.msm(pool, stream, bases_dev, scalars_dev, results_dev, args.log_n)

    for _ in range(max(args.warmup, 3)):
        step_device()
    bc.stream_synchronize(stream)

    # ---- device-resident throughput (value) ----------------------------------
    clocks = ClockSampler(dist.local)
    dist.barrier()
    clocks.start()
    ms_local = time_steps(bc, stream, args.steps, step_device)
    clock_info = clocks.stop()
    ms = dist.max(ms_local)
    value = dist.world * n / (ms * 1e-3) / 1e6

    # ---- end to end: pinned host scalars in, pinned host results out ---------
    host_scalars, hs_ptr = bc.pinned_array(scalars.shape)
    host_scalars[...] = scalars
    host_results, hr_ptr = bc.pinned_array((254, 24))

    def step_e2e():
        bc.msm(pool, stream, bases_dev, hs_ptr, hr_ptr, args.log_n)

    for _ in range(2):
        step_e2e()
    dist.barrier()
    e2e_ms = dist.max(time_steps(bc, stream, args.steps, step_e2e))
    e2e_value = dist.world * n / (e2e_ms * 1e-3) / 1e6

    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Mpoints/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": round(ms, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic",
        "config": {
            "workload": f"plain single MSM, N=2^{args.log_n}, {args.workload} Montgomery-form scalars (seed {seed}), "
                        f"resident bases k_i*G (k_i seed {seed}), device-resident inputs and results",
            "n": n,
            "l2": "no flush: inputs larger than L2 (bases 256 MiB + scalars 128 MiB per step)",
            "parallelism": f"replicas x{dist.world}",
        },
        "e2e": {"value": round(e2e_value, 3), "unit": "Mpoints/s", "ms_per_step": round(e2e_ms, 4),
                "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": 254 * 96},
    }
    if clock_info:
        line["clocks"] = clock_info

    if args.impl == "reference":
        line["impl"] = "reference"
        line["cpu_baseline"] = {"value": line["value"], "unit": "Mpoints/s", "cores": 0, "kind": "reference",
                                "sample": "not a CPU run: the reference's msm_execute_async built for sm_100a from its sources, on this GPU"}
        line["e2e"]["h2d_bytes_per_step"] = n * 32
    else:
        line["impl"] = "b200"
        # ---- stage times over K more steps (events recorded by the library) ----
        events = [[bc.event_create() for _ in range(7)] for _ in range(args.steps)]
        stage_ms = np.zeros(6)
        launches = 0
        bc.stream_synchronize(stream)
        for s in range(args.steps):
            launches = bc.msm_staged(pool, stream, bases_dev, scalars_dev, results_dev, n, events[s])
        bc.stream_synchronize(stream)
        for s in range(args.steps):
            stage_ms += [bc.elapsed_ms(events[s][i], events[s][i + 1]) for i in range(6)]
            for ev in events[s]:
                bc.event_destroy(ev)
        stage_ms /= args.steps
        prof = bc.msm_profiled(pool, stream, bases_dev, scalars_dev, results_dev, n)
        # pipe peak: the better of independent mad.lo and paired lo/hi carry chains
        peak = max(bc.mul_throughput(4), bc.mul_throughput(1))
        montmul_rate = bc.mul_throughput(2)
        madd_rate = bc.mul_throughput(3)
        acc_s = stage_ms[3] * 1e-3
        achieved = prof.madds * MADD_MULOPS / acc_s
        line["gpu_launches"] = launches * args.steps
        line["config"]["window_bits"] = prof.window_bits
        line["config"]["windows"] = prof.windows
        line["stages_ms"] = {name: round(float(v), 4) for name, v in zip(bcm.MsmB200Profile.STAGES, stage_ms)}
        line["roofline"] = {
            "bound": "imad",
            "kernel": "accumulate_kernel",
            "achieved": round(achieved / 1e12, 3),
            "peak": round(peak / 1e12, 3),
            "unit": "T mul-instr/s",
            "frac": round(achieved / peak, 4),
            "traffic": round(ACC_DRAM_BYTES_PER_ENTRY * prof.nonzero_entries),
            "traffic_source": "ncu capture at 2^21 (dram__bytes_read.sum + dram__bytes_write.sum per launch), scaled by the nonzero "
                              "entries of this launch",
            "work": f"{prof.madds} XYZZ+affine additions x {MADD_MULOPS} 32-bit multiply instructions",
            "peak_source": "measured in this run: max of msm_b200_measure_mul_throughput kinds 4 (independent mad.lo) and 1 (paired "
                           "mad.lo.cc/madc.hi.cc chains), i.e. ~64 multiply instructions per clock per SM",
            "probe_montmul_frac": round(montmul_rate / peak, 4),
            "probe_madd_frac": round(madd_rate / peak, 4),
        }
        hbm, hbm_src = hbm_peak()
        sort_bytes = (n * 32 + prof.windows * n * 8) + 2 * (prof.windows * n * 20)
        sort_s = (stage_ms[0] + stage_ms[1]) * 1e-3
        line["roofline_hbm"] = {"kernels": "digits + sort", "achieved": round(sort_bytes / sort_s / 1e9, 1), "peak": hbm, "unit": "GB/s",
                                "frac": round(sort_bytes / sort_s / 1e9 / hbm, 4), "peak_source": hbm_src,
                                "bytes": "32 B scalar + 8 B/entry digit write; 20 B/entry per radix pass (4 histogram + 8 read + 8 write)"}
        # ---- the optional on-device final reduction of the 254 results ---------
        point_dev = bc.malloc(80)  # sizeof(msm_b200_affine_point)

        def step_final_sum():
            bc.check(bc.final_sum_async(results_dev, point_dev, stream), "msm_b200_final_sum_async")

        step_final_sum()
        line["final_sum"] = {"ms": round(time_steps(bc, stream, args.steps, step_final_sum), 4),
                             "what": "msm_b200_final_sum_async: sum 2^i R_i of the 254 results as one canonical affine point, on "
                                     "the device (one block; latency-bound: 255 dependent doublings, 8 additions, one inversion)"}
        bc.free(point_dev)
        if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(bc, scalars, bases_dev, results_dev)
    if dist.rank == 0 and dist.world == 1 and not args.no_batched:
        line["batched"] = batched_section(ours, bc, pool, stream, max(3, args.steps // 2), 2)
    if dist.rank == 0 and dist.world == 1 and not args.no_serving and args.impl == "b200":
        line["serving"] = serving_section(bc, pool, stream, args.serving_requests)
    if dist.rank == 0:
        print(json.dumps(line))
    for p in (scalars_dev, results_dev, bases_dev):
        bc.free(p)
    if bc is not ours:
        ours.free(bases_dev_ours)
    bc.free_host(hs_ptr)
    bc.free_host(hr_ptr)
    dist.close()


if __name__ == "__main__":
    main()
