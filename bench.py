#!/usr/bin/env python
"""Swap-evaluation throughput of the SRO-targeted swap search on B200.

Workload (default): the plain GPU configuration -- BCC 20x20x20 (16000 sites,
8/6/12 shells), 5 species x 3200 atoms, seeded synthetic target alpha
(U(-0.15, 0.15), zero row sums), weights [4, 1, 0.5], 256 solutions x 512
tasks, 50 iterations, converge depth 20.  One step = one whole search
(pyhea/cpp/accelerate.cu:1112-1242 semantics) with a fresh seed.

  value  swap evaluations per second over the K timed steps, device time (CUDA
         events on the search's stream), inputs resident; summed over ranks and
         divided by the slowest rank's time
  e2e    the same metric through the C ABI with host buffers
         (hea_run_local_parallel_hcs): neighbour table and inputs copied from
         pinned memory and the population read back inside the timed region
  roofline  the local-search kernel: algorithmic bytes (2 sum Z (4 B id + 1 B
         species) + 2 B per evaluation) over its CUDA-event time, against the
         measured HBM copy bandwidth
  cpu_baseline  the reference CPU engine (oracle/_ref) on a bounded sample

--impl reference times the reference CPU engine alone (rank 0) on the same
workload and prints the same line with "impl": "reference".
Multi-GPU: replicas -- every rank searches its own copy of the workload with
its own seeds; no collective on the data path.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per swap evaluation of the dominant
# kernel, from one ncu capture each, reported per launch as roofline.traffic, scaled by the
# evaluations of the bench's launches: mc_kernel on the plain GPU workload, 164.5 MB over its first
# local-search launch of 203.7 M evaluations (python -m pyhea_b200.cases plain --iters 1);
# batch_kernel on the 64-structure batch, 152.5 GB over a launch of 631.3 M evaluations
# (python -m pyhea_b200.cases batch --count 64 --iters 1).
DRAM_BYTES_PER_EVAL = {"plain_gpu": 164.5e6 / 203.7e6, "batched": 152.467e9 / 631.335e6}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["plain_gpu", "plain_cpu", "batched", "large", "serving"],
                    default="plain_gpu")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="serving: Poisson arrival rate, requests/s")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving: arrival window, seconds")
    ap.add_argument("--slice-ms", type=float, default=40.0,
                    help="serving: time slice of one server step (measured at 200 req/s: 40 ms best p99 of 2-80)")
    ap.add_argument("--large-rounds", type=int, default=4000,
                    help="large workload: cap on rounds per local search (the uncapped search runs for hours)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=0, help="reference processes (0: all host cores)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def workload(name):
    from pyhea_b200 import workloads as W

    return W.plain_gpu(seed=0) if name == "plain_gpu" else W.plain_cpu(seed=0)


def config_of(st, name):
    return {"workload": f"{name}: {st.name}", "lattice": "FCC" if st.lattice == 0 else "BCC", "cell": st.cell,
            "sites": st.num_sites, "species": [int(x) for x in st.species],
            "shells": [len(v) for v in st.shell_sizes()][: len(st.weight)], "weights": [float(w) for w in st.weight],
            "solutions": st.P, "parallel_task": st.Q, "total_iter": st.I, "converge_depth": st.D,
            "l2": "flushed between timed steps (256 MiB write)", "step": "one whole search, fresh seed"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower().startswith("active")})
        loaded = [r[0] for r in rows if r[0] > 0.5 * r[1]] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def cpu_reference_sample(st, nbor, sizes, procs, nnet_per_proc=5, step=1):
    from oracle.ref_timing import RefPool, available

    if not available():
        return None
    pool = RefPool(procs)
    try:
        r = pool.sample(nbor, sizes[: len(st.weight)], st.species, st.weight, st.target, nnet_per_proc, step, st.Q,
                        st.D)
    finally:
        pool.close()
    r["procs"] = procs
    r["sample"] = (f"{procs} processes x {nnet_per_proc} solutions x {step} iteration(s) of the same structure, "
                   f"task={st.Q}, depth={st.D}; evaluations counted exactly (calls of the engine's incremental fitness)")
    return r


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in ("large", "serving"):
        why = {"large": "one local search of the reference CPU engine on 4,000,000 sites does not end within the "
                        "bench's time bound (every proposal copies the whole occupancy, accelerate.cpp:648)",
               "serving": "the reference has no serving form; its per-structure CPU rate is the plain and "
                          "batched reference lines"}[args.workload]
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    from pyhea_b200 import workloads as W

    structs = W.batched(seed=0) if args.workload == "batched" else [workload(args.workload)]
    procs = args.cpu_procs or host_cores()
    from oracle.ref_timing import RefPool, available

    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_accelerate.so was not built"}))
        return 0
    pool = RefPool(procs)
    nnet = max(1, 2)
    total_evals, total_s = 0.0, 0.0
    try:
        for i in range(args.warmup + args.steps):
            st = structs[(7 * i) % len(structs)]  # the batched workload cycles through its structures
            nbor, sizes = st.neighbors()
            r = pool.sample(nbor, sizes[: len(st.weight)], st.species, st.weight, st.target, nnet, 1, st.Q, st.D)
            if i >= args.warmup:
                total_evals += r["evals"]
                total_s += r["wall_s"]
    finally:
        pool.close()
    value = total_evals / total_s
    st = structs[0]
    what = "one structure of the mixed batch per step (cycling)" if args.workload == "batched" else "the full structure"
    sample = (f"per step: {procs} single-rank processes x {nnet} solutions x 1 iteration of {what}, "
              f"task={st.Q}, depth={st.D}; evaluations counted exactly (calls of the engine's incremental fitness)")
    line = {"metric": "swap_evals_per_sec", "value": value, "unit": "swap-evals/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": (config_of(st, args.workload) if args.workload != "batched" else
                       {"workload": "batched: 64 mixed FCC/BCC structures", "solutions": 64, "parallel_task": 256,
                        "total_iter": 10, "converge_depth": 10}),
            "cpu_baseline": {"value": value, "unit": "swap-evals/s", "cores": procs, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "swap-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_batched(args):
    """Mixed-size batch: 64 structures (FCC/BCC, edge 6..30, 3-6 species, Dirichlet(2)
    compositions), 64 solutions x 256 tasks, 10 iterations, depth 10.  value = swap
    evaluations/s of the batched persistent kernel; plain = the same structures searched one
    structure per launch sequence (device-resident plans), same seeds, same results."""
    import numpy as np
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    structs = W.batched(seed=0)
    problems = [st.problem(device=True) for st in structs]
    params = [dict(num_solutions=st.P, total_iter=st.I, parallel_task=st.Q, converge_depth=st.D) for st in structs]
    seeds = lambda k: [7919 * k + i for i in range(len(structs))]  # noqa: E731
    batch = hb.Batch(problems, params)
    batch.run(seeds(0))
    tuned = batch.autotune()  # launch configuration timed on full runs, before the warm-up
    plans = [hb.Plan(pb, st.P, st.I, st.Q, st.D, autotune=True) for pb, st in zip(problems, structs)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for w in range(args.warmup):
        batch.run(seeds(w))
    b_ms, b_ev, p_ms, p_ev = 0.0, 0, 0.0, 0
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        s = batch.run(seeds(args.warmup + k))
        b_ms += s["gpu_ms"]
        b_ev += s["evals"]
    clocks = sampler.stop()
    evals_of = [int(t[1]) for t in batch.tallies()]  # per structure, last step
    for k in range(args.steps):
        for i, plan in enumerate(plans):
            flush.zero_()
            torch.cuda.synchronize()
            s = plan.run(seeds(args.warmup + k)[i])
            p_ms += s["gpu_ms"]
            p_ev += s["evals"]
    # same seeds, same results: the last step of each path
    same = 0
    for i, plan in enumerate(plans):
        same += int(np.array_equal(batch.read(i)[0], plan.read()[0]))
    for plan in plans:
        plan.close()
    batch.close()
    value = b_ev / (b_ms / 1000.0)
    plain = p_ev / (p_ms / 1000.0)

    # end to end through the public API: every step creates the batch from the host problems in
    # pinned memory (tables uploaded), runs it and reads every structure's population back
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    pinned = [hb.Problem(pin(pb.nbor), pin(pb.shell_sizes), pin(pb.species), pin(pb.weight), pin(pb.target_sro))
              for pb in problems]
    e2e_s, e2e_ev = 0.0, 0
    h2d = sum(pb.nbor.nbytes + pb.shell_sizes.nbytes + pb.species.nbytes + pb.weight.nbytes + pb.target_sro.nbytes
              for pb in pinned)
    d2h = sum(st.P * (st.num_sites + 8) for st in structs)
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eb = hb.Batch(pinned, params)
        s = eb.run(seeds(args.warmup + k))
        for i in range(len(structs)):
            eb.read(i)
        eb.close()
        e2e_s += time.perf_counter() - t0
        e2e_ev += s["evals"]

    # roofline of the persistent kernel: each structure's algorithmic bytes per evaluation
    # (BCC 8/6/12 262 B, FCC 12/6/24 422 B) weighted by its evaluations in the batch's last step, over
    # the batch's device time
    peak, peak_kind = measured_peaks()
    alg_bytes = sum(e * st.evals_bytes() for e, st in zip(evals_of, structs)) / max(1, sum(evals_of)) * b_ev
    achieved = alg_bytes / (b_ms / 1000.0) / 1e9
    line = {"metric": "swap_evals_per_sec", "value": value, "unit": "swap-evals/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched: 64 mixed FCC/BCC structures", "sites_total": int(sum(st.num_sites for st in structs)),
                       "solutions": 64, "parallel_task": 256, "total_iter": 10, "converge_depth": 10,
                       "l2": "flushed between timed steps (256 MiB write)", "batch_launch": tuned},
            "plain": {"value": plain, "ms_per_step": p_ms / args.steps, "evals_per_step": p_ev / args.steps},
            "speedup_vs_plain": value / plain, "identical_structures": same, "structures": len(structs),
            "evals_per_step": b_ev / args.steps, "clocks": clocks,
            "e2e": {"value": e2e_ev / e2e_s, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "kernel": "batch_kernel (persistent job engine)",
                         "bytes_per_eval": alg_bytes / max(1, b_ev), "peak_kind": peak_kind,
                         "traffic": DRAM_BYTES_PER_EVAL["batched"] * b_ev / args.steps},
            # one CUDA graph per step: queue reset, phase-0 seeding, the persistent kernel
            "gpu_launches": 3 * args.steps}
    print(json.dumps(line))
    return 0


def run_large(args):
    """FCC 100^3 (4,000,000 sites, 12/6/24 shells, 672 MB neighbour table), 4 species at 0.25,
    32 solutions x 4096 tasks, depth 20: one iteration per step with every local search capped at
    --large-rounds rounds.  Occupancies stay in HBM; each solution runs on a thread-block cluster."""
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    st = W.large(seed=0)
    pb = st.problem(device=True)
    plan = hb.Plan(pb, st.P, 1, st.Q, st.D, max_rounds=args.large_rounds, time_kernels=True)
    for w in range(args.warmup):
        plan.run(w)
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    ms, ev, mc_ms = 0.0, 0, 0.0
    for k in range(args.steps):  # 4 GB of tables and populations: inputs exceed L2
        s = plan.run(args.warmup + k)
        ms += s["gpu_ms"]
        ev += s["evals"]
        mc_ms += s["mc_ms"]
    clocks = sampler.stop()
    _, fit = plan.read()
    plan.close()

    # end to end through the C ABI with pinned host buffers: the neighbour table uploaded and the
    # population read back every step (same seeds as the device-timed steps, so the same work)
    import numpy as np

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hp = hb.Problem(pin(pb.nbor), pin(pb.shell_sizes), pin(pb.species), pin(pb.weight), pin(pb.target_sro))
    out_occ = torch.empty((st.P, st.num_sites), dtype=torch.uint8).pin_memory().numpy()
    out_fit = torch.empty(st.P, dtype=torch.float64).pin_memory().numpy()
    e2e_s, e2e_ev = 0.0, 0
    for k in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, s = hb.search(hp, st.P, 1, st.Q, st.D, seed=args.warmup + k, max_rounds=args.large_rounds,
                            out_occ=out_occ, out_fitness=out_fit)
        e2e_s += time.perf_counter() - t0
        e2e_ev += s["evals"]
    h2d = hp.nbor.nbytes + hp.shell_sizes.nbytes + hp.species.nbytes + hp.weight.nbytes + hp.target_sro.nbytes
    d2h = out_occ.nbytes + out_fit.nbytes

    peak, peak_kind = measured_peaks()
    B = st.evals_bytes()
    achieved = ev * B / (mc_ms / 1000.0) / 1e9
    line = {"metric": "swap_evals_per_sec", "value": ev / (ms / 1000.0), "unit": "swap-evals/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "large: FCC 100^3, 4,000,000 sites, 12/6/24", "solutions": st.P,
                       "parallel_task": st.Q, "converge_depth": st.D, "total_iter": 1,
                       "max_rounds_per_local_search": args.large_rounds,
                       "l2": "inputs larger than L2 (704 MB table)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "kernel": "mc_large_kernel (cluster local search)", "bytes_per_eval": B,
                         "peak_kind": peak_kind},
            "best_fitness_last_step": float(fit[0]), "evals_per_step": ev / args.steps, "clocks": clocks,
            "e2e": {"value": e2e_ev / e2e_s, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            # per step (one iteration): the slot-order reset; zero counts, generate, recount and fitness
            # for each of the two generations; two cluster local searches; merge and survivor sorts
            "gpu_launches": args.steps * 13}
    print(json.dumps(line))
    return 0


def run_serving(args):
    """Serving loop under a Poisson request stream (workloads.serving): each request an
    FCC/BCC supercell of 4e3..1e6 sites (log-uniform), 3-6 species, 8 solutions x 256 tasks,
    4 iterations, depth 10, fitness tolerance 1e-3; tables built on the device from the
    lattice description.  Requests are submitted at their arrival times while the server
    runs; latency = arrival to the host holding the result.  value = swap evaluations of
    the finished requests / wall time of the run."""
    import math

    import numpy as np
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    P, Q, I, D, tol = 8, 256, 4, 10, 1e-3
    reqs = W.serving(seed=0, rate=args.serve_rate, duration=args.serve_seconds, P=P, Q=Q, I=I, D=D)
    srv = hb.Server(max_requests=1024, arena_bytes=48 << 30, slice_ms=args.slice_ms)
    lo, hi = math.log(4e3), math.log(1e6)

    def level(n):  # smaller requests first
        return min(15, max(0, int(16 * (math.log(n) - lo) / (hi - lo))))

    def submit(st, seed):
        q = dict(num_solutions=P, total_iter=I, parallel_task=Q, converge_depth=D, seed=seed)
        return srv.submit_lattice(st.lattice, st.cell, st.species, st.weight, st.target, q, shell_set=st.shell_set,
                                  tolerance=tol, priority=level(st.num_sites))

    warm = W.serving(seed=1, rate=50.0, duration=1.0, P=P, Q=Q, I=I, D=D)
    warm = sorted(warm, key=lambda r: r[1].num_sites)[: max(args.warmup, 1)]
    for k, (_, st) in enumerate(warm):
        submit(st, 10 ** 6 + k)
    srv.drain()
    for rid in list(srv._meta):
        srv.result(rid)
    srv.take_finished()
    base = srv.status()

    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    arrival, size, lat, evals, bytes_alg, iters, h2d, d2h = {}, {}, [], 0, 0.0, [], 0, 0
    i, t0 = 0, time.perf_counter()
    hard_stop = args.serve_seconds + 120.0
    last_done = 0.0
    lat_by_size = []  # (sites, latency ms)
    step_gap, step_ms, t_prev = 0.0, 0.0, None  # longest gap between steps; longest step (host view)
    while True:
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i][0] <= now:
            st = reqs[i][1]
            rid = submit(st, i)
            arrival[rid], size[rid] = reqs[i][0], (st.num_sites, st.evals_bytes())
            h2d += st.species.nbytes + st.weight.nbytes + st.target.nbytes
            i += 1
        if i == len(reqs) and not arrival:
            break
        if now > hard_stop:
            break
        if not arrival:
            time.sleep(max(0.0, min(reqs[i][0] - now, 0.002)))
            continue
        ts = time.perf_counter()
        if t_prev is not None:
            step_gap = max(step_gap, ts - t_prev)
        srv.step()
        t_prev = time.perf_counter()
        step_ms = max(step_ms, (t_prev - ts) * 1000.0)
        for rid in srv.take_finished():
            if rid not in arrival:
                continue
            r = srv.result(rid)
            occ, fit, info = r
            t = time.perf_counter() - t0
            lat.append((t - arrival.pop(rid)) * 1000.0)
            n, B = size.pop(rid)
            lat_by_size.append((n, lat[-1]))
            evals += info["evals"]
            bytes_alg += info["evals"] * B
            iters.append(info["iterations"])
            d2h += occ.nbytes + fit.nbytes
            last_done = t
    clocks = sampler.stop()
    st_end = srv.status()
    busy = st_end["busy_ms"] - base["busy_ms"]
    srv.close()
    wall = last_done
    lat_a = np.array(lat) if lat else np.array([float("nan")])

    def pct(sel):  # p50 / p99 / max of the requests whose site count passes sel
        v = np.array([ms for n, ms in lat_by_size if sel(n)])
        if v.size == 0:
            return None
        return {"count": int(v.size), "p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
                "max": float(v.max())}

    peak, peak_kind = measured_peaks()
    achieved = bytes_alg / (busy / 1000.0) / 1e9 if busy > 0 else 0.0
    value = evals / wall if wall > 0 else 0.0
    line = {"metric": "swap_evals_per_sec", "value": value, "unit": "swap-evals/s", "n_gpus": 1, "steps": 1,
            "warmup": len(warm), "ms_per_step": wall * 1000.0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "serving: Poisson stream of FCC/BCC requests, 4e3..1e6 sites (log-uniform)",
                       "rate_per_s": args.serve_rate, "arrival_window_s": args.serve_seconds,
                       "solutions": P, "parallel_task": Q, "total_iter": I, "converge_depth": D, "tolerance": tol,
                       "slice_ms": args.slice_ms, "priority": "smaller requests first (16 levels by log size)",
                       "l2": "inputs larger than L2 (tables of the requests on the device exceed 126 MB)"},
            "requests": {"arrived": i, "finished": len(lat), "unfinished": len(arrival),
                         "per_s": len(lat) / wall if wall > 0 else 0.0,
                         "latency_ms": {"p50": float(np.percentile(lat_a, 50)), "p90": float(np.percentile(lat_a, 90)),
                                        "p99": float(np.percentile(lat_a, 99)), "max": float(lat_a.max())},
                         "reached_tolerance_before_last_iteration": int(sum(1 for k in iters if k < I)),
                         "latency_ms_by_sites": {"below_1e5": pct(lambda n: n < 1e5),
                                                 "from_1e5": pct(lambda n: n >= 1e5)},
                         "host_longest_step_ms": step_ms, "host_longest_gap_between_steps_ms": step_gap * 1000.0},
            "gpu_busy_fraction": busy / (wall * 1000.0) if wall > 0 else 0.0,
            "e2e": {"value": value, "unit": "swap-evals/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "the serving line is end to end: one step = the whole run"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "kernel": "batch_kernel (persistent job engine)",
                         "peak_kind": peak_kind, "traffic": None},
            "gpu_launches": int(st_end["launches"] - base["launches"]), "clocks": clocks}
    print(json.dumps(line))
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "serving":
        return run_serving(args)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    import pyhea_b200 as hb

    st = workload(args.workload)
    problem = st.problem(device=True)
    nbor, sizes = st.neighbors(device=True)
    plan = hb.Plan(problem, st.P, st.I, st.Q, st.D, time_kernels=True, autotune=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    from pyhea_b200 import replicas

    for w in range(args.warmup):
        plan.run(replicas.replica_seed(rank, w))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    total_ms, evals, mc_ms, launches, accepts = 0.0, 0, 0.0, 0, 0
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        s = plan.run(replicas.replica_seed(rank, args.warmup + k))
        total_ms += s["gpu_ms"]
        evals += s["evals"]
        mc_ms += s["mc_ms"]
        launches += s["mc_launches"]
        accepts += s["accepts"]
    torch.cuda.synchronize()
    clocks = sampler.stop()
    _, best = plan.read()
    block = plan.local_search_block
    plan.close()

    # end to end through the C ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hp = hb.Problem(pin(problem.nbor), pin(problem.shell_sizes), pin(problem.species), pin(problem.weight),
                    pin(problem.target_sro))
    out_occ = torch.empty((st.P, st.num_sites), dtype=torch.uint8).pin_memory().numpy()
    out_fit = torch.empty(st.P, dtype=torch.float64).pin_memory().numpy()
    e2e_s, e2e_evals = 0.0, 0
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, s = hb.search(hp, st.P, st.I, st.Q, st.D, seed=replicas.replica_seed(rank, 10_000 + k), out_occ=out_occ,
                            out_fitness=out_fit)
        e2e_s += time.perf_counter() - t0
        e2e_evals += s["evals"]
    h2d = (hp.nbor.nbytes + hp.shell_sizes.nbytes + hp.species.nbytes + hp.weight.nbytes + hp.target_sro.nbytes)
    d2h = out_occ.nbytes + out_fit.nbytes

    # time to tolerance: the same search through the serving loop with a fitness tolerance (local
    # searches and the request end once it is reached), submission to result on the host; 1e-3 is
    # PyHEA's default threshold, the looser ones show the time along the way
    time_to_tol = None
    time_to_tol_sweep = []
    if rank == 0:
        srv = hb.Server(max_requests=4, slice_ms=50.0)
        q = dict(num_solutions=st.P, total_iter=st.I, parallel_task=st.Q, converge_depth=st.D,
                 seed=replicas.replica_seed(rank, 20_000))
        for tol in (1e-3, 1.02e-3, 1.1e-3, 1.5e-3):
            t0 = time.perf_counter()
            rid = srv.submit(problem, q, tolerance=tol)
            res = None
            while res is None:
                srv.step()
                res = srv.result(rid)
            tt = time.perf_counter() - t0
            time_to_tol_sweep.append({"tolerance": tol, "wall_ms": 1000.0 * tt, "iterations": res[2]["iterations"],
                                      "best_fitness": float(res[1][0]), "reached": bool(res[1][0] <= tol),
                                      "evals": res[2]["evals"]})
        srv.close()
        time_to_tol = time_to_tol_sweep[0]

    dev = torch.device("cuda", local)
    total_ms_max, evals_all = replicas.combine(total_ms, evals, device=dev)
    e2e_ms_max, e2e_evals_all = replicas.combine(1000.0 * e2e_s, e2e_evals, device=dev)
    e2e_max = e2e_ms_max / 1000.0

    if rank == 0:
        peak, peak_kind = measured_peaks()
        B = st.evals_bytes()
        achieved = evals * B / (mc_ms / 1000.0) / 1e9 if mc_ms > 0 else None
        line = {
            "metric": "swap_evals_per_sec", "value": evals_all / (total_ms_max / 1000.0), "unit": "swap-evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config_of(st, args.workload), parallelism=f"replicas x{world}",
                           local_search_block=block),
            "gpu_launches": None,
            "e2e": {"value": e2e_evals_all / e2e_max, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": (DRAM_BYTES_PER_EVAL[args.workload] * evals / launches
                                     if args.workload in DRAM_BYTES_PER_EVAL and launches else None),
                         "algorithmic_bytes_per_launch": evals * B / launches if launches else None,
                         "kernel": "mc_kernel (local search)", "bytes_per_eval": B, "peak_kind": peak_kind,
                         "kernel_share": mc_ms / total_ms if total_ms else None},
            "search": {"evals_per_step": evals / args.steps, "accepts_per_step": accepts / args.steps,
                       "best_fitness_last_step": float(best[0])},
            "time_to_tol": time_to_tol, "time_to_tol_sweep": time_to_tol_sweep,
            "clocks": clocks,
        }
        # kernels launched per search: 1 generate + per iteration (generate, search, merge, search, sort), plus
        # the iota of the slot order
        line["gpu_launches"] = args.steps * (2 + 5 * st.I)
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_reference_sample(st, nbor, sizes, args.cpu_procs or host_cores())
            if r:
                line["cpu_baseline"] = {"value": r["evals"] / r["wall_s"], "unit": "swap-evals/s", "cores": r["procs"],
                                        "kind": "reference", "sample": r["sample"]}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
