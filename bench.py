#!/usr/bin/env python
"""Swap-evaluation throughput of the SRO-targeted swap search on B200.

Headline (default): the plain GPU configuration -- BCC 20x20x20 (16000 sites,
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
         species) + 2 B per evaluation) over its CUDA-event time against the
         measured HBM copy bandwidth (the normalisation every line uses), and
         the two ceilings that bind the kernel: L2 bytes per evaluation (ncu)
         against an L2 read peak measured here by the library's own probe
         kernel (l2_frac), and warp instructions per evaluation (ncu) against
         the SMs' issue rate at the sampled SM clock (issue_frac)
  cpu_baseline  the reference CPU engine (oracle/_ref) on a bounded sample
  dropin_e2e  the pybind11 drop-in called as pyhea/model/opt.py:89-90 calls it
         (nested Python lists, per-iteration log on), end to end

At one GPU the line also carries the other configurations, each measured here:
  batched   the mixed 64-structure batch on the persistent kernel against the
            same structures searched one plain plan at a time (same seeds, same
            results), with its own roofline
  serving   a Poisson request stream through the serving loop at the stated
            request size (64 solutions x 256 tasks, 10 iterations, tolerance
            1e-3) and the stated 200 requests/s, over a short arrival window:
            that rate is above one B200's capacity at this request size, so
            the run measures the capacity (finished requests / wall time) and
            latency under overload
  serving_sustained  the same requests at a rate below capacity (30/s): latency
            p50/p90/p99 and by request size
  large     FCC 100^3 (4,000,000 sites): iterations of the uncapped search
  time_to_tol  wall time until the best fitness reaches 1e-3 (PyHEA's default
            threshold) on the plain GPU and CPU structures, plus looser tolerances

--workload batched|large|serving|plain_cpu prints that configuration's own line.
--impl reference times the reference CPU engine alone (rank 0) on the same
workload and prints the same line with "impl": "reference".

--case plain|batch|large runs one small fixed case for a profiler capture and
prints its statistics (rounds, evaluations, accepts, device time) as JSON:
  plain [--iters 1]            one search of the plain GPU structure
  batch [--count 16] [--iters 1]  the `count` largest structures of the mixed
                               batch, one batched run
  large [--cell 40] [--rounds 500]  one local search of an FCC cell^3 supercell
                               on the HBM cluster path (32 solutions x 4096 tasks)
Multi-GPU: replicas -- every rank searches its own copy of the workload with
its own seeds; no collective on the data path.
"""
import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

HBM_FALLBACK_GBS = 6650.0
# Per-evaluation counters of the dominant kernel from one ncu capture each (per launch, so they
# scale to the bench's launches by their evaluations):
#   dram   dram__bytes_read.sum + dram__bytes_write.sum      -> roofline.traffic
#   l2     lts__t_sectors_srcunit_tex.sum x 32 B              -> roofline.l2_frac
#   inst   smsp__inst_executed.sum (warp instructions)        -> roofline.issue_frac
#   dram_read  dram__bytes_read.sum                           -> roofline.dram_random (batched)
# mc_kernel<5, ImplicitShells<3>> (the plain structure's table is recognised as a BCC lattice's): the
# first local-search launch of `python bench.py --case plain --iters 1` (203.72 M evaluations):
# 69.81 MB + 92.28 MB DRAM, 428.96 M L2 sectors, 3.9814 G warp instructions.  batch_kernel: the launch
# of `python bench.py --case batch --count 64 --iters 10`, the bench's batch configuration (6268.46 M
# evaluations, lattice tables recognised): 1189.72 GB + 81.32 GB DRAM, 68.43 G L2 sectors, 178.51 G
# warp instructions.  dram_random_probe_kernel (hea_dram_random_probe over 4 GiB, 77.59 M
# random 16-byte loads): 9.833 GB DRAM read, i.e. 126.7 B per load (each load fetches a 128-byte line).
KERNEL_COUNTERS = {
    "plain_gpu": {"dram": (69.81e6 + 92.28e6) / 203.72e6, "l2": 428.96e6 * 32.0 / 203.72e6,
                  "inst": 3.9814e9 / 203.72e6,
                  "capture": "mc_kernel, first local-search launch of bench.py --case plain --iters 1"},
    "batched": {"dram": (1189.72e9 + 81.32e9) / 6268.46e6, "l2": 68.43e9 * 32.0 / 6268.46e6,
                "inst": 178.51e9 / 6268.46e6, "dram_read": 1189.72e9 / 6268.46e6,
                "capture": "batch_kernel, bench.py --case batch --count 64 --iters 10"},
}
DRAM_BYTES_PER_RANDOM_LOAD = 9.833e9 / 77.594624e6
L2_PROBE_BYTES = 32 << 20  # fits in L2 (126 MB) with room to spare


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
    ap.add_argument("--serve-window", type=float, default=2.0,
                    help="headline line's serving object: arrival window at --serve-rate, seconds")
    ap.add_argument("--serve-sustained-rate", type=float, default=30.0,
                    help="headline line's serving_sustained object: arrival rate below capacity, requests/s")
    ap.add_argument("--serve-sustained-seconds", type=float, default=20.0,
                    help="headline line's serving_sustained object: arrival window, seconds")
    ap.add_argument("--serve-solutions", type=int, default=64, help="serving: solutions per request")
    ap.add_argument("--serve-iters", type=int, default=10, help="serving: iterations per request (tolerance ends it)")
    ap.add_argument("--slice-ms", type=float, default=40.0, help="serving: time slice of one server step")
    ap.add_argument("--large-iters", type=int, default=3, help="large: iterations of the uncapped search")
    ap.add_argument("--tol-iters", type=int, default=400, help="time_to_tol: iteration cap")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="headline line only (no batched/serving/large)")
    ap.add_argument("--cpu-procs", type=int, default=0, help="reference processes (0: all host cores)")
    ap.add_argument("--neighbours", choices=["table", "implicit"], default="table",
                    help="batched, large and --case: neighbour table or implicit lattice neighbours")
    ap.add_argument("--case", choices=["plain", "batch", "large"], help="one small case for a profiler capture")
    ap.add_argument("--iters", type=int, default=1, help="--case plain/batch: iterations")
    ap.add_argument("--count", type=int, default=16, help="--case batch: structures")
    ap.add_argument("--cell", type=int, default=40, help="--case large: FCC cell edge")
    ap.add_argument("--rounds", type=int, default=500, help="--case large: round cap")
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
        return self

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


def sm_count():
    import torch

    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def roofline_of(kernel, counters, evals, kernel_s, bytes_per_eval, launches, clocks, l2_peak, sms):
    """Roofline object of one kernel: the algorithmic-byte normalisation against HBM, plus the L2 and
    issue ceilings from the kernel's ncu counters per evaluation (see KERNEL_COUNTERS)."""
    peak, peak_kind = measured_peaks()
    rate = evals / kernel_s if kernel_s > 0 else 0.0
    achieved = rate * bytes_per_eval / 1e9
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "kernel": kernel, "bytes_per_eval": bytes_per_eval, "peak_kind": peak_kind,
           "traffic": counters["dram"] * evals / launches if counters.get("dram") and launches else None,
           "algorithmic_bytes_per_launch": evals * bytes_per_eval / launches if launches else None,
           "counters_from": counters["capture"]}
    if counters.get("l2") and l2_peak:
        l2_gbs = rate * counters["l2"] / 1e9
        out["l2"] = {"bytes_per_eval": counters["l2"], "achieved_gbs": l2_gbs, "peak_gbs": l2_peak,
                     "peak_kind": "measured (hea_l2_read_probe, 32 MiB read through L2)"}
        out["l2_frac"] = l2_gbs / l2_peak
    if counters.get("inst") and sms:
        mhz = (clocks or {}).get("sm_mhz") or 1965.0
        peak_inst = sms * 4 * mhz * 1e6  # one warp instruction per SM sub-partition per cycle
        out["issue"] = {"warp_inst_per_eval": counters["inst"], "achieved_per_s": rate * counters["inst"],
                        "peak_per_s": peak_inst, "sm_mhz": mhz}
        out["issue_frac"] = rate * counters["inst"] / peak_inst
    return out


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
    from pyhea_b200 import workloads as W  # numpy only: maps none of this build's libraries

    structs = W.batched(seed=0) if args.workload == "batched" else [workload(args.workload)]
    procs = args.cpu_procs or host_cores()
    from oracle.ref_timing import RefPool, available

    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_accelerate.so was not built"}))
        return 0
    pool = RefPool(procs)
    nnet = 2
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


# ---------------------------------------------------------------------------
# Batched: the mixed 64-structure batch
# ---------------------------------------------------------------------------
def neighbours_of(lattice_code, implicit):
    """How a line's structures get their neighbours: described by the lattice, a table the library
    recognised as an FCC/BCC cube's (both run on lattice arithmetic, same results), or a table."""
    if implicit:
        return "implicit (lattice arithmetic, no table)"
    if lattice_code:
        return "table, recognised as %s lattice's (lattice arithmetic, table not kept)" % ("an FCC", "a BCC")[lattice_code - 1]
    return "table"


def pinned_problem(pb):
    """The same problem with its host arrays in pinned memory (implicit problems keep no table)."""
    import numpy as np
    import torch

    import pyhea_b200 as hb

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    return hb.Problem(None if pb.nbor is None else pin(pb.nbor), pin(pb.shell_sizes), pin(pb.species),
                      pin(pb.weight), pin(pb.target_sro), lattice=pb.lattice)


def problem_bytes(pb):
    """Host bytes a search copies to the device for a problem."""
    return ((pb.nbor.nbytes if pb.nbor is not None else 0) + pb.shell_sizes.nbytes + pb.species.nbytes +
            pb.weight.nbytes + pb.target_sro.nbytes)


def measure_batched(steps, warmup, l2_peak=None, implicit=False, select=None):
    """64 structures (FCC/BCC, edge 6..30, 3-6 species, Dirichlet(2) compositions), 64 solutions x
    256 tasks, 10 iterations, depth 10.  value = swap evaluations/s of the batched persistent kernel;
    plain = the same structures searched one structure per launch sequence (device-resident plans,
    CTA size autotuned), same seeds, same results.  `select`: indices of the structures this process
    searches (a rank's share of the batch; each keeps the seeds it has in the whole batch)."""
    import numpy as np
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    every = W.batched(seed=0)
    index = list(range(len(every))) if select is None else list(select)
    structs = [every[i] for i in index]
    problems = [st.problem(device=True, implicit=implicit) for st in structs]
    params = [dict(num_solutions=st.P, total_iter=st.I, parallel_task=st.Q, converge_depth=st.D) for st in structs]
    seeds = lambda k: [7919 * k + i for i in index]  # noqa: E731
    batch = hb.Batch(problems, params)
    batch.run(seeds(0))
    tuned = batch.autotune()  # launch configuration timed on full runs, before the warm-up
    plans = [hb.Plan(pb, st.P, st.I, st.Q, st.D, autotune=True) for pb, st in zip(problems, structs)]
    recognised = all(plan.lattice for plan in plans)  # the batch builds its structures the same way
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for w in range(warmup):
        batch.run(seeds(w))
    b_ms, b_ev, p_ms, p_ev = 0.0, 0, 0.0, 0
    sampler = ClockSampler(torch.cuda.current_device()).start()
    for k in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        s = batch.run(seeds(warmup + k))
        b_ms += s["gpu_ms"]
        b_ev += s["evals"]
    clocks = sampler.stop()
    evals_of = [int(t[1]) for t in batch.tallies()]  # per structure, last step
    for k in range(steps):
        for i, plan in enumerate(plans):
            flush.zero_()
            torch.cuda.synchronize()
            s = plan.run(seeds(warmup + k)[i])
            p_ms += s["gpu_ms"]
            p_ev += s["evals"]
    same = 0  # same seeds, same results: the last step of each path
    for i, plan in enumerate(plans):
        same += int(np.array_equal(batch.read(i)[0], plan.read()[0]))
    for plan in plans:
        plan.close()
    batch.close()
    value = b_ev / (b_ms / 1000.0)
    plain = p_ev / (p_ms / 1000.0)

    # end to end through the public API: every step creates the batch from the host problems in
    # pinned memory (tables uploaded), runs it and reads every structure's population back
    pinned = [pinned_problem(pb) for pb in problems]
    e2e_s, e2e_ev = 0.0, 0
    h2d = sum(problem_bytes(pb) for pb in pinned)
    d2h = sum(st.P * (st.num_sites + 8) for st in structs)
    for k in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eb = hb.Batch(pinned, params)
        s = eb.run(seeds(warmup + k))
        last = [eb.read(i)[0] for i in range(len(structs))]
        eb.close()
        e2e_s += time.perf_counter() - t0
        e2e_ev += s["evals"]

    # the same structures described by their lattices (no neighbour tables): device and end-to-end
    # rates, and the results of the last step compared with the tables'
    implicit_block = None
    if not implicit:
        ip = [pinned_problem(st.problem(implicit=True)) for st in structs]
        ib = hb.Batch(ip, params)
        ib.run(seeds(0))
        i_ms = i_ev = 0
        for k in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            s = ib.run(seeds(warmup + k))
            i_ms += s["gpu_ms"]
            i_ev += s["evals"]
        ib.close()
        ie_s, ie_ev = 0.0, 0
        for k in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eb = hb.Batch(ip, params)
            s = eb.run(seeds(warmup + k))
            got = [eb.read(i)[0] for i in range(len(structs))]
            eb.close()
            ie_s += time.perf_counter() - t0
            ie_ev += s["evals"]
        isame = sum(int(np.array_equal(a, b)) for a, b in zip(got, last))
        implicit_block = {"value": i_ev / (i_ms / 1000.0), "unit": "swap-evals/s", "ms_per_step": i_ms / steps,
                          "identical_structures": isame,
                          "e2e": {"value": ie_ev / ie_s, "unit": "swap-evals/s",
                                  "h2d_bytes_per_step": int(sum(problem_bytes(pb) for pb in ip)),
                                  "d2h_bytes_per_step": int(d2h)}}

    # roofline: each structure's algorithmic bytes per evaluation (BCC 8/6/12 262 B, FCC 12/6/24
    # 422 B) weighted by its evaluations in the last step
    bpe = sum(e * st.evals_bytes() for e, st in zip(evals_of, structs)) / max(1, sum(evals_of))
    roof = roofline_of("batch_kernel (persistent job engine)", KERNEL_COUNTERS["batched"], b_ev, b_ms / 1000.0,
                       bpe, steps, clocks, l2_peak, sm_count())
    # the regime that binds the batch: most of its evaluations are on structures whose site
    # histograms stay in DRAM, read at random; random 16-byte DRAM loads are measured here by the
    # library's probe and converted to DRAM bytes with the probe's captured bytes per load (the
    # batch's own DRAM traffic also holds streaming reads, so its fraction can exceed 1)
    loads_per_s = hb.dram_random_probe(4 << 30, 256)
    peak_dram = loads_per_s * DRAM_BYTES_PER_RANDOM_LOAD / 1e9
    got_dram = value * KERNEL_COUNTERS["batched"]["dram_read"] / 1e9
    roof["dram_random"] = {"probe_loads_per_s": loads_per_s, "dram_bytes_per_probe_load": DRAM_BYTES_PER_RANDOM_LOAD,
                           "peak_gbs": peak_dram, "dram_read_bytes_per_eval": KERNEL_COUNTERS["batched"]["dram_read"],
                           "achieved_gbs": got_dram, "unit": "GB/s"}
    roof["dram_random_frac"] = got_dram / peak_dram
    return {"value": value, "unit": "swap-evals/s", "steps": steps, "warmup": warmup, "ms_per_step": b_ms / steps,
            "config": {"workload": "batched: 64 mixed FCC/BCC structures",
                       "sites_total": int(sum(st.num_sites for st in structs)), "solutions": 64,
                       "parallel_task": 256, "total_iter": 10, "converge_depth": 10,
                       "l2": "flushed between timed steps (256 MiB write)", "batch_launch": tuned,
                       "neighbours": neighbours_of(0, True) if implicit else
                       ("tables, each recognised as its FCC/BCC lattice's (lattice arithmetic, tables not kept)"
                        if recognised else "tables")},
            "plain": {"value": plain, "ms_per_step": p_ms / steps, "evals_per_step": p_ev / steps},
            "speedup_vs_plain": value / plain, "identical_structures": same, "structures": len(structs),
            "evals_per_step": b_ev / steps, "clocks": clocks, "roofline": roof,
            "e2e": {"value": e2e_ev / e2e_s, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            **({"implicit_neighbours": implicit_block} if implicit_block else {}),
            # one CUDA graph per step: queue reset, phase-0 seeding, the persistent kernel
            "gpu_launches": 3 * steps,
            "_raw": {"b_ms": b_ms, "b_ev": b_ev, "p_ms": p_ms, "p_ev": p_ev, "e2e_ms": 1000.0 * e2e_s,
                     "e2e_ev": e2e_ev}}


def run_batched(args):
    """The batched line.  Under torchrun the 64 structures are split across the ranks (replicas.shard,
    balanced by sites x solutions); each rank searches its share as one batch with the seeds the
    structures have in the whole batch, and only times (max) and evaluation counts (sum) are combined:
    total work is fixed, so the scaling is strong.  The roofline and the implicit-neighbour block are
    rank 0's."""
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
    from pyhea_b200 import replicas
    from pyhea_b200 import workloads as W

    select = None
    if world > 1:
        every = W.batched(seed=0)
        select = replicas.shard([st.num_sites * st.P for st in every], rank, world)
    sub = measure_batched(args.steps, args.warmup, hb.l2_read_probe(L2_PROBE_BYTES),
                          implicit=args.neighbours == "implicit", select=select)
    raw = sub.pop("_raw")
    if world > 1:
        dev = torch.device("cuda", local)
        b_ms, b_ev = replicas.combine(raw["b_ms"], raw["b_ev"], device=dev)
        p_ms, p_ev = replicas.combine(raw["p_ms"], raw["p_ev"], device=dev)
        e_ms, e_ev = replicas.combine(raw["e2e_ms"], raw["e2e_ev"], device=dev)
        sub["value"] = b_ev / (b_ms / 1000.0)
        sub["ms_per_step"] = b_ms / args.steps
        sub["evals_per_step"] = b_ev / args.steps
        sub["plain"] = {"value": p_ev / (p_ms / 1000.0), "ms_per_step": p_ms / args.steps,
                        "evals_per_step": p_ev / args.steps}
        sub["speedup_vs_plain"] = sub["value"] / sub["plain"]["value"]
        sub["e2e"]["value"] = e_ev / (e_ms / 1000.0)
        sub["config"]["parallelism"] = f"batch split over {world} ranks"
        sub["config"]["structures_on_rank0"] = len(select)
        sub.pop("implicit_neighbours", None)
    line = {"metric": "swap_evals_per_sec", "n_gpus": world, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    line.update(sub)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Large: FCC 100^3
# ---------------------------------------------------------------------------
def measure_large(iters, e2e=True, implicit=False):
    """FCC 100^3 (4,000,000 sites, 12/6/24 shells, 672 MB neighbour table), 4 species at 0.25, 32
    solutions x 4096 tasks, depth 20: `iters` iterations of the uncapped search (the configuration
    states 200).  Occupancies stay in HBM; each solution runs on a thread-block cluster.  With
    `implicit` the neighbour ids come from lattice arithmetic and no table is uploaded or read."""
    import numpy as np
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    st = W.large(seed=0)
    pb = st.problem(device=True, implicit=implicit)
    warm = hb.Plan(pb, st.P, 1, st.Q, st.D, max_rounds=50)  # kernels loaded; capped
    warm.run(0)
    warm.close()
    plan = hb.Plan(pb, st.P, iters, st.Q, st.D, time_kernels=True)
    lattice_code = plan.lattice
    sampler = ClockSampler(torch.cuda.current_device()).start()
    s = plan.run(1)
    clocks = sampler.stop()
    _, fit = plan.read()
    plan.close()
    out = {"value": s["evals"] / (s["gpu_ms"] / 1000.0), "unit": "swap-evals/s", "steps": 1, "warmup": 1,
           "ms_per_step": s["gpu_ms"], "evals_per_step": s["evals"], "rounds_per_step": s["rounds"],
           "best_fitness": float(fit[0]),
           "config": {"workload": "large: FCC 100^3, 4,000,000 sites, 12/6/24", "solutions": st.P,
                      "parallel_task": st.Q, "converge_depth": st.D, "total_iter_run": iters,
                      "total_iter_stated": st.I, "max_rounds_per_local_search": None,
                      "warmup": "one capped (50-round) iteration",
                      "neighbours": neighbours_of(lattice_code, implicit),
                      "l2": "inputs larger than L2 (4.1 GB of site histograms)"},
           "clocks": clocks}
    peak, peak_kind = measured_peaks()
    B = st.evals_bytes()
    achieved = s["evals"] * B / (s["mc_ms"] / 1000.0) / 1e9 if s["mc_ms"] > 0 else 0.0
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "kernel": "mc_large_kernel (cluster local search)", "bytes_per_eval": B,
                       "peak_kind": peak_kind, "traffic": None}
    # per iteration: the slot-order reset; zero counts, generate, recount and fitness for each of the
    # two generations; two cluster local searches; merge and survivor sorts
    out["gpu_launches"] = 1 + 12 * iters
    if e2e:
        # end to end through the C ABI with pinned host buffers: the neighbour table uploaded and the
        # population read back (same seed as the device-timed step, so the same work)
        hp = pinned_problem(pb)
        out_occ = torch.empty((st.P, st.num_sites), dtype=torch.uint8).pin_memory().numpy()
        out_fit = torch.empty(st.P, dtype=torch.float64).pin_memory().numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, e = hb.search(hp, st.P, iters, st.Q, st.D, seed=1, out_occ=out_occ, out_fitness=out_fit)
        dt = time.perf_counter() - t0
        h2d = problem_bytes(hp)
        out["e2e"] = {"value": e["evals"] / dt, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                      "d2h_bytes_per_step": int(out_occ.nbytes + out_fit.nbytes)}
    return out


def run_large(args):
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    line = {"metric": "swap_evals_per_sec", "n_gpus": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    line.update(measure_large(args.large_iters, implicit=args.neighbours == "implicit"))
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# Serving: a Poisson request stream
# ---------------------------------------------------------------------------
def measure_serving(rate, seconds, P, I, slice_ms, warmup=1, Q=256, D=10, tol=1e-3):
    """Serving loop under a Poisson request stream (workloads.serving): each request an FCC/BCC
    supercell of 4e3..1e6 sites (log-uniform), 3-6 species, P solutions x Q tasks, up to I
    iterations, depth D, fitness tolerance `tol`; tables built on the device from the lattice
    description.  Requests are submitted at their arrival times while the server runs; latency =
    arrival to the host holding the result.  value = swap evaluations of the finished requests /
    wall time of the run."""
    import numpy as np
    import torch

    import pyhea_b200 as hb
    from pyhea_b200 import workloads as W

    reqs = W.serving(seed=0, rate=rate, duration=seconds, P=P, Q=Q, I=I, D=D)
    srv = hb.Server(max_requests=1024, arena_bytes=48 << 30, slice_ms=slice_ms)
    lo, hi = math.log(4e3), math.log(1e6)

    def level(n):  # smaller requests first
        return min(15, max(0, int(16 * (math.log(n) - lo) / (hi - lo))))

    def submit(st, seed):
        q = dict(num_solutions=P, total_iter=I, parallel_task=Q, converge_depth=D, seed=seed)
        return srv.submit_lattice(st.lattice, st.cell, st.species, st.weight, st.target, q, shell_set=st.shell_set,
                                  tolerance=tol, priority=level(st.num_sites))

    warm = W.serving(seed=1, rate=50.0, duration=1.0, P=P, Q=Q, I=I, D=D)
    warm = sorted(warm, key=lambda r: r[1].num_sites)[: max(warmup, 1)]
    for k, (_, st) in enumerate(warm):
        submit(st, 10 ** 6 + k)
    srv.drain()
    for rid in list(srv._meta):
        srv.result(rid)
    srv.take_finished()
    base = srv.status()

    sampler = ClockSampler(torch.cuda.current_device()).start()
    arrival, size, lat, evals, bytes_alg, iters, h2d, d2h = {}, {}, [], 0, 0.0, [], 0, 0
    i, t0 = 0, time.perf_counter()
    hard_stop = seconds + 600.0
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
            occ, fit, info = srv.result(rid)
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
    return {"value": value, "unit": "swap-evals/s", "steps": 1, "warmup": len(warm), "ms_per_step": wall * 1000.0,
            "config": {"workload": "serving: Poisson stream of FCC/BCC requests, 4e3..1e6 sites (log-uniform)",
                       "rate_per_s": rate, "arrival_window_s": seconds, "solutions": P, "parallel_task": Q,
                       "total_iter": I, "converge_depth": D, "tolerance": tol, "slice_ms": slice_ms,
                       "priority": "smaller requests first (16 levels by log size)",
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


def run_serving(args):
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    line = {"metric": "swap_evals_per_sec", "n_gpus": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    line.update(measure_serving(args.serve_rate, args.serve_seconds, args.serve_solutions, args.serve_iters,
                                args.slice_ms, args.warmup))
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# Time to tolerance
# ---------------------------------------------------------------------------
def measure_time_to_tol(st, problem, seed, max_iter, tols=(1e-3, 1.02e-3, 1.1e-3, 1.5e-3)):
    """The structure's search through the serving loop with a fitness tolerance (local searches and
    the request end once it is reached) and up to max_iter iterations; submission to result on the
    host.  1e-3 is PyHEA's default threshold (pyhea/model/opt.py:37)."""
    import pyhea_b200 as hb

    srv = hb.Server(max_requests=4, slice_ms=50.0)
    q = dict(num_solutions=st.P, total_iter=max_iter, parallel_task=st.Q, converge_depth=st.D, seed=seed)
    out = []
    for tol in tols:
        t0 = time.perf_counter()
        rid = srv.submit(problem, q, tolerance=tol)
        res = None
        while res is None:
            srv.step()
            res = srv.result(rid)
        tt = time.perf_counter() - t0
        out.append({"tolerance": tol, "wall_ms": 1000.0 * tt, "iterations": res[2]["iterations"],
                    "best_fitness": float(res[1][0]), "reached": bool(res[1][0] <= tol), "evals": res[2]["evals"]})
    srv.close()
    return {"workload": st.name, "solutions": st.P, "parallel_task": st.Q, "converge_depth": st.D,
            "iteration_cap": max_iter, "result": out[0], "sweep": out}


# ---------------------------------------------------------------------------
# The drop-in module as PyHEA calls it
# ---------------------------------------------------------------------------
def measure_dropin(st, nbor, sizes, seed):
    """accelerate.run_local_parallel_hcs_cuda called positionally as pyhea/model/opt.py:89-90 calls
    it: neighbour table as nested Python lists [N][S][Z], element counts, weights, target [S][T*T],
    the per-iteration log line on (the reference prints it); returns lists.  End to end, including
    the flattening of the nested lists and the Python lists built for the result.  The library
    prints the log lines on file descriptor 1; they are counted here, not passed on."""
    import pyhea_b200 as hb
    from pyhea_b200 import lattice as L

    nested = L.as_nested(nbor, sizes)
    species = [int(x) for x in st.species]
    weight = [float(w) for w in st.weight]
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile() as log:
        os.dup2(log.fileno(), 1)
        try:
            t0 = time.perf_counter()
            latts, fits = hb.accelerate.run_local_parallel_hcs_cuda(st.P, st.I, st.Q, st.D, 0.001, nested, species,
                                                                    weight, st.target, seed=seed)
            dt = time.perf_counter() - t0
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        log.seek(0)
        lines = log.read().decode(errors="replace").count("best fitness")
    return {"wall_ms": dt * 1000.0, "logged_lines": lines, "best_fitness": float(fits[0]),
            "note": "value = the plain search's evaluations per step over this call's wall time"}


def run_case(args):
    """One small fixed case for profiler captures; prints its statistics as JSON."""
    import numpy as np

    import pyhea_b200 as hb
    from pyhea_b200 import lattice as L
    from pyhea_b200 import workloads as W

    implicit = args.neighbours == "implicit"
    if args.case == "plain":
        st = W.plain_gpu(seed=0)
        plan = hb.Plan(st.problem(device=True, implicit=implicit), st.P, args.iters, st.Q, st.D)
        out = plan.run(123)
        plan.close()
    elif args.case == "batch":
        structs = sorted(W.batched(seed=0), key=lambda s: -s.num_sites)[: args.count]
        problems = [st.problem(device=True, implicit=implicit) for st in structs]
        params = [dict(num_solutions=st.P, total_iter=args.iters, parallel_task=st.Q, converge_depth=st.D)
                  for st in structs]
        b = hb.Batch(problems, params)
        out = b.run([11 + i for i in range(len(structs))])
        b.close()
    else:
        rng = np.random.default_rng(0)
        n = 4 * args.cell ** 3
        st = W.Structure(L.FCC, args.cell, L.SHELLS_FCC_TRUE3, [n // 4] * 4, W.WEIGHTS,
                         W.zero_row_sum_target(rng, 4, 0.05), P=32, Q=4096, I=1, D=20, name=f"fcc{args.cell}")
        plan = hb.Plan(st.problem(device=True, implicit=implicit), st.P, 1, st.Q, st.D, max_rounds=args.rounds,
                       hbm_occupancy=True)
        out = plan.run(123)
        plan.close()
    print(json.dumps(out))
    return 0


def main():
    args = parse_args()
    if args.case:
        return run_case(args)
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
    from pyhea_b200 import replicas

    l2_peak = hb.l2_read_probe(L2_PROBE_BYTES)
    st = workload(args.workload)
    problem = st.problem(device=True)
    nbor, sizes = st.neighbors(device=True)
    plan = hb.Plan(problem, st.P, st.I, st.Q, st.D, time_kernels=True, autotune=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for w in range(args.warmup):
        plan.run(replicas.replica_seed(rank, w))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    sampler = ClockSampler(local).start()
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
    lattice_code = plan.lattice
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

    dev = torch.device("cuda", local)
    total_ms_max, evals_all = replicas.combine(total_ms, evals, device=dev)
    e2e_ms_max, e2e_evals_all = replicas.combine(1000.0 * e2e_s, e2e_evals, device=dev)
    e2e_max = e2e_ms_max / 1000.0

    if rank == 0:
        B = st.evals_bytes()
        counters = KERNEL_COUNTERS.get(args.workload, {"dram": None, "capture": None})
        roof = roofline_of("mc_kernel (local search)", counters, evals, mc_ms / 1000.0, B, launches, clocks, l2_peak,
                           sm_count())
        roof["kernel_share"] = mc_ms / total_ms if total_ms else None
        line = {
            "metric": "swap_evals_per_sec", "value": evals_all / (total_ms_max / 1000.0), "unit": "swap-evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config_of(st, args.workload), parallelism=f"replicas x{world}",
                           local_search_block=block, neighbours=neighbours_of(lattice_code, False)),
            # kernels launched per search: 1 generate + per iteration (generate, search, merge, search,
            # sort), plus the iota of the slot order
            "gpu_launches": args.steps * (2 + 5 * st.I),
            "e2e": {"value": e2e_evals_all / e2e_max, "unit": "swap-evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": roof,
            "search": {"evals_per_step": evals / args.steps, "accepts_per_step": accepts / args.steps,
                       "best_fitness_last_step": float(best[0])},
            "clocks": clocks,
        }
        if world == 1:
            d = measure_dropin(st, nbor, sizes, replicas.replica_seed(rank, 30_000))
            d["value"] = (evals / args.steps) / (d["wall_ms"] / 1000.0)
            d["unit"] = "swap-evals/s"
            line["dropin_e2e"] = d
            line["time_to_tol"] = measure_time_to_tol(st, problem, replicas.replica_seed(rank, 20_000),
                                                      args.tol_iters)
            if not args.no_extras:
                cpu = workload("plain_cpu")
                line["time_to_tol_plain_cpu"] = measure_time_to_tol(cpu, cpu.problem(device=True), 20_000,
                                                                    args.tol_iters)
                line["batched"] = measure_batched(args.steps, args.warmup, l2_peak)
                line["batched"].pop("_raw", None)
                line["serving"] = measure_serving(args.serve_rate, args.serve_window, args.serve_solutions,
                                                  args.serve_iters, args.slice_ms)
                line["serving"]["capacity_per_s"] = line["serving"]["requests"]["per_s"]
                line["serving_sustained"] = measure_serving(args.serve_sustained_rate, args.serve_sustained_seconds,
                                                            args.serve_solutions, args.serve_iters, args.slice_ms)
                line["large"] = measure_large(args.large_iters)
            if not args.no_cpu_baseline:
                r = cpu_reference_sample(st, nbor, sizes, args.cpu_procs or host_cores())
                if r:
                    line["cpu_baseline"] = {"value": r["evals"] / r["wall_s"], "unit": "swap-evals/s",
                                            "cores": r["procs"], "kind": "reference", "sample": r["sample"]}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
