"""Small fixed cases of the search for profiler captures and quick checks.

    python -m pyhea_b200.cases plain [--iters 1]        one search of the plain GPU structure
    python -m pyhea_b200.cases batch [--count 16] [--iters 1]
                                                         the first `count` structures of the
                                                         mixed batch, one batched run
    python -m pyhea_b200.cases large [--cell 40] [--rounds 500]
                                                         one local search of an FCC cell^3
                                                         supercell on the HBM cluster path
                                                         (32 solutions x 4096 tasks)

Each prints its statistics (rounds, evaluations, accepts, device time) as one
line of JSON.
"""
import argparse
import json

import numpy as np

import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W


def plain(iters):
    st = W.plain_gpu(seed=0)
    plan = hb.Plan(st.problem(device=True), st.P, iters, st.Q, st.D)
    out = plan.run(123)
    plan.close()
    return out


def batch(count, iters):
    structs = sorted(W.batched(seed=0), key=lambda s: -s.num_sites)[:count]
    problems = [st.problem(device=True) for st in structs]
    params = [dict(num_solutions=st.P, total_iter=iters, parallel_task=st.Q, converge_depth=st.D) for st in structs]
    b = hb.Batch(problems, params)
    out = b.run([11 + i for i in range(count)])
    b.close()
    return out


def large(cell, rounds):
    rng = np.random.default_rng(0)
    n = 4 * cell ** 3
    st = W.Structure(L.FCC, cell, L.SHELLS_FCC_TRUE3, [n // 4] * 4, W.WEIGHTS, W.zero_row_sum_target(rng, 4, 0.05),
                     P=32, Q=4096, I=1, D=20, name=f"fcc{cell}")
    plan = hb.Plan(st.problem(device=True), st.P, 1, st.Q, st.D, max_rounds=rounds, hbm_occupancy=True)
    out = plan.run(123)
    plan.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["plain", "batch", "large"])
    ap.add_argument("--iters", type=int, default=1)
    ap.add_argument("--count", type=int, default=16)
    ap.add_argument("--cell", type=int, default=40)
    ap.add_argument("--rounds", type=int, default=500)
    a = ap.parse_args()
    if a.case == "plain":
        out = plain(a.iters)
    elif a.case == "batch":
        out = batch(a.count, a.iters)
    else:
        out = large(a.cell, a.rounds)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
