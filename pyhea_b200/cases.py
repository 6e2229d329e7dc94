"""Small fixed cases of the search for profiler captures and quick checks.

    python -m pyhea_b200.cases plain [--iters 1]        one search of the plain GPU structure
    python -m pyhea_b200.cases batch [--count 16] [--iters 1]
                                                         the first `count` structures of the
                                                         mixed batch, one batched run

Each prints its statistics (rounds, evaluations, accepts, device time) as one
line of JSON.
"""
import argparse
import json

import pyhea_b200 as hb
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["plain", "batch"])
    ap.add_argument("--iters", type=int, default=1)
    ap.add_argument("--count", type=int, default=16)
    a = ap.parse_args()
    out = plain(a.iters) if a.case == "plain" else batch(a.count, a.iters)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
