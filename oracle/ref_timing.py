"""Timing of the reference CPU engine (oracle/_ref/libref_accelerate.so).

TEST INFRASTRUCTURE ONLY: used by bench.py for its CPU baseline and for the
reference arm.  Swap evaluations are counted exactly: the harness counts the
engine's calls of its incremental fitness, one per scored proposal
(pyhea/cpp/accelerate.cpp:659-661).  The rand() call count is kept beside it as
a cross-check: the engine draws two values per attempt and redraws until the
species differ (:649-655), so evaluations ~ rand_calls / 2 * (1 - sum_t c_t^2).

Multi-core follows the reference's own MPI split (accelerate.cpp:728): K
independent single-rank processes, each searching its share of the
solutions; wall time is the slowest process.
"""
import ctypes
import multiprocessing as mp
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_accelerate.so")


def available():
    return os.path.exists(REF_LIB)


def _worker(job):
    (nbor, shell_size, species, weight, target, nnet, step, task, depth) = job
    # the engine logs every iteration on stdout; keep the benchmark's stdout clean
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_rand_calls.restype = ctypes.c_ulonglong
    lib.ref_eval_count.restype = ctypes.c_ulonglong
    P = ctypes.POINTER
    i32 = lambda a: a.ctypes.data_as(P(ctypes.c_int32))  # noqa: E731
    f64 = lambda a: a.ctypes.data_as(P(ctypes.c_double))  # noqa: E731
    n = int(species.sum())
    occ = np.zeros((nnet, n), dtype=np.int32)
    fit = np.zeros(nnet)
    lib.ref_reset_rand_calls()
    lib.ref_reset_eval_count()
    t0 = time.perf_counter()
    lib.ref_run_local_parallel_hcs(nnet, step, task, depth, ctypes.c_double(0.001), n, len(species), len(weight),
                                   i32(nbor), nbor.shape[1], i32(shell_size), i32(species), f64(weight), f64(target),
                                   i32(occ), f64(fit))
    wall = time.perf_counter() - t0
    return wall, int(lib.ref_rand_calls()), float(fit[0]), int(lib.ref_eval_count())


class RefPool:
    """A spawn-context process pool of `procs` workers running the reference engine."""

    def __init__(self, procs):
        self.procs = procs
        self.pool = mp.get_context("spawn").Pool(procs)

    def sample(self, nbor, shell_size, species, weight, target, nnet_per_proc, step, task, depth):
        """One bounded sample: every worker searches nnet_per_proc solutions.
        Returns dict(wall_s, evals, rand_calls, best_fitness)."""
        species = np.ascontiguousarray(species, dtype=np.int32)
        job = (np.ascontiguousarray(nbor, dtype=np.int32), np.ascontiguousarray(shell_size, dtype=np.int32), species,
               np.ascontiguousarray(weight, dtype=np.float64), np.ascontiguousarray(target, dtype=np.float64),
               int(nnet_per_proc), int(step), int(task), int(depth))
        t0 = time.perf_counter()
        res = self.pool.map(_worker, [job] * self.procs)
        wall = time.perf_counter() - t0
        calls = sum(r[1] for r in res)
        c = species / species.sum()
        p_valid = 1.0 - float(np.sum(c * c))
        return {"wall_s": max(max(r[0] for r in res), 1e-9), "pool_wall_s": wall, "rand_calls": calls,
                "evals": sum(r[3] for r in res), "evals_from_rand_calls": calls / 2.0 * p_valid,
                "best_fitness": min(r[2] for r in res)}

    def close(self):
        self.pool.close()
        self.pool.join()
