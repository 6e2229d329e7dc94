"""ctypes front end of the CPU restatement (oracle/hea_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product package.  Every function works
on numpy arrays; the neighbour table is the flattened int32 [N][sum Z] form
(shells concatenated per site, pyhea/lattice/lattice.py:196-323 order).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = ctypes.POINTER
u32, i32, i64, f64, u8 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_uint8


class _Problem(ctypes.Structure):
    _fields_ = [("num_sites", i32), ("num_types", i32), ("num_shells", i32), ("row", i32),
                ("nbor", P(i32)), ("shell_size", P(i32)), ("species", P(i32)), ("weight", P(f64)),
                ("E", P(f64)), ("R", P(f64))]


class Accept(ctypes.Structure):
    _fields_ = [("round", u32), ("task", u32), ("s1", u32), ("s2", u32), ("f2", f64)]


class _Stats(ctypes.Structure):
    _fields_ = [("rounds", i64), ("evals", i64), ("accepts", i64)]


def _load():
    from oracle.build_oracle import build_oracle  # local recipe; compiles once

    lib = ctypes.CDLL(build_oracle())
    lib.hea_oracle_f2.restype = f64
    lib.hea_oracle_delta.restype = f64
    lib.hea_oracle_draw_pair.restype = i64
    lib.hea_oracle_mc.restype = i64
    lib.hea_oracle_permute.restype = u32
    lib.hea_oracle_reject_threshold.restype = u32
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(P(ct))


def key_of(seed):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return (u32 * 2)(seed & 0xFFFFFFFF, seed >> 32)


def philox(ctr, key):
    o = (u32 * 4)()
    lib().hea_oracle_philox((u32 * 4)(*ctr), (u32 * 2)(*key), o)
    return list(o)


class Problem:
    """One structure: neighbour table, species counts, shell weights, target SRO."""

    def __init__(self, nbor, shell_size, species, weight, target):
        self.nbor = np.ascontiguousarray(nbor, dtype=np.int32)
        self.shell_size = np.ascontiguousarray(shell_size, dtype=np.int32)
        self.species = np.ascontiguousarray(species, dtype=np.int32)
        self.weight = np.ascontiguousarray(weight, dtype=np.float64)
        self.num_shells = len(self.weight)
        self.num_types = len(self.species)
        self.num_sites = int(self.species.sum())
        assert self.nbor.shape[0] == self.num_sites
        T, S = self.num_types, self.num_shells
        self.target = np.ascontiguousarray(np.asarray(target, dtype=np.float64).reshape(-1, T * T)[:S])
        self.E = np.zeros((S, T, T))
        self.R = np.zeros((S, T, T))
        lib().hea_oracle_tables(self.num_sites, T, S, _ptr(self.shell_size, i32), _ptr(self.species, i32),
                                _ptr(self.target, f64), _ptr(self.E, f64), _ptr(self.R, f64))
        self._c = _Problem(self.num_sites, T, S, self.nbor.shape[1], _ptr(self.nbor, i32), _ptr(self.shell_size, i32),
                           _ptr(self.species, i32), _ptr(self.weight, f64), _ptr(self.E, f64), _ptr(self.R, f64))

    @property
    def ncount(self):
        return self.num_shells * self.num_types * self.num_types

    def generate(self, seed, generation, slot):
        occ = np.zeros(self.num_sites, dtype=np.uint8)
        lib().hea_oracle_generate(key_of(seed), u32(generation), u32(slot), _ptr(self.species, i32), self.num_types,
                                  self.num_sites, _ptr(occ, u8))
        return occ

    def recount(self, occ):
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        C = np.zeros((self.num_shells, self.num_types, self.num_types), dtype=np.int32)
        lib().hea_oracle_recount(ctypes.byref(self._c), _ptr(occ, u8), _ptr(C, i32))
        return C

    def f2(self, C):
        C = np.ascontiguousarray(C, dtype=np.int32)
        return lib().hea_oracle_f2(ctypes.byref(self._c), _ptr(C, i32))

    def swap_counts(self, occ, C, s1, s2):
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        Cp = np.array(C, dtype=np.int32, copy=True)
        lib().hea_oracle_swap_counts(ctypes.byref(self._c), _ptr(occ, u8), u32(s1), u32(s2), _ptr(Cp, i32))
        return Cp

    def delta(self, occ, C, s1, s2):
        """D: the change of f2 swapping s1 and s2 makes, by the scoring contract (rank-2 form)."""
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        C = np.ascontiguousarray(C, dtype=np.int32)
        return lib().hea_oracle_delta(ctypes.byref(self._c), _ptr(occ, u8), _ptr(C, i32), u32(s1), u32(s2))

    def draw_pair(self, seed, stream, rnd, task, occ):
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        a, b = u32(), u32()
        att = lib().hea_oracle_draw_pair(key_of(seed), u32(stream), u32(rnd), u32(task), _ptr(occ, u8),
                                         u32(self.num_sites), ctypes.byref(a), ctypes.byref(b))
        return (int(att), a.value, b.value)

    def mc(self, seed, stream, occ, tasks, depth, max_rounds=1 << 30, trace_cap=0, trace_counts=False):
        """Search one occupancy (copied); returns dict with occ, counts, f2 (recomputed from the final
        counts), rounds, accepts, evals and the trace (round, task, s1, s2, running f2 after the swap)."""
        occ = np.array(occ, dtype=np.uint8, copy=True)
        C = self.recount(occ)
        f2 = f64(self.f2(C))
        tr = (Accept * max(trace_cap, 1))()
        tc = np.zeros((max(trace_cap, 1), self.num_shells, self.num_types, self.num_types), dtype=np.int32)
        acc, ev = i64(), i64()
        rounds = lib().hea_oracle_mc(ctypes.byref(self._c), key_of(seed), u32(stream), int(tasks), int(depth),
                                     i64(max_rounds), _ptr(occ, u8), _ptr(C, i32), ctypes.byref(f2),
                                     tr if trace_cap else None, _ptr(tc, i32) if (trace_cap and trace_counts) else None,
                                     i64(trace_cap), ctypes.byref(acc), ctypes.byref(ev))
        n = min(acc.value, trace_cap)
        trace = [(tr[i].round, tr[i].task, tr[i].s1, tr[i].s2, tr[i].f2) for i in range(n)]
        return {"occ": occ, "counts": C, "f2": f2.value, "rounds": int(rounds), "accepts": acc.value,
                "evals": ev.value, "trace": trace, "trace_counts": tc[:n] if trace_counts else None}

    def hcs(self, seed, num_solutions, total_iter, tasks, depth, max_rounds=1 << 30):
        """The whole search; returns (occ [P][N] uint8, f2 [P], stats dict)."""
        occ = np.zeros((num_solutions, self.num_sites), dtype=np.uint8)
        f2 = np.zeros(num_solutions)
        st = _Stats()
        rc = lib().hea_oracle_hcs(ctypes.byref(self._c), key_of(seed), int(num_solutions), int(total_iter), int(tasks),
                                  int(depth), i64(max_rounds), _ptr(occ, u8), _ptr(f2, f64), ctypes.byref(st))
        if rc != 0:
            raise MemoryError("oracle allocation failed")
        return occ, f2, {"rounds": st.rounds, "evals": st.evals, "accepts": st.accepts}


def permutation(seed, generation, slot, n):
    rk = (u32 * 6)()
    lib().hea_oracle_round_keys(key_of(seed), u32(generation), u32(slot), rk)
    return np.array([lib().hea_oracle_permute(u32(s), u32(n), rk) for s in range(n)], dtype=np.int64)
