"""B200-native SRO-targeted atom-swap search (the hot path of PyHEA).

Two front ends over one CUDA library (libhea_cuda.so, C ABI in include/hea_cuda.h):

* ``pyhea_b200.accelerate`` -- pybind11 module with the interface of
  ``pyhea.cpp.accelerate`` (pyhea/cpp/bind.cpp): ``run_local_parallel_hcs_cuda``
  and ``cuda_available``.  Drop it in as ``pyhea/cpp/accelerate*.so``.
* the ctypes functions below -- numpy-friendly calls of the same C ABI
  (``search``, ``Plan``, ``generate``, ``recount``, ``local_search``,
  ``build_neighbors``), used by the tests and the benchmark.

The CUDA library is loaded on first use -- any call below, or the ``lib`` and
``accelerate`` attributes -- and raises ImportError then when it has not been
built (``python pyhea_b200/build.py``); there is no CPU fallback.  Importing the
package, or its numpy-only modules (``lattice``, ``workloads``, ``sro``,
``output``), maps no shared library.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_PKG, "libhea_cuda.so")

_P = ctypes.POINTER
_i32, _i64, _u32, _u64, _f64, _u8 = (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_uint64,
                                     ctypes.c_double, ctypes.c_uint8)

HEA_OK, HEA_ERR_INVALID, HEA_ERR_UNSUPPORTED, HEA_ERR_CUDA, HEA_ERR_NOMEM, HEA_PENDING = 0, 1, 2, 3, 4, 5
HEA_FLAG_LOG_ITERS = 1
HEA_FLAG_TIME_KERNELS = 2
HEA_FLAG_HBM_OCCUPANCY = 4
HEA_FLAG_AUTOTUNE = 8
FCC, BCC = 0, 1
SHELLS_REFERENCE, SHELLS_FCC_TRUE3 = 0, 1


class HeaError(RuntimeError):
    """A failed C ABI call; ``code`` is the HEA_ERR_* value."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class HeaValueError(HeaError, ValueError):
    pass


class _Problem(ctypes.Structure):
    _fields_ = [("num_sites", _i32), ("num_types", _i32), ("num_shells", _i32), ("shell_sizes", _P(_i32)),
                ("nbor", _P(_i32)), ("species", _P(_i32)), ("weight", _P(_f64)), ("target_sro", _P(_f64)),
                ("implicit_lattice", _i32), ("lattice_cell", _i32), ("lattice_shell_set", _i32)]


class _Params(ctypes.Structure):
    _fields_ = [("num_solutions", _i32), ("total_iter", _i32), ("parallel_task", _i32), ("converge_depth", _i32),
                ("threshold", _f64), ("seed", _u64), ("max_rounds", _i64), ("flags", _i32)]


class Stats(ctypes.Structure):
    _fields_ = [("rounds", _i64), ("evals", _i64), ("accepts", _i64), ("gpu_ms", _f64), ("mc_ms", _f64),
                ("mc_launches", _i64)]

    def as_dict(self):
        return {"rounds": self.rounds, "evals": self.evals, "accepts": self.accepts, "gpu_ms": self.gpu_ms,
                "mc_ms": self.mc_ms, "mc_launches": self.mc_launches}


class AcceptRecord(ctypes.Structure):
    _fields_ = [("round", _u32), ("task", _u32), ("s1", _u32), ("s2", _u32), ("f2", _f64)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("max_requests", _i32), ("ring_jobs", _i32), ("arena_bytes", _i64), ("smem_bytes", _i32),
                ("hbm_sites", _i32), ("slice_ms", _f64), ("wait_limit_ms", _f64)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", _i32), ("iterations", _i32), ("hbm", _i32), ("pad_", _i32), ("submit_ms", _f64),
                ("admit_ms", _f64), ("finish_ms", _f64), ("device_ms", _f64), ("rounds", _i64), ("evals", _i64),
                ("accepts", _i64), ("device_bytes", _i64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class ServerStatus(ctypes.Structure):
    _fields_ = [("queued", _i32), ("running", _i32), ("finished_unread", _i32), ("slots_free", _i32),
                ("arena_free_bytes", _i64), ("arena_bytes", _i64), ("rounds", _i64), ("evals", _i64),
                ("accepts", _i64), ("finished", _i64), ("busy_ms", _f64), ("launches", _i32), ("smem_bytes", _i32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _declare(lib):
    sig = {
        "hea_cuda_available": (_i32, []),
        "hea_last_error": (ctypes.c_char_p, []),
        "hea_release_cached_memory": (None, []),
        "hea_run_local_parallel_hcs": (_i32, [_P(_Problem), _P(_Params), _P(_u8), _P(_f64), _P(Stats)]),
        "hea_plan_create": (_i32, [_P(_Problem), _P(_Params), _P(ctypes.c_void_p)]),
        "hea_plan_run": (_i32, [ctypes.c_void_p, _u64, _P(Stats)]),
        "hea_plan_read": (_i32, [ctypes.c_void_p, _P(_u8), _P(_f64)]),
        "hea_plan_destroy": (None, [ctypes.c_void_p]),
        "hea_plan_local_search_block": (_i32, [ctypes.c_void_p]),
        "hea_plan_lattice": (_i32, [ctypes.c_void_p]),
        "hea_generate": (_i32, [_P(_Problem), _u64, _u32, _i32, _P(_u8), _P(_i32), _P(_f64)]),
        "hea_recount": (_i32, [_P(_Problem), _i32, _P(_u8), _P(_i32), _P(_f64)]),
        "hea_local_search": (_i32, [_P(_Problem), _u64, _u32, _i32, _i32, _i32, _i64, _P(_u8), _P(_i32), _P(_f64),
                                    _P(_i64), _P(AcceptRecord), _P(_i32), _i64, _P(_i64)]),
        "hea_build_neighbors": (_i32, [_i32, _i32, _i32, _P(_i32), _P(_i32), _P(_i32)]),
        "hea_l2_read_probe": (_i32, [_i64, _i32, _P(_f64)]),
        "hea_dram_random_probe": (_i32, [_i64, _i32, _P(_f64)]),
        "hea_recount_noalloc": (_i32, [_P(_Problem), _i32, _P(_u8), _P(_i32), _P(_f64)]),
        "hea_batch_create": (_i32, [_P(_Problem), _P(_Params), _i32, _P(ctypes.c_void_p)]),
        "hea_batch_run": (_i32, [ctypes.c_void_p, _P(_u64), _P(Stats)]),
        "hea_batch_read": (_i32, [ctypes.c_void_p, _i32, _P(_u8), _P(_f64)]),
        "hea_batch_finish_times": (_i32, [ctypes.c_void_p, _P(_f64)]),
        "hea_batch_tallies": (_i32, [ctypes.c_void_p, _P(_u64)]),
        "hea_batch_autotune": (_i32, [ctypes.c_void_p, _P(_i32), _P(_i32)]),
        "hea_batch_set_wait_limit": (_i32, [ctypes.c_void_p, _f64]),
        "hea_batch_destroy": (None, [ctypes.c_void_p]),
        "hea_server_create": (_i32, [_P(_ServerConfig), _P(ctypes.c_void_p)]),
        "hea_server_submit": (_i32, [ctypes.c_void_p, _P(_Problem), _P(_Params), _f64, _i32, _P(_i64)]),
        "hea_server_submit_lattice": (_i32, [ctypes.c_void_p, _i32, _i32, _i32, _i32, _i32, _P(_i32), _P(_f64),
                                             _P(_f64), _P(_Params), _f64, _i32, _P(_i64)]),
        "hea_server_step": (_i32, [ctypes.c_void_p, _P(_i32)]),
        "hea_server_take_finished": (_i32, [ctypes.c_void_p, _P(_i64), _i32, _P(_i32)]),
        "hea_server_result": (_i32, [ctypes.c_void_p, _i64, _P(_u8), _P(_f64), _P(RequestInfo)]),
        "hea_server_info": (_i32, [ctypes.c_void_p, _i64, _P(RequestInfo)]),
        "hea_server_status_get": (_i32, [ctypes.c_void_p, _P(ServerStatus)]),
        "hea_server_destroy": (None, [ctypes.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def _load():
    """The CUDA library with its C ABI declared; loaded on the first call."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(f"{_LIB_PATH} is missing; build it with `python pyhea_b200/build.py`")
        _lib = _declare(ctypes.CDLL(_LIB_PATH))
    return _lib


def __getattr__(name):
    if name == "lib":
        return _load()
    if name == "accelerate":  # pybind11 module next to the library; it links the library itself
        import importlib

        _load()
        return importlib.import_module(".accelerate", __name__)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def _check(rc):
    if rc != HEA_OK:
        msg = _load().hea_last_error().decode()
        raise (HeaValueError if rc == HEA_ERR_INVALID else HeaError)(rc, msg)


def cuda_available():
    return bool(_load().hea_cuda_available())


def _ptr(a, ct):
    return a.ctypes.data_as(_P(ct)) if a is not None else None


class Problem:
    """One structure: flattened neighbour table [N][sum Z], shell sizes, species
    counts, shell weights and target alpha [S][T*T] (the reference's nbor,
    element, weight and target_sro with nbor cut to len(weight) shells).

    ``Problem.from_lattice`` describes a perfect FCC/BCC cube instead of giving a
    table: the device computes neighbour ids from lattice arithmetic and stores
    no table (same results as with the table ``build_neighbors`` makes).  A
    table that is such a cube's (every shell holding the lattice's ids, in any
    order -- PyHEA's tables are) is recognised and run the same way unless
    ``recognize=False``."""

    def __init__(self, nbor, shell_sizes, species, weight, target_sro, lattice=None, recognize=True):
        self.species = np.ascontiguousarray(species, dtype=np.int32)
        self.weight = np.ascontiguousarray(weight, dtype=np.float64)
        S, T = len(self.weight), len(self.species)
        sizes = np.asarray(shell_sizes, dtype=np.int32)
        self.shell_sizes = np.ascontiguousarray(sizes[:S])
        if nbor is None:
            self.nbor = None
        else:
            nb = np.asarray(nbor)
            self.nbor = np.ascontiguousarray(nb[:, : int(self.shell_sizes.sum())], dtype=np.int32)
        self.target_sro = np.ascontiguousarray(np.asarray(target_sro, dtype=np.float64).reshape(-1, T * T)[:S])
        self.num_sites = int(self.species.sum())
        self.num_types, self.num_shells = T, S
        self.lattice = lattice  # (FCC | BCC, cell, shell_set) of an implicit-neighbour problem, else None
        kind, cell, shell_set = (lattice[0] + 1, lattice[1], lattice[2]) if lattice is not None else (0, 0, 0)
        if lattice is None and self.nbor is not None and not recognize:
            kind = -1  # the table as given
        self._c = _Problem(self.num_sites, T, S, _ptr(self.shell_sizes, _i32), _ptr(self.nbor, _i32),
                           _ptr(self.species, _i32), _ptr(self.weight, _f64), _ptr(self.target_sro, _f64),
                           int(kind), int(cell), int(shell_set))

    @classmethod
    def from_lattice(cls, lattice, cell, species, weight, target_sro, shell_set=SHELLS_REFERENCE):
        """Implicit-neighbour problem of the FCC (0) / BCC (1) cube of edge `cell`."""
        from . import lattice as _lat

        sizes = [len(v) for v in _lat.shell_vectors(lattice, shell_set)]
        return cls(None, sizes, species, weight, target_sro, lattice=(int(lattice), int(cell), int(shell_set)))

    @property
    def ncount(self):
        return self.num_shells * self.num_types * self.num_types


def _params(num_solutions, total_iter, parallel_task, converge_depth, seed, max_rounds=0, flags=0, threshold=0.001):
    return _Params(int(num_solutions), int(total_iter), int(parallel_task), int(converge_depth), float(threshold),
                   int(seed) & 0xFFFFFFFFFFFFFFFF, int(max_rounds), int(flags))


def search(problem, num_solutions, total_iter, parallel_task, converge_depth, seed=0, max_rounds=0, log=False,
           out_occ=None, out_fitness=None, time_kernels=False, hbm_occupancy=False):
    """The whole search with host buffers (hea_run_local_parallel_hcs).
    Returns (occ [P][N] uint8, fitness [P] float64, stats dict)."""
    P, N = int(num_solutions), problem.num_sites
    occ = out_occ if out_occ is not None else np.empty((P, N), dtype=np.uint8)
    fit = out_fitness if out_fitness is not None else np.empty(P, dtype=np.float64)
    st = Stats()
    flags = ((HEA_FLAG_LOG_ITERS if log else 0) | (HEA_FLAG_TIME_KERNELS if time_kernels else 0) |
             (HEA_FLAG_HBM_OCCUPANCY if hbm_occupancy else 0))
    prm = _params(P, total_iter, parallel_task, converge_depth, seed, max_rounds, flags)
    _check(_load().hea_run_local_parallel_hcs(ctypes.byref(problem._c), ctypes.byref(prm), _ptr(occ, _u8),
                                          _ptr(fit, _f64), ctypes.byref(st)))
    return occ, fit, st.as_dict()


class Plan:
    """Device-resident search (hea_plan_*): tables uploaded once, run many times."""

    def __init__(self, problem, num_solutions, total_iter, parallel_task, converge_depth, seed=0, max_rounds=0,
                 time_kernels=False, hbm_occupancy=False, autotune=False):
        self.problem = problem
        self.P = int(num_solutions)
        self._h = ctypes.c_void_p()
        flags = ((HEA_FLAG_TIME_KERNELS if time_kernels else 0) | (HEA_FLAG_HBM_OCCUPANCY if hbm_occupancy else 0)
                 | (HEA_FLAG_AUTOTUNE if autotune else 0))
        prm = _params(num_solutions, total_iter, parallel_task, converge_depth, seed, max_rounds, flags)
        _check(_load().hea_plan_create(ctypes.byref(problem._c), ctypes.byref(prm), ctypes.byref(self._h)))

    @property
    def lattice(self):
        """Neighbours the plan runs on: 0 its table, 1 FCC / 2 BCC lattice arithmetic (implicit, or a
        recognised lattice table)."""
        return int(_load().hea_plan_lattice(self._h))

    @property
    def local_search_block(self):
        """Threads per CTA of the local search (the autotuner's pick when autotune=True)."""
        return int(_load().hea_plan_local_search_block(self._h))

    def run(self, seed):
        st = Stats()
        _check(_load().hea_plan_run(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(st)))
        return st.as_dict()

    def read(self):
        occ = np.empty((self.P, self.problem.num_sites), dtype=np.uint8)
        fit = np.empty(self.P, dtype=np.float64)
        _check(_load().hea_plan_read(self._h, _ptr(occ, _u8), _ptr(fit, _f64)))
        return occ, fit

    def close(self):
        if self._h:
            _load().hea_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many structures searched together by one persistent kernel (hea_batch_*).

    problems: list of Problem; params: list of dicts with num_solutions,
    total_iter, parallel_task, converge_depth (and optional max_rounds).  Each
    structure's result equals search() on it alone with the same seed."""

    def __init__(self, problems, params):
        self.problems = list(problems)
        n = len(self.problems)
        self._pb = (_Problem * n)(*[p._c for p in self.problems])
        self._prm = (_Params * n)(*[_params(q["num_solutions"], q["total_iter"], q["parallel_task"],
                                            q["converge_depth"], 0, q.get("max_rounds", 0)) for q in params])
        self.P = [int(q["num_solutions"]) for q in params]
        self._h = ctypes.c_void_p()
        _check(_load().hea_batch_create(self._pb, self._prm, n, ctypes.byref(self._h)))

    def run(self, seeds):
        arr = (_u64 * len(self.problems))(*[int(s) & 0xFFFFFFFFFFFFFFFF for s in seeds])
        st = Stats()
        _check(_load().hea_batch_run(self._h, arr, ctypes.byref(st)))
        return st.as_dict()

    def read(self, index):
        occ = np.empty((self.P[index], self.problems[index].num_sites), dtype=np.uint8)
        fit = np.empty(self.P[index], dtype=np.float64)
        _check(_load().hea_batch_read(self._h, int(index), _ptr(occ, _u8), _ptr(fit, _f64)))
        return occ, fit

    def autotune(self):
        """Time the launch configurations on full runs (current seeds) and keep the fastest;
        returns {"hbm_all": 0|1, "ctas_per_sm": n}.  Results do not depend on it."""
        h, c = _i32(), _i32()
        _check(_load().hea_batch_autotune(self._h, ctypes.byref(h), ctypes.byref(c)))
        return {"hbm_all": h.value, "ctas_per_sm": c.value}

    def set_wait_limit(self, ms):
        """Bound (ms) on every wait of the persistent kernel for queued work; a run whose wait runs
        out raises HeaError and leaves the batch ready for the next run."""
        _check(_load().hea_batch_set_wait_limit(self._h, float(ms)))

    def finish_times(self):
        """Milliseconds from the start of the last run to each structure's end."""
        out = np.empty(len(self.problems))
        _check(_load().hea_batch_finish_times(self._h, _ptr(out, _f64)))
        return out

    def tallies(self):
        """Per structure of the last run: [rounds, swap evaluations, accepted swaps] (uint64 [count][3])."""
        out = np.empty((len(self.problems), 3), dtype=np.uint64)
        _check(_load().hea_batch_tallies(self._h, _ptr(out, _u64)))
        return out

    def close(self):
        if self._h:
            _load().hea_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop (hea_server_*): searches submitted while others run.

    ``submit`` / ``submit_lattice`` queue a request and return its id;
    ``step`` admits queued requests as request slots, arena memory and job-ring
    room free up, runs one time slice of the persistent kernel and returns the
    ids that finished; ``result`` hands over (occupancies [P][N] ascending by
    fitness, fitness [P], info dict) once and releases the request.  A request's
    result equals search() on it alone with the same seed (with a tolerance:
    with total_iter = info["iterations"])."""

    def __init__(self, max_requests=0, ring_jobs=0, arena_bytes=0, smem_bytes=0, slice_ms=0.0, hbm_sites=0,
                 wait_limit_ms=0.0):
        cfg = _ServerConfig(int(max_requests), int(ring_jobs), int(arena_bytes), int(smem_bytes), int(hbm_sites),
                            float(slice_ms), float(wait_limit_ms))
        self._h = ctypes.c_void_p()
        _check(_load().hea_server_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self._meta = {}  # id -> (P, N)

    @staticmethod
    def _prm(params):
        return _params(params["num_solutions"], params["total_iter"], params["parallel_task"],
                       params["converge_depth"], params.get("seed", 0), params.get("max_rounds", 0))

    def submit(self, problem, params, tolerance=-1.0, priority=0):
        prm = self._prm(params)
        rid = _i64()
        _check(_load().hea_server_submit(self._h, ctypes.byref(problem._c), ctypes.byref(prm), float(tolerance),
                                     int(priority), ctypes.byref(rid)))
        self._meta[rid.value] = (int(params["num_solutions"]), problem.num_sites)
        return rid.value

    def submit_lattice(self, lattice, cell, species, weight, target_sro, params, shell_set=SHELLS_REFERENCE,
                       tolerance=-1.0, priority=0):
        sp = np.ascontiguousarray(species, dtype=np.int32)
        w = np.ascontiguousarray(weight, dtype=np.float64)
        tg = np.ascontiguousarray(target_sro, dtype=np.float64)
        T, S = sp.size, w.size
        if tg.size != S * T * T:
            raise ValueError(f"target_sro needs {S}*{T}*{T} values, got {tg.size}")
        prm = self._prm(params)
        rid = _i64()
        _check(_load().hea_server_submit_lattice(self._h, int(lattice), int(cell), int(shell_set), T, S, _ptr(sp, _i32),
                                             _ptr(w, _f64), _ptr(tg, _f64), ctypes.byref(prm), float(tolerance),
                                             int(priority), ctypes.byref(rid)))
        n = (4 if lattice == FCC else 2) * int(cell) ** 3
        self._meta[rid.value] = (int(params["num_solutions"]), n)
        return rid.value

    def step(self):
        """Wait for the previous time slice, hand over its finished requests, admit queued ones and
        launch the next slice (not waited for); returns the number of requests that finished."""
        fin = _i32()
        _check(_load().hea_server_step(self._h, ctypes.byref(fin)))
        return fin.value

    def take_finished(self, cap=4096):
        """Ids of requests that finished (or failed) since the last call."""
        ids = (_i64 * cap)()
        n = _i32()
        _check(_load().hea_server_take_finished(self._h, ids, int(cap), ctypes.byref(n)))
        return list(ids[: n.value])

    def info(self, rid):
        inf = RequestInfo()
        _check(_load().hea_server_info(self._h, int(rid), ctypes.byref(inf)))
        return inf.as_dict()

    def result(self, rid):
        """(occ, fitness, info) of a finished request, or None while it is queued or running."""
        P, n = self._meta.get(rid, (0, 0))
        occ = np.empty((P, n), dtype=np.uint8)
        fit = np.empty(P, dtype=np.float64)
        inf = RequestInfo()
        rc = _load().hea_server_result(self._h, int(rid), _ptr(occ, _u8), _ptr(fit, _f64), ctypes.byref(inf))
        if rc == HEA_PENDING:
            return None
        self._meta.pop(rid, None)
        _check(rc)
        return occ, fit, inf.as_dict()

    def status(self):
        st = ServerStatus()
        _check(_load().hea_server_status_get(self._h, ctypes.byref(st)))
        return st.as_dict()

    def drain(self, max_steps=1 << 30):
        """Step until nothing is queued or running."""
        for _ in range(max_steps):
            st = self.status()
            if st["queued"] == 0 and st["running"] == 0:
                return
            self.step()
        raise HeaError(HEA_ERR_CUDA, "server did not drain")

    def close(self):
        if self._h:
            _load().hea_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate(problem, seed, generation, count):
    """hea_generate: (occ [count][N], counts [count][S][T][T], f2 [count])."""
    occ = np.empty((count, problem.num_sites), dtype=np.uint8)
    cnt = np.empty((count, problem.num_shells, problem.num_types, problem.num_types), dtype=np.int32)
    f2 = np.empty(count)
    _check(_load().hea_generate(ctypes.byref(problem._c), int(seed), int(generation), int(count), _ptr(occ, _u8),
                            _ptr(cnt, _i32), _ptr(f2, _f64)))
    return occ, cnt, f2


def _rows(problem, occ):
    """Occupancies as a contiguous uint8 [count][N] array; N must be the problem's site count
    (the C ABI reads exactly count x N bytes)."""
    occ = np.ascontiguousarray(np.atleast_2d(occ), dtype=np.uint8)
    if occ.ndim != 2 or occ.shape[1] != problem.num_sites:
        raise ValueError(f"occupancies must be [count][{problem.num_sites}], got shape {occ.shape}")
    return occ


def recount(problem, occ):
    """hea_recount: (counts [count][S][T][T], f2 [count]) of occupancies [count][N]."""
    occ = _rows(problem, occ)
    count = occ.shape[0]
    cnt = np.empty((count, problem.num_shells, problem.num_types, problem.num_types), dtype=np.int32)
    f2 = np.empty(count)
    _check(_load().hea_recount(ctypes.byref(problem._c), int(count), _ptr(occ, _u8), _ptr(cnt, _i32), _ptr(f2, _f64)))
    return cnt, f2


def local_search(problem, seed, mc_call, occ, tasks, depth, max_rounds=0, trace_cap=0, trace_counts=False):
    """hea_local_search on occupancies [count][N] (copied).  Returns a dict with
    occ, counts, f2, rounds and, when trace_cap > 0, per-occupancy traces."""
    occ = np.array(_rows(problem, occ), copy=True)
    count = occ.shape[0]
    cnt = np.empty((count, problem.num_shells, problem.num_types, problem.num_types), dtype=np.int32)
    f2 = np.empty(count)
    rounds = np.empty(count, dtype=np.int64)
    tr = (AcceptRecord * max(1, count * trace_cap))() if trace_cap else None
    tc = (np.empty((count, trace_cap, problem.num_shells, problem.num_types, problem.num_types), dtype=np.int32)
          if trace_cap and trace_counts else None)
    tlen = np.zeros(count, dtype=np.int64) if trace_cap else None
    _check(_load().hea_local_search(ctypes.byref(problem._c), int(seed), int(mc_call), int(count), int(tasks), int(depth),
                                int(max_rounds), _ptr(occ, _u8), _ptr(cnt, _i32), _ptr(f2, _f64), _ptr(rounds, _i64),
                                tr, _ptr(tc, _i32), int(trace_cap), _ptr(tlen, _i64)))
    out = {"occ": occ, "counts": cnt, "f2": f2, "rounds": rounds}
    if trace_cap:
        traces = []
        for p in range(count):
            n = int(min(tlen[p], trace_cap))
            recs = [tr[p * trace_cap + i] for i in range(n)]
            traces.append([(r.round, r.task, r.s1, r.s2, r.f2) for r in recs])
        out["trace"] = traces
        out["trace_len"] = tlen
        out["trace_counts"] = tc
    return out


def recount_noalloc(problem, occ):
    """hea_recount_noalloc: the same results as recount() from a fixed static
    device array instead of allocated buffers (for callers that cannot
    allocate device memory)."""
    occ = _rows(problem, occ)
    count = occ.shape[0]
    cnt = np.empty((count, problem.num_shells, problem.num_types, problem.num_types), dtype=np.int32)
    f2 = np.empty(count)
    _check(_load().hea_recount_noalloc(ctypes.byref(problem._c), int(count), _ptr(occ, _u8), _ptr(cnt, _i32),
                                   _ptr(f2, _f64)))
    return cnt, f2


def build_neighbors(lattice, cell, shell_set=SHELLS_REFERENCE):
    """Device-built neighbour table of an FCC (0) / BCC (1) cube of edge `cell`:
    (nbor int32 [N][sum Z], shell_sizes int32 [3])."""
    sizes = np.zeros(3, dtype=np.int32)
    n = _i32()
    _check(_load().hea_build_neighbors(int(lattice), int(cell), int(shell_set), None, _ptr(sizes, _i32), ctypes.byref(n)))
    nbor = np.empty((n.value, int(sizes.sum())), dtype=np.int32)
    _check(_load().hea_build_neighbors(int(lattice), int(cell), int(shell_set), _ptr(nbor, _i32), _ptr(sizes, _i32),
                                   ctypes.byref(n)))
    return nbor, sizes


def l2_read_probe(nbytes=32 << 20, reps=50):
    """hea_l2_read_probe: L2 read bandwidth of the current device in GB/s (a buffer of
    `nbytes` that fits in L2, read `reps` times by every SM)."""
    out = _f64()
    _check(_load().hea_l2_read_probe(int(nbytes), int(reps), ctypes.byref(out)))
    return out.value


def dram_random_probe(nbytes=4 << 30, per_thread=256):
    """hea_dram_random_probe: random 16-byte loads per second from a buffer of `nbytes` in DRAM
    (the best of L2-cached and evict-first loads at 8 and 32 CTAs per SM)."""
    out = _f64()
    _check(_load().hea_dram_random_probe(int(nbytes), int(per_thread), ctypes.byref(out)))
    return out.value
