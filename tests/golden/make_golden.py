"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has the reference tree (HEA_REFERENCE_ROOT, else a
checkout named `reference` beside this repository) and the reference CPU engine built by
oracle/build_oracle.py:

    python oracle/build_oracle.py && python tests/golden/make_golden.py

Fixtures written:
  nbor_ref.npz       neighbour lists produced by the reference lattice builder
                     (pyhea/lattice/lattice.py:196-323) for FCC/BCC cells of edge 3 and 4
  target_sro.json    lower-triangle TARGET_SRO files expanded by the reference
                     config reader (pyhea/io/input.py:350-465) for 2-4 species
  ref_engine.npz     per-case occupancies and swaps with the reference engine's
                     gamma (accelerate.cpp:370-399), full fitness (:118-180) and
                     incremental fitness (:498-570)
  poscar_*.txt       POSCAR files written by the reference writer
                     (pyhea/io/output.py:62-106) for seeded occupancies of FCC and
                     BCC cells (`python tests/golden/make_golden.py poscar` writes
                     only these)
  opt_call.json      the positional call the reference's own driver makes into its engine
                     (pyhea/model/opt.py:87-90, device: gpu), recorded by running
                     opt_model.run_optimization on an FCC 4^3 configuration read by the
                     reference config reader, with a recording stand-in in place of
                     pyhea.cpp.accelerate (`python tests/golden/make_golden.py opt` writes
                     only this)
  lammps_conf.json   the reference's sample LAMMPS output (examples/conf.lmp, FCC
                     10^3, 4 species): its occupancy in the reference lattice's site
                     order, its lattice constant and the SHA-256 of its text
                     (`python tests/golden/make_golden.py lammps` writes only this)

The reference's Python modules import mpi4py, OVITO, dpdata and matplotlib at
module level; none is needed by the two functions used here, so they are
replaced by stubs in sys.modules before the import.
"""
import ctypes
import json
import os
import sys
import tempfile
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE_ROOT = os.environ.get("HEA_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO), "reference")


def import_reference():
    for name in ["mpi4py", "ovito", "ovito.io", "ovito.modifiers", "ovito.data", "WarrenCowleyParameters", "dpdata",
                 "matplotlib", "matplotlib.pyplot", "psutil"]:
        sys.modules.setdefault(name, mock.MagicMock())
    sys.path.insert(0, REFERENCE_ROOT)
    from pyhea.lattice.lattice import lattice  # noqa: E402
    from pyhea.io.input import input_config  # noqa: E402
    return lattice, input_config


def flat_nbor(nbor):
    return np.array([np.concatenate([np.asarray(sh, dtype=np.int64) for sh in site]) for site in nbor], dtype=np.int32)


POSCAR_CASES = [("poscar_fcc3_t4.txt", "FCC", 3, 4, 11), ("poscar_bcc4_t3.txt", "BCC", 4, 3, 12)]


def poscar_fixtures(lattice):
    from pyhea.io.output import write_poscar  # noqa: E402

    for name, typ, L, T, seed in POSCAR_CASES:
        lat = lattice([L, L, L], typ, 3.6, np.eye(3) * L)
        n = len(lat.coords)
        occ = np.random.default_rng(seed).integers(0, T, size=n)
        write_poscar([int(x) for x in occ], lat, T, [f"E{t}" for t in range(T)], os.path.join(HERE, name))


def lammps_fixture(lattice):
    import hashlib

    path = os.path.join(REFERENCE_ROOT, "examples", "conf.lmp")
    text = open(path).read()
    lines = text.splitlines()
    n = int(lines[1].split()[0])
    T = int(lines[2].split()[0])
    edge = float(lines[3].split()[1])
    cell = 10
    a = edge / cell
    lat = lattice([cell, cell, cell], "FCC", a, np.eye(3) * cell)
    coords = np.asarray(lat.coords, dtype=np.float64)  # cell units, multiples of 1/2
    assert len(coords) == n
    site_of = {tuple(int(round(2 * v)) for v in xyz): i for i, xyz in enumerate(coords)}
    occ = np.full(n, -1, dtype=np.int64)
    start = lines.index("Atoms # atomic") + 2
    for ln in lines[start:start + n]:
        _, typ, x, y, z = ln.split()
        occ[site_of[tuple(int(round(2 * float(v) / a)) for v in (x, y, z))]] = int(typ) - 1
    assert occ.min() >= 0
    fixture = {"source": "examples/conf.lmp", "lattice": "FCC", "cell": cell, "lattice_constant": a, "num_types": T,
               "occupancy": "".join(str(int(t)) for t in occ), "sha256": hashlib.sha256(text.encode()).hexdigest(),
               "head": lines[:11], "tail": lines[-2:]}
    with open(os.path.join(HERE, "lammps_conf.json"), "w") as f:
        json.dump(fixture, f, indent=1)


def opt_call_fixture():
    """Run the reference's opt_model.run_optimization (device: gpu) with a stand-in engine module
    that records the positional arguments of run_local_parallel_hcs_cuda and returns a valid
    population, so the driver completes (and writes its POSCAR) as it would with a real engine."""
    import types

    calls = []

    def run_cuda(*args):
        calls.append(args)
        nnet, element = args[0], args[6]
        occ = [t for t, c in enumerate(element) for _ in range(c)]
        rng = np.random.default_rng(0)
        latts = [[int(x) for x in rng.permutation(occ)] for _ in range(nnet)]
        return latts, [0.1 * (i + 1) for i in range(nnet)]

    fake = types.ModuleType("pyhea.cpp.accelerate")
    fake.run_local_parallel_hcs_cuda = run_cuda
    fake.cuda_available = lambda: True
    fake.run_local_parallel_hcs = None
    sys.modules["pyhea.cpp.accelerate"] = fake
    lattice, input_config = import_reference()
    import pyhea.cpp  # noqa: E402  (package of the stand-in)

    pyhea.cpp.accelerate = fake
    import pyhea.io.input as reference_input  # noqa: E402
    from pyhea.model.opt import opt_model  # noqa: E402

    # the config reader falls back to device: cpu unless it sees a GPU; this machine has none
    reference_input.get_gpu_info = lambda: [{"name": "NVIDIA B200", "memory": "183359 MiB", "driver": "580"}]

    class OneRank:  # mpi4py.MPI.COMM_WORLD of a single process
        def Get_rank(self):
            return 0

        def Get_size(self):
            return 1

    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        cfg = os.path.join(tmp, "config.yaml")
        with open(cfg, "w") as f:
            f.write("type: 4\nelement: [64, 64, 64, 64]\ncell_dim: [4, 4, 4]\ndevice: gpu\nsolutions: 4\n"
                    "total_iter: 2\nparallel_task: 32\nconverge_depth: 4\nweight: [4.0, 1.0, 0.5]\n"
                    f"structure: {os.path.join(REFERENCE_ROOT, 'examples', 'POSCAR_FCC')}\n"
                    f"target_sro: {os.path.join(REFERENCE_ROOT, 'examples', 'TARGET_SRO')}\n")
        conf = input_config(cfg)
        latt = lattice(conf.cell_dim, conf.latt_type, conf.latt_const, conf.latt_vectors, valid=True)
        os.chdir(tmp)
        try:
            opt_model(latt, conf, OneRank()).run_optimization()
            written = sorted(os.listdir(tmp))
        finally:
            os.chdir(cwd)
    assert len(calls) == 1
    args = calls[0]
    def kind(a):  # type of an argument down to its innermost containers, e.g. "list[list[ndarray(int64)]]"
        if isinstance(a, np.ndarray):
            return f"ndarray({a.dtype})"
        if isinstance(a, (list, tuple)):
            return f"{type(a).__name__}[{kind(a[0])}]" if len(a) else f"{type(a).__name__}[]"
        return type(a).__name__

    def plain(a):
        if isinstance(a, np.ndarray):
            return a.tolist()
        if isinstance(a, (list, tuple)):
            return [plain(x) for x in a]
        return a.item() if isinstance(a, np.generic) else a

    kinds = [kind(a) for a in args]
    as_json = [plain(a) for a in args]
    with open(os.path.join(HERE, "opt_call.json"), "w") as f:
        json.dump({"source": "pyhea/model/opt.py:87-90 (device: gpu), FCC 4^3 from examples/POSCAR_FCC, "
                             "target from examples/TARGET_SRO", "arg_types": kinds, "args": as_json,
                   "files_written": written}, f)


def main():
    if sys.argv[1:] == ["opt"]:
        opt_call_fixture()
        return
    lattice, input_config = import_reference()
    if sys.argv[1:] == ["poscar"]:
        poscar_fixtures(lattice)
        return
    if sys.argv[1:] == ["lammps"]:
        lammps_fixture(lattice)
        return
    poscar_fixtures(lattice)
    lammps_fixture(lattice)
    opt_call_fixture()

    # 1. neighbour lists
    nb = {}
    for typ in ("FCC", "BCC"):
        for L in (3, 4):
            lat = lattice([L, L, L], typ, 1.0, np.eye(3) * L)
            nb[f"{typ}_{L}"] = flat_nbor(lat.nbor_list)
            nb[f"{typ}_{L}_shells"] = np.array([len(s) for s in lat.nbor_list[0]], dtype=np.int32)
    np.savez_compressed(os.path.join(HERE, "nbor_ref.npz"), **nb)

    # 2. TARGET_SRO expansion (lower triangle per shell -> full T*T matrices)
    cases = {}
    with tempfile.TemporaryDirectory() as tmp:
        for T in (2, 3, 4):
            m = T * (T + 1) // 2
            shells = [[round(0.01 * (k + 1) * (q + 1) - 0.05, 4) for q in range(m)] for k in range(3)]
            lines = []
            for k, vals in enumerate(shells):
                lines.append(["First Shell", "Second Shell", "Third Shell"][k])
                pos = 0
                for row in range(T):
                    lines.append(" ".join(str(v) for v in vals[pos:pos + row + 1]))
                    pos += row + 1
            path = os.path.join(tmp, f"TARGET_SRO_{T}")
            with open(path, "w") as f:
                f.write("\n".join(lines) + "\n")
            cfg = object.__new__(input_config)
            cfg.config = {"type": T, "target_sro": path}
            cwd = os.getcwd()
            os.chdir("/")
            try:
                full = np.asarray(cfg.target_sro, dtype=float)
            finally:
                os.chdir(cwd)
            cases[str(T)] = {"lower": shells, "full": full.tolist()}
        cfg = object.__new__(input_config)
        cfg.config = {"type": 4}
        cases["default_4"] = {"lower": None, "full": np.asarray(cfg.target_sro, dtype=float).tolist()}
    with open(os.path.join(HERE, "target_sro.json"), "w") as f:
        json.dump(cases, f, indent=1)

    # 3. reference engine functions on fixed occupancies and swaps
    ref = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_accelerate.so"))
    ref.ref_fitness_incremental.restype = ctypes.c_double
    P = ctypes.POINTER
    i32 = lambda a: a.ctypes.data_as(P(ctypes.c_int32))  # noqa: E731
    f64 = lambda a: a.ctypes.data_as(P(ctypes.c_double))  # noqa: E731
    rng = np.random.default_rng(20241203)
    specs = [
        ("fcc4_t4_s3", "FCC_4", [64, 64, 64, 64], [4.0, 1.0, 0.5]),
        ("bcc4_t3_s2", "BCC_4", [40, 44, 44], [1.0, 0.5]),
        ("fcc3_t5_s3", "FCC_3", [20, 22, 22, 22, 22], [4.0, 1.0, 0.5]),
        ("bcc4_t6_s3", "BCC_4", [20, 20, 20, 20, 24, 24], [2.0, 1.0, 0.25]),
        ("fcc4_t2_s1", "FCC_4", [100, 156], [1.0]),
    ]
    out = {}
    for name, key, species, weight in specs:
        nbor_full = nb[key]
        shells_full = nb[key + "_shells"]
        S = len(weight)
        T = len(species)
        N = int(sum(species))
        assert N == nbor_full.shape[0]
        shell_size = shells_full[:S].copy()
        nbor = np.ascontiguousarray(nbor_full[:, : int(shell_size.sum())])
        row = nbor.shape[1]
        tgt = rng.uniform(-0.2, 0.2, size=(S, T, T))
        tgt = 0.5 * (tgt + tgt.transpose(0, 2, 1))
        target = np.ascontiguousarray(tgt.reshape(S, T * T))
        sp = np.array(species, dtype=np.int32)
        w = np.array(weight, dtype=np.float64)
        layout = np.repeat(np.arange(T, dtype=np.int32), species)
        occs = np.stack([rng.permutation(layout) for _ in range(4)]).astype(np.int32)
        gam = np.zeros((4, T, T, S))
        for p in range(4):
            ref.ref_recount(N, T, S, i32(nbor), row, i32(shell_size), i32(sp), i32(np.ascontiguousarray(occs[p])),
                            f64(gam[p]))
        fit = np.zeros(4)
        ref.ref_fitness_of_solutions(4, N, T, S, i32(nbor), row, i32(shell_size), i32(sp), f64(w), f64(target),
                                     i32(occs), f64(fit))
        # swaps on occupancy 0: half random pairs, half first-shell neighbour pairs
        swaps, inc_fit, inc_gam = [], [], []
        occ0 = np.ascontiguousarray(occs[0])
        while len(swaps) < 24:
            a = int(rng.integers(N))
            b = int(rng.integers(N)) if len(swaps) % 2 == 0 else int(nbor[a, rng.integers(shell_size[0])])
            if occ0[a] == occ0[b]:
                continue
            g_out = np.zeros((T, T, S))
            f = ref.ref_fitness_incremental(N, T, S, i32(nbor), row, i32(shell_size), i32(sp), f64(w), f64(target),
                                            i32(occ0), a, b, f64(np.ascontiguousarray(gam[0])), f64(g_out))
            swaps.append((a, b))
            inc_fit.append(f)
            inc_gam.append(g_out)
        out[name + "/lattice"] = np.array(key)
        out[name + "/species"] = sp
        out[name + "/weight"] = w
        out[name + "/target"] = target
        out[name + "/shell_size"] = shell_size
        out[name + "/occ"] = occs
        out[name + "/gamma"] = gam
        out[name + "/fitness"] = fit
        out[name + "/swaps"] = np.array(swaps, dtype=np.int32)
        out[name + "/swap_fitness"] = np.array(inc_fit)
        out[name + "/swap_gamma"] = np.array(inc_gam)
    np.savez_compressed(os.path.join(HERE, "ref_engine.npz"), **out)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
