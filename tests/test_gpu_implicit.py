"""Implicit neighbours: a perfect FCC/BCC cube described by its lattice
(Problem.from_lattice, hea_problem.implicit_lattice) instead of a neighbour
table gives the same results as the table hea_build_neighbors builds -- the
site numbering and shells of pyhea/lattice/lattice.py:146-323 -- on every path,
bit for bit, while no table is kept on the device."""
import numpy as np
import pytest

import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    # lattice, cell, species, shells, shell_set
    (L.FCC, 4, (64, 64, 64, 64), 3, L.SHELLS_REFERENCE),
    (L.FCC, 3, (20, 22, 22, 22, 22), 3, L.SHELLS_FCC_TRUE3),
    (L.BCC, 5, (50, 50, 50, 50, 50), 3, L.SHELLS_REFERENCE),
    (L.BCC, 4, (40, 44, 44), 2, L.SHELLS_REFERENCE),
    (L.FCC, 4, (100, 156), 1, L.SHELLS_REFERENCE),
    (L.FCC, 2, (8, 8, 8, 8), 3, L.SHELLS_FCC_TRUE3),  # edge 2: periodic images repeat neighbours
    (L.BCC, 2, (5, 5, 6), 3, L.SHELLS_REFERENCE),
]


def pair(case, seed=0):
    lat, cell, species, shells, shell_set = case
    st = W.small_case(lattice=lat, cell=cell, species=species, shells=shells, shell_set=shell_set, seed=seed)
    nbor, sizes = hb.build_neighbors(lat, cell, shell_set)
    table = hb.Problem(nbor, sizes, st.species, st.weight, st.target, recognize=False)
    implicit = hb.Problem.from_lattice(lat, cell, st.species, st.weight, st.target, shell_set=shell_set)
    assert implicit.nbor is None
    return table, implicit


@pytest.mark.parametrize("case", CASES)
def test_generate_recount_and_trajectories_equal(case):
    tp, ip = pair(case)
    a, b = hb.generate(tp, 7, 2, 4), hb.generate(ip, 7, 2, 4)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(hb.recount(tp, a[0])[0], hb.recount(ip, a[0])[0])
    for tasks in (16, 300):
        got = hb.local_search(ip, 5, 3, a[0], tasks, 4, trace_cap=4096, trace_counts=True)
        want = hb.local_search(tp, 5, 3, a[0], tasks, 4, trace_cap=4096, trace_counts=True)
        for k in ("occ", "counts", "f2", "rounds", "trace_len"):
            np.testing.assert_array_equal(got[k], want[k])
        assert got["trace"] == want["trace"]
        np.testing.assert_array_equal(got["trace_counts"], want["trace_counts"])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("hbm", [False, True])
def test_whole_search_equal(case, hbm):
    tp, ip = pair(case)
    a = hb.search(tp, 4, 2, 48, 3, seed=11, hbm_occupancy=hbm)
    b = hb.search(ip, 4, 2, 48, 3, seed=11, hbm_occupancy=hbm)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert (a[2]["rounds"], a[2]["evals"], a[2]["accepts"]) == (b[2]["rounds"], b[2]["evals"], b[2]["accepts"])


def test_batch_with_implicit_and_table_structures():
    items = [pair(c, seed=i) for i, c in enumerate(CASES)]
    problems = [p for t, i in items for p in (t, i)]
    params = [dict(num_solutions=3, total_iter=2, parallel_task=64, converge_depth=3)] * len(problems)
    seeds = [50 + i // 2 for i in range(len(problems))]  # each table/implicit pair shares its seed
    b = hb.Batch(problems, params)
    b.run(seeds)
    for i in range(0, len(problems), 2):
        np.testing.assert_array_equal(b.read(i)[0], b.read(i + 1)[0], err_msg=f"case {i // 2}")
        np.testing.assert_array_equal(b.read(i)[1], b.read(i + 1)[1], err_msg=f"case {i // 2}")
    b.close()


def test_server_lattice_requests_keep_no_table():
    """Lattice requests are implicit now: the same results as submitting the table, in less arena memory."""
    lat, cell, species, shells, shell_set = (L.FCC, 6, (200, 264, 200, 200), 3, L.SHELLS_FCC_TRUE3)
    tp, ip = pair((lat, cell, species, shells, shell_set))
    q = dict(num_solutions=4, total_iter=2, parallel_task=64, converge_depth=3, seed=9)
    srv = hb.Server(max_requests=8, slice_ms=20.0)
    r1 = srv.submit(tp, q)
    r2 = srv.submit_lattice(lat, cell, ip.species, ip.weight, ip.target_sro, q, shell_set=shell_set)
    r3 = srv.submit(ip, q)
    res = {}
    while len(res) < 3:
        srv.step()
        for rid in (r1, r2, r3):
            if rid not in res:
                got = srv.result(rid)
                if got is not None:
                    res[rid] = got
    srv.close()
    for rid in (r2, r3):
        np.testing.assert_array_equal(res[rid][0], res[r1][0])
        np.testing.assert_array_equal(res[rid][1], res[r1][1])
        assert res[rid][2]["device_bytes"] < res[r1][2]["device_bytes"]


@pytest.mark.parametrize("case", CASES)
def test_lattice_tables_are_recognised(case):
    """A lattice table, also with its shells' entries permuted, runs on lattice arithmetic with the
    table's results; the same table with recognition off, or relabelled by a site permutation (a valid
    table, not the lattice's), runs on the table."""
    lat, cell, species, shells, shell_set = case
    st = W.small_case(lattice=lat, cell=cell, species=species, shells=shells, shell_set=shell_set, seed=3)
    nbor, sizes = hb.build_neighbors(lat, cell, shell_set)
    nbor = nbor[:, : int(sizes[:shells].sum())]
    rng = np.random.default_rng(0)
    shuffled = nbor.copy()
    off = np.concatenate([[0], np.cumsum(sizes[:shells])])
    for k in range(shells):
        seg = shuffled[:, off[k]:off[k + 1]]
        shuffled[:, off[k]:off[k + 1]] = np.take_along_axis(seg, rng.permuted(np.tile(np.arange(seg.shape[1]), (len(seg), 1)), axis=1), axis=1)
    perm = rng.permutation(len(nbor)).astype(np.int32)  # site s of the new labels is perm[s] of the old
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm), dtype=np.int32)
    relabelled = inv[nbor[perm]]
    q = dict(num_solutions=4, total_iter=2, parallel_task=48, converge_depth=3)
    want = None
    for table, recognize, lattice in ((nbor, False, 0), (nbor, True, lat + 1), (shuffled, True, lat + 1),
                                      (relabelled, True, 0)):
        pb = hb.Problem(table, sizes, st.species, st.weight, st.target, recognize=recognize)
        plan = hb.Plan(pb, q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"])
        assert plan.lattice == lattice
        plan.run(21)
        got = plan.read()
        plan.close()
        if table is relabelled:
            continue  # another labelling of the sites: other trajectories
        if want is None:
            want = got
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


def test_server_recognises_lattice_tables():
    """A lattice table submitted to the server runs as a lattice request: same result as the table
    as given, and no table in the arena."""
    case = (L.BCC, 5, (50, 50, 50, 50, 50), 3, L.SHELLS_REFERENCE)
    tp, _ = pair(case)
    rp = hb.Problem(tp.nbor, tp.shell_sizes, tp.species, tp.weight, tp.target_sro)  # recognised
    q = dict(num_solutions=4, total_iter=2, parallel_task=64, converge_depth=3, seed=5)
    srv = hb.Server(max_requests=4, slice_ms=20.0)
    ids = [srv.submit(tp, q), srv.submit(rp, q)]
    res = {}
    while len(res) < 2:
        srv.step()
        for rid in ids:
            if rid not in res:
                got = srv.result(rid)
                if got is not None:
                    res[rid] = got
    srv.close()
    a, b = res[ids[0]], res[ids[1]]
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert b[2]["device_bytes"] < a[2]["device_bytes"]
