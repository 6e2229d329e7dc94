"""CUDA path vs the CPU oracle, through the C ABI (and the pybind11 drop-in).

Integer results (occupancies, pair counts, accepted-swap traces) must be
bit-exact; f2 is computed with the same fused multiply-adds in the same order
on both sides, so it must be bit-exact too.  Fitness against the reference
engine's own floating-point accumulation: 1e-12 relative.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import REPO, engine_case_problem, opt_call_args
from oracle import hea_oracle as ho
import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import sro
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    # lattice, cell, species, shells, shell_set
    (L.FCC, 4, (64, 64, 64, 64), 3, L.SHELLS_REFERENCE),
    (L.BCC, 5, (40, 42, 42, 42, 42, 42), 3, L.SHELLS_REFERENCE),
    (L.FCC, 3, (20, 22, 22, 22, 22), 3, L.SHELLS_FCC_TRUE3),
    (L.BCC, 4, (40, 44, 44), 2, L.SHELLS_REFERENCE),
    (L.FCC, 4, (100, 156), 1, L.SHELLS_REFERENCE),
    (L.BCC, 3, (1, 53), 3, L.SHELLS_REFERENCE),  # 54 sites (not a multiple of 16), one minority atom
    # the layouts and species counts of the benchmarked structures: BCC 8/6/12 with 5 species
    # (mc_kernel<5, Shells<2,2,3>>) and FCC 12/6/24 with 4 species (mc_kernel<4, Shells<3,2,6>>)
    (L.BCC, 5, (50, 50, 50, 50, 50), 3, L.SHELLS_REFERENCE),
    (L.FCC, 3, (27, 27, 27, 27), 3, L.SHELLS_FCC_TRUE3),
]
FULL_SEARCH_CASES = CASES[:4] + CASES[6:]


def pair(case, seed=0, recognize=True):
    """(library problem, oracle problem).  The cases' tables are lattice tables: with `recognize` the
    library runs them on lattice arithmetic, without it on the table as given."""
    lat, cell, species, shells, shell_set = case
    st = W.small_case(lattice=lat, cell=cell, species=species, shells=shells, shell_set=shell_set, seed=seed)
    nbor, sizes = st.neighbors()
    return (hb.Problem(nbor, sizes, st.species, st.weight, st.target, recognize=recognize),
            ho.Problem(nbor[:, : int(sizes[:shells].sum())], sizes[:shells], st.species, st.weight, st.target))


@pytest.mark.parametrize("recognize", [True, False])
@pytest.mark.parametrize("case", CASES)
def test_generate_bit_exact(case, recognize):
    gp, op = pair(case, recognize=recognize)
    occ, cnt, f2 = hb.generate(gp, seed=1234, generation=3, count=5)
    for s in range(5):
        want = op.generate(1234, 3, s)
        np.testing.assert_array_equal(occ[s], want)
        C = op.recount(want)
        np.testing.assert_array_equal(cnt[s], C)
        assert f2[s] == op.f2(C)


def test_recount_matches_reference_engine(golden_engine, golden_nbor):
    for name, case in golden_engine.items():
        gp = engine_case_problem(case, golden_nbor, hb)
        op = engine_case_problem(case, golden_nbor, ho)
        cnt, f2 = hb.recount(gp, case["occ"].astype(np.uint8))
        ss = case["shell_size"]
        for p in range(len(case["occ"])):
            ref = np.rint(case["gamma"][p].transpose(2, 0, 1) * ss[:, None, None] * gp.num_sites).astype(np.int64)
            np.testing.assert_array_equal(cnt[p], ref, err_msg=name)
            assert f2[p] == op.f2(ref)
            assert abs(np.sqrt(f2[p]) - case["fitness"][p]) <= 1e-12 * case["fitness"][p]


@pytest.mark.parametrize("recognize", [True, False])
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("tasks", [1, 37, 64, 600])
def test_local_search_trajectory_bit_exact(case, tasks, recognize):
    """Every accepted swap (round, task, sites, f2) and the counts after it equal the oracle's."""
    gp, op = pair(case, recognize=recognize)
    count, depth, call = 3, 4, 7
    occ0 = np.stack([op.generate(99, 2, s) for s in range(count)])
    got = hb.local_search(gp, 99, call, occ0, tasks, depth, trace_cap=4096, trace_counts=True)
    for s in range(count):
        want = op.mc(99, (call << 16) | s, occ0[s], tasks, depth, trace_cap=4096, trace_counts=True)
        assert got["rounds"][s] == want["rounds"]
        assert got["trace_len"][s] == want["accepts"]
        assert got["trace"][s] == want["trace"]
        n = len(want["trace"])
        np.testing.assert_array_equal(got["trace_counts"][s][:n], want["trace_counts"])
        np.testing.assert_array_equal(got["occ"][s], want["occ"])
        np.testing.assert_array_equal(got["counts"][s], want["counts"])
        assert got["f2"][s] == want["f2"]
        # counts maintained on the device == a recount of the final occupancy
        np.testing.assert_array_equal(got["counts"][s], op.recount(got["occ"][s]))


@pytest.mark.parametrize("recognize", [True, False])
@pytest.mark.parametrize("case", FULL_SEARCH_CASES)
def test_full_search_bit_exact(case, recognize):
    gp, op = pair(case, recognize=recognize)
    occ, fit, stats = hb.search(gp, num_solutions=4, total_iter=2, parallel_task=32, converge_depth=4, seed=77)
    wocc, wf2, wstats = op.hcs(77, 4, 2, 32, 4)
    np.testing.assert_array_equal(occ, wocc)
    np.testing.assert_array_equal(fit, np.sqrt(wf2))
    assert stats["evals"] == wstats["evals"] and stats["accepts"] == wstats["accepts"]
    assert stats["rounds"] == wstats["rounds"]


@pytest.mark.parametrize("lat,cell,species", [
    (L.BCC, 15, (2250, 2250, 2250)),     # 6750 sites: 2^16 mod N = 4786 > 4096
    (L.BCC, 33, (23958, 23958, 23958)),  # 71 874 sites, above 2^16
])
def test_32bit_draws_bit_exact(lat, cell, species):
    """Structures outside the 16-bit draw mode (two attempts per Philox call
    from 32-bit words): trajectories and a whole search equal the oracle's."""
    lib = ho.lib()
    lib.hea_oracle_use_draw16.restype = ctypes.c_int
    assert lib.hea_oracle_use_draw16(L.num_sites(lat, cell)) == 0
    gp, op = pair((lat, cell, species, 3, L.SHELLS_REFERENCE), seed=1)
    count, depth, call, tasks = 2, 4, 3, 64
    occ0 = np.stack([op.generate(41, 1, s) for s in range(count)])
    got = hb.local_search(gp, 41, call, occ0, tasks, depth, trace_cap=4096)
    for s in range(count):
        want = op.mc(41, (call << 16) | s, occ0[s], tasks, depth, trace_cap=4096)
        assert got["rounds"][s] == want["rounds"] and got["trace"][s] == want["trace"]
        np.testing.assert_array_equal(got["occ"][s], want["occ"])
        np.testing.assert_array_equal(got["counts"][s], want["counts"])
        assert got["f2"][s] == want["f2"]
    occ, fit, stats = hb.search(gp, num_solutions=2, total_iter=1, parallel_task=48, converge_depth=3, seed=13)
    wocc, wf2, wstats = op.hcs(13, 2, 1, 48, 3)
    np.testing.assert_array_equal(occ, wocc)
    np.testing.assert_array_equal(fit, np.sqrt(wf2))
    assert stats["evals"] == wstats["evals"] and stats["rounds"] == wstats["rounds"]


def test_plan_reruns_match_search():
    gp, _ = pair(CASES[0])
    occ, fit, _ = hb.search(gp, 6, 2, 48, 3, seed=5)
    plan = hb.Plan(gp, 6, 2, 48, 3)
    for _ in range(2):
        plan.run(5)
        pocc, pfit = plan.read()
        np.testing.assert_array_equal(pocc, occ)
        np.testing.assert_array_equal(pfit, fit)
    plan.run(6)
    assert not np.array_equal(plan.read()[0], occ)
    plan.close()


def test_dropin_module_call_as_pyhea_model_makes_it():
    """The positional call of pyhea/model/opt.py:89-90 with nested neighbour lists."""
    lat, cell, species = L.FCC, 4, [64, 64, 64, 64]
    nbor, sizes = L.neighbors(lat, cell)
    nested = L.as_nested(nbor, sizes)
    st = W.small_case(lattice=lat, cell=cell, species=species)
    target = st.target  # ndarray [3][T*T], as input_config.target_sro returns
    assert hb.accelerate.cuda_available() is True
    latts, fitss = hb.accelerate.run_local_parallel_hcs_cuda(4, 2, 32, 4, 0.001, nested, species, [4.0, 1.0, 0.5],
                                                             target, seed=77, verbose=False)
    assert isinstance(latts, list) and isinstance(latts[0], list) and isinstance(latts[0][0], int)
    assert isinstance(fitss, list) and fitss == sorted(fitss)
    op = ho.Problem(nbor, sizes, species, [4.0, 1.0, 0.5], target)
    wocc, wf2, _ = op.hcs(77, 4, 2, 32, 4)
    np.testing.assert_array_equal(np.array(latts), wocc)
    np.testing.assert_array_equal(np.array(fitss), np.sqrt(wf2))


def test_dropin_replays_the_reference_driver_call(capfd):
    """The call recorded from the reference driver (pyhea/model/opt.py:89-90, device: gpu) through
    the drop-in module: with a seed it equals the oracle's search; as recorded (no keywords: fresh
    seed, log on) it returns a valid population and prints one log line per iteration."""
    args = opt_call_args()
    nnet, step, task, depth, thr, nbor, element, weight, target = args
    nb = np.array([np.concatenate(site) for site in nbor], dtype=np.int32)
    sizes = np.array([len(s) for s in nbor[0]], dtype=np.int32)
    op = ho.Problem(nb, sizes, element, weight, target)
    latts, fitss = hb.accelerate.run_local_parallel_hcs_cuda(*args, seed=2024, verbose=False)
    wocc, wf2, _ = op.hcs(2024, nnet, step, task, depth)
    np.testing.assert_array_equal(np.array(latts), wocc)
    np.testing.assert_array_equal(np.array(fitss), np.sqrt(wf2))
    capfd.readouterr()
    latts, fitss = hb.accelerate.run_local_parallel_hcs_cuda(*args)
    out = capfd.readouterr().out
    assert out.count("best fitness") == step
    assert len(latts) == nnet and fitss == sorted(fitss)
    for o, f in zip(latts, fitss):
        o = np.array(o, dtype=np.uint8)
        np.testing.assert_array_equal(np.bincount(o, minlength=len(element)), element)
        assert f == np.sqrt(op.f2(op.recount(o)))


def test_search_fitness_agrees_with_reference_engine():
    """Final structures scored by the reference's calculate_fitness_of_solutions."""
    path = os.path.join(REPO, "oracle", "_ref", "libref_accelerate.so")
    if not os.path.exists(path):
        pytest.skip("reference engine not built")
    ref = ctypes.CDLL(path)
    gp, op = pair(CASES[1])
    occ, fit, _ = hb.search(gp, 4, 2, 64, 4, seed=3)
    rf = np.zeros(4)
    P = ctypes.POINTER
    occ32 = occ.astype(np.int32)
    ref.ref_fitness_of_solutions(4, gp.num_sites, gp.num_types, gp.num_shells, gp.nbor.ctypes.data_as(P(ctypes.c_int32)),
                                 gp.nbor.shape[1], gp.shell_sizes.ctypes.data_as(P(ctypes.c_int32)),
                                 gp.species.ctypes.data_as(P(ctypes.c_int32)), gp.weight.ctypes.data_as(P(ctypes.c_double)),
                                 gp.target_sro.ctypes.data_as(P(ctypes.c_double)), occ32.ctypes.data_as(P(ctypes.c_int32)),
                                 rf.ctypes.data_as(P(ctypes.c_double)))
    np.testing.assert_allclose(fit, rf, rtol=1e-12, atol=0)


@pytest.mark.parametrize("lat", [L.FCC, L.BCC])
@pytest.mark.parametrize("shell_set", [L.SHELLS_REFERENCE, L.SHELLS_FCC_TRUE3])
@pytest.mark.parametrize("cell", [2, 3, 5, 7])
def test_device_neighbor_builder(lat, shell_set, cell):
    d, ds = hb.build_neighbors(lat, cell, shell_set)
    h, hs = L.neighbors(lat, cell, shell_set)
    np.testing.assert_array_equal(ds, hs)
    np.testing.assert_array_equal(d, h)


def test_edge_controls():
    gp, op = pair(CASES[0])
    # no iterations: the initial population in generation order
    occ, fit, st = hb.search(gp, 3, 0, 8, 3, seed=9)
    for s in range(3):
        np.testing.assert_array_equal(occ[s], op.generate(9, 0, s))
    assert st["evals"] == 0
    # depth 0: no rounds; one solution, one task
    occ, fit, st = hb.search(gp, 1, 2, 1, 0, seed=9)
    assert st["rounds"] == 0
    wocc, wf2, _ = op.hcs(9, 1, 2, 1, 0)
    np.testing.assert_array_equal(occ, wocc)
    # round cap
    r = hb.local_search(gp, 9, 0, op.generate(9, 1, 0)[None], 16, 1000, max_rounds=5)
    assert r["rounds"][0] == 5


def test_bad_tables_are_rejected():
    nbor, sizes = L.neighbors(L.FCC, 4)
    T = 4
    bad = nbor.copy()
    bad[3, 0] = 10_000
    with pytest.raises(ValueError, match="outside"):
        hb.search(hb.Problem(bad, sizes, [64] * T, [4.0, 1.0, 0.5], np.zeros((3, 16))), 2, 1, 8, 2)
    bad = nbor.copy()
    bad[3, 0] = bad[3, 1]  # duplicate breaks symmetry with multiplicity
    with pytest.raises(hb.HeaError, match="symmetric"):
        hb.search(hb.Problem(bad, sizes, [64] * T, [4.0, 1.0, 0.5], np.zeros((3, 16))), 2, 1, 8, 2)
    bad = nbor.copy()
    bad[3, 0] = 3
    with pytest.raises(hb.HeaError, match="own neighbour"):
        hb.search(hb.Problem(bad, sizes, [64] * T, [4.0, 1.0, 0.5], np.zeros((3, 16))), 2, 1, 8, 2)


def test_full_size_plain_gpu_properties():
    """The BCC 20^3 five-species structure at full size (fewer iterations):
    composition kept, output ascending, every fitness equal to a recount's."""
    st = W.plain_gpu(seed=0)
    gp = st.problem(device=True)
    occ, fit, stats = hb.search(gp, st.P, 2, st.Q, st.D, seed=11)
    assert np.all(np.diff(fit) >= 0)
    for o in occ[:: max(1, st.P // 16)]:
        np.testing.assert_array_equal(np.bincount(o, minlength=5), st.species)
    cnt, f2 = hb.recount(gp, occ)
    np.testing.assert_array_equal(np.sqrt(f2), fit)
    op = ho.Problem(gp.nbor, gp.shell_sizes, gp.species, gp.weight, gp.target_sro)
    for p in (0, st.P - 1):
        np.testing.assert_array_equal(cnt[p], op.recount(occ[p]))
    assert stats["evals"] > 0 and stats["accepts"] > 0
    init = hb.generate(gp, 11, 0, st.P)[2]
    assert fit[0] ** 2 < init.min()


def test_plans_of_different_sizes_coexist():
    """Kernels are shared by all plans: creating a plan for a small structure
    must not shrink the shared-memory allowance of a larger plan made before."""
    big = W.small_case(lattice=L.FCC, cell=14, species=(2744,) * 4, shell_set=L.SHELLS_FCC_TRUE3)
    small = W.small_case(lattice=L.FCC, cell=3, species=(27,) * 4, shell_set=L.SHELLS_FCC_TRUE3)
    pb_big, pb_small = big.problem(), small.problem()
    plan_big = hb.Plan(pb_big, 2, 1, 64, 2)
    plan_small = hb.Plan(pb_small, 2, 1, 64, 2)
    hb.recount_noalloc(pb_small, hb.generate(pb_small, 1, 0, 1)[0])
    plan_big.run(3)
    plan_small.run(3)
    occ, fit = plan_big.read()
    np.testing.assert_array_equal(np.sqrt(hb.recount(pb_big, occ)[1]), fit)
    plan_big.close()
    plan_small.close()


def test_autotuned_plan_gives_the_same_search():
    """The autotuner only picks the local search's CTA size; the search is the same."""
    st = W.small_case(lattice=L.BCC, cell=6, species=(150, 150, 132), shells=3, seed=3, P=6, Q=384, I=2, D=5)
    pb = st.problem()
    ref = hb.Plan(pb, st.P, st.I, st.Q, st.D)
    tuned = hb.Plan(pb, st.P, st.I, st.Q, st.D, autotune=True)
    assert ref.local_search_block == 384
    assert tuned.local_search_block in (384, 256, 128)
    for seed in (5, 6):
        a, b = ref.run(seed), tuned.run(seed)
        assert a["evals"] == b["evals"] and a["accepts"] == b["accepts"]
        np.testing.assert_array_equal(ref.read()[0], tuned.read()[0])
        np.testing.assert_array_equal(ref.read()[1], tuned.read()[1])
    ref.close()
    tuned.close()


@pytest.mark.parametrize("case", [CASES[0], CASES[6], CASES[7]])
def test_searched_alpha_in_the_analyzer_convention(case):
    """Final alpha of searched structures: alpha from the device's pair counts (the engine's
    convention) equals the analyzer-convention restatement (neighbour ranks [0, 12, 18] FCC /
    [0, 8, 14] BCC, pyhea/utils/analyze.py:35) computed from the occupancies, shells 1-2."""
    lat, cell = case[0], case[1]
    gp, _ = pair(case)
    occ, fit, _ = hb.search(gp, 4, 2, 64, 4, seed=3)
    cnt, f2 = hb.recount(gp, occ)
    np.testing.assert_array_equal(np.sqrt(f2), fit)
    for p in range(len(occ)):
        a = sro.alpha_from_counts(cnt[p], gp.shell_sizes, gp.species)
        wc = sro.warren_cowley_of_occupancy(occ[p], lat, cell, gp.num_types)
        np.testing.assert_allclose(wc, a[:2], rtol=0, atol=1e-12)
