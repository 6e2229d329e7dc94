"""The CPU restatement (oracle/) pinned against the reference engine and its
published primitives; CPU only."""
import ctypes

import numpy as np
import pytest

from conftest import engine_case_problem
from oracle import hea_oracle as ho
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

# Random123 known-answer vectors for Philox4x32-10 (kat_vectors of the SC'11 release)
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(ho.philox(ctr, key)) == want


def test_recount_matches_reference_engine(golden_engine, golden_nbor):
    """Counts == gamma * Z_k * N of calculate_sro_coefficient (accelerate.cpp:370-399), exactly."""
    for name, case in golden_engine.items():
        pr = engine_case_problem(case, golden_nbor, ho)
        ss = case["shell_size"]
        for occ, gam in zip(case["occ"], case["gamma"]):
            C = pr.recount(occ.astype(np.uint8))
            scaled = gam.transpose(2, 0, 1) * ss[:, None, None] * pr.num_sites
            ref = np.rint(scaled).astype(np.int64)
            assert np.abs(scaled - ref).max() < 1e-6, name
            np.testing.assert_array_equal(C, ref, err_msg=name)


def test_fitness_matches_reference_engine(golden_engine, golden_nbor):
    """sqrt(f2) agrees with calculate_fitness_of_solutions (accelerate.cpp:118-180) to 1e-12 relative."""
    for name, case in golden_engine.items():
        pr = engine_case_problem(case, golden_nbor, ho)
        for occ, fit in zip(case["occ"], case["fitness"]):
            f = np.sqrt(pr.f2(pr.recount(occ.astype(np.uint8))))
            assert abs(f - fit) <= 1e-12 * fit, (name, f, fit)


def test_incremental_matches_reference_engine(golden_engine, golden_nbor):
    """Swap update == calculate_fitness_incremental (accelerate.cpp:498-570): counts exact, fitness 1e-12."""
    for name, case in golden_engine.items():
        pr = engine_case_problem(case, golden_nbor, ho)
        ss = case["shell_size"]
        occ = case["occ"][0].astype(np.uint8)
        C0 = pr.recount(occ)
        for (a, b), fit, gam in zip(case["swaps"], case["swap_fitness"], case["swap_gamma"]):
            Cp = pr.swap_counts(occ, C0, a, b)
            ref = np.rint(gam.transpose(2, 0, 1) * ss[:, None, None] * pr.num_sites).astype(np.int64)
            np.testing.assert_array_equal(Cp, ref, err_msg=name)
            after = occ.copy()
            after[a], after[b] = after[b], after[a]
            np.testing.assert_array_equal(Cp, pr.recount(after))
            assert abs(np.sqrt(pr.f2(Cp)) - fit) <= 1e-12 * fit, name


def test_generate_keeps_composition_and_is_a_permutation():
    st = W.small_case(species=(50, 70, 80, 56))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    for slot in range(3):
        perm = ho.permutation(7, 1, slot, pr.num_sites)
        assert sorted(perm.tolist()) == list(range(pr.num_sites))
        occ = pr.generate(7, 1, slot)
        np.testing.assert_array_equal(np.bincount(occ, minlength=4), st.species)
    assert not np.array_equal(pr.generate(7, 1, 0), pr.generate(7, 1, 1))
    assert not np.array_equal(pr.generate(7, 1, 0), pr.generate(8, 1, 0))


def test_generate_is_uniform_per_site():
    """Species frequency at fixed sites over many keys matches the composition (chi-square)."""
    st = W.small_case(lattice=L.BCC, cell=3, species=(9, 18, 27))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    hits = np.zeros((pr.num_sites, 3))
    R = 600
    for seed in range(R):
        occ = pr.generate(seed, 0, 0)
        hits[np.arange(pr.num_sites), occ] += 1
    expect = R * st.species / st.species.sum()
    chi2 = (((hits - expect) ** 2) / expect).sum()
    dof = pr.num_sites * 2
    assert abs(chi2 - dof) < 6 * np.sqrt(2 * dof), (chi2, dof)


def test_draw_pair_uniform_and_valid():
    st = W.small_case(lattice=L.BCC, cell=3, species=(20, 34))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    occ = pr.generate(1, 0, 0)
    seen = np.zeros(pr.num_sites)
    for q in range(4000):
        att, a, b = pr.draw_pair(3, 5, 0, q, occ)
        assert att >= 0 and occ[a] != occ[b]
        seen[a] += 1
    # s1 is uniform over sites given validity weight: species-0 sites are picked with prob ∝ n1
    p0 = seen[occ == 0].sum() / seen.sum()
    assert abs(p0 - 0.5) < 0.05


def test_mc_counts_match_recount_after_every_accept():
    st = W.small_case(species=(64, 64, 64, 64))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    occ0 = pr.generate(11, 1, 0)
    res = pr.mc(11, 5, occ0, tasks=16, depth=4, trace_cap=5000, trace_counts=True)
    assert res["accepts"] > 10
    occ = occ0.copy()
    last = pr.f2(pr.recount(occ0))
    for (rnd, task, s1, s2, f2), cnt in zip(res["trace"], res["trace_counts"]):
        occ[s1], occ[s2] = occ[s2], occ[s1]
        np.testing.assert_array_equal(cnt, pr.recount(occ))
        # the running f2 (sum of the accepted deltas) tracks a recount's to rounding
        assert abs(f2 - pr.f2(cnt)) <= 1e-12 * pr.f2(cnt) and f2 < last
        last = f2
    np.testing.assert_array_equal(occ, res["occ"])
    np.testing.assert_array_equal(res["counts"], pr.recount(occ))
    assert res["f2"] == pr.f2(res["counts"])
    assert res["evals"] <= res["rounds"] * 16


@pytest.mark.parametrize("lat,cell,species,shell_set", [
    (L.FCC, 4, (100, 156), L.SHELLS_REFERENCE),
    (L.BCC, 5, (40, 42, 42, 42, 42, 42), L.SHELLS_REFERENCE),
    (L.FCC, 3, (20, 22, 22, 22, 22), L.SHELLS_FCC_TRUE3),
    (L.BCC, 4, (40, 44, 44), L.SHELLS_REFERENCE),
    (L.FCC, 4, (64, 64, 64, 64), L.SHELLS_FCC_TRUE3),
])
def test_delta_is_the_change_of_fitness(lat, cell, species, shell_set):
    """The scoring contract's D equals f2(counts after the swap) - f2(counts before) -- the
    reference's full fitness of the swapped state minus the current one (accelerate.cpp:555-569)
    -- to rounding, for random states and swaps, including neighbouring pairs (m > 0)."""
    st = W.small_case(lattice=lat, cell=cell, species=species, shell_set=shell_set, seed=3)
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    rng = np.random.default_rng(5)
    near = 0
    for trial in range(300):
        occ = pr.generate(trial, 0, 0)
        C = pr.recount(occ)
        f0 = pr.f2(C)
        s1 = int(rng.integers(pr.num_sites))
        cand = nbor[s1] if trial % 3 == 0 else rng.integers(pr.num_sites, size=8)
        s2 = next((int(x) for x in cand if occ[int(x)] != occ[s1]), None)
        if s2 is None:
            continue
        near += int(s2 in nbor[s1])
        f1 = pr.f2(pr.swap_counts(occ, C, s1, s2))
        D = pr.delta(occ, C, s1, s2)
        assert abs(D - (f1 - f0)) <= 1e-13 * max(f0, f1), (trial, D, f1 - f0)
        assert (D < 0) == (f1 < f0) or abs(f1 - f0) <= 1e-13 * f0
    assert near > 20


def test_hcs_sorted_deterministic_and_improving():
    st = W.small_case(species=(64, 64, 64, 64))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    occ, f2, stats = pr.hcs(3, num_solutions=4, total_iter=2, tasks=16, depth=4)
    assert np.all(np.diff(f2) >= 0)
    for o, f in zip(occ, f2):
        np.testing.assert_array_equal(np.bincount(o, minlength=4), st.species)
        assert pr.f2(pr.recount(o)) == f
    occ2, f22, _ = pr.hcs(3, num_solutions=4, total_iter=2, tasks=16, depth=4)
    np.testing.assert_array_equal(occ, occ2)
    np.testing.assert_array_equal(f2, f22)
    init = [pr.f2(pr.recount(pr.generate(3, 0, s))) for s in range(4)]
    assert f2[0] < min(init)
    assert stats["evals"] > 0 and stats["accepts"] > 0


def test_draw_modes():
    """Structures of at most 2^16 sites with few rejected 16-bit words draw four
    attempts per Philox call from 16-bit halves; the others two from 32-bit words."""
    lib = ho.lib()
    lib.hea_oracle_use_draw16.restype = ctypes.c_int
    assert lib.hea_oracle_use_draw16(16000) == 1 and lib.hea_oracle_use_draw16(4000) == 1
    assert lib.hea_oracle_use_draw16(35152) == 0 and lib.hea_oracle_use_draw16(65537) == 0
    st = W.small_case(lattice=L.BCC, cell=26, species=(17576, 17576))
    nbor, ss = st.neighbors()
    pr = ho.Problem(nbor, ss, st.species, st.weight, st.target)
    occ = pr.generate(2, 0, 0)
    atts, seen = [], np.zeros(pr.num_sites)
    for q in range(3000):
        att, a, b = pr.draw_pair(9, 5, 0, q, occ)
        assert att >= 0 and occ[a] != occ[b]
        atts.append(att)
        seen[a] += 1
    assert max(atts) >= 2  # 32-bit mode: attempt 2 is the second Philox call
    assert abs(seen[occ == 0].sum() / seen.sum() - 0.5) < 0.05
