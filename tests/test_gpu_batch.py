"""Batched persistent search: every structure's result equals the plain path
on that structure alone (same seed), bit for bit -- the "same result alone and
in the mix" property -- over structures of different lattice, size, species
count, composition and search sizes."""
import numpy as np
import pytest

import pyhea_b200 as hb
from oracle import hea_oracle as ho
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


def mixed_structures(seed=0, count=7):
    rng = np.random.default_rng(seed)
    out = []
    specs = [(L.FCC, 4, L.SHELLS_FCC_TRUE3, 3), (L.BCC, 6, L.SHELLS_REFERENCE, 3), (L.FCC, 5, L.SHELLS_REFERENCE, 3),
             (L.BCC, 5, L.SHELLS_REFERENCE, 2), (L.FCC, 6, L.SHELLS_FCC_TRUE3, 3), (L.BCC, 8, L.SHELLS_REFERENCE, 1),
             (L.FCC, 3, L.SHELLS_FCC_TRUE3, 3)]
    for i in range(count):
        lat, cell, shell_set, S = specs[i % len(specs)]
        T = int(rng.integers(2, 7))
        n = L.num_sites(lat, cell)
        species = W.dirichlet_counts(rng, T, n)
        st = W.small_case(lattice=lat, cell=cell, species=species, shells=S, shell_set=shell_set, seed=i)
        nbor, sizes = st.neighbors()
        prm = dict(num_solutions=int(rng.integers(2, 9)), total_iter=int(rng.integers(0, 4)),
                   parallel_task=int(rng.choice([16, 37, 64, 300])), converge_depth=int(rng.integers(1, 6)))
        out.append((hb.Problem(nbor, sizes, st.species, st.weight, st.target), prm))
    return out


def test_batch_equals_plain_per_structure():
    items = mixed_structures(0, 7)
    seeds = [1000 + 17 * i for i in range(len(items))]
    b = hb.Batch([p for p, _ in items], [q for _, q in items])
    st = b.run(seeds)
    tallies = b.tallies()
    total_evals = 0
    for i, (pb, q) in enumerate(items):
        occ, fit = b.read(i)
        pocc, pfit, pst = hb.search(pb, q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"],
                                    seed=seeds[i])
        np.testing.assert_array_equal(occ, pocc, err_msg=f"structure {i}")
        np.testing.assert_array_equal(fit, pfit, err_msg=f"structure {i}")
        assert list(tallies[i]) == [pst["rounds"], pst["evals"], pst["accepts"]], f"structure {i}"
        total_evals += pst["evals"]
    assert st["evals"] == total_evals
    # a second run with other seeds, then the first seeds again: same as before
    b.run([s + 1 for s in seeds])
    b.run(seeds)
    occ0, fit0 = b.read(0)
    pocc, pfit, _ = hb.search(items[0][0], items[0][1]["num_solutions"], items[0][1]["total_iter"],
                              items[0][1]["parallel_task"], items[0][1]["converge_depth"], seed=seeds[0])
    np.testing.assert_array_equal(occ0, pocc)
    b.close()


def test_batch_matches_oracle_on_one_structure():
    items = mixed_structures(3, 3)
    pb, q = items[1]
    q = dict(q, total_iter=2)
    b = hb.Batch([items[0][0], pb, items[2][0]], [items[0][1], q, items[2][1]])
    b.run([5, 6, 7])
    occ, fit = b.read(1)
    op = ho.Problem(pb.nbor, pb.shell_sizes, pb.species, pb.weight, pb.target_sro)
    wocc, wf2, _ = op.hcs(6, q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"])
    np.testing.assert_array_equal(occ, wocc)
    np.testing.assert_array_equal(fit, np.sqrt(wf2))
    b.close()


def test_batch_matches_oracle_for_every_kernel_instance():
    """One structure of every (species count, shell layout) the batch engine
    compiles -- T = 2..6 on the BCC 8/6/12 and FCC 12/6/24 layouts of the mixed
    batch and on the runtime layouts (FCC 12/6/12, two shells, one shell) --
    in one batch, each equal to the oracle's whole search."""
    specs = [(L.BCC, 4, L.SHELLS_REFERENCE, 3), (L.FCC, 3, L.SHELLS_FCC_TRUE3, 3), (L.FCC, 3, L.SHELLS_REFERENCE, 3),
             (L.BCC, 4, L.SHELLS_REFERENCE, 2), (L.FCC, 3, L.SHELLS_REFERENCE, 1)]
    rng = np.random.default_rng(11)
    items = []
    for lat, cell, shell_set, S in specs:
        for T in range(2, 7):
            n = L.num_sites(lat, cell)
            st = W.small_case(lattice=lat, cell=cell, species=W.dirichlet_counts(rng, T, n), shells=S,
                              shell_set=shell_set, seed=len(items))
            nbor, sizes = st.neighbors()
            q = dict(num_solutions=3, total_iter=2, parallel_task=int(rng.choice([24, 64, 130])), converge_depth=3)
            items.append((hb.Problem(nbor, sizes, st.species, st.weight, st.target), q))
    seeds = [300 + i for i in range(len(items))]
    b = hb.Batch([p for p, _ in items], [q for _, q in items])
    b.run(seeds)
    for i, (pb, q) in enumerate(items):
        occ, fit = b.read(i)
        op = ho.Problem(pb.nbor, pb.shell_sizes, pb.species, pb.weight, pb.target_sro)
        wocc, wf2, _ = op.hcs(seeds[i], q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"])
        np.testing.assert_array_equal(occ, wocc, err_msg=f"structure {i}")
        np.testing.assert_array_equal(fit, np.sqrt(wf2), err_msg=f"structure {i}")
    b.close()


def test_autotuned_batch_gives_the_same_results():
    """The batch autotuner only changes where occupancies live and how many CTAs share an SM."""
    items = mixed_structures(4, 5)
    seeds = [77 + 3 * i for i in range(len(items))]
    b = hb.Batch([p for p, _ in items], [q for _, q in items])
    b.run(seeds)
    choice = b.autotune()
    assert choice["hbm_all"] in (0, 1) and 1 <= choice["ctas_per_sm"] <= 3
    b.run(seeds)
    for i, (pb, q) in enumerate(items):
        occ, fit = b.read(i)
        pocc, pfit, _ = hb.search(pb, q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"],
                                  seed=seeds[i])
        np.testing.assert_array_equal(occ, pocc, err_msg=f"structure {i}")
        np.testing.assert_array_equal(fit, pfit, err_msg=f"structure {i}")
    b.close()


def test_streaming_histogram_loads_give_the_same_results():
    """Two FCC 30^3 structures (108 000 sites, 64 solutions): 221 MB of site histograms each, 442 MB
    together, more than twice the L2, so the batch reads both with evict-first loads; searched alone
    each fits the plain path's cached policy.  The load policy must not change a result."""
    rng = np.random.default_rng(5)
    items = []
    for i, implicit in enumerate((False, True)):
        n = L.num_sites(L.FCC, 30)
        species = W.dirichlet_counts(rng, 4, n)
        st = W.small_case(lattice=L.FCC, cell=30, species=species, shells=3, shell_set=L.SHELLS_FCC_TRUE3, seed=40 + i)
        items.append(st.problem(device=True, implicit=implicit))
    q = dict(num_solutions=64, total_iter=1, parallel_task=64, converge_depth=3)
    seeds = [71, 72]
    b = hb.Batch(items, [q, q])
    b.run(seeds)
    for i, pb in enumerate(items):
        occ, fit = b.read(i)
        pocc, pfit, _ = hb.search(pb, q["num_solutions"], q["total_iter"], q["parallel_task"], q["converge_depth"],
                                  seed=seeds[i])
        np.testing.assert_array_equal(occ, pocc, err_msg=f"structure {i}")
        np.testing.assert_array_equal(fit, pfit, err_msg=f"structure {i}")
    b.close()
