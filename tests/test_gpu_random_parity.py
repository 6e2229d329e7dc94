"""A seeded sweep of random small structures through the whole search, against
the CPU oracle: lattice kind, edge 2-6, 2-6 species with random compositions,
1-3 shells of either shell set, task counts around the warp and CTA sizes,
neighbours from the table as given or recognised (lattice arithmetic), and the
HBM cluster path on some.  Occupancies, fitness and the evaluation, accept and
round counts must be bit-exact."""
import numpy as np
import pytest

from oracle import hea_oracle as ho
import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


def draw_case(rng):
    lat = L.FCC if rng.random() < 0.5 else L.BCC
    cell = int(rng.integers(2, 7))
    n = L.num_sites(lat, cell)
    T = int(rng.integers(2, min(6, n // 2) + 1))
    S = int(rng.integers(1, 4))
    shell_set = L.SHELLS_FCC_TRUE3 if (lat == L.FCC and rng.random() < 0.5) else L.SHELLS_REFERENCE
    species = W.dirichlet_counts(rng, T, n)
    prm = dict(P=int(rng.integers(1, 6)), I=int(rng.integers(0, 3)), Q=int(rng.choice([1, 31, 32, 33, 100, 513])),
               D=int(rng.integers(1, 5)))
    return lat, cell, species, S, shell_set, prm, bool(rng.random() < 0.5), bool(rng.random() < 0.25)


@pytest.mark.parametrize("index", range(64))
def test_random_structures_match_the_oracle(index):
    rng = np.random.default_rng(1000 + index)
    lat, cell, species, S, shell_set, prm, recognize, hbm = draw_case(rng)
    st = W.small_case(lattice=lat, cell=cell, species=species, shells=S, shell_set=shell_set, seed=index)
    nbor, sizes = st.neighbors()
    gp = hb.Problem(nbor, sizes, st.species, st.weight, st.target, recognize=recognize)
    op = ho.Problem(nbor[:, : int(sizes[:S].sum())], sizes[:S], st.species, st.weight, st.target)
    seed = 500 + index
    occ, fit, stats = hb.search(gp, prm["P"], prm["I"], prm["Q"], prm["D"], seed=seed, hbm_occupancy=hbm)
    wocc, wf2, wstats = op.hcs(seed, prm["P"], prm["I"], prm["Q"], prm["D"])
    case = f"{'FCC' if lat == L.FCC else 'BCC'} {cell} T={len(species)} S={S} {prm} recognize={recognize} hbm={hbm}"
    np.testing.assert_array_equal(occ, wocc, err_msg=case)
    np.testing.assert_array_equal(fit, np.sqrt(wf2), err_msg=case)
    assert (stats["evals"], stats["accepts"], stats["rounds"]) == (wstats["evals"], wstats["accepts"], wstats["rounds"]), case
