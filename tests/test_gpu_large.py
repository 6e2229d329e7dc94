"""The large-structure path (occupancy in HBM, one thread-block cluster per
solution) gives the same results as the shared-memory path and the oracle, and
handles structures too large for shared memory."""
import numpy as np
import pytest

import pyhea_b200 as hb
from oracle import hea_oracle as ho
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lat,cell,species,shells,shell_set,tasks", [
    (L.FCC, 4, (64, 64, 64, 64), 3, L.SHELLS_FCC_TRUE3, 48),      # one CTA per cluster
    (L.BCC, 6, (100, 100, 132, 100), 3, L.SHELLS_REFERENCE, 700),  # clusters of 2
    (L.FCC, 5, (100, 150, 250), 2, L.SHELLS_REFERENCE, 3000),      # clusters of 6
    (L.BCC, 4, (40, 44, 44), 1, L.SHELLS_REFERENCE, 4096),         # clusters of 8
    (L.BCC, 33, (23958, 23958, 23958), 3, L.SHELLS_REFERENCE, 600),  # 71 874 sites: 32-bit draws
])
def test_hbm_path_equals_shared_path_and_oracle(lat, cell, species, shells, shell_set, tasks):
    st = W.small_case(lattice=lat, cell=cell, species=species, shells=shells, shell_set=shell_set, seed=2)
    nbor, sizes = st.neighbors()
    pb = hb.Problem(nbor, sizes, st.species, st.weight, st.target)
    a = hb.search(pb, 4, 2, tasks, 3, seed=31)
    b = hb.search(pb, 4, 2, tasks, 3, seed=31, hbm_occupancy=True)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2]["evals"] == b[2]["evals"] and a[2]["rounds"] == b[2]["rounds"]
    if tasks <= 700:
        op = ho.Problem(nbor[:, : int(sizes[:shells].sum())], sizes[:shells], st.species, st.weight, st.target)
        wocc, wf2, _ = op.hcs(31, 4, 2, tasks, 3)
        np.testing.assert_array_equal(b[0], wocc)
        np.testing.assert_array_equal(b[1], np.sqrt(wf2))


def test_structure_beyond_shared_memory():
    """FCC 40^3 (256 000 sites) exceeds one block's shared memory: the search
    takes the HBM path by itself; composition, order and counts hold."""
    rng = np.random.default_rng(4)
    n = 4 * 40 ** 3
    species = W.dirichlet_counts(rng, 4, n)
    st = W.Structure(L.FCC, 40, L.SHELLS_FCC_TRUE3, species, W.WEIGHTS, W.projected_target(rng, species / n, 0.1),
                     P=4, Q=2048, I=1, D=3)
    pb = st.problem(device=True)
    occ, fit, stats = hb.search(pb, st.P, st.I, st.Q, st.D, seed=8, max_rounds=300)
    assert np.all(np.diff(fit) >= 0)
    for o in occ:
        np.testing.assert_array_equal(np.bincount(o, minlength=4), species)
    cnt, f2 = hb.recount(pb, occ)
    np.testing.assert_array_equal(np.sqrt(f2), fit)
    init = hb.generate(pb, 8, 0, st.P)[2]
    assert fit[0] ** 2 < init.min()
    assert stats["evals"] > 0
