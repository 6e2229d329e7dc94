"""The benchmarked structures at full size, bit for bit against the oracle.

The plain GPU configuration (BCC 20^3, 16000 sites, 8/6/12 shells, 5 x 3200
atoms) runs the kernel instance mc_kernel<5, Shells<2,2,3>>; the CPU
configuration's structure (FCC 10^3, 4000 sites, 12/6/24 shells, 4 x 1000
atoms) runs mc_kernel<4, Shells<3,2,6>>.  Each is compared with the oracle on
its own targets and search sizes (Q, D of the configuration): every accepted
swap and the counts after it, the final occupancies, counts and f2, and whole
searches of a few solutions.  The reference semantics restated by the oracle
are pyhea/cpp/accelerate.cpp:601-694 (local search) and :713-763 (global loop).
"""
import numpy as np
import pytest

import pyhea_b200 as hb
from oracle import hea_oracle as ho
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu

CONFIGS = {"plain_gpu": W.plain_gpu, "plain_cpu": W.plain_cpu}


def _pair(name):
    st = CONFIGS[name](seed=0)
    nbor, sizes = st.neighbors()
    S = len(st.weight)
    gp = hb.Problem(nbor, sizes, st.species, st.weight, st.target)
    op = ho.Problem(nbor[:, : int(sizes[:S].sum())], sizes[:S], st.species, st.weight, st.target)
    return st, gp, op


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_full_size_trajectories_bit_exact(name):
    st, gp, op = _pair(name)
    count, call = 3, 5
    occ0 = np.stack([op.generate(2024, 1, s) for s in range(count)])
    cap = 20000
    got = hb.local_search(gp, 2024, call, occ0, st.Q, st.D, trace_cap=cap, trace_counts=True)
    for s in range(count):
        want = op.mc(2024, (call << 16) | s, occ0[s], st.Q, st.D, trace_cap=cap, trace_counts=True)
        assert want["accepts"] < cap
        assert got["rounds"][s] == want["rounds"]
        assert got["trace_len"][s] == want["accepts"]
        assert got["trace"][s] == want["trace"]
        np.testing.assert_array_equal(got["trace_counts"][s][: want["accepts"]], want["trace_counts"])
        np.testing.assert_array_equal(got["occ"][s], want["occ"])
        np.testing.assert_array_equal(got["counts"][s], want["counts"])
        assert got["f2"][s] == want["f2"]


@pytest.mark.parametrize("name", sorted(CONFIGS))
@pytest.mark.parametrize("hbm", [False, True])
def test_full_size_whole_search_bit_exact(name, hbm):
    """Two iterations of the global loop on four solutions, on the shared-memory
    path and on the occupancy-in-HBM cluster path."""
    st, gp, op = _pair(name)
    occ, fit, stats = hb.search(gp, 4, 2, st.Q, st.D, seed=31, hbm_occupancy=hbm)
    wocc, wf2, wstats = op.hcs(31, 4, 2, st.Q, st.D)
    np.testing.assert_array_equal(occ, wocc)
    np.testing.assert_array_equal(fit, np.sqrt(wf2))
    assert (stats["rounds"], stats["evals"], stats["accepts"]) == (wstats["rounds"], wstats["evals"],
                                                                  wstats["accepts"])


def test_full_size_batch_of_both_structures_bit_exact():
    """Both structures in one batch (the persistent job engine's instances for
    these layouts) equal the oracle's whole searches."""
    items = [_pair(n) for n in sorted(CONFIGS)]
    b = hb.Batch([gp for _, gp, _ in items],
                 [dict(num_solutions=3, total_iter=2, parallel_task=st.Q, converge_depth=st.D) for st, _, _ in items])
    b.run([41, 42])
    for i, (st, _, op) in enumerate(items):
        occ, fit = b.read(i)
        wocc, wf2, _ = op.hcs(41 + i, 3, 2, st.Q, st.D)
        np.testing.assert_array_equal(occ, wocc)
        np.testing.assert_array_equal(fit, np.sqrt(wf2))
    b.close()
