"""The allocation-free recount (hea_recount_noalloc) through the C ABI.

It serves callers that cannot allocate device memory -- a process whose GPU
memory is reserved up front by another allocator, or code that must not pay
cudaMalloc's device-wide synchronisation -- by keeping its scratch in a fixed
static device array.  This file is collected last so that a run stopping at
the first failure has run every other test; it passes alone and after them.
Its results must equal the allocating hea_recount bit for bit (integer counts,
and f2 from the same fma order), on two calls in a row sharing the array.
"""
import numpy as np
import pytest

import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _problem(lattice, cell, species, shell_set, seed):
    st = W.small_case(lattice=lattice, cell=cell, species=species, shell_set=shell_set, seed=seed)
    nbor, sizes = st.neighbors()
    return hb.Problem(nbor, sizes, st.species, st.weight, st.target)


def test_noalloc_recount_matches_recount_twice_in_a_row():
    cases = [
        (_problem(L.BCC, 20, (3200,) * 5, L.SHELLS_REFERENCE, 3), 40),   # the plain GPU structure size
        (_problem(L.FCC, 6, (200, 264, 200, 200), L.SHELLS_FCC_TRUE3, 4), 9),
    ]
    for pb, count in cases:
        occ = hb.generate(pb, seed=21, generation=2, count=count)[0]
        want_cnt, want_f2 = hb.recount(pb, occ)
        # two calls in a row share the static scratch; both must match
        for _ in range(2):
            cnt, f2 = hb.recount_noalloc(pb, occ)
            np.testing.assert_array_equal(cnt, want_cnt)
            np.testing.assert_array_equal(f2, want_f2)


def test_noalloc_recount_rejects_inputs_beyond_its_scratch():
    pb = _problem(L.FCC, 20, (8000,) * 4, L.SHELLS_FCC_TRUE3, 5)  # 32000 sites, 42 neighbours
    occ = np.tile(np.repeat(np.arange(4, dtype=np.uint8), 8000), (200, 1))
    with pytest.raises(hb.HeaError, match="scratch"):
        hb.recount_noalloc(pb, occ)
