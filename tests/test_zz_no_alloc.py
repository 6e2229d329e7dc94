"""The allocation-free recount (hea_recount_noalloc) through the C ABI.

It serves callers that cannot allocate device memory -- a process whose GPU
memory is reserved up front by another allocator, or code that must not pay
cudaMalloc's device-wide synchronisation -- by keeping its scratch in a fixed
static device array.  This file is collected last so that a run stopping at
the first failure has run every other test; it passes alone and after them.
Its results must equal the allocating hea_recount bit for bit (integer counts,
and f2 from the same fma order), on two calls in a row sharing the array, and
the CPU oracle's recount and f2.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO
import pyhea_b200 as hb
from oracle import hea_oracle as ho
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _problem(lattice, cell, species, shell_set, seed):
    st = W.small_case(lattice=lattice, cell=cell, species=species, shell_set=shell_set, seed=seed)
    nbor, sizes = st.neighbors()
    return hb.Problem(nbor, sizes, st.species, st.weight, st.target)


def _oracle(pb):
    return ho.Problem(pb.nbor, pb.shell_sizes, pb.species, pb.weight, pb.target_sro)


def test_noalloc_recount_matches_recount_twice_in_a_row():
    cases = [
        (_problem(L.BCC, 20, (3200,) * 5, L.SHELLS_REFERENCE, 3), 40),   # the plain GPU structure size
        (_problem(L.FCC, 6, (200, 264, 200, 200), L.SHELLS_FCC_TRUE3, 4), 9),
    ]
    for pb, count in cases:
        occ = hb.generate(pb, seed=21, generation=2, count=count)[0]
        want_cnt, want_f2 = hb.recount(pb, occ)
        op = _oracle(pb)
        for p in (0, count - 1):
            np.testing.assert_array_equal(want_cnt[p], op.recount(occ[p]))
            assert want_f2[p] == op.f2(want_cnt[p])
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


def test_noalloc_recount_after_a_failed_call():
    """A call that fails inside the scratch (an asymmetric table caught by the
    device check, which sets the array's error flag) leaves the next call exact."""
    nbor, sizes = L.neighbors(L.FCC, 4)
    st = W.small_case(lattice=L.FCC, cell=4, species=(64, 64, 64, 64), seed=2)
    bad = nbor.copy()
    bad[3, 0] = bad[3, 1]  # a duplicate breaks symmetry with multiplicity
    occ = np.stack([np.random.default_rng(s).permutation(np.repeat(np.arange(4, dtype=np.uint8), 64))
                    for s in range(3)])
    with pytest.raises(hb.HeaError, match="symmetric"):
        hb.recount_noalloc(hb.Problem(bad, sizes, st.species, st.weight, st.target), occ)
    pb = hb.Problem(nbor, sizes, st.species, st.weight, st.target)
    cnt, f2 = hb.recount_noalloc(pb, occ)
    want_cnt, want_f2 = hb.recount(pb, occ)
    np.testing.assert_array_equal(cnt, want_cnt)
    np.testing.assert_array_equal(f2, want_f2)


def test_noalloc_recount_null_outputs_and_shape():
    pb = _problem(L.BCC, 5, (50, 50, 50, 50, 50), L.SHELLS_REFERENCE, 6)
    occ = hb.generate(pb, seed=3, generation=0, count=2)[0]
    _, want_f2 = hb.recount(pb, occ)
    f2 = np.empty(2)
    P = ctypes.POINTER
    optr = occ.ctypes.data_as(P(ctypes.c_uint8))
    assert hb.lib.hea_recount_noalloc(ctypes.byref(pb._c), 2, optr, None, f2.ctypes.data_as(P(ctypes.c_double))) == 0
    np.testing.assert_array_equal(f2, want_f2)
    assert hb.lib.hea_recount_noalloc(ctypes.byref(pb._c), 2, optr, None, None) == 0
    with pytest.raises(ValueError, match="occupancies"):
        hb.recount_noalloc(pb, occ[:, :-1])
    with pytest.raises(ValueError, match="occupancies"):
        hb.recount(pb, occ[:, :-1])


_CONTEXT_SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import pyhea_b200 as hb
from oracle import hea_oracle as ho
from pyhea_b200 import lattice as L, workloads as W

st = W.small_case(lattice=L.FCC, cell=6, species=(200, 264, 200, 200), shell_set=L.SHELLS_FCC_TRUE3, seed=4)
nbor, sizes = st.neighbors()
pb = hb.Problem(nbor, sizes, st.species, st.weight, st.target)
op = ho.Problem(pb.nbor, pb.shell_sizes, pb.species, pb.weight, pb.target_sro)
occ = np.stack([np.random.default_rng(s).permutation(np.repeat(np.arange(4, dtype=np.uint8), st.species))
                for s in range(5)])
want = np.stack([op.recount(o) for o in occ])
first = hb.recount_noalloc(pb, occ)                    # the primary context
cu = ctypes.CDLL("libcuda.so.1")
dev, ctx = ctypes.c_int(), ctypes.c_void_p()
assert cu.cuDeviceGet(ctypes.byref(dev), 0) == 0
assert cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev) == 0  # another context, current on this thread
other = hb.recount_noalloc(pb, occ)
assert cu.cuCtxDestroy_v2(ctx) == 0                    # back to the primary context
again = hb.recount_noalloc(pb, occ)
for cnt, f2 in (first, other, again):
    np.testing.assert_array_equal(cnt, want)
    assert all(f2[p] == op.f2(want[p]) for p in range(len(occ)))
print("contexts ok")
"""


def test_noalloc_recount_under_another_context():
    """The scratch array's address belongs to one context: with another
    context current on the thread the call must use that context's copy, and
    the primary context's again afterwards.  Run in a process of its own (no
    other library holds the device there)."""
    r = subprocess.run([sys.executable, "-c", _CONTEXT_SCRIPT, REPO], capture_output=True, text=True, timeout=300,
                       cwd=REPO, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "contexts ok" in r.stdout
