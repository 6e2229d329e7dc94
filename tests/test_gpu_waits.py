"""Bounded device-side waits of the persistent job engine run out cleanly.

Every spin of batch_kernel -- a CTA waiting in claim_job for queued work, or
for the producer's sequence number in a ring slot -- is bounded by a wall-time
limit counted from the last finished job.  Here the limit is set to a few
milliseconds while one structure's single local search runs far longer, so the
idle CTAs' waits run out: the kernel must return, the host must report the
error with a message, and a following run with the normal limit must give the
same result as searching the structure alone.  Nothing here faults or hangs a
GPU: the expiry is the designed exit of a bounded wait.
"""
import numpy as np
import pytest

import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu

# one solution, 20000 rounds of 64 tasks (the depth never ends it): tens of milliseconds
LONG = dict(num_solutions=1, total_iter=1, parallel_task=64, converge_depth=1 << 20, max_rounds=20000)


def _problem():
    st = W.small_case(lattice=L.BCC, cell=10, species=(700, 650, 650), shells=3, seed=5)
    nbor, sizes = st.neighbors()
    return hb.Problem(nbor, sizes, st.species, st.weight, st.target)


def test_batch_wait_limit_runs_out_and_the_next_run_is_exact():
    pb = _problem()
    want_occ, want_fit, want = hb.search(pb, LONG["num_solutions"], LONG["total_iter"], LONG["parallel_task"],
                                         LONG["converge_depth"], seed=9, max_rounds=LONG["max_rounds"])
    b = hb.Batch([pb], [LONG])
    b.set_wait_limit(2.0)
    with pytest.raises(hb.HeaError, match="time limit"):
        b.run([9])
    b.set_wait_limit(60_000.0)
    st = b.run([9])
    occ, fit = b.read(0)
    np.testing.assert_array_equal(occ, want_occ)
    np.testing.assert_array_equal(fit, want_fit)
    assert (st["rounds"], st["evals"], st["accepts"]) == (want["rounds"], want["evals"], want["accepts"])
    b.close()


def test_server_wait_limit_runs_out_with_a_message():
    pb = _problem()
    srv = hb.Server(max_requests=4, slice_ms=100.0, wait_limit_ms=2.0)
    srv.submit(pb, dict(LONG, seed=9))
    with pytest.raises(hb.HeaError, match="time limit"):
        for _ in range(1000):
            srv.step()
    with pytest.raises(hb.HeaError, match="server stopped"):
        srv.step()
    srv.close()
    # a server with the normal limit serves the same request
    srv = hb.Server(max_requests=4, slice_ms=100.0)
    rid = srv.submit(pb, dict(LONG, seed=9))
    res = None
    while res is None:
        srv.step()
        res = srv.result(rid)
    occ, fit, info = res
    want_occ, want_fit, _ = hb.search(pb, 1, 1, 64, 1 << 20, seed=9, max_rounds=20000)
    np.testing.assert_array_equal(occ, want_occ)
    np.testing.assert_array_equal(fit, want_fit)
    srv.close()
