"""Serving loop: requests admitted while others run give the same result as the
plain path on each request alone (same seed), bit for bit, however the time
slices fall, whatever shares the GPU, and whether the occupancy sits in shared
memory or HBM."""
import numpy as np
import pytest

import pyhea_b200 as hb
from pyhea_b200 import lattice as L
from pyhea_b200 import workloads as W

pytestmark = pytest.mark.gpu


def requests(seed=0, count=6):
    rng = np.random.default_rng(seed)
    specs = [(L.FCC, 4, L.SHELLS_FCC_TRUE3, 3), (L.BCC, 6, L.SHELLS_REFERENCE, 3), (L.FCC, 5, L.SHELLS_REFERENCE, 3),
             (L.BCC, 5, L.SHELLS_REFERENCE, 2), (L.FCC, 6, L.SHELLS_FCC_TRUE3, 3), (L.BCC, 8, L.SHELLS_REFERENCE, 1)]
    out = []
    for i in range(count):
        lat, cell, shell_set, S = specs[i % len(specs)]
        T = int(rng.integers(2, 7))
        species = W.dirichlet_counts(rng, T, L.num_sites(lat, cell))
        st = W.small_case(lattice=lat, cell=cell, species=species, shells=S, shell_set=shell_set, seed=i)
        nbor, sizes = st.neighbors()
        prm = dict(num_solutions=int(rng.integers(2, 7)), total_iter=int(rng.integers(0, 4)),
                   parallel_task=int(rng.choice([16, 37, 64, 300])), converge_depth=int(rng.integers(2, 8)),
                   seed=500 + 11 * i)
        out.append((st, hb.Problem(nbor, sizes, st.species, st.weight, st.target), prm))
    return out


def alone(pb, q, total_iter=None):
    occ, fit, _ = hb.search(pb, q["num_solutions"], q["total_iter"] if total_iter is None else total_iter,
                            q["parallel_task"], q["converge_depth"], seed=q["seed"])
    return occ, fit


def serve_all(srv, ids):
    got = {}
    for _ in range(100000):
        srv.step()
        for rid in ids:
            if rid not in got:
                r = srv.result(rid)
                if r is not None:
                    got[rid] = r
        if len(got) == len(ids):
            return got
    raise AssertionError("requests did not finish")


@pytest.mark.parametrize("slice_ms,hbm_sites", [(50.0, -1), (0.05, -1), (0.2, 0), (0.5, 400), (1.0, 1)])
def test_mix_equals_alone(slice_ms, hbm_sites):
    """Requests arriving over several steps, short slices (searches stop and resume
    many times), and occupancy in HBM for all or some requests."""
    items = requests(1, 6)
    srv = hb.Server(max_requests=4, slice_ms=slice_ms, hbm_sites=hbm_sites)
    ids = []
    for i, (_, pb, q) in enumerate(items):
        ids.append(srv.submit(pb, q, priority=i % 3))
        if i % 2:
            srv.step()  # later requests arrive while earlier ones run
    got = serve_all(srv, ids)
    assert srv.status()["launches"] >= 2
    for rid, (_, pb, q) in zip(ids, items):
        occ, fit, info = got[rid]
        aocc, afit = alone(pb, q)
        np.testing.assert_array_equal(occ, aocc, err_msg=f"request {rid}")
        np.testing.assert_array_equal(fit, afit, err_msg=f"request {rid}")
        assert info["state"] == 2 and info["iterations"] == q["total_iter"]
        assert info["hbm"] == (1 if hbm_sites == 0 or 0 < hbm_sites <= pb.num_sites else 0)
        assert info["finish_ms"] >= info["admit_ms"] >= info["submit_ms"]
    srv.close()


def test_lattice_request_equals_table_request():
    st = W.small_case(lattice=L.FCC, cell=5, species=(100, 200, 200), shells=3, shell_set=L.SHELLS_FCC_TRUE3, seed=4)
    q = dict(num_solutions=4, total_iter=2, parallel_task=64, converge_depth=5, seed=99)
    srv = hb.Server(slice_ms=1.0)
    a = srv.submit_lattice(st.lattice, st.cell, st.species, st.weight, st.target, q, shell_set=st.shell_set)
    b = srv.submit(st.problem(), q)
    got = serve_all(srv, [a, b])
    np.testing.assert_array_equal(got[a][0], got[b][0])
    np.testing.assert_array_equal(got[a][1], got[b][1])
    aocc, afit = alone(st.problem(), q)
    np.testing.assert_array_equal(got[a][0], aocc)
    srv.close()


def test_tolerance_same_alone_and_in_mix():
    """With a tolerance the request ends early (searches stop once they reach
    it); its result is the same served alone or among other requests."""
    st = W.small_case(lattice=L.BCC, cell=6, species=(216, 216), shells=2, seed=7)
    pb = st.problem()
    q = dict(num_solutions=4, total_iter=6, parallel_task=64, converge_depth=6, seed=3)
    full = alone(pb, q, total_iter=2)[1][0]  # fitness the plain path reaches after two iterations
    tol = float(full) * 1.5
    srv = hb.Server(slice_ms=5.0)
    rid = srv.submit(pb, q, tolerance=tol)
    occ, fit, info = serve_all(srv, [rid])[rid]
    k = info["iterations"]
    assert 1 <= k <= 2 and fit[0] <= tol
    srv.close()
    others = requests(5, 4)
    mix = hb.Server(slice_ms=0.1, max_requests=3)
    ids = [mix.submit(p, qq) for _, p, qq in others[:2]]
    mix.step()
    rid2 = mix.submit(pb, q, tolerance=tol)
    ids += [mix.submit(p, qq) for _, p, qq in others[2:]]
    got = serve_all(mix, ids + [rid2])
    np.testing.assert_array_equal(got[rid2][0], occ)
    np.testing.assert_array_equal(got[rid2][1], fit)
    assert got[rid2][2]["iterations"] == k
    for rid_o, (_, p, qq) in zip(ids, others):
        np.testing.assert_array_equal(got[rid_o][0], alone(p, qq)[0])
    mix.close()


def test_admission_waits_for_memory():
    """An arena that holds one request at a time: the others wait in the queue
    and are admitted as memory frees; every result is still the alone one."""
    st = W.small_case(lattice=L.FCC, cell=5, species=(150, 150, 200), shells=3, seed=2)
    pb = st.problem()
    qs = [dict(num_solutions=3, total_iter=2, parallel_task=48, converge_depth=4, seed=40 + i) for i in range(3)]
    probe = hb.Server(slice_ms=2.0)
    rid = probe.submit(pb, qs[0])
    probe.step()
    need = probe.info(rid)["device_bytes"]
    probe.close()
    assert need > 0
    srv = hb.Server(slice_ms=2.0, arena_bytes=need + need // 2)
    ids = [srv.submit(pb, q) for q in qs]
    assert srv.status()["queued"] == 3
    got = {}
    srv.step()
    assert srv.status()["queued"] == 2  # one admitted, two wait for its memory
    for _ in range(100000):
        srv.step()
        for rid in ids:
            if rid not in got:
                r = srv.result(rid)
                if r is not None:
                    got[rid] = r
        if len(got) == len(ids):
            break
    assert len(got) == 3
    spans = sorted((got[r][2]["admit_ms"], got[r][2]["finish_ms"]) for r in ids)
    for (_, fin), (adm, _) in zip(spans, spans[1:]):
        assert adm >= fin  # served one after the other
    for rid, q in zip(ids, qs):
        aocc, afit = alone(pb, q)
        np.testing.assert_array_equal(got[rid][0], aocc)
        np.testing.assert_array_equal(got[rid][1], afit)
    st = srv.status()
    assert st["arena_free_bytes"] == st["arena_bytes"]
    srv.close()


def test_bad_table_fails_only_that_request():
    st = W.small_case(lattice=L.BCC, cell=4, species=(64, 64), shells=2, seed=1)
    nbor, sizes = st.neighbors()
    bad = nbor.copy()
    bad[3, 0] = bad[3, 1]  # site 3 lists one neighbour twice: asymmetric
    q = dict(num_solutions=2, total_iter=1, parallel_task=32, converge_depth=3, seed=1)
    srv = hb.Server(slice_ms=2.0)
    rb = srv.submit(hb.Problem(bad, sizes, st.species, st.weight, st.target), q)
    rg = srv.submit(st.problem(), q)
    for _ in range(1000):
        srv.step()
        if srv.status()["running"] == 0 and srv.status()["queued"] == 0:
            break
    with pytest.raises(hb.HeaError, match="symmetric"):
        srv.result(rb)
    occ, fit, info = srv.result(rg)
    np.testing.assert_array_equal(occ, alone(st.problem(), q)[0])
    srv.close()


def test_submit_rejects_bad_arguments():
    st = W.small_case(lattice=L.BCC, cell=4, species=(64, 64), shells=2, seed=1)
    srv = hb.Server(slice_ms=2.0, ring_jobs=8)
    q = dict(num_solutions=8, total_iter=1, parallel_task=32, converge_depth=3, seed=1)
    with pytest.raises(hb.HeaError, match="job ring"):
        srv.submit(st.problem(), q)
    with pytest.raises(hb.HeaValueError, match="priority"):
        srv.submit(st.problem(), dict(q, num_solutions=2), priority=16)
    with pytest.raises(hb.HeaValueError):
        srv.result(12345)
    srv.close()
