"""Host-side inputs of the search pinned against the reference: neighbour
tables (pyhea/lattice/lattice.py) and TARGET_SRO expansion (pyhea/io/input.py)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from pyhea_b200 import lattice as L
from pyhea_b200 import sro


@pytest.mark.parametrize("typ,lat", [("FCC", L.FCC), ("BCC", L.BCC)])
@pytest.mark.parametrize("cell", [3, 4])
def test_neighbors_match_reference(golden_nbor, typ, lat, cell):
    nbor, sizes = L.neighbors(lat, cell)
    np.testing.assert_array_equal(nbor, golden_nbor[f"{typ}_{cell}"])
    np.testing.assert_array_equal(sizes, golden_nbor[f"{typ}_{cell}_shells"])


@pytest.mark.parametrize("lat,shell_set,dist", [
    (L.FCC, L.SHELLS_REFERENCE, [0.5 ** 0.5, 1.0, 2 ** 0.5]),
    (L.FCC, L.SHELLS_FCC_TRUE3, [0.5 ** 0.5, 1.0, 1.5 ** 0.5]),
    (L.BCC, L.SHELLS_REFERENCE, [0.75 ** 0.5, 1.0, 2 ** 0.5]),
])
def test_neighbor_distances_and_symmetry(lat, shell_set, dist):
    cell = 5
    nbor, sizes = L.neighbors(lat, cell, shell_set)
    pos = L.positions(lat, cell) / 2.0
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for k in range(3):
        ids = nbor[:, offs[k]:offs[k + 1]]
        d = pos[ids] - pos[:, None, :]
        d -= cell * np.round(d / cell)
        np.testing.assert_allclose(np.sqrt((d ** 2).sum(-1)), dist[k], atol=1e-12)
        assert all(len(set(r)) == len(r) for r in ids.tolist())
        # symmetric: n in shell k of s  <=>  s in shell k of n
        pairs = set(zip(np.repeat(np.arange(len(ids)), ids.shape[1]).tolist(), ids.ravel().tolist()))
        assert all((b, a) in pairs for a, b in pairs)
    assert list(sizes) == ([12, 6, 24] if shell_set == L.SHELLS_FCC_TRUE3 and lat == L.FCC else
                           [12, 6, 12] if lat == L.FCC else [8, 6, 12])


def test_target_sro_expansion_matches_reference():
    cases = json.load(open(os.path.join(GOLDEN, "target_sro.json")))
    for T in ("2", "3", "4"):
        lower = cases[T]["lower"]
        full = np.array(cases[T]["full"])
        for k in range(3):
            np.testing.assert_array_equal(sro.expand_lower_triangle(lower[k], int(T)), full[k])
    np.testing.assert_array_equal(sro.read_target_sro(None, 4), np.array(cases["default_4"]["full"]))


def test_target_sro_file_any_species(tmp_path):
    T = 6
    vals = np.arange(T * (T + 1) // 2) / 100.0
    text = ["# comment", "First Shell"]
    pos = 0
    for r in range(T):
        text.append(" ".join(str(v) for v in vals[pos:pos + r + 1]))
        pos += r + 1
    text += ["Second Shell"] + [" ".join(["0.5"] * (r + 1)) for r in range(T)]
    p = tmp_path / "TARGET_SRO"
    p.write_text("\n".join(text) + "\n")
    full = sro.read_target_sro(str(p), T)
    assert full.shape == (3, T * T)
    m = full[0].reshape(T, T)
    np.testing.assert_array_equal(m, m.T)
    assert m[5, 2] == vals[5 * 6 // 2 + 2]
    np.testing.assert_array_equal(full[1], 0.5)
    np.testing.assert_array_equal(full[2], 0.0)
    p.write_text("Shell\n0.1 0.2\n")
    with pytest.raises(ValueError):
        sro.read_target_sro(str(p), 2)


def test_weighted_error_matches_oracle_fitness(golden_engine, golden_nbor):
    from conftest import engine_case_problem
    from oracle import hea_oracle as ho

    case = golden_engine["fcc4_t4_s3"]
    pr = engine_case_problem(case, golden_nbor, ho)
    C = pr.recount(case["occ"][0].astype(np.uint8))
    f = sro.weighted_sro_error(C, case["shell_size"], case["species"], case["weight"], case["target"])
    assert abs(f - case["fitness"][0]) < 1e-12 * case["fitness"][0]


def test_alpha_matches_reference_gamma(golden_engine, golden_nbor):
    """alpha from the oracle's integer counts equals 1 - gamma/(c_i c_j) with the
    reference engine's own gamma (accelerate.cpp:370-399, :171)."""
    from conftest import engine_case_problem
    from oracle import hea_oracle as ho

    for name in ("fcc4_t4_s3", "bcc4_t3_s2", "bcc4_t6_s3"):
        case = golden_engine[name]
        pr = engine_case_problem(case, golden_nbor, ho)
        sp = np.asarray(case["species"], dtype=np.float64)
        c = sp / sp.sum()
        for p in range(len(case["occ"])):
            C = pr.recount(case["occ"][p].astype(np.uint8))
            a = sro.alpha_from_counts(C, case["shell_size"], case["species"])
            gamma = np.moveaxis(np.asarray(case["gamma"][p]), -1, 0)  # [T][T][S] -> [S][T][T]
            ref_alpha = 1.0 - gamma / np.outer(c, c)[None]
            np.testing.assert_allclose(a, ref_alpha, rtol=0, atol=1e-12)


@pytest.mark.parametrize("lat,cell,T", [(L.FCC, 5, 4), (L.BCC, 6, 3), (L.FCC, 4, 6), (L.BCC, 10, 5)])
def test_analyzer_restatement_equals_alpha_from_counts(lat, cell, T):
    """The analyzer's convention (pyhea/utils/analyze.py:35: neighbour ranks [0, 12, 18] FCC,
    [0, 8, 14] BCC) gives, on perfect lattices, the engine-convention alpha of shells 1-2."""
    from oracle import hea_oracle as ho

    nbor, sizes = L.neighbors(lat, cell)
    n = L.num_sites(lat, cell)
    for seed in range(3):
        occ = np.random.default_rng(seed).permutation(np.arange(n) % T).astype(np.uint8)
        sp = np.bincount(occ, minlength=T)
        op = ho.Problem(nbor, sizes, sp, [4.0, 1.0, 0.5], np.zeros((3, T * T)))
        wc = sro.warren_cowley_of_occupancy(occ, lat, cell, T)
        a = sro.alpha_from_counts(op.recount(occ), sizes, sp)
        assert wc.shape == (2, T, T)
        np.testing.assert_allclose(wc, a[:2], rtol=0, atol=1e-12)
        np.testing.assert_allclose(wc, wc.transpose(0, 2, 1), rtol=0, atol=1e-12)


def test_analyzer_restatement_on_a_written_structure_file(tmp_path):
    """End to end as the reference post-processes (write the structure, analyse the file): a POSCAR
    written by the reference-format writer and read back gives the same parameters."""
    from pyhea_b200 import output

    lat, cell, T = L.FCC, 4, 4
    n = L.num_sites(lat, cell)
    occ = np.random.default_rng(7).permutation(np.arange(n) % T)
    path = str(tmp_path / "out.poscar")
    output.write_poscar(path, occ, lat, cell, lattice_constant=3.6, num_types=T)
    scale, vec, labels, counts, coords = output.read_poscar(path)
    types = np.repeat(np.arange(T), counts)
    got = sro.warren_cowley(coords * scale, np.diag(vec) * scale, types, T, sro.ANALYZER_NNEIGH["FCC"])
    want = sro.warren_cowley_of_occupancy(occ, lat, cell, T)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
