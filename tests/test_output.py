"""POSCAR writer against files written by the reference writer
(pyhea/io/output.py:62-106, fixtures from tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from pyhea_b200 import lattice as L
from pyhea_b200 import output

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = [("poscar_fcc3_t4.txt", L.FCC, 3, 4, 11), ("poscar_bcc4_t3.txt", L.BCC, 4, 3, 12)]


@pytest.mark.parametrize("name,lat,cell,T,seed", CASES)
def test_poscar_matches_reference_writer(name, lat, cell, T, seed):
    occ = np.random.default_rng(seed).integers(0, T, size=L.num_sites(lat, cell))
    ref = output.read_poscar(os.path.join(GOLDEN, name))
    ours = output.read_poscar(output.poscar_text(occ, lat, cell, lattice_constant=float(np.float16(3.6)), num_types=T))
    assert ours[0] == pytest.approx(ref[0])
    np.testing.assert_array_equal(ours[1], ref[1])
    assert ours[2] == ref[2] and ours[3] == ref[3]
    np.testing.assert_array_equal(ours[4], ref[4])


def test_poscar_counts_and_grouping():
    occ = np.array([2, 0, 1, 0, 2, 2, 1, 0], dtype=np.uint8)  # BCC 2^3 = 16 sites needs 16 entries
    with pytest.raises(ValueError):
        output.poscar_text(occ, L.BCC, 2)
    occ = np.tile(occ, 2)
    scale, vec, labels, counts, xyz = output.read_poscar(output.poscar_text(occ, L.BCC, 2))
    assert labels == ["A", "B", "C"] and counts == [6, 4, 6]
    pos = output.site_coordinates(L.BCC, 2)
    np.testing.assert_array_equal(xyz, pos[np.argsort(occ, kind="stable")])
