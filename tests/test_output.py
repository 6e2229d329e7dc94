"""Structure writers against the reference's own output: POSCAR files written
by the reference writer (pyhea/io/output.py:62-106) and the reference's sample
LAMMPS output (examples/conf.lmp); fixtures from tests/golden/make_golden.py."""
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


def test_lammps_matches_reference_sample():
    """Byte-identical to the reference's sample LAMMPS output (examples/conf.lmp,
    fixture from tests/golden/make_golden.py lammps)."""
    import hashlib
    import json

    fx = json.load(open(os.path.join(GOLDEN, "lammps_conf.json")))
    occ = np.array([int(c) for c in fx["occupancy"]], dtype=np.uint8)
    text = output.lammps_text(occ, L.FCC, fx["cell"], fx["lattice_constant"], fx["num_types"])
    lines = text.splitlines()
    assert lines[:11] == fx["head"] and lines[-2:] == fx["tail"]
    assert hashlib.sha256(text.encode()).hexdigest() == fx["sha256"]


def test_lammps_roundtrip_and_write_structure(tmp_path):
    occ = np.random.default_rng(5).integers(0, 3, size=L.num_sites(L.BCC, 3))
    edges, tilts, ids, types, xyz = output.read_lammps(output.lammps_text(occ, L.BCC, 3, 2.5, 3))
    order = np.argsort(occ, kind="stable")
    np.testing.assert_array_equal(edges, [7.5, 7.5, 7.5])
    np.testing.assert_array_equal(tilts, [0.0, 0.0, 0.0])
    np.testing.assert_array_equal(ids, np.arange(1, occ.size + 1))
    np.testing.assert_array_equal(types, occ[order] + 1)
    np.testing.assert_array_equal(xyz, output.site_coordinates(L.BCC, 3)[order] * 2.5)
    # the reference writer's format names and file naming (pyhea/io/output.py:14-58)
    p = output.write_structure(str(tmp_path / "best.vasp"), occ, L.BCC, 3, 2.5, 3)
    assert p.endswith("best.vasp") and output.read_poscar(p)[3] == list(np.bincount(occ, minlength=3))
    p = output.write_structure(str(tmp_path / "best.vasp"), occ, L.BCC, 3, 2.5, 3, output_format="lammps/lmp")
    assert p.endswith("best.lmp") and open(p).read() == output.lammps_text(occ, L.BCC, 3, 2.5, 3)
    with pytest.raises(ValueError):
        output.write_structure(str(tmp_path / "x"), occ, L.BCC, 3, output_format="xyz")
