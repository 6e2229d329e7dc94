"""Structure files from searched occupancies.

`write_poscar` writes a VASP POSCAR in the layout of PyHEA's writer
(pyhea/io/output.py:62-106): title, scale (the lattice constant), the cubic
supercell vectors (edge = cell, in units of the scale), element labels A, B,
C, ... (one per species, as the reference writes them), atom counts per
species, "Cartesian", then the site coordinates grouped by species, each
group in site order.  Site coordinates are those of the reference lattice
builder (pyhea/lattice/lattice.py:146-190): site id = nb (x cell^2 + y cell +
z) + basis, basis offsets FCC (0,0,0) (½,½,0) (½,0,½) (0,½,½), BCC (0,0,0)
(½,½,½), in cell units.

Coordinates are multiples of ½, written with one decimal, so the text is
exact; large structures are formatted with numpy in one pass.
"""
import io

import numpy as np

from . import lattice as _lat


def site_coordinates(lattice, cell):
    """[N][3] float64 Cartesian coordinates in cell units."""
    return _lat.positions(lattice, cell) * 0.5


def poscar_text(occupancy, lattice, cell, lattice_constant=1.0, num_types=None, title="pyhea_b200"):
    """POSCAR text of one occupancy (species ids per site, [N])."""
    occ = np.asarray(occupancy).astype(np.int64).ravel()
    n = _lat.num_sites(lattice, cell)
    if occ.size != n:
        raise ValueError(f"occupancy has {occ.size} sites; the {cell}^3 supercell has {n}")
    T = int(num_types) if num_types is not None else int(occ.max()) + 1
    if occ.min() < 0 or occ.max() >= T:
        raise ValueError("species ids must lie in [0, num_types)")
    counts = np.bincount(occ, minlength=T)
    order = np.argsort(occ, kind="stable")  # grouped by species, site order inside a group
    xyz = site_coordinates(lattice, cell)[order]
    out = io.StringIO()
    out.write(f"{title}\n{float(lattice_constant)}\n")
    for r in range(3):
        v = [0.0, 0.0, 0.0]
        v[r] = float(cell)
        out.write("\t".join(str(x) for x in v) + "\n")
    out.write("   ".join(chr(65 + t) for t in range(T)) + "\n")
    out.write("   ".join(str(int(c)) for c in counts) + "\n")
    out.write("Cartesian\n")
    np.savetxt(out, xyz, fmt="%.1f", delimiter="\t")
    return out.getvalue()


def write_poscar(path, occupancy, lattice, cell, lattice_constant=1.0, num_types=None, title="pyhea_b200"):
    with open(path, "w") as f:
        f.write(poscar_text(occupancy, lattice, cell, lattice_constant, num_types, title))


def read_poscar(path_or_text):
    """(scale, vectors [3][3], labels, counts, coordinates [N][3]) of a Cartesian POSCAR."""
    text = path_or_text if "\n" in path_or_text else open(path_or_text).read()
    lines = text.splitlines()
    scale = float(lines[1])
    vec = np.array([[float(x) for x in lines[2 + r].split()] for r in range(3)])
    labels = lines[5].split()
    counts = [int(x) for x in lines[6].split()]
    assert lines[7].strip().lower().startswith("c")
    coords = np.array([[float(x) for x in ln.split()] for ln in lines[8:8 + sum(counts)]])
    return scale, vec, labels, counts, coords
