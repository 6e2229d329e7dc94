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

`write_lammps` writes the LAMMPS data file PyHEA produces for
`output_format="lammps/lmp"` (pyhea/io/output.py:14-58, pyhea/model/opt.py:
104-114), which converts its POSCAR with the third-party dpdata package.  The
layout restated here is the one of the reference's sample output
(examples/conf.lmp): a blank first line, "<N> atoms", "<T> atom types", the
orthogonal box [0, cell a] on each axis ("%15.10f %15.10f xlo xhi", ...), the
three zero tilt factors ("... xy xz yz"), a blank line, "Atoms # atomic", a
blank line, then one line per atom "%6d %6d %15.10f %15.10f %15.10f" (id from
1, type = species + 1, Cartesian x y z in Å), in the POSCAR order.
`write_structure` picks the format by name as the reference's writer does.
"""
import io
import os

import numpy as np

from . import lattice as _lat


def site_coordinates(lattice, cell):
    """[N][3] float64 Cartesian coordinates in cell units."""
    return _lat.positions(lattice, cell) * 0.5


def poscar_text(occupancy, lattice, cell, lattice_constant=1.0, num_types=None, title="pyhea_b200"):
    """POSCAR text of one occupancy (species ids per site, [N])."""
    occ, order, T = _grouped(occupancy, lattice, cell, num_types)
    counts = np.bincount(occ, minlength=T)
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


def _grouped(occupancy, lattice, cell, num_types):
    occ = np.asarray(occupancy).astype(np.int64).ravel()
    n = _lat.num_sites(lattice, cell)
    if occ.size != n:
        raise ValueError(f"occupancy has {occ.size} sites; the {cell}^3 supercell has {n}")
    T = int(num_types) if num_types is not None else int(occ.max()) + 1
    if occ.min() < 0 or occ.max() >= T:
        raise ValueError("species ids must lie in [0, num_types)")
    order = np.argsort(occ, kind="stable")  # grouped by species, site order inside a group
    return occ, order, T


def lammps_text(occupancy, lattice, cell, lattice_constant=1.0, num_types=None):
    """LAMMPS data text ("atomic" style) of one occupancy (species ids per site, [N])."""
    occ, order, T = _grouped(occupancy, lattice, cell, num_types)
    a = float(lattice_constant)
    edge = float(cell) * a
    out = io.StringIO()
    out.write(f"\n{occ.size} atoms\n{T} atom types\n")
    for axis in ("x", "y", "z"):
        out.write("%15.10f %15.10f %slo %shi\n" % (0.0, edge, axis, axis))
    out.write("%15.10f %15.10f %15.10f xy xz yz\n" % (0.0, 0.0, 0.0))
    out.write("\nAtoms # atomic\n\n")
    xyz = site_coordinates(lattice, cell)[order] * a
    ids = np.arange(1, occ.size + 1, dtype=np.int64)
    types = occ[order] + 1
    for i in range(0, occ.size, 1 << 16):  # chunks keep the temporary strings small
        rows = zip(ids[i:i + (1 << 16)].tolist(), types[i:i + (1 << 16)].tolist(), *xyz[i:i + (1 << 16)].T.tolist())
        out.write("".join("%6d %6d %15.10f %15.10f %15.10f\n" % r for r in rows))
    return out.getvalue()


def write_lammps(path, occupancy, lattice, cell, lattice_constant=1.0, num_types=None):
    with open(path, "w") as f:
        f.write(lammps_text(occupancy, lattice, cell, lattice_constant, num_types))


def read_lammps(path_or_text):
    """(box edges [3], tilts [3], ids [N], types [N], coordinates [N][3]) of an atomic-style data file."""
    text = path_or_text if "\n" in path_or_text else open(path_or_text).read()
    lines = text.splitlines()
    n = int(next(ln for ln in lines if ln.endswith(" atoms")).split()[0])
    edges = [float(next(ln for ln in lines if ln.endswith(f"{x}lo {x}hi")).split()[1]) for x in "xyz"]
    tilts = [float(v) for v in next(ln for ln in lines if ln.endswith("xy xz yz")).split()[:3]]
    start = lines.index("Atoms # atomic") + 2
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[start:start + n]])
    return np.array(edges), np.array(tilts), rows[:, 0].astype(np.int64), rows[:, 1].astype(np.int64), rows[:, 2:5]


def write_structure(path, occupancy, lattice, cell, lattice_constant=1.0, num_types=None,
                    output_format="vasp/poscar"):
    """The reference's writer entry (pyhea/io/output.py:14-58): "vasp/poscar"
    writes `path`; "lammps/lmp" writes `path` with its extension replaced by
    ".lmp".  Returns the path written; other formats raise ValueError."""
    if output_format == "vasp/poscar":
        write_poscar(path, occupancy, lattice, cell, lattice_constant, num_types)
        return path
    if output_format == "lammps/lmp":
        out = os.path.splitext(path)[0] + ".lmp"
        write_lammps(out, occupancy, lattice, cell, lattice_constant, num_types)
        return out
    raise ValueError(f"Unsupported output format: {output_format}")
