"""Host-side FCC/BCC neighbour tables (numpy), the same tables the device
builder hea_build_neighbors makes.

Site numbering and shell order follow pyhea/lattice/lattice.py:
  FCC  id = 4 (x L^2 + y L + z) + basis, basis (0,0,0) (1/2,1/2,0) (1/2,0,1/2) (0,1/2,1/2)
       (calc_atom_id_fcc, lattice.py:109-144)
  BCC  id = 2 (x L^2 + y L + z) + basis, basis (0,0,0) (1/2,1/2,1/2)
       (calc_atom_id_bcc, lattice.py:72-107)
Each shell lists its neighbour ids in ascending order (np.sort at
lattice.py:236,245,256,302,311,320), periodic in every axis.

Shell sets:
  SHELLS_REFERENCE  FCC 12/6/12 with the third shell at sqrt(2) a, as the
                    reference builds it (lattice.py:283-287); BCC 8/6/12.
  SHELLS_FCC_TRUE3  FCC 12/6/24 with the third shell at sqrt(3/2) a; BCC 8/6/12.
"""
import itertools

import numpy as np

FCC, BCC = 0, 1
SHELLS_REFERENCE, SHELLS_FCC_TRUE3 = 0, 1

_BASIS = {FCC: np.array([[0, 0, 0], [1, 1, 0], [1, 0, 1], [0, 1, 1]]), BCC: np.array([[0, 0, 0], [1, 1, 1]])}


def _vectors(a, b, c):
    """All distinct axis/sign placements of (a, b, c), half lattice units."""
    out = set()
    for p in itertools.permutations((a, b, c)):
        for s in itertools.product((-1, 1), repeat=3):
            out.add(tuple(int(x * y) for x, y in zip(p, s)))
    return np.array(sorted(out))


def shell_vectors(lattice, shell_set=SHELLS_REFERENCE):
    if lattice == FCC:
        third = (2, 2, 0) if shell_set == SHELLS_REFERENCE else (2, 1, 1)
        return [_vectors(1, 1, 0), _vectors(2, 0, 0), _vectors(*third)]
    if lattice == BCC:
        return [_vectors(1, 1, 1), _vectors(2, 0, 0), _vectors(2, 2, 0)]
    raise ValueError(f"lattice must be FCC (0) or BCC (1), got {lattice}")


def num_sites(lattice, cell):
    return len(_BASIS[lattice]) * cell ** 3


def positions(lattice, cell):
    """Site positions in half lattice units, [N][3] int."""
    basis = _BASIS[lattice]
    nb = len(basis)
    s = np.arange(nb * cell ** 3)
    b, c = s % nb, s // nb
    xyz = np.stack([c // (cell * cell), (c // cell) % cell, c % cell], axis=1)
    return 2 * xyz + basis[b]


def neighbors(lattice, cell, shell_set=SHELLS_REFERENCE):
    """(nbor int32 [N][sum Z], shell_sizes int32 [3])."""
    basis = _BASIS[lattice]
    nb = len(basis)
    lut = -np.ones(8, dtype=np.int64)
    for i, (x, y, z) in enumerate(basis):
        lut[(x & 1) * 4 + (y & 1) * 2 + (z & 1)] = i
    pos = positions(lattice, cell)
    m = 2 * cell
    cols, sizes = [], []
    for vec in shell_vectors(lattice, shell_set):
        q = (pos[:, None, :] + vec[None, :, :]) % m
        bidx = lut[(q[..., 0] & 1) * 4 + (q[..., 1] & 1) * 2 + (q[..., 2] & 1)]
        if (bidx < 0).any():
            raise AssertionError("neighbour vector left the lattice")
        ids = nb * ((q[..., 0] >> 1) * cell * cell + (q[..., 1] >> 1) * cell + (q[..., 2] >> 1)) + bidx
        cols.append(np.sort(ids, axis=1))
        sizes.append(len(vec))
    return np.concatenate(cols, axis=1).astype(np.int32), np.array(sizes, dtype=np.int32)


def as_nested(nbor, shell_sizes):
    """The reference's nbor form: list[N] of list[S] of int arrays."""
    offs = np.concatenate([[0], np.cumsum(shell_sizes)])
    return [[row[offs[k]:offs[k + 1]] for k in range(len(shell_sizes))] for row in nbor]
