"""TARGET_SRO files and alpha matrices for any number of species.

The reference reads a per-shell lower triangle of the target Warren-Cowley
matrix and expands it to the full row-major [3][T*T] array the engine indexes
as target_sro[k][i*T + j] (pyhea/io/input.py:350-465).  It does so only for
T <= 4 (input.py:423-458); the expansion here is the same map written for any
T: full[i*T + j] = lower[max(i,j) * (max(i,j) + 1) / 2 + min(i,j)].

It also restates the per-shell alpha of a set of pair counts with the
reference's formula alpha_ij = 1 - gamma_ij / (c_i c_j), gamma = C / (Z_k N)
(pyhea/cpp/accelerate.cpp:171), so a searched structure can be compared to its
target without the third-party analyzer.

And it restates the analyzer the reference runs on its output files
(pyhea/utils/analyze.py:12-45): OVITO's WarrenCowleyParameters modifier with
nneigh = [0, 12, 18] (FCC) or [0, 8, 14] (BCC), the third-party package
WarrenCowleyParameters >= 2.0.0 (pyhea requirements.txt:10; not installed
here, so this restatement is unpinned against it).  Its published definition
(Cowley, Phys. Rev. 77, 669 (1950)): for each atom the neighbours are ranked
by distance (periodic images), shell m holds ranks nneigh[m] .. nneigh[m+1]-1,
and alpha^m_ij = 1 - P^m(j | i) / c_j, where P^m(j | i) is the fraction of
species-j atoms among the shell-m neighbours of species-i atoms and c_j the
concentration of j.  warren_cowley() computes that from positions and types;
where the rank ranges are whole coordination shells (FCC 12 + 6, BCC 8 + 6)
it equals alpha_from_counts on the engine's first two shells.
"""
import os

import numpy as np


def expand_lower_triangle(lower, num_types):
    """Lower triangle (row-major, T(T+1)/2 values) -> full T*T row-major list."""
    T = int(num_types)
    lower = np.asarray(lower, dtype=np.float64).ravel()
    if lower.size != T * (T + 1) // 2:
        raise ValueError(f"expected {T * (T + 1) // 2} values for {T} species, got {lower.size}")
    full = np.empty(T * T)
    for i in range(T):
        for j in range(T):
            hi, lo = max(i, j), min(i, j)
            full[i * T + j] = lower[hi * (hi + 1) // 2 + lo]
    return full


def _is_marker(line):
    low = line.lower()
    return low.startswith("shell") or low.startswith("second shell") or low.startswith("third shell")


def read_target_sro(path, num_types, shells=3):
    """Parse a TARGET_SRO file as pyhea/io/input.py:373-421 does and return the
    full [shells][T*T] array.  None -> all zeros (input.py:371-372).  Comment
    lines start with '#'; a line starting with 'shell', 'second shell' or
    'third shell' closes the current shell; other non-numeric lines are
    skipped; missing shells stay zero."""
    T = int(num_types)
    expected = T * (T + 1) // 2
    if path is None:
        return np.zeros((shells, T * T))
    if not os.path.exists(path):
        raise FileNotFoundError(f"Target SRO file not found: {path}")
    blocks, cur = [], []
    with open(path) as f:
        for raw in f:
            line = raw.strip()
            if not line or line.startswith("#"):
                continue
            if _is_marker(line):
                if cur:
                    if len(cur) != expected:
                        raise ValueError(f"Shell {len(blocks) + 1} has incorrect number of values. "
                                         f"Expected {expected}, got {len(cur)}")
                    blocks.append(cur)
                    cur = []
                continue
            try:
                cur.extend(float(v) for v in line.split())
            except ValueError:
                continue
    if cur:
        if len(cur) != expected:
            raise ValueError(f"Shell {len(blocks) + 1} has incorrect number of values. "
                             f"Expected {expected}, got {len(cur)}")
        blocks.append(cur)
    out = np.zeros((shells, T * T))
    for k, b in enumerate(blocks[:shells]):
        out[k] = expand_lower_triangle(b, T)
    return out


def alpha_from_counts(counts, shell_sizes, species):
    """Warren-Cowley alpha [S][T][T] from pair counts [S][T][T]."""
    counts = np.asarray(counts, dtype=np.float64)
    n = float(np.sum(species))
    c = np.asarray(species, dtype=np.float64) / n
    z = np.asarray(shell_sizes, dtype=np.float64)[:, None, None]
    gamma = counts / (z * n)
    return 1.0 - gamma / np.outer(c, c)[None]


def weighted_sro_error(counts, shell_sizes, species, weight, target):
    """sqrt(sum_k w_k sum_ij (alpha - target)^2): the reference fitness, in numpy."""
    a = alpha_from_counts(counts, shell_sizes, species)
    t = np.asarray(target, dtype=np.float64).reshape(a.shape)
    w = np.asarray(weight, dtype=np.float64)
    return float(np.sqrt(np.sum(w * np.sum((a - t) ** 2, axis=(1, 2)))))


ANALYZER_NNEIGH = {"FCC": (0, 12, 18), "BCC": (0, 8, 14)}  # pyhea/utils/analyze.py:35


def warren_cowley(positions, box, types, num_types=None, nneigh=(0, 12, 18)):
    """Warren-Cowley parameters [len(nneigh)-1][T][T] of a periodic structure, by neighbour rank.

    positions [N][3] Cartesian, box [3] edge lengths of an orthogonal periodic cell, types [N] in
    [0, T).  For every atom its nneigh[-1] nearest other atoms (minimum image) are ranked by
    distance; shell m is ranks [nneigh[m], nneigh[m+1]).  alpha^m_ij = 1 - P^m(j|i) / c_j with
    P^m(j|i) = (species-j neighbours in shell m of species-i atoms) / (n_i * shell size).
    A rank range that splits a set of equidistant neighbours depends on their order; keep the
    ranges at whole coordination shells."""
    from scipy.spatial import cKDTree

    pos = np.asarray(positions, dtype=np.float64)
    box = np.asarray(box, dtype=np.float64)
    types = np.asarray(types, dtype=np.int64)
    T = int(num_types) if num_types is not None else int(types.max()) + 1
    edges = [int(x) for x in nneigh]
    if edges[0] != 0 or any(b <= a for a, b in zip(edges, edges[1:])):
        raise ValueError("nneigh must start at 0 and increase")
    tree = cKDTree(np.mod(pos, box), boxsize=box)
    _, idx = tree.query(np.mod(pos, box), k=edges[-1] + 1)
    nb = idx[:, 1:]  # rank 0 is the atom itself
    counts = np.bincount(types, minlength=T).astype(np.float64)
    c = counts / counts.sum()
    out = np.zeros((len(edges) - 1, T, T))
    for m in range(len(edges) - 1):
        ranks = nb[:, edges[m]:edges[m + 1]]
        pair = np.zeros((T, T))
        np.add.at(pair, (np.repeat(types, ranks.shape[1]), types[ranks].ravel()), 1.0)
        P = pair / (counts[:, None] * ranks.shape[1])
        out[m] = 1.0 - P / c[None, :]
    return out


def warren_cowley_of_occupancy(occupancy, lattice, cell, num_types=None, nneigh=None):
    """warren_cowley() of an occupancy on the FCC (0) / BCC (1) cube of edge `cell` in the
    engine's site numbering, with the reference analyzer's rank ranges by default."""
    from . import lattice as _lat

    if nneigh is None:
        nneigh = ANALYZER_NNEIGH["FCC" if lattice == _lat.FCC else "BCC"]
    pos = _lat.positions(lattice, cell).astype(np.float64) * 0.5  # lattice units
    return warren_cowley(pos, np.full(3, float(cell)), occupancy, num_types, nneigh)
