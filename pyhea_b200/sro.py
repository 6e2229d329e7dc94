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
