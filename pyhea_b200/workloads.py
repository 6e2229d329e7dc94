"""Seeded synthetic structures of the benchmark configurations.

Every structure is generated from a recorded seed with numpy's default_rng; the
search itself draws from Philox with its own seed.  Target alpha matrices are
symmetric; zero (concentration-weighted) row sums make them consistent with a
pair-probability matrix (sum_j c_j alpha_ij = 0).

  plain_cpu   FCC 10^3 (4000 sites, 12/6/24 shells), 4 x 1000 atoms, off-diagonal
              alpha ~ U(-0.1, 0.1) with diagonals making each row sum to zero,
              weights [4, 1, 0.5]; P=128, Q=256, I=10, D=10
  plain_gpu   BCC 20^3 (16000 sites, 8/6/12), 5 x 3200 atoms, alpha ~ U(-0.15, 0.15)
              with zero row sums; P=256, Q=512, I=50, D=20
  batched     64 structures: FCC/BCC (p=0.5), edge U{6..30}, 3-6 species with
              Dirichlet(2) compositions (largest remainder, every count >= 1),
              alpha ~ U(-0.1, 0.1) projected onto sum_j c_j alpha_ij = 0;
              P=64, Q=256 (I=10, D=10)
  large       FCC 100^3 (4,000,000 sites, 12/6/24), 4 species at 0.25, alpha ~
              U(-0.05, 0.05) with zero row sums; P=32, Q=4096, I=200, D=20
  serving     Poisson request stream; FCC/BCC supercells with log-uniform site
              counts in [4e3, 1e6], 3-6 species (Dirichlet(2)), projected
              alpha ~ U(-0.1, 0.1)
"""
import numpy as np

from . import lattice as _lat

WEIGHTS = [4.0, 1.0, 0.5]


def zero_row_sum_target(rng, T, amp, shells=3):
    """Symmetric [S][T*T]: off-diagonals U(-amp, amp), diagonals set so each row sums to 0."""
    out = np.zeros((shells, T, T))
    for k in range(shells):
        a = rng.uniform(-amp, amp, size=(T, T))
        a = np.triu(a, 1)
        a = a + a.T
        np.fill_diagonal(a, -a.sum(axis=1))
        out[k] = a
    return out.reshape(shells, T * T)


def projected_target(rng, conc, amp, shells=3):
    """Symmetric [S][T*T]: U(-amp, amp) symmetrised, then projected onto sum_j c_j a_ij = 0
    (A -> P A P with P = I - c c^T / c^T c, the orthogonal projection onto that subspace)."""
    c = np.asarray(conc, dtype=float)
    T = len(c)
    Pm = np.eye(T) - np.outer(c, c) / c.dot(c)
    out = np.zeros((shells, T, T))
    for k in range(shells):
        a = rng.uniform(-amp, amp, size=(T, T))
        a = 0.5 * (a + a.T)
        out[k] = Pm @ a @ Pm
    return out.reshape(shells, T * T)


def dirichlet_counts(rng, T, n, alpha=2.0):
    """Integer composition summing to n from Dirichlet(alpha), largest remainder, all >= 1."""
    p = rng.dirichlet([alpha] * T)
    raw = p * (n - T)
    base = np.floor(raw).astype(np.int64)
    rem = int((n - T) - base.sum())
    order = np.argsort(-(raw - base), kind="stable")
    base[order[:rem]] += 1
    return (base + 1).astype(np.int32)


class Structure:
    """One search problem: neighbour table, shells, species, weights, target and search sizes."""

    def __init__(self, lattice, cell, shell_set, species, weight, target, P, Q, I, D, name=""):
        self.lattice, self.cell, self.shell_set = lattice, cell, shell_set
        self.species = np.asarray(species, dtype=np.int32)
        self.weight = np.asarray(weight, dtype=np.float64)
        self.target = np.asarray(target, dtype=np.float64)
        self.P, self.Q, self.I, self.D = P, Q, I, D
        self.name = name
        self._nbor = None

    @property
    def num_sites(self):
        return _lat.num_sites(self.lattice, self.cell)

    def neighbors(self, device=False):
        if self._nbor is None:
            if device:
                from . import build_neighbors

                self._nbor = build_neighbors(self.lattice, self.cell, self.shell_set)
            else:
                self._nbor = _lat.neighbors(self.lattice, self.cell, self.shell_set)
        return self._nbor

    def shell_sizes(self):
        return _lat.shell_vectors(self.lattice, self.shell_set)

    def problem(self, device=False, implicit=False):
        """Problem with the neighbour table (built on the device when `device`), or, with
        `implicit`, the lattice description instead of a table."""
        from . import Problem

        if implicit:
            return Problem.from_lattice(self.lattice, self.cell, self.species, self.weight, self.target,
                                        shell_set=self.shell_set)
        nbor, sizes = self.neighbors(device)
        return Problem(nbor, sizes, self.species, self.weight, self.target)

    def evals_bytes(self):
        """Algorithmic bytes of one swap evaluation: 2 sum Z (4 B id + 1 B species) + 2 B centres."""
        z = sum(len(v) for v in _lat.shell_vectors(self.lattice, self.shell_set)[: len(self.weight)])
        return 2 * z * 5 + 2


def plain_cpu(seed=0):
    rng = np.random.default_rng(seed)
    return Structure(_lat.FCC, 10, _lat.SHELLS_FCC_TRUE3, [1000] * 4, WEIGHTS, zero_row_sum_target(rng, 4, 0.1),
                     P=128, Q=256, I=10, D=10, name="fcc10_t4_12-6-24")


def plain_gpu(seed=0):
    rng = np.random.default_rng(seed)
    return Structure(_lat.BCC, 20, _lat.SHELLS_REFERENCE, [3200] * 5, WEIGHTS, zero_row_sum_target(rng, 5, 0.15),
                     P=256, Q=512, I=50, D=20, name="bcc20_t5_8-6-12")


def batched(seed=0, count=64, P=64, Q=256, I=10, D=10):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        lat = _lat.FCC if rng.random() < 0.5 else _lat.BCC
        cell = int(rng.integers(6, 31))
        T = int(rng.integers(3, 7))
        n = _lat.num_sites(lat, cell)
        species = dirichlet_counts(rng, T, n)
        target = projected_target(rng, species / n, 0.1)
        shells = _lat.SHELLS_FCC_TRUE3 if lat == _lat.FCC else _lat.SHELLS_REFERENCE
        out.append(Structure(lat, cell, shells, species, WEIGHTS, target, P=P, Q=Q, I=I, D=D,
                             name=f"{'fcc' if lat == _lat.FCC else 'bcc'}{cell}_t{T}"))
    return out


def large(seed=0):
    rng = np.random.default_rng(seed)
    return Structure(_lat.FCC, 100, _lat.SHELLS_FCC_TRUE3, [1_000_000] * 4, WEIGHTS,
                     zero_row_sum_target(rng, 4, 0.05), P=32, Q=4096, I=200, D=20, name="fcc100_t4_12-6-24")


def serving(seed=0, rate=200.0, duration=60.0, P=8, Q=256, I=4, D=10, n_min=4e3, n_max=1e6):
    """Request stream of the serving loop: Poisson arrivals at `rate` per second
    for `duration` seconds; each request an FCC/BCC (p=0.5) supercell whose site
    count is log-uniform in [n_min, n_max] (rounded to the nearest cubic cell
    inside the range), 3-6 species with Dirichlet(2) compositions, alpha ~
    U(-0.1, 0.1) projected onto sum_j c_j alpha_ij = 0.  Returns a list of
    (arrival seconds, Structure)."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        lat = _lat.FCC if rng.random() < 0.5 else _lat.BCC
        nb = 4 if lat == _lat.FCC else 2
        n_goal = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        cell = max(2, int(round((n_goal / nb) ** (1.0 / 3.0))))
        while nb * cell ** 3 > n_max and cell > 2:
            cell -= 1
        while nb * cell ** 3 < n_min:
            cell += 1
        n = nb * cell ** 3
        T = int(rng.integers(3, 7))
        species = dirichlet_counts(rng, T, n)
        target = projected_target(rng, species / n, 0.1)
        shells = _lat.SHELLS_FCC_TRUE3 if lat == _lat.FCC else _lat.SHELLS_REFERENCE
        out.append((t, Structure(lat, cell, shells, species, WEIGHTS, target, P=P, Q=Q, I=I, D=D,
                                 name=f"{'fcc' if lat == _lat.FCC else 'bcc'}{cell}_t{T}")))


def small_case(lattice=_lat.FCC, cell=4, species=(64, 64, 64, 64), shells=3, shell_set=_lat.SHELLS_REFERENCE, seed=0,
               P=4, Q=32, I=2, D=4):
    """A structure small enough for the CPU oracle."""
    rng = np.random.default_rng(seed)
    species = np.asarray(species, dtype=np.int32)
    target = projected_target(rng, species / species.sum(), 0.1)
    return Structure(lattice, cell, shell_set, species, WEIGHTS[:shells], target[:shells], P=P, Q=Q, I=I, D=D,
                     name="small")
