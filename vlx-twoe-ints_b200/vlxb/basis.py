"""Synthetic molecules, contracted Cartesian s/p/d basis sets and densities.

This is the caller side of the path (the role VeloxChem's host code plays for
the reference's emitted kernels): it defines the primitives, the AO map and
the density that the J/K entry points consume.  The workload recipes are those
of the benchmark configurations:

  * atoms placed uniformly at random in a cube by rejection sampling with a
    minimum separation of 1.5 bohr;
  * per atom, for each shell type, n contracted shells of `degree`
    primitives; primitive j of shell n has exponent alpha0 * ratio**(degree*n + j)
    (even-tempered, distinct for every primitive of the atom);
  * contraction coefficients drawn U(0.2, 1) (seeded), then the contracted
    function is normalised;
  * Cartesian d (and f) shells; every component of a shell shares the normalisation
    of its x^l component (so d_xx is unit-normalised, d_xy is not);
  * density D = C C^T with C ~ N(0,1)^(nao x nocc), orthonormalised in the
    overlap metric: C <- C (C^T S C)^(-1/2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Cartesian components in the reference's order (x^l first, then by
# decreasing y power); f follows the same rule.
CART = {0: [(0, 0, 0)],
        1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
        2: [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)],
        3: [(3, 0, 0), (2, 1, 0), (2, 0, 1), (1, 2, 0), (1, 1, 1), (1, 0, 2), (0, 3, 0), (0, 2, 1), (0, 1, 2),
            (0, 0, 3)]}
NCART = {0: 1, 1: 3, 2: 6, 3: 10}


def _dfact(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def prim_norm(alpha: float, l: int) -> float:
    """Normalisation of x^l exp(-alpha r^2)."""
    return math.sqrt((2.0 * alpha / math.pi) ** 1.5 * (4.0 * alpha) ** l / _dfact(2 * l - 1))


@dataclass
class Shell:
    atom: int
    l: int
    exps: np.ndarray
    coefs: np.ndarray   # includes primitive and contraction normalisation
    ao0: int = 0        # first Cartesian AO of the shell


@dataclass
class Molecule:
    coords: np.ndarray               # (natoms, 3) bohr
    shells: list = field(default_factory=list)
    naos: int = 0

    @property
    def natoms(self):
        return len(self.coords)


def place_atoms(n: int, side: float, rng: np.random.Generator, min_sep: float = 1.5,
                max_tries: int = 200000) -> np.ndarray:
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the requested minimum separation")
        p = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(p - q) >= min_sep for q in pts):
            pts.append(p)
    return np.array(pts)


def build_molecule(coords: np.ndarray, recipe: dict, degree: int, alpha0: float, ratio: float,
                   rng: np.random.Generator) -> Molecule:
    """recipe: {l: number of contracted shells of angular momentum l per atom}."""
    mol = Molecule(coords=np.asarray(coords, dtype=np.float64))
    ao = 0
    for a in range(len(coords)):
        for l in sorted(recipe):
            for n in range(recipe[l]):
                exps = np.array([alpha0 * ratio ** (degree * n + j) for j in range(degree)])
                c = rng.uniform(0.2, 1.0, size=degree)
                c = c * np.array([prim_norm(e, l) for e in exps])
                # normalise the contracted x^l component
                s = 0.0
                for i in range(degree):
                    for j in range(degree):
                        p = exps[i] + exps[j]
                        s += c[i] * c[j] * (math.pi / p) ** 1.5 * _dfact(2 * l - 1) / (2.0 * p) ** l
                c = c / math.sqrt(s)
                mol.shells.append(Shell(atom=a, l=l, exps=exps, coefs=c, ao0=ao))
                ao += NCART[l]
    mol.naos = ao
    return mol


# ------------------------------------------------------------------ overlap

def _overlap_1d(la, lb, PA, PB, p):
    """Obara-Saika 1D overlap factors s[i][j] (without the prefactor)."""
    s = np.zeros((la + 1, lb + 1) + np.shape(PA))
    s[0, 0] = 1.0
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = PA * s[i - 1, j]
                if i > 1:
                    v = v + (i - 1) / (2 * p) * s[i - 2, j]
                if j > 0:
                    v = v + j / (2 * p) * s[i - 1, j - 1]
            else:
                v = PB * s[i, j - 1]
                if j > 1:
                    v = v + (j - 1) / (2 * p) * s[i, j - 2]
            s[i, j] = v
    return s


def overlap_matrix(mol: Molecule) -> np.ndarray:
    """AO overlap matrix, one vectorised block per pair of shell types (all
    shell pairs and primitive pairs of the block at once)."""
    n = mol.naos
    S = np.zeros((n, n))
    by_l = {}
    for sh in mol.shells:
        by_l.setdefault(sh.l, []).append(sh)
    for la, sa in by_l.items():
        ea = np.array([sh.exps for sh in sa])                # (na, ka)
        ca = np.array([sh.coefs for sh in sa])
        A = np.array([mol.coords[sh.atom] for sh in sa])     # (na, 3)
        ao_a = np.array([sh.ao0 for sh in sa])
        for lb, sb in by_l.items():
            eb = np.array([sh.exps for sh in sb])
            cb = np.array([sh.coefs for sh in sb])
            B = np.array([mol.coords[sh.atom] for sh in sb])
            ao_b = np.array([sh.ao0 for sh in sb])
            # axes: shell a, shell b, primitive a, primitive b
            a_ = ea[:, None, :, None]
            b_ = eb[None, :, None, :]
            p = a_ + b_
            AB2 = np.sum((A[:, None, :] - B[None, :, :]) ** 2, axis=-1)[:, :, None, None]
            K = np.exp(-a_ * b_ / p * AB2) * (math.pi / p) ** 1.5
            cc = ca[:, None, :, None] * cb[None, :, None, :] * K
            s1 = []
            for x in range(3):
                Px = (a_ * A[:, None, None, None, x] + b_ * B[None, :, None, None, x]) / p
                s1.append(_overlap_1d(la, lb, Px - A[:, None, None, None, x], Px - B[None, :, None, None, x], p))
            for ia, (ax, ay, az) in enumerate(CART[la]):
                for ib, (bx, by, bz) in enumerate(CART[lb]):
                    v = (cc * s1[0][ax, bx] * s1[1][ay, by] * s1[2][az, bz]).sum(axis=(2, 3))
                    S[np.ix_(ao_a + ia, ao_b + ib)] = v
    return S


def make_density(mol: Molecule, nocc: int, rng: np.random.Generator, S: np.ndarray | None = None) -> np.ndarray:
    if S is None:
        S = overlap_matrix(mol)
    C = rng.standard_normal((mol.naos, nocc))
    M = C.T @ S @ C
    w, V = np.linalg.eigh(M)
    C = C @ (V @ np.diag(w ** -0.5) @ V.T)
    return C @ C.T


# ------------------------------------------------------------------ configs

@dataclass
class Workload:
    name: str
    mol: Molecule
    D: np.ndarray
    threshold: float
    nocc: int


def config_small(seed: int = 0) -> Workload:
    """5 atoms in a 6-bohr cube, 3s+2p shells of degree 3, alpha = 0.1 * 3^k,
    10 occupied orbitals, Schwarz threshold 1e-12 (plain FP64 build)."""
    rng = np.random.default_rng(seed)
    coords = place_atoms(5, 6.0, rng)
    mol = build_molecule(coords, {0: 3, 1: 2}, degree=3, alpha0=0.1, ratio=3.0, rng=rng)
    D = make_density(mol, 10, np.random.default_rng(seed + 1))
    return Workload("5 atoms 3s2p (45 Cartesian AOs)", mol, D, 1e-12, 10)


def config_medium(seed: int = 0) -> Workload:
    """40 atoms in a 14-bohr cube, 4s+3p+2d shells of degree 3,
    alpha = 0.05 * 2.5^k, 80 occupied orbitals (1000 Cartesian AOs)."""
    rng = np.random.default_rng(seed)
    coords = place_atoms(40, 14.0, rng)
    mol = build_molecule(coords, {0: 4, 1: 3, 2: 2}, degree=3, alpha0=0.05, ratio=2.5, rng=rng)
    D = make_density(mol, 80, np.random.default_rng(seed + 1))
    return Workload("40 atoms 4s3p2d (1000 Cartesian AOs)", mol, D, 1e-12, 80)


def config_custom(natoms: int, side: float, recipe: dict, degree: int, alpha0: float, ratio: float,
                  nocc: int, threshold: float = 1e-12, seed: int = 0) -> Workload:
    rng = np.random.default_rng(seed)
    coords = place_atoms(natoms, side, rng)
    mol = build_molecule(coords, recipe, degree=degree, alpha0=alpha0, ratio=ratio, rng=rng)
    D = make_density(mol, nocc, np.random.default_rng(seed + 1))
    return Workload(f"{natoms} atoms custom", mol, D, threshold, nocc)


def molecule_at_density(natoms: int, bohr3_per_atom: float, seed: int, threshold: float = 1e-12) -> Workload:
    """One molecule of the batched / served workloads: `natoms` atoms placed in a
    cube of side (natoms * bohr3_per_atom)^(1/3) bohr, the 4s+3p+2d recipe of
    degree 3 (alpha = 0.05 * 2.5^k), 2 occupied orbitals per atom."""
    side = (natoms * bohr3_per_atom) ** (1.0 / 3.0)
    wl = config_custom(natoms, side, {0: 4, 1: 3, 2: 2}, 3, 0.05, 2.5, 2 * natoms, threshold, seed)
    wl.name = f"{natoms} atoms 4s3p2d at {bohr3_per_atom:g} bohr^3/atom"
    return wl


def config_batch(n_mols: int = 256, atoms=(3, 30), bohr3_per_atom: float = 30.0, seed: int = 0) -> list:
    """Batched workload: n_mols independent molecules, atom counts uniform in
    [atoms[0], atoms[1]], 1 atom per 30 bohr^3, the 4s+3p+2d recipe."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(atoms[0], atoms[1] + 1, size=n_mols)
    return [molecule_at_density(int(n), bohr3_per_atom, seed * 100003 + t) for t, n in enumerate(counts)]


def serve_atom_counts(n_req: int, lo: int = 5, hi: int = 120, seed: int = 0) -> np.ndarray:
    """Atom counts of served requests: log-uniform on [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=n_req)).astype(int).clip(lo, hi)
