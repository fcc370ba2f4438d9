"""Seeded synthetic structures for the benchmark and parity workloads.

All generators return ``Molecule`` objects in Bohr with species indices that
refer to the synthetic H/C/O parameter file (H=0, C=1, O=2).  The inputs are
synthetic stand-ins built from the workload rules (no dataset is involved):

* n-alkanes C_nH_{2n+2}, all-trans, C-C 1.54 A, C-H 1.09 A, tetrahedral angles,
  seeded Gaussian jitter (sigma 0.02 A) on every coordinate;
* water clusters of rigid H2O (O-H 0.96 A, H-O-H 104.5 deg) placed on a cubic
  grid of 3.1 A spacing filled in seeded random order, uniformly random
  orientation (random unit quaternion), sigma 0.05 A jitter;
* a 10x10x10 water box (3000 atoms) from the same rules;
* a Poisson-arrival request stream with log-uniform sizes, 50/50 water/alkane.

Seeds follow ``numpy.random.default_rng(1000 + workload_index)`` unless a seed
is given explicitly.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

ANGSTROM = 1.0 / 0.529177210903  # Bohr per Angstrom
H, C, O = 0, 1, 2
TETRA = math.acos(-1.0 / 3.0)  # 109.4712 deg


@dataclasses.dataclass
class Molecule:
    """One structure: species indices, Cartesian coordinates (Bohr), charge, uhf."""

    id: np.ndarray          # int32 [nat]
    xyz: np.ndarray         # float64 [nat, 3], Bohr
    charge: float = 0.0
    uhf: int = 0
    label: str = ""

    @property
    def nat(self) -> int:
        return int(self.id.shape[0])


def _unit(v):
    return v / np.linalg.norm(v)


def _rotation_from_quaternion(q):
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _random_rotation(rng):
    q = rng.normal(size=4)
    return _rotation_from_quaternion(q / np.linalg.norm(q))


def alkane_ideal(n: int) -> tuple[np.ndarray, np.ndarray]:
    """All-trans C_nH_{2n+2} in Angstrom (ideal geometry, no jitter)."""
    rcc, rch = 1.54, 1.09
    half = 0.5 * TETRA
    dx, dy = rcc * math.sin(half), rcc * math.cos(half)

    def cpos_of(k):  # zig-zag backbone in the xy plane, also for virtual k=-1, n
        return np.array([k * dx, (k % 2) * dy, 0.0])

    cpos = np.array([cpos_of(k) for k in range(n)])
    hpos = []
    for k in range(n):
        if n == 1:  # methane
            for d in ([1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]):
                hpos.append(cpos[k] + rch * _unit(np.array(d, float)))
            continue
        nbrs = [cpos[j] - cpos[k] for j in (k - 1, k + 1) if 0 <= j < n]
        if len(nbrs) == 2:
            u1, u2 = _unit(nbrs[0]), _unit(nbrs[1])
            b = -_unit(u1 + u2)
            nrm = _unit(np.cross(u1, u2))
            for sgn in (1.0, -1.0):
                hpos.append(cpos[k] + rch * (b * math.cos(half) + sgn * nrm * math.sin(half)))
        else:
            u = _unit(nbrs[0])
            virt = cpos_of(-1) if k == 0 else cpos_of(n)
            d0 = _unit(virt - cpos[k])                 # trans H, in the backbone plane
            e1 = _unit(d0 - np.dot(d0, u) * u)
            e2 = np.cross(u, e1)
            ct = math.cos(TETRA)
            st = math.sin(TETRA)
            for phi in (0.0, 2.0 * math.pi / 3.0, -2.0 * math.pi / 3.0):
                d = ct * u + st * (math.cos(phi) * e1 + math.sin(phi) * e2)
                hpos.append(cpos[k] + rch * d)
    xyz = np.vstack([cpos, np.array(hpos)])
    species = np.array([C] * n + [H] * len(hpos), dtype=np.int32)
    return species, xyz


def alkane(n: int, rng: np.random.Generator, sigma: float = 0.02) -> Molecule:
    sp, xyz = alkane_ideal(n)
    xyz = xyz + rng.normal(scale=sigma, size=xyz.shape)
    return Molecule(sp, np.ascontiguousarray(xyz * ANGSTROM), label=f"C{n}H{2 * n + 2}")


def water_cluster(nwat: int, rng: np.random.Generator, spacing: float = 3.1,
                  sigma: float = 0.05, grid: int | None = None) -> Molecule:
    """nwat rigid waters on a cubic grid (spacing in Angstrom), random order/orientation."""
    roh, ang = 0.96, math.radians(104.5)
    mono = np.array([
        [0.0, 0.0, 0.0],
        [roh * math.sin(0.5 * ang), 0.0, roh * math.cos(0.5 * ang)],
        [-roh * math.sin(0.5 * ang), 0.0, roh * math.cos(0.5 * ang)],
    ])
    com = (16.0 * mono[0] + 1.008 * (mono[1] + mono[2])) / (16.0 + 2 * 1.008)
    mono = mono - com
    side = grid if grid is not None else int(math.ceil(round(nwat ** (1.0 / 3.0), 9)))
    while side ** 3 < nwat:
        side += 1
    sites = np.array([[i, j, k] for i in range(side) for j in range(side) for k in range(side)],
                     dtype=float) * spacing
    order = rng.permutation(len(sites))[:nwat]
    xyz, sp = [], []
    for s in order:
        rot = _random_rotation(rng)
        xyz.append(sites[s] + mono @ rot.T)
        sp.extend([O, H, H])
    xyz = np.vstack(xyz)
    xyz = xyz + rng.normal(scale=sigma, size=xyz.shape)
    return Molecule(np.array(sp, dtype=np.int32), np.ascontiguousarray(xyz * ANGSTROM),
                    label=f"(H2O){nwat}")


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

def octane(seed: int = 1000) -> Molecule:
    """n-octane C8H18, all-trans, sigma 0.02 A (single plain FP64 singlepoint)."""
    return alkane(8, np.random.default_rng(seed))


def water_clusters(count: int = 1024, seed: int = 1001, nmin: int = 8, nmax: int = 64):
    """`count` water clusters with U{nmin..nmax} molecules each (uneven batch)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [water_cluster(int(n), rng) for n in sizes]


def alkanes(count: int = 256, seed: int = 1002, nmin: int = 20, nmax: int = 200):
    """`count` alkane chains C_nH_{2n+2}, n ~ U{nmin..nmax}."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [alkane(int(n), rng) for n in sizes]


def request_stream(count: int = 20000, seed: int = 1003, rate: float = 2000.0,
                   amin: int = 10, amax: int = 600):
    """Poisson arrivals (rate per second) of log-uniform sized water/alkane requests.

    Returns a list of (arrival_time_s, Molecule).
    """
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps)
    out = []
    for i in range(count):
        target = math.exp(rng.uniform(math.log(amin), math.log(amax)))
        if rng.uniform() < 0.5:
            nw = max(1, int(round(target / 3.0)))
            mol = water_cluster(nw, rng)
        else:
            n = max(1, int(round((target - 2.0) / 3.0)))
            mol = alkane(n, rng)
        out.append((float(t[i]), mol))
    return out


def water_box(seed: int = 1004) -> Molecule:
    """1000 H2O on a 10x10x10 grid at 3.1 A (3000 atoms)."""
    return water_cluster(1000, np.random.default_rng(seed), grid=10)


def write_xyz(mol: Molecule, path: str, symbols=("H", "C", "O")) -> None:
    """Write a structure in the XYZ format (Angstrom); symbols[i] names species i."""
    lines = [str(mol.nat), mol.label or "tblite-b200 structure"]
    for s, (x, y, z) in zip(mol.id, np.asarray(mol.xyz) / ANGSTROM):
        lines.append(f"{symbols[int(s)]:2s} {x:22.15f} {y:22.15f} {z:22.15f}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
