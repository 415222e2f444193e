"""Seeded synthetic molecules for the benchmark workloads.

No public dataset is involved: every molecule is generated here with numpy's PCG64
(``numpy.random.default_rng(seed)``), so the library, the CPU oracle and the CPU baseline
read identical coordinates.  Two generators, both in Angstrom:

* water clusters: monomers with O-H 0.9572 A and H-O-H 104.52 deg, each rotated about its
  oxygen by a uniformly random rotation (a unit quaternion from four standard normals),
  placed on a cubic grid of 3.0 A spacing filled x-fastest (side = the smallest s with
  s^3 >= k, the fill order of the reference's tools/make_water_cluster.py:67-77), each
  centre jittered by U(-0.3, 0.3) A per coordinate;
* linear alkanes CnH2n+2: all-trans zig-zag carbon chain (C-C 1.54 A, C-C-C 109.47 deg),
  C-H 1.09 A along tetrahedral directions, then N(0, 0.05 A) jitter on every coordinate.
  A radical drops one terminal hydrogen (multiplicity 2).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

R_OH = 0.9572
THETA_HOH = math.radians(104.52)
R_CC = 1.54
R_CH = 1.09
TET = math.acos(-1.0 / 3.0)  # 109.47 deg


@dataclass
class Mol:
    numbers: np.ndarray          # int32 [natoms]
    xyz: np.ndarray              # float64 [natoms, 3], Angstrom
    charge: float = 0.0
    multiplicity: int = 1
    kind: str = ""
    tags: dict = field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return int(self.numbers.shape[0])

    def nao(self) -> int:
        return int(np.sum(np.where(self.numbers == 1, 1, 4)))


def _quat_rotation(q: np.ndarray) -> np.ndarray:
    q = q / np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


_MONOMER = np.array([
    [0.0, 0.0, 0.0],
    [R_OH, 0.0, 0.0],
    [R_OH * math.cos(THETA_HOH), R_OH * math.sin(THETA_HOH), 0.0],
])


def grid_side(k: int) -> int:
    s = 1
    while s ** 3 < k:
        s += 1
    return s


def water_cluster(k: int, rng: np.random.Generator, spacing: float = 3.0, jitter: float = 0.3,
                  grid: tuple[int, int, int] | None = None) -> Mol:
    if grid is None:
        s = grid_side(k)
        grid = (s, s, s)
    gx, gy, _ = grid
    z = []
    xyz = []
    for i in range(k):
        a, b, c = i % gx, (i // gx) % gy, i // (gx * gy)
        rot = _quat_rotation(rng.standard_normal(4))
        centre = np.array([a, b, c], dtype=float) * spacing + rng.uniform(-jitter, jitter, 3)
        xyz.append(_MONOMER @ rot.T + centre)
        z += [8, 1, 1]
    return Mol(np.array(z, dtype=np.int32), np.concatenate(xyz), kind="water", tags={"k": k})


def _unit(v):
    return v / np.linalg.norm(v)


def alkane(n: int, rng: np.random.Generator, jitter: float = 0.05, radical: bool = False) -> Mol:
    half = TET / 2.0
    dx = R_CC * math.sin(half)
    dy = R_CC * math.cos(half)
    carbons = np.array([[i * dx, (i % 2) * dy, 0.0] for i in range(n)])
    hyd = []
    zhat = np.array([0.0, 0.0, 1.0])
    if n == 1:
        for d in ([1, 1, 1], [-1, -1, 1], [-1, 1, -1], [1, -1, -1]):
            hyd.append(carbons[0] + R_CH * _unit(np.array(d, dtype=float)))
    else:
        for i in range(n):
            c = carbons[i]
            bonds = []
            if i > 0:
                bonds.append(_unit(carbons[i - 1] - c))
            if i < n - 1:
                bonds.append(_unit(carbons[i + 1] - c))
            if len(bonds) == 2:
                m = -_unit(bonds[0] + bonds[1])
                for sgn in (1.0, -1.0):
                    hyd.append(c + R_CH * (m * math.cos(half) + sgn * zhat * math.sin(half)))
            else:
                b = bonds[0]
                # The in-plane terminal hydrogen is anti to the next carbon along the chain:
                # opposite side of the C(i)-C(j) line from C(k).
                j = i + 1 if i == 0 else i - 1
                k = j + (j - i)
                if 0 <= k < n:
                    off = carbons[k] - carbons[j]
                    inplane = -_unit(off - np.dot(off, b) * b)
                else:
                    inplane = _unit(np.cross(zhat, b))
                for phi in (0.0, 2 * math.pi / 3, 4 * math.pi / 3):
                    perp = inplane * math.cos(phi) + zhat * math.sin(phi)
                    d = b * math.cos(TET) + perp * math.sin(TET)
                    hyd.append(c + R_CH * _unit(d))
    if radical:
        hyd = hyd[:-1] if n == 1 else hyd[:2] + hyd[3:]  # drop one terminal H
    xyz = np.concatenate([carbons, np.array(hyd)])
    xyz = xyz + rng.normal(0.0, jitter, xyz.shape)
    z = np.array([6] * n + [1] * len(hyd), dtype=np.int32)
    return Mol(z, xyz, multiplicity=2 if radical else 1, kind="alkane_radical" if radical else "alkane",
               tags={"n": n})


# ---------------------------------------------------------------------------------------
# The benchmark workloads
# ---------------------------------------------------------------------------------------
def water32_cluster() -> Mol:
    """32 H2O on a 4x4x2 grid, seed 0 (96 atoms, 192 AOs)."""
    return water_cluster(32, np.random.default_rng(0), grid=(4, 4, 2))


def alkane_water_batch(n_alkanes: int = 2048, n_waters: int = 2048) -> list[Mol]:
    """4096 molecules of uneven size, seed 1: alkanes n ~ U{1..40}, water clusters k ~ U{1..64}."""
    rng = np.random.default_rng(1)
    ns = rng.integers(1, 41, n_alkanes)
    ks = rng.integers(1, 65, n_waters)
    mols = [alkane(int(n), rng) for n in ns]
    mols += [water_cluster(int(k), rng) for k in ks]
    return mols


def alkane_water_radical_batch(n_radicals: int = 512) -> list[Mol]:
    """alkane_water_batch plus 512 alkyl radicals (one terminal H removed, doublets) from the same stream."""
    rng = np.random.default_rng(1)
    ns = rng.integers(1, 41, 2048)
    ks = rng.integers(1, 65, 2048)
    mols = [alkane(int(n), rng) for n in ns]
    mols += [water_cluster(int(k), rng) for k in ks]
    nr = rng.integers(1, 41, n_radicals)
    mols += [alkane(int(n), rng, radical=True) for n in nr]
    return mols


def water1024_cluster() -> Mol:
    """1024 H2O on a jittered 16x8x8 grid, seed 3 (3072 atoms, 6144 AOs)."""
    return water_cluster(1024, np.random.default_rng(3), grid=(16, 8, 8))


@dataclass
class Request:
    arrival_s: float
    mol: Mol


def serving_stream(n_requests: int = 100_000, rate: float = 2000.0, seed: int = 2) -> list[Request]:
    """Open-loop Poisson stream: sizes log-uniform on [3, 600] atoms, RHF:UHF = 9:1."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n_requests)
    t = np.cumsum(gaps)
    out = []
    for i in range(n_requests):
        natoms = math.exp(rng.uniform(math.log(3.0), math.log(600.0)))
        uhf = rng.uniform() < 0.1
        if uhf:
            m = alkane(max(1, round((natoms - 1) / 3)), rng, radical=True)
        elif rng.uniform() < 0.5:
            m = alkane(max(1, round((natoms - 2) / 3)), rng)
        else:
            m = water_cluster(max(1, round(natoms / 3)), rng)
        out.append(Request(float(t[i]), m))
    return out


def min_contact(m: Mol) -> float:
    """Smallest interatomic distance (Angstrom)."""
    d = m.xyz[:, None, :] - m.xyz[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    r[np.diag_indices_from(r)] = np.inf
    return float(r.min())
