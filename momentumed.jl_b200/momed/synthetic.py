"""Synthetic Hamiltonians of the benchmark workloads (seeded; no dataset involved).

Mesh a x b: Nk = a b, k_list[:, i] = ((i-1) mod a, (i-1) div a), Gk = (a, b).
  H_one(k, cf, ci) = d(cf, ci) (cos(2 pi kx / a) + cos(2 pi ky / b))
  H_two(a1, a2, a3, a4, cf1, cf2, ci2, ci1) (positions kf1, kf2, ki2, ki1)
      = comp * exp(-|q|^2 / 2) / (|q| + 0.5) * exp(i theta(a1 a2 a3 a4))
      q = k(a3) - k(a1) folded per direction to the nearest image, |q| = 2 pi |q_frac|
      comp = d(cf1,ci1) d(cf2,ci2) + beta [cf1 != cf2] d(cf1,ci2) d(cf2,ci1)
  theta is tabulated over momentum-conserving quadruples in lexicographic order from
  a SplitMix64 stream seeded with `seed` (its first draw is beta), one draw per
  {(a1 a2 a3 a4), (a3 a4 a1 a2)} pair with theta(a3 a4 a1 a2) = -theta(a1 a2 a3 a4)
  and theta = 0 on self-paired quadruples.
The arithmetic is written operation by operation so that every amplitude is
bit-identical to the CPU oracle's C restatement of the same recipe.
"""
from __future__ import annotations

import math

import numpy as np

from .preparation import EDPara

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def u01(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def mesh_klist(a: int, b: int) -> np.ndarray:
    i = np.arange(a * b)
    return np.stack([i % a, i // a]).astype(np.int64)


class MeshHamiltonian:
    """Callables H_one / H_two (index mode) of the recipe on an a x b mesh."""

    def __init__(self, a: int, b: int, seed: int):
        self.a, self.b, self.Nk = a, b, a * b
        Nk = self.Nk
        rng = SplitMix64(seed)
        self.beta = rng.u01()
        theta = np.zeros((Nk, Nk, Nk, Nk))
        xs = [i % a for i in range(Nk)]
        ys = [i // a for i in range(Nk)]
        for a1 in range(Nk):
            for a2 in range(Nk):
                sx, sy = xs[a1] + xs[a2], ys[a1] + ys[a2]
                for a3 in range(Nk):
                    for a4 in range(Nk):
                        if (sx - xs[a3] - xs[a4]) % a or (sy - ys[a3] - ys[a4]) % b:
                            continue
                        if a1 < a3 or (a1 == a3 and a2 < a4):
                            th = 2.0 * math.pi * rng.u01()
                            theta[a1, a2, a3, a4] = th
                            theta[a3, a4, a1, a2] = -th
                        elif a1 == a3 and a2 == a4:
                            theta[a1, a2, a3, a4] = 0.0
        self.theta = theta
        self._xs, self._ys = xs, ys

    def H_one(self, k: int, cf: int, ci: int) -> complex:
        if cf != ci:
            return 0j
        kx, ky = (k - 1) % self.a, (k - 1) // self.a
        return complex(math.cos(2.0 * math.pi * kx / self.a) + math.cos(2.0 * math.pi * ky / self.b), 0.0)

    def H_two(self, a1: int, a2: int, a3: int, a4: int, cf1: int = 1, cf2: int = 1, ci2: int = 1,
              ci1: int = 1) -> complex:
        comp = 0.0
        if cf1 == ci1 and cf2 == ci2:
            comp = comp + 1.0
        if cf1 != cf2 and cf1 == ci2 and cf2 == ci1:
            comp = comp + self.beta
        if comp == 0.0:
            return 0j
        qx = self._xs[a3 - 1] - self._xs[a1 - 1]
        qy = self._ys[a3 - 1] - self._ys[a1 - 1]
        tx = qx / self.a
        ty = qy / self.b
        fx = tx - math.floor(tx + 0.5)
        fy = ty - math.floor(ty + 0.5)
        qn = 2.0 * math.pi * math.sqrt(fx * fx + fy * fy)
        mag = math.exp(-(qn * qn) / 2.0) / (qn + 0.5)
        th = float(self.theta[a1 - 1, a2 - 1, a3 - 1, a4 - 1])
        m = comp * mag
        return complex(m * math.cos(th), m * math.sin(th))


def mesh_para(a: int, b: int, seed: int, Nc_mix: int = 1, Nc_conserve: int = 1, with_one: bool = True,
              with_two: bool = True):
    """EDPara of the recipe plus the MeshHamiltonian it uses."""
    mh = MeshHamiltonian(a, b, seed)
    para = EDPara(k_list=mesh_klist(a, b), Gk=(a, b), Nc_mix=Nc_mix, Nc_conserve=Nc_conserve,
                  H_one=mh.H_one if with_one else None, H_two=mh.H_two if with_two else None,
                  one_momentum_coordinate=False, two_momentum_coordinate=False)
    return para, mh


# Workloads (mesh a x b, electrons per conserved component, nev, seed)
WORKLOADS = {
    "plain_3x5": dict(a=3, b=5, N_each=(5,), nev=10, seed=0, Nc_conserve=1),
    "plain_3x10": dict(a=3, b=10, N_each=(10,), nev=6, seed=1, Nc_conserve=1, krylovdim=64),
    "plain_3x9": dict(a=3, b=9, N_each=(9,), nev=4, seed=2, Nc_conserve=1),
    "batch_3x9": dict(a=3, b=9, N_each=(9,), nev=4, seed=2, Nc_conserve=1, n_u=32, u_range=(0.5, 2.0)),
    "two_comp_4x6": dict(a=4, b=6, N_each=(4, 4), nev=8, seed=3, Nc_conserve=2),
}

# Meshes of the serving stream (Poisson arrivals at 50 req/s, seed 4): mesh -> (electrons, recipe seed)
SERVE_MESHES = {"3x5": (5, 0), "3x9": (9, 2), "3x10": (10, 1), "4x9": (12, 4)}


def serve_requests(n: int, meshes, sector_counts, rate: float = 50.0, seed: int = 4):
    """The serving stream: n requests with Poisson arrivals at `rate` per second.  Each picks a
    mesh uniformly from `meshes`, a uniform sector of it (`sector_counts[mesh]` sectors),
    U0 ~ U(0.5, 2), nev in 1..20 and tolerance 1e-10.  Returns dicts sorted by arrival (s)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        mesh = meshes[int(rng.integers(len(meshes)))]
        out.append(dict(arrival=float(t[i]), mesh=mesh, sector=int(rng.integers(sector_counts[mesh])),
                        u=float(rng.uniform(0.5, 2.0)), nev=int(rng.integers(1, 21)), tol=1e-10))
    return out


def u_grid(n: int = 32, lo: float = 0.5, hi: float = 2.0) -> np.ndarray:
    """Interaction strengths U0 of the sweep, evenly spaced over [lo, hi]."""
    return lo + (hi - lo) * np.arange(n) / (n - 1)
