"""Two-body interactions whose amplitudes the device regenerates for twisted-boundary sweeps.

The reference rebuilds the whole two-body list on the host for every kshift of a sweep
(ED_scatterlist_twobody with momentum coordinates, MomentumED/src/preparation/scat_list.jl:
442-497 and 5-50).  Here the list's structure is described to the library once
(momed_set_twobody_recipe) and each sweep point is one momed_set_kshift call: the device
evaluates the interaction for every raw term and writes the Hermitian-completed amplitudes into
the operator in place.

LandauCoulomb is the interaction of the reference's own test (MomentumED/test/
example1_FQH_Laughlin.jl:20-89): the screened Coulomb interaction projected to the lowest Landau
level, with the magnetic-translation phases, on momentum coordinates.  Its H_two is the host
form of the same formula (usable with ED_scatterlist_twobody); the device evaluates it in FP64
with CUDA's sincospi / tanh / exp, agreeing with the host to ~1e-15 relative.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .core import MBOperator, ScatterList, hermitian_complete
from .preparation import EDPara, _shift_decipher, twobody_recipe_table


class LandauCoulomb:
    """V(q) = W0 / |q l| tanh(|q l| D) exp(-|q l|^2 / 2) (W0 D at q = 0) in the lowest Landau
    level, summed over reciprocal vectors g with |g1|, |g2|, |g1 - g2| <= nshell, with the
    magnetic-translation phase and the parity signs of the shifted reciprocal vectors; the
    metric has angle `angle` between the reciprocal vectors and length scale `mag_length`."""

    kind = _lib.RECIPE_LANDAU_COULOMB

    def __init__(self, mag_length: float = math.sqrt(2.0 * math.pi / math.sqrt(0.75)), screening: float = 5.0,
                 strength: float = 1.0, angle: float = 2.0 * math.pi / 3.0, nshell: int = 2):
        self.mag_length, self.screening, self.strength = float(mag_length), float(screening), float(strength)
        self.angle, self.nshell = float(angle), int(nshell)

    @property
    def params(self) -> np.ndarray:
        return np.array([self.mag_length, self.screening, self.strength, self.angle, self.nshell], np.float64)

    def vff(self, q1: float, q2: float) -> float:
        ql = math.sqrt(q1 * q1 + q2 * q2 + 2.0 * math.cos(self.angle) * q1 * q2) * self.mag_length
        if ql == 0.0:
            return self.strength * self.screening
        return self.strength / ql * math.tanh(ql * self.screening) * math.exp(-0.5 * (ql * ql))

    def H_two(self, kf1: tuple, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1) -> complex:
        def rn(v):
            return int(round(v))

        q = [(ki1[i] - kf1[i]) - rn(ki1[i] - kf1[i]) for i in range(2)]
        gs1 = [rn(ki1[i] - kf1[i] - q[i]) for i in range(2)]
        gs2 = [rn(kf2[i] - ki2[i] - q[i]) for i in range(2)]
        vr = vi = 0.0
        ns = self.nshell
        for g1 in range(-ns, ns + 1):
            for g2 in range(-ns, ns + 1):
                if abs(g1 - g2) > ns:
                    continue
                qq1, qq2 = q[0] + g1, q[1] + g2
                pa = 0.5 * (ki1[0] * kf1[1] - ki1[1] * kf1[0])
                pa += 0.5 * ((ki1[0] + kf1[0]) * qq2 - (ki1[1] + kf1[1]) * qq1)
                pa += 0.5 * (ki2[0] * kf2[1] - ki2[1] * kf2[0])
                pa += 0.5 * ((ki2[0] + kf2[0]) * (-qq2) - (ki2[1] + kf2[1]) * (-qq1))
                x = 2.0 * pa
                c, s = math.cos(math.pi * x), math.sin(math.pi * x)
                sg = (1 if (g1 + gs1[0]) % 2 == 0 and (g2 + gs1[1]) % 2 == 0 else -1) * \
                     (1 if (g1 + gs2[0]) % 2 == 0 and (g2 + gs2[1]) % 2 == 0 else -1)
                v = self.vff(float(qq1), float(qq2))
                vr += (sg * c) * v
                vi += (sg * s) * v
        return complex(vr, vi)


class KShiftOperator:
    """The two-body operator of `recipe` on para's mesh (plus an optional static upper list, e.g.
    one-body terms) set on `handle` as its working operator, with its two-body amplitudes
    regenerated on the device by set_kshift.  kshift takes the forms of ED_scatterlist_twobody's
    keyword: a tuple (every conserved component), a list of Nc_conserve tuples or a dim x
    Nc_conserve array (scat_list.jl:29-50)."""

    def __init__(self, para: EDPara, recipe: LandauCoulomb, handle: _lib.Handle, static: ScatterList | None = None,
                 kshift=None):
        if para.dim != 2:
            raise AssertionError("the Landau-level recipe needs a 2D mesh")
        self.para, self.recipe, self.h = para, recipe, handle
        t = twobody_recipe_table(para)
        bits = para.bits
        upper = ScatterList(np.zeros(len(t["out"]), np.complex128), t["out"], t["in_"], t["pm"], bits, np.complex128)
        parts = [upper] if static is None else [upper, static]
        self.op = MBOperator(*parts, upper_hermitian=True)
        full = hermitian_complete(self.op)
        index = {(int(i), int(o)): u for u, (i, o) in enumerate(zip(t["in_"], t["out"]))}
        eu = np.full(len(full), -1, np.int64)
        ep = np.zeros(len(full), np.int32)
        for e, (i, o) in enumerate(zip(full.in_, full.out)):
            u = index.get((int(i), int(o)))
            if u is not None:
                eu[e] = u
            else:
                u = index.get((int(o), int(i)))
                if u is not None:
                    eu[e], ep[e] = u, 1
        self.full = full
        self.n_upper = len(t["out"])
        handle.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
        handle.set_twobody_recipe(para, recipe.kind, recipe.params, t["raw"], t["upper_start"], eu, ep)
        self.set_kshift(kshift)

    def set_kshift(self, kshift=None):
        sh = _shift_decipher(kshift, self.para.Nc_conserve, self.para.dim)     # sh[d][c]
        arr = np.array([[float(sh[d][c]) for d in range(self.para.dim)] for c in range(self.para.Nc_conserve)])
        self.h.set_kshift(arr.reshape(-1))
        self.kshift = kshift


def kshift_sweep(subspace, para: EDPara, recipe: LandauCoulomb, kshifts, N: int, *, handle=None, static=None,
                 krylovdim: int = 30, tol: float = 1e-12, want_vectors: bool = False):
    """Lowest N eigenpairs of the recipe's Hamiltonian in `subspace` at every kshift of `kshifts`
    (the twisted-boundary loop of a Wilson-loop / Chern-number calculation): one device
    regeneration of the amplitudes and one FP64 device solve per point.  Returns a list of
    (energies, vectors or None, residuals) per point."""
    h = handle if handle is not None else _lib.Handle(0)
    try:
        h.set_basis(subspace.list)
        op = KShiftOperator(para, recipe, h, static=static)
        out = []
        for ks in kshifts:
            op.set_kshift(ks)
            vals, vecs, res, _ = h.eigsolve(N, krylovdim=krylovdim, tol=tol, want_vectors=want_vectors)
            out.append((vals, vecs, res))
        return out
    finally:
        if handle is None:
            h.close()
