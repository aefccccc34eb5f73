"""Host mirror of MomentumED's preparation layer for the matrix-free path.

  - ``EDPara`` ........................ MomentumED/src/preparation/init_parameter.jl:62-146
  - ``momentum_residue`` / ``MBS_totalmomentum`` .. init_parameter.jl:148-152, momentum_decomposition.jl:49-77
  - ``ED_momentum_subspaces`` ......... momentum_decomposition.jl:188-273 (device kernel (a))
  - ``group_momentum_pairs`` .......... scat_list.jl:174-200
  - ``ED_scatterlist_onebody/twobody`` . scat_list.jl:78-142, 425-572

The scatter-list builders call the user's H_one / H_two on the host (as the
reference does) with the reference's loop order, filters and arithmetic
(including Complex{Float32} arithmetic when element_type is float32).
"""
from __future__ import annotations

import inspect
from fractions import Fraction

import numpy as np

from .core import HilbertSubspace, MBS64, Scatter, ScatterList, parity_mask, sort_merge_scatlist


class EDPara:
    """Parameters of a momentum-conserving system (init_parameter.jl:62-146).

    ``k_list`` is a dim x Nk integer matrix; orbital index i = k + Nk (c - 1) with
    c = c_mix + Nc_mix (c_conserve - 1).  ``H_one(k, cf, ci)`` and
    ``H_two(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1)`` take momentum indices (1-based)
    or, in coordinate mode, tuples of coordinates (k / Gk when Gk != 0).
    The mode is read from the callables' annotations (a ``tuple`` first parameter
    means coordinates) unless given explicitly.
    """

    def __init__(self, *, k_list, Gk, Nc_mix: int = 1, Nc_conserve: int = 1, H_one=None, H_two=None,
                 one_momentum_coordinate: bool | None = None, two_momentum_coordinate: bool | None = None):
        self.k_list = np.asarray(k_list, np.int64)
        if self.k_list.ndim != 2:
            raise AssertionError("k_list must be a dim x Nk matrix")
        self.Gk = tuple(int(g) for g in Gk)
        self.dim = len(self.Gk)
        if self.k_list.shape[0] != self.dim:
            raise AssertionError("k_list rows must match the length of Gk")
        self.Nk = self.k_list.shape[1]
        self.Nc_mix, self.Nc_conserve = int(Nc_mix), int(Nc_conserve)
        self.Nc = self.Nc_mix * self.Nc_conserve
        if self.Nc <= 0:
            raise AssertionError("Number of components must be positive")
        if self.Nk * self.Nc > 64:
            raise AssertionError("The total orbital number exceeds 64 bits.")
        if any(g < 0 for g in self.Gk):
            raise AssertionError("Gk must all be non-negative integers.")
        self.H_one = H_one if H_one is not None else (lambda *a, **k: 0j)
        self.H_two = H_two if H_two is not None else (lambda *a, **k: 0j)
        self.one_momentum_coordinate = (_detect_coordinate(self.H_one) if one_momentum_coordinate is None
                                        else bool(one_momentum_coordinate))
        self.two_momentum_coordinate = (_detect_coordinate(self.H_two) if two_momentum_coordinate is None
                                        else bool(two_momentum_coordinate))

    @property
    def bits(self) -> int:
        return self.Nk * self.Nc


def _detect_coordinate(fn) -> bool:
    try:
        params = list(inspect.signature(fn).parameters.values())
    except (TypeError, ValueError):
        return False
    if not params:
        return False
    ann = params[0].annotation
    return ann is tuple or getattr(ann, "__origin__", None) is tuple


def momentum_residue(k, Gk):
    return tuple(kd if g == 0 else kd % g for kd, g in zip(k, Gk))


def MBS_totalmomentum(para: EDPara, mbs) -> tuple:
    """Total momentum of a state (or of a tuple of 1-based orbitals, repeats counted)."""
    if isinstance(mbs, tuple):
        orbs = list(mbs)
    else:
        n = mbs.n if isinstance(mbs, MBS64) else int(mbs)
        orbs = []
        while n:
            orbs.append((n & -n).bit_length())
            n &= n - 1
    k = [0] * para.dim
    for i in orbs:
        ik = (i - 1) % para.Nk
        for d in range(para.dim):
            k[d] += int(para.k_list[d, ik])
    return momentum_residue(k, para.Gk)


# ------------------------------------------------------------------------------- sectors
def ED_momentum_subspaces(para: EDPara, N_each_component, *, momentum_restriction: bool = False,
                          momentum_list=None, mask=None, selection_rule=None, handle=None):
    """Per-sector sorted bases and their momenta, enumerated on the GPU (kernel (a)).

    Returns ``(subspaces, subspace_k)`` in the reference's sector order, empty sectors
    dropped.  ``selection_rule`` (a predicate on ``MBS64``) is applied to every state.
    """
    from ._lib import Handle

    if isinstance(N_each_component, int):
        N_each_component = (N_each_component,)
    N_each = [int(v) for v in N_each_component]
    if len(N_each) != para.Nc_conserve:
        raise AssertionError(f"The length of number_list must be equal to the number of conserved components "
                             f"{para.Nc_conserve}")
    h = handle if handle is not None else Handle(0)
    moms = None
    if momentum_restriction:
        moms = [tuple(m) for m in (momentum_list or [])]
        if not moms:
            return [], []
    sectors = h.enumerate_basis(para.k_list, para.Gk, para.Nc_mix, para.Nc_conserve, N_each, mask=mask,
                                momentum_list=moms)
    subspaces, ks = [], []
    bits = para.bits
    for k, basis in sectors:
        if selection_rule is not None:
            keep = np.fromiter((bool(selection_rule(MBS64(bits, int(s)))) for s in basis), bool, len(basis))
            basis = basis[keep]
            if len(basis) == 0:
                continue
        subspaces.append(HilbertSubspace(basis, bits))
        ks.append(k)
    return subspaces, ks


# ------------------------------------------------------------------------------- scatter lists
def _coords(para: EDPara, shifts, rational: bool):
    """k coordinates (k / Gk when Gk != 0) and per-conserved-component shifts (scat_list.jl:5-28)."""
    kl = [[(Fraction(int(para.k_list[d, i])) if rational else float(para.k_list[d, i])) for i in range(para.Nk)]
          for d in range(para.dim)]
    sh = [[(Fraction(shifts[d][c]) if rational else float(shifts[d][c])) for c in range(para.Nc_conserve)]
          for d in range(para.dim)]
    for d in range(para.dim):
        g = para.Gk[d]
        if g != 0:
            kl[d] = [v / g for v in kl[d]]
            sh[d] = [v / g for v in sh[d]]
    return kl, sh


def _shift_decipher(kshift, Ncc: int, dim: int):
    """scat_list.jl:29-50: shifts[d][c]."""
    if kshift is None:
        return [[0] * Ncc for _ in range(dim)]
    if isinstance(kshift, tuple):
        return [[kshift[d]] * Ncc for d in range(dim)]
    if isinstance(kshift, list):
        if len(kshift) != Ncc:
            raise AssertionError("length of kshift isn't equal to para.Nc_conserve.")
        return [[kshift[c][d] for c in range(Ncc)] for d in range(dim)]
    arr = np.asarray(kshift)
    if arr.shape != (dim, Ncc):
        raise AssertionError("size of kshift isn't equal to para.Nc_conserve.")
    return [[arr[d, c].item() for c in range(Ncc)] for d in range(dim)]


def _is_rational(shifts) -> bool:
    return all(isinstance(v, (int, np.integer, Fraction)) for row in shifts for v in row)


def _to_et(v, element_type):
    v = complex(v)
    return element_type(v)


def ED_scatterlist_onebody(para: EDPara, *, element_type=np.float64, kshift=None, H_one: dict | None = None
                           ) -> ScatterList:
    """One-body terms at equal k with i_in >= i_out, upper-Hermitian, sorted and merged (scat_list.jl:78-142)."""
    ct = np.complex64 if element_type in (np.float32, np.complex64) else np.complex128
    kw = H_one or {}
    Nk, Ncc, Ncm, bits = para.Nk, para.Nc_conserve, para.Nc_mix, para.bits
    terms = []
    if para.one_momentum_coordinate:
        shifts = _shift_decipher(kshift, Ncc, para.dim)
        kl, sh = _coords(para, shifts, _is_rational(shifts))
    for cc in range(1, Ncc + 1):
        for cmi in range(1, Ncm + 1):
            for cmf in range(1, Ncm + 1):
                cf = cmf + (cc - 1) * Ncm
                ci = cmi + (cc - 1) * Ncm
                for k in range(1, Nk + 1):
                    i_out = k + Nk * (cf - 1)
                    i_in = k + Nk * (ci - 1)
                    if i_in >= i_out:
                        if para.one_momentum_coordinate:
                            kc = tuple(kl[d][k - 1] + sh[d][cc - 1] for d in range(para.dim))
                            V = _to_et(para.H_one(kc, cf, ci, **kw), ct)
                        else:
                            V = _to_et(para.H_one(k, cf, ci, **kw), ct)
                        if V != 0:
                            terms.append(Scatter(V, i_out, i_in, bits=bits, upper_hermitian=True, element_type=ct))
    if not terms:
        return ScatterList(np.zeros(0, ct), [], [], [], bits, ct)
    return sort_merge_scatlist(ScatterList.from_terms(terms, bits, ct))


def group_momentum_pairs(para: EDPara) -> dict:
    """Pairs (i, j), i >= j, of momentum indices keyed by their total momentum (scat_list.jl:174-200)."""
    groups: dict = {}
    for i in range(1, para.Nk + 1):
        for j in range(1, i + 1):
            K = MBS_totalmomentum(para, (i, j))
            groups.setdefault(K, []).append((i, j))
    return groups


def ED_scatterlist_twobody(para: EDPara, *, element_type=np.float64, kshift=None, H_two: dict | None = None
                           ) -> ScatterList:
    """Antisymmetrised, Nk-normalised upper-triangle two-body terms (scat_list.jl:425-572)."""
    ct = np.complex64 if element_type in (np.float32, np.complex64) else np.complex128
    ft = np.float32 if ct is np.complex64 else np.float64
    kw = H_two or {}
    Nk, Nc, Ncm, bits = para.Nk, para.Nc, para.Nc_mix, para.bits
    sys_size = Nk if all(g != 0 for g in para.Gk) else 1
    groups = group_momentum_pairs(para)
    coord = para.two_momentum_coordinate
    if coord:
        shifts = _shift_decipher(kshift, para.Nc_conserve, para.dim)
        kl, sh = _coords(para, shifts, _is_rational(shifts))
    H = para.H_two
    terms = []
    for _, pairs in groups.items():
        for (ki1, ki2) in pairs:
            for (kf1, kf2) in pairs:
                for ci1 in range(1, Nc + 1):
                    for ci2 in range(1, Nc + 1):
                        for cf1 in range(1, Nc + 1):
                            for cf2 in range(1, Nc + 1):
                                f1 = kf1 + Nk * (cf1 - 1)
                                f2 = kf2 + Nk * (cf2 - 1)
                                i1 = ki1 + Nk * (ci1 - 1)
                                i2 = ki2 + Nk * (ci2 - 1)
                                if i1 == i2 or f1 == f2:
                                    continue
                                if ki1 == ki2 and i1 < i2:
                                    continue
                                if kf1 == kf2 and f1 < f2:
                                    continue
                                if not ((min(i1, i2), max(i1, i2)) >= (min(f1, f2), max(f1, f2))):
                                    continue
                                if coord:
                                    ccs = [(c - 1) // Ncm + 1 for c in (cf1, cf2, ci2, ci1)]
                                    kc = [tuple(kl[d][kq - 1] + sh[d][cq - 1] for d in range(para.dim))
                                          for kq, cq in zip((kf1, kf2, ki2, ki1), ccs)]
                                    d_ = H(kc[0], kc[1], kc[2], kc[3], cf1, cf2, ci2, ci1, **kw)
                                    e_ = H(kc[0], kc[1], kc[3], kc[2], cf1, cf2, ci1, ci2, **kw)
                                else:
                                    d_ = H(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1, **kw)
                                    e_ = H(kf1, kf2, ki1, ki2, cf1, cf2, ci1, ci2, **kw)
                                d_, e_ = complex(d_), complex(e_)
                                if ct is np.complex64:
                                    re = (ft(d_.real) - ft(e_.real)) / ft(sys_size)
                                    im = (ft(d_.imag) - ft(e_.imag)) / ft(sys_size)
                                    amp = ct(complex(float(re), float(im)))
                                else:
                                    amp = complex((d_.real - e_.real) / sys_size, (d_.imag - e_.imag) / sys_size)
                                if amp != 0:
                                    terms.append(Scatter(amp, f1, f2, i2, i1, bits=bits, upper_hermitian=True,
                                                         element_type=ct))
    if not terms:
        return ScatterList(np.zeros(0, ct), [], [], [], bits, ct)
    return sort_merge_scatlist(ScatterList.from_terms(terms, bits, ct))


# the names the README and older releases use (scat_list.jl:573-574)
ED_sortedScatterList_onebody = ED_scatterlist_onebody
ED_sortedScatterList_twobody = ED_scatterlist_twobody


# ------------------------------------------------------------------------------- device recipes
def twobody_recipe_table(para: EDPara) -> dict:
    """Structure of the coordinate-mode two-body list without evaluating H_two: the loop, filters
    and normal ordering of ED_scatterlist_twobody (scat_list.jl:442-497), recording for every raw
    term its momenta and components and what the Scatter constructor does to its amplitude (sign;
    as is, conjugated on the upper swap, or reduced to the real part on the diagonal), grouped by
    upper term (out, in) in the order sort_merge_scatlist sums them.

    Returns dict(out, in_, pm: the upper terms (sorted by in, out); raw: int32 [nraw][9] = kf1, kf2,
    ki2, ki1 (0-based), cf1, cf2, ci2, ci1, flags (bit 0 negate, bits 1-2: 0 as is, 1 conjugate,
    2 real part); upper_start: int64 [nupper + 1]).  Every structurally allowed term is kept, also
    those whose amplitude vanishes at some kshift."""
    Nk, Nc, Ncm, bits = para.Nk, para.Nc, para.Nc_mix, para.bits
    probe = complex(1.0, 2.0)
    recs, keys = [], []
    for _, pairs in group_momentum_pairs(para).items():
        for (ki1, ki2) in pairs:
            for (kf1, kf2) in pairs:
                for ci1 in range(1, Nc + 1):
                    for ci2 in range(1, Nc + 1):
                        for cf1 in range(1, Nc + 1):
                            for cf2 in range(1, Nc + 1):
                                f1, f2 = kf1 + Nk * (cf1 - 1), kf2 + Nk * (cf2 - 1)
                                i1, i2 = ki1 + Nk * (ci1 - 1), ki2 + Nk * (ci2 - 1)
                                if i1 == i2 or f1 == f2:
                                    continue
                                if ki1 == ki2 and i1 < i2:
                                    continue
                                if kf1 == kf2 and f1 < f2:
                                    continue
                                if not ((min(i1, i2), max(i1, i2)) >= (min(f1, f2), max(f1, f2))):
                                    continue
                                s = Scatter(probe, f1, f2, i2, i1, bits=bits, upper_hermitian=True)
                                a = complex(s.Amp)
                                if a == probe:
                                    fl = 0
                                elif a == -probe:
                                    fl = 1
                                elif a == probe.conjugate():
                                    fl = 2
                                elif a == -probe.conjugate():
                                    fl = 3
                                elif a == 1:
                                    fl = 4
                                elif a == -1:
                                    fl = 5
                                else:
                                    raise AssertionError(f"unexpected normal ordering {a}")
                                recs.append((kf1 - 1, kf2 - 1, ki2 - 1, ki1 - 1, cf1, cf2, ci2, ci1, fl))
                                keys.append((s.in_, s.out))
    if not recs:
        z = np.zeros(0, np.uint64)
        return dict(out=z, in_=z.copy(), pm=z.copy(), raw=np.zeros((0, 9), np.int32),
                    upper_start=np.zeros(1, np.int64))
    order = sorted(range(len(recs)), key=lambda r: keys[r])        # stable: merge order within a key
    raw = np.array([recs[r] for r in order], np.int32)
    sk = [keys[r] for r in order]
    starts = [0] + [i for i in range(1, len(sk)) if sk[i] != sk[i - 1]] + [len(sk)]
    uin = np.array([sk[i][0] for i in starts[:-1]], np.uint64)
    uout = np.array([sk[i][1] for i in starts[:-1]], np.uint64)
    pm = np.array([parity_mask(int(o)) ^ parity_mask(int(i)) for o, i in zip(uout, uin)], np.uint64)
    return dict(out=uout, in_=uin, pm=pm, raw=raw, upper_start=np.array(starts, np.int64))
