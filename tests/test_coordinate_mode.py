"""Coordinate-mode scatter lists: the reference's own test workload (CPU, no GPU needed).

MomentumED/test/example1_FQH_Laughlin.jl defines H_two on momentum COORDINATES, so
ED_scatterlist_twobody takes its coordinate branch (scat_list.jl:442-497): coordinates are
k / Gk plus the conserved component's kshift / Gk, exact Rationals for integer or rational
shifts (the default, kshift = nothing) and Float64 otherwise (scat_list.jl:5-50).  These tests
hold the host builders bit-exact to the oracle's C restatement on that workload (default,
rational and float kshift), on a two-component system with per-component shifts and in Float32,
and check the physics of the restated workload (three-fold Laughlin ground states).
"""
from fractions import Fraction

import numpy as np
import pytest

import laughlin as L
import momed
import oracle as O
from test_host_mirror import same_bits


def laughlin_para():
    return momed.EDPara(k_list=L.K_LIST, Gk=L.GK, H_two=L.V_int, two_momentum_coordinate=True)


@pytest.mark.parametrize("kshift", [None, (Fraction(1, 3), Fraction(1, 4)), (1, 0), (0.25, 0.5), (0.1, 0.0)],
                         ids=["default", "rational", "integer", "float", "float-small"])
def test_laughlin_twobody_bit_exact(kshift):
    para = laughlin_para()
    got = momed.ED_scatterlist_twobody(para, kshift=kshift)
    ref = O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int, kshift=kshift)
    assert len(ref) > 100
    assert same_bits(got, ref)


def test_laughlin_twobody_float32_bit_exact():
    para = laughlin_para()
    got = momed.ED_scatterlist_twobody(para, element_type=np.float32, kshift=(Fraction(1, 2), 0))
    ref = O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int, kshift=(Fraction(1, 2), 0), prec=32)
    assert same_bits(got, ref)


def test_rational_coordinates_reach_the_callable_exactly():
    seen = []

    def H2(kf1, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1):
        seen.append((kf1, ki1))
        return 0j

    O.scatterlist_twobody_coord(L.K_LIST, L.GK, H2, kshift=(Fraction(1, 3), 0))
    assert seen and all(isinstance(v, Fraction) for k, _ in seen for v in k)
    # k = (1, 2) of the 3 x 4 mesh shifted by (1/3, 0): (1/3 + 1/9, 2/4)
    assert (Fraction(4, 9), Fraction(1, 2)) in {k for k, _ in seen}


def two_component_coord():
    """Two conserved components on a 3 x 3 mesh, coordinate-mode one- and two-body callables."""
    def H1(k, cf, ci):
        return complex(np.cos(2 * np.pi * float(k[0])) + 0.5 * np.cos(2 * np.pi * float(k[1])), 0.0)

    def H2(kf1, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1):
        if not (cf1 == ci1 and cf2 == ci2):
            return 0j
        q = [float(ki1[d]) - float(kf1[d]) for d in range(2)]
        v = np.exp(-(q[0] ** 2 + q[1] ** 2)) * (1.0 + 0.25 * (cf1 + cf2))
        return complex(v * np.cos(q[0] - 2 * q[1]), v * np.sin(q[0] + q[1]))

    kl = O.mesh_klist(3, 3)
    para = momed.EDPara(k_list=kl, Gk=(3, 3), Nc_conserve=2, H_one=H1, H_two=H2,
                        one_momentum_coordinate=True, two_momentum_coordinate=True)
    return kl, para, H1, H2


@pytest.mark.parametrize("kshift", [None, [(Fraction(1, 2), 0), (0, Fraction(1, 3))], [(0.5, 0.0), (0.0, 0.25)],
                                    np.array([[0.5, 0.0], [0.0, 0.25]])],
                         ids=["default", "rational-per-component", "float-per-component", "matrix"])
@pytest.mark.parametrize("prec", [64, 32])
def test_two_component_coordinate_builders_bit_exact(kshift, prec):
    kl, para, H1, H2 = two_component_coord()
    et = np.float32 if prec == 32 else np.float64
    ks = kshift.tolist() if isinstance(kshift, np.ndarray) else kshift
    o1 = O.scatterlist_onebody_coord(kl, (3, 3), H1, Nc_conserve=2, kshift=kshift, prec=prec)
    o2 = O.scatterlist_twobody_coord(kl, (3, 3), H2, Nc_conserve=2, kshift=kshift, prec=prec)
    assert same_bits(momed.ED_scatterlist_onebody(para, element_type=et, kshift=kshift), o1)
    assert same_bits(momed.ED_scatterlist_twobody(para, element_type=et, kshift=kshift), o2)
    assert len(o2) > 0 and ks is not None or kshift is None


def test_kshift_length_checked():
    kl, para, _, _ = two_component_coord()
    with pytest.raises(AssertionError):
        momed.ED_scatterlist_twobody(para, kshift=[(0.5, 0.0)])
    with pytest.raises(AssertionError):
        O.scatterlist_twobody_coord(kl, (3, 3), lambda *a: 0j, Nc_conserve=2, kshift=[(0.5, 0.0)])


def test_laughlin_three_fold_ground_state():
    """The restated workload is the Laughlin state at filling 1/3: over all 12 sectors the three
    lowest levels lie in the three sectors of ky = 2, split by < 1e-7, below a gap of > 0.04."""
    full = O.hermitian_complete(O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int))
    bases, ks = O.momentum_subspaces(L.K_LIST, L.GK, (L.NE,))
    assert len(bases) == 12 and sum(len(b) for b in bases) == 495
    levels = []
    for b, k in zip(bases, ks):
        w = np.linalg.eigvalsh(O.dense_hamiltonian(b, full))
        levels += [(e, k) for e in w]
    levels.sort()
    low = levels[:3]
    assert sorted(k for _, k in low) == [(0, 2), (1, 2), (2, 2)]
    assert low[2][0] - low[0][0] < 1e-7
    assert levels[3][0] - low[2][0] > 0.04


# ---------------------------------------------------------------------------- device recipe tables
def replay_table(para, t, H, kshift):
    """The upper amplitudes a recipe table describes, evaluated on the host in its order."""
    from momed.preparation import _coords, _shift_decipher
    sh = _shift_decipher(kshift, para.Nc_conserve, para.dim)
    kl, shv = _coords(para, sh, False)
    sys_size = para.Nk if all(g != 0 for g in para.Gk) else 1
    out = []
    for u in range(len(t["out"])):
        acc = 0j
        for r in t["raw"][t["upper_start"][u]:t["upper_start"][u + 1]]:
            ks, cs, fl = r[:4], r[4:8], int(r[8])
            cc = [(int(c) - 1) // para.Nc_mix for c in cs]
            kc = [tuple(kl[d][int(k)] + shv[d][c] for d in range(para.dim)) for k, c in zip(ks, cc)]
            d_ = complex(H(kc[0], kc[1], kc[2], kc[3], *[int(c) for c in cs]))
            e_ = complex(H(kc[0], kc[1], kc[3], kc[2], int(cs[0]), int(cs[1]), int(cs[3]), int(cs[2])))
            v = complex((d_.real - e_.real) / sys_size, (d_.imag - e_.imag) / sys_size)
            if fl & 1:
                v = -v
            mode = (fl >> 1) & 3
            if mode == 1:
                v = v.conjugate()
            elif mode == 2:
                v = complex(v.real, 0.0)
            acc = acc + v
        out.append(acc)
    return np.array(out)


@pytest.mark.parametrize("kshift", [(0.0, 0.0), (0.25, 0.5), (0.1, 0.7)])
def test_recipe_table_replays_the_builder(kshift):
    """The structure table that the device recipe evaluates, replayed on the host with the same
    H_two and float kshift, gives the builder's merged upper list bit for bit (terms the builder
    dropped as exactly zero replay to zero)."""
    rec = momed.LandauCoulomb()
    para = momed.EDPara(k_list=L.K_LIST, Gk=L.GK, H_two=rec.H_two, two_momentum_coordinate=True)
    from momed.preparation import twobody_recipe_table
    t = twobody_recipe_table(para)
    got = replay_table(para, t, rec.H_two, kshift)
    ref = momed.ED_scatterlist_twobody(para, kshift=kshift)
    keys = {(int(i), int(o)): a for i, o, a in zip(ref.in_, ref.out, ref.amp)}
    assert len(t["out"]) >= len(ref)
    for i, o, a in zip(t["in_"], t["out"], got):
        want = keys.get((int(i), int(o)), 0j)
        assert a == want or (want == 0 and a == 0), (i, o, a, want)


def test_recipe_interaction_is_the_reference_test_formula():
    """LandauCoulomb.H_two (the host form of the device recipe) against the port of the reference
    test's V_int, on random float coordinates (1e-14 relative; cispi there, cos/sin of pi x here)."""
    rec = momed.LandauCoulomb()
    rng = np.random.default_rng(3)
    for _ in range(200):
        ks = [tuple(rng.uniform(-1.5, 1.5, 2)) for _ in range(4)]
        a = rec.H_two(*ks)
        b = L.V_int(*ks)
        assert abs(a - b) <= 1e-14 * max(1.0, abs(b))
