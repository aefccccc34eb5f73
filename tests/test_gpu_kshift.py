"""Twisted-boundary sweeps with the two-body amplitudes regenerated on the device.

The reference's own test workload (Laughlin state, 3 x 4 torus, Ne = 4; MomentumED/test/
example1_FQH_Laughlin.jl) with the flux-insertion twist kshift that its notebooks sweep for
Wilson loops: the reference rebuilds ED_scatterlist_twobody on the host for every kshift
(scat_list.jl:442-497); here the list's structure is set once and each point regenerates the
amplitudes on the device (momed_set_kshift).

Bars: the device operator's map equals the oracle map of the host-built list (the reference
test's V_int, float kshift) to 1e-12 relative; swept eigenvalues equal those of a host-built
operator solved on the device to 1e-10 relative.
"""
import numpy as np
import pytest

import laughlin as L
import momed
import oracle as O

pytestmark = pytest.mark.gpu

KSHIFTS = [(0.0, 0.0), (0.25, 0.5), (0.5, 0.0), (1.0 / 3.0, 2.0 / 3.0), (0.9, 0.15)]


@pytest.fixture(scope="module")
def system():
    rec = momed.LandauCoulomb()
    para = momed.EDPara(k_list=L.K_LIST, Gk=L.GK, H_two=rec.H_two, two_momentum_coordinate=True)
    subs, ks = momed.ED_momentum_subspaces(para, (L.NE,))
    return rec, para, subs, ks


def host_list(kshift):
    return O.hermitian_complete(O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int, kshift=kshift))


def test_device_amplitudes_match_host_builder(system):
    rec, para, subs, _ = system
    h = momed.Handle(0)
    try:
        for si in (0, 6):
            basis = subs[si].list
            h.set_basis(basis)
            op = momed.KShiftOperator(para, rec, h)
            rng = np.random.default_rng(si)
            x = rng.standard_normal(len(basis)) + 1j * rng.standard_normal(len(basis))
            for ks in KSHIFTS:
                op.set_kshift(ks)
                y = h.matvec(x)
                ref = O.matvec(basis, host_list(ks), x)
                assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref)), ks
    finally:
        h.close()


def test_kshift_sweep_eigenvalues(system):
    rec, para, subs, _ = system
    sub = subs[7]
    res = momed.kshift_sweep(sub, para, rec, KSHIFTS, L.NEIGEN, want_vectors=True)
    for ks, (vals, vecs, resid) in zip(KSHIFTS, res):
        op = momed.MBOperator(momed.ED_scatterlist_twobody(para, kshift=ks), upper_hermitian=True)
        E, _ = momed.EDsolve(sub, op, N=L.NEIGEN, method_info=False, tol=1e-12)
        assert np.max(np.abs(vals - E) / np.abs(E)) < 1e-10, ks
        assert np.max(resid) <= 1e-9
        w = np.linalg.eigvalsh(O.dense_hamiltonian(sub.list, host_list(ks)))[:L.NEIGEN]
        assert np.max(np.abs(vals - w) / np.abs(w)) < 1e-10, ks


def test_recipe_refuses_wrong_use(system):
    rec, para, subs, _ = system
    h = momed.Handle(0)
    try:
        h.set_basis(subs[0].list)
        with pytest.raises(momed.MomedError):
            h.set_kshift(np.zeros(2))                 # no recipe attached
        op = momed.KShiftOperator(para, rec, h)
        with pytest.raises(momed.MomedError):
            h.set_kshift(np.array([np.nan, 0.0]))
        # a new operator drops the recipe
        full = op.full
        h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
        with pytest.raises(momed.MomedError):
            h.set_kshift(np.zeros(2))
    finally:
        h.close()
