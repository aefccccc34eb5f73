"""The reference's own test workload on the GPU (MomentumED/test/example1_FQH_Laughlin.jl).

Laughlin state at filling 1/3: 3 x 4 torus mesh, Ne = 4, the screened Coulomb interaction with
magnetic-translation phases given on momentum coordinates (the coordinate branch of
ED_scatterlist_twobody, scat_list.jl:442-497).  Every one of the 12 momentum sectors is solved
on the device for the test's N = 10 lowest eigenpairs (the reference loops EDsolve over the
sectors, example1_FQH_Laughlin.jl:103-113), by the matrix-free map and by the sparse method, and
compared with LAPACK on the oracle's dense matrix.

Bars: bases bit-exact; eigenvalues within 1e-10 relative of LAPACK; each eigenvector's FP64
residual ||H psi - E psi|| (oracle map) <= 1e-8; the eigenspace of each cluster of equal
eigenvalues overlaps LAPACK's to >= 1 - 1e-9.
"""
from fractions import Fraction

import numpy as np
import pytest

import laughlin as L
import momed
import oracle as O

pytestmark = pytest.mark.gpu


def para():
    return momed.EDPara(k_list=L.K_LIST, Gk=L.GK, H_two=L.V_int, two_momentum_coordinate=True)


def lapack(basis, full_oracle, n):
    w, v = np.linalg.eigh(O.dense_hamiltonian(basis, full_oracle))
    return w[:n], v[:, :n]


def subspace_overlap(V, W):
    """min singular value of V^H W for orthonormal columns V, W of the same span size."""
    return float(np.min(np.linalg.svd(V.conj().T @ W, compute_uv=False)))


def check_solution(basis, ofull, E, vecs, tol=1e-10):
    n = len(E)
    w, V = lapack(basis, ofull, n)
    assert np.max(np.abs(E - w) / np.abs(w)) < tol, (E, w)
    X = np.stack([np.asarray(v.vec if hasattr(v, "vec") else v) for v in vecs], axis=1)
    for i in range(n):
        r = O.matvec(basis, ofull, X[:, i]) - E[i] * X[:, i]
        assert np.linalg.norm(r) <= 1e-8
    # clusters of (near-)equal eigenvalues compared as subspaces
    i = 0
    while i < n:
        j = i + 1
        while j < n and abs(w[j] - w[j - 1]) < 1e-6 * max(1.0, abs(w[j])):
            j += 1
        if j < n or i == 0:                       # a cluster cut at N has no well-defined span
            assert subspace_overlap(V[:, i:j], X[:, i:j]) >= 1 - 1e-9
        i = j


@pytest.fixture(scope="module")
def workload():
    p = para()
    scat = momed.ED_scatterlist_twobody(p)
    op = momed.MBOperator(scat, upper_hermitian=True)
    ofull = O.hermitian_complete(O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int))
    subs, ks = momed.ED_momentum_subspaces(p, (L.NE,))
    return p, scat, op, ofull, subs, ks


def test_laughlin_sectors_bit_exact(workload):
    _, _, _, _, subs, ks = workload
    ref, rks = O.momentum_subspaces(L.K_LIST, L.GK, (L.NE,))
    assert ks == rks and all(np.array_equal(s.list, r) for s, r in zip(subs, ref))


@pytest.mark.parametrize("method", ["map", "sparse"])
def test_laughlin_all_sectors_edsolve(workload, method):
    _, _, op, ofull, subs, ks = workload
    lows = []
    for s, k in zip(subs, ks):
        E, vecs = momed.EDsolve(s, op, N=L.NEIGEN, method=method, method_info=False, tol=1e-12)
        check_solution(s.list, ofull, E, vecs)
        lows += [(e, k) for e in E]
    lows.sort()
    # the three-fold Laughlin ground state in the ky = 2 sectors, below the gap
    assert sorted(k for _, k in lows[:3]) == [(0, 2), (1, 2), (2, 2)]
    assert lows[2][0] - lows[0][0] < 1e-7 and lows[3][0] - lows[2][0] > 0.04


def test_laughlin_scatter_list_form(workload):
    """EDsolve(subspace, scat; N) as the reference test calls it (the scatter-list form)."""
    _, scat, _, ofull, subs, _ = workload
    E, vecs = momed.EDsolve(subs[6], scat, N=L.NEIGEN, method_info=False, tol=1e-12)
    check_solution(subs[6].list, ofull, E, vecs)
    with pytest.raises(ValueError):
        momed.EDsolve(subs[6], scat, N=2, method="map")


@pytest.mark.parametrize("kshift", [(0.5, 0.25), (Fraction(1, 3), Fraction(2, 3))], ids=["float", "rational"])
def test_laughlin_twisted_boundary(workload, kshift):
    """A twisted boundary (kshift), the ingredient of the reference's Wilson-loop sweeps."""
    p, _, _, _, subs, _ = workload
    scat = momed.ED_scatterlist_twobody(p, kshift=kshift)
    op = momed.MBOperator(scat, upper_hermitian=True)
    ofull = O.hermitian_complete(O.scatterlist_twobody_coord(L.K_LIST, L.GK, L.V_int, kshift=kshift))
    for si in (0, 7):
        E, vecs = momed.EDsolve(subs[si], op, N=L.NEIGEN, method="map", method_info=False, tol=1e-12)
        check_solution(subs[si].list, ofull, E, vecs)
