"""Non-Hermitian eigensolve on the device (EDsolve(...; ishermitian = false)).

The reference passes the map of an operator whose term list is not Hermitian-completed to
krylov_map_solve(H, N; ishermitian = false) (MomentumEDCUDAExt.jl:159-179), i.e. KrylovKit's
Arnoldi with Krylov-Schur restarts, eigenvalues ordered by real part (:SR).  Bars: eigenvalues
within 1e-10 relative of LAPACK (numpy.linalg.eig on the oracle's dense matrix of the same term
list), residuals ||H x - e x|| <= 1e-9; on a sector too large for LAPACK, the eigenvalues of the
adjoint map are the complex conjugates of the map's (1e-9 relative).
"""
import numpy as np
import pytest

import momed
import oracle as O
from momed import core
from momed.synthetic import mesh_para

pytestmark = pytest.mark.gpu


def as_oracle(sl):
    o = np.zeros(len(sl), O.SCAT_DTYPE)
    o["re"], o["im"] = sl.amp.real, sl.amp.imag
    o["out"], o["in"], o["pm"] = sl.out, sl.in_, sl.pm
    return o


def non_hermitian(a, b, seed):
    """A genuinely non-Hermitian operator: the Hermitian-completed list of the recipe with the
    amplitudes of the terms below the diagonal (in < out) multiplied by 1.3 exp(0.7 i), taken as it
    is (upper_hermitian = false).  (The upper list alone is triangular in the sorted basis, with the
    real diagonal as its spectrum.)"""
    para, _ = mesh_para(a, b, seed)
    herm = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                            upper_hermitian=True)
    full = core.hermitian_complete(herm)
    amp = full.amp.copy()
    low = full.in_ < full.out
    amp[low] *= 1.3 * np.exp(0.7j)
    sl = core.ScatterList(amp, full.out, full.in_, full.pm, full.bits, full.element_type)
    return para, momed.MBOperator(sl, upper_hermitian=False)


def lapack_sr(basis, op):
    w, v = np.linalg.eig(O.dense_hamiltonian(basis, as_oracle(op.scats)))
    order = np.lexsort((w.imag, w.real))
    return w[order], v[:, order]


def nev_with_gap(w, top=8):
    for n in range(top, 1, -1):
        if w[n].real - w[n - 1].real > 1e-6 * max(1.0, abs(w[n - 1])):
            return n
    return 1


@pytest.mark.parametrize("sector", [0, 7])
def test_arnoldi_vs_lapack(sector):
    para, op = non_hermitian(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    space = core.HilbertSubspace(ref[sector], 15)
    w, _ = lapack_sr(ref[sector], op)
    assert np.max(np.abs(w.imag)) > 1e-3          # genuinely complex spectrum
    nev = nev_with_gap(w)
    M = momed.create_gpu_linearmap(momed.LinearMap(op, space))
    try:
        vals, vecs, info = momed.krylov_map_solve(M, nev, ishermitian=False, tol=1e-12, krylovdim=40)
    finally:
        M.release()
    assert np.max(np.abs(vals - w[:nev]) / np.abs(w[:nev])) < 1e-10, (vals, w[:nev])
    assert info["converged"] >= nev
    full = as_oracle(op.scats)
    for lam, x in zip(vals, vecs):
        r = O.matvec(ref[sector], full, x) - lam * x
        assert np.linalg.norm(r) <= 1e-9 * max(1.0, abs(lam))
        assert abs(np.linalg.norm(x) - 1.0) < 1e-12


def test_edsolve_non_hermitian_dropin():
    para, op = non_hermitian(3, 5, 0)
    subs, _ = momed.ED_momentum_subspaces(para, (5,))
    w, _ = lapack_sr(subs[3].list, op)
    E, vecs = momed.EDsolve(subs[3], op, N=3, ishermitian=False, method_info=False)
    assert E.dtype == np.complex128 and len(vecs) == 3
    assert np.max(np.abs(E - w[:3]) / np.abs(w[:3])) < 1e-10
    with pytest.raises(AssertionError):
        momed.EDsolve(subs[3], op, N=3)           # ishermitian=true needs an upper-Hermitian operator


def test_adjoint_spectrum_is_conjugate_3x8():
    """~30k states: the adjoint map's eigenvalues are the conjugates of the map's."""
    para, op = non_hermitian(3, 8, 5)
    subs, _ = momed.ED_momentum_subspaces(para, (8,))
    space = subs[2]
    M = momed.create_gpu_linearmap(momed.LinearMap(op, space))
    Ma = M.adjoint()
    try:
        v1, x1, i1 = momed.krylov_map_solve(M, 4, ishermitian=False, tol=1e-10, krylovdim=60, maxiter=300)
        v2, x2, i2 = momed.krylov_map_solve(Ma, 4, ishermitian=False, tol=1e-10, krylovdim=60, maxiter=300)
    finally:
        Ma.release()
        M.release()
    assert i1["converged"] >= 4 and i2["converged"] >= 4
    assert np.max(np.abs(v2 - np.conj(v1)) / np.abs(v1)) < 1e-9
    assert np.max(i1["residuals"]) <= 1e-8 and np.max(i2["residuals"]) <= 1e-8
