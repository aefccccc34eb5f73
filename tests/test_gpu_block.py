"""Block Lanczos (several Krylov vectors per map launch) against LAPACK and the single-vector solver.

momed_eigsolve switches to the block solver for nev >= 2 on sectors of >= 500k states; the
MOMED_BLOCK environment variable forces a block size (4, 8, 16) or the single-vector solver (0),
so these tests also run it on small sectors where LAPACK gives the exact answer.

Bars: eigenvalues within 1e-10 relative of LAPACK (or of the single-vector FP64 solver on
sectors too large for LAPACK); FP64 solves: residuals <= 1e-9, eigenspace overlap >= 1 - 1e-9; mixed
solves are accepted on eigenvalue accuracy (error ~ r^2 / gap), their residuals (~1e-6) stated.
"""
import os
from contextlib import contextmanager

import numpy as np
import pytest

import momed
import oracle as O
from momed import _lib, core
from momed.synthetic import mesh_para

pytestmark = pytest.mark.gpu


@contextmanager
def block(b):
    old = os.environ.get("MOMED_BLOCK")
    os.environ["MOMED_BLOCK"] = str(b)
    try:
        yield
    finally:
        if old is None:
            del os.environ["MOMED_BLOCK"]
        else:
            os.environ["MOMED_BLOCK"] = old


@pytest.fixture(scope="module")
def h():
    hd = momed.Handle(0)
    yield hd
    hd.close()


def setup(h, a, b, seed, ne, sector, ncc=1):
    para, _ = mesh_para(a, b, seed, Nc_conserve=ncc)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    full = core.hermitian_complete(op)
    secs = h.enumerate_basis(para.k_list, para.Gk, 1, ncc, ne)
    basis = secs[sector][1]
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    S = O.Synth(a, b, seed, Nc_conserve=ncc)
    ofull = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    return basis, ofull


def overlap(V, W):
    return float(np.min(np.linalg.svd(V.conj().T @ W, compute_uv=False)))


@pytest.mark.parametrize("bsize", [4, 8, 16])
@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED])
def test_block_vs_lapack_3x6(h, bsize, precision):
    basis, ofull = setup(h, 3, 6, 0, (6,), 4)
    assert len(basis) >= 16 * bsize
    w, V = np.linalg.eigh(O.dense_hamiltonian(basis, ofull))
    nev = 10
    with block(bsize):
        vals, vecs, resid, info = h.eigsolve(nev, krylovdim=30, tol=1e-12, seed=3, precision=precision)
    assert np.max(np.abs(vals - w[:nev]) / np.abs(w[:nev])) < 1e-10
    assert np.max(resid) <= 1e-9
    assert info["converged"] >= nev
    # whole clusters only (the 10th value may be cut inside a degenerate cluster)
    n = nev
    while n > 1 and abs(w[n] - w[n - 1]) < 1e-8:
        n -= 1
    assert overlap(V[:, :n], vecs[:n].T) >= 1 - 1e-9


def test_block_matches_single_vector_3x8(h):
    """A ~30k-state sector: block FP64 and mixed against the single-vector FP64 solver."""
    setup(h, 3, 8, 5, (8,), 2)
    with block(0):
        ref, rvecs, _, _ = h.eigsolve(6, krylovdim=40, tol=1e-12, seed=1)
    for b in (4, 8):
        for prec in (_lib.PREC_FP64, _lib.PREC_MIXED):
            with block(b):
                vals, vecs, resid, info = h.eigsolve(6, krylovdim=40, tol=1e-12, seed=1, precision=prec)
            assert np.max(np.abs(vals - ref) / np.abs(ref)) < 1e-10, (b, prec, vals, ref)
            if prec == _lib.PREC_FP64:
                assert np.max(resid) <= 1e-9
                assert overlap(rvecs.T, vecs.T) >= 1 - 1e-9
            else:                     # accepted on eigenvalue accuracy: residuals ~1e-6, stated
                assert np.max(resid) <= 1e-5
                assert overlap(rvecs.T, vecs.T) >= 1 - 1e-6


def test_block_is_default_for_large_sectors_without_hit_cache(h):
    """nev >= 6 on >= 500k states takes the block solver when the map has no hit cache: its maps
    are block-map launches.  Over a hit cache (below 2M states) the single-vector solver runs."""
    setup(h, 3, 10, 1, (10,), 3)
    assert h.n >= 500000
    with env(MOMED_HITCACHE=0):
        h.profile(True)
        vals, _, resid, info = h.eigsolve(6, krylovdim=30, tol=1e-12, seed=1, want_vectors=False)
        nblk, _ = h.profile_read(_lib.KERNEL_BLOCK_MATVEC_C128)
        nsingle, _ = h.profile_read(_lib.KERNEL_MATVEC_C128)
        h.profile(False)
    assert h.hit_cache_info() is None
    assert nblk > 0 and info["converged"] >= 6
    assert nsingle <= 6 * 2            # only the final FP64 residual maps are single-vector
    with block(0):                     # and MOMED_BLOCK=0 keeps the single-vector solver
        ref, _, _, _ = h.eigsolve(6, krylovdim=30, tol=1e-12, seed=1, want_vectors=False)
    assert np.max(np.abs(vals - ref) / np.abs(ref)) < 1e-10
    h.profile(True)                    # with the hit cache (built by the solver): single-vector maps
    vals2, _, _, _ = h.eigsolve(6, krylovdim=30, tol=1e-12, seed=1, want_vectors=False)
    nhc, _ = h.profile_read(_lib.KERNEL_HC_MATVEC_C128)
    nhb, _ = h.profile_read(_lib.KERNEL_HC_BLOCK_C128)
    h.profile(False)
    assert h.hit_cache_info() is not None and nhc > 0 and nhb == 0
    assert np.max(np.abs(vals2 - ref) / np.abs(ref)) < 1e-10


def test_block_start_vector_and_two_component(h):
    basis, ofull = setup(h, 4, 3, 3, (2, 2), 5, ncc=2)
    w = np.linalg.eigvalsh(O.dense_hamiltonian(basis, ofull))
    v0 = np.random.default_rng(4).standard_normal(len(basis)) + 0j
    with block(4):
        vals, _, resid, _ = h.eigsolve(5, krylovdim=24, tol=1e-12, vec0=v0)
    assert np.max(np.abs(vals - w[:5]) / np.abs(w[:5])) < 1e-10
    assert np.max(resid) <= 1e-9


@contextmanager
def env(**kv):
    old = {k: os.environ.get(k) for k in kv}
    os.environ.update({k: str(v) for k, v in kv.items()})
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("bsize", [8, 16])
def test_tensor_core_projection_matches_cuda_cores(h, bsize):
    """The mixed block solver's basis projections Q^H W run on the tensor cores (tcgen05.mma
    kind::tf32, split hi/lo); with MOMED_TC_CHECK=1 every projection is also computed on the CUDA
    cores in FP64 and the solve fails if any coefficient differs by more than 1e-5 (unit-norm
    FP32 vectors).  Then the solve is repeated with the tensor cores off: same eigenvalues to
    1e-10, and a similar number of maps."""
    setup(h, 3, 8, 5, (8,), 2)
    with env(MOMED_BLOCK=bsize, MOMED_TC_CHECK=1):
        v_tc, _, r_tc, i_tc = h.eigsolve(8, krylovdim=40, tol=1e-12, seed=2, want_vectors=False,
                                         precision=_lib.PREC_MIXED)
    with env(MOMED_BLOCK=bsize, MOMED_TC_PROJ=0):
        v_cc, _, r_cc, i_cc = h.eigsolve(8, krylovdim=40, tol=1e-12, seed=2, want_vectors=False,
                                         precision=_lib.PREC_MIXED)
    assert np.max(np.abs(v_tc - v_cc) / np.abs(v_cc)) < 1e-10
    assert max(np.max(r_tc), np.max(r_cc)) <= 1e-9
    assert i_tc["matvecs"] <= 1.25 * i_cc["matvecs"] + 8 * bsize
