"""Hit cache of the matrix-free map (momed_build_hit_cache): the map over the cached (target row,
term slot, sign) of every hit against the candidate map and the oracle's dense restatement, and
the eigensolvers over it against LAPACK and against the same solves without it.

The test operator mixes the three amplitude kinds the cache sorts hits into (B part only, A part
only, both) while staying Hermitian: the kind of a term is chosen from in ^ out, which a term and
its Hermitian partner share.

Bars:
  - complex128 map within 1e-13 relative of the candidate map and of the dense product
    (same values, another summation order), complex64 within 2e-6;
  - the cache holds exactly the off-diagonal entries of the sparse method's matrix;
  - eigenvalues within 1e-10 relative of LAPACK and 1e-11 of the solves without the cache (the
    batched solves converge to tol 1e-12; a near-degenerate pair, as the sixth and fifth levels
    here, 6.0492 / 6.0477, moves by a few 1e-12 with the summation order).
"""
import os
from contextlib import contextmanager

import numpy as np
import pytest

import oracle as O
import momed
from momed import _lib
from momed.core import pair_operator
from momed.synthetic import mesh_para

pytestmark = pytest.mark.gpu


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


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def kind_mix_pair(a, b, seed):
    """H(u) = A2 + u B2 with off-diagonal terms of all three kinds, Hermitian for real u."""
    para, _ = mesh_para(a, b, seed)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    amp_a, amp_b, in_, out, pm = pair_operator(A, B)
    sel = (in_ ^ out) % np.uint64(3)
    a2 = amp_a.copy()
    b2 = amp_b.copy()
    both, aonly = sel == 0, sel == 1
    a2[both] += 0.4 * amp_b[both]
    a2[aonly] += 0.7 * amp_b[aonly]
    b2[aonly] = 0.0
    return para, (a2, b2, in_, out, pm)


def dense(basis, pair, u):
    a2, b2, in_, out, pm = pair
    amp = a2 + u * b2
    o = np.zeros(len(amp), O.SCAT_DTYPE)
    o["re"], o["im"], o["out"], o["in"], o["pm"] = amp.real, amp.imag, out, in_, pm
    return O.dense_hamiltonian(basis, o)


@pytest.fixture(scope="module")
def setup():
    h = momed.Handle(0)
    para, pair = kind_mix_pair(3, 6, 0)
    secs = h.enumerate_basis(para.k_list, para.Gk, 1, 1, (6,))
    basis = secs[4][1]
    h.set_basis(basis)
    h.set_scatter_pair(*pair)
    a2, b2, in_, out, _ = pair
    offd = in_ != out
    kinds = {(bool(np.any(x != 0)), bool(np.any(y != 0))) for x, y in zip(a2[offd], b2[offd])}
    assert {(False, True), (True, False), (True, True)} <= kinds     # all three kinds present
    yield h, basis, pair
    h.close()


def test_cached_map_matches_candidate_map_and_dense(setup):
    h, basis, pair = setup
    n = len(basis)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for u in (0.0, 0.7, 1.9):
        h.set_param(u)
        h.release_hit_cache()
        y_cand = h.matvec(x)
        y32_cand = h.matvec(x.astype(np.complex64))
        info = h.build_hit_cache()
        assert info is not None and info["hits"] > 0 and info["bytes"] >= 8 * info["hits"]
        y_hc = h.matvec(x)
        y32_hc = h.matvec(x.astype(np.complex64))
        y_ref = dense(basis, pair, u) @ x
        assert rel(y_hc, y_ref) < 1e-13
        assert rel(y_hc, y_cand) < 1e-13
        assert rel(y32_hc.astype(np.complex128), y_ref) < 2e-6
        assert rel(y32_hc.astype(np.complex128), y32_cand.astype(np.complex128)) < 2e-6


def test_cache_holds_the_sparse_matrix_offdiagonal_entries(setup):
    h, basis, _ = setup
    hits = h.build_hit_cache()["hits"]
    nnz = h.build_sparse()                 # one entry per off-diagonal hit plus the diagonal
    assert h.hit_cache_info() is None      # dropped: maps read the matrix while it is built
    assert hits == nnz - len(basis)
    h.release_sparse()


def test_cache_lifetime(setup):
    h, basis, pair = setup
    h.set_param(1.0)
    h.release_hit_cache()
    assert h.hit_cache_info() is None
    h.eigsolve(4, tol=1e-10)                       # the solvers build it when it fits
    assert h.hit_cache_info() is not None
    h.set_param(1.3)                               # a new u keeps it (values come from the term list)
    assert h.hit_cache_info() is not None
    with env(MOMED_HITCACHE=0):
        h.set_basis(basis)                         # a new basis drops it
        assert h.hit_cache_info() is None
        h.eigsolve(4, tol=1e-10)
        assert h.hit_cache_info() is None          # and MOMED_HITCACHE=0 keeps the solvers off it
    h.build_hit_cache()
    h.set_scatter_pair(*pair)                      # a new operator drops it
    assert h.hit_cache_info() is None


def test_solvers_over_the_cache_vs_lapack(setup):
    h, basis, pair = setup
    us = np.array([0.5, 1.0, 1.5, 2.0])
    nev = 6
    ref = [np.linalg.eigvalsh(dense(basis, pair, u))[:nev] for u in us]
    res = {}
    for flag in ("1", "0"):
        with env(MOMED_HITCACHE=flag):
            h.set_basis(basis)
            h.profile(True)
            vals, _, _, info = h.batch_solve(us, nev, krylovdim=30, tol=1e-12, precision=_lib.PREC_MIXED)
            n_hc, _ = h.profile_read(_lib.KERNEL_HC_BLOCK_C64)
            n_cand, _ = h.profile_read(_lib.KERNEL_BLOCK_MATVEC_C64)
            h.profile(False)
            if flag == "1":
                assert n_hc > 0 and n_cand == 0
            else:
                assert n_hc == 0 and n_cand > 0
            for r, v in zip(ref, vals):
                assert np.max(np.abs(v - r) / np.abs(r)) < 1e-10
            res[flag] = vals
    assert np.max(np.abs(res["1"] - res["0"]) / np.abs(res["0"])) < 1e-11

    # block Lanczos (c128 block maps over the cache) and the single-vector solver
    h.set_basis(basis)
    h.set_param(1.25)
    w = np.linalg.eigvalsh(dense(basis, pair, 1.25))[:8]
    with env(MOMED_BLOCK=4):
        vals, _, resid, info = h.eigsolve(8, krylovdim=48, tol=1e-12)
    assert h.hit_cache_info() is not None
    assert np.max(np.abs(vals - w) / np.abs(w)) < 1e-10
    with env(MOMED_BLOCK=0):
        vals1, _, _, _ = h.eigsolve(8, krylovdim=48, tol=1e-12)
    assert np.max(np.abs(vals1 - w) / np.abs(w)) < 1e-10


def test_block_map_at_32_right_hand_sides(setup):
    """The 32-wide block map of the batched solver (FP32 Lanczos and FP64 checks) over the cache
    against LAPACK and against the candidate block map; with a B part (32 parameter values) and
    without one (the operator set as one term list, all right-hand sides the same matrix)."""
    h, basis, pair = setup
    us = np.linspace(0.5, 2.0, 32)
    nev = 3
    ref = {i: np.linalg.eigvalsh(dense(basis, pair, us[i]))[:nev] for i in (0, 13, 31)}
    res = {}
    for flag in ("1", "0"):
        with env(MOMED_HITCACHE=flag):
            h.set_basis(basis)
            vals, _, _, _ = h.batch_solve(us, nev, krylovdim=24, tol=1e-12, precision=_lib.PREC_MIXED)
        assert vals.shape == (32, nev)
        for i, r in ref.items():
            assert np.max(np.abs(vals[i] - r) / np.abs(r)) < 1e-10
        res[flag] = vals
    assert np.max(np.abs(res["1"] - res["0"]) / np.abs(res["0"])) < 1e-11

    a2, b2, in_, out, pm = pair
    u = 1.1
    w = np.linalg.eigvalsh(dense(basis, pair, u))[:nev]
    h.set_scatter(a2 + u * b2, in_, out, pm)
    try:
        with env(MOMED_HITCACHE=1):
            vals, _, _, _ = h.batch_solve(us, nev, krylovdim=24, tol=1e-12, precision=_lib.PREC_MIXED)
        assert np.max(np.abs(vals - w[None, :]) / np.abs(w[None, :])) < 1e-10
    finally:
        h.set_scatter_pair(*pair)
        h.set_basis(basis)


def test_slot_mode_matches_full_cache(setup):
    """Slot mode (term slot per hit, the target formed at each application): the same hits as
    the full cache and the same products."""
    h, basis, pair = setup
    n = len(basis)
    rng = np.random.default_rng(8)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    h.set_param(0.9)
    full = h.build_hit_cache()
    y_full, y32_full = h.matvec(x), h.matvec(x.astype(np.complex64))
    with env(MOMED_HITCACHE=2):
        slots = h.build_hit_cache()
    assert slots["hits"] == full["hits"] and slots["bytes"] < full["bytes"]
    assert full["mode"] == "full" and slots["mode"] == "slots"
    y_sl, y32_sl = h.matvec(x), h.matvec(x.astype(np.complex64))
    y_ref = dense(basis, pair, 0.9) @ x
    assert rel(y_sl, y_ref) < 1e-13 and rel(y_sl, y_full) < 1e-13
    assert rel(y32_sl.astype(np.complex128), y32_full.astype(np.complex128)) < 2e-6
    w = np.linalg.eigvalsh(dense(basis, pair, 0.9))[:4]
    vals, _, _, _ = h.eigsolve(4, tol=1e-12)            # the single-vector solver over the slots
    assert np.max(np.abs(vals - w) / np.abs(w)) < 1e-10
    h.release_hit_cache()
