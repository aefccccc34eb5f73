"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

Bars (stated per test):
  - basis enumeration, sector order, index lookups: bit-exact;
  - matvec: complex128 within 1e-13 relative (max |dy| / max |y|), complex64
    within 2e-6 relative of the FP64 oracle (different summation order only);
  - eigenvalues within 1e-10 relative of LAPACK (numpy.linalg.eigh) on the
    dense matrix, eigenvector subspace overlap >= 1 - 1e-9, residual reported.
"""
import os

import numpy as np
import pytest

import oracle as O
import momed
from momed import core
from momed.synthetic import mesh_para, u_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    hd = momed.Handle(0)
    yield hd
    hd.close()


def operator_lists(a, b, seed, ncc=1):
    """(upper MBOperator, full completed ScatterList, oracle full list) of the synthetic recipe."""
    para, mh = mesh_para(a, b, seed, Nc_conserve=ncc)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    full = core.hermitian_complete(op)
    S = O.Synth(a, b, seed, Nc_conserve=ncc)
    ofull = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    return para, op, full, ofull


def load(h, basis, full):
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# ------------------------------------------------------------------------------ kernel (a)
@pytest.mark.parametrize("a,b,ne", [(3, 5, (5,)), (3, 9, (9,)), (4, 4, (6,))])
def test_enumeration_bit_exact(h, a, b, ne):
    got = h.enumerate_basis(O.mesh_klist(a, b), (a, b), 1, 1, ne)
    ref, ks = O.momentum_subspaces(O.mesh_klist(a, b), (a, b), ne)
    assert [k for k, _ in got] == ks
    for (k, g), r in zip(got, ref):
        assert np.array_equal(g, r)


def test_enumeration_two_component(h):
    kl = O.mesh_klist(4, 3)
    got = h.enumerate_basis(kl, (4, 3), 1, 2, (3, 3))
    ref, ks = O.momentum_subspaces(kl, (4, 3), (3, 3), Nc_conserve=2)
    assert [k for k, _ in got] == ks and all(np.array_equal(g, r) for (_, g), r in zip(got, ref))
    assert sum(len(r) for r in ref) == 220 * 220


def test_enumeration_mask_holes_restriction(h):
    kl = O.mesh_klist(3, 4)
    # mask over both conserved components, a hole component, a momentum restriction with duplicates
    mask = [1, 2, 4, 5, 7, 8, 10, 11, 13, 14, 16, 19, 20, 22, 23]
    for ne, kw in [((2, -3), dict(mask=mask)), ((3, 2), dict(momentum_list=[(1, 2), (0, 0), (4, 6), (1, 2)])),
                   ((-2, 2), {})]:
        got = h.enumerate_basis(kl, (3, 4), 1, 2, ne, **kw)
        ref, ks = O.momentum_subspaces(kl, (3, 4), ne, Nc_conserve=2, **kw)
        assert [k for k, _ in got] == ks
        assert all(np.array_equal(g, r) for (_, g), r in zip(got, ref))


def test_enumeration_open_direction(h):
    # Gk = 0 in one direction: raw momentum sums, range min..max * Ne (momentum_decomposition.jl:360-368)
    kl = np.array([[0, 1, 2, 0, 1, 2, 0, 1], [0, 0, 0, 1, 1, 1, 2, 2]], np.int64)
    got = h.enumerate_basis(kl, (3, 0), 1, 1, (3,))
    ref, ks = O.momentum_subspaces(kl, (3, 0), (3,))
    assert [k for k, _ in got] == ks and all(np.array_equal(g, r) for (_, g), r in zip(got, ref))


def test_ed_momentum_subspaces_api(h):
    para, _ = mesh_para(3, 5, 0)
    subs, ks = momed.ED_momentum_subspaces(para, (5,), handle=h)
    ref, rks = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    assert ks == rks and all(np.array_equal(s.list, r) for s, r in zip(subs, ref))
    # selection_rule filters states (leaf test at momentum_decomposition.jl:293)
    subs2, _ = momed.ED_momentum_subspaces(para, (5,), handle=h, selection_rule=lambda m: (m.n & 1) == 0)
    assert all(np.all((s.list & np.uint64(1)) == 0) for s in subs2)


# ------------------------------------------------------------------------------ kernel (b)
def test_matvec_config1_all_sectors(h):
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    rng = np.random.default_rng(0)
    for basis in ref:
        load(h, basis, full)
        x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
        y = h.matvec(x)
        yo = O.matvec(basis, ofull, x)
        assert rel(y, yo) < 1e-13
        assert h.stats()["index_mode"] == 0          # ranked tables, validated
        y32 = h.matvec(x.astype(np.complex64))
        assert rel(y32.astype(np.complex128), yo) < 2e-6


def test_matvec_two_component(h):
    para, op, full, ofull = operator_lists(4, 3, 5, ncc=2)
    ref, _ = O.momentum_subspaces(O.mesh_klist(4, 3), (4, 3), (3, 3), Nc_conserve=2)
    rng = np.random.default_rng(1)
    for basis in ref[:3]:
        load(h, basis, full)
        x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
        assert rel(h.matvec(x), O.matvec(basis, ofull, x)) < 1e-13
        st = h.stats()
        assert st["nnz"] == O.count_hits(basis, ofull)


def test_matvec_3x8_sector(h):
    para, op, full, ofull = operator_lists(3, 8, 4)
    got = h.enumerate_basis(O.mesh_klist(3, 8), (3, 8), 1, 1, (8,), momentum_list=[(1, 3)])
    basis = got[0][1]
    load(h, basis, full)
    x = np.random.default_rng(2).normal(size=(len(basis), 2)) @ np.array([1, 1j])
    assert rel(h.matvec(x), O.matvec(basis, ofull, x)) < 1e-13
    assert h.stats()["nnz"] == O.count_hits(basis, ofull)


def test_matvec_search_mode_subset_basis(h):
    # a basis that is not a whole sector: ranked tables are refused, the search fallback is exact
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[2][np.random.default_rng(3).random(len(ref[2])) < 0.6]
    load(h, basis, full)
    x = np.random.default_rng(4).normal(size=len(basis)) + 0j
    assert rel(h.matvec(x), O.matvec(basis, ofull, x)) < 1e-13
    assert h.stats()["index_mode"] == 2


def test_matvec_checked_mode_dropped_targets(h):
    # an operator that leaves the sector: targets outside the basis are dropped (index_fit / j == 0)
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    extra = momed.sort_merge_scatlist([momed.Scatter(0.7 + 0.2j, 1, 2, bits=15, upper_hermitian=True),
                                       momed.Scatter(0.3, 4, 9, 2, 1, bits=15, upper_hermitian=True)])
    op2 = momed.MBOperator(op.scats, extra, upper_hermitian=True)
    full2 = core.hermitian_complete(op2)
    ofull2 = np.zeros(len(full2), O.SCAT_DTYPE)
    ofull2["re"], ofull2["im"] = full2.amp.real, full2.amp.imag
    ofull2["out"], ofull2["in"], ofull2["pm"] = full2.out, full2.in_, full2.pm
    basis = ref[4]
    load(h, basis, full2)
    x = np.random.default_rng(5).normal(size=len(basis)) + 1j
    assert rel(h.matvec(x), O.matvec(basis, ofull2, x)) < 1e-13
    assert h.stats()["index_mode"] == 1


def test_matvec_device_pointers(h):
    import torch
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[0]
    load(h, basis, full)
    x = torch.randn(len(basis), dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    h.matvec_device(x.data_ptr(), y.data_ptr())
    yo = O.matvec(basis, ofull, x.cpu().numpy())
    assert rel(y.cpu().numpy(), yo) < 1e-13


def test_matvec_3x10_sector_properties(h):
    """A full 3x10 Ne=10 sector (~1.0M states): Hermiticity, linearity and sampled rows vs the oracle."""
    para, op, full, ofull = operator_lists(3, 10, 1)
    got = h.enumerate_basis(O.mesh_klist(3, 10), (3, 10), 1, 1, (10,), momentum_list=[(0, 0)])
    basis = got[0][1]
    assert len(basis) > 900_000
    load(h, basis, full)
    rng = np.random.default_rng(6)
    x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    z = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    hx, hz = h.matvec(x), h.matvec(z)
    assert abs(np.vdot(z, hx) - np.vdot(hz, x)) < 1e-10 * abs(np.vdot(z, hx))
    assert rel(h.matvec(2 * x - 3j * z), 2 * hx - 3j * hz) < 1e-12
    rows = rng.choice(len(basis), 3000, replace=False)
    assert rel(hx[rows], O.matvec_rows(basis, ofull, x, rows)) < 1e-13
    st = h.stats()
    assert st["index_mode"] == 0 and st["nnz"] > 300 * len(basis)


def sector_count(a, b, ne, K):
    """States of ne electrons on the a x b mesh with total momentum K (mod (a, b)), by a DP over
    orbitals (no enumeration)."""
    dp = np.zeros((ne + 1, a, b), np.int64)
    dp[0, 0, 0] = 1
    for i in range(a * b):
        kx, ky = i % a, i // a
        dp[1:] = dp[1:] + np.roll(np.roll(dp[:-1], kx, axis=1), ky, axis=2)
    return int(dp[ne, K[0] % a, K[1] % b])


def test_matvec_4x9_ne12_largest_sector(h):
    """The largest configured size: a 4x9 Ne=12 sector (~34.8M states, 36-bit states, from a
    1.25G-rank enumeration).  Size against a DP count, sorted and unique, momentum of sampled
    states, Hermiticity and sampled rows of the c128 map against the oracle."""
    para, op, full, ofull = operator_lists(4, 9, 4)
    got = h.enumerate_basis(O.mesh_klist(4, 9), (4, 9), 1, 1, (12,), momentum_list=[(1, 2)])
    k, basis = got[0]
    assert tuple(k) == (1, 2)
    assert len(basis) == sector_count(4, 9, 12, (1, 2)) > 34_000_000
    assert np.all(basis[1:] > basis[:-1])
    rng = np.random.default_rng(11)
    for st in basis[rng.choice(len(basis), 2000, replace=False)]:
        occ = [i for i in range(36) if (int(st) >> i) & 1]
        assert len(occ) == 12
        assert (sum(i % 4 for i in occ) % 4, sum(i // 4 for i in occ) % 9) == (1, 2)
    load(h, basis, full)
    x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    z = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    hx, hz = h.matvec(x), h.matvec(z)
    assert abs(np.vdot(z, hx) - np.vdot(hz, x)) < 1e-10 * abs(np.vdot(z, hx))
    rows = rng.choice(len(basis), 2000, replace=False)
    assert rel(hx[rows], O.matvec_rows(basis, ofull, x, rows)) < 1e-13
    assert h.stats()["nnz"] > 500 * len(basis)
    # the slot-mode hit cache (2 bytes per hit, ~43 GB here; a full cache would need ~170 GB)
    old = os.environ.get("MOMED_HITCACHE")
    os.environ["MOMED_HITCACHE"] = "2"
    try:
        info = h.build_hit_cache()
    finally:
        if old is None:
            del os.environ["MOMED_HITCACHE"]
        else:
            os.environ["MOMED_HITCACHE"] = old
    assert info["mode"] == "slots" and info["hits"] > 500 * len(basis)
    assert rel(h.matvec(x), hx) < 1e-13
    h.release_hit_cache()


# ------------------------------------------------------------------------------ Lanczos
def check_eigs(vals, vecs, H, tol_rel=1e-10, overlap_tol=1e-9):
    w, U = np.linalg.eigh(H)
    nev = len(vals)
    assert np.max(np.abs(vals - w[:nev]) / np.maximum(np.abs(w[:nev]), 1.0)) < tol_rel
    for i in range(nev):
        cluster = np.abs(w - vals[i]) < 1e-6
        ov = np.linalg.norm(U[:, cluster].conj().T @ vecs[i])
        assert ov > 1 - overlap_tol, (i, ov)


@pytest.mark.parametrize("sector", [0, 5, 11])
def test_eigsolve_fp64_vs_lapack(h, sector):
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[sector]
    load(h, basis, full)
    vals, vecs, resid, info = h.eigsolve(10, krylovdim=30, tol=1e-12, seed=1)
    assert info["converged"] >= 10
    assert np.all(resid < 1e-10)
    check_eigs(vals, vecs, O.dense_hamiltonian(basis, ofull))


def test_eigsolve_mixed_precision_vs_lapack(h):
    para, op, full, ofull = operator_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[3]
    load(h, basis, full)
    vals, vecs, resid, info = h.eigsolve(10, krylovdim=30, tol=1e-12, seed=2, precision=momed._lib.PREC_MIXED)
    check_eigs(vals, vecs, O.dense_hamiltonian(basis, ofull), tol_rel=1e-10, overlap_tol=1e-6)


def test_eigsolve_matches_oracle_lanczos_3x8(h):
    para, op, full, ofull = operator_lists(3, 8, 4)
    got = h.enumerate_basis(O.mesh_klist(3, 8), (3, 8), 1, 1, (8,), momentum_list=[(2, 5)])
    basis = got[0][1]
    load(h, basis, full)
    vals, vecs, resid, info = h.eigsolve(6, krylovdim=40, tol=1e-12, seed=3)
    ovals, ovecs, ores, oinfo = O.eigsolve(basis, ofull, 6, krylovdim=40, tol=1e-12, seed=3, want_vectors=True)
    assert np.max(np.abs(vals - ovals) / np.abs(ovals)) < 1e-10
    for i in range(6):
        assert abs(abs(np.vdot(ovecs[i], vecs[i])) - 1) < 1e-8 or abs(vals[i] - vals[min(i + 1, 5)]) < 1e-6


def test_edsolve_dropin_two_component(h):
    """EDsolve(subspace, H; method=:map, device=:gpu) end to end on a two-component sector."""
    para, mh = mesh_para(4, 3, 5, Nc_conserve=2)
    subs, ks = momed.ED_momentum_subspaces(para, (3, 3), handle=h)
    sub = subs[0]
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    E, vecs = momed.EDsolve(sub, op, N=8, method="map", device="gpu", method_info=False)
    S = O.Synth(4, 3, 5, Nc_conserve=2)
    ofull = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    check_eigs(E, [v.vec for v in vecs], O.dense_hamiltonian(sub.list, ofull))
    assert all(isinstance(v, momed.MBS64Vector) for v in vecs)


def test_eigsolve_small_sector_krylov_exhausts(h):
    # N < krylovdim: the Krylov space is the whole space (invariant subspace path)
    para, op, full, ofull = operator_lists(2, 2, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(2, 2), (2, 2), (2,))
    basis = max(ref, key=len)
    load(h, basis, full)
    vals, vecs, resid, info = h.eigsolve(len(basis), krylovdim=30, tol=1e-12, seed=4)
    check_eigs(vals, vecs, O.dense_hamiltonian(basis, ofull))


# ------------------------------------------------------------------------------ batched solver
def pair_lists(a, b, seed):
    from momed.core import pair_operator
    para, _ = mesh_para(a, b, seed)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    return pair_operator(A, B)


def oracle_list(amp, in_, out, pm):
    o = np.zeros(len(amp), O.SCAT_DTYPE)
    o["re"], o["im"], o["out"], o["in"], o["pm"] = amp.real, amp.imag, out, in_, pm
    return o


def test_parametrised_matvec(h):
    amp_a, amp_b, in_, out, pm = pair_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[1]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    x = np.random.default_rng(7).normal(size=len(basis)) + 0.3j
    for u0 in (0.5, 1.25, 2.0):
        h.set_param(u0)
        yo = O.matvec(basis, oracle_list(amp_a + u0 * amp_b, in_, out, pm), x)
        assert rel(h.matvec(x), yo) < 1e-13
    h.set_param(1.0)


@pytest.mark.parametrize("precision", [momed._lib.PREC_MIXED, momed._lib.PREC_FP64])
@pytest.mark.parametrize("nu", [8, 32, 5])
def test_batch_solve_vs_lapack(h, precision, nu):
    amp_a, amp_b, in_, out, pm = pair_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[6]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    u = u_grid(nu, 0.5, 2.0)
    vals, vecs, resid, info = h.batch_solve(u, 4, krylovdim=30, tol=1e-12, precision=precision, want_vectors=True)
    assert vals.shape == (nu, 4)
    for q in range(nu):
        H = O.dense_hamiltonian(basis, oracle_list(amp_a + u[q] * amp_b, in_, out, pm))
        check_eigs(vals[q], vecs[q], H, tol_rel=1e-10, overlap_tol=1e-6)
        assert np.all(resid[q] < 1e-5)


def test_batch_solve_3x8_matches_plain_fp64(h):
    """The 32-wide mixed-precision batch on a 3x8 sector agrees with one-at-a-time FP64 solves."""
    amp_a, amp_b, in_, out, pm = pair_lists(3, 8, 4)
    got = h.enumerate_basis(O.mesh_klist(3, 8), (3, 8), 1, 1, (8,), momentum_list=[(0, 2)])
    basis = got[0][1]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    u = u_grid(32, 0.5, 2.0)
    vals, _, resid, info = h.batch_solve(u, 4, krylovdim=30, tol=1e-12, precision=momed._lib.PREC_MIXED)
    for q in (0, 13, 31):
        h.set_param(float(u[q]))
        pv, _, pr, pinfo = h.eigsolve(4, krylovdim=30, tol=1e-12, seed=5, want_vectors=False)
        assert np.max(np.abs(vals[q] - pv) / np.abs(pv)) < 1e-10
    h.set_param(1.0)


@pytest.mark.parametrize("nu,nev", [(32, 4), (8, 10)])
def test_batch_solve_3x9_refinement_matches_plain_fp64(h, nu, nev):
    """A full 3x9 Ne=9 sector (173,583 states): the FP32 phase stops at its floor and the anchored
    refinement (FP32 extension of FP64 Ritz vectors) finishes; eigenvalues, residuals and
    eigenvectors agree with one-at-a-time FP64 solves."""
    amp_a, amp_b, in_, out, pm = pair_lists(3, 9, 2)
    got = h.enumerate_basis(O.mesh_klist(3, 9), (3, 9), 1, 1, (9,), momentum_list=[(1, 4)])
    basis = got[0][1]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    u = u_grid(nu, 0.5, 2.0)
    vals, vecs, resid, info = h.batch_solve(u, nev, krylovdim=30, tol=1e-12, precision=momed._lib.PREC_MIXED,
                                             want_vectors=True)
    assert info["converged"] >= nev
    for q in sorted({0, nu // 2, nu - 1}):
        h.set_param(float(u[q]))
        pv, pvecs, pr, pinfo = h.eigsolve(nev, krylovdim=30, tol=1e-12, seed=5, want_vectors=True)
        assert np.max(np.abs(vals[q] - pv) / np.abs(pv)) < 1e-10
        for i in range(nev):
            gap = np.min(np.abs(np.delete(pv, i) - pv[i])) if nev > 1 else 1.0
            if gap > 1e-6:                                   # nondegenerate: vectors agree up to phase,
                ov = abs(np.vdot(pvecs[i], vecs[q, i]))      # within the residual-over-gap bound
                assert 1 - ov <= max(1e-9, 4 * (resid[q, i] / gap) ** 2)
    h.set_param(1.0)
