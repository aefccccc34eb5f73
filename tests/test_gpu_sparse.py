"""GPU sparse method (EDsolve(...; method=:sparse, device=:gpu)): the CSR matrix built on the
device against the oracle's restatement of the reference's matrix builder, the CSR SpMV against
the matrix-free map, and eigenpairs against LAPACK.

Bars:
  - structure (column pointers, row indices after merging duplicates): identical to the oracle's
    CSC of ED_HamiltonianMatrix_threaded_CSCdirect;
  - values: within 1e-13 relative (the diagonal is summed in another order);
  - SpMV: complex128 within 1e-13 relative of the matrix-free map, complex64 within 2e-6;
  - eigenvalues within 1e-10 relative of LAPACK, eigenvector overlap >= 1 - 1e-9.
"""
import numpy as np
import pytest
import scipy.sparse as sps

import oracle as O
import momed
from momed import core
from momed.synthetic import mesh_para

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    hd = momed.Handle(0)
    yield hd
    hd.close()


def full_lists(a, b, seed, ncc=1):
    para, _ = mesh_para(a, b, seed, Nc_conserve=ncc)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    full = core.hermitian_complete(op)
    S = O.Synth(a, b, seed, Nc_conserve=ncc)
    ofull = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    return full, ofull


def oracle_list(amp, in_, out, pm):
    o = np.zeros(len(amp), O.SCAT_DTYPE)
    o["re"], o["im"], o["out"], o["in"], o["pm"] = amp.real, amp.imag, out, in_, pm
    return o


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def device_csc(h, n):
    rp, col, val = h.sparse_copy()
    assert rp[0] == 0 and rp[-1] == len(col)
    assert np.all(np.diff(rp) >= 1)
    assert np.array_equal(col[rp[:-1]], np.arange(n))            # the diagonal leads every row
    assert col.min() >= 0 and col.max() < n
    H = sps.csr_matrix((val, col, rp), shape=(n, n)).tocsc()
    H.sum_duplicates()
    H.eliminate_zeros()
    return H


def oracle_csc(basis, olist):
    cp, rv, nz = O.sparse_csc(basis, olist)
    H = sps.csc_matrix((nz, rv, cp), shape=(len(basis), len(basis)))
    H.eliminate_zeros()
    return H


def assert_same_matrix(Hd, Ho):
    assert np.array_equal(Hd.indptr, Ho.indptr)
    assert np.array_equal(Hd.indices, Ho.indices)
    assert rel(Hd.data, Ho.data) < 1e-13


def test_sparse_matches_oracle_matrix_config1(h):
    full, ofull = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    for basis in ref[::4]:
        h.set_basis(basis)
        h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
        nnz = h.build_sparse()
        Hd = device_csc(h, len(basis))
        Ho = oracle_csc(basis, ofull)
        assert_same_matrix(Hd, Ho)
        # one entry per row for the diagonal plus one per off-diagonal hit
        assert nnz == len(basis) + (Ho.nnz - np.count_nonzero(Ho.diagonal()))


def test_sparse_two_component_matches_oracle(h):
    full, ofull = full_lists(4, 3, 5, ncc=2)
    ref, _ = O.momentum_subspaces(O.mesh_klist(4, 3), (4, 3), (3, 3), Nc_conserve=2)
    basis = ref[1]
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    h.build_sparse()
    assert_same_matrix(device_csc(h, len(basis)), oracle_csc(basis, ofull))


def test_sparse_pair_operator_at_u_and_dropped_on_new_u(h):
    from momed.core import pair_operator
    para, _ = mesh_para(3, 5, 0)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    amp_a, amp_b, in_, out, pm = pair_operator(A, B)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[2]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    h.set_param(0.7)
    h.build_sparse()
    assert_same_matrix(device_csc(h, len(basis)), oracle_csc(basis, oracle_list(amp_a + 0.7 * amp_b, in_, out, pm)))
    x = np.random.default_rng(3).normal(size=len(basis)) + 0.5j
    assert rel(h.matvec(x), O.matvec(basis, oracle_list(amp_a + 0.7 * amp_b, in_, out, pm), x)) < 1e-13
    h.set_param(1.6)                       # values were built at 0.7: the matrix is dropped
    with pytest.raises(momed.MomedError):
        h.sparse_copy()
    assert rel(h.matvec(x), O.matvec(basis, oracle_list(amp_a + 1.6 * amp_b, in_, out, pm), x)) < 1e-13
    h.set_param(1.0)


def test_spmv_matches_map_3x9_sector(h):
    """Full-size sector of the batched workload (173,583 states): SpMV against the map."""
    full, _ = full_lists(3, 9, 2)
    got = h.enumerate_basis(O.mesh_klist(3, 9), (3, 9), 1, 1, (9,), momentum_list=[(1, 4)])
    basis = got[0][1]
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    rng = np.random.default_rng(5)
    x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    y_map = h.matvec(x)
    y32_map = h.matvec(x.astype(np.complex64))
    nnz = h.build_sparse()
    assert nnz >= len(basis)
    y_sp = h.matvec(x)
    assert rel(y_sp, y_map) < 1e-13
    y32_sp = h.matvec(x.astype(np.complex64))
    assert rel(y32_sp.astype(np.complex128), y_map) < 2e-6
    assert rel(y32_map.astype(np.complex128), y_map) < 2e-6
    h.release_sparse()
    assert rel(h.matvec(x), y_map) == 0.0      # back on the map, same kernel, same bits


def test_sparse_eigsolve_vs_lapack(h):
    full, ofull = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[7]
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    h.build_sparse()
    vals, vecs, resid, info = h.eigsolve(10, krylovdim=30, tol=1e-12, seed=1)
    assert info["converged"] >= 10 and np.all(resid < 1e-10)
    H = O.dense_hamiltonian(basis, ofull)
    w, U = np.linalg.eigh(H)
    assert np.max(np.abs(vals - w[:10]) / np.maximum(np.abs(w[:10]), 1.0)) < 1e-10
    for i in range(10):
        cl = np.abs(w - vals[i]) < 1e-6
        assert np.linalg.norm(U[:, cl].conj().T @ vecs[i]) > 1 - 1e-9


def test_edsolve_sparse_dropin_matches_map(h):
    para, _ = mesh_para(4, 3, 5, Nc_conserve=2)
    subs, ks = momed.ED_momentum_subspaces(para, (3, 3), handle=h)
    sub = subs[0]
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    E_sp, v_sp = momed.EDsolve(sub, op, N=8, method="sparse", device="gpu", method_info=False)
    E_map, _ = momed.EDsolve(sub, op, N=8, method="map", device="gpu", method_info=False)
    assert np.max(np.abs(E_sp - E_map) / np.maximum(np.abs(E_map), 1.0)) < 1e-10
    _, ofull = full_lists(4, 3, 5, ncc=2)
    w = np.linalg.eigvalsh(O.dense_hamiltonian(sub.list, ofull))
    assert np.max(np.abs(E_sp - w[:8]) / np.maximum(np.abs(w[:8]), 1.0)) < 1e-10
    assert all(isinstance(v, momed.MBS64Vector) for v in v_sp)


def test_sparse_budget_refusal(h):
    full, _ = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    h.set_basis(ref[0])
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    h.set_hbm_budget(1024)
    try:
        with pytest.raises(momed.MomedError) as e:
            h.build_sparse()
        assert e.value.code == momed._lib.ENOMEM
    finally:
        h.set_hbm_budget(0)
    x = np.ones(len(ref[0]), np.complex128)
    assert np.all(np.isfinite(h.matvec(x)))   # the handle still maps (matrix-free)


def test_batch_solve_on_sparse_entries_matches_map(h):
    """The batched solver's FP32 maps as a block SpMV over the sparse method's entries (A and B
    parts per entry): same eigenvalues as with the matrix-free block map, and LAPACK's."""
    from momed.core import pair_operator
    from momed.synthetic import u_grid
    para, _ = mesh_para(3, 5, 0)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    amp_a, amp_b, in_, out, pm = pair_operator(A, B)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[6]
    h.set_basis(basis)
    h.set_scatter_pair(amp_a, amp_b, in_, out, pm)
    u = u_grid(8, 0.5, 2.0)
    v_map, _, _, _ = h.batch_solve(u, 4, krylovdim=30, tol=1e-12)
    h.build_sparse()
    h.profile(True)
    v_sp, vecs, res, info = h.batch_solve(u, 4, krylovdim=30, tol=1e-12, want_vectors=True)
    n_bsp, _ = h.profile_read(momed._lib.KERNEL_BLOCK_SPMV_C64)
    n_bmv, _ = h.profile_read(momed._lib.KERNEL_BLOCK_MATVEC_C64)
    h.profile(False)
    assert n_bsp > 0 and n_bmv == 0
    assert np.max(np.abs(v_sp - v_map) / np.maximum(np.abs(v_map), 1.0)) < 1e-10
    for q in range(len(u)):
        w = np.linalg.eigvalsh(O.dense_hamiltonian(basis, oracle_list(amp_a + u[q] * amp_b, in_, out, pm)))
        assert np.max(np.abs(v_sp[q] - w[:4]) / np.maximum(np.abs(w[:4]), 1.0)) < 1e-10
    h.release_sparse()


def test_batch_solve_on_sparse_entries_3x9_sector(h):
    """The headline's shape (173,583 states, 32 U0 values, nev 4) on the sparse entries."""
    from momed.core import pair_operator
    from momed.synthetic import u_grid
    para, _ = mesh_para(3, 9, 2)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    got = h.enumerate_basis(O.mesh_klist(3, 9), (3, 9), 1, 1, (9,), momentum_list=[(2, 5)])
    h.set_basis(got[0][1])
    h.set_scatter_pair(*pair_operator(A, B))
    u = u_grid(32, 0.5, 2.0)
    v_map, _, _, _ = h.batch_solve(u, 4, krylovdim=30, tol=1e-10)
    h.build_sparse()
    v_sp, _, res, info = h.batch_solve(u, 4, krylovdim=30, tol=1e-10)
    h.release_sparse()
    assert info["converged"] >= 4
    assert np.max(np.abs(v_sp - v_map) / np.maximum(np.abs(v_map), 1.0)) < 1e-10


def test_batch_solve_single_operator_on_sparse_entries(h):
    full, ofull = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[4]
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    h.build_sparse()
    v, _, _, _ = h.batch_solve(np.array([0.3, 1.0, 2.0, 5.0]), 5, krylovdim=30, tol=1e-12)
    h.release_sparse()
    w = np.linalg.eigvalsh(O.dense_hamiltonian(basis, ofull))
    for q in range(4):                                   # a single operator: every u solves H = A
        assert np.max(np.abs(v[q] - w[:5]) / np.maximum(np.abs(w[:5]), 1.0)) < 1e-10


def test_sparse_subset_basis_drops_absent_targets(h):
    """A basis that is not a whole sector (every other state): targets outside it are dropped as
    index_fit drops them (hilbert_subspace.jl:67-72), in the matrix and in its SpMV."""
    full, ofull = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[3][::2].copy()
    h.set_basis(basis)
    h.set_scatter(full.amp.astype(np.complex128), full.in_, full.out, full.pm)
    h.build_sparse()
    assert_same_matrix(device_csc(h, len(basis)), oracle_csc(basis, ofull))
    x = np.random.default_rng(9).normal(size=len(basis)) + 0.2j
    assert rel(h.matvec(x), O.matvec(basis, ofull, x)) < 1e-13
    h.release_sparse()


def test_uploaded_host_matrix_dropin(h):
    """create_gpu_matrix of a host matrix (the reference's sparse GPU hook receives the CSC that
    SparseHmltMatrix builds): the oracle's CSC uploaded, multiplied and solved on the device."""
    full, ofull = full_lists(3, 5, 0)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[9]
    Hcsc = oracle_csc(basis, ofull)
    G = momed.create_gpu_matrix(Hcsc)
    try:
        x = np.random.default_rng(11).normal(size=len(basis)) + 0.4j
        assert rel(G(x), O.matvec(basis, ofull, x)) < 1e-13
        vals, vecs, info = momed.krylov_matrix_solve(G, 10, krylovdim=30, tol=1e-12, seed=2)
        w = np.linalg.eigvalsh(O.dense_hamiltonian(basis, ofull))
        assert np.max(np.abs(vals - w[:10]) / np.maximum(np.abs(w[:10]), 1.0)) < 1e-10
        with pytest.raises(momed.MomedError) as e:        # no basis: operator calls are refused
            G.handle.stats()
        assert e.value.code == momed._lib.ESTATE
    finally:
        G.release()
    # the Hermitian CSC passed as CSR with conjugated values (what the Julia hook does)
    hd = momed.Handle(0)
    try:
        hd.set_sparse_csr(Hcsc.indptr, Hcsc.indices, np.conj(Hcsc.data))
        assert rel(hd.matvec(x), O.matvec(basis, ofull, x)) < 1e-13
        with pytest.raises(momed.MomedError):
            hd.set_sparse_csr(np.array([0, 1]), np.array([5], np.int32), np.ones(1))   # column out of range
    finally:
        hd.close()
