"""Pin the oracle to the reference's own known answers (EDCore unit tests).

Every case comes from tests/golden/edcore_known_answers.json, which cites the
reference test line it transcribes.  A failure here means the oracle no longer
restates the reference's conventions (bit layout, colex order, fermionic sign,
Scatter normal ordering, sort/merge, operator application).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "edcore_known_answers.json")))


def occ_to_mask(occ):
    m = 0
    for i in occ:
        m |= 1 << (i - 1)
    return m


@pytest.mark.parametrize("case", GOLD["scat_occ_number"], ids=lambda c: c["cite"])
def test_scat_occ_number(case):
    assert O.scat_occ_number_tuple(case["n"], case["orbitals"], case["bits"]) == case["expect"]
    # the mask form (manybodystate_basis.jl:397) agrees with the tuple form for pairs
    assert O.scat_occ_number(case["n"], occ_to_mask(case["orbitals"])) == case["expect"]


def test_mbs_ops():
    c = GOLD["mbs_ops"]
    assert (c[0]["hi"] << c[0]["lo_bits"]) | c[0]["lo"] == c[0]["expect"]
    assert c[1]["a"] | c[1]["b"] == c[1]["expect"]
    assert occ_to_mask(c[2]["occ"]) == c[2]["n"]
    assert c[3]["n"] ^ occ_to_mask(c[3]["flip"]) == c[3]["expect"]


@pytest.mark.parametrize("case", GOLD["colex"], ids=lambda c: c["cite"])
def test_colex(case):
    got = O.colex(case["n"], case["t"])
    if "expect_occ" in case:
        assert [int(v) for v in got] == [occ_to_mask(o) for o in case["expect_occ"]]
    if "expect_len" in case:
        assert len(got) == case["expect_len"] == O.binomial(case["n"], case["t"])
    if case.get("expect_sorted"):
        assert np.all(np.diff(got.astype(np.int64)) > 0)


@pytest.mark.parametrize("case", GOLD["colex_mask"], ids=lambda c: c["cite"])
def test_colex_mask(case):
    got = O.colex(case["n"], case["t"], mask=case["mask"])
    if "expect_occ" in case:
        assert [int(v) for v in got] == [occ_to_mask(o) for o in case["expect_occ"]]
    if "expect_len" in case:
        assert len(got) == case["expect_len"]
    if case.get("expect_sorted"):
        assert np.all(np.diff(got.astype(np.int64)) > 0)


def test_colex_chunks_concatenate():
    # unrank_colex chunk starts (colex_mbslist.jl:2-21) reproduce the full iteration
    full = O.colex(12, 5)
    parts = [O.colex(12, 5, s, e) for s, e in ((1, 100), (101, 500), (501, 792))]
    assert np.array_equal(np.concatenate(parts), full)


@pytest.mark.parametrize("case", GOLD["scatter"], ids=lambda c: c["cite"])
def test_scatter_normal_ordering(case):
    s = O.scatter(complex(*case["V"]), *case["out_in"], upper_hermitian=case["upper"])[0]
    assert int(s["out"]) == occ_to_mask(case["expect_out"])
    assert int(s["in"]) == occ_to_mask(case["expect_in"])
    assert (s["re"], s["im"]) == tuple(case["expect_amp"])
    assert int(s["pm"]) == O.parity_mask(int(s["out"])) ^ O.parity_mask(int(s["in"]))


def test_adjoint_and_diagonal():
    s1 = O.scatter(1.0, 1, 2)[0]
    s3 = O.scatter(1.0, 2, 1)[0]
    adj = O.hermitian_complete(np.array([s1]))
    assert any(int(t["out"]) == int(s3["out"]) and int(t["in"]) == int(s3["in"]) for t in adj)
    d = O.scatter(1.0, 1, 1)[0]
    assert int(d["in"]) == int(d["out"])


def test_generic_nbody_matches_twobody():
    # the generic constructor (scattering.jl:63-100) agrees with the 2-body one (121-153)
    rng = np.random.default_rng(0)
    for _ in range(200):
        i1, i2, j2, j1 = (int(v) for v in rng.choice(np.arange(1, 20), 4, replace=False))
        V = complex(rng.normal(), rng.normal())
        for up in (False, True):
            a = O.scatter(V, i1, i2, j2, j1, upper_hermitian=up)[0]
            b = np.zeros(1, O.SCAT_DTYPE)
            import ctypes as C
            arr = np.array([i1, i2, j2, j1], np.int64)
            rec = O._Scat()
            O.lib().or_scatter_n(V.real, V.imag, arr.ctypes.data_as(C.c_void_p), 4, int(up), C.byref(rec))
            assert (rec.re, rec.im, rec.out, rec.in_, rec.pm) == tuple(a.tolist())


@pytest.mark.parametrize("case", GOLD["sort_merge"], ids=lambda c: c["cite"])
def test_sort_merge(case):
    terms = np.concatenate([O.scatter(complex(*t["V"]), *t["out_in"], upper_hermitian=t.get("upper", False))
                            for t in case["terms"]])
    if case.get("expect_error"):
        with pytest.raises(AssertionError):
            O.sort_merge(terms, check_upper=case["check_upper"])
        return
    m = O.sort_merge(terms, check_upper=case["check_upper"])
    assert len(m) == case["expect_len"]
    if "expect_amp0" in case:
        assert (m[0]["re"], m[0]["im"]) == tuple(case["expect_amp0"])
    if case.get("expect_sorted"):
        assert (int(m[0]["in"]), int(m[0]["out"])) < (int(m[1]["in"]), int(m[1]["out"]))


@pytest.mark.parametrize("case", GOLD["scatter_apply"], ids=lambda c: c["cite"])
def test_scatter_apply(case):
    s = O.scatter(complex(*case["V"]), *case["out_in"])
    amp, st = O.scat_apply(s, occ_to_mask(case["state_occ"]))
    assert amp == complex(*case["expect_amp"])
    assert st == occ_to_mask(case["expect_state_occ"])
    # mbs_out * scat inverts it (multiplication.jl:51)
    amp2, st2 = O.scat_apply(s, st, right=True)
    assert amp2 == amp and st2 == occ_to_mask(case["state_occ"])


@pytest.mark.parametrize("case", GOLD["operator_matvec"], ids=lambda c: c["cite"])
def test_operator_matvec(case):
    terms = np.concatenate([O.scatter(complex(*t["V"]), *t["out_in"], upper_hermitian=t.get("upper", False))
                            for t in case["terms"]])
    merged = O.sort_merge(terms, check_upper=case["upper"])
    full = O.hermitian_complete(merged) if case["upper"] else merged
    basis = np.array([occ_to_mask(o) for o in case["basis_occ"]], np.uint64)
    for c in case["cases"]:
        x = np.zeros(len(basis), np.complex128)
        x[c["x_at"]] = 1.0
        y = O.matvec(basis, full, x)
        for idx, val in c["expect"].items():
            assert abs(y[int(idx)] - complex(*val)) < 1e-14


@pytest.mark.parametrize("case", GOLD["subspace_search"], ids=lambda c: c["cite"])
def test_subspace_search(case):
    lst = np.array(case["list"], np.uint64)
    j = int(np.searchsorted(lst, case["query"], side="left"))     # searchsortedfirst, 0-based
    if "expect_index1" in case:
        assert j + 1 == case["expect_index1"]
    if "expect_fit" in case:
        fit = j < len(lst) and int(lst[j]) == case["query"]
        assert fit == case["expect_fit"]


def test_parity_mask_julia_shift_semantics():
    # odd bit count: the trailing (1 << 64) term is 0 in Julia (scattering.jl:14)
    assert O.parity_mask(1 << 3) == (~((1 << 4) - 1)) & (2**64 - 1)
    assert O.parity_mask(1 << 63) == 0
    assert O.parity_mask((1 << 1) | (1 << 5)) == 0b011100
    assert O.parity_mask(0) == 0


def test_sparse_csc_restatement_matches_dense():
    """The oracle's restatement of the sparse method's matrix builder (sparse_matrix.jl:64-190)
    against its row-oriented dense builder: same matrix, rows sorted and unique per column."""
    S = O.Synth(3, 5, 0)
    full = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    sectors, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    for basis in sectors[::5]:
        cp, rv, nz = O.sparse_csc(basis, full)
        D = O.dense_hamiltonian(basis, full)
        N = len(basis)
        M = np.zeros((N, N), np.complex128)
        for j in range(N):
            seg = rv[cp[j]:cp[j + 1]]
            assert np.all(np.diff(seg) > 0)
            M[seg, j] = nz[cp[j]:cp[j + 1]]
        assert np.array_equal(M, D)
        assert len(nz) == np.count_nonzero(D)


def test_bracket_restatement_forms_agree():
    """mul_add_bracket with the upper_hermitian list (multiplication.jl:153-173) equals the bracket
    with the completed list and the dot product with the oracle map."""
    S = O.Synth(3, 5, 0)
    upper = O.sort_merge(np.concatenate([S.onebody(), S.twobody()]))
    full = O.hermitian_complete(upper)
    sectors, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    b = sectors[2]
    rng = np.random.default_rng(0)
    x = rng.normal(size=len(b)) + 1j * rng.normal(size=len(b))
    y = rng.normal(size=len(b)) + 1j * rng.normal(size=len(b))
    v_up = O.bracket(b, y, b, x, upper, upper=True)
    v_full = O.bracket(b, y, b, x, full, upper=False)
    v_map = np.vdot(y, O.matvec(b, full, x))
    assert abs(v_up - v_map) < 1e-12 * abs(v_map)
    assert abs(v_full - v_map) < 1e-12 * abs(v_map)


def test_rdm1_restatement_properties():
    """PES_1rdm restated (particle_reduced_density_matrix.jl:4-33): Hermitian, trace = electrons,
    diagonal = occupations, and within one momentum sector (one component) diagonal."""
    sectors, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    b = sectors[0]
    rng = np.random.default_rng(0)
    x = rng.normal(size=len(b)) + 1j * rng.normal(size=len(b))
    x /= np.linalg.norm(x)
    R = O.rdm1(b, x, 15)
    occ = np.array([[(int(s) >> i) & 1 for i in range(15)] for s in b])
    assert np.allclose(R, R.conj().T)
    assert abs(np.trace(R) - 5) < 1e-12
    assert np.allclose(np.diag(R).real, (np.abs(x) ** 2) @ occ)
    assert np.max(np.abs(R - np.diag(np.diag(R)))) == 0.0


def test_step_inner_prod_restatement_matches_numpy():
    """ED_step_inner_prod restated (manybody_quantum_geometry.jl:48-94) against a direct numpy
    evaluation of sum_x conj(f[j][x]) i[k][x] prod_{occupied o} orb[o]."""
    sectors, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    b = sectors[3]
    rng = np.random.default_rng(5)
    g = 2
    f = rng.normal(size=(g, len(b))) + 1j * rng.normal(size=(g, len(b)))
    i = rng.normal(size=(g, len(b))) + 1j * rng.normal(size=(g, len(b)))
    orb = np.exp(1j * rng.uniform(0, 2 * np.pi, 15))
    occ = np.array([[(int(s) >> o) & 1 for o in range(15)] for s in b], bool)
    prod = np.array([np.prod(orb[row]) for row in occ])
    want = np.einsum("jx,kx,x->jk", f.conj(), i, prod)
    got = O.step_inner_prod(b, f, i, orb)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
