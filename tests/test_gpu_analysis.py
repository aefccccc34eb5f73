"""Analysis of eigenvectors on the device: ED_bracket (EDCore/src/multiplication.jl:153-245)
against the oracle's restatement of mul_add_bracket, within 1e-12 relative."""
import numpy as np
import pytest

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


def as_oracle(lst):
    o = np.zeros(len(lst.amp), O.SCAT_DTYPE)
    o["re"], o["im"], o["out"], o["in"], o["pm"] = lst.amp.real, lst.amp.imag, lst.out, lst.in_, lst.pm
    return o


def relc(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_bracket_same_space_hamiltonian(h):
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    space = core.HilbertSubspace(ref[4])
    rng = np.random.default_rng(0)
    x = rng.normal(size=len(space)) + 1j * rng.normal(size=len(space))
    y = rng.normal(size=len(space)) + 1j * rng.normal(size=len(space))
    got = momed.ED_bracket(core.MBS64Vector(y, space), op, core.MBS64Vector(x, space), handle=h)
    want = O.bracket(ref[4], y, ref[4], x, as_oracle(op.scats), upper=True)
    assert relc(got, want) < 1e-12
    assert relc(got, np.vdot(y, O.matvec(ref[4], as_oracle(core.hermitian_complete(op)), x))) < 1e-12


def test_bracket_across_momentum_sectors(h):
    """rho_q = sum_k c+_{k+q} c_k moves a state from sector K to K + q: bra and ket on different
    subspaces, targets outside the bra space dropped."""
    a, b = 3, 5
    kl = O.mesh_klist(a, b)
    Nk = a * b
    q = (1, 2)
    amp, out, inn = [], [], []
    for k in range(Nk):
        kq = ((kl[0, k] + q[0]) % a) + a * ((kl[1, k] + q[1]) % b)
        amp.append(1.0 + 0.1j * k)
        out.append(1 << int(kq))
        inn.append(1 << k)
    lst = core.ScatterList(np.array(amp), np.array(out, np.uint64), np.array(inn, np.uint64))
    op = momed.MBOperator(lst, upper_hermitian=False)
    ref, ks = O.momentum_subspaces(kl, (a, b), (5,))
    ks = [tuple(int(v) for v in k) for k in np.asarray(ks).reshape(len(ref), -1)]
    iK = 3
    K = ks[iK]
    target = ((K[0] + q[0]) % a, (K[1] + q[1]) % b)
    iB = ks.index(target)
    rng = np.random.default_rng(1)
    ket = rng.normal(size=len(ref[iK])) + 1j * rng.normal(size=len(ref[iK]))
    bra = rng.normal(size=len(ref[iB])) + 1j * rng.normal(size=len(ref[iB]))
    got = momed.ED_bracket(core.MBS64Vector(bra, core.HilbertSubspace(ref[iB])), op,
                           core.MBS64Vector(ket, core.HilbertSubspace(ref[iK])), handle=h)
    want = O.bracket(ref[iB], bra, ref[iK], ket, as_oracle(op.scats), upper=False)
    assert abs(want) > 1e-6
    assert relc(got, want) < 1e-12
    # a bra in the ket's own sector sees nothing: every target leaves it
    self_b = rng.normal(size=len(ref[iK])) + 0j
    got0 = momed.ED_bracket(core.MBS64Vector(self_b, core.HilbertSubspace(ref[iK])), op,
                            core.MBS64Vector(ket, core.HilbertSubspace(ref[iK])), handle=h)
    assert abs(got0) < 1e-12


def test_bracket_expectation_of_eigenvector(h):
    """<psi| H |psi> of a computed eigenvector equals its eigenvalue."""
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    subs, _ = momed.ED_momentum_subspaces(para, (5,), handle=h)
    E, vecs = momed.EDsolve(subs[1], op, N=3, method="map", device="gpu", method_info=False)
    for e, v in zip(E, vecs):
        val = momed.ED_bracket(v, op, v, handle=h)
        assert abs(val.imag) < 1e-10 and abs(val.real - e) / abs(e) < 1e-10


def test_rdm1_matches_oracle_across_sectors(h):
    """PES_1rdm on a basis that holds every momentum sector (c+_i c_j moves between them, so the
    matrix has off-diagonal entries) and on one sector (diagonal: the occupations)."""
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    union = np.sort(np.concatenate(ref))
    rng = np.random.default_rng(2)
    psi = rng.normal(size=len(union)) + 1j * rng.normal(size=len(union))
    psi /= np.linalg.norm(psi)
    got = momed.PES_1rdm(core.MBS64Vector(psi, core.HilbertSubspace(union, 15)), handle=h)
    want = O.rdm1(union, psi, 15)
    assert np.max(np.abs(got - want)) < 1e-12
    assert np.max(np.abs(want - np.diag(np.diag(want)))) > 1e-3          # off-diagonal entries present
    assert abs(np.trace(got) - 5) < 1e-12
    one = ref[6]
    phi = rng.normal(size=len(one)) + 1j * rng.normal(size=len(one))
    phi /= np.linalg.norm(phi)
    got1 = momed.PES_1rdm(core.MBS64Vector(phi, core.HilbertSubspace(one, 15)), handle=h)
    assert np.max(np.abs(got1 - O.rdm1(one, phi, 15))) < 1e-12


def test_rdm1_two_component_eigenvector(h):
    """Two conserved components (48 orbitals at 4x6; here 4x3, 24 orbitals): the matrix of a
    computed eigenvector against the oracle."""
    para, _ = mesh_para(4, 3, 5, Nc_conserve=2)
    subs, _ = momed.ED_momentum_subspaces(para, (3, 3), handle=h)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    E, vecs = momed.EDsolve(subs[0], op, N=2, method="map", device="gpu", method_info=False)
    bits = subs[0].bits
    got = momed.PES_1rdm(vecs[0], handle=h)
    want = O.rdm1(subs[0].list, vecs[0].vec, bits)
    assert got.shape == (bits, bits)
    assert np.max(np.abs(got - want)) < 1e-12
    assert abs(np.trace(got).real - 6) < 1e-9


@pytest.mark.parametrize("g", [1, 3])
def test_step_inner_prod_matches_oracle(h, g):
    """ED_step_inner_prod (manybody_quantum_geometry.jl:48-94), Abelian (g = 1) and non-Abelian."""
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    basis = ref[5]
    space = core.HilbertSubspace(basis, 15)
    rng = np.random.default_rng(g)
    f = rng.normal(size=(g, len(basis))) + 1j * rng.normal(size=(g, len(basis)))
    i = rng.normal(size=(g, len(basis))) + 1j * rng.normal(size=(g, len(basis)))
    orb = np.exp(1j * rng.uniform(0, 2 * np.pi, 15)) * rng.uniform(0.9, 1.0, 15)
    want = O.step_inner_prod(basis, f, i, orb)
    if g == 1:
        got = momed.ED_step_inner_prod(core.MBS64Vector(f[0], space), core.MBS64Vector(i[0], space), orb, handle=h)
        assert abs(got - want[0, 0]) < 1e-12 * abs(want[0, 0])
    else:
        got = momed.ED_step_inner_prod([core.MBS64Vector(v, space) for v in f],
                                       [core.MBS64Vector(v, space) for v in i], orb, handle=h)
        assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))


def test_adjoint_map_of_non_hermitian_operator(h):
    """A non-Hermitian operator (the upper two-body list taken as it is): the device map and its
    adjoint satisfy <y, A x> = <A^H y, x>, and A^H y matches the oracle map of the adjoint terms."""
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=False)
    ref, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    space = core.HilbertSubspace(ref[8], 15)
    M = momed.create_gpu_linearmap(momed.LinearMap(op, space))
    Madj = M.adjoint()
    try:
        assert Madj is not M
        rng = np.random.default_rng(4)
        x = rng.normal(size=len(space)) + 1j * rng.normal(size=len(space))
        y = rng.normal(size=len(space)) + 1j * rng.normal(size=len(space))
        ax, ay = M(x), Madj(y)
        assert relc(np.vdot(y, ax), np.vdot(ay, x)) < 1e-12
        from momed.methods import adjoint_list
        assert np.max(np.abs(ay - O.matvec(ref[8], as_oracle(adjoint_list(op.scats)), y))) < 1e-12 * np.max(np.abs(ay))
        assert np.max(np.abs(ax - O.matvec(ref[8], as_oracle(op.scats), x))) < 1e-12 * np.max(np.abs(ax))
        # the adjoint of a Hermitian-completed operator is the map itself
        H = momed.create_gpu_linearmap(momed.LinearMap(momed.MBOperator(
            momed.ED_scatterlist_twobody(para), upper_hermitian=True), space))
        assert H.adjoint() is H
        H.release()
    finally:
        Madj.release()
        M.release()


def test_two_operator_bracket(h):
    """<bra| op2 op1 |ket> (multiplication.jl:174-190, 215-222) through unrestricted intermediate
    states: the density-density correlation <psi| rho_-q rho_q |psi> (intermediate sector K + q)
    and <y| H H |x> = <H y, H x>, against the oracle."""
    a, b = 3, 5
    kl = O.mesh_klist(a, b)
    q = (1, 2)

    def rho(qx, qy):
        amp, out, inn = [], [], []
        for k in range(a * b):
            kq = ((kl[0, k] + qx) % a) + a * ((kl[1, k] + qy) % b)
            amp.append(1.0)
            out.append(1 << int(kq))
            inn.append(1 << k)
        return momed.MBOperator(core.ScatterList(np.array(amp, complex), np.array(out, np.uint64),
                                                 np.array(inn, np.uint64)), upper_hermitian=False)

    r_q, r_mq = rho(*q), rho(-q[0], -q[1])
    ref, _ = O.momentum_subspaces(kl, (a, b), (5,))
    space = core.HilbertSubspace(ref[2], 15)
    rng = np.random.default_rng(7)
    psi = rng.normal(size=len(space)) + 1j * rng.normal(size=len(space))
    v = core.MBS64Vector(psi, space)
    got = momed.ED_bracket(v, r_mq, r_q, v, handle=h)
    want = O.bracket2(ref[2], psi, ref[2], psi, as_oracle(r_mq.scats), as_oracle(r_q.scats))
    assert abs(want) > 1e-6 and relc(got, want) < 1e-12
    para, _ = mesh_para(3, 5, 0)
    H = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                         upper_hermitian=True)
    full = as_oracle(core.hermitian_complete(H))
    y = core.MBS64Vector(rng.normal(size=len(space)) + 0.5j, space)
    got2 = momed.ED_bracket(y, H, H, v, handle=h)
    assert relc(got2, np.vdot(O.matvec(ref[2], full, y.vec), O.matvec(ref[2], full, psi))) < 1e-12
