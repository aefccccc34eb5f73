"""CPU tests of the host-side mirror of the reference API (no GPU needed).

The Python host builds scatter lists, merges and completes operators exactly as
the reference does; these tests hold it bit-exact to the oracle's C restatement
and to the reference's own known answers, and check that the C-ABI library
exports every entry point include/momed.h declares.
"""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import momed
from momed import core
from momed.synthetic import mesh_para

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "edcore_known_answers.json")))


def same_bits(sl, o):
    return (len(sl) == len(o) and np.array_equal(sl.out, o["out"]) and np.array_equal(sl.in_, o["in"])
            and np.array_equal(sl.pm, o["pm"])
            and np.array_equal(sl.amp.real.astype(np.float64).view(np.uint64), o["re"].view(np.uint64))
            and np.array_equal(sl.amp.imag.astype(np.float64).view(np.uint64), o["im"].view(np.uint64)))


@pytest.mark.parametrize("a,b,seed,ncc", [(3, 5, 0, 1), (3, 4, 7, 1), (2, 3, 3, 2), (4, 3, 11, 2)])
@pytest.mark.parametrize("prec", [64, 32])
def test_builders_bit_exact(a, b, seed, ncc, prec):
    para, mh = mesh_para(a, b, seed, Nc_conserve=ncc)
    et = np.float32 if prec == 32 else np.float64
    h1 = momed.ED_scatterlist_onebody(para, element_type=et)
    h2 = momed.ED_scatterlist_twobody(para, element_type=et)
    S = O.Synth(a, b, seed, Nc_conserve=ncc)
    assert same_bits(h1, S.onebody(prec))
    assert same_bits(h2, S.twobody(prec))


def test_builders_user_callable_vs_oracle():
    # an arbitrary index-mode H_two through both builders
    def H2(kf1, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1):
        return complex(np.sin(kf1 + 2 * kf2) - ki1 * 0.25, np.cos(ki2 * kf1) * 0.5) * (1 + 0.1 * (cf1 + ci1))

    def H1(k, cf, ci):
        return complex(0.3 * k, 0.1 * (cf - ci))

    kl = O.mesh_klist(3, 3)
    para = momed.EDPara(k_list=kl, Gk=(3, 3), Nc_mix=2, Nc_conserve=1, H_one=H1, H_two=H2,
                        one_momentum_coordinate=False, two_momentum_coordinate=False)
    assert same_bits(momed.ED_scatterlist_twobody(para), O.scatterlist_twobody(kl, (3, 3), H2, Nc_mix=2))
    assert same_bits(momed.ED_scatterlist_onebody(para), O.scatterlist_onebody(kl, (3, 3), H1, Nc_mix=2))


def test_hermitian_complete_matches_oracle():
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), momed.ED_scatterlist_twobody(para),
                          upper_hermitian=True)
    full = core.hermitian_complete(op)
    S = O.Synth(3, 5, 0)
    ofull = O.hermitian_complete(O.sort_merge(np.concatenate([S.onebody(), S.twobody()])))
    assert same_bits(full, ofull)


@pytest.mark.parametrize("case", GOLD["scatter"], ids=lambda c: c["cite"])
def test_scatter_known_answers(case):
    s = momed.Scatter(complex(*case["V"]), *case["out_in"], bits=10, upper_hermitian=case["upper"])
    assert s.out == momed.make_mask64(case["expect_out"])
    assert s.in_ == momed.make_mask64(case["expect_in"])
    assert (s.Amp.real, s.Amp.imag) == tuple(case["expect_amp"])


@pytest.mark.parametrize("case", GOLD["scatter_apply"], ids=lambda c: c["cite"])
def test_scatter_apply_known_answers(case):
    s = momed.Scatter(complex(*case["V"]), *case["out_in"], bits=4)
    amp, st = s.apply(momed.make_mask64(case["state_occ"]))
    assert amp == complex(*case["expect_amp"]) and st == momed.make_mask64(case["expect_state_occ"])


def test_sort_merge_known_answers():
    s1 = momed.Scatter(1.0, 1, 2, bits=10)
    s2 = momed.Scatter(2.0, 1, 2, bits=10)
    s3 = momed.Scatter(1.0, 2, 1, bits=10)
    s4 = momed.Scatter(1.0, 1, 1, bits=10, upper_hermitian=True)
    m = momed.sort_merge_scatlist([s1, s2], check_upper=False)
    assert len(m) == 1 and m[0].Amp == 3.0
    m = momed.sort_merge_scatlist([s1, s3], check_upper=False)
    assert len(m) == 2 and m[0] < m[1]
    with pytest.raises(AssertionError):
        momed.sort_merge_scatlist([s3], check_upper=True)
    assert len(momed.sort_merge_scatlist([s4], check_upper=True)) == 1


def test_generic_nbody_scatter_matches_oracle():
    rng = np.random.default_rng(1)
    for _ in range(100):
        orbs = [int(v) for v in rng.choice(np.arange(1, 30), 6, replace=False)]
        V = complex(rng.normal(), rng.normal())
        for up in (False, True):
            s = momed.Scatter(V, *orbs, bits=30, upper_hermitian=up)
            o = O.scatter(V, *orbs, upper_hermitian=up)[0]
            assert (s.Amp.real, s.Amp.imag, s.out, s.in_, s.parity_mask) == \
                   (o["re"], o["im"], int(o["out"]), int(o["in"]), int(o["pm"]))


def test_parity_mask_matches_oracle():
    rng = np.random.default_rng(2)
    for _ in range(500):
        occ = int(rng.integers(0, 2**63)) | (int(rng.integers(0, 2)) << 63)
        assert momed.parity_mask(occ) == O.parity_mask(occ)


def test_hilbert_subspace_search():
    sp = momed.HilbertSubspace(np.arange(5, dtype=np.uint64), bits=8)
    assert sp.get(2) == 3
    assert not momed.index_fit(sp.get(5), sp, 5)


def test_momentum_and_pairs():
    para, _ = mesh_para(3, 5, 0)
    groups = momed.group_momentum_pairs(para)
    assert sum(len(v) for v in groups.values()) == 15 * 16 // 2
    for K, pairs in groups.items():
        for (i, j) in pairs:
            assert momed.MBS_totalmomentum(para, (i, j)) == K


def test_library_exports_every_declared_symbol():
    """libmomed_b200.so loads without a GPU and exports each function include/momed.h declares."""
    from momed import _lib
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "momentumed.jl_b200")], check=True)
    header = open(os.path.join(ROOT, "include", "momed.h")).read()
    declared = set(re.findall(r"\b(momed_[a-z_0-9]+)\s*\(", header))
    assert declared, "no declarations parsed"
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"
    assert set(_lib.SIGNATURES) == declared
    assert lib.momed_version
    v = ctypes.CDLL(_lib.LIB_PATH)
    v.momed_version.restype = ctypes.c_char_p
    assert b"sm_100a" in v.momed_version()


def test_no_device_fails_loudly():
    """Without a CUDA device the product path raises instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(momed.MomedError):
        momed.Handle(0)


def test_serving_stream_is_seeded_poisson():
    """The serving stream: seeded, arrivals increasing at about 50/s, fields in their ranges."""
    from momed.synthetic import SERVE_MESHES, serve_requests
    counts = {"3x5": 15, "3x9": 27, "3x10": 30, "4x9": 36}
    meshes = list(SERVE_MESHES)
    a = serve_requests(2000, meshes, counts)
    b = serve_requests(2000, meshes, counts)
    assert a == b
    t = np.array([r["arrival"] for r in a])
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 50.0) < 5.0
    assert {r["mesh"] for r in a} == set(meshes)
    assert all(0 <= r["sector"] < counts[r["mesh"]] for r in a)
    assert all(1 <= r["nev"] <= 20 and 0.5 <= r["u"] <= 2.0 and r["tol"] == 1e-10 for r in a)
    assert serve_requests(5, meshes, counts, seed=5) != a[:5]


def test_connection_gaugefixing_host():
    """ED_connection_gaugefixing (manybody_quantum_geometry.jl:14-45): the suggested element (one
    vector) or the determinant of the suggested elements (g vectors) becomes real and positive."""
    import momed
    from momed import core
    space = core.HilbertSubspace(np.arange(1, 9, dtype=np.uint64), 4)
    rng = np.random.default_rng(0)
    v = core.MBS64Vector(rng.normal(size=8) + 1j * rng.normal(size=8), space)
    momed.ED_connection_gaugefixing(v, 3)
    assert abs(v.vec[2].imag) < 1e-14 and v.vec[2].real > 0
    vs = [core.MBS64Vector(rng.normal(size=8) + 1j * rng.normal(size=8), space) for _ in range(2)]
    momed.ED_connection_gaugefixing(vs, [2, 5])
    d = np.linalg.det(np.array([[w.vec[i - 1] for w in vs] for i in (2, 5)]))
    assert abs(d.imag) < 1e-12 and d.real > 0


def test_analysis_input_checks_on_host():
    """ED_step_inner_prod refuses mismatched subspaces, vector counts and orbital-overlap lengths
    before touching a device (the reference's @assert lines, manybody_quantum_geometry.jl:52-53,
    67-71)."""
    import momed
    from momed import core
    s1 = core.HilbertSubspace(np.array([3, 5, 6], np.uint64), 3)
    s2 = core.HilbertSubspace(np.array([3, 5], np.uint64), 3)
    v1 = core.MBS64Vector(np.ones(3, complex), s1)
    v2 = core.MBS64Vector(np.ones(2, complex), s2)
    with pytest.raises(AssertionError):
        momed.ED_step_inner_prod(v1, v2, np.ones(3))
    with pytest.raises(AssertionError):
        momed.ED_step_inner_prod(v1, v1, np.ones(4))
    with pytest.raises(AssertionError):
        momed.ED_step_inner_prod([v1, v1], [v1], np.ones(3))
    with pytest.raises(AssertionError):
        momed.ED_connection_gaugefixing([v1, v1], [1])


def test_edsolve_method_checks_on_host():
    """EDsolve's argument checks (MomentumED.jl:381-387) and the methods this backend leaves to
    the reference (dense, CPU) fail before any device work."""
    import momed
    from momed import core
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    space = core.HilbertSubspace(np.array([31], np.uint64), 15)
    with pytest.raises(AssertionError):
        momed.EDsolve(space, op, N=1, method="lanczos")
    with pytest.raises(AssertionError):
        momed.EDsolve(space, op, N=0)
    with pytest.raises(NotImplementedError):
        momed.EDsolve(space, op, N=1, method="dense", device="gpu")
    with pytest.raises(NotImplementedError):
        momed.EDsolve(space, op, N=1, method="sparse", device="cpu")


def test_forward_images_host():
    """The intermediate states of the two-operator bracket: every state one term reaches from the
    ket space (scat * mbs_in, multiplication.jl:20-34), against a brute-force application."""
    from momed.analysis import forward_images
    from momed import core
    para, _ = mesh_para(3, 5, 0)
    op = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    lst = core.hermitian_complete(op)
    sectors, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    states = sectors[1]
    want = set()
    for s in (int(v) for v in states):
        for i_m, o_m in zip(lst.in_.tolist(), lst.out.tolist()):
            if s & i_m != i_m:
                continue
            mid = s & ~i_m
            if mid & o_m:
                continue
            want.add(mid | o_m)
    got = forward_images(states, lst)
    assert list(got) == sorted(want)
    assert np.all(np.diff(got.astype(np.float64)) > 0)
    # a momentum-conserving operator keeps the sector: the images are the sector's own states
    assert set(got.tolist()) <= set(int(v) for v in states)
