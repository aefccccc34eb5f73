"""GPU tests of the serving form (continuous-batching solve server).

Bar: a request's eigenvalues are the same alone and in a concurrent mix of uneven
requests (tolerance 1e-12 relative; solves are deterministic, so they agree to the bit in
practice), and they match the one-at-a-time solver within 1e-10 relative.  Failure paths
are exercised on the host: over-budget refusal, cancellation of a queued request, bounded
polls.  Nothing here faults, traps or hangs the GPU.
"""
import os
import time

import numpy as np
import pytest

import oracle as O
import momed
from momed import _lib
from momed.core import pair_operator
from momed.synthetic import mesh_para

pytestmark = pytest.mark.gpu


def pair(a, b, seed):
    para, _ = mesh_para(a, b, seed)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    return pair_operator(A, B)


@pytest.fixture(scope="module")
def workload():
    p35 = pair(3, 5, 0)
    p38 = pair(3, 8, 4)
    b35, _ = O.momentum_subspaces(O.mesh_klist(3, 5), (3, 5), (5,))
    h = momed.Handle(0)
    s38 = h.enumerate_basis(O.mesh_klist(3, 8), (3, 8), 1, 1, (8,), momentum_list=[(0, 1), (2, 3)])
    h.close()
    return p35, p38, b35, [b for _, b in s38]


def wait_all(srv, rids, nev, timeout_s=600):
    out = {}
    t0 = time.time()
    while len(out) < len(rids):
        assert time.time() - t0 < timeout_s, "server did not finish in time"
        for rid in rids:
            if rid in out:
                continue
            st, vals, resid, info, q, lat = srv.poll(rid, nev[rid], wait_ms=50)
            if st == _lib.DONE:
                out[rid] = (vals, resid, info, q, lat)
    return out


def test_same_result_alone_and_in_mix(workload):
    p35, p38, b35, b38 = workload
    srv = _lib.Server(0, slots=4)
    op35 = srv.register_operator(*p35)
    op38 = srv.register_operator(*p38)
    # alone
    rid = srv.submit(op38, b38[0], 1.3, 5, tol=1e-12, seed=7)
    alone = wait_all(srv, [rid], {rid: 5})[rid][0]
    # in a mix of uneven requests that arrive while others run
    rng = np.random.default_rng(0)
    rids, nev = [], {}
    for k in range(10):
        if k == 4:
            r = srv.submit(op38, b38[0], 1.3, 5, tol=1e-12, seed=7)
            target = r
            nev[r] = 5
        else:
            big = rng.random() < 0.4
            basis = b38[k % 2] if big else b35[int(rng.integers(len(b35)))]
            n = int(rng.integers(1, 8))
            r = srv.submit(op38 if big else op35, basis, float(rng.uniform(0.5, 2.0)), n, tol=1e-12, seed=k)
            nev[r] = min(n, len(basis))
        rids.append(r)
        time.sleep(0.01)
    res = wait_all(srv, rids, nev)
    mixed = res[target][0]
    assert np.max(np.abs(mixed - alone) / np.abs(alone)) < 1e-12
    st = srv.stats()
    assert st["completed"] >= 11 and st["failed"] == 0
    srv.stop()
    # against the one-at-a-time solver
    h = momed.Handle(0)
    h.set_basis(b38[0])
    h.set_scatter_pair(*p38)
    h.set_param(1.3)
    v, _, _, _ = h.eigsolve(5, tol=1e-12, seed=7, want_vectors=False)
    h.close()
    assert np.max(np.abs(v - alone) / np.abs(v)) < 1e-10


def test_budget_refusal_and_cancel(workload):
    p35, p38, b35, b38 = workload
    # a budget that admits the small requests but never a large one
    srv = _lib.Server(0, slots=1, hbm_budget=64 << 20)
    op35 = srv.register_operator(*p35)
    op38 = srv.register_operator(*p38)
    big = srv.submit(op38, b38[0], 1.0, 4, krylovdim=120)
    with pytest.raises(momed.MomedError) as ei:
        srv.poll(big, 4)
    assert ei.value.code == _lib.ENOMEM
    first = srv.submit(op35, b35[0], 1.0, 4)
    queued = [srv.submit(op35, b35[i], 1.0, 4) for i in range(1, 4)]
    assert srv.cancel(queued[-1]) in (_lib.OK, _lib.ESTATE)
    st, *_ = srv.poll(first, 4, wait_ms=1)           # bounded poll returns promptly
    res = wait_all(srv, [first] + queued[:-1], {r: 4 for r in [first] + queued})
    assert len(res) == 3
    st, *_ = srv.poll(queued[-1], 4)
    assert st in (_lib.CANCELLED, _lib.DONE)
    srv.stop()


def test_unknown_operator_and_bad_request(workload):
    p35, _, b35, _ = workload
    srv = _lib.Server(0, slots=1)
    with pytest.raises(momed.MomedError):
        srv.submit(99, b35[0], 1.0, 4)
    op = srv.register_operator(*p35)
    with pytest.raises(momed.MomedError):
        srv.submit(op, b35[0], 1.0, 0)          # nev < 1
    srv.stop()


def test_mixed_precision_requests(workload):
    """Mixed-precision requests (batched solver with one right-hand side): the same result alone
    and in a mix with FP64 and other mixed requests, and within 1e-10 of the FP64 solver."""
    p35, p38, b35, b38 = workload
    srv = _lib.Server(0, slots=4)
    op35 = srv.register_operator(*p35)
    op38 = srv.register_operator(*p38)
    rid = srv.submit(op38, b38[1], 0.8, 6, tol=1e-10, seed=3, precision=_lib.PREC_MIXED)
    alone, _, info, _, _ = wait_all(srv, [rid], {rid: 6})[rid]
    assert info["converged"] >= 6
    rids, nev = [], {}
    for k in range(8):
        if k == 3:
            r = srv.submit(op38, b38[1], 0.8, 6, tol=1e-10, seed=3, precision=_lib.PREC_MIXED)
            target, n = r, 6
        else:
            n = 1 + k
            prec = _lib.PREC_MIXED if k % 2 else _lib.PREC_FP64
            r = srv.submit(op35, b35[k], 1.0 + 0.1 * k, n, tol=1e-10, seed=k, precision=prec)
        nev[r] = n
        rids.append(r)
    res = wait_all(srv, rids, nev)
    assert np.max(np.abs(res[target][0] - alone) / np.abs(alone)) < 1e-12
    assert srv.stats()["failed"] == 0
    srv.stop()
    h = momed.Handle(0)
    h.set_scatter_pair(*p38)
    h.set_basis(b38[1])
    h.set_param(0.8)
    v, _, _, _ = h.eigsolve(6, tol=1e-12, seed=1, want_vectors=False)
    h.set_scatter_pair(*p35)
    for r, k in zip(rids, range(8)):
        if k == 3:
            continue
        h.set_basis(b35[k])
        h.set_param(1.0 + 0.1 * k)
        ref, _, _, _ = h.eigsolve(nev[r], tol=1e-12, seed=1, want_vectors=False)
        assert np.max(np.abs(res[r][0] - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-10
    h.close()
    assert np.max(np.abs(v - alone) / np.abs(v)) < 1e-10


def test_queued_requests_on_one_sector_are_batched(workload):
    """Requests queued behind a running one that share its operator, sector and precision are
    solved together (continuous batching): they finish as one group, each with its own u, and
    every result matches the one-at-a-time FP64 solver within 1e-10."""
    p35, p38, b35, b38 = workload
    srv = _lib.Server(0, slots=1)
    op35 = srv.register_operator(*p35)
    op38 = srv.register_operator(*p38)
    blocker = srv.submit(op38, b38[0], 1.0, 6, tol=1e-10)           # keeps the only slot busy
    us = [0.6, 0.9, 1.2, 1.5]
    rids = [srv.submit(op35, b35[2], u, 3, tol=1e-10, precision=_lib.PREC_MIXED) for u in us]
    nev = {r: 3 for r in rids}
    nev[blocker] = 6
    res = wait_all(srv, [blocker] + rids, nev)
    srv.stop()
    infos = [res[r][2] for r in rids]
    assert len({(i["matvecs"], i["seconds"]) for i in infos}) == 1      # one group, one solve
    h = momed.Handle(0)
    h.set_scatter_pair(*p35)
    h.set_basis(b35[2])
    for r, u in zip(rids, us):
        h.set_param(u)
        ref, _, _, _ = h.eigsolve(3, tol=1e-12, seed=1, want_vectors=False)
        assert np.max(np.abs(res[r][0] - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-10
    h.close()


def test_sparse_method_and_map_fallback_by_budget(workload):
    """A 3x8 request (~30k states) is solved over the map's hit cache when it fits the budget, on
    the sparse method when the cache is switched off and the matrix fits, and over the cache's slot
    mode when neither fits (96 MB: ~50 MB for the solve, ~50 MB for a full cache, ~265 MB for the
    matrix, ~14 MB for the slots): the same eigenvalues every way."""
    p35, p38, b35, b38 = workload
    vals = {}
    for budget, knobs in ((8 << 30, {}), (8 << 30, {"MOMED_SERVE_HITCACHE": "0"}), (96 << 20, {})):
        old = {k: os.environ.get(k) for k in knobs}
        os.environ.update(knobs)
        try:
            srv = _lib.Server(0, slots=1, hbm_budget=budget)
            op = srv.register_operator(*p38)
            rid = srv.submit(op, b38[1], 1.1, 4, tol=1e-12, seed=5)
            vals[(budget, tuple(knobs))] = wait_all(srv, [rid], {rid: 4})[rid][0]
            assert srv.stats()["failed"] == 0
            srv.stop()
        finally:
            for k, v in old.items():
                if v is None:
                    del os.environ[k]
                else:
                    os.environ[k] = v
    ref = vals[(96 << 20, ())]
    for v in vals.values():
        assert np.max(np.abs(v - ref) / np.abs(ref)) < 1e-10
