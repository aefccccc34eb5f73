"""The batching form's launch machinery: captured CUDA graphs and the block-map autotuner.

The batched solver replays each restart cycle after the first from a captured CUDA graph
(MOMED_GRAPHS=0 launches every kernel one by one); the block map's launch (rows per warp, grid)
is chosen by timing candidates at the first launch of each (operator, sector size class, block
width, precision) and reported by momed_block_tuning (MOMED_AUTOTUNE=0 keeps the default).
Both change only how the same kernels are launched (each row is still computed by one warp with
the same instruction sequence); results agree to rounding (the Gram-Schmidt norms are summed with
atomics, whose order is not fixed).
"""
import os
from contextlib import contextmanager

import numpy as np
import pytest

import momed
from momed import _lib
from momed.core import pair_operator
from momed.synthetic import mesh_para, u_grid

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


@pytest.fixture(scope="module")
def h3x8():
    para, _ = mesh_para(3, 8, 5)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    h = momed.Handle(0)
    secs = h.enumerate_basis(para.k_list, para.Gk, 1, 1, (8,))
    h.set_scatter_pair(*pair_operator(A, B))
    h.select_sector(3, len(secs[3][1]))
    yield h
    h.close()


def test_graph_replay_matches_eager_launches(h3x8):
    u = u_grid(8, 0.5, 2.0)
    with env(MOMED_GRAPHS=0):
        v0, _, r0, i0 = h3x8.batch_solve(u, 4, krylovdim=30, tol=1e-12, precision=_lib.PREC_MIXED)
    v1, _, r1, i1 = h3x8.batch_solve(u, 4, krylovdim=30, tol=1e-12, precision=_lib.PREC_MIXED)
    assert i1["restarts"] >= 1                         # cycles after the first ran as graph replays
    # the norms of the Gram-Schmidt update are summed with atomics (order not fixed), so two runs
    # agree to rounding, graphs or not
    assert np.max(np.abs(v0 - v1) / np.abs(v0)) < 1e-12
    # a convergence test that sits at its threshold can take one restart cycle more or less
    assert abs(i0["restarts"] - i1["restarts"]) <= 1


def test_autotuner_records_a_choice(h3x8):
    """The tuner times the candidate block map (the map over a hit cache has no tuned launch)."""
    u = u_grid(4, 0.5, 2.0)
    h3x8.release_hit_cache()
    with env(MOMED_HITCACHE=0):
        h3x8.batch_solve(u, 2, krylovdim=20, tol=1e-10, precision=_lib.PREC_MIXED)
    t = h3x8.block_tuning(4, _lib.PREC_MIXED, True)
    assert t is not None
    assert t["rows_per_warp"] in (1, 2, 4) and t["grid"] in ("resident-1", "resident", "2x resident")
    assert 0 < t["ms"] <= t["ms_default"] * 1.0001    # the default launch is one of the candidates
