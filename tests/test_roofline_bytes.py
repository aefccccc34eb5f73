"""The algorithmic bytes behind the bench line's roofline, recomputed on the CPU for the headline
workload (3x9 mesh, Ne = 9, the 173,583-state sectors, 32 right-hand sides, c64): the per-launch
figures of the block map over the hit cache (10.19 GB: row metadata, x and y, one 8-byte record
and one 256-byte x-row gather per off-diagonal hit, the amplitude tables) and of the candidate
block map (11.88 GB: one gather per (row, term) hit), from the oracle's hit counts of the same
operator, so the formulas the bench divides by its CUDA-event times are pinned to the counts."""
import numpy as np

import bench
import oracle as O
import momed
from momed.core import pair_operator
from momed.synthetic import mesh_para


def test_headline_algorithmic_bytes():
    para, _ = mesh_para(3, 9, 2)
    A = momed.MBOperator(momed.ED_scatterlist_onebody(para), upper_hermitian=True)
    B = momed.MBOperator(momed.ED_scatterlist_twobody(para), upper_hermitian=True)
    amp_a, amp_b, in_, out, pm = pair_operator(A, B)
    amp = amp_a + amp_b
    o = np.zeros(len(amp), O.SCAT_DTYPE)
    o["re"], o["im"], o["out"], o["in"], o["pm"] = amp.real, amp.imag, out, in_, pm
    bases, _ = O.momentum_subspaces(O.mesh_klist(3, 9), (3, 9), (9,))
    basis = next(b for b in bases if len(b) == 173583)
    N, nscat = len(basis), len(amp_a)
    assert nscat == 4590
    nnz = O.count_hits(basis, o)                      # every (row, term) hit, diagonal ones too
    cp, rv, _ = O.sparse_csc(basis, o)
    offd = int(np.count_nonzero(np.repeat(np.arange(N), np.diff(cp)) != rv))
    assert offd == 38242368                           # the hit cache's record count on the GPU
    assert abs(bench.hc_bytes(N, offd, nscat, 32, 8) - 10.19e9) < 0.01e9
    assert abs(bench.block_bytes(N, nnz, nscat, 32, 8) - 11.88e9) < 0.01e9
