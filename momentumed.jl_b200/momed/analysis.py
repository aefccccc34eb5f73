"""Analysis of eigenvectors on the device.

  - ``ED_bracket`` ........ EDCore/src/multiplication.jl:226-245 (mul_add_bracket 153-173,
                            mul_add_bracket_scatlist 180-190): <bra| op |ket>, the bra and the
                            ket on their own subspaces (targets outside the bra space dropped
                            as index_fit drops them)

  - ``PES_1rdm`` .......... MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33:
                            <psi| c+_i c_j |psi> over the subspace's orbitals

The bracket runs as one fused map-and-dot kernel (``momed_bracket``): the map's rows run over
the bra space and its targets are looked up in the ket space, and conj(bra) is folded in per
row, so H ket is never written.  The two-operator bracket <bra| op2 op1 |ket> of the reference
scatters through intermediate states outside any subspace and is not provided.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .core import MBOperator, MBS64Vector, hermitian_complete


def ED_bracket(bra: MBS64Vector, op: MBOperator, ket: MBS64Vector, *, handle: _lib.Handle | None = None) -> complex:
    """<bra| op |ket> (complex).  An upper_hermitian operator contributes its conjugate terms too."""
    lst = hermitian_complete(op)
    h = handle or _lib.Handle(0)
    try:
        h.set_basis(ket.space.list)
        h.set_scatter(lst.amp.astype(np.complex128), lst.in_, lst.out, lst.pm)
        same = len(bra.space.list) == len(ket.space.list) and np.array_equal(bra.space.list, ket.space.list)
        return h.bracket(np.asarray(bra.vec, np.complex128), np.asarray(ket.vec, np.complex128),
                         None if same else bra.space.list)
    finally:
        if handle is None:
            h.close()


def PES_1rdm(psi: MBS64Vector, *, handle: _lib.Handle | None = None) -> np.ndarray:
    """One-body reduced density matrix (bits x bits, bits = the subspace's orbital count)."""
    bits = int(getattr(psi.space, "bits", 64))
    h = handle or _lib.Handle(0)
    try:
        h.set_basis(psi.space.list)
        return h.rdm1(np.asarray(psi.vec, np.complex128), bits)
    finally:
        if handle is None:
            h.close()
