"""Analysis of eigenvectors on the device.

  - ``ED_bracket`` ........ EDCore/src/multiplication.jl:226-245 (mul_add_bracket 153-173,
                            mul_add_bracket_scatlist 180-190): <bra| op |ket>, the bra and the
                            ket on their own subspaces (targets outside the bra space dropped
                            as index_fit drops them)

  - ``PES_1rdm`` .......... MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33:
                            <psi| c+_i c_j |psi> over the subspace's orbitals

  - ``ED_step_inner_prod`` MomentumED/src/analysis/manybody_quantum_geometry.jl:48-94: the
                            many-body connection step between eigenvectors at two kshift points
  - ``ED_connection_gaugefixing`` (same file, 14-45): the phase fix before a Wilson loop (host)

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


def ED_step_inner_prod(psi_f, psi_i, orbital_inner_prod, *, handle: _lib.Handle | None = None):
    """sum_x conj(psi_f[x]) psi_i[x] prod_{occupied o} orbital_inner_prod[o]: a complex for two
    MBS64Vector, a [g, g] matrix for two lists of g vectors (the non-Abelian connection step)."""
    single = isinstance(psi_f, MBS64Vector)
    fs = [psi_f] if single else list(psi_f)
    is_ = [psi_i] if single else list(psi_i)
    if len(fs) != len(is_):
        raise AssertionError("Number of eigenvectors must match in non-Abelian connection")
    space = fs[0].space
    for v in fs + is_:
        if not np.array_equal(v.space.list, space.list):
            raise AssertionError("The Hilbert subspaces of eigenvectors must match.")
    orb = np.asarray(orbital_inner_prod, np.complex128)
    if len(orb) != space.bits:
        raise AssertionError(f"orbital inner product length should be {space.bits}.")
    h = handle or _lib.Handle(0)
    try:
        h.set_basis(space.list)
        out = h.step_inner_prod(np.array([v.vec for v in fs]), np.array([v.vec for v in is_]), orb)
    finally:
        if handle is None:
            h.close()
    return complex(out[0, 0]) if single else out


def ED_connection_gaugefixing(psi, suggest_dims=None, warning_tol: float = 1e-8):
    """Fix the overall phase in place: one vector by its element suggest_dims (1-based, default 1),
    a list of g vectors by the determinant of their elements at suggest_dims (default 1..g),
    applied to the first vector (manybody_quantum_geometry.jl:14-45)."""
    import warnings
    if isinstance(psi, MBS64Vector):
        d = 1 if suggest_dims is None else int(suggest_dims)
        x = psi.vec[d - 1]
        if abs(x) < warning_tol:
            warnings.warn(f"Gauge fixing may be unstable. Element at position {d} has amplitude {abs(x)}.")
        psi.vec *= np.exp(-1j * np.angle(x))
        return psi
    dims = list(range(1, len(psi) + 1)) if suggest_dims is None else list(suggest_dims)
    if len(dims) != len(psi):
        raise AssertionError("number of suggested vectors mismatches number of eigenvectors.")
    m = np.array([[v.vec[i - 1] for v in psi] for i in dims])
    x = np.linalg.det(m)
    if abs(x) < warning_tol:
        warnings.warn(f"Gauge fixing may be unstable. Determinant of elements at position {dims} has amplitude {abs(x)}.")
    psi[0].vec *= np.exp(-1j * np.angle(x))
    return psi
