"""Analysis of eigenvectors on the device.

  - ``ED_bracket`` ........ EDCore/src/multiplication.jl:226-245 (mul_add_bracket 153-190,
                            mul_add_bracket_scatlist 195-222): <bra| op |ket> and
                            <bra| op2 op1 |ket>, the bra and the ket on their own subspaces
                            (targets outside the bra space dropped as index_fit drops them)

  - ``PES_1rdm`` .......... MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33:
                            <psi| c+_i c_j |psi> over the subspace's orbitals

  - ``ED_step_inner_prod`` MomentumED/src/analysis/manybody_quantum_geometry.jl:48-94: the
                            many-body connection step between eigenvectors at two kshift points
  - ``ED_connection_gaugefixing`` (same file, 14-45): the phase fix before a Wilson loop (host)

The bracket runs as one fused map-and-dot kernel (``momed_bracket``): the map's rows run over
the bra space and its targets are looked up in the ket space, and conj(bra) is folded in per
row, so H ket is never written.  The two-operator bracket <bra| op2 op1 |ket> of the reference
scatters through intermediate states outside any subspace: they are collected on the host as
the forward images of the ket space, op1 |ket> is mapped on their union with it, and op2 is
bracketed against that.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .core import MBOperator, MBS64Vector, hermitian_complete


def ED_bracket_threaded(bra: MBS64Vector, op: MBOperator, op1_or_ket, ket: MBS64Vector | None = None, *,
                        handle: _lib.Handle | None = None) -> complex:
    """ED_bracket_threaded (multiplication.jl:247-286), the reference's multithreaded form: the
    device bracket is parallel already, so it is ED_bracket."""
    return ED_bracket(bra, op, op1_or_ket, ket, handle=handle)


def forward_images(states: np.ndarray, lst) -> np.ndarray:
    """Sorted distinct states that one term of lst reaches from any of states (scat * mbs_in,
    EDCore/src/multiplication.jl:20-34): in within the state, out empty after removing in."""
    states = np.asarray(states, np.uint64)
    imgs = []
    for i_m, o_m in {(int(i), int(o)) for i, o in zip(lst.in_, lst.out)}:
        im, om = np.uint64(i_m), np.uint64(o_m)
        mid = states[(states & im) == im] & ~im
        imgs.append(mid[(mid & om) == 0] | om)
    return np.unique(np.concatenate(imgs)) if imgs else np.zeros(0, np.uint64)


def ED_bracket(bra: MBS64Vector, op: MBOperator, op1_or_ket, ket: MBS64Vector | None = None, *,
               handle: _lib.Handle | None = None) -> complex:
    """<bra| op |ket>, or <bra| op2 op1 |ket> called as ED_bracket(bra, op2, op1, ket) (complex).
    Upper_hermitian operators contribute their conjugate terms too.  The two-operator form
    passes through every intermediate state op1 reaches: the ket is mapped by op1 on the union
    of the ket space and those states (found on the host), then bracketed with op2."""
    h = handle or _lib.Handle(0)
    try:
        if ket is None:
            ket = op1_or_ket
            lst = hermitian_complete(op)
            h.set_basis(ket.space.list)
            h.set_scatter(lst.amp.astype(np.complex128), lst.in_, lst.out, lst.pm)
            kvec = np.asarray(ket.vec, np.complex128)
            kspace = ket.space.list
        else:
            l1, l2 = hermitian_complete(op1_or_ket), hermitian_complete(op)
            kspace = np.union1d(forward_images(ket.space.list, l1), ket.space.list).astype(np.uint64)
            x = np.zeros(len(kspace), np.complex128)
            x[np.searchsorted(kspace, ket.space.list)] = ket.vec
            h.set_basis(kspace)
            h.set_scatter(l1.amp.astype(np.complex128), l1.in_, l1.out, l1.pm)
            kvec = h.matvec(x)                                   # op1 |ket> on the union
            h.set_scatter(l2.amp.astype(np.complex128), l2.in_, l2.out, l2.pm)
        same = len(bra.space.list) == len(kspace) and np.array_equal(bra.space.list, kspace)
        return h.bracket(np.asarray(bra.vec, np.complex128), kvec, None if same else bra.space.list)
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
