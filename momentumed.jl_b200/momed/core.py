"""Host-side mirror of the EDCore types on the matrix-free path.

Names, argument meaning and error behaviour follow the reference:
  - ``MBS64`` / bit helpers ........ EDCore/src/types/manybodystate_basis.jl
  - ``Scatter`` (normal ordering) .. EDCore/src/types/scattering.jl:52-153
  - ``sort_merge_scatlist`` ........ EDCore/src/types/scattering.jl:258-282
  - ``MBOperator`` ................. EDCore/src/types/operator.jl:24-32, 59-88
  - ``HilbertSubspace`` ............ EDCore/src/types/hilbert_subspace.jl:19-72
  - ``MBS64Vector`` ................ EDCore/src/types/manybodystate_vector.jl:21-116

A term list is a ``ScatterList``: struct-of-arrays (amp, out, in, parity_mask)
that iterates as ``Scatter`` objects, which is the layout the device library
consumes.  Bits: bit i-1 of a uint64 is orbital i.
"""
from __future__ import annotations

from typing import Iterable, Sequence

import numpy as np

U64 = (1 << 64) - 1


# ------------------------------------------------------------------------------- bits
def _shl1(s: int) -> int:
    """UInt64(1) << s with Julia semantics (0 for s >= 64)."""
    return 0 if s >= 64 or s < 0 else (1 << s)


def _tz(x: int) -> int:
    return (x & -x).bit_length() - 1 if x else 64


def parity_mask(occ: int) -> int:
    """scattering.jl:7-18: bits strictly between consecutive pairs of set bits (wrapping UInt64 arithmetic)."""
    mask = 0
    while occ > 0:
        tz1 = _tz(occ)
        occ &= occ - 1
        tz2 = _tz(occ)
        occ &= (occ - 1) & U64
        mask = (mask + _shl1(tz2)) & U64
        mask = (mask - _shl1(tz1 + 1)) & U64
    return mask


def make_mask64(occ: Iterable[int]) -> int:
    """manybodystate_basis.jl:161-182 (1-based orbitals)."""
    m = 0
    for i in occ:
        if not 1 <= i <= 64:
            raise AssertionError("orbital index must be between 1 and 64")
        m |= 1 << (i - 1)
    return m


def occ_list(n: int) -> list[int]:
    out = []
    while n:
        tz = _tz(n)
        out.append(tz + 1)
        n &= n - 1
    return out


def scat_occ_number(n: int, i_mask: int) -> int:
    """manybodystate_basis.jl:397-408."""
    return bin(n & parity_mask(i_mask)).count("1")


class MBS64:
    """A many-body state: bit i-1 of ``n`` is orbital i, ``bits`` physical orbitals."""

    __slots__ = ("bits", "n")

    def __init__(self, bits: int, n: int):
        if not (0 <= bits <= 64):
            raise AssertionError("The number of bits must be an integer between 0 and 64.")
        if n > (_shl1(bits) - 1 if bits < 64 else U64) or n < 0:
            raise AssertionError("State representation out of range for given bits")
        self.bits, self.n = bits, int(n)

    @classmethod
    def from_occ(cls, bits: int, occ: Iterable[int]) -> "MBS64":
        occ = sorted(occ)
        if len(set(occ)) != len(occ):
            raise AssertionError("Duplicate orbital indices when constructing MBS64.")
        return cls(bits, make_mask64(occ))

    def __mul__(self, other: "MBS64") -> "MBS64":     # concatenation, manybodystate_basis.jl:81-83
        return MBS64(self.bits + other.bits, ((self.n << other.bits) & U64) | other.n)

    def __add__(self, other: "MBS64") -> "MBS64":
        return MBS64(self.bits, self.n | other.n)

    def __eq__(self, other) -> bool:
        if isinstance(other, MBS64):
            return self.bits == other.bits and self.n == other.n
        return self.n == other

    def __lt__(self, other: "MBS64") -> bool:
        return self.n < other.n

    def __hash__(self):
        return hash(self.n)

    def __repr__(self):
        return f"MBS64{{{self.bits}}}({self.n})"


# ------------------------------------------------------------------------------- scatter
def _desc_sort_parity(v: Sequence[int]) -> int:
    inv = 0
    for a in range(len(v)):
        for b in range(a + 1, len(v)):
            if v[a] < v[b]:
                inv ^= 1
    return inv


class Scatter:
    """One term Amp * c+_out... c_in... (scattering.jl:52-62).

    ``Scatter(V, i, j; bits, upper_hermitian)``, ``Scatter(V, i1, i2, j2, j1; ...)`` and the
    generic N-body form follow scattering.jl:63-153 (normal ordering signs, upper-triangle swap
    with conj, real-only diagonal).  ``in_`` is the annihilation mask (``in`` is a Python keyword).
    """

    __slots__ = ("Amp", "out", "in_", "parity_mask", "bits")

    def __init__(self, V, *out_in: int, bits: int, upper_hermitian: bool = False,
                 element_type=np.complex128):
        V = element_type(V)
        n2 = len(out_in)
        if n2 % 2:
            raise AssertionError("number conservation requires annihilated and created indices number being even")
        if n2 == 2:
            i, j = out_in
            i_mask, j_mask = make_mask64((i,)), make_mask64((j,))
            if upper_hermitian:
                if j_mask < i_mask:
                    i_mask, j_mask, V = j_mask, i_mask, np.conj(V)
                elif j_mask == i_mask:
                    V = element_type(V.real)
        elif n2 == 4:
            i1, i2, j2, j1 = out_in
            i_mask, j_mask = make_mask64((i1, i2)), make_mask64((j1, j2))
            if j1 == j2 or i1 == i2:
                self._set(element_type(0), i_mask, j_mask, bits)
                return
            if i1 < i2:
                V = -V
            if j1 < j2:
                V = -V
            if upper_hermitian:
                if j_mask < i_mask:
                    i_mask, j_mask, V = j_mask, i_mask, np.conj(V)
                elif j_mask == i_mask:
                    V = element_type(V.real)
        else:
            N = n2 // 2
            is_ = list(out_in[:N])
            js = list(out_in[::-1][:N])
            i_mask, j_mask = make_mask64(is_), make_mask64(js)
            if bin(i_mask).count("1") < N or bin(j_mask).count("1") < N:
                self._set(element_type(0), i_mask, j_mask, bits)
                return
            if (_desc_sort_parity(is_) + _desc_sort_parity(js)) & 1:
                V = -V
            if upper_hermitian:
                if j_mask < i_mask:
                    i_mask, j_mask, V = j_mask, i_mask, np.conj(V)
                elif j_mask == i_mask:
                    V = element_type(V.real)
        self._set(V, i_mask, j_mask, bits)

    def _set(self, amp, out: int, in_: int, bits: int):
        self.Amp, self.out, self.in_, self.bits = amp, int(out), int(in_), bits
        self.parity_mask = parity_mask(self.out) ^ parity_mask(self.in_)

    @classmethod
    def raw(cls, amp, out: int, in_: int, bits: int) -> "Scatter":
        s = cls.__new__(cls)
        s._set(amp, out, in_, bits)
        return s

    def adjoint(self) -> "Scatter":                   # scattering.jl:185-187
        return Scatter.raw(np.conj(self.Amp), self.in_, self.out, self.bits)

    def isdiagonal(self) -> bool:
        return self.in_ == self.out

    def isupper(self) -> bool:                        # scattering.jl:170
        return self.in_ > self.out or (self.in_ == self.out and self.Amp.imag == 0)

    def get_body(self):
        return (bin(self.out).count("1"), bin(self.in_).count("1"))

    def key(self):
        return (self.in_, self.out)

    def __eq__(self, other) -> bool:                  # scattering.jl:215-217 (amplitude-blind)
        return isinstance(other, Scatter) and self.in_ == other.in_ and self.out == other.out

    def __lt__(self, other) -> bool:                  # scattering.jl:205-207
        return self.key() < other.key()

    def __repr__(self):
        return (f"Scatter: c+_out {list(reversed(occ_list(self.out)))} c_in {occ_list(self.in_)}, "
                f"Amp = {self.Amp}")

    def apply(self, state: int):
        """scat * mbs_in (multiplication.jl:19-33): (amp, out_state), amp 0 when not mapped."""
        if state & self.in_ != self.in_:
            return 0, state
        if self.in_ == self.out:
            return self.Amp, state
        mid = state & ~self.in_ & U64
        if mid & self.out:
            return 0, state
        sign = 1 - 2 * (bin(mid & self.parity_mask).count("1") & 1)
        return sign * self.Amp, mid | self.out

    def apply_right(self, state: int):
        """mbs_out * scat (multiplication.jl:55-69): (amp, in_state)."""
        if state & self.out != self.out:
            return 0, state
        if self.in_ == self.out:
            return self.Amp, state
        mid = state & ~self.out & U64
        if mid & self.in_:
            return 0, state
        sign = 1 - 2 * (bin(mid & self.parity_mask).count("1") & 1)
        return sign * self.Amp, mid | self.in_


class ScatterList:
    """Struct-of-arrays term list; iterates as ``Scatter``."""

    def __init__(self, amp, out, in_, pm=None, bits: int = 64, element_type=np.complex128):
        self.amp = np.asarray(amp, element_type)
        self.out = np.asarray(out, np.uint64)
        self.in_ = np.asarray(in_, np.uint64)
        if pm is None:
            pm = [parity_mask(int(o)) ^ parity_mask(int(i)) for o, i in zip(self.out, self.in_)]
        self.pm = np.asarray(pm, np.uint64)
        self.bits = bits
        self.element_type = element_type

    @classmethod
    def from_terms(cls, terms: Sequence[Scatter], bits: int | None = None, element_type=np.complex128):
        if bits is None:
            bits = terms[0].bits if len(terms) else 64
        return cls([t.Amp for t in terms], [t.out for t in terms], [t.in_ for t in terms],
                   [t.parity_mask for t in terms], bits, element_type)

    def __len__(self):
        return len(self.amp)

    def __getitem__(self, i) -> Scatter:
        return Scatter.raw(self.element_type(self.amp[i]), int(self.out[i]), int(self.in_[i]), self.bits)

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def concat(self, *others: "ScatterList") -> "ScatterList":
        lists = (self,) + others
        return ScatterList(np.concatenate([l.amp for l in lists]), np.concatenate([l.out for l in lists]),
                           np.concatenate([l.in_ for l in lists]), np.concatenate([l.pm for l in lists]),
                           self.bits, self.element_type)

    def isupper(self) -> np.ndarray:
        return (self.in_ > self.out) | ((self.in_ == self.out) & (self.amp.imag == 0))

    def equal(self, other: "ScatterList") -> bool:
        """Bit-exact equality of masks, parity masks and amplitudes."""
        return (len(self) == len(other) and np.array_equal(self.out, other.out)
                and np.array_equal(self.in_, other.in_) and np.array_equal(self.pm, other.pm)
                and np.array_equal(self.amp.view(np.uint8), other.amp.astype(self.element_type).view(np.uint8)))


def _as_list(x) -> ScatterList:
    if isinstance(x, ScatterList):
        return x
    return ScatterList.from_terms(list(x))


def sort_merge_scatlist(*lists, check_upper: bool = True) -> ScatterList:
    """scattering.jl:258-282: stable sort by (in, out), then sum amplitudes of equal keys
    starting from 0 * first (so the arithmetic order matches the reference)."""
    parts = [_as_list(l) for l in lists]
    L = parts[0].concat(*parts[1:]) if len(parts) > 1 else parts[0]
    if len(L) == 0:
        return L
    if check_upper and not np.all(L.isupper()):
        raise AssertionError("All Scatter terms must be in the upper triangular.")
    order = np.lexsort((L.out, L.in_))          # stable: primary in, secondary out
    amp, out, in_, pm = L.amp[order], L.out[order], L.in_[order], L.pm[order]
    et = L.element_type
    new_group = np.ones(len(amp), bool)
    new_group[1:] = (in_[1:] != in_[:-1]) | (out[1:] != out[:-1])
    starts = np.flatnonzero(new_group)
    merged = amp[starts].copy()
    zero = et(0)
    # first entry: (0 * a1) + a1 in the element type
    merged[0] = et(zero * et(amp[0])) + et(amp[0])
    dup = np.flatnonzero(~new_group)
    if len(dup):
        gid = np.cumsum(new_group) - 1
        for g in np.unique(gid[dup]):
            idx = np.flatnonzero(gid == g)
            acc = (et(zero * et(amp[idx[0]])) + et(amp[idx[0]])) if g == 0 else et(amp[idx[0]])
            for k in idx[1:]:
                acc = et(acc + et(amp[k]))
            merged[g] = acc
    return ScatterList(merged, out[starts], in_[starts], pm[starts], L.bits, et)


class MBOperator:
    """Sorted, merged term list plus the upper_hermitian flag (operator.jl:24-32)."""

    def __init__(self, *scats, upper_hermitian: bool):
        self.scats = sort_merge_scatlist(*scats, check_upper=upper_hermitian)
        self.upper_hermitian = upper_hermitian

    def isupper(self) -> bool:
        return self.upper_hermitian

    def __repr__(self):
        return (f"Many Body Operator {'(Hermitian, upper triangle entries only) ' * self.upper_hermitian}:\n"
                f"\t{len(self.scats)} scattering terms")

    def adjoint(self) -> "MBOperator":                # operator.jl:59-67 on a copy
        op = MBOperator.__new__(MBOperator)
        op.upper_hermitian = self.upper_hermitian
        s = self.scats
        if self.upper_hermitian:
            op.scats = ScatterList(s.amp.copy(), s.out.copy(), s.in_.copy(), s.pm.copy(), s.bits, s.element_type)
        else:
            adj = ScatterList(np.conj(s.amp), s.in_, s.out, s.pm, s.bits, s.element_type)
            order = np.lexsort((adj.out, adj.in_))
            op.scats = ScatterList(adj.amp[order], adj.out[order], adj.in_[order], adj.pm[order], s.bits,
                                   s.element_type)
        return op


def hermitian_complete(op: MBOperator) -> ScatterList:
    """The full term list of LinearMap (linear_map.jl:22-37): the upper list plus s' for every
    non-diagonal term, stably sorted by (in, out)."""
    s = op.scats
    if not op.upper_hermitian:
        return s
    nd = s.in_ != s.out
    amp = np.concatenate([s.amp, np.conj(s.amp[nd])])
    out = np.concatenate([s.out, s.in_[nd]])
    in_ = np.concatenate([s.in_, s.out[nd]])
    pm = np.concatenate([s.pm, s.pm[nd]])
    order = np.lexsort((out, in_))
    return ScatterList(amp[order], out[order], in_[order], pm[order], s.bits, s.element_type)


def pair_operator(A: MBOperator, B: MBOperator):
    """Term arrays of H(u) = A + u B on the union of both completed term lists, sorted by (in, out):
    returns (amp_a, amp_b, in, out, parity).  A term present in one operator only gets amplitude 0
    in the other.  Used by the batched solver, where u is an interaction strength."""
    fa, fb = hermitian_complete(A), hermitian_complete(B)
    keys_a = {(int(i), int(o)): k for k, (i, o) in enumerate(zip(fa.in_, fa.out))}
    keys_b = {(int(i), int(o)): k for k, (i, o) in enumerate(zip(fb.in_, fb.out))}
    keys = sorted(set(keys_a) | set(keys_b))
    amp_a = np.zeros(len(keys), np.complex128)
    amp_b = np.zeros(len(keys), np.complex128)
    for n, key in enumerate(keys):
        if key in keys_a:
            amp_a[n] = fa.amp[keys_a[key]]
        if key in keys_b:
            amp_b[n] = fb.amp[keys_b[key]]
    in_ = np.array([k[0] for k in keys], np.uint64)
    out = np.array([k[1] for k in keys], np.uint64)
    pm = np.array([parity_mask(int(o)) ^ parity_mask(int(i)) for i, o in keys], np.uint64)
    return amp_a, amp_b, in_, out, pm


# ------------------------------------------------------------------------------- containers
class HilbertSubspace:
    """Sorted list of basis states (hilbert_subspace.jl:19-30); ``list`` is a uint64 array."""

    def __init__(self, lst, bits: int = 64):
        arr = np.asarray([m.n for m in lst] if len(lst) and isinstance(lst[0], MBS64) else lst, np.uint64)
        if len(arr) > 1 and not np.all(arr[1:] >= arr[:-1]):
            import warnings
            warnings.warn("The input list for HilbertSubspace is not sorted. It will be sorted now.")
            arr = np.sort(arr)
        self.list = arr
        self.bits = bits

    @property
    def length(self) -> int:
        return len(self.list)

    def __len__(self):
        return len(self.list)

    def get(self, mbs) -> int:
        """searchsortedfirst, 1-based (hilbert_subspace.jl:67-69)."""
        n = mbs.n if isinstance(mbs, MBS64) else int(mbs)
        return int(np.searchsorted(self.list, np.uint64(n), side="left")) + 1

    def index_fit(self, index: int, mbs) -> bool:
        n = mbs.n if isinstance(mbs, MBS64) else int(mbs)
        return 0 < index <= len(self.list) and int(self.list[index - 1]) == n

    def get_bits(self) -> int:
        return self.bits

    def __repr__(self):
        return f"Hilbert subspace {{bits = {self.bits}, dim = {len(self.list)}}}"


def index_fit(index: int, space: HilbertSubspace, mbs) -> bool:
    return space.index_fit(index, mbs)


class MBS64Vector:
    """Coefficient vector bound to a subspace (manybodystate_vector.jl:21-29)."""

    def __init__(self, vec, space: HilbertSubspace):
        vec = np.asarray(vec)
        if len(vec) != len(space):
            raise AssertionError("vector length mismatches Hilbert space dimension.")
        self.vec, self.space = vec, space

    def __len__(self):
        return len(self.vec)

    @property
    def size(self):
        return (len(self.vec),)

    def similar(self) -> "MBS64Vector":
        return MBS64Vector(np.empty_like(self.vec), self.space)

    def dot(self, other: "MBS64Vector"):
        if other.space is not self.space:
            raise AssertionError("mbs vectors are not in the same subspace.")
        return np.vdot(self.vec, other.vec)

    def __add__(self, other):
        return MBS64Vector(self.vec + other.vec, self.space)

    def __sub__(self, other):
        return MBS64Vector(self.vec - other.vec, self.space)
