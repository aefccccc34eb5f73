"""Python driver for the parity oracle (TEST INFRASTRUCTURE ONLY).

Wraps ``libmomed_oracle.so`` (built from ``momed_oracle.c`` by the Makefile in
this directory) with ctypes.  The oracle is a CPU restatement of
MomentumED.jl's matrix-free path; only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference arm may import this module.  The
product library never imports it.

Scatter lists are numpy structured arrays with the layout of ``or_scat``
(re, im, out, in, pm).  Complex vectors are numpy complex128/complex64.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmomed_oracle.so")

SCAT_DTYPE = np.dtype([("re", "<f8"), ("im", "<f8"), ("out", "<u8"), ("in", "<u8"), ("pm", "<u8")])


class _Scat(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double), ("out", C.c_uint64),
                ("in_", C.c_uint64), ("pm", C.c_uint64)]


class _Para(C.Structure):
    _fields_ = [("dim", C.c_int32), ("Nk", C.c_int32), ("Nc_mix", C.c_int32),
                ("Nc_conserve", C.c_int32), ("k_list", C.POINTER(C.c_int64)),
                ("Gk", C.POINTER(C.c_int64))]


class _Synth(C.Structure):
    _fields_ = [("a", C.c_int32), ("b", C.c_int32), ("Nk", C.c_int32), ("pad", C.c_int32),
                ("beta", C.c_double), ("theta", C.POINTER(C.c_double))]


class _Info(C.Structure):
    _fields_ = [("converged", C.c_int32), ("restarts", C.c_int32), ("matvecs", C.c_int64)]


H1_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                    C.POINTER(C.c_double), C.POINTER(C.c_double))
H2_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                    C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                    C.POINTER(C.c_double), C.POINTER(C.c_double))

H1C_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.c_int64,
                     C.POINTER(C.c_double), C.POINTER(C.c_double))
H2C_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                     C.POINTER(C.c_double), C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                     C.POINTER(C.c_double), C.POINTER(C.c_double))
H1R_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_int64), C.c_int64, C.c_int64,
                     C.POINTER(C.c_double), C.POINTER(C.c_double))
H2R_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                     C.POINTER(C.c_int64), C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                     C.POINTER(C.c_double), C.POINTER(C.c_double))

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "momed_oracle.c"))):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_parity_mask.restype = C.c_uint64
        L.or_parity_mask.argtypes = [C.c_uint64]
        L.or_scat_occ_number.argtypes = [C.c_uint64, C.c_uint64]
        L.or_scat_occ_number_1.argtypes = [C.c_uint64, C.c_int, C.c_int]
        L.or_scat_occ_number_2.argtypes = [C.c_uint64, C.c_int, C.c_int]
        L.or_scatter_1.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.or_scatter_2.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.or_scatter_n.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.or_isupper.argtypes = [C.c_void_p]
        for fn in (L.or_scat_apply, L.or_scat_apply_right):
            fn.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                           C.POINTER(C.c_uint64)]
        L.or_sort_merge.restype = C.c_int64
        L.or_sort_merge.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p]
        L.or_hermitian_complete.restype = C.c_int64
        L.or_hermitian_complete.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.or_binomial.restype = C.c_int64
        L.or_binomial.argtypes = [C.c_int64, C.c_int64]
        L.or_unrank_colex.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_void_p]
        L.or_colex.restype = C.c_int64
        L.or_colex.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_void_p, C.c_int64]
        L.or_colex_mask.restype = C.c_int64
        L.or_colex_mask.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int64, C.c_int64,
                                    C.c_void_p, C.c_int64]
        L.or_momentum_subspaces.restype = C.c_int64
        L.or_momentum_subspaces.argtypes = [C.POINTER(_Para), C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                            C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.POINTER(C.c_int64)]
        L.or_scatterlist_onebody.restype = C.c_int64
        L.or_scatterlist_onebody.argtypes = [C.POINTER(_Para), H1_FN, C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        L.or_scatterlist_twobody.restype = C.c_int64
        L.or_scatterlist_twobody.argtypes = [C.POINTER(_Para), H2_FN, C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        L.or_scatterlist_onebody_coord.restype = C.c_int64
        L.or_scatterlist_onebody_coord.argtypes = [C.POINTER(_Para), H1C_FN, C.c_void_p, C.c_void_p, C.c_int,
                                                   C.c_void_p, C.c_int64]
        L.or_scatterlist_twobody_coord.restype = C.c_int64
        L.or_scatterlist_twobody_coord.argtypes = [C.POINTER(_Para), H2C_FN, C.c_void_p, C.c_void_p, C.c_int,
                                                   C.c_void_p, C.c_int64]
        L.or_scatterlist_onebody_rational.restype = C.c_int64
        L.or_scatterlist_onebody_rational.argtypes = [C.POINTER(_Para), H1R_FN, C.c_void_p, C.c_void_p, C.c_int,
                                                      C.c_void_p, C.c_int64]
        L.or_scatterlist_twobody_rational.restype = C.c_int64
        L.or_scatterlist_twobody_rational.argtypes = [C.POINTER(_Para), H2R_FN, C.c_void_p, C.c_void_p, C.c_int,
                                                      C.c_void_p, C.c_int64]
        L.or_synth_init.argtypes = [C.POINTER(_Synth), C.c_int, C.c_int, C.c_uint64]
        L.or_synth_free.argtypes = [C.POINTER(_Synth)]
        L.or_synth_onebody.restype = C.c_int64
        L.or_synth_onebody.argtypes = [C.POINTER(_Para), C.POINTER(_Synth), C.c_int, C.c_void_p, C.c_int64]
        L.or_synth_twobody.restype = C.c_int64
        L.or_synth_twobody.argtypes = [C.POINTER(_Para), C.POINTER(_Synth), C.c_int, C.c_void_p, C.c_int64]
        L.or_synth_h2.argtypes = [C.c_void_p] + [C.c_int64] * 8 + [C.POINTER(C.c_double)] * 2
        L.or_synth_h1.argtypes = [C.c_void_p] + [C.c_int64] * 3 + [C.POINTER(C.c_double)] * 2
        L.or_matvec_c128.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]
        L.or_matvec_c64.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]
        L.or_dense_hamiltonian.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
        L.or_bracket.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                 C.c_int64, C.c_int, C.c_void_p]
        L.or_rdm1.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int, C.c_void_p]
        L.or_step_inner_prod.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                         C.c_void_p]
        L.or_bracket2.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                  C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
        L.or_sparse_csc.restype = C.c_int64
        L.or_sparse_csc.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_int64]
        L.or_count_hits.restype = C.c_int64
        L.or_count_hits.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int]
        L.or_symeig.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_eigsolve.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_double,
                                  C.c_int, C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.POINTER(_Info)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


# --------------------------------------------------------------------------- bits
def parity_mask(occ: int) -> int:
    return int(lib().or_parity_mask(C.c_uint64(occ)))


def scat_occ_number(n: int, imask: int) -> int:
    return int(lib().or_scat_occ_number(n, imask))


def scat_occ_number_tuple(n: int, orbitals, bits: int) -> int:
    if len(orbitals) == 1:
        return int(lib().or_scat_occ_number_1(n, orbitals[0], bits))
    if len(orbitals) == 2:
        return int(lib().or_scat_occ_number_2(n, orbitals[0], orbitals[1]))
    raise ValueError("tuple form covers one and two orbitals")


# --------------------------------------------------------------------------- scatter
def _rec_to_np(rec: _Scat) -> np.ndarray:
    a = np.zeros(1, SCAT_DTYPE)
    a[0] = (rec.re, rec.im, rec.out, rec.in_, rec.pm)
    return a


def scatter(V, *out_in, upper_hermitian=False) -> np.ndarray:
    """Scatter(V, out_in...; upper_hermitian) as one structured record."""
    V = complex(V)
    rec = _Scat()
    L = lib()
    if len(out_in) == 2:
        L.or_scatter_1(V.real, V.imag, out_in[0], out_in[1], int(upper_hermitian), C.byref(rec))
    elif len(out_in) == 4:
        L.or_scatter_2(V.real, V.imag, *out_in, int(upper_hermitian), C.byref(rec))
    else:
        arr = np.asarray(out_in, dtype=np.int64)
        if L.or_scatter_n(V.real, V.imag, _ptr(arr), len(out_in), int(upper_hermitian), C.byref(rec)) != 0:
            raise ValueError("odd operator count")
    return _rec_to_np(rec)


def scat_apply(rec, state: int, right: bool = False):
    """scat * mbs (right=False) or mbs * scat (right=True); returns (amp, state) or None."""
    a = np.ascontiguousarray(np.asarray(rec, SCAT_DTYPE).reshape(1))
    re, im, st = C.c_double(), C.c_double(), C.c_uint64()
    fn = lib().or_scat_apply_right if right else lib().or_scat_apply
    ok = fn(_ptr(a), C.c_uint64(state), C.byref(re), C.byref(im), C.byref(st))
    return (complex(re.value, im.value), int(st.value)) if ok else None


def isupper(rec) -> bool:
    a = np.ascontiguousarray(np.asarray(rec, SCAT_DTYPE).reshape(1))
    return bool(lib().or_isupper(_ptr(a)))


def sort_merge(lst: np.ndarray, check_upper=True, prec=64) -> np.ndarray:
    lst = np.ascontiguousarray(lst, SCAT_DTYPE)
    out = np.zeros(max(len(lst), 1), SCAT_DTYPE)
    m = lib().or_sort_merge(_ptr(lst), len(lst), int(check_upper), prec, _ptr(out))
    if m < 0:
        raise AssertionError("All Scatter terms must be in the upper triangular.")
    return out[:m].copy()


def hermitian_complete(upper: np.ndarray) -> np.ndarray:
    upper = np.ascontiguousarray(upper, SCAT_DTYPE)
    out = np.zeros(max(2 * len(upper), 1), SCAT_DTYPE)
    m = lib().or_hermitian_complete(_ptr(upper), len(upper), _ptr(out))
    return out[:m].copy()


# --------------------------------------------------------------------------- colex
def binomial(n, k) -> int:
    return int(lib().or_binomial(n, k))


def unrank_colex(n, t, k):
    out = np.zeros(max(t, 1), np.int64)
    m = lib().or_unrank_colex(n, t, k, _ptr(out))
    return [int(v) for v in out[:m]]


def colex(n, t, start=1, end=None, mask=None) -> np.ndarray:
    full = binomial(len(mask) if mask is not None else n, t)
    end = full if end is None else end
    cap = max(0, min(end, full) - start + 1)
    out = np.zeros(max(cap, 1), np.uint64)
    if mask is None:
        m = lib().or_colex(n, t, start, end, _ptr(out), cap)
    else:
        marr = np.asarray(mask, np.int64)
        m = lib().or_colex_mask(n, t, _ptr(marr), len(marr), start, end, _ptr(out), cap)
    return out[:m].copy()


# --------------------------------------------------------------------------- sectors
def _para(k_list: np.ndarray, Gk, Nc_mix=1, Nc_conserve=1):
    k_list = np.asarray(k_list, np.int64)
    dim, Nk = k_list.shape
    kl = np.ascontiguousarray(k_list.T).reshape(-1)          # kl[d + dim*i]
    g = np.asarray(Gk, np.int64)
    p = _Para(dim, Nk, Nc_mix, Nc_conserve, kl.ctypes.data_as(C.POINTER(C.c_int64)),
              g.ctypes.data_as(C.POINTER(C.c_int64)))
    p._keep = (kl, g)
    return p


def momentum_subspaces(k_list, Gk, N_each, Nc_mix=1, Nc_conserve=1, mask=None, momentum_list=None):
    """Sector bases (list of uint64 arrays) and their momenta, in the reference's order."""
    p = _para(k_list, Gk, Nc_mix, Nc_conserve)
    ne = np.asarray(N_each, np.int64)
    marr = np.asarray(mask, np.int64) if mask is not None else None
    restrict = momentum_list is not None
    mom = np.asarray(momentum_list if restrict else [], np.int64).reshape(-1)
    nsec = C.c_int64(0)
    L = lib()
    total = L.or_momentum_subspaces(C.byref(p), _ptr(ne), len(ne), _ptr(marr),
                                    len(marr) if marr is not None else -1, int(restrict), _ptr(mom),
                                    len(mom) // p.dim if restrict else 0, None, None, None, C.byref(nsec))
    if total < 0:
        raise ValueError("invalid arguments")
    ks = np.zeros(max(nsec.value * p.dim, 1), np.int64)
    sizes = np.zeros(max(nsec.value, 1), np.int64)
    basis = np.zeros(max(total, 1), np.uint64)
    L.or_momentum_subspaces(C.byref(p), _ptr(ne), len(ne), _ptr(marr),
                            len(marr) if marr is not None else -1, int(restrict), _ptr(mom),
                            len(mom) // p.dim if restrict else 0, _ptr(ks), _ptr(sizes), _ptr(basis),
                            C.byref(nsec))
    out, kout, off = [], [], 0
    for s in range(nsec.value):
        out.append(basis[off:off + sizes[s]].copy())
        kout.append(tuple(int(v) for v in ks[s * p.dim:(s + 1) * p.dim]))
        off += sizes[s]
    return out, kout


def mesh_klist(a: int, b: int) -> np.ndarray:
    i = np.arange(a * b)
    return np.stack([i % a, i // a]).astype(np.int64)


# --------------------------------------------------------------------------- builders
class Synth:
    """The synthetic Hamiltonian recipe (one-body band + random-phase two-body) on an a x b mesh."""

    def __init__(self, a: int, b: int, seed: int, Nc_mix=1, Nc_conserve=1):
        self.a, self.b = a, b
        self.s = _Synth()
        if lib().or_synth_init(C.byref(self.s), a, b, seed) != 0:
            raise MemoryError
        self.para = _para(mesh_klist(a, b), (a, b), Nc_mix, Nc_conserve)

    @property
    def beta(self) -> float:
        return float(self.s.beta)

    def h1(self, k, cf, ci) -> complex:
        re, im = C.c_double(), C.c_double()
        lib().or_synth_h1(C.addressof(self.s), k, cf, ci, C.byref(re), C.byref(im))
        return complex(re.value, im.value)

    def h2(self, kf1, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1) -> complex:
        re, im = C.c_double(), C.c_double()
        lib().or_synth_h2(C.addressof(self.s), kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1, C.byref(re), C.byref(im))
        return complex(re.value, im.value)

    def _build(self, fn, prec):
        L = lib()
        n = fn(C.byref(self.para), C.byref(self.s), prec, None, 0)
        out = np.zeros(max(n, 1), SCAT_DTYPE)
        m = fn(C.byref(self.para), C.byref(self.s), prec, _ptr(out), len(out))
        if m < 0:
            raise RuntimeError("builder failed")
        return out[:m].copy()

    def onebody(self, prec=64) -> np.ndarray:
        return self._build(lib().or_synth_onebody, prec)

    def twobody(self, prec=64) -> np.ndarray:
        return self._build(lib().or_synth_twobody, prec)

    def __del__(self):
        try:
            lib().or_synth_free(C.byref(self.s))
        except Exception:
            pass


def scatterlist_onebody(k_list, Gk, H_one, Nc_mix=1, Nc_conserve=1, prec=64) -> np.ndarray:
    """ED_scatterlist_onebody with an index-mode Python callable H_one(k, cf, ci)."""
    p = _para(k_list, Gk, Nc_mix, Nc_conserve)

    @H1_FN
    def cb(ctx, k, cf, ci, re, im):
        v = complex(H_one(k, cf, ci))
        re[0], im[0] = v.real, v.imag

    L = lib()
    n = L.or_scatterlist_onebody(C.byref(p), cb, None, prec, None, 0)
    out = np.zeros(max(n, 1), SCAT_DTYPE)
    m = L.or_scatterlist_onebody(C.byref(p), cb, None, prec, _ptr(out), len(out))
    return out[:m].copy()


def scatterlist_twobody(k_list, Gk, H_two, Nc_mix=1, Nc_conserve=1, prec=64) -> np.ndarray:
    """ED_scatterlist_twobody with an index-mode Python callable H_two(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1)."""
    p = _para(k_list, Gk, Nc_mix, Nc_conserve)

    @H2_FN
    def cb(ctx, kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1, re, im):
        v = complex(H_two(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1))
        re[0], im[0] = v.real, v.imag

    L = lib()
    n = L.or_scatterlist_twobody(C.byref(p), cb, None, prec, None, 0)
    out = np.zeros(max(n, 1), SCAT_DTYPE)
    m = L.or_scatterlist_twobody(C.byref(p), cb, None, prec, _ptr(out), len(out))
    return out[:m].copy()


# --------------------------------------------------------------------------- matvec / eig
def shift_matrix(kshift, Ncc: int, dim: int):
    """kshift -> shifts[d][c] (scat_list.jl:29-50): None -> zeros, a tuple -> the same shift for
    every conserved component, a list of Ncc tuples -> one per component, a dim x Ncc array."""
    if kshift is None:
        return [[0] * Ncc for _ in range(dim)]
    if isinstance(kshift, tuple):
        return [[kshift[d] for _ in range(Ncc)] for d in range(dim)]
    if isinstance(kshift, list):
        assert len(kshift) == Ncc, "length of kshift isn't equal to para.Nc_conserve."
        return [[kshift[c][d] for c in range(Ncc)] for d in range(dim)]
    a = np.asarray(kshift)
    assert a.shape == (dim, Ncc), "size of kshift isn't equal to para.Nc_conserve."
    return [[a[d, c].item() for c in range(Ncc)] for d in range(dim)]


def _exact(shifts) -> bool:
    """scat_list.jl:453-457: integer and rational shifts keep coordinates exact (Rational), any
    float makes them Float64."""
    return all(isinstance(v, (int, np.integer, Fraction)) for row in shifts for v in row)


def _coord_call(k_list, Gk, Nc_mix, Nc_conserve, kshift, prec, onebody, fn):
    p = _para(k_list, Gk, Nc_mix, Nc_conserve)
    dim = p.dim
    shifts = shift_matrix(kshift, Nc_conserve, dim)
    L = lib()
    if _exact(shifts):
        rs = np.zeros(2 * dim * Nc_conserve, np.int64)
        for d in range(dim):
            for c in range(Nc_conserve):
                f = Fraction(shifts[d][c])
                rs[2 * (d + dim * c)], rs[2 * (d + dim * c) + 1] = f.numerator, f.denominator

        def co(k):
            return tuple(Fraction(int(k[2 * d]), int(k[2 * d + 1])) for d in range(dim))

        if onebody:
            @H1R_FN
            def cb(ctx, k, cf, ci, re, im):
                v = complex(fn(co(k), cf, ci))
                re[0], im[0] = v.real, v.imag
            build = L.or_scatterlist_onebody_rational
        else:
            @H2R_FN
            def cb(ctx, a, b, c, d, cf1, cf2, ci2, ci1, re, im):
                v = complex(fn(co(a), co(b), co(c), co(d), cf1, cf2, ci2, ci1))
                re[0], im[0] = v.real, v.imag
            build = L.or_scatterlist_twobody_rational
        sh = rs
    else:
        sh = np.zeros(dim * Nc_conserve, np.float64)
        for d in range(dim):
            for c in range(Nc_conserve):
                sh[d + dim * c] = float(shifts[d][c])

        def co(k):
            return tuple(float(k[d]) for d in range(dim))

        if onebody:
            @H1C_FN
            def cb(ctx, k, cf, ci, re, im):
                v = complex(fn(co(k), cf, ci))
                re[0], im[0] = v.real, v.imag
            build = L.or_scatterlist_onebody_coord
        else:
            @H2C_FN
            def cb(ctx, a, b, c, d, cf1, cf2, ci2, ci1, re, im):
                v = complex(fn(co(a), co(b), co(c), co(d), cf1, cf2, ci2, ci1))
                re[0], im[0] = v.real, v.imag
            build = L.or_scatterlist_twobody_coord
        sh = sh
    n = build(C.byref(p), cb, None, _ptr(sh), prec, None, 0)
    out = np.zeros(max(n, 1), SCAT_DTYPE)
    m = build(C.byref(p), cb, None, _ptr(sh), prec, _ptr(out), len(out))
    if m < 0:
        raise RuntimeError("builder failed")
    return out[:m].copy()


def scatterlist_onebody_coord(k_list, Gk, H_one, Nc_mix=1, Nc_conserve=1, kshift=None, prec=64) -> np.ndarray:
    """ED_scatterlist_onebody with a coordinate-mode callable H_one(k::tuple, cf, ci)
    (scat_list.jl:78-142): k is k/Gk (+ the component's kshift/Gk) as Fractions for integer or
    rational shifts (the default) and as floats otherwise."""
    return _coord_call(k_list, Gk, Nc_mix, Nc_conserve, kshift, prec, True, H_one)


def scatterlist_twobody_coord(k_list, Gk, H_two, Nc_mix=1, Nc_conserve=1, kshift=None, prec=64) -> np.ndarray:
    """ED_scatterlist_twobody with a coordinate-mode callable H_two(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1)
    (scat_list.jl:442-514), coordinates as in scatterlist_onebody_coord."""
    return _coord_call(k_list, Gk, Nc_mix, Nc_conserve, kshift, prec, False, H_two)


def matvec(basis: np.ndarray, full_list: np.ndarray, x: np.ndarray, nthreads: int = 0) -> np.ndarray:
    """Reference CPU map y = H x over the Hermitian-completed list (complex128 or complex64)."""
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    L = lib()
    if x.dtype == np.complex64:
        x = np.ascontiguousarray(x)
        y = np.empty_like(x)
        L.or_matvec_c64(_ptr(basis), len(basis), _ptr(full_list), len(full_list), _ptr(x), _ptr(y), nthreads)
    else:
        x = np.ascontiguousarray(x, np.complex128)
        y = np.empty_like(x)
        L.or_matvec_c128(_ptr(basis), len(basis), _ptr(full_list), len(full_list), _ptr(x), _ptr(y), nthreads)
    return y


def matvec_rows(basis, full_list, x, rows, nthreads: int = 0) -> np.ndarray:
    """(H x)[rows] for the given row indices (complex128)."""
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    x = np.ascontiguousarray(x, np.complex128)
    rows = np.ascontiguousarray(rows, np.int64)
    y = np.zeros(len(rows), np.complex128)
    L = lib()
    L.or_matvec_rows_c128.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_int64, C.c_void_p, C.c_int]
    L.or_matvec_rows_c128(_ptr(basis), len(basis), _ptr(full_list), len(full_list), _ptr(x), _ptr(rows),
                          len(rows), _ptr(y), nthreads)
    return y


def dense_hamiltonian(basis: np.ndarray, full_list: np.ndarray) -> np.ndarray:
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    H = np.zeros((len(basis), len(basis)), np.complex128)
    lib().or_dense_hamiltonian(_ptr(basis), len(basis), _ptr(full_list), len(full_list), _ptr(H))
    return H


def bracket(bra_basis, bra, ket_basis, ket, scat_list, upper: bool = False) -> complex:
    """<bra| op |ket> over a term list (multiplication.jl:153-190); upper: upper_hermitian list."""
    bb = np.ascontiguousarray(bra_basis, np.uint64)
    kb = np.ascontiguousarray(ket_basis, np.uint64)
    bv = np.ascontiguousarray(bra, np.complex128)
    kv = np.ascontiguousarray(ket, np.complex128)
    lst = np.ascontiguousarray(scat_list, SCAT_DTYPE)
    out = np.zeros(2)
    lib().or_bracket(_ptr(bb), len(bb), _ptr(bv), _ptr(kb), len(kb), _ptr(kv), _ptr(lst), len(lst), int(upper),
                     _ptr(out))
    return complex(out[0], out[1])


def rdm1(basis, psi, bits: int) -> np.ndarray:
    """PES_1rdm (particle_reduced_density_matrix.jl:4-33): [bits, bits] complex matrix."""
    bb = np.ascontiguousarray(basis, np.uint64)
    v = np.ascontiguousarray(psi, np.complex128)
    out = np.zeros((bits, bits), np.complex128)
    lib().or_rdm1(_ptr(bb), len(bb), _ptr(v), int(bits), _ptr(out))
    return out


def step_inner_prod(basis, psi_f, psi_i, orb) -> np.ndarray:
    """ED_step_inner_prod (manybody_quantum_geometry.jl:48-94): [g, g] from [g, N] vectors."""
    bb = np.ascontiguousarray(basis, np.uint64)
    f = np.ascontiguousarray(np.atleast_2d(psi_f), np.complex128)
    i = np.ascontiguousarray(np.atleast_2d(psi_i), np.complex128)
    o = np.ascontiguousarray(orb, np.complex128)
    g = f.shape[0]
    out = np.zeros((g, g), np.complex128)
    lib().or_step_inner_prod(_ptr(bb), len(bb), _ptr(f), _ptr(i), g, _ptr(o), len(o), _ptr(out))
    return out


def bracket2(bra_basis, bra, ket_basis, ket, list2, list1) -> complex:
    """<bra| op2 op1 |ket> over two completed term lists (multiplication.jl:174-190, 215-222)."""
    bb = np.ascontiguousarray(bra_basis, np.uint64)
    kb = np.ascontiguousarray(ket_basis, np.uint64)
    bv = np.ascontiguousarray(bra, np.complex128)
    kv = np.ascontiguousarray(ket, np.complex128)
    l2 = np.ascontiguousarray(list2, SCAT_DTYPE)
    l1 = np.ascontiguousarray(list1, SCAT_DTYPE)
    out = np.zeros(2)
    lib().or_bracket2(_ptr(bb), len(bb), _ptr(bv), _ptr(kb), len(kb), _ptr(kv), _ptr(l2), len(l2), _ptr(l1),
                      len(l1), _ptr(out))
    return complex(out[0], out[1])


def sparse_csc(basis: np.ndarray, full_list: np.ndarray):
    """The sparse method's matrix (sparse_matrix.jl:64-190): 0-based CSC (colptr, rowval, nzval)
    with rows sorted inside each column and duplicates summed."""
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    N = len(basis)
    colptr = np.zeros(N + 1, np.int64)
    nnz = lib().or_sparse_csc(_ptr(basis), N, _ptr(full_list), len(full_list), _ptr(colptr), None, None, 0)
    rowval = np.zeros(max(nnz, 1), np.int64)
    nzval = np.zeros(max(nnz, 1), np.complex128)
    lib().or_sparse_csc(_ptr(basis), N, _ptr(full_list), len(full_list), _ptr(colptr), _ptr(rowval), _ptr(nzval),
                        nnz)
    return colptr, rowval[:nnz], nzval[:nnz]


def count_hits(basis: np.ndarray, full_list: np.ndarray, nthreads: int = 0) -> int:
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    return int(lib().or_count_hits(_ptr(basis), len(basis), _ptr(full_list), len(full_list), nthreads))


def eigsolve(basis, full_list, nev, krylovdim=30, tol=1e-12, maxiter=100, vec0=None, seed=0,
             nthreads=0, want_vectors=True):
    """FP64 thick-restart Lanczos (the eigensolver restatement). Returns (vals, vecs[nev, N], resid, info)."""
    basis = np.ascontiguousarray(basis, np.uint64)
    full_list = np.ascontiguousarray(full_list, SCAT_DTYPE)
    N = len(basis)
    nev = min(nev, N)
    vals = np.zeros(nev)
    resid = np.zeros(nev)
    vecs = np.zeros((nev, N), np.complex128) if want_vectors else None
    v0 = None if vec0 is None else np.ascontiguousarray(vec0, np.complex128)
    info = _Info()
    rc = lib().or_eigsolve(_ptr(basis), N, _ptr(full_list), len(full_list), nev, krylovdim, tol, maxiter,
                           _ptr(v0), seed, nthreads, _ptr(vals), _ptr(vecs), _ptr(resid), C.byref(info))
    if rc != 0:
        raise RuntimeError(f"or_eigsolve failed ({rc})")
    return vals, vecs, resid, {"converged": info.converged, "restarts": info.restarts, "matvecs": info.matvecs}
