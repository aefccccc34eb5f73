"""ctypes bindings of libmomed_b200.so (include/momed.h).

The shared library is built in-tree by ``make -C momentumed.jl_b200`` (or
``__graft_entry__.build()``) into ``momentumed.jl_b200/lib/``.  There is no
CPU fallback: if the library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libmomed_b200.so")

OK, EINVAL, ENOMEM, ECUDA, ENOTCONV, ETIMEOUT, ESTATE, ENODEV = range(8)
C128, C64 = 0, 1
RECIPE_LANDAU_COULOMB = 1
PREC_FP64, PREC_MIXED = 0, 1


class MomedError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"momed error {code}: {msg}")
        self.code = code


class NotConverged(MomedError):
    pass


class Para(C.Structure):
    _fields_ = [("dim", C.c_int32), ("Nk", C.c_int32), ("Nc_mix", C.c_int32), ("Nc_conserve", C.c_int32),
                ("k_list", C.POINTER(C.c_int64)), ("Gk", C.POINTER(C.c_int64))]


class SolveOpts(C.Structure):
    _fields_ = [("nev", C.c_int32), ("krylovdim", C.c_int32), ("maxiter", C.c_int32), ("precision", C.c_int32),
                ("tol", C.c_double), ("seed", C.c_uint64), ("want_vectors", C.c_int32),
                ("vecs_on_device", C.c_int32)]


class Info(C.Structure):
    _fields_ = [("converged", C.c_int32), ("restarts", C.c_int32), ("matvecs", C.c_int64),
                ("matvecs_fp64", C.c_int64), ("seconds", C.c_double)]


_lib = None

# every symbol include/momed.h declares, with its ctypes signature
SIGNATURES = {
    "momed_version": (C.c_char_p, []),
    "momed_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "momed_destroy": (C.c_int, [C.c_void_p]),
    "momed_last_error": (C.c_char_p, [C.c_void_p]),
    "momed_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "momed_set_hbm_budget": (C.c_int, [C.c_void_p, C.c_int64]),
    "momed_enumerate_basis": (C.c_int, [C.c_void_p, C.POINTER(Para), C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                        C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "momed_enumeration_copy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "momed_select_sector": (C.c_int, [C.c_void_p, C.c_int64]),
    "momed_enumerate_sector_noalloc": (C.c_int, [C.POINTER(Para), C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                                 C.c_int64, C.POINTER(C.c_int64), C.c_void_p]),
    "momed_set_basis": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]),
    "momed_set_scatter": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "momed_set_scatter_pair": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int64]),
    "momed_set_param": (C.c_int, [C.c_void_p, C.c_double]),
    "momed_matvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "momed_eigsolve": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(Info)]),
    "momed_set_twobody_recipe": (C.c_int, [C.c_void_p, C.POINTER(Para), C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                           C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64]),
    "momed_set_kshift": (C.c_int, [C.c_void_p, C.c_void_p]),
    "momed_block_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "momed_eigsolve_general": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.POINTER(Info)]),
    "momed_batch_solve": (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_int32, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(Info)]),
    "momed_build_sparse": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "momed_sparse_copy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "momed_release_sparse": (C.c_int, [C.c_void_p]),
    "momed_build_hit_cache": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "momed_hit_cache_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "momed_release_hit_cache": (C.c_int, [C.c_void_p]),
    "momed_set_sparse_csr": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "momed_bracket": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "momed_rdm1": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "momed_step_inner_prod": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                        C.c_void_p]),
    "momed_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "momed_last_kernel_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "momed_kernel_launches": (C.c_int64, []),
    "momed_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "momed_profile_read": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
}

SIGNATURES.update({
    "momed_serve_start": (C.c_int, [C.c_int, C.c_int32, C.c_int64, C.POINTER(C.c_void_p)]),
    "momed_serve_register_operator": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_int64, C.POINTER(C.c_int32)]),
    "momed_serve_submit": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_double,
                                     C.POINTER(SolveOpts), C.POINTER(C.c_int64)]),
    "momed_serve_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "momed_serve_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p,
                                   C.POINTER(Info), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "momed_serve_stats": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_int64)] * 5),
    "momed_serve_last_error": (C.c_char_p, [C.c_void_p]),
    "momed_serve_stop": (C.c_int, [C.c_void_p]),
})

(KERNEL_MATVEC_C128, KERNEL_MATVEC_C64, KERNEL_BLOCK_MATVEC_C64, KERNEL_BLOCK_MATVEC_C128, KERNEL_SPMV_C128,
 KERNEL_SPMV_C64, KERNEL_BLOCK_SPMV_C64, KERNEL_HC_MATVEC_C128, KERNEL_HC_MATVEC_C64, KERNEL_HC_BLOCK_C64,
 KERNEL_HC_BLOCK_C128) = range(11)
QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)


class Server:
    """Continuous-batching solve server (momed_serve_*): submit requests any time, poll results."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: int = 0):
        s = C.c_void_p()
        rc = lib().momed_serve_start(device, slots, hbm_budget, C.byref(s))
        if rc != OK:
            raise MomedError(rc, "momed_serve_start failed")
        self._s = s

    def _err(self, rc):
        raise MomedError(rc, lib().momed_serve_last_error(self._s).decode())

    def register_operator(self, amp_a, amp_b, in_, out, parity=None) -> int:
        a = np.ascontiguousarray(amp_a, np.complex128)
        b = None if amp_b is None else np.ascontiguousarray(amp_b, np.complex128)
        i = np.ascontiguousarray(in_, np.uint64)
        o = np.ascontiguousarray(out, np.uint64)
        p = None if parity is None else np.ascontiguousarray(parity, np.uint64)
        op = C.c_int32()
        rc = lib().momed_serve_register_operator(self._s, _p(a), _p(b), _p(i), _p(o), _p(p), len(a), C.byref(op))
        if rc != OK:
            self._err(rc)
        return op.value

    def submit(self, op_id: int, basis, u: float, nev: int, tol: float = 1e-12, krylovdim: int = 30,
               maxiter: int = 100, precision: int = PREC_FP64, seed: int = 0) -> int:
        b = np.ascontiguousarray(basis, np.uint64)
        opts = SolveOpts(nev, krylovdim, maxiter, precision, tol, seed, 0, 0)
        rid = C.c_int64()
        rc = lib().momed_serve_submit(self._s, op_id, _p(b), len(b), float(u), C.byref(opts), C.byref(rid))
        if rc != OK:
            self._err(rc)
        return rid.value

    def cancel(self, rid: int) -> int:
        return lib().momed_serve_cancel(self._s, rid)

    def poll(self, rid: int, nev: int, wait_ms: int = 0):
        """(status, vals, resid, info, queue_s, latency_s); raises on a failed request."""
        st = C.c_int32()
        vals, resid = np.zeros(nev), np.zeros(nev)
        info = Info()
        q, lat = C.c_double(), C.c_double()
        rc = lib().momed_serve_poll(self._s, rid, wait_ms, C.byref(st), _p(vals), _p(resid), C.byref(info),
                                    C.byref(q), C.byref(lat))
        if rc not in (OK, ETIMEOUT):
            self._err(rc)
        return st.value, vals, resid, {"converged": info.converged, "matvecs": info.matvecs,
                                       "seconds": info.seconds}, q.value, lat.value

    def stats(self):
        v = [C.c_int64() for _ in range(5)]
        lib().momed_serve_stats(self._s, *[C.byref(x) for x in v])
        return dict(zip(("queued", "completed", "failed", "hbm_used", "hbm_budget"), (x.value for x in v)))

    def stop(self):
        if getattr(self, "_s", None):
            lib().momed_serve_stop(self._s)
            self._s = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def kernel_launches() -> int:
    """Kernels the library has launched in this process."""
    return int(lib().momed_kernel_launches())


def lib():
    """Load the library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MomedError(ENODEV, f"{LIB_PATH} is missing: build it with `make -C momentumed.jl_b200` "
                                     "(this backend has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def version() -> str:
    return lib().momed_version().decode()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Handle:
    """One device context of the library: a working basis, an operator and scratch buffers."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        rc = L.momed_create(device, C.byref(h))
        if rc != OK:
            raise MomedError(rc, L.momed_last_error(None).decode())
        self._h = h
        self.n = 0

    # ---------------------------------------------------------------- plumbing
    def _check(self, rc: int):
        if rc == OK:
            return
        msg = lib().momed_last_error(self._h).decode()
        if rc == ENOTCONV:
            raise NotConverged(rc, msg or "not converged")
        raise MomedError(rc, msg)

    def close(self):
        if getattr(self, "_h", None):
            lib().momed_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        self._check(lib().momed_set_stream(self._h, C.c_void_p(stream_ptr)))

    # ---------------------------------------------------------------- basis
    def enumerate_basis(self, k_list: np.ndarray, Gk, Nc_mix: int, Nc_conserve: int, N_each, mask=None,
                        momentum_list=None):
        k_list = np.asarray(k_list, np.int64)
        dim, Nk = k_list.shape
        kl = np.ascontiguousarray(k_list.T).reshape(-1)
        g = np.asarray(Gk, np.int64)
        para = Para(dim, Nk, Nc_mix, Nc_conserve, kl.ctypes.data_as(C.POINTER(C.c_int64)),
                    g.ctypes.data_as(C.POINTER(C.c_int64)))
        ne = np.asarray(N_each, np.int64)
        marr = None if mask is None else np.asarray(sorted(mask), np.int64)
        mom = None if momentum_list is None else np.asarray(momentum_list, np.int64).reshape(-1)
        nsec, ntot = C.c_int64(), C.c_int64()
        self._check(lib().momed_enumerate_basis(self._h, C.byref(para), _p(ne), len(ne), _p(marr),
                                                -1 if marr is None else len(marr), _p(mom),
                                                -1 if mom is None else len(mom) // dim, C.byref(nsec),
                                                C.byref(ntot)))
        ks = np.zeros(max(nsec.value * dim, 1), np.int64)
        sizes = np.zeros(max(nsec.value, 1), np.int64)
        basis = np.zeros(max(ntot.value, 1), np.uint64)
        self._check(lib().momed_enumeration_copy(self._h, _p(ks), _p(sizes), _p(basis), 0))
        out, off = [], 0
        for s in range(nsec.value):
            out.append((tuple(int(v) for v in ks[s * dim:(s + 1) * dim]), basis[off:off + sizes[s]]))
            off += int(sizes[s])
        return out

    def set_twobody_recipe(self, para, kind: int, params, raw, upper_start, entry_upper, entry_partner):
        """Attach the device recipe of the working operator's two-body terms (momed_set_twobody_recipe)."""
        k_list = np.asarray(para.k_list, np.int64)
        dim, Nk = k_list.shape
        kl = np.ascontiguousarray(k_list.T).reshape(-1)
        g = np.asarray(para.Gk, np.int64)
        p = Para(dim, Nk, para.Nc_mix, para.Nc_conserve, kl.ctypes.data_as(C.POINTER(C.c_int64)),
                 g.ctypes.data_as(C.POINTER(C.c_int64)))
        prm = np.ascontiguousarray(params, np.float64)
        raw = np.ascontiguousarray(raw, np.int32).reshape(-1, 9)
        us = np.ascontiguousarray(upper_start, np.int64)
        eu = np.ascontiguousarray(entry_upper, np.int64)
        ep = np.ascontiguousarray(entry_partner, np.int32)
        self._check(lib().momed_set_twobody_recipe(self._h, C.byref(p), kind, _p(prm), len(prm), _p(raw), len(raw),
                                                   _p(us), len(us) - 1, _p(eu), _p(ep), len(eu)))

    def block_tuning(self, nb: int, precision: int = PREC_MIXED, has_param: bool = True):
        """The block map autotuner's choice for this operator / sector class (None before tuning)."""
        r, g, a, b = C.c_int32(), C.c_int32(), C.c_double(), C.c_double()
        rc = lib().momed_block_tuning(self._h, nb, precision, int(has_param), C.byref(r), C.byref(g), C.byref(a),
                                      C.byref(b))
        if rc == ESTATE:
            return None
        self._check(rc)
        return {"rows_per_warp": r.value, "grid": ["resident-1", "resident", "2x resident"][g.value],
                "ms": a.value, "ms_default": b.value}

    def set_kshift(self, kshift):
        """Regenerate the recipe's amplitudes on the device at kshift [Nc_conserve][dim]."""
        k = np.ascontiguousarray(kshift, np.float64)
        self._check(lib().momed_set_kshift(self._h, _p(k)))

    def select_sector(self, s: int, n: int):
        self._check(lib().momed_select_sector(self._h, s))
        self.n = n

    def set_basis(self, basis, on_device: bool = False, n: int | None = None):
        if on_device:
            self._check(lib().momed_set_basis(self._h, C.c_void_p(basis), n, 1))
            self.n = n
        else:
            b = np.ascontiguousarray(basis, np.uint64)
            self._check(lib().momed_set_basis(self._h, _p(b), len(b), 0))
            self.n = len(b)

    # ---------------------------------------------------------------- operator
    def set_scatter(self, amp: np.ndarray, in_: np.ndarray, out: np.ndarray, parity: np.ndarray | None = None):
        a = np.ascontiguousarray(amp, np.complex128)
        i = np.ascontiguousarray(in_, np.uint64)
        o = np.ascontiguousarray(out, np.uint64)
        p = None if parity is None else np.ascontiguousarray(parity, np.uint64)
        self._check(lib().momed_set_scatter(self._h, _p(a), _p(i), _p(o), _p(p), len(a)))

    def set_scatter_pair(self, amp_a, amp_b, in_, out, parity=None):
        a = np.ascontiguousarray(amp_a, np.complex128)
        b = np.ascontiguousarray(amp_b, np.complex128)
        i = np.ascontiguousarray(in_, np.uint64)
        o = np.ascontiguousarray(out, np.uint64)
        p = None if parity is None else np.ascontiguousarray(parity, np.uint64)
        self._check(lib().momed_set_scatter_pair(self._h, _p(a), _p(b), _p(i), _p(o), _p(p), len(a)))

    def set_param(self, u: float):
        self._check(lib().momed_set_param(self._h, float(u)))

    def set_hbm_budget(self, nbytes: int):
        """Device-memory limit for this handle's admissions (0 = free memory)."""
        self._check(lib().momed_set_hbm_budget(self._h, int(nbytes)))

    # ---------------------------------------------------------------- compute
    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = H x with host arrays (complex128 or complex64)."""
        prec = C64 if x.dtype == np.complex64 else C128
        x = np.ascontiguousarray(x, np.complex64 if prec == C64 else np.complex128)
        y = np.empty_like(x)
        self._check(lib().momed_matvec(self._h, _p(x), _p(y), prec, 0))
        return y

    def matvec_device(self, x_ptr: int, y_ptr: int, precision: int = C128):
        self._check(lib().momed_matvec(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), precision, 1))

    def last_kernel_ms(self) -> float:
        v = C.c_double()
        self._check(lib().momed_last_kernel_ms(self._h, C.byref(v)))
        return v.value

    def profile(self, enable: bool = True):
        self._check(lib().momed_profile(self._h, int(enable)))

    def profile_read(self, kind: int = KERNEL_BLOCK_MATVEC_C64):
        """(launches, summed device ms) of one matvec kernel kind since profile(True)."""
        n, ms = C.c_int64(), C.c_double()
        self._check(lib().momed_profile_read(self._h, kind, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def bracket(self, bra: np.ndarray, ket: np.ndarray, bra_basis=None) -> complex:
        """<bra| H |ket>: ket on the working basis, bra on bra_basis (None: the working basis)."""
        k = np.ascontiguousarray(ket, np.complex128)
        b = np.ascontiguousarray(bra, np.complex128)
        out = np.zeros(2)
        if bra_basis is None:
            self._check(lib().momed_bracket(self._h, None, 0, _p(b), _p(k), _p(out)))
        else:
            bb = np.ascontiguousarray(bra_basis, np.uint64)
            if len(bb) != len(b):
                raise MomedError(EINVAL, "bra and bra_basis lengths differ")
            self._check(lib().momed_bracket(self._h, _p(bb), len(bb), _p(b), _p(k), _p(out)))
        return complex(out[0], out[1])

    def rdm1(self, psi: np.ndarray, norb: int) -> np.ndarray:
        """One-body reduced density matrix [norb, norb] of psi on the working basis."""
        v = np.ascontiguousarray(psi, np.complex128)
        out = np.zeros((norb, norb), np.complex128)
        self._check(lib().momed_rdm1(self._h, _p(v), int(norb), _p(out)))
        return out

    def step_inner_prod(self, psi_f: np.ndarray, psi_i: np.ndarray, orb: np.ndarray) -> np.ndarray:
        """[g, g] many-body connection step of [g, N] vectors on the working basis."""
        f = np.ascontiguousarray(np.atleast_2d(psi_f), np.complex128)
        i = np.ascontiguousarray(np.atleast_2d(psi_i), np.complex128)
        o = np.ascontiguousarray(orb, np.complex128)
        if f.shape != i.shape or f.shape[1] != self.n:
            raise MomedError(EINVAL, "psi_f and psi_i must both be [g, N] on the working basis")
        out = np.zeros((f.shape[0], f.shape[0]), np.complex128)
        self._check(lib().momed_step_inner_prod(self._h, _p(f), _p(i), f.shape[0], _p(o), len(o), _p(out)))
        return out

    # ---------------------------------------------------------------- sparse method
    def build_sparse(self) -> int:
        """CSR matrix of the working operator (at the current u) on the device; maps and
        eigsolve use it until the basis, operator or u changes.  Returns the stored entries."""
        nnz = C.c_int64()
        self._check(lib().momed_build_sparse(self._h, C.byref(nnz)))
        self._sparse_nnz = nnz.value
        return nnz.value

    def sparse_copy(self):
        """(row_ptr int64[n + 1], col int32[nnz], val complex128[nnz]) of the built matrix."""
        nnz = getattr(self, "_sparse_nnz", None)
        if nnz is None:
            raise MomedError(ESTATE, "no sparse matrix (build_sparse)")
        rp = np.empty(self.n + 1, np.int64)
        col = np.empty(max(nnz, 1), np.int32)
        val = np.empty(max(nnz, 1), np.complex128)
        self._check(lib().momed_sparse_copy(self._h, _p(rp), _p(col), _p(val)))
        return rp, col[:nnz], val[:nnz]

    def set_sparse_csr(self, row_ptr, col, val):
        """Upload a host CSR matrix (int64 row_ptr[n + 1], int32 col, complex128 val); the handle
        then multiplies by it with no basis or operator (create_gpu_matrix of a host matrix)."""
        rp = np.ascontiguousarray(row_ptr, np.int64)
        c = np.ascontiguousarray(col, np.int32)
        v = np.ascontiguousarray(val, np.complex128)
        if len(c) != rp[-1] or len(v) != rp[-1]:
            raise MomedError(EINVAL, "col and val must hold row_ptr[-1] entries")
        self._check(lib().momed_set_sparse_csr(self._h, len(rp) - 1, _p(rp), _p(c), _p(v)))
        self.n = len(rp) - 1
        self._sparse_nnz = int(rp[-1])

    def release_sparse(self):
        self._check(lib().momed_release_sparse(self._h))
        self._sparse_nnz = None

    # ---------------------------------------------------------------- hit cache of the map
    def build_hit_cache(self) -> dict:
        """Record every off-diagonal hit's target row and term slot for the working basis and
        operator, so that maps skip the candidate stage; the eigensolvers build it by themselves
        when it fits a quarter of the free device memory (MOMED_HITCACHE=0 turns that off)."""
        hits, nbytes = C.c_int64(), C.c_int64()
        self._check(lib().momed_build_hit_cache(self._h, C.byref(hits), C.byref(nbytes)))
        return self.hit_cache_info()

    def hit_cache_info(self):
        """{"hits", "bytes", "build_ms", "mode"} of the built hit cache (mode "full": target and
        term slot per hit; "slots": the term slot only), or None."""
        built, hits, nbytes, ms = C.c_int32(), C.c_int64(), C.c_int64(), C.c_double()
        self._check(lib().momed_hit_cache_info(self._h, C.byref(built), C.byref(hits), C.byref(nbytes), C.byref(ms)))
        if not built.value:
            return None
        return {"hits": hits.value, "bytes": nbytes.value, "build_ms": ms.value,
                "mode": "full" if built.value == 1 else "slots"}

    def release_hit_cache(self):
        self._check(lib().momed_release_hit_cache(self._h))

    def stats(self):
        nnz, mode, tb = C.c_int64(), C.c_int32(), C.c_int64()
        self._check(lib().momed_stats(self._h, C.byref(nnz), C.byref(mode), C.byref(tb)))
        return {"nnz": nnz.value, "index_mode": mode.value, "table_bytes": tb.value}

    def eigsolve(self, nev: int, krylovdim: int = 30, tol: float = 1e-12, maxiter: int = 100,
                 vec0: np.ndarray | None = None, seed: int = 0, precision: int = PREC_FP64,
                 want_vectors: bool = True, raise_on_notconv: bool = False):
        n = self.n
        nev_eff = min(nev, n)
        opts = SolveOpts(nev, krylovdim, maxiter, precision, tol, seed, int(want_vectors), 0)
        vals = np.zeros(nev_eff)
        resid = np.zeros(nev_eff)
        vecs = np.zeros((nev_eff, n), np.complex128) if want_vectors else None
        v0 = None if vec0 is None else np.ascontiguousarray(vec0, np.complex128)
        info = Info()
        rc = lib().momed_eigsolve(self._h, C.byref(opts), _p(v0), _p(vals), _p(resid), _p(vecs), C.byref(info))
        if rc not in (OK, ENOTCONV) or (rc == ENOTCONV and raise_on_notconv):
            self._check(rc)
        return vals, vecs, resid, {"converged": info.converged, "restarts": info.restarts,
                                   "matvecs": info.matvecs, "matvecs_fp64": info.matvecs_fp64,
                                   "seconds": info.seconds}

    def eigsolve_general(self, nev: int, krylovdim: int = 30, tol: float = 1e-12, maxiter: int = 100,
                         vec0: np.ndarray | None = None, seed: int = 0, want_vectors: bool = True,
                         raise_on_notconv: bool = False):
        """Non-Hermitian operator (its term list set as it is): complex eigenvalues ordered by
        real part, right eigenvectors, residuals (momed_eigsolve_general)."""
        n = self.n
        nev_eff = min(nev, n)
        opts = SolveOpts(nev, krylovdim, maxiter, PREC_FP64, tol, seed, int(want_vectors), 0)
        vals = np.zeros(2 * nev_eff)
        resid = np.zeros(nev_eff)
        vecs = np.zeros((nev_eff, n), np.complex128) if want_vectors else None
        v0 = None if vec0 is None else np.ascontiguousarray(vec0, np.complex128)
        info = Info()
        rc = lib().momed_eigsolve_general(self._h, C.byref(opts), _p(v0), _p(vals), _p(resid), _p(vecs),
                                          C.byref(info))
        if rc not in (OK, ENOTCONV) or (rc == ENOTCONV and raise_on_notconv):
            self._check(rc)
        return (vals[0::2] + 1j * vals[1::2], vecs, resid,
                {"converged": info.converged, "restarts": info.restarts, "matvecs": info.matvecs,
                 "matvecs_fp64": info.matvecs_fp64, "seconds": info.seconds})

    def batch_solve(self, u: np.ndarray, nev: int, krylovdim: int = 30, tol: float = 1e-12, maxiter: int = 100,
                    seed: int = 0, precision: int = PREC_MIXED, want_vectors: bool = False,
                    out_vecs: np.ndarray | None = None):
        """out_vecs: optional caller-owned C-contiguous complex128 array of shape (len(u), nev, n)
        (pinned host memory makes the copy-out fast); used instead of a fresh array."""
        u = np.ascontiguousarray(u, np.float64)
        n = self.n
        nev_eff = min(nev, n)
        opts = SolveOpts(nev, krylovdim, maxiter, precision, tol, seed, int(want_vectors), 0)
        vals = np.zeros((len(u), nev_eff))
        resid = np.zeros((len(u), nev_eff))
        vecs = None
        if want_vectors:
            if out_vecs is not None:
                if (out_vecs.dtype != np.complex128 or out_vecs.shape != (len(u), nev_eff, n)
                        or not out_vecs.flags.c_contiguous):
                    raise ValueError(f"out_vecs must be C-contiguous complex128 of shape {(len(u), nev_eff, n)}")
                vecs = out_vecs
            else:
                vecs = np.zeros((len(u), nev_eff, n), np.complex128)
        info = Info()
        rc = lib().momed_batch_solve(self._h, C.byref(opts), _p(u), len(u), _p(vals), _p(resid), _p(vecs),
                                     C.byref(info))
        if rc not in (OK, ENOTCONV):
            self._check(rc)
        return vals, vecs, resid, {"converged": info.converged, "restarts": info.restarts,
                                   "matvecs": info.matvecs, "matvecs_fp64": info.matvecs_fp64,
                                   "seconds": info.seconds}
