"""The enumeration entry point that allocates no device memory.

Some callers cannot call cudaMalloc: their device memory belongs to another allocator (a
Julia CUDA.jl pool, a framework's caching allocator) or was reserved up front for solve
slots.  momed_enumerate_sector_noalloc lets them enumerate a sector straight into a buffer
they own; its working space is a static device array shared by all calls.

This test drives it through the C ABI with a caller-owned (torch) buffer and checks it
against the existing entry point (momed_enumerate_basis) bit for bit, for several sectors
and on two calls in a row (the shared scratch keeps the previous call's contents), plus the
too-small-buffer path, which must write nothing and report the size needed.
"""
import ctypes as C

import numpy as np
import pytest

import momed
from momed import _lib

pytestmark = pytest.mark.gpu


def _para(k_list, Gk, Nc_mix=1, Nc_conserve=1):
    k_list = np.asarray(k_list, np.int64)
    dim, Nk = k_list.shape
    kl = np.ascontiguousarray(k_list.T).reshape(-1)
    g = np.asarray(Gk, np.int64)
    p = _lib.Para(dim, Nk, Nc_mix, Nc_conserve, kl.ctypes.data_as(C.POINTER(C.c_int64)),
                  g.ctypes.data_as(C.POINTER(C.c_int64)))
    return p, (kl, g)


def noalloc(para, N_each, momentum, out, stream=None):
    ne = np.asarray(N_each, np.int64)
    mom = np.asarray(momentum, np.int64)
    n = C.c_int64(-1)
    rc = _lib.lib().momed_enumerate_sector_noalloc(C.byref(para), ne.ctypes.data_as(C.c_void_p), len(ne),
                                                    mom.ctypes.data_as(C.c_void_p),
                                                    C.c_void_p(out.data_ptr()), out.numel(), C.byref(n),
                                                    C.c_void_p(stream))
    return rc, n.value


@pytest.mark.parametrize("mesh,N_each,ncc", [((3, 9), (9,), 1), ((3, 5), (5,), 1), ((4, 3), (3, 3), 2)])
def test_noalloc_matches_enumerate_basis(mesh, N_each, ncc):
    import torch
    from momed.synthetic import mesh_klist

    a, b = mesh
    kl = mesh_klist(a, b)
    h = momed.Handle(0)
    ref = h.enumerate_basis(kl, (a, b), 1, ncc, N_each)        # existing entry point
    h.close()
    para, keep = _para(kl, (a, b), 1, ncc)
    out = torch.zeros(max(len(s) for _, s in ref) + 7, dtype=torch.int64, device="cuda")
    for call in range(2):                                         # two calls in a row
        for k, basis in ref[::max(1, len(ref) // 5)]:
            out.fill_(-1)
            torch.cuda.synchronize()
            rc, n = noalloc(para, N_each, k, out)
            assert rc == _lib.OK and n == len(basis)
            got = out[:n].cpu().numpy().view(np.uint64)
            assert np.array_equal(got, basis), (call, k)
            assert int(out[n].item()) == -1                       # nothing written past the sector


def test_noalloc_rejects_small_buffer_and_empty_sector():
    import torch
    from momed.synthetic import mesh_klist

    kl = mesh_klist(3, 5)
    para, keep = _para(kl, (3, 5))
    out = torch.full((10,), -1, dtype=torch.int64, device="cuda")
    rc, n = noalloc(para, (5,), (1, 2), out)
    assert rc == _lib.EINVAL and n > 10
    assert bool((out == -1).all())                                # nothing written
    big = torch.zeros(n, dtype=torch.int64, device="cuda")
    rc, n2 = noalloc(para, (5,), (1, 2), big)
    assert rc == _lib.OK and n2 == n
    # a momentum outside the reachable box is an empty sector
    kl2 = np.array([[0, 1, 2, 0, 1, 2], [0, 0, 0, 1, 1, 1]], np.int64)
    para2, keep2 = _para(kl2, (3, 0))
    rc, n3 = noalloc(para2, (2,), (0, 9), big)
    assert rc == _lib.OK and n3 == 0
