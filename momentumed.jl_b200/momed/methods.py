"""Host mirror of MomentumED's matrix-free methods, backed by libmomed_b200.

  - ``LinearMap`` ........... MomentumED/src/method/linear_map.jl:18-42 (Hermitian completion + sort)
  - GPU plugin hooks ........ MomentumED/src/method/gpu_interface.jl:13-94
      GPU_AVAILABLE, DEFAULT_GPU, activate_gpu_device, create_gpu_linearmap,
      krylov_map_solve, release_gpu_memory
  - ``EDsolve`` ............. MomentumED/src/MomentumED.jl:375-480 (method=:map or :sparse, device=:gpu)
  - sparse method ........... create_gpu_matrix / krylov_matrix_solve (MomentumEDCUDAExt.jl:145-200), the
                              matrix built on the device instead of by sparse_matrix.jl:64-190

The device map computes H x (the CPU LinearMap semantics, linear_map.jl:100-118);
the reference's KernelAbstractions kernel computes conj(H) x, so its eigenvectors
are the complex conjugates of these.  Eigenvalues are identical.
"""
from __future__ import annotations

import warnings

import numpy as np

from . import _lib
from .core import HilbertSubspace, MBOperator, MBS64Vector, ScatterList, hermitian_complete

GPU_AVAILABLE = {"cuda": False, "oneapi": False, "metal": False, "multi_cuda": False, "b200": False}
DEFAULT_GPU = ["nogpu"]
GPU_RESTART_CHUNKSIZE = [262144]   # kept for API parity; the device restart needs no chunking
GPU_MEMORY_MONITOR = [False]


def activate_b200(device: int = 0, set_default_gpu: bool = True) -> bool:
    """Probe the B200 backend (loads the library and opens a device context)."""
    try:
        h = _lib.Handle(device)
        h.close()
        GPU_AVAILABLE["b200"] = True
        if set_default_gpu or DEFAULT_GPU[0] == "nogpu":
            DEFAULT_GPU[0] = "b200"
    except _lib.MomedError:
        GPU_AVAILABLE["b200"] = False
    return GPU_AVAILABLE["b200"]


def activate_gpu_device(device: str, set_default_gpu: bool = True):
    if device not in GPU_AVAILABLE:
        raise ValueError(f"Unknown GPU {device}. Valid options are: {list(GPU_AVAILABLE)}.")
    if device in ("b200", "cuda"):
        return activate_b200(set_default_gpu=set_default_gpu)
    GPU_AVAILABLE[device] = False
    return False


def _throw_gpu_unavailable(device: str):
    if GPU_AVAILABLE.get(device, False):
        return
    try:
        activate_gpu_device(device, set_default_gpu=False)
    except ValueError:
        pass
    if GPU_AVAILABLE.get(device, False):
        return
    raise ValueError(f"device=:{device} requires functional GPU(s) of the type. "
                     "Load the required package(s) and verify GPU availability.")


class LinearMap:
    """Matrix-free map: the Hermitian-completed sorted term list over a subspace (linear_map.jl:18-42)."""

    def __init__(self, op: MBOperator, space: HilbertSubspace):
        et = op.scats.element_type
        if et not in (np.complex128, np.complex64):
            raise AssertionError(f"element_type={et}. Use Complex of Float64, Float32.")
        self.scat_list: ScatterList = hermitian_complete(op)
        self.space = space
        self.element_type = et
        self.hermitian = op.upper_hermitian      # the completed list of an upper operator is Hermitian

    @property
    def size(self):
        n = len(self.space)
        return (n, n)


def adjoint_list(s: ScatterList) -> ScatterList:
    """Terms of the adjoint operator: conj(amp), in and out swapped, sorted by (in, out)."""
    order = np.lexsort((s.in_, s.out))
    return ScatterList(np.conj(s.amp[order]), s.in_[order], s.out[order], s.pm[order], s.bits, s.element_type)


class B200LinearMap:
    """The device map (the role of CuLinearMap, MomentumEDCUDAExt.jl:55-139)."""

    def __init__(self, A: LinearMap, device: int = 0, handle: _lib.Handle | None = None, adjoint: bool = False):
        self.space = A.space
        self.element_type = A.element_type
        self._A, self._device, self._adjoint = A, device, adjoint
        self.handle = handle or _lib.Handle(device)
        self.handle.set_basis(A.space.list)
        s = adjoint_list(A.scat_list) if adjoint else A.scat_list
        self.handle.set_scatter(s.amp.astype(np.complex128), s.in_, s.out, s.pm)

    @property
    def size(self):
        n = len(self.space)
        return (n, n)

    @property
    def eltype(self):
        return self.element_type

    def __call__(self, x, y=None):
        prec_dtype = np.complex64 if self.element_type is np.complex64 else np.complex128
        out = self.handle.matvec(np.asarray(x, prec_dtype))
        if y is not None:
            y[...] = out
            return y
        return out

    def adjoint(self):
        """The adjoint map (AdjointLinearMap, linear_map.jl:48-55, 120-139; the GPU kernel
        ka_adjoint_linearmap_kernel!, gpu_interface.jl:170-205): the map of a Hermitian-completed
        operator is itself; otherwise a device map over the adjoint terms (conjugated amplitudes,
        creation and annihilation masks swapped), on its own handle."""
        if self._A.hermitian:
            return self
        return B200LinearMap(self._A, self._device, adjoint=not self._adjoint)

    def release(self):
        self.handle.close()


def create_gpu_linearmap(A: LinearMap, device: str = "b200") -> B200LinearMap:
    return B200LinearMap(A)


def krylov_map_solve(H: B200LinearMap, N_eigen: int, *, ishermitian: bool = True, vec0=None,
                     krylovdim: int = 30, tol: float = 1e-12, maxiter: int = 100, seed: int = 0,
                     precision: str = "fp64", verbosity: int = 0):
    """Lowest N_eigen eigenpairs (:SR) of the device map; returns (vals, vecs, info).

    ishermitian=False (a map of a non-Hermitian operator): Arnoldi with Krylov-Schur restarts,
    complex eigenvalues ordered by real part (KrylovKit eigsolve(:SR; ishermitian = false))."""
    m = H.size[0]
    if not ishermitian:
        if getattr(H, "hermitian", False):
            warnings.warn("ishermitian=false on a Hermitian map: solved as a general matrix")
        vals, vecs, resid, info = H.handle.eigsolve_general(min(N_eigen, m), krylovdim=krylovdim, tol=tol,
                                                            maxiter=maxiter, vec0=vec0, seed=seed)
        info = dict(info)
        info["residuals"] = resid
        return vals, [vecs[i] for i in range(len(vals))], info
    N_eigen = min(N_eigen, m)
    prec = _lib.PREC_MIXED if precision == "mixed" else _lib.PREC_FP64
    vals, vecs, resid, info = H.handle.eigsolve(N_eigen, krylovdim=krylovdim, tol=tol, maxiter=maxiter,
                                                vec0=vec0, seed=seed, precision=prec)
    info = dict(info)
    info["residuals"] = resid
    return vals, [vecs[i] for i in range(len(vals))], info


class B200SparseMatrix:
    """The device CSR matrix of the sparse method (the role of the CuSparseMatrixCSR that
    create_gpu_matrix uploads, MomentumEDCUDAExt.jl:145-152).  The reference builds the matrix on
    host threads (ED_HamiltonianMatrix_threaded_CSCdirect, sparse_matrix.jl:64-190) and uploads
    it; here it is built on the device from the same Hermitian-completed term list."""

    def __init__(self, A: LinearMap, device: int = 0):
        self._map = B200LinearMap(A, device)
        self.handle = self._map.handle
        self.space = A.space
        self.element_type = A.element_type
        self.nnz = self.handle.build_sparse()

    @property
    def size(self):
        n = len(self.space)
        return (n, n)

    def __call__(self, x, y=None):
        return self._map(x, y)           # the handle multiplies by the CSR matrix while it is built

    def to_host(self):
        """(row_ptr, col, val) of the CSR matrix: row i lists the diagonal first, then one entry
        per off-diagonal (row, term) hit."""
        return self.handle.sparse_copy()

    def release(self):
        self.handle.close()


class B200HostSparseMatrix:
    """A host sparse matrix uploaded to the device (create_gpu_matrix of the reference's host
    matrix, MomentumEDCUDAExt.jl:145-152): any scipy.sparse matrix, stored as CSR."""

    def __init__(self, H, device: int = 0):
        import scipy.sparse as sps
        csr = sps.csr_matrix(H, dtype=np.complex128)
        csr.sort_indices()
        self.handle = _lib.Handle(device)
        self.handle.set_sparse_csr(csr.indptr, csr.indices, csr.data)
        self.nnz = csr.nnz
        self.size = csr.shape
        self.element_type = np.complex128

    def __call__(self, x, y=None):
        out = self.handle.matvec(np.asarray(x, np.complex128))
        if y is not None:
            y[...] = out
            return y
        return out

    def release(self):
        self.handle.close()


def create_gpu_matrix(A, device: str = "b200"):
    """A LinearMap: the matrix is built on the device from its basis and term list.  A host
    scipy.sparse matrix (what SparseHmltMatrix builds, sparse_matrix.jl:64-190): uploaded."""
    if isinstance(A, LinearMap):
        return B200SparseMatrix(A)
    return B200HostSparseMatrix(A)


def krylov_matrix_solve(H: B200SparseMatrix, N_eigen: int, **kw):
    """Lowest N_eigen eigenpairs (:SR) of the device CSR matrix (krylov_matrix_solve,
    MomentumEDCUDAExt.jl:180-200); same keywords and results as krylov_map_solve."""
    return krylov_map_solve(H, N_eigen, **kw)


def release_gpu_memory(device: str = "b200", level: int = 2):
    """Device buffers belong to handles and are freed when a handle closes; nothing to collect."""
    return None


def EDsolve(subspace: HilbertSubspace, *Hamiltonian, N: int, method: str | None = None,
            device: str = "gpu", showtime: bool = False, ishermitian: bool = True, element_type=None,
            index_type=np.int32, map_warning_dim: int = 20000, method_info: bool = True, **krylovkit_kwargs):
    """Lowest N eigenpairs of the Hamiltonian in ``subspace`` on the GPU.

    Two forms, as in the reference: ``EDsolve(subspace, H::MBOperator; N, method=:map)``
    (MomentumED.jl:375-480; :map or :sparse) and ``EDsolve(subspace, scat_lists...; N,
    method=:sparse)`` (MomentumED.jl:217-372) with one or more scatter lists, whose matrix is built
    on the device from their sum (upper-Hermitian lists when ``ishermitian``).  The list form has
    no matrix-free method (the reference refuses :map there too), and this backend has no dense
    method, so small sectors also run on the device's sparse method.

    Returns ``(energies, vectors)`` with ``vectors`` a list of ``MBS64Vector``.
    ``krylovkit_kwargs`` accepts krylovdim, tol, maxiter, vec0, seed and precision ("fp64"/"mixed").
    """
    import time
    import warnings

    if len(Hamiltonian) == 1 and isinstance(Hamiltonian[0], MBOperator):
        Hamiltonian = Hamiltonian[0]
        method = "map" if method is None else method
    else:
        if not Hamiltonian or not all(isinstance(h, ScatterList) for h in Hamiltonian):
            raise TypeError("EDsolve takes one MBOperator or one or more scatter lists")
        method = "sparse" if method is None else method
        if method == "map":
            raise ValueError("Linear map methods are only supported when input Hamitonian is MBOperator instead of "
                             "Vector{Scatter}.")
        Hamiltonian = MBOperator(*Hamiltonian, upper_hermitian=ishermitian)
    if N < 1:
        raise AssertionError("N should be at least 1.")
    if len(subspace) > np.iinfo(index_type).max:
        raise AssertionError(f"Hilbert space dimension {len(subspace)} exceeds limit of index_type={index_type}.")
    if method not in ("sparse", "dense", "map"):
        raise AssertionError(f"Unknown method: {method}. Use :sparse, :dense, :map.")
    if device not in ("cpu", "gpu", "cuda", "oneapi", "metal", "multi_cuda", "b200"):
        raise AssertionError(f"Unknown device: {device}.")
    if ishermitian and not Hamiltonian.isupper():
        raise AssertionError("Use upper_hermitian form of Hamiltonian operator when ishermitian = true.")
    if method == "dense" or device == "cpu":
        raise NotImplementedError("this backend provides method=:map and method=:sparse on the GPU; the dense "
                                  "and CPU paths stay in the reference")
    if method == "map" and len(subspace) < map_warning_dim and method_info:
        warnings.warn(f"Linear map may be slow for dim={len(subspace)}. Consider using :sparse method.")
    if device == "gpu":
        if DEFAULT_GPU[0] == "nogpu":
            activate_b200(set_default_gpu=True)
        device = DEFAULT_GPU[0]
        if device == "nogpu":
            raise ValueError("No GPU available. Please load a supported GPU extension and verify availability.")
    if device == "cuda":
        device = "b200"
    _throw_gpu_unavailable(device)
    t0 = time.perf_counter()
    H_map = LinearMap(Hamiltonian, subspace)
    if method == "sparse":
        H_gpu = create_gpu_matrix(H_map, device)
        solve = krylov_matrix_solve
    else:
        H_gpu = create_gpu_linearmap(H_map, device)
        solve = krylov_map_solve
    try:
        vals, vecs, info = solve(H_gpu, N, ishermitian=ishermitian, **krylovkit_kwargs)
    finally:
        H_gpu.release()
    if showtime:
        print(f"EDsolve: {time.perf_counter() - t0:.4f} s ({info['matvecs']} matvecs, "
              f"{info['restarts']} restarts)")
    if len(vals) < N:
        raise RuntimeError(f"Krylov method fails. Cannot find {N} eigenvectors.")
    energies = np.asarray(vals[:N])
    vectors = [MBS64Vector(vecs[i], subspace) for i in range(N)]
    return energies, vectors
