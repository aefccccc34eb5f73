/*
 * momed.h -- C ABI of libmomed_b200.so, the B200 (sm_100a) backend for
 * MomentumED.jl's matrix-free Hamiltonian map and Lanczos eigensolve.
 *
 * The reference binds this path through its GPU plugin hooks
 * (MomentumED/src/method/gpu_interface.jl:13-21); each entry point below names
 * the hook or function it replaces.  Conventions:
 *   - every call returns an int status (MOMED_OK == 0); the message of the last
 *     failure on a handle is momed_last_error(h).  Nothing traps or throws.
 *   - orbitals are bits: bit i-1 of a uint64 is orbital i (EDCore MBS64).
 *   - complex arrays are interleaved (re, im) of double (c128) or float (c64).
 *   - basis indices are 0-based inside the ABI (the Julia shim adds 1).
 *   - inputs are copied; the caller keeps ownership of its buffers.  Device
 *     buffers inside a handle are owned by the handle.
 *   - one handle per host thread; distinct handles are independent.
 */
#ifndef MOMED_H
#define MOMED_H

#include <stdint.h>

#if defined(__GNUC__)
#define MOMED_API __attribute__((visibility("default")))
#else
#define MOMED_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MOMED_OK        0
#define MOMED_EINVAL    1   /* bad argument or size */
#define MOMED_ENOMEM    2   /* device memory / HBM budget refused */
#define MOMED_ECUDA     3   /* CUDA runtime error (message carries the CUDA text) */
#define MOMED_ENOTCONV  4   /* eigensolver stopped at maxiter (results still written) */
#define MOMED_ETIMEOUT  5   /* a bounded wait gave up */
#define MOMED_ESTATE    6   /* call order (e.g. matvec before set_basis) */
#define MOMED_ENODEV    7   /* no usable CUDA device */

#define MOMED_C128      0   /* complex double vectors / FP64 arithmetic */
#define MOMED_C64       1   /* complex float vectors, FP32 accumulate */

#define MOMED_PREC_FP64   0 /* plain: c128 matvec, FP64 Lanczos */
#define MOMED_PREC_MIXED  1 /* c64 matvec + FP64 recurrences, then FP64 Rayleigh-Ritz / refinement */

typedef struct momed_handle momed_handle;

/* EDPara subset the basis enumerator needs (init_parameter.jl:62-146). */
typedef struct {
    int32_t dim, Nk, Nc_mix, Nc_conserve;
    const int64_t* k_list;   /* k_list[d + dim*i], column i of the Julia dim x Nk matrix */
    const int64_t* Gk;       /* [dim]; 0 = no periodicity in that direction */
} momed_para;

typedef struct {
    int32_t nev;          /* eigenpairs wanted (EDsolve N) */
    int32_t krylovdim;    /* Krylov subspace size (KrylovKit krylovdim; default 30) */
    int32_t maxiter;      /* restarts (KrylovKit maxiter; default 100) */
    int32_t precision;    /* MOMED_PREC_FP64 or MOMED_PREC_MIXED */
    double  tol;          /* residual-norm tolerance (KrylovKit tol; default 1e-12) */
    uint64_t seed;        /* start vector seed when vec0 == NULL */
    int32_t want_vectors; /* 0: eigenvalues only */
    int32_t vecs_on_device;
} momed_solve_opts;

typedef struct {
    int32_t converged;     /* leading eigenpairs with residual <= tol */
    int32_t restarts;
    int64_t matvecs;       /* all matvecs */
    int64_t matvecs_fp64;  /* of which FP64 (mixed mode) */
    double  seconds;       /* device time of the solve */
} momed_info;

/* Library */
MOMED_API const char* momed_version(void);
MOMED_API int  momed_create(int device, momed_handle** out);             /* activate_gpu_device (gpu_interface.jl:41-55) */
MOMED_API int  momed_destroy(momed_handle* h);                           /* release_gpu_memory (MomentumEDCUDAExt.jl:43-47) */
MOMED_API const char* momed_last_error(const momed_handle* h);
MOMED_API int  momed_set_stream(momed_handle* h, void* cuda_stream);      /* optional; default: the handle's own stream */
MOMED_API int  momed_set_hbm_budget(momed_handle* h, int64_t bytes);      /* admission limit for this handle (0 = free memory) */

/* Kernel (a): basis enumeration per momentum sector.
 * Replaces ED_momentum_subspaces (momentum_decomposition.jl:188-273) without selection_rule.
 * mask (sorted 1-based orbitals) may be NULL (mlen < 0).  momentum_list (nmom * dim) restricts
 * the sectors when nmom >= 0; nmom < 0 enumerates every momentum in the reference order.
 * The result stays on the device; fetch it with momed_enumeration_copy. */
MOMED_API int  momed_enumerate_basis(momed_handle* h, const momed_para* p, const int64_t* N_each, int32_t ncc,
                           const int64_t* mask, int32_t mlen, const int64_t* momentum_list, int32_t nmom,
                           int64_t* n_sectors, int64_t* n_total);
/* sector_k [n_sectors*dim], sector_sizes [n_sectors], basis [n_total] (host, or device if basis_on_device). */
MOMED_API int  momed_enumeration_copy(momed_handle* h, int64_t* sector_k, int64_t* sector_sizes, uint64_t* basis,
                            int32_t basis_on_device);
/* Use sector s of the last enumeration as the working basis (device to device). */
MOMED_API int  momed_select_sector(momed_handle* h, int64_t s);

/* The basis of ONE momentum sector (total momentum `momentum[dim]`, no mask) written into the
 * caller's device buffer out_dev[out_capacity], allocating no device memory: for callers that
 * cannot call cudaMalloc (device memory owned by another allocator such as a Julia CUDA.jl
 * pool, or services that reserve all HBM up front).  No counterpart in the reference, whose
 * enumeration runs on the host.  Runs on the current device and the given stream (NULL: the
 * default stream) and returns after the stream has finished it.  Working space is a static
 * 148,864-byte device array per GPU, kept until process exit; the first call on a device
 * looks its address up and should come before any stream capture; calls that overlap on the
 * GPU race on it.  Limits: momentum box (product of Gk, or of the momentum ranges where
 * Gk == 0) <= 4096 entries.  *n_states receives the sector size; when it exceeds
 * out_capacity nothing is written and MOMED_EINVAL is returned. */
MOMED_API int  momed_enumerate_sector_noalloc(const momed_para* p, const int64_t* N_each, int32_t ncc,
                                              const int64_t* momentum, uint64_t* out_dev, int64_t out_capacity,
                                              int64_t* n_states, void* cuda_stream);

/* Working basis: the sorted HilbertSubspace list (hilbert_subspace.jl:19-30), uploaded as in
 * create_gpu_linearmap (MomentumEDCUDAExt.jl:94-113). */
MOMED_API int  momed_set_basis(momed_handle* h, const uint64_t* basis, int64_t n, int32_t on_device);

/* Operator: the Hermitian-completed, sorted scatter list of LinearMap (linear_map.jl:22-37),
 * flattened as in create_gpu_linearmap: amp[2*nscat] (c128), in/out/parity masks.
 * parity may be NULL (recomputed).  Amplitudes of c64 matvecs are rounded from these. */
MOMED_API int  momed_set_scatter(momed_handle* h, const double* amp, const uint64_t* in, const uint64_t* out,
                       const uint64_t* parity, int64_t nscat);
/* Parametrised operator H(u) = A + u B on one term list (amp_b may be NULL = zeros): used by
 * the batched solver where u is an interaction strength (two-body amplitudes scaled by u). */
MOMED_API int  momed_set_scatter_pair(momed_handle* h, const double* amp_a, const double* amp_b, const uint64_t* in,
                            const uint64_t* out, const uint64_t* parity, int64_t nscat);

/* Twisted-boundary sweeps: the two-body amplitudes regenerated on the device for each kshift.
 * With momentum coordinates, ED_scatterlist_twobody (scat_list.jl:442-497) evaluates H_two at
 * k/Gk + kshift/Gk of each conserved component (scat_list.jl:5-50), so the reference rebuilds
 * the list on the host for every point of a sweep.  momed_set_twobody_recipe attaches to the
 * working operator (set by momed_set_scatter, a single operator) the structure of its two-body
 * terms: raw[nraw][9] = (kf1, kf2, ki2, ki1) 0-based momentum indices, (cf1, cf2, ci2, ci1)
 * 1-based components, flags (bit 0: negate; bits 1-2: 0 as is, 1 conjugate, 2 real part: the
 * normal ordering of the Scatter constructor), grouped per upper term by upper_start[nupper + 1]
 * in the order the terms are summed; for each entry e of the list passed to momed_set_scatter,
 * entry_upper[e] (its upper term, -1 for a term the recipe leaves as uploaded) and
 * entry_partner[e] (1 for the Hermitian partner, whose amplitude is the conjugate).
 * momed_set_kshift(h, kshift[Nc_conserve][dim]) evaluates the recipe's interaction on the device
 * for every contribution, (direct - exchange) / Nk as scat_list.jl does, and overwrites the term
 * amplitudes (a built sparse matrix is dropped).  Recipe MOMED_RECIPE_LANDAU_COULOMB: the
 * screened Coulomb interaction in the lowest Landau level with magnetic-translation phases
 * (the H_two of MomentumED/test/example1_FQH_Laughlin.jl:20-89), params [Gl, D, W0, angle,
 * nshell], 2D meshes.  FP64 on the device: amplitudes agree with the host builder to ~1e-15. */
#define MOMED_RECIPE_LANDAU_COULOMB 1
MOMED_API int  momed_set_twobody_recipe(momed_handle* h, const momed_para* p, int32_t recipe, const double* params,
                                        int32_t nparams, const int32_t* raw, int64_t nraw, const int64_t* upper_start,
                                        int64_t nupper, const int64_t* entry_upper, const int32_t* entry_partner,
                                        int64_t nentries);
MOMED_API int  momed_set_kshift(momed_handle* h, const double* kshift);

/* Parameter u of the operator H(u) = A + u B set by momed_set_scatter_pair (default 1). */
MOMED_API int  momed_set_param(momed_handle* h, double u);

/* y = H x: the callable (y, x) of CuLinearMap (MomentumEDCUDAExt.jl:119-122, kernel at
 * gpu_interface.jl:128-163), computing H*x as the CPU LinearMap does (linear_map.jl:100-118).
 * precision MOMED_C128 / MOMED_C64; x, y host or device (on_device). */
MOMED_API int  momed_matvec(momed_handle* h, const void* x, void* y, int32_t precision, int32_t on_device);

/* Lowest nev eigenpairs: krylov_map_solve (MomentumEDCUDAExt.jl:159-179) -> KrylovKit eigsolve(:SR).
 * vals[nev] ascending; resid[nev] = ||H x - e x|| per pair (may be NULL);
 * vecs [nev][N] c128 (host, or device if opts->vecs_on_device).  vec0 (c128, host) may be NULL.
 * Returns MOMED_ENOTCONV when fewer than nev pairs met tol (results still written). */
MOMED_API int  momed_eigsolve(momed_handle* h, const momed_solve_opts* opts, const double* vec0,
                    double* vals, double* resid, void* vecs, momed_info* info);

/* Eigenpairs of a NON-Hermitian operator (a term list set as it is, without Hermitian
 * completion): krylov_map_solve(H, N; ishermitian = false) (MomentumEDCUDAExt.jl:159-179) ->
 * KrylovKit eigsolve(:SR; ishermitian = false).  Arnoldi with Krylov-Schur restarts in FP64 on
 * the matrix-free map.  vals [2 nev]: complex eigenvalues (re, im) ordered by real part
 * (ascending); resid [nev] = ||H x - e x||; vecs [nev][N] c128 right eigenvectors (unit norm).
 * opts->precision is ignored (FP64).  Returns MOMED_ENOTCONV when fewer than nev pairs met tol. */
MOMED_API int  momed_eigsolve_general(momed_handle* h, const momed_solve_opts* opts, const double* vec0,
                                      double* vals, double* resid, void* vecs, momed_info* info);

/* Batched solve of H(u) = A + u B (momed_set_scatter_pair) for nu values of u at once on the
 * working basis: block matvec over all u, one Lanczos per u.  vals [nu][nev], resid [nu][nev];
 * vecs [nu][nev][N] c128 host (may be NULL).  Mixed precision is opts->precision.  With a
 * single operator (momed_set_scatter) every u solves H = A. */
MOMED_API int  momed_batch_solve(momed_handle* h, const momed_solve_opts* opts, const double* u, int32_t nu,
                       double* vals, double* resid, double* vecs, momed_info* info);

/* GPU sparse method: EDsolve(...; method = :sparse, device = :gpu), whose matrix the reference
 * builds on host threads (ED_HamiltonianMatrix_threaded_CSCdirect, sparse_matrix.jl:64-190),
 * uploads (create_gpu_matrix, MomentumEDCUDAExt.jl:145-152) and multiplies inside
 * krylov_matrix_solve (MomentumEDCUDAExt.jl:180-200).  momed_build_sparse builds H (at the
 * current u) as a CSR matrix on the device from the working operator and basis: row i = output
 * state, entry row_ptr[i] is the diagonal, then one entry per off-diagonal (row, term) hit
 * (a pair reached by two terms keeps two entries).  While it is built, momed_matvec and
 * momed_eigsolve use the CSR SpMV instead of the matrix-free map; a new basis, operator or u
 * drops it, as does momed_release_sparse.  momed_batch_solve then runs its FP32 maps as a
 * block SpMV over the same entries (values A + u B per right-hand side; its FP64 maps stay
 * matrix-free).  nnz receives the stored entries; the matrix takes 8 (N + 1) + 28 nnz bytes
 * (44 nnz for H(u) = A + u B, which also keeps the A and B parts) and MOMED_ENOMEM is
 * returned when that exceeds the handle's budget or 90% of free device memory.
 * momed_sparse_copy copies it to host arrays row_ptr[N + 1], col[nnz], val[2 nnz] (c128);
 * any of them may be NULL. */
MOMED_API int  momed_build_sparse(momed_handle* h, int64_t* nnz);
MOMED_API int  momed_sparse_copy(momed_handle* h, int64_t* row_ptr, int32_t* col, double* val);
MOMED_API int  momed_release_sparse(momed_handle* h);
/* create_gpu_matrix(H::SparseMatrixCSC, Val(:b200)) (MomentumEDCUDAExt.jl:145-152): upload a
 * host matrix of size n as CSR (0-based row_ptr[n + 1], col[nnz], val[2 nnz] c128; for the
 * Hermitian CSC matrix that SparseHmltMatrix returns, pass its colptr and rowval with conjugated
 * values).  Validated on the host (monotone row_ptr from 0, columns in [0, n)).  The handle then
 * multiplies by it (momed_matvec, momed_eigsolve) with no basis or operator; a later basis drops
 * it, and momed_release_sparse empties the handle. */
MOMED_API int  momed_set_sparse_csr(momed_handle* h, int64_t n, const int64_t* row_ptr, const int32_t* col,
                                    const double* val);

/* ED_bracket(bra, op, ket) (EDCore/src/multiplication.jl:153-190, 239-245): <bra| H |ket> with
 * the working operator (its Hermitian-completed list, at the current u), ket (c128, host) on the
 * working basis and bra (c128, host) on bra_basis[n_bra] (sorted; NULL = the working basis, then
 * n_bra is ignored).  Targets outside the bra space are dropped (index_fit).  Computed as one
 * fused map-and-dot kernel (no H ket vector is written); out[2] = (re, im). */
MOMED_API int  momed_bracket(momed_handle* h, const uint64_t* bra_basis, int64_t n_bra, const double* bra,
                             const double* ket, double* out);

/* PES_1rdm(psi) (MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33): the one-body
 * reduced density matrix rdm[i][j] = <psi| c+_i c_j |psi> over orbitals 0..norb-1 (norb <= 64;
 * the reference's bits), psi (c128, host) on the working basis (no operator needed).  rdm:
 * [norb][norb] c128 row-major, Hermitian. */
MOMED_API int  momed_rdm1(momed_handle* h, const double* psi, int32_t norb, double* rdm);

/* ED_step_inner_prod (MomentumED/src/analysis/manybody_quantum_geometry.jl:48-94): for g
 * vectors psi_f[g][N], psi_i[g][N] (c128, host) on the working basis and orbital overlaps
 * orb[norb] (c128), out[j][k] = sum_x conj(psi_f[j][x]) psi_i[k][x] prod_{o occupied in x} orb[o]
 * ([g][g] c128; g <= 32, norb <= 64). */
MOMED_API int  momed_step_inner_prod(momed_handle* h, const double* psi_f, const double* psi_i, int32_t g,
                                     const double* orb, int32_t norb, double* out);

/* Diagnostics for roofline accounting: exact (row, term) hit count of the working operator
 * on the working basis, the index mode (0 = ranked tables, 1 = checked tables, 2 = search),
 * and the bytes of the lookup tables. */
MOMED_API int  momed_stats(momed_handle* h, int64_t* nnz, int32_t* index_mode, int64_t* table_bytes);

/* Device time (ms) of the last matvec kernel launch on the handle's stream. */
MOMED_API int  momed_last_kernel_ms(momed_handle* h, double* ms);

/* Serving form: a continuous-batching solve server (no reference counterpart: the reference
 * runs one EDsolve at a time).  `slots` worker contexts, each with its own stream, take
 * queued requests in arrival order as soon as a slot is free and the request's HBM estimate
 * fits the budget (0 = 85% of free memory); admitted solves run concurrently on the device.
 * Queued mixed-precision requests (nev <= 12) on the same operator and sector basis are solved
 * together as one batched solve (3 to 32 of them, one right-hand side per u); any other request
 * runs alone on the FP64 single-vector solver.  A solve of at least 4096 states uses the sparse
 * method (momed_build_sparse) when its matrix fits what the budget has left; requests of at
 * least 131072 states run one at a time.
 * Requests larger than the budget fail at once with MOMED_ENOMEM.  poll waits at most
 * wait_ms and returns MOMED_ETIMEOUT when the request is still queued or running;
 * status: 0 queued, 1 running, 2 done, 3 failed (return code is the failure's), 4 cancelled. */
typedef struct momed_server momed_server;
MOMED_API int  momed_serve_start(int device, int32_t slots, int64_t hbm_budget, momed_server** out);
MOMED_API int  momed_serve_register_operator(momed_server* s, const double* amp_a, const double* amp_b,
                                             const uint64_t* in, const uint64_t* out, const uint64_t* parity,
                                             int64_t nscat, int32_t* op_id);
MOMED_API int  momed_serve_submit(momed_server* s, int32_t op_id, const uint64_t* basis, int64_t n, double u,
                                  const momed_solve_opts* opts, int64_t* request_id);
MOMED_API int  momed_serve_cancel(momed_server* s, int64_t request_id);
MOMED_API int  momed_serve_poll(momed_server* s, int64_t request_id, int32_t wait_ms, int32_t* status,
                                double* vals, double* resid, momed_info* info, double* queue_s, double* latency_s);
MOMED_API int  momed_serve_stats(momed_server* s, int64_t* queued, int64_t* completed, int64_t* failed,
                                 int64_t* hbm_used, int64_t* hbm_budget);
MOMED_API const char* momed_serve_last_error(momed_server* s);
MOMED_API int  momed_serve_stop(momed_server* s);

/* The block map's autotuned launch for the working operator and basis (its sector size class)
 * at block width nb (1..32), precision MOMED_PREC_FP64 (c128) or MOMED_PREC_MIXED (c64), with
 * (has_param = 1) or without the H(u) = A + u B form: rows per warp (1, 2, 4), grid (0: one
 * CTA per SM fewer than resident, 1: resident, 2: twice resident), the chosen and the default
 * launch's device time (ms).  The tuner runs at a key's first launch (MOMED_AUTOTUNE=0 turns it
 * off); MOMED_ESTATE until then.  No reference counterpart (a measurement aid). */
MOMED_API int  momed_block_tuning(momed_handle* h, int32_t nb, int32_t precision, int32_t has_param,
                                  int32_t* rows_per_warp, int32_t* grid_mult, double* ms, double* ms_default);

/* Hit cache of the matrix-free map: for the current sector basis and term list, the target row
 * and term slot of every off-diagonal (row, term) hit (8 bytes each) and each row's diagonal
 * sums, so that a map skips the candidate stage (mask tests, signs, index lookups) and forms
 * only the values, from the term list, at each application.  The eigensolvers build it at their
 * start when it fits a quarter of the free device memory and no HBM budget is set; when it does
 * not, its slot mode (the term slot of each hit only, 2 bytes, for at most 65536 terms; the
 * single-vector map then forms each target itself) when that fits 30% (MOMED_HITCACHE=0: never,
 * =1: full whatever its size, =2: slot mode); momed_build_hit_cache builds it on request (the
 * slot mode under MOMED_HITCACHE=2; MOMED_ENOMEM when it does not fit, MOMED_ESTATE while a
 * sparse matrix is built).  It is
 * dropped with the basis, the operator, a sparse-matrix build, or new amplitudes of a
 * parametrised operator.  No reference counterpart: the reference map evaluates every term at
 * every application (ka_linearmap_kernel!, MomentumED/src/method/gpu_interface.jl:128-163). */
MOMED_API int  momed_build_hit_cache(momed_handle* h, int64_t* hits, int64_t* bytes);
MOMED_API int  momed_hit_cache_info(momed_handle* h, int32_t* built, int64_t* hits, int64_t* bytes,
                                    double* build_ms);          /* built: 0 none, 1 full, 2 slot mode */
MOMED_API int  momed_release_hit_cache(momed_handle* h);

/* Kernels this library has launched in the process so far (all handles). */
MOMED_API int64_t momed_kernel_launches(void);

/* Per-launch device timing of the matvec kernels (CUDA events on the handle's stream).
 * momed_profile(h, 1) starts a fresh record; momed_profile_read returns, for one kernel
 * kind, the launches recorded since and their summed device time in ms. */
#define MOMED_KERNEL_MATVEC_C128        0
#define MOMED_KERNEL_MATVEC_C64         1
#define MOMED_KERNEL_BLOCK_MATVEC_C64   2
#define MOMED_KERNEL_BLOCK_MATVEC_C128  3
#define MOMED_KERNEL_SPMV_C128          4
#define MOMED_KERNEL_SPMV_C64           5
#define MOMED_KERNEL_BLOCK_SPMV_C64     6
#define MOMED_KERNEL_HC_MATVEC_C128     7   /* the map over its hit cache */
#define MOMED_KERNEL_HC_MATVEC_C64      8
#define MOMED_KERNEL_HC_BLOCK_C64       9
#define MOMED_KERNEL_HC_BLOCK_C128      10
#define MOMED_KERNEL_KINDS              11
MOMED_API int  momed_profile(momed_handle* h, int32_t enable);
MOMED_API int  momed_profile_read(momed_handle* h, int32_t kind, int64_t* launches, double* total_ms);

#ifdef __cplusplus
}
#endif
#endif /* MOMED_H */
