# MomentumEDB200Ext — package extension that plugs libmomed_b200.so into MomentumED.jl's
# GPU hooks (MomentumED/src/method/gpu_interface.jl:13-21) so that
#     EDsolve(subspace, H::MBOperator; method=:map, device=:gpu, N=...)
#     EDsolve(subspace, H::MBOperator; method=:sparse, device=:gpu, N=...)
# run on a B200.  No reference file is edited: the extension registers :b200 in the
# mutable GPU_AVAILABLE dict and makes it the DEFAULT_GPU, and EDsolve resolves :gpu to it
# (MomentumED.jl:446-453).
#
# Written against the C ABI in include/momed.h.  (This file is not executed by the test
# suite of this repository: no Julia toolchain is available where it was built.)
module MomentumEDB200Ext

using MomentumED
using MomentumED: EDPara, HilbertSubspace, MBS64
using MomentumED.Methods: GPU_AVAILABLE, DEFAULT_GPU, LinearMap, AbstractGPULinearMap
import MomentumED.Methods: create_gpu_linearmap, krylov_map_solve, release_gpu_memory
import MomentumED.Methods: create_gpu_matrix, krylov_matrix_solve
using SparseArrays: SparseMatrixCSC, sparse
using LinearAlgebra: Hermitian

const libmomed = get(ENV, "MOMED_B200_LIB", joinpath(@__DIR__, "..", "lib", "libmomed_b200.so"))

struct MomedSolveOpts
    nev::Int32
    krylovdim::Int32
    maxiter::Int32
    precision::Int32
    tol::Float64
    seed::UInt64
    want_vectors::Int32
    vecs_on_device::Int32
end

struct MomedPara
    dim::Int32
    Nk::Int32
    Nc_mix::Int32
    Nc_conserve::Int32
    k_list::Ptr{Int64}
    Gk::Ptr{Int64}
end

mutable struct MomedInfo
    converged::Int32
    restarts::Int32
    matvecs::Int64
    matvecs_fp64::Int64
    seconds::Float64
end
MomedInfo() = MomedInfo(0, 0, 0, 0, 0.0)

function check(h::Ptr{Cvoid}, rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:momed_last_error, libmomed), Cstring, (Ptr{Cvoid},), h))
    rc == 4 && (@warn "B200 eigensolver: $msg"; return nothing)      # MOMED_ENOTCONV
    error("libmomed_b200 error $rc: $msg")
end

function __init__()
    h = Ref{Ptr{Cvoid}}(C_NULL)
    rc = try
        ccall((:momed_create, libmomed), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h)
    catch
        Cint(7)
    end
    if rc == 0
        ccall((:momed_destroy, libmomed), Cint, (Ptr{Cvoid},), h[])
        GPU_AVAILABLE[:b200] = Ref(true)
        DEFAULT_GPU[] = :b200
        @info "MomentumED B200 extension loaded ($(unsafe_string(ccall((:momed_version, libmomed), Cstring, ()))))."
    else
        GPU_AVAILABLE[:b200] = Ref(false)
    end
end

# The device map: one library handle holding the sorted basis and the term list of the LinearMap
# (Hermitian-completed for an upper-Hermitian operator, as it is otherwise).
mutable struct B200LinearMap{bits, F <: AbstractFloat} <: AbstractGPULinearMap{bits, F}
    handle::Ptr{Cvoid}
    space::HilbertSubspace{bits}
    hermitian::Bool
    terms::Tuple{Vector{ComplexF64}, Vector{UInt64}, Vector{UInt64}, Vector{UInt64}}   # amp, in, out, parity
end

Base.size(A::B200LinearMap) = (length(A.space), length(A.space))
Base.eltype(::B200LinearMap{bits, F}) where {bits, F} = Complex{F}
# AdjointLinearMap (linear_map.jl:46-55, 120-139): a completed Hermitian list is its own adjoint;
# otherwise a device map over the adjoint terms (conjugated amplitudes, creation and annihilation
# masks exchanged).
function Base.adjoint(A::B200LinearMap{bits, F}) where {bits, F}
    A.hermitian && return A
    amp, inm, outm, par = A.terms
    return device_map(B200LinearMap{bits, F}, A.space, false, (conj.(amp), outm, inm, par))
end

function device_map(::Type{T}, space, hermitian::Bool, terms) where {T}
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:momed_create, libmomed), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h))
    basis = UInt64[mbs.n for mbs in space.list]
    check(h[], ccall((:momed_set_basis, libmomed), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Int64, Int32),
                     h[], basis, length(basis), 0))
    amp, inm, outm, par = terms
    check(h[], ccall((:momed_set_scatter, libmomed), Cint,
                     (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{UInt64}, Ptr{UInt64}, Ptr{UInt64}, Int64),
                     h[], amp, inm, outm, par, length(amp)))
    M = T(h[], space, hermitian, terms)
    finalizer(m -> (m.handle != C_NULL && ccall((:momed_destroy, libmomed), Cint, (Ptr{Cvoid},), m.handle);
                    m.handle = C_NULL), M)
    return M
end

# create_gpu_linearmap hook (pattern of MomentumEDCUDAExt.jl:94-113): flatten and upload.
function create_gpu_linearmap(A::LinearMap{bits, F}, ::Val{:b200}) where {bits, F}
    amp = ComplexF64[ComplexF64(s.Amp) for s in A.scat_list]
    inm = UInt64[s.in.n for s in A.scat_list]
    outm = UInt64[s.out.n for s in A.scat_list]
    par = UInt64[s.parity_mask for s in A.scat_list]
    return device_map(B200LinearMap{bits, F}, A.space, is_hermitian_list(amp, inm, outm), (amp, inm, outm, par))
end

# A list is Hermitian when every term's adjoint (masks exchanged, amplitude conjugated) is in it,
# as the completion of an upper-Hermitian operator makes it (linear_map.jl:22-33).
function is_hermitian_list(amp, inm, outm)
    d = Dict{Tuple{UInt64, UInt64}, ComplexF64}()
    for (a, i, o) in zip(amp, inm, outm)
        d[(i, o)] = a
    end
    return all(get(d, (o, i), NaN + 0im) == conj(a) for (a, i, o) in zip(amp, inm, outm))
end

# callable (y, x): H*x with host vectors (the CPU LinearMap convention, linear_map.jl:100-118)
function (A::B200LinearMap{bits, F})(y::Vector{Complex{F}}, x::Vector{Complex{F}}) where {bits, F}
    prec = F === Float64 ? Int32(0) : Int32(1)
    check(A.handle, ccall((:momed_matvec, libmomed), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int32, Int32),
                          A.handle, x, y, prec, 0))
    return y
end
(A::B200LinearMap{bits, F})(x::Vector{Complex{F}}) where {bits, F} = A(similar(x), x)

# krylov_map_solve hook: the device-resident Lanczos; vecs are host vectors (Array(vecs[i]) works).
function krylov_map_solve(H::B200LinearMap{bits, F}, N_eigen::Int64; ishermitian::Bool = true,
                          vec0 = nothing, krylovdim::Int = 30, tol::Real = 1e-12, maxiter::Int = 100,
                          seed::Integer = 0, precision::Symbol = :fp64, kwargs...) where {bits, F}
    m = length(H.space)
    nev = min(N_eigen, m)
    vecs = zeros(ComplexF64, m, nev)            # column i = eigenvector i (layout [nev][N] in C)
    resid = zeros(Float64, nev)
    info = MomedInfo()
    if !ishermitian
        # Arnoldi with Krylov-Schur restarts: complex eigenvalues ordered by real part (:SR)
        opts = MomedSolveOpts(nev, krylovdim, maxiter, 0, tol, seed, 1, 0)
        vri = zeros(Float64, 2nev)
        v0buf = vec0 === nothing ? ComplexF64[] : Vector{ComplexF64}(vec0)
        GC.@preserve v0buf begin
            v0 = vec0 === nothing ? Ptr{ComplexF64}(C_NULL) : pointer(v0buf)
            check(H.handle, ccall((:momed_eigsolve_general, libmomed), Cint,
                                  (Ptr{Cvoid}, Ref{MomedSolveOpts}, Ptr{ComplexF64}, Ptr{Float64}, Ptr{Float64},
                                   Ptr{ComplexF64}, Ref{MomedInfo}),
                                  H.handle, opts, v0, vri, resid, vecs, info))
        end
        vals = ComplexF64[complex(vri[2i - 1], vri[2i]) for i in 1:nev]
        return vals, [Vector{Complex{F}}(vecs[:, i]) for i in 1:nev], info
    end
    opts = MomedSolveOpts(nev, krylovdim, maxiter, precision === :mixed ? 1 : 0, tol, seed, 1, 0)
    vals = zeros(Float64, nev)
    eigsolve_call(H.handle, opts, vec0, vals, resid, vecs, info)
    return vals, [Vector{Complex{F}}(vecs[:, i]) for i in 1:nev], info
end

# momed_eigsolve with the start vector converted to a ComplexF64 buffer that stays rooted for the
# whole call (the conversion makes a new array: it must be bound to a live variable, not passed as
# a temporary's pointer, or the collector may free it while the library reads it).
function eigsolve_call(h::Ptr{Cvoid}, opts::MomedSolveOpts, vec0, vals::Vector{Float64},
                       resid::Vector{Float64}, vecs::Matrix{ComplexF64}, info::MomedInfo)
    v0buf = vec0 === nothing ? ComplexF64[] : Vector{ComplexF64}(vec0)
    vec0 === nothing || length(v0buf) == size(vecs, 1) || error("vec0 has length $(length(v0buf)), expected $(size(vecs, 1))")
    GC.@preserve v0buf begin
        v0 = vec0 === nothing ? Ptr{ComplexF64}(C_NULL) : pointer(v0buf)
        check(h, ccall((:momed_eigsolve, libmomed), Cint,
                       (Ptr{Cvoid}, Ref{MomedSolveOpts}, Ptr{ComplexF64}, Ptr{Float64}, Ptr{Float64}, Ptr{ComplexF64},
                        Ref{MomedInfo}),
                       h, opts, v0, vals, resid, vecs, info))
    end
    return nothing
end

# Sparse method hooks (EDsolve(...; method=:sparse, device=:gpu), MomentumEDCUDAExt.jl:145-200).
# create_gpu_matrix receives the host CSC that SparseHmltMatrix built; H is Hermitian, so its
# CSC columns with conjugated values are the CSR rows of H (momed_set_sparse_csr).
mutable struct B200SparseMatrix{F <: AbstractFloat}
    handle::Ptr{Cvoid}
    n::Int
end
Base.size(A::B200SparseMatrix) = (A.n, A.n)

function create_gpu_matrix(H::SparseMatrixCSC{Complex{F}}, ::Val{:b200}) where {F}
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:momed_create, libmomed), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h))
    n = size(H, 2)
    rowptr = Int64.(H.colptr) .- 1
    col = Int32.(H.rowval) .- Int32(1)
    val = conj.(ComplexF64.(H.nzval))
    check(h[], ccall((:momed_set_sparse_csr, libmomed), Cint,
                     (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int32}, Ptr{ComplexF64}), h[], n, rowptr, col, val))
    M = B200SparseMatrix{F}(h[], n)
    finalizer(m -> (m.handle != C_NULL && ccall((:momed_destroy, libmomed), Cint, (Ptr{Cvoid},), m.handle);
                    m.handle = C_NULL), M)
    return M
end
create_gpu_matrix(H::Hermitian{C, SparseMatrixCSC{C}}, v::Val{:b200}) where {C <: Complex} =
    create_gpu_matrix(sparse(H), v)

function krylov_matrix_solve(H::B200SparseMatrix{F}, N_eigen::Int64; ishermitian::Bool = true,
                             vec0 = nothing, krylovdim::Int = 30, tol::Real = 1e-12, maxiter::Int = 100,
                             seed::Integer = 0, precision::Symbol = :fp64, kwargs...) where {F}
    ishermitian || error("the B200 sparse method solves Hermitian problems")
    nev = min(N_eigen, H.n)
    opts = MomedSolveOpts(nev, krylovdim, maxiter, precision === :mixed ? 1 : 0, tol, seed, 1, 0)
    vals = zeros(Float64, nev)
    resid = zeros(Float64, nev)
    vecs = zeros(ComplexF64, H.n, nev)
    info = MomedInfo()
    eigsolve_call(H.handle, opts, vec0, vals, resid, vecs, info)
    return vals, [Vector{Complex{F}}(vecs[:, i]) for i in 1:nev], info
end

# ED_momentum_subspaces on the device (kernel (a)): the reference enumerates on host threads
# (MomentumED/src/preparation/momentum_decomposition.jl:188-273).  Selected with a trailing
# Val(:b200), so the reference's own methods stay as they are:
#     subspaces, subspace_k = ED_momentum_subspaces(para, (Ne,), Val(:b200))
# Same keywords, same result (sectors in the reference order, empty ones dropped, each list
# sorted); a selection_rule other than the default is applied on the host to each sector.
function MomentumED.ED_momentum_subspaces(para::EDPara{dim}, N_each_component, ::Val{:b200};
        momentum_restriction::Bool = false, momentum_list::Vector{NTuple{dim, Int64}} = NTuple{dim, Int64}[],
        mask::Union{Nothing, Vector{Int64}} = nothing,
        selection_rule::Function = Returns(true)) where {dim}
    Ns = N_each_component isa Integer ? Int64[N_each_component] : Int64[n for n in N_each_component]
    @assert length(Ns) == para.Nc_conserve "The length of number_list must be equal to the number of conserved components $(para.Nc_conserve)"
    bits = para.Nk * para.Nc
    momentum_restriction && isempty(momentum_list) &&
        return HilbertSubspace{bits}[], NTuple{dim, Int64}[]
    klist = Matrix{Int64}(para.k_list)                 # dim x Nk, column-major: k_list[d + dim*i]
    Gk = Int64[para.Gk...]
    maskv = mask === nothing ? Int64[] : sort(mask)
    moms = momentum_restriction ? Int64[m[d] for m in momentum_list for d in 1:dim] : Int64[]
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:momed_create, libmomed), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h))
    try
        nsec, ntot = Ref{Int64}(0), Ref{Int64}(0)
        GC.@preserve klist Gk maskv moms Ns begin
            p = MomedPara(Int32(dim), Int32(para.Nk), Int32(para.Nc_mix), Int32(para.Nc_conserve),
                          pointer(klist), pointer(Gk))
            check(h[], ccall((:momed_enumerate_basis, libmomed), Cint,
                             (Ptr{Cvoid}, Ref{MomedPara}, Ptr{Int64}, Int32, Ptr{Int64}, Int32, Ptr{Int64}, Int32,
                              Ref{Int64}, Ref{Int64}),
                             h[], p, Ns, Int32(length(Ns)),
                             mask === nothing ? Ptr{Int64}(C_NULL) : pointer(maskv),
                             Int32(mask === nothing ? -1 : length(maskv)),
                             momentum_restriction ? pointer(moms) : Ptr{Int64}(C_NULL),
                             Int32(momentum_restriction ? length(momentum_list) : -1), nsec, ntot))
        end
        sector_k = Vector{Int64}(undef, max(nsec[] * dim, 1))
        sizes = Vector{Int64}(undef, max(nsec[], 1))
        basis = Vector{UInt64}(undef, max(ntot[], 1))
        check(h[], ccall((:momed_enumeration_copy, libmomed), Cint,
                         (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int64}, Ptr{UInt64}, Int32),
                         h[], sector_k, sizes, basis, Int32(0)))
        subspaces = HilbertSubspace{bits}[]
        subspace_k = NTuple{dim, Int64}[]
        off = 0
        for s in 1:nsec[]
            list = MBS64{bits}[MBS64{bits}(basis[off + i]) for i in 1:sizes[s]]
            off += sizes[s]
            selection_rule === Returns(true) || filter!(selection_rule, list)
            isempty(list) && continue
            push!(subspaces, HilbertSubspace(list))
            push!(subspace_k, ntuple(d -> sector_k[(s - 1) * dim + d], Val(dim)))
        end
        return subspaces, subspace_k
    finally
        ccall((:momed_destroy, libmomed), Cint, (Ptr{Cvoid},), h[])
    end
end

# release_gpu_memory hook: device buffers belong to handles (freed by their finalizers).
release_gpu_memory(::Val{:b200}, level::Int64 = 2) = (level >= 1 && GC.gc(); nothing)

end # module
