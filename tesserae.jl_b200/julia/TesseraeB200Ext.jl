# TesseraeB200Ext.jl -- Tesserae.jl package extension that runs the explicit MPM
# hot path on a B200 (sm_100) through libtesserae_b200.so's C ABI
# (include/tesserae_b200.h).
#
# Where it plugs in. Tesserae dispatches its GPU work on the device tag of the
# data (src/Core/devices.jl:16-20) at these points; this extension adds more
# specific methods for CUDA data of the recognised equation sets:
#
#   update!(bs::GPUBlockStrategy, xₚ)        src/Parallel/gpu_block_strategy.jl:142-166  -> tb_bin_particles_*
#   update!(weights, particles, mesh)        src/Basis/basis_weight.jl:714-752           -> tb_update_weights_*
#   P2G(::P2GBodies, ::GPUDevice, ..., ::Partition{<:GPUBlockStrategy})
#                                            src/Transfer/gpu.jl:196-223                 -> tb_p2g_*
#   foreach_loop(f, ::GPUDevice, ...)        src/Transfer/foreach.jl:308-339 (the @P2G grid half)
#                                                                                        -> tb_grid_update_*
#   G2P(f, ::GPUDevice, ...)                 src/Transfer/gpu.jl:226-232                 -> tb_g2p_*
#   reorder_particles!(particles, bs)        src/Parallel/gpu_block_strategy.jl:193-238  -> tb_reorder_particles_*
#   block_ordered_particle_contiguity(bs)    src/Parallel/gpu_block_strategy.jl:172-191  -> tb_particle_contiguity
#
# plus the device seam of ext/TesseraeCUDAExt.jl:11-39 for the B200Device tag
# (get_backend, get_device, has_device, adapt_storage, free_temporary!) and a
# ChainRulesCore rrule over a checkpointed rollout (tb_tape_forward_* /
# tb_tape_backward_*; the reference has no adjoint of its transfers).
#
# Layout. The C ABI takes one device pointer per vector or tensor component.
# `b200(x)`, `b200_x64(x)` and `b200_preserve(x)` adapt particles and grids to
# StructArrays whose Vec / Tensor fields are unwrapped into component CuArrays
# (`particles.x[p]` still returns a Vec), with F always Float64, and in
# `b200_x64` the positions too (the tb_*_f32x64 form). Data in another layout
# takes Tesserae's own generic GPU kernels.
#
# Recognising the transfer bodies. `@P2G` hands the block-scheduled GPU path a
# `P2GBodies{names}` whose names are the scattered grid fields
# (src/Transfer/gpu.jl:23-28); `@G2P` and the grid half hand over a bare closure
# (src/Transfer/g2p.jl:87-92, src/Transfer/runtime.jl:174-175). Neither names
# its equations, so each closure is recognised by what it computes: it is run
# once on the host on a one-particle probe (a 4^3-cell mesh, the same field
# names and element types, random state) and its outputs are compared with
# this extension's host statement of every supported equation set, the set's
# scalars (dt, flip alpha, mu, lambda, bulk modulus, gravity) being solved for
# from the probe's own outputs; a second probe with another random state must
# then agree to rounding. The equation set is cached per closure type (one per
# macro call site); the scalars are solved again on every call, since closures
# capture values such as an adaptive dt anew each step (a one-particle host
# evaluation, microseconds). A body that matches no supported set runs on
# Tesserae's generic GPU kernels, or raises with TESSERAE_B200_STRICT=1.
# Supported sets: README.md:71-87 (FLIP / PIC blend, Neo-Hookean), APIC
# (docs/src/transfer.md:166-186), the weakly compressible fluid sigma = K (J - 1) I,
# gravity in f, slip-wall slices.
module TesseraeB200Ext

using Tesserae
using Tesserae: CUDADevice, GPUDevice, EltypePolicy, CastFloat32, PreserveEltype, Partition,
                GPUBlockStrategy, P2GBodies, CartesianMesh, BSpline, Quadratic, uGIMP, WLS,
                KernelCorrection, Vec, Mat, SymmetricSecondOrderTensor
using CUDA
using KernelAbstractions
using Adapt
using StructArrays
using ChainRulesCore
using LinearAlgebra
using Libdl
using Random

const libtb = "libtesserae_b200"  # resolved through Libdl.DL_LOAD_PATH / LD_LIBRARY_PATH

const TB_OK = Int32(0)
const TB_ERR_CAPACITY = Int32(-3)
const TB_ERR_UNSUPPORTED = Int32(-4)
const TB_BSPLINE_QUADRATIC, TB_UGIMP, TB_WLS_BSPLINE_QUADRATIC, TB_WLS_UGIMP, TB_KC_BSPLINE_QUADRATIC, TB_KC_UGIMP =
    Int32.(0:5)
const TB_MATERIAL_NEOHOOKEAN, TB_MATERIAL_FLUID, TB_MATERIAL_VONMISES = Int32.(0:2)
const TB_TRANSFER_FLIP, TB_TRANSFER_APIC = Int32.(0:1)

# ---- POD descriptors, field for field as in include/tesserae_b200.h ----------

struct TbMesh
    dim::Int32
    block_log2::Int32
    n_nodes::NTuple{3,Int64}
    xmin::NTuple{3,Float64}
    h::Float64
    h_inv::Float64
end

struct TbParticles
    n::Int64
    x::NTuple{3,Ptr{Cvoid}}
    v::NTuple{3,Ptr{Cvoid}}
    V::Ptr{Cvoid}
    m::Ptr{Cvoid}
    l::Ptr{Cvoid}
    grad_v::NTuple{9,Ptr{Cvoid}}
    sigma::NTuple{6,Ptr{Cvoid}}
    F::NTuple{9,Ptr{Cvoid}}
    B::NTuple{9,Ptr{Cvoid}}
    V0::Ptr{Cvoid}
    mu::Ptr{Cvoid}
    lambda::Ptr{Cvoid}
    eps_p::Ptr{Cvoid}
    Cp_inv::NTuple{6,Ptr{Cvoid}}
end

struct TbGrid
    m::Ptr{Cvoid}
    mv::NTuple{3,Ptr{Cvoid}}
    f::NTuple{3,Ptr{Cvoid}}
    v::NTuple{3,Ptr{Cvoid}}
    vn::NTuple{3,Ptr{Cvoid}}
    block_numbering::Ptr{Int32}   # SpGrid only (C_NULL for a dense grid)
    active_blocks::Ptr{Int32}
    nactive::Ptr{Int32}
    capacity::Int64
end

struct TbPartition
    blockids::Ptr{Int32}
    counts::Ptr{Int32}
    offsets::Ptr{Int32}
    blocklist::Ptr{Int32}
    particleindices::Ptr{Int32}
    nblocks::Int64
end

struct TbWeights
    w::Ptr{Cvoid}
    grad_w::Ptr{Cvoid}
    window::Ptr{Int64}
end

struct TbParams
    dt::Float64
    mass::Float64
    V0::Float64
    mu::Float64
    lambda::Float64
    gravity::NTuple{3,Float64}
    gimp_l::Float64
    flip_alpha::Float64
    basis::Int32
    transfer::Int32
    material::Int32
    wall_mask::Int32
    wall_layers::Int32
    reserved::Int32
    hardening::Float64
    yield_stress::Float64
end

struct TbAdjoint
    x::NTuple{3,Ptr{Float64}}
    v::NTuple{3,Ptr{Float64}}
    F::NTuple{9,Ptr{Float64}}
    mu::Ptr{Float64}
    lambda::Ptr{Float64}
    B::NTuple{9,Ptr{Float64}}
end

struct TbKernelTime
    name::NTuple{32,UInt8}
    launches::Int64
    ms::Float64
end

# ---- context: one tb_ctx per (device, stream) -------------------------------

const CTXS = Dict{Tuple{Int,UInt},Ptr{Cvoid}}()
const CTX_LOCK = ReentrantLock()
const ACTIVE = Ref(false)   # an sm_100 device and the library are present
const STRICT = Ref(false)   # unrecognised bodies raise instead of taking the generic kernels

function ctx()
    dev = CUDA.deviceid(CUDA.device())
    st = CUDA.stream()
    key = (dev, UInt(st.handle))
    lock(CTX_LOCK) do
        get!(CTXS, key) do
            c = ccall((:tb_create, libtb), Ptr{Cvoid}, (Int32, Ptr{Cvoid}), Int32(dev), st.handle)
            c == C_NULL && error("tb_create failed on device $dev")
            c
        end
    end
end

function check(rc::Int32, what)
    rc == TB_OK && return nothing
    msg = unsafe_string(ccall((:tb_last_error, libtb), Cstring, (Ptr{Cvoid},), ctx()))
    error("$what: libtesserae_b200 status $rc: $msg")
end

function __init__()
    dir = get(ENV, "TESSERAE_B200_LIBDIR", "")
    isempty(dir) || pushfirst!(Libdl.DL_LOAD_PATH, dir)
    STRICT[] = get(ENV, "TESSERAE_B200_STRICT", "0") == "1"
    ACTIVE[] = CUDA.functional() && CUDA.capability(CUDA.device()) == v"10.0" &&
               Libdl.dlopen(libtb; throw_error=false) !== nothing
    atexit() do
        for c in values(CTXS)
            ccall((:tb_destroy, libtb), Cvoid, (Ptr{Cvoid},), c)
        end
    end
end

# ---- device tag and the seam of ext/TesseraeCUDAExt.jl:11-39 -----------------

# `keep` names the fields that stay Float64 under CastFloat32 (F always; x too
# in the FP64-position form).
struct B200Device{P,keep} <: GPUDevice{P} end
const b200 = B200Device{CastFloat32,(:F,)}()
const b200_x64 = B200Device{CastFloat32,(:F, :x)}()
const b200_preserve = B200Device{PreserveEltype,()}()

KernelAbstractions.get_backend(::B200Device) = CUDABackend()
Tesserae.has_device(::B200Device) = ACTIVE[]
Tesserae.free_temporary!(a::CuArray) = CUDA.unsafe_free!(a)

# Component arrays of an unwrapped Vec / Tensor field, or nothing when the
# field is stored AoS.
unwrap_schema(T) = T <: Union{Tesserae.Tensor,NTuple}
to_float(::Type{CastFloat32}, ::Type{T}) where {T<:AbstractFloat} = Float32
to_float(::Type{PreserveEltype}, ::Type{T}) where {T} = T
retype(::Type{P}, ::Type{T}, keep::Bool) where {P,T<:Number} = keep ? T : to_float(P, T)
retype(::Type{P}, ::Type{Tesserae.Tensor{S,T,N,L}}, keep::Bool) where {P,S,T,N,L} =
    Tesserae.Tensor{S,retype(P, T, keep),N,L}
retype(::Type{P}, ::Type{T}, keep::Bool) where {P,T} = T

function Adapt.adapt_storage(::B200Device{P,keep}, A::StructArray{T}) where {P,keep,T<:NamedTuple}
    names = fieldnames(T)
    cols = map(names) do name
        col = getproperty(A, name)
        col isa AbstractArray || return col  # e.g. the grid's lazy mesh column
        E = retype(P, eltype(col), name in keep)
        S = StructArray{E}(undef, size(col); unwrap=unwrap_schema)
        copyto!(S, col)
        replace_storage(CuArray, S)
    end
    StructArray(NamedTuple{names}(cols))
end
Adapt.adapt_storage(::B200Device{CastFloat32}, A::AbstractArray) = cu(A)
Adapt.adapt_storage(::B200Device{PreserveEltype}, A::AbstractArray) = adapt(CuArray, A)

# Flat list of the component CuArrays of one StructArray column (scalars give one).
components_of(col::CuArray{<:Number}) = (col,)
components_of(col::StructArray) = Tuple(Iterators.flatten(map(components_of, StructArrays.components(col))))
components_of(col) = nothing

devptr(a::CuArray) = reinterpret(Ptr{Cvoid}, pointer(a))
function ptrs(col, k::Int)
    cs = components_of(col)
    cs === nothing && return nothing
    ntuple(i -> i <= length(cs) ? devptr(cs[i]) : C_NULL, k)
end
optptr(A, name) = hasproperty(A, name) ? first(something(ptrs(getproperty(A, name), 1), (C_NULL,))) : C_NULL

# ---- descriptors from Tesserae objects --------------------------------------

function tbmesh(mesh::CartesianMesh{dim}) where {dim}
    n = size(mesh)
    TbMesh(Int32(dim), Int32(Tesserae.block_size_log2(mesh)),
           ntuple(d -> d <= dim ? Int64(n[d]) : Int64(1), 3),
           ntuple(d -> d <= dim ? Float64(Tesserae.get_xmin(mesh)[d]) : 0.0, 3),
           Float64(Tesserae.spacing(mesh)), Float64(Tesserae.spacing_inv(mesh)))
end

# Symmetric tensors: the ABI's order (11, 21, 31, 22, 32, 33) is Tensorial's
# independent-component order, which unwrapping yields as is. A full stress
# tensor has no ABI slot: such data takes the generic kernels.
function tbparticles(P::StructArray)
    n = Int64(length(P))
    x = ptrs(P.x, 3)
    v = hasproperty(P, :v) ? ptrs(P.v, 3) : ntuple(_ -> C_NULL, 3)
    gv = hasproperty(P, :∇v) ? ptrs(P.∇v, 9) : ntuple(_ -> C_NULL, 9)
    sg = hasproperty(P, :σ) ? ptrs(P.σ, 6) : ntuple(_ -> C_NULL, 6)
    F = hasproperty(P, :F) ? ptrs(P.F, 9) : ntuple(_ -> C_NULL, 9)
    B = hasproperty(P, :B) ? ptrs(P.B, 9) : ntuple(_ -> C_NULL, 9)
    Cp = hasproperty(P, :Cᵖ⁻¹) ? ptrs(P.Cᵖ⁻¹, 6) : ntuple(_ -> C_NULL, 6)
    any(isnothing, (x, v, gv, sg, F, B, Cp)) && return nothing
    TbParticles(n, x, v, optptr(P, :V), optptr(P, :m), optptr(P, :l), gv, sg, F, B,
                optptr(P, :V⁰), optptr(P, :μ), optptr(P, :λ), optptr(P, :ε̄ᵖ), Cp)
end

function tbgrid(G::StructArray)
    m = first(something(ptrs(G.m, 1), (nothing,)))
    mv, f, v, vn = ptrs(G.mv, 3), ptrs(G.f, 3), ptrs(G.v, 3), ptrs(G.vⁿ, 3)
    any(isnothing, (m, mv, f, v, vn)) && return nothing
    sp = get(SPARSITY, G, nothing)  # the numbering b200_update_sparsity! keeps for this SpGrid
    sp === nothing && return TbGrid(m, mv, f, v, vn, C_NULL, C_NULL, C_NULL, 0)
    TbGrid(m, mv, f, v, vn, pointer(sp.numbering), pointer(sp.active), pointer(sp.nactive), sp.capacity)
end

# SpGrid (src/Grids/sparray.jl) on the B200 path: the library numbers the active
# node blocks into Int32 arrays kept here per grid; the SpIndices' own Int
# numbering gets a copy, so Tesserae's indexing of the SpArray agrees, and each
# field's data vector is resized to the stored node count.
mutable struct B200Sparsity
    numbering::CuVector{Int32}
    active::CuVector{Int32}
    nactive::CuVector{Int32}
    capacity::Int64
end
const SPARSITY = IdDict{Any,B200Sparsity}()

"""
    b200_update_sparsity!(grid::SpGrid, particles, partition)

`update_sparsity!(grid, particles.x)` through `tb_update_sparsity_*`: bins the
particles into `partition`, numbers the node blocks within one block of an
occupied block (src/Grids/sparsity.jl:19-60), resizes the grid's SpArray data
to the stored node count and zero-fills it. Returns that count.
"""
function b200_update_sparsity!(grid, particles, partition)
    spinds = Tesserae.get_spinds(grid)
    nb = length(Tesserae.blocknumbering(spinds))
    sp = get!(SPARSITY, grid) do
        B200Sparsity(CUDA.zeros(Int32, nb), CUDA.zeros(Int32, nb), CUDA.zeros(Int32, 2), 0)
    end
    bl = Tesserae.blocklength(spinds)
    nstored = Ref{Int64}(0)
    for attempt in 1:2
        sp.capacity = length(Tesserae.get_data(grid.m))
        gd = tbgrid(grid)
        GC.@preserve grid particles partition sp begin
            rc = ccall((sym(:tb_update_sparsity, form(particles)), libtb), Int32,
                       (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{TbGrid}, Ref{Int64}),
                       ctx(), tbmesh(grid.x), tbparticles(particles), tbpartition(Tesserae.strategy(partition)),
                       gd, nstored)
        end
        if rc == TB_ERR_CAPACITY && attempt == 1
            for name in propertynames(grid)
                A = getproperty(grid, name)
                A isa Tesserae.SpArray && resize!(Tesserae.get_data(A), nstored[])
            end
            continue
        end
        check(rc, "update_sparsity")
        break
    end
    Tesserae.blocknumbering(spinds) .= sp.numbering
    nstored[]
end

tbpartition(bs::GPUBlockStrategy) =
    TbPartition(pointer(bs.blockids), pointer(bs.counts), pointer(bs.offsets), pointer(bs.blocklist),
                pointer(bs.particleindices), Int64(length(bs.counts)))

function basis_kind(basis)
    basis isa BSpline{Quadratic} && return TB_BSPLINE_QUADRATIC
    basis isa uGIMP && return TB_UGIMP
    basis isa WLS{<:BSpline{Quadratic}} && return TB_WLS_BSPLINE_QUADRATIC
    basis isa WLS{<:uGIMP} && return TB_WLS_UGIMP
    basis isa KernelCorrection{<:BSpline{Quadratic}} && return TB_KC_BSPLINE_QUADRATIC
    basis isa KernelCorrection{<:uGIMP} && return TB_KC_UGIMP
    return nothing
end

# precision form from the element types: all Float64, Float32 state (F Float64),
# or Float32 state with Float64 positions
function form(P::StructArray)
    Tv = eltype(eltype(P.v))
    Tx = eltype(eltype(P.x))
    Tv === Float64 && return :f64
    Tx === Float64 ? :f32x64 : :f32
end
sym(name, f::Symbol) = Symbol(name, "_", f)

# ---- binning: update!(bs::GPUBlockStrategy, xₚ) ------------------------------

function Tesserae.update!(bs::GPUBlockStrategy, xₚ::StructVector{<:Vec{dim,T}}) where {dim,T}
    xs = ptrs(xₚ, 3)
    (ACTIVE[] && xs !== nothing) || return invoke(Tesserae.update!, Tuple{GPUBlockStrategy,AbstractVector}, bs, xₚ)
    n = length(xₚ)
    length(bs.blockids) == n || resize!(bs.blockids, n)
    length(bs.particleindices) == n || resize!(bs.particleindices, n)
    na, nass = Ref{Int64}(0), Ref{Int64}(0)
    desc = TbParticles(Int64(n), xs, ntuple(_ -> C_NULL, 3), C_NULL, C_NULL, C_NULL, ntuple(_ -> C_NULL, 9),
                       ntuple(_ -> C_NULL, 6), ntuple(_ -> C_NULL, 9), ntuple(_ -> C_NULL, 9), C_NULL, C_NULL,
                       C_NULL, C_NULL, ntuple(_ -> C_NULL, 6))
    GC.@preserve xₚ bs begin
        rc = ccall((T === Float32 ? :tb_bin_particles_f32 : :tb_bin_particles_f64, libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{Int64}, Ref{Int64}),
                   ctx(), tbmesh(bs.mesh), desc, tbpartition(bs), na, nass)
    end
    check(rc, "update!(partition)")
    bs.nactive[] = na[]
    bs.nassigned[] = nass[]
    bs
end

# ---- stored weights: update!(weights, particles, mesh) -----------------------

function Tesserae.update!(weights::Tesserae.BasisWeightArray{B,<:NamedTuple,<:CuArray}, particles::StructArray,
                          mesh::CartesianMesh; deferred::Bool=Tesserae.storageless(weights)) where {B}
    kind = basis_kind(Tesserae.basis(weights))
    desc = tbparticles(particles)
    generic() = invoke(Tesserae.update!, Tuple{AbstractArray{<:Tesserae.BasisWeight},StructArray,Tesserae.AbstractMesh},
                       weights, particles, mesh; deferred)
    (ACTIVE[] && kind !== nothing && desc !== nothing && !deferred) || return generic()
    Tesserae.set_deferring!(weights, false)
    vals = getfield(weights, :vals)
    wt = TbWeights(devptr(vals.w), devptr(vals.∇w), pointer(reinterpret(Int64, getfield(weights, :indices))))
    l = hasproperty(particles, :l) ? 0.0 : Float64(get(Tesserae.basis(weights), :l, 0.0))
    prm = TbParams(0.0, 0.0, 0.0, 0.0, 0.0, (0.0, 0.0, 0.0), l, 1.0, kind, TB_TRANSFER_FLIP, TB_MATERIAL_NEOHOOKEAN,
                   Int32(0), Int32(0), Int32(0), 0.0, 0.0)
    GC.@preserve weights particles begin
        rc = ccall((sym(:tb_update_weights, form(particles) === :f64 ? :f64 : :f32), libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbParams}, Ref{TbWeights}),
                   ctx(), tbmesh(mesh), desc, prm, wt)
    end
    check(rc, "update!(weights)")
    weights
end

# ---- recognition of transfer bodies by probing --------------------------------

# A one-particle host fixture: the particle's support lies inside a 4^3-cell mesh
# of spacing 1/4; every state field gets a random value of its type.
function probe_fixture(particles, grid, weights, rng)
    dim = length(eltype(particles.x))
    mesh = CartesianMesh(0.25, ntuple(_ -> (0.0, 1.0), dim)...)
    P = StructArray{eltype(particles)}(undef, 1)
    Tesserae.fillzero!(P)
    for name in propertynames(P)
        col = getproperty(P, name)
        E = eltype(col)
        col[1] = name === :x ? E(ntuple(_ -> 0.4 + 0.2rand(rng), dim)) :
                 name === :F ? E(I + 0.01randn(rng, dim, dim)) :
                 name in (:m, :V, :V⁰, :μ, :λ) ? E(0.5 + rand(rng)) :
                 E <: Number ? E(randn(rng)) : E(Tuple(randn(rng, length(E))))
    end
    G = Tesserae.generate_grid(eltype(grid), mesh)
    for name in (:m, :mv, :f, :v, :vⁿ)
        hasproperty(G, name) || continue
        col = getproperty(G, name)
        for i in eachindex(col)
            E = eltype(col)
            col[i] = E <: Number ? E(0.5 + rand(rng)) : E(Tuple(randn(rng, length(E))))
        end
    end
    W = Tesserae.generate_basis_weights(Tesserae.basis(weights), mesh, 1)
    Tesserae.update!(W, P, mesh)
    (; mesh, P, G, W)
end

# Host statement of the supported @G2P sets on the probe: FLIP/PIC blend or APIC,
# then F = (I + dt grad v) F and the material (README.md:79-86).
function g2p_candidate(fx, transfer, material, dt, alpha, a, b)
    (; P, G, W) = fx
    bw = W[1]
    xp, vp, Fp = P.x[1], P.v[1], P.F[1]
    vpic = zero(vp); dvf = zero(vp); L = zero(Fp); Bn = zero(Fp)
    for (ip, i) in enumerate(Tesserae.supportnodes(bw, G))
        w, ∇w = bw.w[ip], bw.∇w[ip]
        vpic += w * G.v[i]
        dvf += w * (G.v[i] - G.vⁿ[i])
        L += G.v[i] ⊗ ∇w
        Bn += w * G.v[i] ⊗ (G.x[i] - xp)
    end
    v = transfer === :apic ? vpic : (1 - alpha) * vpic + alpha * (vp + dvf)
    x = xp + vpic * dt
    F = (I + dt * L) * Fp
    J = det(F)
    σ = material === :neohookean ? (a * (F ⋅ F' - I) + b * log(J) * I) / J : b * (J - 1) * one(F)
    (; v, ∇v=L, x, F, σ=Tesserae.symmetric(σ), B=Bn)
end

# Scalars of a FLIP/APIC x Neo-Hookean/fluid set from a probe's outputs (least
# squares on the relations that are linear in each scalar).
function solve_scalars(fx, out, transfer, material)
    c0 = g2p_candidate(fx, transfer, material, 1.0, 1.0, 0.0, 0.0)
    vpic = (c0.x - fx.P.x[1])            # the PIC velocity times dt = 1
    dt = dot(out.x - fx.P.x[1], vpic) / max(dot(vpic, vpic), eps())
    alpha = 1.0
    if transfer === :flip
        cpic = g2p_candidate(fx, :flip, material, dt, 0.0, 0.0, 0.0).v
        cflip = g2p_candidate(fx, :flip, material, dt, 1.0, 0.0, 0.0).v
        d = cflip - cpic
        alpha = dot(out.v - cpic, d) / max(dot(d, d), eps())
    end
    F = out.F
    J = det(F)
    A1 = vec((F ⋅ F' - I) / J)
    A2 = vec(log(J) * one(F) / J)
    s = vec(Tesserae.Tensor{Tuple{length(fx.P.x[1]),length(fx.P.x[1])}}(out.σ))
    a, b = material === :neohookean ? hcat(A1, A2) \ s : (0.0, (vec((J - 1) * one(F)) \ s)[1])
    (dt, alpha, a, b)
end

approx(a, b) = isapprox(collect(Tuple(a)), collect(Tuple(b)); rtol=1e-5, atol=1e-8)

run_probe!(f, fx) = (f(fx.G, fx.P, fx.W, 1); fx)

const G2P_SETS = IdDict{DataType,Any}()

# (transfer, material) of a @G2P closure, or nothing.
function classify_g2p(f, particles, grid, weights)
    get!(G2P_SETS, typeof(f)) do
        for transfer in (:flip, :apic), material in (:neohookean, :fluid)
            (transfer === :apic) == hasproperty(particles, :B) || continue
            ok = true
            for seed in (1, 2)
                fx = probe_fixture(particles, grid, weights, MersenneTwister(seed))
                P0 = deepcopy(fx.P)
                run_probe!(f, fx)
                out = fx.P[1]
                fx0 = (; fx..., P=P0)
                dt, alpha, a, b = solve_scalars(fx0, out, transfer, material)
                ref = g2p_candidate(fx0, transfer, material, dt, alpha, a, b)
                ok &= approx(out.v, ref.v) && approx(out.x, ref.x) && approx(out.F, ref.F) &&
                      approx(out.σ, ref.σ) && (transfer === :flip || approx(out.B, ref.B))
                ok || break
            end
            ok && return (transfer, material)
        end
        nothing
    end
end

# ---- P2G: the scatter half of @P2G -------------------------------------------

const P2G_SETS = IdDict{DataType,Any}()

# (apic, gravity) of a block-scheduled @P2G body scattering m, mv, f: run the
# particle body on the probe and compare with m = sum w m_p,
# mv = sum w m_p (v_p [+ B D^-1 (x_i - x_p)]), f = sum (-V sigma grad w + w m_p g).
function classify_p2g(bodies, particles, grid, weights)
    fx = probe_fixture(particles, grid, weights, MersenneTwister(3))
    Tesserae.fillzero!(fx.G.m); Tesserae.fillzero!(fx.G.mv); Tesserae.fillzero!(fx.G.f)
    bodies.particle(fx.G, fx.P, fx.W, 1)
    bw = fx.W[1]
    mp = hasproperty(fx.P, :m) ? fx.P.m[1] : 1.0
    nodes = collect(Tesserae.supportnodes(bw, fx.G))
    msum = sum(bw.w[ip] * mp for ip in eachindex(nodes))
    fint = sum(-fx.P.V[1] * fx.P.σ[1] ⋅ bw.∇w[ip] for ip in eachindex(nodes))
    g = (sum(fx.G.f[i] for i in nodes) - fint) / msum
    apic = hasproperty(fx.P, :B)
    for (ip, i) in enumerate(nodes)
        w = bw.w[ip]
        vv = fx.P.v[1] + (apic ? fx.P.B[1] ⋅ (4 / 0.25^2) ⋅ (fx.G.x[i] - fx.P.x[1]) : zero(fx.P.v[1]))
        approx((fx.G.m[i],), (w * mp,)) && approx(fx.G.mv[i], w * mp * vv) &&
            approx(fx.G.f[i], -fx.P.V[1] * fx.P.σ[1] ⋅ bw.∇w[ip] + w * mp * g) || return nothing
    end
    (apic, Tuple(g))
end

function params(weights, particles, transfer, material; dt=0.0, alpha=1.0, a=0.0, b=0.0, g=(0.0, 0.0, 0.0))
    kind = basis_kind(Tesserae.basis(weights))
    mu, lam = material === :fluid ? (0.0, b) : (a, b)
    TbParams(dt, 0.0, 0.0, mu, lam, ntuple(d -> d <= length(g) ? Float64(g[d]) : 0.0, 3),
             Float64(get(Tesserae.basis(weights), :l, 0.0)), alpha, kind,
             transfer === :apic ? TB_TRANSFER_APIC : TB_TRANSFER_FLIP,
             material === :fluid ? TB_MATERIAL_FLUID : TB_MATERIAL_NEOHOOKEAN,
             Int32(0), Int32(0), Int32(0), 0.0, 0.0)
end

function Tesserae.P2G(bodies::P2GBodies{(:m, :mv, :f)}, device::CUDADevice, sched::Val, grid, particles, weights,
                      partition::Partition{<:GPUBlockStrategy}, zeroed::Tuple=())
    generic() = invoke(Tesserae.P2G, Tuple{P2GBodies,GPUDevice,Val,Any,Any,Any,Partition{<:GPUBlockStrategy},Tuple},
                       bodies, device, sched, grid, particles, weights, partition, zeroed)
    pd, gd, kind = tbparticles(particles), tbgrid(grid), basis_kind(Tesserae.basis(weights))
    (ACTIVE[] && pd !== nothing && gd !== nothing && kind !== nothing) || return STRICT[] ? unsupported("@P2G") : generic()
    set = get!(() -> classify_p2g(bodies, particles, grid, weights), P2G_SETS, typeof(bodies))
    set === nothing && return STRICT[] ? unsupported("@P2G") : generic()
    apic, _ = set
    _, g = classify_p2g(bodies, particles, grid, weights)  # gravity as captured this call
    prm = params(weights, particles, apic ? :apic : :flip, :neohookean; g)
    f = form(particles)
    GC.@preserve grid particles partition begin
        rc = ccall((sym(:tb_p2g, f === :f64 ? :f64 : :f32), libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{TbGrid}, Ref{TbParams}),
                   ctx(), tbmesh(grid.x), pd, tbpartition(Tesserae.strategy(partition)), gd, prm)
    end
    check(rc, "@P2G")
end

unsupported(what) = error("$what: this transfer body is not one of the equation sets libtesserae_b200 implements " *
                          "(TESSERAE_B200_STRICT=1)")

# ---- the @P2G grid half: vn = mv/m, v = vn + dt f/m (guarded) -----------------

const GRID_SETS = IdDict{DataType,Bool}()

# dt of a grid-half closure, or nothing: run it on a probe grid node and compare
# with vⁿ = mv/m and v = vⁿ + dt f/m (docs/src/gpu.md:309-310).
function grid_half_dt(f, grid)
    mesh = CartesianMesh(0.25, ntuple(_ -> (0.0, 1.0), length(eltype(grid.x)))...)
    G = Tesserae.generate_grid(eltype(grid), mesh)
    rng = MersenneTwister(4)
    i = CartesianIndex(ntuple(_ -> 2, ndims(G)))
    G.m[i] = 0.5 + rand(rng)
    G.mv[i] = eltype(G.mv)(Tuple(randn(rng, length(eltype(G.mv)))))
    G.f[i] = eltype(G.f)(Tuple(randn(rng, length(eltype(G.f)))))
    f(G, i)
    approx(G.vⁿ[i], G.mv[i] / G.m[i]) || return nothing
    a = G.f[i] / G.m[i]
    dot(G.v[i] - G.vⁿ[i], a) / max(dot(a, a), eps())
end

function Tesserae.foreach_loop(f, device::CUDADevice, sched::Val, grid::StructArray)
    generic() = invoke(Tesserae.foreach_loop, Tuple{Any,GPUDevice,Val,Any}, f, device, sched, grid)
    gd = tbgrid(grid)
    (ACTIVE[] && gd !== nothing && hasproperty(grid, :vⁿ)) || return generic()
    recognised = get!(() -> grid_half_dt(f, grid) !== nothing, GRID_SETS, typeof(f))
    recognised || return generic()
    dt = grid_half_dt(f, grid)
    prm = TbParams(dt, 0.0, 0.0, 0.0, 0.0, (0.0, 0.0, 0.0), 0.0, 1.0, TB_BSPLINE_QUADRATIC, TB_TRANSFER_FLIP,
                   TB_MATERIAL_NEOHOOKEAN, Int32(0), Int32(0), Int32(0), 0.0, 0.0)
    GC.@preserve grid begin
        rc = ccall((eltype(eltype(grid.v)) === Float64 ? :tb_grid_update_f64 : :tb_grid_update_f32, libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbGrid}, Ref{TbParams}), ctx(), tbmesh(grid.x), gd, prm)
    end
    check(rc, "@P2G grid half")
end
# Slip-wall slices (`@foreach grid[:, :, begin]=>i`) keep Tesserae's generic GPU
# kernel: a masked store on a face, no scatter or gather.

# ---- G2P ---------------------------------------------------------------------

function Tesserae.G2P(f, device::CUDADevice, sched::Val, grid, particles::StructArray, weights)
    generic() = invoke(Tesserae.G2P, Tuple{Any,GPUDevice,Val,Any,Any,Any}, f, device, sched, grid, particles, weights)
    pd, gd = tbparticles(particles), tbgrid(grid)
    (ACTIVE[] && pd !== nothing && gd !== nothing && basis_kind(Tesserae.basis(weights)) !== nothing) ||
        return STRICT[] ? unsupported("@G2P") : generic()
    set = classify_g2p(f, particles, grid, weights)
    set === nothing && return STRICT[] ? unsupported("@G2P") : generic()
    transfer, material = set
    fx = probe_fixture(particles, grid, weights, MersenneTwister(1))
    P0 = deepcopy(fx.P)
    run_probe!(f, fx)
    dt, alpha, a, b = solve_scalars((; fx..., P=P0), fx.P[1], transfer, material)
    prm = params(weights, particles, transfer, material; dt, alpha, a, b)
    GC.@preserve grid particles begin
        rc = ccall((sym(:tb_g2p, form(particles) === :f64 ? :f64 : :f32), libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbGrid}, Ref{TbParticles}, Ref{TbParams}),
                   ctx(), tbmesh(grid.x), gd, pd, prm)
    end
    check(rc, "@G2P")
end

# ---- reorder_particles! and the contiguity score ------------------------------

function Tesserae.reorder_particles!(particles::StructVector, bs::GPUBlockStrategy; threshold=1)
    pd = tbparticles(particles)
    (ACTIVE[] && pd !== nothing) ||
        return invoke(Tesserae.reorder_particles!, Tuple{StructVector,GPUBlockStrategy}, particles, bs; threshold)
    did = Ref{Int32}(0)
    GC.@preserve particles bs begin
        rc = ccall((sym(:tb_reorder_particles, form(particles)), libtb), Int32,
                   (Ptr{Cvoid}, Int32, Ref{TbParticles}, Ref{TbPartition}, Float64, Ref{Int32}),
                   ctx(), Int32(length(eltype(particles.x))), pd, tbpartition(bs), Float64(threshold), did)
    end
    check(rc, "reorder_particles!")
    did[] != 0
end

function Tesserae.block_ordered_particle_contiguity(bs::GPUBlockStrategy{dim,<:Any,<:CuArray}) where {dim}
    ACTIVE[] || return invoke(Tesserae.block_ordered_particle_contiguity, Tuple{GPUBlockStrategy}, bs)
    score = Ref{Float64}(0.0)
    GC.@preserve bs begin
        rc = ccall((:tb_particle_contiguity, libtb), Int32, (Ptr{Cvoid}, Ref{TbPartition}, Int64, Ref{Float64}),
                   ctx(), tbpartition(bs), Int64(length(bs.blockids)), score)
    end
    check(rc, "block_ordered_particle_contiguity")
    score[]
end

# ---- the fused loop body and its adjoint --------------------------------------

"""
    b200_step!(grid, particles, partition, params::TbParams, nsteps)

The whole README.md:66-87 loop body (bin, P2G, grid half, G2P) `nsteps` times on
the device without host synchronisation (`tb_step_*`; the precision form follows
the element types).
"""
function b200_step!(grid, particles, partition, prm::TbParams, nsteps::Integer)
    pd, gd = tbparticles(particles), tbgrid(grid)
    (pd === nothing || gd === nothing) && error("b200_step!: particles and grid must be in the b200 layout")
    GC.@preserve grid particles partition begin
        rc = ccall((sym(:tb_step, form(particles)), libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{TbGrid}, Ref{TbParams}, Int32),
                   ctx(), tbmesh(grid.x), pd, tbpartition(Tesserae.strategy(partition)), gd, prm, Int32(nsteps))
    end
    check(rc, "b200_step!")
end

"""
    xT = b200_rollout(v0, particles, grid, partition, params, nsteps; checkpoint_every=nothing)

Final positions (a dim x n Float64 matrix) of a rollout from the initial
velocities `v0` (dim x n). Differentiable: the `rrule` below runs the
checkpointed tape (`tb_tape_forward_*`) forward and `tb_tape_backward_*` in the
pullback, giving d loss / d v0 (the Julia counterpart of the torch
autograd.Function of the Python host mirror). `checkpoint_every = nothing`
keeps the whole tape (interval 1: the pullback runs no forward step) when
`tb_tape_bytes` says it takes at most 60% of the device's free memory, else
checkpoints every 20 steps.
"""
function b200_rollout(v0::CuMatrix, particles, grid, partition, prm::TbParams, nsteps::Integer;
                      checkpoint_every::Union{Integer,Nothing}=nothing)
    if checkpoint_every === nothing
        elem = form(particles) === :f64 ? 8 : 4
        bytes = GC.@preserve grid ccall((:tb_tape_bytes, libtb), Int64,
                                        (Ref{TbMesh}, Int64, Int32, Int32, Int32, Int32, Int32),
                                        tbmesh(grid.x), length(particles), Int32(elem),
                                        Int32(prm.transfer == TB_TRANSFER_APIC), Int32(form(particles) === :f32x64),
                                        Int32(nsteps), Int32(1))
        checkpoint_every = 0 <= bytes <= 0.6 * CUDA.available_memory() ? 1 : 20
    end
    setv!(particles, v0)
    pd, gd = tbparticles(particles), tbgrid(grid)
    GC.@preserve grid particles partition begin
        rc = ccall((sym(:tb_tape_forward, form(particles)), libtb), Int32,
                   (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{TbGrid}, Ref{TbParams},
                    Int32, Int32),
                   ctx(), tbmesh(grid.x), pd, tbpartition(Tesserae.strategy(partition)), gd, prm, Int32(nsteps),
                   Int32(checkpoint_every))
    end
    check(rc, "tape forward")
    xT = CUDA.zeros(Float64, length(eltype(particles.x)), length(particles))
    for (d, c) in enumerate(components_of(particles.x))
        xT[d, :] .= Float64.(c)
    end
    xT
end

function setv!(particles, v0)
    for (d, c) in enumerate(components_of(particles.v))
        c .= view(v0, d, :)
    end
end

function ChainRulesCore.rrule(::typeof(b200_rollout), v0, particles, grid, partition, prm, nsteps;
                              checkpoint_every=nothing)
    xT = b200_rollout(v0, particles, grid, partition, prm, nsteps; checkpoint_every)
    function pullback(x̄)
        dim, n = size(xT)
        gx = CuArray{Float64}(unthunk(x̄))
        gv = CUDA.zeros(Float64, dim, n)
        gF = CUDA.zeros(Float64, dim * dim, n)
        row(A, d) = reinterpret(Ptr{Float64}, pointer(view(A, d, :)))
        adj = TbAdjoint(ntuple(d -> d <= dim ? row(gx, d) : Ptr{Float64}(0), 3),
                        ntuple(d -> d <= dim ? row(gv, d) : Ptr{Float64}(0), 3),
                        ntuple(k -> k <= dim * dim ? row(gF, k) : Ptr{Float64}(0), 9),
                        Ptr{Float64}(0), Ptr{Float64}(0), ntuple(_ -> Ptr{Float64}(0), 9))
        pd, gd = tbparticles(particles), tbgrid(grid)
        GC.@preserve grid particles partition gx gv gF begin
            rc = ccall((sym(:tb_tape_backward, form(particles)), libtb), Int32,
                       (Ptr{Cvoid}, Ref{TbMesh}, Ref{TbParticles}, Ref{TbPartition}, Ref{TbGrid}, Ref{TbParams},
                        Ref{TbAdjoint}),
                       ctx(), tbmesh(grid.x), pd, tbpartition(Tesserae.strategy(partition)), gd, prm, adj)
        end
        check(rc, "tape backward")
        (NoTangent(), gv, NoTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent())
    end
    xT, pullback
end

export b200, b200_x64, b200_preserve, b200_step!, b200_rollout, b200_update_sparsity!

end # module
