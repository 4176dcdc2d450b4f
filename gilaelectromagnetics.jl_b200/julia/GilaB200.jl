#=
GilaB200.jl -- drop-in device path for GilaElectromagnetics.jl's Green operator.

Keeps the reference's operator API (src/glaMemSup.jl GlaOprMem / GlaOpr
constructors, src/glaAct.jl egoOpr!, src/glaLinAlg.jl *, mul!, adjoint, size,
eltype, glaSze and predicates) and runs every matvec in libgila_b200.so (sm_100a
CUDA) through ccall.  The C declarations are in include/gila_b200.h.

Usage (a maintainer would swap these in for the CUDA.jl device path):

    using GilaElectromagnetics          # GlaVol, GlaKerOpt, glaSze, ...
    include("GilaB200.jl"); using .GilaB200
    mem = GilaB200.GlaOprMem(GlaKerOpt(true), GlaVol((32,32,32), (1//32,1//32,1//32), (0//1,0//1,0//1)))
    y = GilaB200.egoOpr!(mem, x)        # x::Array{ComplexF64,4} or CuArray

This file is not exercised in the build's test-suite (no Julia toolchain in
the build image); the same entry points are tested through Python ctypes.
=#
module GilaB200

using LinearAlgebra

const LIB = get(ENV, "GILA_B200_LIB", joinpath(@__DIR__, "..", "libgila_b200.so"))

# gila_status codes (include/gila_b200.h)
const GILA_OK = Cint(0)
const GILA_ERR_SIZE = Cint(2)
const GILA_ERR_TYPE = Cint(3)
const GILA_C64 = Cint(0)
const GILA_C128 = Cint(1)

struct CVol               # gila_vol
    cel::NTuple{3,Int64}
    scl_num::NTuple{3,Int64}; scl_den::NTuple{3,Int64}
    org_num::NTuple{3,Int64}; org_den::NTuple{3,Int64}
    grd_num::NTuple{3,Int64}; grd_den::NTuple{3,Int64}
end

struct CKopt              # gila_kopt
    frq_re::Cdouble; frq_im::Cdouble
    int_ord::Int32; adj_mod::Int32; dev_mod::Int32
    num_trd::NTuple{3,Int32}; num_blk::NTuple{3,Int32}
end

cvol(v) = CVol(Int64.(Tuple(v.cel)),
    Int64.(numerator.(v.scl)), Int64.(denominator.(v.scl)),
    Int64.(numerator.(v.org)), Int64.(denominator.(v.org)),
    Int64.(numerator.(Rational.(step.(v.grd)))), Int64.(denominator.(Rational.(step.(v.grd)))))

function ckopt(o)
    t = isempty(o.numTrd) ? (0, 0, 0) : o.numTrd
    b = isempty(o.numBlk) ? (0, 0, 0) : o.numBlk
    CKopt(real(o.frqPhz), imag(o.frqPhz), Int32(o.intOrd), Int32(o.adjMod), Int32(1), Int32.(t), Int32.(b))
end

dtcode(::Type{ComplexF64}) = GILA_C128
dtcode(::Type{ComplexF32}) = GILA_C64
dtcode(T) = throw(ArgumentError("setTyp must be a subtype of Complex"))

lasterr() = unsafe_string(ccall((:gila_last_error, LIB), Cstring, ()))

function check(st)
    st == GILA_OK && return nothing
    msg = lasterr()
    st == GILA_ERR_TYPE && throw(AssertionError(msg))
    error(msg)
end

const CTX = Ref{Ptr{Cvoid}}(C_NULL)
function ctx()
    if CTX[] == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:gila_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, r))
        CTX[] = r[]
    end
    CTX[]
end

"""GlaOprMem backed by libgila_b200 (src/glaMemSup.jl:16-20)."""
mutable struct GlaOprMem{T}
    h::Ptr{Cvoid}
    cmpInf::Any
    trgVol::Any
    srcVol::Any
    function GlaOprMem{T}(h, c, t, s) where {T}
        m = new{T}(h, c, t, s)
        finalizer(x -> ccall((:gila_opr_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), m)
        m
    end
end

function GlaOprMem(cmpInf, trgVol, srcVol=nothing; egoFur=nothing, setTyp::DataType=ComplexF64)
    code = dtcode(setTyp)
    tv = Ref(cvol(trgVol)); o = Ref(ckopt(cmpInf))
    sv = srcVol === nothing ? C_NULL : Ref(cvol(srcVol))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    if egoFur === nothing
        check(ccall((:gila_opr_create, LIB), Cint,
            (Ptr{Cvoid}, Ref{CVol}, Ptr{CVol}, Ref{CKopt}, Cint, Ref{Ptr{Cvoid}}),
            ctx(), tv, srcVol === nothing ? C_NULL : sv, o, code, r))
    else
        fur = [Array(f) for f in egoFur]                 # host copies, reference layout
        ptrs = Ptr{Cvoid}[pointer(f) for f in fur]
        dims = zeros(Int64, 6, 8)
        for e in 1:8, k in 1:6
            dims[k, e] = size(fur[e], k)
        end
        GC.@preserve fur begin
            check(ccall((:gila_opr_create_from_fur, LIB), Cint,
                (Ptr{Cvoid}, Ref{CVol}, Ptr{CVol}, Ref{CKopt}, Cint, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Cint,
                 Ref{Ptr{Cvoid}}),
                ctx(), tv, srcVol === nothing ? C_NULL : sv, o, code, ptrs, dims,
                dtcode(eltype(fur[1])), r))
        end
    end
    GlaOprMem{setTyp}(r[], cmpInf, trgVol, srcVol === nothing ? trgVol : srcVol)
end

"""GlaOpr wrapper (src/glaMem.jl:116-119)."""
struct GlaOpr
    mem::GlaOprMem
end

function GlaOpr(cel::NTuple{3,Int}, scl::NTuple{3,Rational}, org::NTuple{3,Rational}=(0//1, 0//1, 0//1);
                useGpu::Bool=true, setTyp::DataType=ComplexF64)
    setTyp <: Complex || throw(ArgumentError("setTyp must be a subtype of Complex"))
    vol = (cel=cel, scl=scl, org=org, grd=[StepRange(o, s, o) for (o, s) in zip(org, scl)])
    GlaOpr(GlaOprMem((frqPhz=1.0 + 0im, intOrd=32, adjMod=false, numTrd=(), numBlk=()), vol; setTyp=setTyp))
end

function sizes(m::GlaOprMem)
    i = zeros(Int64, 4); o = zeros(Int64, 4)
    check(ccall((:gila_opr_input_size, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}), m.h, i))
    check(ccall((:gila_opr_output_size, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}), m.h, o))
    Tuple(i), Tuple(o)
end

"""egoOpr!(egoMem, actVec) (src/glaAct.jl:33-49).  Host Arrays and CuArrays
(any pointer the CUDA runtime can classify) are accepted; the result has the
input's array type."""
function egoOpr!(m::GlaOprMem{T}, actVec::AbstractArray{T}) where {T}
    insz, outsz = sizes(m)
    size(actVec) == insz || error("Size of input vector does not match size of source volume. " *
                                  "Required data layout is (srcCelX, srcCelY, srcCelZ, 3).")
    out = similar(actVec, T, outsz...)
    check(ccall((:gila_opr_apply, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64, Int64, Ptr{Cvoid}),
        m.h, dtcode(T), pointer(actVec), length(actVec), pointer(out), length(out), 1, C_NULL))
    out
end

Base.eltype(o::GlaOpr) = typeof(o.mem).parameters[1]
glaSze(o::GlaOpr) = ((Tuple(o.mem.trgVol.cel)..., 3), (Tuple(o.mem.srcVol.cel)..., 3))
glaSze(o::GlaOpr, d::Int) = glaSze(o)[d]
Base.size(o::GlaOpr) = (3 * prod(o.mem.trgVol.cel), 3 * prod(o.mem.srcVol.cel))
Base.size(o::GlaOpr, d::Int) = size(o)[d]
LinearAlgebra.issymmetric(::GlaOpr) = false
LinearAlgebra.ishermitian(::GlaOpr) = false
LinearAlgebra.isposdef(::GlaOpr) = false
LinearAlgebra.isdiag(::GlaOpr) = false
isadjoint(o::GlaOpr) = o.mem.cmpInf.adjMod
isselfoperator(o::GlaOpr) = o.mem.srcVol == o.mem.trgVol
isexternaloperator(o::GlaOpr) = !isselfoperator(o)

function Base.adjoint(o::GlaOpr)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:gila_opr_adjoint, LIB), Cint, (Ptr{Cvoid}, Ref{Ptr{Cvoid}}), o.mem.h, r))
    c = o.mem.cmpInf
    c2 = merge(NamedTuple{propertynames(c)}(getproperty.(Ref(c), propertynames(c))), (adjMod=!c.adjMod,))
    GlaOpr(GlaOprMem{eltype(o)}(r[], c2, o.mem.srcVol, o.mem.trgVol))
end

function Base.:*(o::GlaOpr, x::AbstractArray{T,4}) where {T<:Complex}
    @assert T <: eltype(o) "Input array must have the same element type as the operator. eltype(opr) = $(eltype(o))"
    egoOpr!(o.mem, x)              # the library never mutates its input
end

function Base.:*(o::GlaOpr, x::AbstractArray{T}) where {T<:Complex}
    y = o * reshape(x, glaSze(o, 2))
    length(x) == prod(glaSze(o, 1)) && return reshape(y, size(x))
    ndims(x) == 1 && return vec(y)
    reshape(y, glaSze(o, 1))
end

"""mul!(y, G, x, α, β) (src/glaLinAlg.jl:61-69) with the axpby fused on the GPU."""
function LinearAlgebra.mul!(y::AbstractArray{T}, o::GlaOpr, x::AbstractArray{T}, α::Number, β::Number) where {T<:Complex}
    @assert T <: eltype(o) "Input array must have the same element type as the operator."
    length(x) == prod(glaSze(o, 2)) || throw(DimensionMismatch("input length"))
    a = Cdouble[real(α), imag(α)]; b = Cdouble[real(β), imag(β)]
    check(ccall((:gila_opr_apply_axpby, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cvoid}, Int64, Ptr{Cdouble}, Ptr{Cvoid}, Int64, Int64, Ptr{Cvoid}),
        o.mem.h, dtcode(T), a, pointer(x), length(x), b, pointer(y), length(y), 1, C_NULL))
    y
end

# ---- kernel cache files ----------------------------------------------------
# The reference keeps egoFur between sessions with Serialization / JLD2
# (test/runtests.jl:38-98, examples/GilaOperators.jl:28-55).  GILAFUR1 is the
# library's raw little-endian format (layout in include/gila_b200.h,
# gila_opr_save): a 768-byte header, then the 8 branches in the reference
# layout.  readGilaFur / writeGilaFur read and write it in plain Julia, so a
# kernel cached by either side feeds GlaOprMem(...; egoFur = fur) on the other.

littleendian() = ENDIAN_BOM == 0x04030201 || error("GILAFUR files are little-endian; this host is not")

function furvol(a::Vector{Int64})
    scl = Tuple(a[4:6] .// a[7:9]); org = Tuple(a[10:12] .// a[13:15]); grd = Tuple(a[16:18] .// a[19:21])
    (cel=Tuple(a[1:3]), scl=scl, org=org, grd=[StepRange(o, g, o) for (o, g) in zip(org, grd)])
end

"""Header of a GILAFUR1 file: element type, self flag, GlaKerOpt fields,
volumes (after GlaOprMem's even-cell regeneration) and branch extents."""
function readGilaFurHeader(io::IO)
    littleendian()
    String(read(io, 8)) == "GILAFUR1" || error("not a GILAFUR1 kernel file")
    h = [read(io, Int32) for _ in 1:6]
    h[1] == 1 || error("unsupported GILAFUR version $(h[1])")
    frq = complex(read(io, Float64), read(io, Float64))
    v = [read(io, Int64) for _ in 1:42]
    dims = reshape([read(io, Int64) for _ in 1:48], 6, 8)
    (T=h[2] == 1 ? ComplexF64 : ComplexF32, self=h[3] == 1, adjMod=h[4] == 1, intOrd=Int(h[5]),
     frqPhz=frq, trgVol=furvol(v[1:21]), srcVol=furvol(v[22:42]), dims=dims)
end
readGilaFurHeader(path::AbstractString) = open(readGilaFurHeader, path, "r")

"""(egoFur, header) of a GILAFUR1 file; egoFur is the Vector{Array{T,6}} that
GlaOprMem(...; egoFur = egoFur) accepts (src/glaMemSup.jl:16-20)."""
function readGilaFur(path::AbstractString)
    open(path, "r") do io
        meta = readGilaFurHeader(io)
        seek(io, 768)
        fur = [read!(io, Array{meta.T,6}(undef, Tuple(meta.dims[:, e])...)) for e in 1:8]
        fur, meta
    end
end

"""Write a reference egoFur (host or device arrays) with its operator's
volumes and GlaKerOpt as a GILAFUR1 file that gila_opr_load reads."""
function writeGilaFur(path::AbstractString, egoFur::AbstractVector, trgVol, srcVol, cmpInf)
    littleendian()
    T = eltype(egoFur[1])
    slf = srcVol === nothing || srcVol == trgVol
    open(path, "w") do io
        write(io, b"GILAFUR1")
        write(io, Int32(1), dtcode(T), Int32(slf), Int32(cmpInf.adjMod), Int32(cmpInf.intOrd), Int32(0))
        write(io, Float64(real(cmpInf.frqPhz)), Float64(imag(cmpInf.frqPhz)))
        for v in (trgVol, slf ? trgVol : srcVol)
            c = cvol(v)
            write(io, Int64[c.cel..., c.scl_num..., c.scl_den..., c.org_num..., c.org_den..., c.grd_num..., c.grd_den...])
        end
        write(io, Int64[size(egoFur[e], k) for k in 1:6, e in 1:8])
        for e in 1:8
            write(io, Array{T}(egoFur[e]))
        end
    end
    nothing
end

"""Save an operator's kernel to a GILAFUR1 file (gila_opr_save)."""
glaSave(m::GlaOprMem, path::AbstractString) =
    check(ccall((:gila_opr_save, LIB), Cint, (Ptr{Cvoid}, Cstring), m.h, path))

"""The operator stored in a GILAFUR1 file, cast to setTyp (gila_opr_load)."""
function glaLoad(path::AbstractString; setTyp::DataType=ComplexF64)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:gila_opr_load, LIB), Cint, (Ptr{Cvoid}, Cstring, Cint, Ref{Ptr{Cvoid}}),
                ctx(), path, dtcode(setTyp), r))
    h = readGilaFurHeader(path)
    opt = (frqPhz=h.frqPhz, intOrd=h.intOrd, adjMod=h.adjMod, numTrd=(), numBlk=())
    GlaOprMem{setTyp}(r[], opt, h.trgVol, h.self ? h.trgVol : h.srcVol)
end

# ---- the scattering solve (examples/GilaOperators.jl:57-96) ---------------

struct CSolveOpts         # gila_solve_opts
    tol::Cdouble; ell::Int32; mixed::Int32; max_matvecs::Int32; max_restarts::Int32
    delta::Cdouble; x0::Int32; no_graph::Int32; keep::Int32
end

struct CSolveInfo         # gila_solve_info
    iters::Int32; outer::Int32; matvecs_f64::Int32; matvecs_f32::Int32
    rel_res::Cdouble; converged::Int32; breakdowns::Int32
end

"""LippmannSchwinger(G, medium): x -> x - medium .* (G x) (examples/GilaOperators.jl:57-82)."""
struct LippmannSchwinger
    greens_op::GlaOpr
    medium::Array{ComplexF64,3}
    g32::Base.RefValue{Any}
end
function LippmannSchwinger(G::GlaOpr, medium::AbstractArray{<:Complex,3})
    glaSze(G, 1)[1:3] == size(medium) ||
        throw(DimensionMismatch("Green's operator and medium must have the same size."))
    LippmannSchwinger(G, ComplexF64.(medium), Ref{Any}(nothing))
end

function Base.:*(ls::LippmannSchwinger, x::AbstractArray)
    gx = reshape(ls.greens_op * x, glaSze(ls.greens_op, 1))
    x - reshape(ls.medium .* gx, size(x))
end
LinearAlgebra.mul!(y::AbstractArray, ls::LippmannSchwinger, x::AbstractArray) = y .= ls * x

function g32(ls::LippmannSchwinger)
    if ls.g32[] === nothing
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:gila_opr_cast, LIB), Cint, (Ptr{Cvoid}, Cint, Ref{Ptr{Cvoid}}),
                    ls.greens_op.mem.h, GILA_C64, r))
        m = ls.greens_op.mem
        ls.g32[] = GlaOprMem{ComplexF32}(r[], m.cmpInf, m.trgVol, m.srcVol)
    end
    ls.g32[]
end

"""solve(ls, i) (examples/scattering_film.jl:58-61): BiCGStab(l) on the GPU,
`i` of size (Nx,Ny,Nz,3) or (Nx,Ny,Nz,3,nrhs); mixed = ComplexF32 Krylov with
FP64 reliable updates.  Returns the solution (same shape) and the info."""
function solve(ls::LippmannSchwinger, i::AbstractArray{ComplexF64}; tol=1e-6, mixed=true, ell=2,
               max_matvecs=4000, keep=false)
    n = 3 * prod(glaSze(ls.greens_op, 1)[1:3])
    nrhs = length(i) ÷ n
    b = Array(i); x = similar(b)
    opts = Ref(CSolveOpts(tol, ell, mixed, max_matvecs, 0, 0.0, 0, 0, keep))  # delta 0: the library default
    info = Ref{CSolveInfo}()
    G32 = mixed ? g32(ls).h : C_NULL
    check(ccall((:gila_ls_solve, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Int64,
                 Ref{CSolveOpts}, Ref{CSolveInfo}, Ptr{Cdouble}, Ptr{Cvoid}),
                ls.greens_op.mem.h, G32, ls.medium, b, x, nrhs, opts, info, C_NULL, C_NULL))
    x, info[]
end

end # module
