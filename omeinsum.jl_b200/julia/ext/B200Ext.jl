# B200Ext: OMEinsum.jl's B200 backend, calling libomeb200 (include/ome_b200.h)
# through its C ABI.
#
# Loaded as a package extension when CUDA.jl is loaded; __init__ stores the
# implementations in the Refs of src/b200_backend.jl (the registry pattern of
# src/backends.jl:170-184 and ext/CuTENSORExt.jl:13-16).  The dispatch points
# in ext/CUDAExt.jl (ext/CUDAExt_b200_hooks.jl) call them when
# `get_einsum_backend() isa B200Backend`.
#
# The library path comes from the environment variable OME_B200_LIB at load
# time (default: "libomeb200" on the loader's search path).
module B200Ext

using CUDA
using Libdl
import OMEinsum
using OMEinsum: EinCode, NestedEinsum, SlicedEinsum, getixs, getiy, getixsv, getiyv, isleaf, siblings,
                tensorindex, rootcode, get_einsum_backend, B200Backend

# ----------------------------------------------------------------------------
# library handle and symbols
# ----------------------------------------------------------------------------

const HANDLE = Ref{Ptr{Cvoid}}(C_NULL)
const SYMBOLS = Dict{Symbol,Ptr{Cvoid}}()

function sym(name::Symbol)
    p = get(SYMBOLS, name, C_NULL)
    if p == C_NULL
        p = Libdl.dlsym(HANDLE[], name)
        SYMBOLS[name] = p
    end
    return p
end

# include/ome_b200.h: ome_tensor (C layout: pointer, int32 + padding, 3 pointers)
struct OmeTensor
    data::Ptr{Cvoid}
    ndim::Int32
    dims::Ptr{Int64}
    strides::Ptr{Int64}   # elements; CuArrays are column-major like the ABI's default
    labels::Ptr{Int32}
end

# ome_status -> Julia exceptions (src/interfaces.jl:78-88, 100)
function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(@ccall $(sym(:ome_last_error))()::Cstring)
    rc == 1 && throw(ArgumentError(msg))
    rc == 2 && throw(DimensionMismatch(msg))
    rc == 4 && throw(OutOfMemoryError())
    error("libomeb200 status $rc: $msg")
end

# ome_dtype
ome_dtype(::Type{Float32}) = Cint(0)
ome_dtype(::Type{Float64}) = Cint(1)
ome_dtype(::Type{ComplexF32}) = Cint(2)
ome_dtype(::Type{ComplexF64}) = Cint(3)
ome_dtype(::Type{Int64}) = Cint(4)
ome_dtype(::Type{Bool}) = Cint(5)
function ome_dtype(::Type{T}) where {T}
    # TropicalNumbers.jl's Tropical{Float32} / Tropical{Float64}: one isbits field, the content
    if nameof(T) === :Tropical && isbitstype(T) && fieldcount(T) == 1
        fieldtype(T, 1) === Float32 && return Cint(6)
        fieldtype(T, 1) === Float64 && return Cint(7)
    end
    throw(ArgumentError("B200Backend: element type $T is not supported"))
end

# sx, sy as one value of the call's element type (Bool -> one/zero, as
# OMEinsum's @addmul! treats true/false)
scalar(::Type{T}, v::Bool) where {T} = Ref(v ? one(T) : zero(T))
scalar(::Type{T}, v) where {T} = Ref(convert(T, v))

prec() = (b = get_einsum_backend(); b isa B200Backend ? b.prec : Int32(0))
stream() = CUDA.stream().handle

# ----------------------------------------------------------------------------
# contexts (one per device; the workspace holds intermediates and scratch)
# ----------------------------------------------------------------------------

const CONTEXTS = Dict{Int,Ptr{Cvoid}}()
const CONTEXT_BYTES = Dict{Int,Int}()

function ctx(min_bytes::Integer = 0)
    dev = CUDA.deviceid(CUDA.device())
    c = get(CONTEXTS, dev, C_NULL)
    need = max(Int(min_bytes), 256 << 20)
    if c == C_NULL || CONTEXT_BYTES[dev] < min_bytes
        if c != C_NULL
            CUDA.synchronize()
            @ccall $(sym(:ome_ctx_destroy))(c::Ptr{Cvoid})::Cint
            need = max(need, 2 * CONTEXT_BYTES[dev])
        end
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(@ccall $(sym(:ome_ctx_create))(dev::Cint, need::Csize_t, r::Ref{Ptr{Cvoid}})::Cint)
        CONTEXTS[dev] = r[]
        CONTEXT_BYTES[dev] = need
        c = r[]
    end
    return c
end

# ----------------------------------------------------------------------------
# labelled tensors
# ----------------------------------------------------------------------------

# labels of any type -> consecutive Int32 ids, per call (only equality matters)
struct LabelMap
    ids::Dict{Any,Int32}
end
LabelMap() = LabelMap(Dict{Any,Int32}())
(m::LabelMap)(l) = get!(m.ids, l, Int32(length(m.ids)))

function ome_tensor(x::CuArray, ix, lm::LabelMap, keep::Vector{Any})
    length(ix) == ndims(x) || throw(ArgumentError("indices $ix invalid for tensor with ndims = $(ndims(x))"))
    d = collect(Int64, size(x))
    s = collect(Int64, strides(x))
    l = Int32[lm(i) for i in ix]
    push!(keep, d, s, l)
    return OmeTensor(reinterpret(Ptr{Cvoid}, pointer(x)), Int32(ndims(x)), pointer(d), pointer(s), pointer(l))
end

# inputs in the output's element type (mixed eltypes are converted first, as
# ext/CUDAExt.jl:116 and align_eltypes do)
aligned(::Type{T}, x::CuArray{T}) where {T} = x
aligned(::Type{T}, x::CuArray) where {T} = T.(x)
aligned(::Type{T}, x::AbstractArray) where {T} = CuArray{T}(x)

# ----------------------------------------------------------------------------
# einsum! / loop_einsum! / einsum_grad (single contractions)
# ----------------------------------------------------------------------------

function _call_einsum!(fn::Symbol, ixs, iy, xs, y::CuArray{T}, sx, sy) where {T}
    N = length(xs)
    cxs = map(x -> aligned(T, x), xs)
    lm = LabelMap()
    keep = Any[]
    GC.@preserve cxs y keep begin
        ts = OmeTensor[ome_tensor(x, ix, lm, keep) for (x, ix) in zip(cxs, ixs)]
        yt = Ref(ome_tensor(y, iy, lm, keep))
        a, b = scalar(T, sx), scalar(T, sy)
        if fn === :ome_einsum
            check(@ccall $(sym(:ome_einsum))(ctx()::Ptr{Cvoid}, stream()::Ptr{Cvoid}, ome_dtype(T)::Cint, Int32(N)::Int32,
                                             ts::Ptr{OmeTensor}, yt::Ref{OmeTensor}, a::Ref{T}, b::Ref{T},
                                             prec()::Int32)::Cint)
        else
            check(@ccall $(sym(:ome_loop_einsum))(ctx()::Ptr{Cvoid}, stream()::Ptr{Cvoid}, ome_dtype(T)::Cint,
                                                  Int32(N)::Int32, ts::Ptr{OmeTensor}, yt::Ref{OmeTensor}, a::Ref{T},
                                                  b::Ref{T})::Cint)
        end
    end
    return y
end

"""einsum!(ixs, iy, xs, y, sx, sy, size_dict) for any number of CuArray inputs
(replaces ext/CUDAExt.jl:181-192 and the unary / n-ary generic paths)."""
b200_einsum!(ixs, iy, xs, y::CuArray, sx, sy, size_dict) = _call_einsum!(:ome_einsum, ixs, iy, xs, y, sx, sy)

"""loop_einsum! (src/loop_einsum.jl:21-45, ext/CUDAExt.jl:60-91)."""
b200_loop_einsum!(ixs, iy, xs, y::CuArray, sx, sy, size_dict) = _call_einsum!(:ome_loop_einsum, ixs, iy, xs, y, sx, sy)

"""einsum_grad(ixs, xs, iy, size_dict, dy, i) (src/autodiff.jl:24-30): one
ome_einsum_grad call; the conjugations run in the library."""
function b200_einsum_grad(ixs, xs, iy, size_dict, dy, i::Integer)
    T = promote_type(map(eltype, xs)..., eltype(dy))
    cxs = map(x -> aligned(T, x), xs)
    cdy = aligned(T, dy)
    dx = CuArray{T}(undef, map(l -> size_dict[l], ixs[i])...)
    lm = LabelMap()
    keep = Any[]
    GC.@preserve cxs cdy dx keep begin
        ts = OmeTensor[ome_tensor(x, ix, lm, keep) for (x, ix) in zip(cxs, ixs)]
        dyt = Ref(ome_tensor(cdy, iy, lm, keep))
        dxt = Ref(ome_tensor(dx, ixs[i], lm, keep))
        check(@ccall $(sym(:ome_einsum_grad))(ctx()::Ptr{Cvoid}, stream()::Ptr{Cvoid}, ome_dtype(T)::Cint,
                                              Int32(length(xs))::Int32, ts::Ptr{OmeTensor}, dyt::Ref{OmeTensor},
                                              Int32(i - 1)::Int32, dxt::Ref{OmeTensor}, prec()::Int32)::Cint)
    end
    # ProjectTo(xs[i]): a real input of a complex contraction takes the real part
    return eltype(xs[i]) <: Real && T <: Complex ? real.(dx) : dx
end

# ----------------------------------------------------------------------------
# contraction trees: NestedEinsum / SlicedEinsum / cost_and_gradient
# ----------------------------------------------------------------------------

"""
    flatten_tree(code) -> NamedTuple

The arrays ome_plan_create takes (include/ome_b200.h), built from a
NestedEinsum (or the tree inside a SlicedEinsum) in post-order, root last:
per node its child references (r >= 0: node r; r < 0: input -r-1, i.e. the
1-based tensorindex t becomes -t) and output labels; per input its labels
(getixsv order); label ids with their extents; the sliced labels.
"""
function flatten_tree(code, size_dict)
    ne = code isa SlicedEinsum ? code.eins : code
    slicing = code isa SlicedEinsum ? collect(code.slicing) : Any[]
    lm = LabelMap()
    ixsv = getixsv(ne)
    input_nlabels = Int32[length(ix) for ix in ixsv]
    input_labels = Int32[lm(l) for ix in ixsv for l in ix]
    node_nargs = Int32[]
    node_args = Int32[]
    node_niy = Int32[]
    node_iy = Int32[]
    function rec(n)
        refs = Int32[isleaf(a) ? Int32(-tensorindex(a)) : rec(a) for a in siblings(n)]
        iy = getiy(rootcode(n))
        push!(node_nargs, Int32(length(refs)))
        append!(node_args, refs)
        push!(node_niy, Int32(length(iy)))
        append!(node_iy, Int32[lm(l) for l in iy])
        return Int32(length(node_nargs) - 1)
    end
    isleaf(ne) && throw(ArgumentError("a bare leaf is not a contraction"))
    rec(ne)
    sliced = Int32[lm(l) for l in slicing]
    labels = collect(keys(lm.ids))
    label_ids = Int32[lm.ids[l] for l in labels]
    label_extents = Int64[size_dict[l] for l in labels]
    return (; input_nlabels, input_labels, node_nargs, node_args, node_niy, node_iy, label_ids, label_extents,
            sliced, nin = Int32(length(ixsv)), out_labels = getiyv(ne))
end

# plans by (tree, extents, element type, precision); freed with the process
const PLANS = Dict{Any,Ptr{Cvoid}}()

function plan(code, size_dict, ::Type{T}) where {T}
    key = (code, sort!([(string(k), v) for (k, v) in size_dict]), T, prec())
    p = get(PLANS, key, C_NULL)
    p == C_NULL || return p
    f = flatten_tree(code, size_dict)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve f begin
        check(@ccall $(sym(:ome_plan_create))(ctx()::Ptr{Cvoid}, ome_dtype(T)::Cint, f.nin::Int32,
                                              f.input_nlabels::Ptr{Int32}, f.input_labels::Ptr{Int32},
                                              Int32(length(f.node_nargs))::Int32, f.node_nargs::Ptr{Int32},
                                              f.node_args::Ptr{Int32}, f.node_niy::Ptr{Int32}, f.node_iy::Ptr{Int32},
                                              Int32(length(f.label_ids))::Int32, f.label_ids::Ptr{Int32},
                                              f.label_extents::Ptr{Int64}, Int32(length(f.sliced))::Int32,
                                              f.sliced::Ptr{Int32}, prec()::Int32, r::Ref{Ptr{Cvoid}})::Cint)
    end
    PLANS[key] = r[]
    return r[]
end

function peak_bytes(p)
    fwd, grad = Ref{Csize_t}(0), Ref{Csize_t}(0)
    check(@ccall $(sym(:ome_plan_peak_bytes))(p::Ptr{Cvoid}, fwd::Ref{Csize_t}, grad::Ref{Csize_t})::Cint)
    return Int(fwd[]), Int(grad[])
end

dense(::Type{T}, x) where {T} = (c = aligned(T, x); c isa CuArray && strides(c) == strides(similar(c)) ? c : copy(c))

"""einsum!(::NestedEinsum / ::SlicedEinsum, xs, y, sx, sy, size_dict): the whole
tree in one ome_plan_execute (intermediates in the context workspace, which
replaces active_free of ext/CUDAExt.jl:121-147; slices summed in FP64 for
Float32/Float64 trees).  y === nothing allocates the output."""
function b200_tree!(code, xs, y, sx, sy, size_dict)
    T = y === nothing ? promote_type(map(eltype, xs)...) : eltype(y)
    ne = code isa SlicedEinsum ? code.eins : code
    yy = y === nothing ? CuArray{T}(undef, map(l -> size_dict[l], getiyv(ne))...) : y
    p = plan(code, size_dict, T)
    fwd, _ = peak_bytes(p)
    c = ctx(fwd)
    ins = map(x -> dense(T, x), xs)
    ptrs = Ptr{Cvoid}[reinterpret(Ptr{Cvoid}, pointer(x)) for x in ins]
    a, b = scalar(T, sx), scalar(T, sy)
    GC.@preserve ins ptrs yy begin
        check(@ccall $(sym(:ome_plan_execute))(c::Ptr{Cvoid}, p::Ptr{Cvoid}, stream()::Ptr{Cvoid}, ptrs::Ptr{Ptr{Cvoid}},
                                               reinterpret(Ptr{Cvoid}, pointer(yy))::Ptr{Cvoid}, a::Ref{T},
                                               b::Ref{T})::Cint)
    end
    return yy
end

"""cost_and_gradient(code, xs, dy) (src/bp.jl:122-130): forward with every
intermediate kept in the workspace, then einsum_grad per node; unsliced, as
in the reference (src/bp.jl:26-28)."""
function b200_cost_and_gradient(code, xs, dy = nothing)
    ne = code isa SlicedEinsum ? code.eins : code
    size_dict = OMEinsum.get_size_dict!(getixsv(ne), xs, Dict{OMEinsum.labeltype(ne),Int}())
    T = promote_type(map(eltype, xs)...)
    p = plan(ne, size_dict, T)
    _, gb = peak_bytes(p)
    c = ctx(gb)
    ins = map(x -> dense(T, x), xs)
    y = CuArray{T}(undef, map(l -> size_dict[l], getiyv(ne))...)
    dxs = map(x -> CuArray{T}(undef, size(x)...), ins)
    if dy === nothing
        ndims(y) == 0 || throw(ArgumentError("the output must be a scalar, or pass the output gradient"))
    end
    cdy = dy === nothing ? nothing : dense(T, dy)
    ptrs = Ptr{Cvoid}[reinterpret(Ptr{Cvoid}, pointer(x)) for x in ins]
    gptrs = Ptr{Cvoid}[reinterpret(Ptr{Cvoid}, pointer(g)) for g in dxs]
    dyp = cdy === nothing ? C_NULL : reinterpret(Ptr{Cvoid}, pointer(cdy))
    GC.@preserve ins ptrs gptrs dxs y cdy begin
        check(@ccall $(sym(:ome_plan_gradient))(c::Ptr{Cvoid}, p::Ptr{Cvoid}, stream()::Ptr{Cvoid}, ptrs::Ptr{Ptr{Cvoid}},
                                                dyp::Ptr{Cvoid}, reinterpret(Ptr{Cvoid}, pointer(y))::Ptr{Cvoid},
                                                gptrs::Ptr{Ptr{Cvoid}})::Cint)
    end
    return y, dxs
end

# ---------------------------------------------------------------------------
# Serving through the library's own loop (ome_server_*): a Julia service
# submits whole trees and polls; slots, admission and issue threads are C++.

struct OmeServerJob        # ome_server_job
    id::Int64
    outcome::Int32         # 0 completed, 1 failed, 2 rejected (memory), 3 rejected (work cap)
    status::Int32
    arrival_s::Float64
    admitted_s::Float64
    done_s::Float64
end

mutable struct B200Server
    handle::Ptr{Cvoid}
    live::Dict{Int64,Any}  # job id -> the arrays the library reads or writes until poll reports it
end

"""B200Server(; slots, budget_bytes, max_work): a serving loop on the current
device; jobs above a slot's share run alone, jobs above the budget or the work
cap are rejected at admission."""
function B200Server(; slots::Integer = 8, budget_bytes::Integer = 150 * 10^9, max_work::Real = 0)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(@ccall $(sym(:ome_server_create))(CUDA.deviceid(CUDA.device())::Cint, Int32(slots)::Int32,
                                            Csize_t(budget_bytes)::Csize_t, Float64(max_work)::Float64,
                                            r::Ref{Ptr{Cvoid}})::Cint)
    srv = B200Server(r[], Dict{Int64,Any}())
    finalizer(close, srv)
    return srv
end

"""submit!(srv, code, xs; grad = false) -> (id, y, dxs): queue the tree's value
(or cost_and_gradient, unsliced as src/bp.jl:26-28) on the server; y and dxs
are filled when poll! reports the job."""
function submit!(srv::B200Server, code, xs; grad::Bool = false, work::Real = 0)
    ne0 = code isa SlicedEinsum ? code.eins : code
    size_dict = OMEinsum.get_size_dict!(getixsv(ne0), xs, Dict{OMEinsum.labeltype(ne0),Int}())
    T = promote_type(map(eltype, xs)...)
    tree = grad ? ne0 : code
    p = plan(tree, size_dict, T)
    ins = map(x -> dense(T, x), xs)
    y = CuArray{T}(undef, map(l -> size_dict[l], getiyv(ne0))...)
    dxs = grad ? map(x -> CuArray{T}(undef, size(x)...), ins) : nothing
    ptrs = Ptr{Cvoid}[reinterpret(Ptr{Cvoid}, pointer(x)) for x in ins]
    gptrs = grad ? Ptr{Cvoid}[reinterpret(Ptr{Cvoid}, pointer(g)) for g in dxs] : Ptr{Cvoid}[]
    id = Ref{Int64}(0)
    GC.@preserve ptrs gptrs begin
        check(@ccall $(sym(:ome_server_submit))(srv.handle::Ptr{Cvoid}, p::Ptr{Cvoid}, Int32(length(ins))::Int32,
                                                ptrs::Ptr{Ptr{Cvoid}}, reinterpret(Ptr{Cvoid}, pointer(y))::Ptr{Cvoid},
                                                (grad ? pointer(gptrs) : C_NULL)::Ptr{Ptr{Cvoid}}, Float64(work)::Float64,
                                                stream()::Ptr{Cvoid}, id::Ref{Int64})::Cint)
    end
    srv.live[id[]] = (ins, y, dxs)
    return id[], y, dxs
end

"""poll!(srv) -> (records, running): retire finished jobs, admit queued ones."""
function poll!(srv::B200Server)
    recs = Vector{OmeServerJob}(undef, 64)
    n, running = Ref{Int32}(0), Ref{Int32}(0)
    out = OmeServerJob[]
    while true
        check(@ccall $(sym(:ome_server_poll))(srv.handle::Ptr{Cvoid}, Int32(64)::Int32, recs::Ptr{OmeServerJob},
                                              n::Ref{Int32}, running::Ref{Int32})::Cint)
        for r in view(recs, 1:n[])
            delete!(srv.live, r.id)
            push!(out, r)
        end
        n[] < 64 && return out, Int(running[])
    end
end

function Base.close(srv::B200Server)
    if srv.handle != C_NULL
        @ccall $(sym(:ome_server_destroy))(srv.handle::Ptr{Cvoid})::Cint
        srv.handle = C_NULL
        empty!(srv.live)
    end
    return nothing
end

"""Synchronise the stream and raise if a bounded device-side wait gave up."""
device_status() = check(@ccall $(sym(:ome_device_status))(stream()::Ptr{Cvoid})::Cint)

function __init__()
    HANDLE[] = Libdl.dlopen(get(ENV, "OME_B200_LIB", "libomeb200"))
    empty!(SYMBOLS)
    OMEinsum._B200_EINSUM_IMPL[] = b200_einsum!
    OMEinsum._B200_LOOP_IMPL[] = b200_loop_einsum!
    OMEinsum._B200_TREE_IMPL[] = b200_tree!
    OMEinsum._B200_GRAD_IMPL[] = b200_einsum_grad
    OMEinsum._B200_COSTGRAD_IMPL[] = b200_cost_and_gradient
    OMEinsum._B200_AVAILABLE[] = true
end

end  # module
