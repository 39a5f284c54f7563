# Dispatch points for the B200 backend, `include`d at the end of
# ext/CUDAExt.jl (inside `module CUDAExt`, after its own methods).
#
# Every method first checks `get_einsum_backend() isa B200Backend`; with
# another backend selected it runs exactly what ext/CUDAExt.jl runs today.
# With B200Backend selected, the call goes to the implementation that
# B200Ext stored in OMEinsum's Refs (src/b200_backend.jl); a missing
# extension or an unsupported case raises, nothing falls back to the CPU.

using OMEinsum: _b200_selected, _b200_impl, _B200_EINSUM_IMPL, _B200_LOOP_IMPL, _B200_TREE_IMPL,
                _B200_GRAD_IMPL, _B200_COSTGRAD_IMPL, SlicedEinsum

# --- binary einsum! (ext/CUDAExt.jl:181-192): one more branch, placed first
# in the body of the existing `OMEinsum.einsum!(ixs, iy, xs::NTuple{2,CuArray{T}}, ...)`:
#
#     _b200_selected() && return _b200_impl(_B200_EINSUM_IMPL, "einsum!")(ixs, iy, xs, y, sx, sy, size_dict)
#
# The methods below are new; they cover the cases ext/CUDAExt.jl leaves to
# the generic CPU-shaped code paths.

# --- unary einsum! on a CuArray (src/einsum.jl:84-101)
function OMEinsum.einsum!(ixs, iy, xs::NTuple{1,CuArray{T}}, y::CuArray{T}, sx, sy,
                          size_dict::Dict{LT}) where {T,LT}
    _b200_selected() && return _b200_impl(_B200_EINSUM_IMPL, "einsum!")(ixs, iy, xs, y, sx, sy, size_dict)
    return invoke(OMEinsum.einsum!, Tuple{Any,Any,NTuple{1,Any},Any,Any,Any,Dict{LT}}, ixs, iy, xs, y, sx, sy,
                  size_dict)
end

# --- n-ary einsum! (src/einsum.jl:47-50 -> loop_einsum!)
function OMEinsum.einsum!(ixs, iy, xs::NTuple{N,CuArray{T}}, y::CuArray{T}, sx, sy,
                          size_dict::Dict) where {N,T}
    if _b200_selected()
        return _b200_impl(_B200_EINSUM_IMPL, "einsum!")(ixs, iy, xs, y, sx, sy, size_dict)
    end
    return loop_einsum!(ixs, iy, xs, y, sx, sy, size_dict)
end

# --- loop_einsum! (src/loop_einsum.jl:21-45; the CUDA method at ext/CUDAExt.jl:60-91
# gains this branch first in its body):
#
#     _b200_selected() && return _b200_impl(_B200_LOOP_IMPL, "loop_einsum!")(ixs0, iy0, xs, y, sx, sy, size_dict)

# --- NestedEinsum (ext/CUDAExt.jl:121-147): both methods gain, first in their body,
#
#     einsum!:  _b200_selected() && return _b200_impl(_B200_TREE_IMPL, "NestedEinsum")(neinsum, xs, y, sx, sy, size_dict)
#     einsum:   _b200_selected() && return _b200_impl(_B200_TREE_IMPL, "NestedEinsum")(neinsum, xs, nothing, true, false, size_dict)

# --- SlicedEinsum on CuArrays (src/slicing.jl:112-137): the whole slice loop in one plan
function OMEinsum.einsum!(se::SlicedEinsum, xs::NTuple{N,CuArray}, y::CuArray, sx, sy, size_dict::Dict) where {N}
    _b200_selected() && return _b200_impl(_B200_TREE_IMPL, "SlicedEinsum")(se, xs, y, sx, sy, size_dict)
    return invoke(OMEinsum.einsum!, Tuple{SlicedEinsum,NTuple{N,AbstractArray} where N,Any,Any,Any,Dict}, se, xs, y,
                  sx, sy, size_dict)
end
function OMEinsum.einsum(se::SlicedEinsum, xs::NTuple{N,CuArray}, size_dict::Dict) where {N}
    _b200_selected() && return _b200_impl(_B200_TREE_IMPL, "SlicedEinsum")(se, xs, nothing, true, false, size_dict)
    return invoke(OMEinsum.einsum, Tuple{SlicedEinsum,NTuple{N,AbstractArray} where N,Dict}, se, xs, size_dict)
end

# --- einsum_grad (src/autodiff.jl:24-30), the pullback of rrule(einsum)
# (src/autodiff.jl:35-44), for CuArray inputs
function OMEinsum.einsum_grad(ixs, xs::NTuple{N,CuArray}, iy, size_dict, dy::CuArray, i) where {N}
    _b200_selected() && return _b200_impl(_B200_GRAD_IMPL, "einsum_grad")(ixs, xs, iy, size_dict, dy, i)
    return invoke(OMEinsum.einsum_grad, Tuple{Any,Any,Any,Any,Any,Any}, ixs, xs, iy, size_dict, dy, i)
end

# --- cost_and_gradient (src/bp.jl:122-130) for CuArray inputs
function OMEinsum.cost_and_gradient(code, xs::NTuple{N,CuArray}, ȳ = nothing) where {N}
    _b200_selected() && return _b200_impl(_B200_COSTGRAD_IMPL, "cost_and_gradient")(code, xs, ȳ)
    return invoke(OMEinsum.cost_and_gradient, Tuple{Any,Tuple,Any}, code, xs, ȳ)
end
