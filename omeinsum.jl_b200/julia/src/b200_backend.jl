# B200 backend registration for OMEinsum.jl.
#
# `include`d from src/OMEinsum.jl right after src/backends.jl.  It follows the
# registry pattern of src/backends.jl:170-184: the backend type lives in the
# package, while the implementation is a function reference that the B200
# extension (ext/B200Ext.jl) stores at load time, so that no method is
# overwritten during precompilation (src/backends.jl:172).
#
# Exports to add in src/OMEinsum.jl: B200Backend.

"""
    B200Backend(; prec = 0)

Einsum on NVIDIA B200 GPUs through `libomeb200` (hand-written sm_100a
kernels).  `prec` selects how Float32 contractions use the tensor cores:
0 = automatic (BF16x6 split products, FP32-faithful), 1 = plain FP32 on CUDA
cores, 2 = BF16x3, 3 = BF16x6.  Other element types (Float64, complex,
Int64, Bool, Tropical) are exact on CUDA cores.  With this backend selected,
an unsupported case is an error, never a CPU fallback.
"""
struct B200Backend <: EinsumBackend
    prec::Int32
end
B200Backend(; prec::Integer = 0) = B200Backend(Int32(prec))

const _B200_AVAILABLE = Ref{Bool}(false)
# function references set by B200Ext.__init__
const _B200_EINSUM_IMPL = Ref{Any}(nothing)       # einsum!(ixs, iy, xs, y, sx, sy, size_dict), any input count
const _B200_LOOP_IMPL = Ref{Any}(nothing)         # loop_einsum!(ixs, iy, xs, y, sx, sy, size_dict)
const _B200_TREE_IMPL = Ref{Any}(nothing)         # einsum!(::NestedEinsum / ::SlicedEinsum, xs, y, sx, sy, size_dict)
const _B200_GRAD_IMPL = Ref{Any}(nothing)         # einsum_grad(ixs, xs, iy, size_dict, dy, i)
const _B200_COSTGRAD_IMPL = Ref{Any}(nothing)     # cost_and_gradient(code, xs, dy)

function check_backend_availability(::B200Backend)
    _B200_AVAILABLE[] && return (true, "")
    return (false, "the B200 extension is not loaded - run `using CUDA` with libomeb200 available first")
end

function set_einsum_backend!(backend::B200Backend)
    available, msg = check_backend_availability(backend)
    # unlike CuTensorBackend there is no silent fallback: the calls raise
    available || @warn "B200Backend: $msg. Contractions on CuArrays will raise until it is loaded."
    EINSUM_BACKEND[] = backend
end

_b200_selected() = get_einsum_backend() isa B200Backend

function _b200_impl(r::Ref{Any}, what::AbstractString)
    impl = r[]
    impl === nothing && error("B200Backend selected but the B200 extension is not loaded ($what)")
    return impl
end
