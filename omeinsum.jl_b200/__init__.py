"""omeinsum_b200: a B200 (sm_100a) einsum backend with OMEinsum.jl's interface.

The package directory is ``omeinsum.jl_b200``; it is imported under the module
name ``omeinsum_b200`` (see ``load_package`` in the repository's
``__graft_entry__.py`` / ``tests/conftest.py``).

Public API (names follow OMEinsum.jl; ``!`` becomes a trailing ``_``):

* codes: ``ein``, ``EinCode``, ``NestedEinsum``, ``SlicedEinsum``,
  ``get_size_dict``, ``getixsv``, ``getiyv``, ``flatten``, ``uniformsize``;
* execution: ``einsum``, ``einsum_``, ``loop_einsum``, ``loop_einsum_``,
  ``einsum_grad``, ``cost_and_gradient``, ``get_output_array``;
* backends: ``set_einsum_backend``, ``get_einsum_backend``, ``B200Backend``,
  ``DefaultBackend``, ``CuTensorBackend``, ``EinsumBackend``;
* planning: ``optimize_code``, ``slice_code``, ``GreedyMethod``,
  ``GreedySlicer``, ``contraction_complexity``, ``flop``, ``peak_memory``,
  ``label_elimination_order``, ``writejson``, ``readjson``;
* batching: ``BatchedEinsum`` (one grouped launch for many contractions of
  uneven shapes), ``capture_graph``, ``einsum_many`` (independent
  contractions of host tensors with uploads and downloads overlapped);
* serving: ``TNServer`` / ``Job`` (continuous batching of whole networks by
  peak workspace bytes, p50/p99 latency);
* element types: torch float32/float64/complex64/complex128/int64/bool and
  ``TropicalTensor`` (max-plus).

Every contraction runs in libomeb200.so; there is no CPU fallback.
"""
from ._lib import ArgumentError, DimensionMismatch, OMEError, device_status, load as load_library, release_workspaces
from .backends import (B200Backend, CuTensorBackend, DefaultBackend, EinsumBackend, get_einsum_backend,
                       set_einsum_backend)
from .core import (AbstractEinsum, DynamicEinCode, DynamicNestedEinsum, EinCode, NestedEinsum, SlicedEinsum,
                   StaticEinCode, StaticNestedEinsum, drop_slicedim, ein, flatten, get_size_dict, getixsv, getiyv,
                   parse_nested, slice_iterator, uniformsize)
from .engine import (TropicalTensor, cost_and_gradient, einsum, einsum_, einsum_grad, einsum_many,
                     get_output_array, loop_einsum, loop_einsum_, promote_dtype)
from .batch import BatchGraph, BatchedEinsum, capture_graph
from .serve import Job, NativeTNServer, TNServer, pow2_rescale
from .distributed import ShardedSlices, allreduce_partial, sharded_einsum, slice_range
from .autograd import ad_einsum
from .planner import (GreedyMethod, GreedySlicer, MergeVectors, ScoreFunction, TreeSA, TreeSASlicer,
                      contraction_complexity, flop, label_elimination_order, optimize_code, peak_memory, readjson,
                      slice_code, writejson)

__all__ = [n for n in dir() if not n.startswith("_")]
