"""B200-native CPML acoustic time stepping behind AcousticWaveCPML.jl's API.

Python mirror of the reference's public surface for the GPU solvers:
``Acoustic2D_CUDA.solve2D``, ``Acoustic3D_CUDA.solve3D``, ``Sources``,
``Receivers``, ``rickersource1D`` and ``calc_Kab_CPML``, plus ``solve2D_batch`` for many shots over several
models in one launch sequence. The compute runs in
libawcpml.so (hand-written sm_100a kernels behind the C ABI of
include/awcpml.h); ``julia/AcousticWaveCPML_B200.jl`` is the equivalent Julia
shim that `ccall`s the same library.

The directory name is not a Python identifier; load it with
``__graft_entry__.load_package()`` (registers it as ``acousticwavecpml_b200``).
"""
from . import Acoustic1D, Acoustic2D_CUDA, Acoustic3D_CUDA, adjoint  # noqa: F401
from ._lib import AWC_F32, AWC_F64, AwcError, AwcInvalidArgument, Problem  # noqa: F401
from . import batch, models  # noqa: F401
from .batch import (Batch, forward_batch, prepare_batch, solve2D_batch,  # noqa: F401
                    solve2D_batch_sharded, solve_sharded)
from .core import Context, Plan, default_context, prepare  # noqa: F401
from .utils import Receivers, Sources, calc_Kab_CPML, rickersource1D  # noqa: F401

__all__ = ["Acoustic1D", "Acoustic2D_CUDA", "Acoustic3D_CUDA", "Sources", "Receivers", "rickersource1D",
           "calc_Kab_CPML", "Context", "Plan", "prepare", "default_context", "Problem",
           "AwcError", "AwcInvalidArgument", "AWC_F32", "AWC_F64", "Batch",
           "forward_batch", "prepare_batch", "adjoint", "solve2D_batch", "solve2D_batch_sharded",
           "solve_sharded", "batch", "models"]
