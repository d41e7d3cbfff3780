"""B200-native (sm_100a) evaluation hot path of FastMultipole.jl.

``fmm`` / ``direct`` mirror the reference's ``fmm!`` / ``direct!``; the work runs
in libfmmb200.so (CUDA) behind the C ABI of include/fmm_b200.h.
"""
from .api import (Barba, DerivativesSwitch, PointSources, PowerAbsoluteGradient, PowerAbsolutePotential,
                  PowerRelativeGradient, PowerRelativePotential,
                  ProbeSystem, RotatedCoefficientsAbsoluteGradient, RotatedCoefficientsRelativeGradient,
                  SelfTuning, SelfTuningTreeStop, System, VortexParticles, default_context, direct, fmm,
                  Server, get_lists, get_tree, make_options, request_footprint, solve_buffers,
                  solve_multi_buffers, vjp, vjp_buffers)
from ._lib import Context, FMMError, lib

__all__ = ["fmm", "direct", "System", "PointSources", "VortexParticles", "ProbeSystem", "DerivativesSwitch",
           "SelfTuningTreeStop", "Barba", "SelfTuning", "PowerAbsoluteGradient", "PowerRelativeGradient",
           "RotatedCoefficientsAbsoluteGradient", "RotatedCoefficientsRelativeGradient", "PowerAbsolutePotential",
           "PowerRelativePotential", "Context", "FMMError",
           "lib", "default_context", "get_tree", "get_lists", "make_options", "solve_buffers", "vjp",
           "vjp_buffers", "Server", "solve_multi_buffers", "request_footprint"]
