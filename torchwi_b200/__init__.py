"""torchwi_b200 -- B200-native (sm_100a) time-domain 2D acoustic propagator
with the interface of TorchWI's time operator.

Public API (mirrors torchwi.operator / torchwi.propagator):
    Time2d, Time2dForward        reference-compatible modules
    Time2dBatch                  all shots of a survey in one plan
    Time2dModels                 several models of different sizes in one batch
    ShotPlan, PlanOptions        the underlying C-ABI plan
    autotune                     fastest launch shape for a grid and shot count
    inversion.Inversion          FWI driver over the batched plan
    io, workflows                RSF / gather files and the example programs
    propagator.td2d_b200         drop-in for the native td2d_cuda module
    source.ricker, source.fdgaus input wavelets

The CUDA library (torchwi_b200/_lib/libtwi_b200.so) is loaded on first use;
build it with ``python -m torchwi_b200.build``.
"""

from .operator import Time2d, Time2dBatch, Time2dForward, Time2dModels  # noqa: F401
from .plan import PlanBatch, PlanOptions, ShotPlan, autotune, footprint_bytes  # noqa: F401
from .source import fdgaus, ricker  # noqa: F401
from ._capi import TwiError, TwiInvalid  # noqa: F401

__version__ = "0.1.0"
