"""B200-native cross-correlation PIV (drop-in for multi_quickPIV's PIV hot path).

The public names mirror the Julia package: ``PIV``, ``setPIVParameters``,
``PIVParameters``, ``get_vectorfield_size`` and the ``_isize``/``_smarg``/
``_ssize``/``_step``/``_ovp`` accessors.  All compute runs in hand-written
sm_100a CUDA kernels behind the C ABI declared in ``include/mqp.h``.
"""
from .piv import (PIV, PIVParameters, _isize, _ovp, _smarg, _ssize, _step,  # noqa: F401
                  correlation_planes, get_vectorfield_size, maxval, parseCorr,
                  setPIVParameters, toDims3)
from ._lib import Context, MQPError  # noqa: F401
from . import postprocessing  # noqa: F401

__all__ = ["PIV", "PIVParameters", "setPIVParameters", "get_vectorfield_size", "correlation_planes",
           "Context", "MQPError", "maxval"]
