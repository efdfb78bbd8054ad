"""RFSignalTracer: lensless specular RF renderer and along-ray resampler (sm_100a).

Exports as in the reference (``geraf/ops/RFSignalTracer/__init__.py:6-18``).
"""
_EXPORTS = {
    "signal_tracer_cuda": ".signal_tracer_cuda",
    "bilinear_raysample_cuda": ".bilinear_raysample_cuda",
}

__all__ = list(_EXPORTS)


# The exported functions share their submodules' names.  Importing them here,
# once, binds the package attribute to the function after the import system has
# bound it to the submodule; later imports of the submodule leave it alone.  The
# compiled library is still loaded lazily, at the first operator call.
from .signal_tracer_cuda import signal_tracer_cuda  # noqa: E402
from .bilinear_raysample_cuda import bilinear_raysample_cuda  # noqa: E402

