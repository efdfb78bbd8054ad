"""RFSignalTracer: lensless specular RF renderer and along-ray resampler (sm_100a).

Lazy exports, as in the reference (``geraf/ops/RFSignalTracer/__init__.py:6-18``).
"""
from importlib import import_module

_EXPORTS = {
    "signal_tracer_cuda": ".signal_tracer_cuda",
    "bilinear_raysample_cuda": ".bilinear_raysample_cuda",
}

__all__ = list(_EXPORTS)


def __getattr__(name):
    if name not in _EXPORTS:
        raise AttributeError(name)
    fn = getattr(import_module(_EXPORTS[name], __name__), name)
    # Importing the submodule binds its module object under the same name;
    # rebind the function so later `from ... import name` keeps returning it.
    globals()[name] = fn
    return fn
