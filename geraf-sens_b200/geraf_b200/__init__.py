"""geraf_b200 -- B200-native (sm_100a) implementation of GeRaF's RF operators.

``geraf_b200.ops.RFMatchedFilter`` and ``geraf_b200.ops.RFSignalTracer`` are
drop-in replacements of ``geraf.ops.RFMatchedFilter`` / ``geraf.ops.RFSignalTracer``
(same call signatures, tensor layouts, autograd behaviour and errors), backed
by the C-ABI library ``libgeraf_rf.so`` (``include/geraf_rf.h``).
``geraf_b200.model_utils`` mirrors the reference's ``geraf.models.model_utils``
op adapters.
"""
from .runtime import default_precision, precision  # noqa: F401

__version__ = "0.1.0"


def library_path() -> str:
    from . import _lib

    return _lib.LIB_PATH


def load_library():
    """Loads ``libgeraf_rf.so`` (raises ImportError if it has not been built)."""
    from . import _lib

    return _lib.load()
