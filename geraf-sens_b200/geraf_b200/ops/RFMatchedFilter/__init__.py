"""RFMatchedFilter: FMCW matched-filter backprojection (sm_100a).

Lazy exports, as in the reference (``geraf/ops/RFMatchedFilter/__init__.py:6-18``).
"""
from importlib import import_module

_EXPORTS = {
    "matched_filter_cuda": ".matched_filter_cuda",
    "faster_matched_filter_cuda": ".faster_matched_filter_cuda",
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
