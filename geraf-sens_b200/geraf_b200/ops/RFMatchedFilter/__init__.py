"""RFMatchedFilter: FMCW matched-filter backprojection (sm_100a).

Exports as in the reference (``geraf/ops/RFMatchedFilter/__init__.py:6-18``).
"""
_EXPORTS = {
    "matched_filter_cuda": ".matched_filter_cuda",
    "faster_matched_filter_cuda": ".faster_matched_filter_cuda",
}

__all__ = list(_EXPORTS)


# The exported functions share their submodules' names.  Importing them here,
# once, binds the package attribute to the function after the import system has
# bound it to the submodule; later imports of the submodule leave it alone.  The
# compiled library is still loaded lazily, at the first operator call.
from .matched_filter_cuda import matched_filter_cuda  # noqa: E402
from .faster_matched_filter_cuda import faster_matched_filter_cuda  # noqa: E402

