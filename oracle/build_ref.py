"""Build the reference GeRaF CUDA extensions, unmodified, for sm_100a into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY.  The two ``_C`` modules of the reference
(``geraf/ops/RFMatchedFilter/csrc`` and ``geraf/ops/RFSignalTracer/csrc``) are
compiled straight from their sources in the reference checkout with the
reference's own preprocessor flags (``setup.py:36-53``: ``WITH_CUDA``, ``-O3``,
the ``-U__CUDA_NO_HALF*`` trio) but with ``-gencode arch=compute_100a,code=sm_100a``
instead of the sm_70..sm_90 list, which has no Blackwell target.  Nothing is
copied into this repository: the sources are read in place and only build
products land in ``oracle/_ref/`` (git-ignored, shipped to the GPU machine with
the rest of the tree).

The built modules are the GPU parity pin: ``tests/golden/make_golden.py`` runs
them on seeded inputs to produce the committed golden vectors, and the ``-m gpu``
tests compare this repository's kernels against them.  Nothing in the product
path loads them.

Usage:  python oracle/build_ref.py [--reference PATH] [--verbose] [--clean]
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
OPS = ("RFMatchedFilter", "RFSignalTracer")
DEFAULT_REFERENCE = "/root/reference"

_CFLAGS = ["-O3", "-DWITH_CUDA"]
_CUDA_CFLAGS = [
    "-O3",
    "-DWITH_CUDA",
    "-gencode=arch=compute_100a,code=sm_100a",
    "-U__CUDA_NO_HALF_OPERATORS__",
    "-U__CUDA_NO_HALF_CONVERSIONS__",
    "-U__CUDA_NO_HALF2_OPERATORS__",
]


def module_name(op: str) -> str:
    return f"geraf_ref_{op}"


def built_path(op: str) -> str | None:
    hits = glob.glob(os.path.join(REF_OUT, op, module_name(op) + "*.so"))
    return hits[0] if hits else None


def build(reference_root: str = DEFAULT_REFERENCE, verbose: bool = False) -> dict:
    """Compile and link both modules without importing them (import needs libcuda)."""
    from torch.utils import cpp_extension

    out = {}
    for op in OPS:
        csrc = os.path.join(reference_root, "geraf", "ops", op, "csrc")
        if not os.path.isdir(csrc):
            raise FileNotFoundError(csrc)
        sources = sorted(glob.glob(os.path.join(csrc, "**", "*.cpp"), recursive=True))
        sources += sorted(glob.glob(os.path.join(csrc, "**", "*.cu"), recursive=True))
        build_dir = os.path.join(REF_OUT, op)
        os.makedirs(build_dir, exist_ok=True)
        # load() would import the module right away; only the build half is wanted here.
        cpp_extension._write_ninja_file_and_build_library(  # noqa: SLF001
            name=module_name(op),
            sources=sources,
            extra_cflags=_CFLAGS,
            extra_cuda_cflags=_CUDA_CFLAGS,
            extra_sycl_cflags=None,
            extra_ldflags=[],
            extra_include_paths=[csrc],
            build_directory=build_dir,
            verbose=verbose,
            with_cuda=True,
            with_sycl=False,
            is_standalone=False,
        )
        out[op] = built_path(op)
    return out


def load(op: str):
    """Import a prebuilt reference module (GPU machine only: it needs libcuda)."""
    import importlib.machinery
    import importlib.util

    import torch  # noqa: F401  (the module links against torch's libraries)

    path = built_path(op)
    if path is None:
        raise FileNotFoundError(f"reference module {op} not built; run oracle/build_ref.py")
    name = module_name(op)
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--clean", action="store_true")
    args = ap.parse_args(argv)
    if args.clean and os.path.isdir(REF_OUT):
        shutil.rmtree(REF_OUT)
    res = build(args.reference, verbose=args.verbose)
    for op, path in res.items():
        print(op, "->", path)
    return 0 if all(res.values()) else 1


if __name__ == "__main__":
    sys.exit(main())
