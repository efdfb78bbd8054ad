"""The C-ABI boundary: the library loads without a GPU, exports every symbol
``include/geraf_rf.h`` declares, the ctypes binding matches the header, and the
Python drop-in modules expose the reference's names (no compute calls here)."""
import ctypes
import inspect
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "geraf_rf.h")
TESTING_HEADER = os.path.join(ROOT, "include", "geraf_rf_testing.h")


def header_functions(path=HEADER):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    decls = re.findall(r"\b(?:int32_t|const char\*)\s+(geraf_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.S)
    return {name: [a.strip() for a in args.split(",") if a.strip() and a.strip() != "void"]
            for name, args in decls}


def test_header_parses():
    fns = header_functions()
    assert "geraf_mf_forward" in fns and "geraf_tracer_backward" in fns
    assert len(fns) == 21
    assert list(header_functions(TESTING_HEADER)) == ["geraf_rf_selftest_wait_timeout"]


def test_library_exports_every_declared_symbol():
    from geraf_b200 import _lib

    lib = _lib.load()
    for name in list(header_functions()) + list(header_functions(TESTING_HEADER)):
        assert hasattr(lib, name), name


def test_ctypes_signatures_match_header():
    from geraf_b200 import _lib

    for path, table in ((HEADER, _lib.SIGNATURES), (TESTING_HEADER, _lib.TEST_SIGNATURES)):
        fns = header_functions(path)
        assert set(fns) == set(table)
        for name, args in fns.items():
            assert len(table[name][1]) == len(args), name


def test_measurement_probes_are_not_in_the_operator_library():
    """The FP32 peak probes live in benchkit's libgeraf_probe.so, not here."""
    from geraf_b200 import _lib

    lib = _lib.load()
    for name in ("geraf_rf_fma_probe", "geraf_rf_horner_probe", "geraf_rf_sincos_identity_check"):
        assert not hasattr(lib, name), name


def test_probe_library_exports_its_probes():
    from benchkit import probes

    lib = probes.lib()
    for name in probes.SIGNATURES:
        assert hasattr(lib, name), name


def test_selftest_rejects_bad_arguments_without_gpu():
    from geraf_b200 import _lib

    lib = _lib.load()
    fn = lib.geraf_rf_selftest_wait_timeout
    assert fn(0, 1, 8, None) == _lib.GERAF_ERR_INVALID_ARGUMENT          # no limit
    assert fn(3_000_000_000, 1, 8, None) == _lib.GERAF_ERR_INVALID_ARGUMENT  # above the operators' 2 s
    assert fn(1_000_000, 0, 8, None) == _lib.GERAF_ERR_INVALID_ARGUMENT  # no blocks
    assert fn(1_000_000, 1, None, None) == _lib.GERAF_ERR_INVALID_ARGUMENT


def test_info_entry_points_run_without_gpu():
    from geraf_b200 import _lib

    lib = _lib.load()
    assert lib.geraf_rf_cudart_version() >= 12000
    assert b"sm_100a" in lib.geraf_rf_build_info()
    assert lib.geraf_rf_last_error() == b""


def test_validation_errors_without_gpu():
    """Argument checks run before any CUDA call, so they work on a CPU host."""
    from geraf_b200 import _lib

    lib = _lib.load()
    rc = lib.geraf_mf_forward(None, None, None, None, None, None, None, -1, 4, 5e6, 1.0, 8,
                              _lib.DTYPE_F32, _lib.MODE_MIXED, None, None, 0, None)
    assert rc == _lib.GERAF_ERR_INVALID_ARGUMENT
    assert b"non-negative" in lib.geraf_rf_last_error()
    rc = lib.geraf_tracer_forward(None, None, None, None, None, None, None, None, 4, 5e6, 770.0,
                                  1.0, 2, 3, _lib.DTYPE_F16, _lib.MODE_PLAIN, None, None, 0, None)
    assert rc == _lib.GERAF_ERR_INVALID_ARGUMENT
    assert b"not implemented for 'Half'" in lib.geraf_rf_last_error()
    rc = lib.geraf_bilinear_forward(None, None, None, None, None, None, None, 1, 2, 1, 3,
                                    _lib.DTYPE_F32, None)
    assert rc == _lib.GERAF_ERR_INVALID_ARGUMENT
    assert b"at least 2 samples" in lib.geraf_rf_last_error()


def test_workspace_query_without_gpu():
    from geraf_b200 import _lib

    # Plain forms never need a workspace; explicit splits make the mixed forward need one.
    assert _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", 64, 32, 1000, 0, 0, None) == 0
    t = _lib.Tuning.from_dict({"splits": 4})
    n = _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", 64, 32, 1000, 0, 1, ctypes.byref(t))
    assert n == 4 * 1000 * 8
    # NUFFT: deconvolution factors (S floats, 256-aligned) + the [A][M + 16] float2 range
    # grid (M = 64 for S = 32), plus [splits][N] partials / [splits][A][M] adjoint grids.
    t = _lib.Tuning.from_dict({"splits": 1})
    n = _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", 64, 32, 1000, 0, _lib.MODE_NUFFT, ctypes.byref(t))
    assert n == 256 + 64 * 80 * 8
    t = _lib.Tuning.from_dict({"splits": 3})
    n = _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", 64, 32, 1000, 0, _lib.MODE_NUFFT, ctypes.byref(t))
    assert n == 256 + 64 * 80 * 8 + 24064  # 3 * 1000 float2, 256-aligned
    n = _lib.workspace_bytes("geraf_mf_backward_workspace_bytes", 64, 32, 1000, 0, _lib.MODE_NUFFT,
                             ctypes.byref(t))
    assert n == 256 + 6400 + 3 * 64 * 64 * 8  # + voxel bounding-box scratch (257 x 6 floats)
    lib = _lib.load()
    size = ctypes.c_size_t(0)
    rc = lib.geraf_mf_forward_workspace_bytes(4, 5000, 10, 0, _lib.MODE_NUFFT, None, ctypes.byref(size))
    assert rc == _lib.GERAF_ERR_UNSUPPORTED and b"4096" in lib.geraf_rf_last_error()


REFERENCE_C_NAMES = {
    "RFMatchedFilter": ["MatchedFilter_forward", "MatchedFilter_fft_forward",
                        "MatchedFilter_backward_realimag", "MatchedFilter_fft_backward_realimag",
                        "get_cuda_version", "has_cuda", "get_compiler_version"],
    "RFSignalTracer": ["SignalTracer_forward", "SignalTracer_backward_normal_sigma",
                       "BilinearRaysample_forward", "BilinearRaysample_backward",
                       "get_cuda_version", "has_cuda", "get_compiler_version"],
}

REFERENCE_ARITY = {
    "MatchedFilter_forward": 12, "MatchedFilter_fft_forward": 13,
    "MatchedFilter_backward_realimag": 14, "MatchedFilter_fft_backward_realimag": 15,
    "SignalTracer_forward": 14, "SignalTracer_backward_normal_sigma": 16,
    "BilinearRaysample_forward": 11, "BilinearRaysample_backward": 10,
}


@pytest.mark.parametrize("op", sorted(REFERENCE_C_NAMES))
def test_c_module_surface(op):
    import importlib

    mod = importlib.import_module(f"geraf_b200.ops.{op}._C")
    for name in REFERENCE_C_NAMES[op]:
        assert callable(getattr(mod, name)), name
    for name, arity in REFERENCE_ARITY.items():
        if hasattr(mod, name) and name.split("_")[0] in ("MatchedFilter", "SignalTracer", "BilinearRaysample"):
            params = [p for p in inspect.signature(getattr(mod, name)).parameters.values()
                      if p.kind == p.POSITIONAL_OR_KEYWORD]
            assert len(params) == arity, name
    assert mod.has_cuda() is True
    assert mod.get_cuda_version().startswith("CUDA 12.")
    assert mod.get_compiler_version().startswith("GCC")


def test_lazy_exports():
    import geraf_b200.ops.RFMatchedFilter as mf
    import geraf_b200.ops.RFSignalTracer as st

    assert set(mf.__all__) == {"matched_filter_cuda", "faster_matched_filter_cuda"}
    assert set(st.__all__) == {"signal_tracer_cuda", "bilinear_raysample_cuda"}
    assert callable(mf.matched_filter_cuda) and callable(st.bilinear_raysample_cuda)
    with pytest.raises(AttributeError):
        getattr(mf, "nope")


def test_public_signatures_match_reference():
    from geraf_b200.ops.RFMatchedFilter import faster_matched_filter_cuda, matched_filter_cuda
    from geraf_b200.ops.RFSignalTracer import bilinear_raysample_cuda, signal_tracer_cuda

    def positional(fn):
        return [p.name for p in inspect.signature(fn).parameters.values()
                if p.kind == p.POSITIONAL_OR_KEYWORD]

    assert positional(matched_filter_cuda) == ["real", "image", "tpos", "rpos", "voxel",
                                               "total_ant_size", "numADCSample", "adcSampleRate",
                                               "As_sci", "N"]
    assert positional(faster_matched_filter_cuda)[:9] == ["real_sel", "image_sel", "real_unsel",
                                                          "image_unsel", "tpos_sel", "rpos_sel",
                                                          "tpos_unsel", "rpos_unsel", "voxel"]
    assert positional(signal_tracer_cuda) == ["normals", "sigmas", "points", "antenna_t",
                                              "antenna_r", "inbounds", "numADCSample",
                                              "adcSampleRate", "fc_start", "As_sci",
                                              "total_ant_size", "total_point_size", "use_diff",
                                              "nomralization"]
    assert positional(bilinear_raysample_cuda) == ["normals", "sigmas", "z_vals", "tgt_z_vals",
                                                   "N_ant", "N_ray", "Nz", "Nz_tgt"]
