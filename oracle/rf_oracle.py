"""numpy interface of the CPU oracle (``oracle/rf_oracle.c``).

TEST INFRASTRUCTURE ONLY -- imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by ``bench.py``'s CPU-baseline leg; never by the product.

Every function takes FP32 numpy arrays in the reference's layouts (voxels as
[3, N]) and returns new arrays: ``*_f64`` functions return float64 results of
the exact-arithmetic model, ``*_f32`` functions float32 results of the
reference's FP32 operation order.  Which reference lines each follows is
stated in ``rf_oracle.c``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_f = ctypes.c_float


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        mf = [_f32p, _f32p, _f32p, _f32p, _f32p, _i64, _i64, _i64, _f, _f]
        L.oracle_mf_forward_f64.argtypes = mf + [_f64p, _f64p]
        L.oracle_mf_forward_f32.argtypes = mf + [_f32p, _f32p]
        L.oracle_mf_backward_f64.argtypes = mf + [_f64p, _f64p]
        L.oracle_mf_backward_f32.argtypes = mf + [_f32p, _f32p]
        L.oracle_mf_forward_f64r.argtypes = mf + [_f64p, _f64p]
        L.oracle_mf_backward_f64r.argtypes = mf + [_f64p, _f64p]
        fft = [_f32p, _f32p, _f32p, _f32p, _f32p, _i64, _i64, _i64, _f, ctypes.c_int, _f32p, _f32p]
        L.oracle_mf_fft_forward_f32.argtypes = fft
        L.oracle_mf_fft_backward_f32.argtypes = fft
        tr = [_f32p, _f32p, _f32p, _f32p, _f32p, _u8p, _i64, _i64, _i64, _f, _f, _f]
        L.oracle_tracer_forward_f64.argtypes = tr + [_f64p, _f64p]
        L.oracle_tracer_forward_f32.argtypes = tr + [_f32p, _f32p]
        trb = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _u8p, _i64, _i64, _i64, _f, _f, _f]
        L.oracle_tracer_backward_f64.argtypes = trb + [_f64p, _f64p, ctypes.c_void_p]
        L.oracle_tracer_backward_f32.argtypes = trb + [_f32p, _f32p]
        L.oracle_bilinear_forward_f32.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i64, _i64,
                                                  _i64, _f32p, _f32p, _u8p]
        L.oracle_bilinear_backward_f32.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i64, _i64,
                                                   _i64, _f32p, _f32p]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def _f32(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float32)


def _u8(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.uint8)


# ---- matched filter ---------------------------------------------------------
def _mf_fn(kind, form):
    if form not in ("f64", "f64r", "f32"):
        raise ValueError(f"unknown oracle form {form!r}")
    return getattr(lib(), f"oracle_mf_{kind}_{form}")


def mf_forward(real, imag, tx, rx, voxel_3n, fs, As, form="f64"):
    """y[N] complex of the matched filter (MatchedFilter_cuda_kernel.cu:65-115).

    ``form``: "f64" (libm cos/sin per sample), "f64r" (the same FP64 model with
    phasors by FP64 rotation, re-seeded every 16 samples; for full-size
    workloads) or "f32" (the reference's FP32 order)."""
    real, imag, tx, rx, vox = map(_f32, (real, imag, tx, rx, voxel_3n))
    A, S = real.shape
    N = vox.shape[1]
    dt = np.float32 if form == "f32" else np.float64
    out_r = np.zeros(N, dt)
    out_i = np.zeros(N, dt)
    _mf_fn("forward", form)(real, imag, tx, rx, vox, A, S, N, fs, As, out_r, out_i)
    return out_r, out_i


def mf_backward(grad_r, grad_i, tx, rx, voxel_3n, A, S, fs, As, form="f64"):
    """grad[A,S] complex of the adjoint (MatchedFilter_cuda_kernel.cu:171-220);
    ``form`` as for :func:`mf_forward`."""
    gr, gi, tx, rx, vox = map(_f32, (grad_r, grad_i, tx, rx, voxel_3n))
    N = vox.shape[1]
    dt = np.float32 if form == "f32" else np.float64
    out_r = np.zeros((A, S), dt)
    out_i = np.zeros((A, S), dt)
    _mf_fn("backward", form)(gr, gi, tx, rx, vox, A, S, N, fs, As, out_r, out_i)
    return out_r, out_i


def mf_fft_forward(real, imag, tx, rx, voxel_3n, spacing, consistent_bins=False):
    """Range-bin forward (MatchedFilter_cuda_kernel.cu:117-169); ``consistent_bins``
    keeps delays up to 2 * spacing * bins instead of the reference's spacing * bins."""
    real, imag, tx, rx, vox = map(_f32, (real, imag, tx, rx, voxel_3n))
    A, B = real.shape
    N = vox.shape[1]
    out_r = np.zeros(N, np.float32)
    out_i = np.zeros(N, np.float32)
    lib().oracle_mf_fft_forward_f32(real, imag, tx, rx, vox, A, B, N, spacing, int(consistent_bins), out_r,
                                    out_i)
    return out_r, out_i


def mf_fft_backward(grad_r, grad_i, tx, rx, voxel_3n, A, B, spacing, consistent_bins=False):
    """Range-bin adjoint (MatchedFilter_cuda_kernel.cu:222-279)."""
    gr, gi, tx, rx, vox = map(_f32, (grad_r, grad_i, tx, rx, voxel_3n))
    N = vox.shape[1]
    out_r = np.zeros((A, B), np.float32)
    out_i = np.zeros((A, B), np.float32)
    lib().oracle_mf_fft_backward_f32(gr, gi, tx, rx, vox, A, B, N, spacing, int(consistent_bins), out_r,
                                     out_i)
    return out_r, out_i


# ---- signal tracer ----------------------------------------------------------
def tracer_forward(normals, sigmas, points, tx, rx, inbounds, S, fs, f0, As, form="f64"):
    """x[A,S] complex of the tracer (SignalTracer_cuda_kernel.cu:351-450)."""
    normals, sigmas, points, tx, rx = map(_f32, (normals, sigmas, points, tx, rx))
    inb = _u8(inbounds)
    A, P = sigmas.shape
    dt = np.float64 if form == "f64" else np.float32
    out_r = np.zeros((A, S), dt)
    out_i = np.zeros((A, S), dt)
    fn = lib().oracle_tracer_forward_f64 if form == "f64" else lib().oracle_tracer_forward_f32
    fn(normals, sigmas, points, tx, rx, inb, A, S, P, fs, f0, As, out_r, out_i)
    return out_r, out_i


def tracer_backward(grad_r, grad_i, normals, sigmas, points, tx, rx, inbounds, fs, f0, As,
                    form="f64", with_points=True):
    """(grad_normals [P,3], grad_sigmas [A,P], grad_points [P,3] or None)
    (SignalTracer_cuda_kernel.cu:452-587; positions: no reference counterpart)."""
    gr, gi, normals, sigmas, points, tx, rx = map(_f32, (grad_r, grad_i, normals, sigmas, points,
                                                          tx, rx))
    inb = _u8(inbounds)
    A, P = sigmas.shape
    S = gr.shape[1]
    if form == "f64":
        gn = np.zeros((P, 3), np.float64)
        gs = np.zeros((A, P), np.float64)
        gp = np.zeros((P, 3), np.float64) if with_points else None
        lib().oracle_tracer_backward_f64(gr, gi, normals, sigmas, points, tx, rx, inb, A, S, P, fs,
                                         f0, As, gn, gs,
                                         gp.ctypes.data if gp is not None else None)
        return gn, gs, gp
    gn = np.zeros((P, 3), np.float32)
    gs = np.zeros((A, P), np.float32)
    lib().oracle_tracer_backward_f32(gr, gi, normals, sigmas, points, tx, rx, inb, A, S, P, fs, f0,
                                     As, gn, gs)
    return gn, gs, None


# ---- along-ray resampler ---------------------------------------------------
def bilinear_forward(normals, sigmas, z_vals, tgt_z_vals):
    normals, sigmas, z, tz = map(_f32, (normals, sigmas, z_vals, tgt_z_vals))
    R, S, _ = normals.shape
    A = sigmas.shape[0]
    T = tz.shape[1]
    out_n = np.zeros((R, T, 3), np.float32)
    out_s = np.zeros((A, R, T), np.float32)
    out_b = np.zeros((R, T), np.uint8)
    lib().oracle_bilinear_forward_f32(normals, sigmas, z, tz, A, R, S, T, out_n, out_s, out_b)
    return out_n, out_s, out_b.astype(bool)


def bilinear_backward(grad_out_normals, grad_out_sigmas, z_vals, tgt_z_vals, grad_normals=None,
                      grad_sigmas=None):
    gon, gos, z, tz = map(_f32, (grad_out_normals, grad_out_sigmas, z_vals, tgt_z_vals))
    R, T, _ = gon.shape
    A = gos.shape[0]
    S = z.shape[1]
    gn = _f32(grad_normals).copy() if grad_normals is not None else np.zeros((R, S, 3), np.float32)
    gs = _f32(grad_sigmas).copy() if grad_sigmas is not None else np.zeros((A, R, S), np.float32)
    lib().oracle_bilinear_backward_f32(gon, gos, z, tz, A, R, S, T, gn, gs)
    return gn, gs


# ---- matched-filter volume at target points ---------------------------------
def sample_volume(volume, points_norm, mode="bilinear", align_corners=True):
    """FP64 restatement of the reference's ``_sample_volume``
    (geraf/datasets/transforms/loading.py:20-25): torch ``grid_sample`` (the
    published 3-D algorithm of torch, pinned at 2.4.1 by the reference) of a
    [1,1,Nx,Ny,Nz] volume at a grid given as (z, y, x) -- so normalised x
    selects along Nx -- with zero padding; ``mode`` "bilinear" (trilinear in
    3-D) or "nearest" (ties to even).  Returns float64 [P]."""
    vol = np.asarray(volume, np.float64)
    pts = np.asarray(points_norm, np.float64).reshape(-1, 3)
    dims = vol.shape

    def src(c, n):
        return (c + 1.0) * 0.5 * (n - 1) if align_corners else ((c + 1.0) * n - 1.0) * 0.5

    f = [src(pts[:, k], dims[k]) for k in range(3)]
    out = np.zeros(pts.shape[0])

    def gather(idx):
        ok = np.ones(pts.shape[0], bool)
        for k in range(3):
            ok &= (idx[k] >= 0) & (idx[k] < dims[k])
        vals = np.zeros(pts.shape[0])
        safe = [np.where(ok, idx[k], 0).astype(np.int64) for k in range(3)]
        vals[ok] = vol[safe[0][ok], safe[1][ok], safe[2][ok]]
        return vals

    if mode == "nearest":
        return gather([np.rint(f[k]) for k in range(3)])  # numpy rint rounds half to even
    if mode != "bilinear":
        raise ValueError(f"unsupported mode {mode!r}")
    lo = [np.floor(f[k]) for k in range(3)]
    w1 = [f[k] - lo[k] for k in range(3)]
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = ((w1[0] if dx else 1 - w1[0]) * (w1[1] if dy else 1 - w1[1]) *
                     (w1[2] if dz else 1 - w1[2]))
                out += w * gather([lo[0] + dx, lo[1] + dy, lo[2] + dz])
    return out
