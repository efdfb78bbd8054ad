"""CPU model of the matched filter's NUFFT form (FP64 numpy): the parameter
choices of ``nufft_kernels.cu`` (mode centring, Gauss-Legendre deconvolution,
power-of-two grid >= 2S, ES kernel with beta = 2.30 W) give the stated
truncation errors, and the model reproduces the FP64 oracle's matched filter."""
import numpy as np
import pytest

from conftest import rel_l2
from benchkit import scenes
from oracle import rf_oracle as orc

NODES, WEIGHTS = np.polynomial.legendre.leggauss(48)


def grid_points(S):
    M = 16
    while M < 2 * S:
        M *= 2
    return M


def es(t, beta):
    return np.exp(beta * (np.sqrt(np.maximum(0.0, 1.0 - t * t)) - 1.0))


def nufft_sum(s, d, W):
    """sum_n s[n] e^{-j 2 pi n d} at every d, the library's way."""
    S = s.shape[0]
    M, h, beta = grid_points(S), S // 2, 2.30 * W
    u = 0.25 * W * (1.0 + NODES)
    wu = 0.25 * W * WEIGHTS
    m = np.arange(S) - h
    phi_hat = 2.0 * (wu * es(u * 2.0 / W, beta) * np.cos(2 * np.pi * np.outer(m / M, u))).sum(1)
    c = np.zeros(M, complex)
    c[m % M] = s / phi_hat
    g = np.fft.fft(c)
    d = d - np.rint(d)
    uu = d * M
    fl = np.floor(uu)
    f = uu - fl
    base = fl.astype(np.int64) - W // 2 + 1
    q = np.zeros(d.shape, complex)
    for k in range(W):
        q += es((f + W / 2 - 1 - k) * 2.0 / W, beta) * g[(base + k) % M]
    return np.exp(-2j * np.pi * h * d) * q


# truncation bound per width (FP64 model); the FP32 library adds ~1e-6 of rounding
BOUNDS = {4: 2e-3, 6: 2e-5, 8: 3e-7, 10: 5e-9, 12: 1e-10}


@pytest.mark.parametrize("S", [1, 2, 7, 64, 100, 256])
@pytest.mark.parametrize("W", sorted(BOUNDS))
def test_truncation_error(S, W):
    rng = np.random.default_rng(S * 31 + W)
    s = rng.standard_normal(S) + 1j * rng.standard_normal(S)
    d = rng.uniform(-0.5, 0.5, 3000)
    ref = np.exp(-2j * np.pi * np.outer(d, np.arange(S))) @ s
    assert rel_l2(nufft_sum(s, d, W), ref) < BOUNDS[W]


def test_error_falls_with_width():
    rng = np.random.default_rng(1)
    s = rng.standard_normal(128) + 1j * rng.standard_normal(128)
    d = rng.uniform(-0.5, 0.5, 2000)
    ref = np.exp(-2j * np.pi * np.outer(d, np.arange(128))) @ s
    errs = [rel_l2(nufft_sum(s, d, W), ref) for W in (4, 6, 8, 10)]
    assert all(a > 10 * b for a, b in zip(errs, errs[1:]))


def test_model_reproduces_oracle_matched_filter():
    """The MIXED phase model (cycles c0 and per-sample step d from the FP64 path
    length) with the model's sample sum equals the FP64 oracle's matched filter."""
    rng = np.random.default_rng(3)
    tx, rx = scenes.virtual_array(2)
    pos, amp = scenes.point_scene(rng, 4, size=0.1)
    ch = scenes.chirp(48)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0, rng=rng)
    vox = scenes.voxel_grid(5, size=0.1)
    ref = orc.mf_forward(re, im, tx, rx, vox, ch.adc_sample_rate, ch.As_sci)
    ref = ref[0] + 1j * ref[1]
    # constants of the MIXED form: pi_f is the FP32 value of pi the reference uses
    pi_f = float(np.float32(np.pi))
    c = float(np.float32(2.9979))
    k0 = (pi_f / np.pi) * float(np.float32(773.704)) / c
    k1 = (pi_f / np.pi) * float(np.float32(ch.As_sci)) / (float(np.float32(ch.adc_sample_rate)) * c)
    bias = float(np.float32(0.15))
    s = re.astype(np.float64) + 1j * im.astype(np.float64)
    y = np.zeros(vox.shape[1], complex)
    for a in range(tx.shape[0]):
        dist = (np.linalg.norm(tx[a].astype(np.float64)[:, None] - vox.astype(np.float64), axis=0)
                + np.linalg.norm(rx[a].astype(np.float64)[:, None] - vox.astype(np.float64), axis=0))
        c0 = (dist + bias) * k0
        d = (dist + bias) * k1
        y += np.exp(-2j * np.pi * (c0 - np.rint(c0))) * nufft_sum(s[a], d, 10)
    y /= tx.shape[0]
    assert rel_l2(y, ref) < 1e-6


# degree of each tap's weight polynomial (nufft_kernels.cu, poly_degree) and its bound
POLY = {4: (5, 1e-4), 6: (6, 3e-6), 8: (7, 1.5e-7), 10: (9, 1.5e-7), 12: (11, 1.5e-7)}


@pytest.mark.parametrize("W", sorted(POLY))
def test_tap_weight_polynomials(W):
    """Chebyshev interpolants of the tap weights at P + 1 nodes, in monomial form,
    evaluated by FP32 Horner, stay within the stated absolute error."""
    from numpy.polynomial import chebyshev as C

    P, bound = POLY[W]
    beta = 2.30 * W
    nodes = np.cos(np.pi * (np.arange(P + 1) + 0.5) / (P + 1))
    f = np.linspace(0.0, 1.0, 20001)[:-1]
    z32 = (2.0 * f - 1.0).astype(np.float32)
    worst = 0.0
    for k in range(W):
        def w(zz):
            return es(((zz + 1.0) / 2.0 + W / 2 - 1 - k) * 2.0 / W, beta)
        mono = C.cheb2poly(C.chebfit(nodes, w(nodes), P)).astype(np.float32)
        acc = np.full_like(z32, mono[-1])
        for c in mono[-2::-1]:
            acc = acc * z32 + c
        worst = max(worst, float(np.abs(acc.astype(np.float64) - w(2.0 * f - 1.0)).max()))
    assert worst < bound
