"""CPU known-answer tests of the oracle (no GPU).

The reference ships no tests or golden vectors and cannot be built here, so
the oracle is pinned by properties that the reference's algorithm has by
construction (cubic.rs Lagrange weights, convolve_rv.rs kernels and
resampling, continuum_fitting.rs least squares), plus regression against the
committed fixtures in tests/golden/.
"""
import os

import numpy as np
import pytest

import oracle as O
from pasta_b200 import synth as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def small():
    spec = S.config0_grid(n_px=4000)
    labels, spectra, factors = S.make_grid(spec)
    g = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    return spec, labels, spectra, g


def test_grid_axes_and_order(small):
    spec, labels, spectra, g = small
    t, m, lg = g.axes()
    np.testing.assert_array_equal(t, spec.teffs)
    np.testing.assert_array_equal(m, np.sort(spec.ms))
    np.testing.assert_array_equal(lg, spec.loggs)


def test_interpolation_at_nodes_reproduces_models(small):
    """Lagrange property (cubic.rs:29-60): weights are one-hot at a grid node."""
    spec, labels, spectra, g = small
    n = spec.n_px - spec.n_px % 128
    for i in (0, 57, 211, 494):
        out = g.interpolate(*labels[i], O.F32)
        assert np.abs(out[:n] - spectra[i][:n] / np.float32(65535.0)).max() < 1e-6
        # tail pixels carry the extra 1/65535 (interpolate.rs:978)
        np.testing.assert_allclose(out[n:], spectra[i][n:] / 65535.0 / 65535.0, rtol=1e-6, atol=1e-12)


def _poly_grid(deg):
    """Grid whose spectra are a polynomial of total degree `deg` in the labels."""
    t = np.arange(6000.0, 8001.0, 250.0)
    m = np.round(np.arange(-0.5, 0.501, 0.1), 2)
    lg = np.arange(3.5, 4.501, 0.25)
    pts = np.array([(a, b, c) for a in t for c in lg for b in m])
    rng = np.random.default_rng(0)
    npx = 256
    coef = rng.uniform(0.0, 1.0, (npx, 3))
    x = np.stack([(pts[:, 0] - 6000) / 2000, (pts[:, 1] + 0.5), (pts[:, 2] - 3.5)], axis=1)
    vals = 0.1 + 0.25 * (x[:, 0][:, None] ** deg * coef[:, 0] + x[:, 1][:, None] ** deg * coef[:, 1]
                         + x[:, 2][:, None] ** deg * coef[:, 2])
    spectra = np.clip(np.rint(vals * 65535.0), 0, 65535).astype(np.uint16)
    return pts, spectra, coef


def test_cubic_spectra_are_reproduced_inside_the_grid():
    """cubic Lagrange interpolation is exact for cubic dependence on the labels."""
    pts, spectra, coef = _poly_grid(3)
    g = O.Grid(pts, spectra, None, O.WL_LOGSPACE, 3.6, 1e-5)
    # exact reference: interpolate the quantized node values with the f64 weights
    for lab in [(6700.0, 0.03, 3.9), (7333.0, -0.27, 4.11)]:
        cols, w = g.local_grid(*lab)
        data = spectra.astype(np.float64)
        # column order is list_gridpoints (teff, logg, m inner) = pts order here
        exact = sum(w[j] * data[cols[j]] for j in range(64) if cols[j] >= 0) / 65535.0
        out = g.interpolate(*lab, O.F64)
        np.testing.assert_allclose(out[:128], exact[:128], rtol=1e-12)
        # and the polynomial itself (up to the uint16 quantisation)
        x = np.array([(lab[0] - 6000) / 2000, lab[1] + 0.5, lab[2] - 3.5])
        poly = 0.1 + 0.25 * (x[0] ** 3 * coef[:, 0] + x[1] ** 3 * coef[:, 1] + x[2] ** 3 * coef[:, 2])
        assert np.abs(out[:128] - poly[:128]).max() < 3e-5


def test_weights_sum_to_one(small):
    spec, labels, spectra, g = small
    rng = np.random.default_rng(1)
    for _ in range(20):
        lab = (rng.uniform(6000, 8000), rng.uniform(-0.5, 0.5), rng.uniform(3.5, 4.5))
        cols, w = g.local_grid(*lab)
        assert abs(w.sum() - 1.0) < 1e-12
        assert (w[cols < 0] == 0).all()


def test_outside_grid_is_an_error(small):
    g = small[3]
    with pytest.raises(O.OracleError):
        g.interpolate(9000.0, 0.0, 4.0)
    with pytest.raises(O.OracleError):
        g.interpolate(7000.0, 0.7, 4.0)


@pytest.mark.parametrize("vsini", [1.0, 10.0, 50.0, 300.0])
def test_rotation_kernel(vsini):
    """convolve_rv.rs:438-475: odd width from the formula, normalised, symmetric."""
    dvelo = np.log(10.0) * 1.2e-6
    k = O.rotation_kernel(vsini, dvelo)
    vrot = vsini / 299792.0
    n = max(1, int(np.ceil(2 * vrot / dvelo * np.sqrt(1 + (4 * (0.6 - 1) / (np.pi * 0.6)) ** 2))) + 2)
    n = n + 1 - n % 2
    assert len(k) == n
    assert abs(k.sum() - 1.0) < 1e-6
    np.testing.assert_allclose(k, k[::-1], atol=1e-6)


def test_identity_resampling_and_exact_shift(small):
    """rv = 0 on the synthetic pixels is the identity (convolve_rv.rs:586-594)."""
    spec, labels, spectra, g = small
    wl = spec.wl()[300:3500]
    d = O.Disp(g, O.DISP_NONE, wl)
    lab = [7000.0, 0.0, 4.0, 0.0, 0.0]
    m = d.produce_model(lab, O.F64)
    ref = g.interpolate(7000.0, 0.0, 4.0, O.F64)[300:3500]
    assert np.abs(m - ref).max() < 1e-6


def test_chunk_fitter_recovers_polynomial_continuum(small):
    """observed = model * polynomial of degree <= p: chi2 -> 0 and the continuum is recovered."""
    spec, labels, spectra, g = small
    wl = spec.wl()[200:3800]
    model = np.linspace(0.5, 1.0, len(wl))
    x = (wl - wl[0]) / (wl[-1] - wl[0])
    cont = 1.0 + 0.3 * x - 0.2 * x ** 2 + 0.05 * x ** 3
    flux = (model * cont).astype(np.float32)
    var = np.full(len(wl), 1e-4, np.float32)
    c = O.Cont(O.CONT_CHUNK, wl, 5, 8, 0.2)
    params, chi2 = c.fit(flux, var, model, O.F64)
    assert chi2 < 1e-6
    built = c.build(params, O.F64)
    np.testing.assert_allclose(built, cont, rtol=1e-5)


def test_f32_mirror_vs_f64(small):
    spec, labels, spectra, g = small
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 3000, 100.0, 85000.0, seed=2)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    m32, m64 = d.produce_model(star.label, O.F32), d.produce_model(star.label, O.F64)
    assert np.abs(m32 - m64).max() / np.abs(m64).max() < 2e-6
    c = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    x32, _ = O.chi2(g, d, c, star.flux, star.var, star.label[None], O.F32)
    x64, _ = O.chi2(g, d, c, star.flux, star.var, star.label[None], O.F64)
    assert abs(x32[0] - x64[0]) / x64[0] < 1e-4


def test_draw_stream():
    a = [O.draw_u01(7, 3, i, 2, 1) for i in range(2000)]
    assert min(a) >= 0.0 and max(a) < 1.0
    assert abs(np.mean(a) - 0.5) < 0.03
    assert O.draw_u01(7, 3, 5, 2, 1) == O.draw_u01(7, 3, 5, 2, 1)
    assert O.draw_u01(7, 3, 5, 2, 1) != O.draw_u01(8, 3, 5, 2, 1)


def test_seeded_fit_is_deterministic(small):
    spec, labels, spectra, g = small
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 3000, 100.0, 85000.0, seed=2)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    c = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    st = O.settings(12, 6, (0.0, 300.0), (-150.0, 150.0))
    r1, rc1 = O.fit(g, d, c, st, star.flux[None], star.var[None], [5], O.F32, nthreads=4, over_stars=False)
    r2, rc2 = O.fit(g, d, c, st, star.flux[None], star.var[None], [5], O.F32, nthreads=1, over_stars=True)
    assert rc1 == 0 and rc2 == 0
    np.testing.assert_array_equal(r1[0]["label"], r2[0]["label"])
    assert r1[0]["chi2"] == r2[0]["chi2"]


def test_brent_root_known_answer():
    # x^2 - 0.25 on [0, 1] has its root at 0.5; on [-1, 0] at -0.5
    r = O._brent(lambda x: x * x - 0.25, 0.0, 1.0, tol=1e-10)
    assert abs(r - 0.5) < 1e-9
    r = O._brent(lambda x: x * x - 0.25, -1.0, 0.0, tol=1e-10)
    assert abs(r + 0.5) < 1e-9
    with pytest.raises(ValueError):
        O._brent(lambda x: x * x + 1.0, 0.0, 1.0)


def test_uncertainty_crossings_bracket_the_target(small):
    spec, labels, spectra, g = small
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 3000, 100.0, 85000.0, seed=2)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    c = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    sr = np.array([0.05, 0.3, 0.3, 0.5, 40.0])
    res = O.compute_uncertainty(g, d, c, star.flux, star.var, 85000.0, star.label, sr)
    best, _ = O.chi2(g, d, c, star.flux, star.var, star.label, O.F64)
    n = 4.0 * 85000.0 * (star.wl[-1] - star.wl[0]) / (star.wl[0] + star.wl[-1])
    target = best[0] * (1.0 + np.sqrt(2.0 / n))
    radius = sr * np.array([star.label[0], 1, 1, 1, 1])
    radius[3] = max(star.label[3] * sr[3], 100.0)
    found = 0
    for i in range(5):
        for side, dist in zip((-1, 1), res[i]):
            if dist is None:
                continue
            # Brent stops with the crossing inside +-tol (1e-3 of the radius)
            # of its estimate; chi2 may jump there (vsini changes the kernel width)
            f = []
            for off in (-2e-3, 2e-3):
                lab = star.label.copy()
                lab[i] += side * (dist + off * radius[i])
                x, st = O.chi2(g, d, c, star.flux, star.var, lab, O.F64)
                assert st[0] == 0
                f.append(x[0] - target)
            assert f[0] * f[1] <= 0.0, (i, side, dist, f)
            found += 1
    assert found >= 8


# ------------------------------------------------------------------ binaries
def test_linear_interpolation_known_answers():
    """interpolate_linear (interpolate.rs:985-1028, cubic.rs:6-10): at a node the
    weights are one-hot, every pixel is u16 / 65535 * factor; spectra linear in
    each label (a trilinear field) are reproduced anywhere inside the grid;
    the weights sum to one; outside the grid is an error."""
    pts, spectra, coef = _poly_grid(1)
    g = O.Grid(pts, spectra, None, O.WL_LOGSPACE, 3.6, 1e-5)
    for i in (0, 17, 240, len(pts) - 1):
        out = g.interpolate_linear(*pts[i], O.F64)
        np.testing.assert_allclose(out, spectra[i] / 65535.0 / 65535.0, rtol=1e-12)
    for lab in [(7130.0, 0.07, 4.02), (6000.0, -0.5, 3.5), (7999.0, 0.49, 4.49), (6250.0, 0.0, 3.75)]:
        cols, w = g.local_grid_linear(*lab)
        assert abs(w.sum() - 1.0) < 1e-12
        assert (cols >= 0).all()
        out = g.interpolate_linear(*lab, O.F64) * 65535.0 * 65535.0
        x = np.array([(lab[0] - 6000) / 2000, lab[1] + 0.5, lab[2] - 3.5])
        exact = (0.1 + 0.25 * (x[0] * coef[:, 0] + x[1] * coef[:, 1] + x[2] * coef[:, 2])) * 65535.0
        assert np.abs(out - exact).max() <= 0.51  # quantisation of the nodes
    for bad in [(5999.0, 0.0, 4.0), (7000.0, 0.6, 4.0), (7000.0, 0.0, 4.6)]:
        with pytest.raises(O.OracleError):
            g.interpolate_linear(*bad)


@pytest.fixture(scope="module")
def binary_small(small):
    spec, labels, spectra, g = small
    cl, cs, cf = S.make_continuum_grid(spec)
    gc = O.Grid(cl, cs, cf, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    star = S.make_binary_star(spec, [7600.0, 0.1, 4.1, 30.0, -40.0], [6300.0, -0.2, 3.8, 10.0, 45.0], 0.6,
                              3000, 150.0, 85000.0, seed=5)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    return spec, g, gc, d, star


def test_binary_model_identities(binary_small):
    """produce_binary_model_norm (interpolate.rs:868-893): two identical stars
    give the single-star model, a zero light ratio gives star 1 alone, and
    swapping the stars with light ratio r -> the model with 1/r."""
    spec, g, gc, d, star = binary_small
    l1 = [7600.0, 0.1, 4.1, 30.0, -40.0]
    l2 = [6300.0, -0.2, 3.8, 10.0, 45.0]
    single = d.produce_model(l1, O.F64)
    np.testing.assert_allclose(O.binary_model(g, gc, d, l1 + l1 + [0.4], O.F64), single, rtol=1e-12)
    np.testing.assert_allclose(O.binary_model(g, gc, d, l1 + l2 + [0.0], O.F64), single, rtol=1e-12)
    a = O.binary_model(g, gc, d, l1 + l2 + [0.5], O.F64)
    b = O.binary_model(g, gc, d, l2 + l1 + [2.0], O.F64)
    np.testing.assert_allclose(a, b, rtol=1e-12)
    m32 = O.binary_model(g, gc, d, l1 + l2 + [0.5], O.F32)
    assert np.abs(m32 - a).max() / np.abs(a).max() < 1e-5


def test_binary_chi2_is_smallest_at_the_truth(binary_small):
    spec, g, gc, d, star = binary_small
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    truth = list(star.label)
    labs = [truth]
    for k, dx in [(0, 150.0), (4, 8.0), (5, -150.0), (9, -8.0), (10, 0.2)]:
        x = list(truth)
        x[k] += dx
        labs.append(x)
    c, st = O.binary_chi2(g, gc, d, oc, star.flux, star.var, labs, O.F64)
    assert (st == 0).all()
    assert c[0] < 1.1 and (c[1:] > c[0]).all(), c
    bad = list(truth)
    bad[5] = 9000.0  # star 2 outside the grid
    c, st = O.binary_chi2(g, gc, d, oc, star.flux, star.var, [bad], O.F64)
    assert st[0] != 0 and np.isnan(c[0])


def test_binary_fit_is_deterministic_and_bounded(binary_small):
    spec, g, gc, d, star = binary_small
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    st = O.binary_settings(12, 4, (0.0, 100.0), (-100.0, 100.0), constraints=[(10, 1, 0.6, 0.6)])
    r1, rc1 = O.binary_fit(g, gc, d, oc, st, star.flux, star.var, 9, O.F64, nthreads=2)
    r2, rc2 = O.binary_fit(g, gc, d, oc, st, star.flux, star.var, 9, O.F64, nthreads=3)
    assert rc1 == 0 and rc2 == 0
    assert r1["chi2"] == r2["chi2"]
    np.testing.assert_array_equal(r1["label1"], r2["label1"])
    assert r1["light_ratio"] == 0.6
    assert 0.0 <= r1["label1"][3] <= 100.0 and -100.0 <= r1["label2"][4] <= 100.0


def _oa_convolve_numpy32(x, k):
    """convolve_rv.rs:121-157 restated with numpy's float32 FFT (pocketfft), an
    FFT implementation independent of the oracle's own radix-2 transform:
    overlap-add blocks of 2048 - (m - 1) inputs, forward real FFT, product
    with the kernel's spectrum, inverse, summed into the output."""
    n, m = 2048, len(k)
    step, L = n - (m - 1), len(x)
    nx = -(-L // step) * step
    pad = np.zeros(n, np.float32)
    pad[:m] = k
    H = np.fft.rfft(pad)
    y = np.zeros(nx + m - 1 + n, np.float32)
    for pos in range(0, nx, step):
        ln = min(step, L - pos)
        pad = np.zeros(n, np.float32)
        pad[:ln] = x[pos:pos + ln]
        r = np.fft.irfft(np.fft.rfft(pad) * H, n).astype(np.float32)
        y[pos:pos + n] += r
    return y


@pytest.mark.parametrize("vsini", [8.0, 60.0, 300.0])
def test_fft_substitution_matches_an_independent_float32_fft(small, vsini):
    """The oracle's FP32 mirror replaces rustfft/realfft by its own radix-2
    real FFT with the reference's overlap-add blocking.  The same blocking
    with numpy's float32 FFT (an independent implementation, as rustfft is)
    agrees with it to float32 roundoff, and both sit at the same distance
    from the FP64 (direct) convolution."""
    spec, labels, spectra, g = small
    x = g.interpolate(7000.0, 0.0, 4.0, O.F32)
    k = O.rotation_kernel(vsini, np.log(10.0) * spec.log_step).astype(np.float32)
    start = len(k) // 2
    ref_np = _oa_convolve_numpy32(x.astype(np.float32), k)[start:start + len(x)].astype(np.float64)
    y32 = g.convolve_rotation(x, vsini, O.F32)
    y64 = g.convolve_rotation(x, vsini, O.F64)
    scale = np.abs(y64).max()
    # measured: 3-5e-7 of the maximum between the two float32 FFTs, and 2-5e-7 from FP64 for each
    assert np.abs(y32 - ref_np).max() <= 1e-6 * scale
    e_oracle, e_numpy = np.abs(y32 - y64).max() / scale, np.abs(ref_np - y64).max() / scale
    assert e_oracle <= 1e-6 and e_numpy <= 1e-6


def test_qr_substitution_matches_svd_least_squares(small):
    """The oracle's FP32 mirror solves each chunk's unweighted least squares
    (continuum_fitting.rs:216-226) by Householder QR instead of nalgebra's f32
    SVD.  LAPACK's float32 SVD least squares (numpy lstsq, sgelsd) on the same
    float32 design matrix and ratios gives the same chunk continua within
    5e-6 of their maximum (degree 8: measured up to 2.3e-6, all of it the QR
    mirror's own roundoff: sgelsd lands within 1e-7 of the FP64 solution).
    How close nalgebra's f32 SVD lands is not known here; the model tolerance
    of the parity tests (1e-5) covers either."""
    spec, labels, spectra, g = small
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 3000, 100.0, 85000.0, seed=4)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    model = d.produce_model(star.label, O.F64)
    p = 8
    c = O.Cont(O.CONT_CHUNK, star.wl, 5, p, 0.2)
    par32, _ = c.fit(star.flux, star.var, model.astype(np.float32), O.F32)
    par64, _ = c.fit(star.flux, star.var, model, O.F64)
    y32 = (star.flux.astype(np.float32) / model.astype(np.float32)).astype(np.float32)
    for ch, (s0, e0) in enumerate(c.chunk_bounds()):
        wl = star.wl[s0:e0]
        xx = -1.0 + 2.0 * (wl - wl[0]) / (wl[-1] - wl[0])
        A64 = np.vander(xx, p + 1, increasing=True)
        A32 = A64.astype(np.float32)
        sol_np = np.linalg.lstsq(A32, y32[s0:e0], rcond=None)[0].astype(np.float64)
        c_np = A64 @ sol_np
        c_32 = A64 @ par32[ch * (p + 1):(ch + 1) * (p + 1)]
        c_64 = A64 @ par64[ch * (p + 1):(ch + 1) * (p + 1)]
        scale = np.abs(c_64).max()
        assert np.abs(c_32 - c_np).max() <= 5e-6 * scale
        assert np.abs(c_32 - c_64).max() <= 5e-6 * scale
        assert np.abs(c_np - c_64).max() <= 3e-7 * scale


def test_linear_model_substitution_matches_svd_least_squares(small):
    """LinearModelFitter (continuum_fitting.rs:44-107) solves D sol = flux /
    model with nalgebra's f32 SVD; the oracle's FP32 mirror uses Householder
    QR.  On a 40-column Legendre design both it and LAPACK's float32 SVD least
    squares give the same fitted continuum within 1e-5 of its maximum
    (measured: the QR mirror 5.6e-6 from FP64, sgelsd 4e-8), and the same
    ratio-space chi2 within 1e-4 relative (measured 2e-7)."""
    spec, labels, spectra, g = small
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 3000, 100.0, 85000.0, seed=6)
    d = O.Disp(g, O.DISP_FIXED, star.wl, 85000.0)
    model = d.produce_model(star.label, O.F64)
    x = np.linspace(-1.0, 1.0, len(star.wl))
    D = np.polynomial.legendre.legvander(x, 39).astype(np.float32)
    c = O.Cont(O.CONT_LINEAR, design=D)
    par32, chi32 = c.fit(star.flux, star.var, model.astype(np.float32), O.F32)
    par64, chi64 = c.fit(star.flux, star.var, model, O.F64)
    b32 = (star.flux.astype(np.float32) / model.astype(np.float32)).astype(np.float32)
    sol_np = np.linalg.lstsq(D, b32, rcond=None)[0].astype(np.float64)
    D64 = D.astype(np.float64)
    f_np, f_32, f_64 = D64 @ sol_np, D64 @ par32, D64 @ par64
    scale = np.abs(f_64).max()
    assert np.abs(f_32 - f_np).max() <= 1e-5 * scale
    assert np.abs(f_np - f_64).max() <= 1e-5 * scale
    r = (f_np - b32)[50:-50]
    chi_np = float(np.sum(r / star.var[50:-50] * r) / len(b32))
    assert abs(chi_np - chi64) <= 1e-4 * chi64 and abs(chi32 - chi64) <= 1e-4 * chi64
