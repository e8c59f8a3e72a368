"""Seeded synthetic grids and observed stars in PASTA's on-disk format.

There is no public dataset for this path, so every workload is synthetic:

* A grid model is ``F = 1 - sum_l d_l(theta) * G_l(lambda)`` over a fixed line
  list of Gaussian absorption lines (centres seeded-uniform, widths
  0.05-0.3 A).  Each depth ``d_l`` is linear in the normalised labels
  (Teff, [M/H], logg) and clipped to 0-0.8.  Models are stored as
  ``round(F * 65535)`` uint16, one spectrum per model
  (model_fetchers.rs:48-67 reads the same format).
* With ``includes_factor`` the model is a blackbody continuum times the line
  spectrum, divided by its own maximum, and the f32 maximum is stored in the
  first two uint16 of the file (README.md "The grid", model_fetchers.rs:53-63).
* An observed star is the noiseless model at its labels, broadened by
  rotation (the limb-darkened profile of convolve_rv.rs:438-475) and a
  Gaussian instrument profile.  It is then Doppler shifted, resampled to
  log-uniform observed pixels, multiplied by a seeded quadratic response and
  given Gaussian noise at the requested SNR.  This is computed directly from
  the line list in float64 with numpy.  It shares no code with the product.

Wavelength grids are log-uniform over 4000-5000 A.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np

C_KMS = 299792.0  # the speed of light used by the reference (convolve_rv.rs:440)


@dataclasses.dataclass
class GridSpec:
    teffs: np.ndarray
    ms: np.ndarray
    loggs: np.ndarray
    n_px: int
    wl_lo: float = 4000.0
    wl_hi: float = 5000.0
    n_lines: int = 400
    includes_factor: bool = False
    seed: int = 0
    # optional staircase: per teff index, (lo, hi) logg index limits
    logg_limits: Optional[list] = None

    @property
    def log_first(self) -> float:
        return float(np.log10(self.wl_lo))

    @property
    def log_step(self) -> float:
        return float((np.log10(self.wl_hi) - np.log10(self.wl_lo)) / (self.n_px - 1))

    def wl(self) -> np.ndarray:
        return 10.0 ** (self.log_first + self.log_step * np.arange(self.n_px))


def config0_grid(n_px: int = 20000, seed: int = 0) -> GridSpec:
    """9 x 11 x 5 = 495 models (Teff 6000-8000 step 250, [M/H] -0.5..0.5, logg 3.5-4.5)."""
    return GridSpec(
        teffs=np.arange(6000.0, 8001.0, 250.0),
        ms=np.round(np.arange(-0.5, 0.5001, 0.1), 2),
        loggs=np.arange(3.5, 4.501, 0.25),
        n_px=n_px, seed=seed)


def config1_grid(n_px: int = 80000, seed: int = 1) -> GridSpec:
    """60 (nonuniform) x 21 x 11 = 13,860 models: Teff 4000-30000, [M/H] -1..0.5, logg 2.5-5."""
    teffs = np.round(4000.0 * (30000.0 / 4000.0) ** (np.arange(60) / 59.0) / 10.0) * 10.0
    return GridSpec(
        teffs=teffs,
        ms=np.round(np.linspace(-1.0, 0.5, 21), 2),
        loggs=np.arange(2.5, 5.001, 0.25),
        n_px=n_px, seed=seed)


def config4_grid(n_px: int = 120000, seed: int = 4) -> GridSpec:
    """80 x 26 x 13 = 27,040 models with a blackbody continuum (includes_factor)."""
    teffs = np.round(4000.0 * (30000.0 / 4000.0) ** (np.arange(80) / 79.0) / 10.0) * 10.0
    return GridSpec(
        teffs=teffs,
        ms=np.round(np.arange(-2.0, 0.5001, 0.1), 2),
        loggs=np.arange(2.0, 5.001, 0.25),
        n_px=n_px, includes_factor=True, seed=seed)


def _norm(v, lo, hi):
    return (v - lo) / (hi - lo) if hi > lo else np.zeros_like(v)


class LineModel:
    """The continuous line-list model the grid is sampled from."""

    def __init__(self, spec: GridSpec):
        rng = np.random.default_rng(spec.seed)
        n = spec.n_lines
        self.spec = spec
        self.centre = rng.uniform(spec.wl_lo, spec.wl_hi, n)
        self.width = rng.uniform(0.05, 0.3, n)
        self.a0 = rng.uniform(0.05, 0.55, n)
        self.coef = rng.uniform(-0.25, 0.25, (n, 3))
        self.tlim = (float(spec.teffs.min()), float(spec.teffs.max()))
        self.mlim = (float(spec.ms.min()), float(spec.ms.max()))
        self.glim = (float(spec.loggs.min()), float(spec.loggs.max()))

    def depths(self, labels: np.ndarray) -> np.ndarray:
        """labels [k, 3] (teff, m, logg) -> depths [k, n_lines], linear then clipped to 0-0.8."""
        lab = np.atleast_2d(labels)
        x = np.stack([_norm(lab[:, 0], *self.tlim), _norm(lab[:, 1], *self.mlim),
                      _norm(lab[:, 2], *self.glim)], axis=1)
        d = self.a0[None, :] + x @ self.coef.T
        return np.clip(d, 0.0, 0.8)

    def profiles(self, wl: np.ndarray, dtype=np.float64) -> np.ndarray:
        """[n_lines, len(wl)] Gaussian line profiles (peak 1)."""
        out = np.zeros((len(self.centre), len(wl)), dtype=dtype)
        for i, (c, w) in enumerate(zip(self.centre, self.width)):
            lo, hi = np.searchsorted(wl, [c - 7 * w, c + 7 * w])
            out[i, lo:hi] = np.exp(-0.5 * ((wl[lo:hi] - c) / w) ** 2)
        return out

    def flux(self, labels: np.ndarray, wl: np.ndarray, profiles=None) -> np.ndarray:
        """Normalised flux [k, len(wl)] in float64, clipped at 0."""
        if profiles is None:
            profiles = self.profiles(wl)
        f = 1.0 - self.depths(labels) @ profiles
        return np.clip(f, 0.0, None)


HC_K = 1.4387769e8  # h c / k in Angstrom K
# Planck's wavelength dependence of a 5772 K blackbody at 5000 A: the unit of
# blackbody(), so that grid maxima and flux ratios are of order one
BB_REF = 1.0 / (5000.0 ** 5 * np.expm1(HC_K / (5000.0 * 5772.0)))


def blackbody(wl_a: np.ndarray, teff: float) -> np.ndarray:
    """Planck B_lambda(T) relative to a 5772 K blackbody at 5000 A, wavelengths in Angstrom."""
    x = HC_K / (wl_a * teff)
    return 1.0 / (wl_a ** 5 * np.expm1(x)) / BB_REF


def gridpoints(spec: GridSpec) -> np.ndarray:
    """All (teff, m, logg) models, honouring an optional staircase."""
    pts = []
    for i, t in enumerate(spec.teffs):
        lo, hi = (0, len(spec.loggs) - 1) if spec.logg_limits is None else spec.logg_limits[i]
        for lg in spec.loggs[lo:hi + 1]:
            for m in spec.ms:
                pts.append((t, m, lg))
    return np.array(pts, dtype=np.float64)


def make_grid(spec: GridSpec, batch: int = 512):
    """Returns (labels [n,3] f64, spectra [n, n_px] u16, factors [n] f32 or None)."""
    labels = gridpoints(spec)
    wl = spec.wl()
    lm = LineModel(spec)
    prof = lm.profiles(wl, dtype=np.float32)
    n = len(labels)
    spectra = np.empty((n, spec.n_px), dtype=np.uint16)
    factors = np.empty(n, dtype=np.float32) if spec.includes_factor else None
    for s in range(0, n, batch):
        lab = labels[s:s + batch]
        f = 1.0 - lm.depths(lab).astype(np.float32) @ prof
        np.clip(f, 0.0, None, out=f)
        if spec.includes_factor:
            bb = np.stack([blackbody(wl, t) for t in lab[:, 0]]).astype(np.float32)
            f = f * bb
            mx = f.max(axis=1).astype(np.float32)
            factors[s:s + batch] = mx
            f = f / mx[:, None]
        spectra[s:s + batch] = np.clip(np.rint(f * 65535.0), 0, 65535).astype(np.uint16)
    return labels, spectra, factors


def filename_from_labels(teff: float, m: float, logg: float) -> str:
    """model_fetchers.rs:39-46 naming: l{m|p}MMMM_TTTTT_GGGG.npy"""
    t = int(round(teff))
    mm = int(round(m * 100.0))
    g = int(round(logg * 100.0))
    return "l%s%04d_%05d_%04d.npy" % ("m" if mm < 0 else "p", abs(mm), t, g)


def write_grid_dir(directory: str, labels, spectra, factors=None) -> None:
    """Write one .npy per model, with the f32 maximum prefix when factors is given."""
    os.makedirs(directory, exist_ok=True)
    for i, (t, m, g) in enumerate(labels):
        arr = spectra[i]
        if factors is not None:
            pre = np.frombuffer(np.float32(factors[i]).tobytes(), dtype=np.uint16)
            arr = np.concatenate([pre, arr])
        np.save(os.path.join(directory, filename_from_labels(t, m, g)), arr)


# ------------------------------------------------------------------- stars
def rotation_profile(vsini: float, dvelo: float) -> np.ndarray:
    """Limb-darkened rotation profile (epsilon 0.6) sampled like convolve_rv.rs:438-475, in float64."""
    eps = 0.6
    vrot = vsini / C_KMS
    n = max(1, int(np.ceil(2.0 * vrot / dvelo * np.sqrt(1.0 + (4.0 * (eps - 1.0) / (np.pi * eps)) ** 2))) + 2)
    n = n + 1 - n % 2
    v = np.arange(n) * dvelo
    v -= v[-1] / 2.0
    y = 1.0 - (v / vrot) ** 2
    k = np.where(y > 0, (2 * (1 - eps) * np.sqrt(np.clip(y, 0, None)) + np.pi * eps / 2 * y)
                 / (np.pi * vrot * (1 - eps / 3)), 0.0)
    return k / k.sum()


def _fft_convolve_same(x: np.ndarray, k: np.ndarray) -> np.ndarray:
    n = len(x) + len(k) - 1
    nf = 1 << int(np.ceil(np.log2(n)))
    y = np.fft.irfft(np.fft.rfft(x, nf) * np.fft.rfft(k, nf), nf)[:n]
    h = (len(k) - 1) // 2
    return y[h:h + len(x)]


@dataclasses.dataclass
class Star:
    wl: np.ndarray        # observed wavelengths (f64)
    flux: np.ndarray      # f32
    var: np.ndarray       # f32
    label: np.ndarray     # true (teff, m, logg, vsini, rv)
    snr: float


def observed_window(spec: GridSpec, rv_max: float, vsini_max: float, resolution: float,
                    extra_px: int = 128):
    """Observed wavelength range that stays clear of the grid edges for any |RV| <= rv_max."""
    dv = np.log(10.0) * spec.log_step * C_KMS  # km/s per synth pixel
    hw_rot = len(rotation_profile(vsini_max, np.log(10.0) * spec.log_step)) // 2 if vsini_max > 0 else 0
    sig = 1.0 / (np.log(10.0) * 2.355 * resolution * spec.log_step) if resolution > 0 else 0.0
    hw_g = int(np.ceil(6 * sig)) // 2 + 1
    shift_px = int(np.ceil(rv_max / dv)) + 2
    margin = hw_rot + hw_g + shift_px + extra_px
    wl = spec.wl()
    return float(wl[margin]), float(wl[spec.n_px - 1 - margin - spec.n_px % 128])


def _broadened(spec: GridSpec, label, resolution: float, lm: "LineModel", profiles=None) -> np.ndarray:
    """Noiseless model at label on the synthetic grid, rotated and broadened."""
    wl = spec.wl()
    f = lm.flux(np.asarray(label[:3])[None, :], wl, profiles)[0]
    if spec.includes_factor:
        f = f * blackbody(wl, label[0])
        f = f / f.max()
    dvelo = np.log(10.0) * spec.log_step
    if label[3] > 0:
        f = _fft_convolve_same(f, rotation_profile(label[3], dvelo))
    if resolution > 0:
        sig = 1.0 / (np.log(10.0) * 2.355 * resolution * spec.log_step)
        n = int(np.ceil(6 * sig))
        n = n + 1 - n % 2
        x = np.arange(n) - (n - 1) / 2
        g = np.exp(-0.5 * (x / sig) ** 2)
        f = _fft_convolve_same(f, g / g.sum())
    return f


def make_star(spec: GridSpec, label, n_obs: int, snr: float, resolution: float, seed: int,
              rv_max: float = 150.0, vsini_max: float = 300.0, lm: Optional[LineModel] = None,
              profiles=None) -> Star:
    """Noisy observed spectrum for label = (teff, m, logg, vsini, rv)."""
    rng = np.random.default_rng(seed)
    lm = lm or LineModel(spec)
    wl = spec.wl()
    f = _broadened(spec, label, resolution, lm, profiles)
    lo, hi = observed_window(spec, rv_max, vsini_max, resolution)
    wl_obs = np.geomspace(lo, hi, n_obs)
    src = wl_obs * (1.0 - label[4] / C_KMS)
    model = np.interp(np.log10(src), np.log10(wl), f)
    x = np.linspace(-1.0, 1.0, n_obs)
    a1, a2 = rng.uniform(-0.2, 0.2, 2)
    signal = model * (1.0 + a1 * x + a2 * x * x)
    sigma = np.abs(signal) / snr + 1e-6
    flux = signal + sigma * rng.standard_normal(n_obs)
    return Star(wl_obs, flux.astype(np.float32), (sigma ** 2).astype(np.float32),
                np.asarray(label, dtype=np.float64), snr)


def random_labels(spec: GridSpec, n: int, seed: int, vsini=(0.0, 300.0), rv=(-150.0, 150.0),
                  inset: float = 0.02) -> np.ndarray:
    """Seeded labels uniform inside the grid (a small inset keeps them off the edges)."""
    rng = np.random.default_rng(seed)

    def u(lo, hi):
        w = hi - lo
        return rng.uniform(lo + inset * w, hi - inset * w, n)

    return np.stack([u(spec.teffs.min(), spec.teffs.max()), u(spec.ms.min(), spec.ms.max()),
                     u(spec.loggs.min(), spec.loggs.max()), rng.uniform(*vsini, n),
                     rng.uniform(*rv, n)], axis=1)


def legendre_design(wl: np.ndarray, k: int) -> np.ndarray:
    """n x k Legendre design matrix on wl mapped to [-1, 1] (config-4 linear continuum model)."""
    x = (wl - wl[0]) / (wl[-1] - wl[0]) * 2.0 - 1.0
    return np.polynomial.legendre.legvander(x, k - 1).astype(np.float32)


def make_stars(spec: GridSpec, labels: np.ndarray, n_obs, snr, resolution: float, seed: int,
               rv_max: float = 150.0, vsini_max: float = 300.0, chunk: int = 32) -> list:
    """Vectorised make_star for many stars (same physics, batched FFTs)."""
    labels = np.asarray(labels, dtype=np.float64)
    n_stars = len(labels)
    n_obs = np.broadcast_to(np.asarray(n_obs), (n_stars,))
    snr = np.broadcast_to(np.asarray(snr, dtype=np.float64), (n_stars,))
    lm = LineModel(spec)
    wl = spec.wl()
    prof = lm.profiles(wl, dtype=np.float32)
    dvelo = np.log(10.0) * spec.log_step
    lo, hi = observed_window(spec, rv_max, vsini_max, resolution)
    npx = spec.n_px
    nf = 1 << int(np.ceil(np.log2(npx + 4096)))
    if resolution > 0:
        sig = 1.0 / (np.log(10.0) * 2.355 * resolution * spec.log_step)
        n = int(np.ceil(6 * sig))
        n = n + 1 - n % 2
        x = np.arange(n) - (n - 1) / 2
        g = np.exp(-0.5 * (x / sig) ** 2)
        g /= g.sum()
        G = np.fft.rfft(np.roll(np.pad(g, (0, nf - n)), -((n - 1) // 2)))
    else:
        G = None
    out = []
    for s0 in range(0, n_stars, chunk):
        lab = labels[s0:s0 + chunk]
        f = 1.0 - (lm.depths(lab[:, :3]).astype(np.float32) @ prof).astype(np.float64)
        np.clip(f, 0.0, None, out=f)
        if spec.includes_factor:
            bb = np.stack([blackbody(wl, t) for t in lab[:, 0]])
            f = f * bb
            f = f / f.max(axis=1, keepdims=True)
        F = np.fft.rfft(f, nf, axis=1)
        for k in range(len(lab)):
            if lab[k, 3] > 0:
                kk = rotation_profile(lab[k, 3], dvelo)
                m = len(kk)
                F[k] *= np.fft.rfft(np.roll(np.pad(kk, (0, nf - m)), -((m - 1) // 2)))
        if G is not None:
            F *= G[None, :]
        conv = np.fft.irfft(F, nf, axis=1)[:, :npx]
        for k in range(len(lab)):
            i = s0 + k
            rng = np.random.default_rng([seed, i])
            wl_obs = np.geomspace(lo, hi, int(n_obs[i]))
            src = wl_obs * (1.0 - lab[k, 4] / C_KMS)
            model = np.interp(np.log10(src), np.log10(wl), conv[k])
            xx = np.linspace(-1.0, 1.0, len(wl_obs))
            a1, a2 = rng.uniform(-0.2, 0.2, 2)
            signal = model * (1.0 + a1 * xx + a2 * xx * xx)
            sigma = np.abs(signal) / snr[i] + 1e-6
            flux = signal + sigma * rng.standard_normal(len(wl_obs))
            out.append(Star(wl_obs, flux.astype(np.float32), (sigma ** 2).astype(np.float32), lab[k].copy(),
                            float(snr[i])))
    return out


# ------------------------------------------------------------------ binaries
def continuum_shape(wl: np.ndarray, teff: float, m: float, logg: float) -> np.ndarray:
    """Unnormalised continuum of a model: the blackbody at Teff relative to a
    5772 K blackbody at 5000 A, scaled smoothly with [M/H] and logg."""
    return blackbody(wl, teff) * (1.0 + 0.05 * m + 0.02 * (logg - 4.0))


def make_continuum_grid(spec: GridSpec):
    """Grid of unnormalised continua on the axes and wavelengths of spec,
    stored like an includes_factor grid (u16 of flux / max, f32 max per
    model).  Returns (labels, spectra, maxima)."""
    labels = gridpoints(spec)
    wl = spec.wl()
    n = len(labels)
    spectra = np.empty((n, spec.n_px), dtype=np.uint16)
    maxima = np.empty(n, dtype=np.float32)
    for i, (t, m, g) in enumerate(labels):
        f = continuum_shape(wl, t, m, g).astype(np.float32)
        mx = np.float32(f.max())
        maxima[i] = mx
        spectra[i] = np.clip(np.rint(f / mx * 65535.0), 0, 65535).astype(np.uint16)
    return labels, spectra, maxima


def make_binary_star(spec: GridSpec, label1, label2, light_ratio: float, n_obs: int, snr: float,
                     resolution: float, seed: int, rv_max: float = 150.0, vsini_max: float = 300.0) -> Star:
    """Noisy normalised spectrum of a binary: each star's broadened model
    weighted by its continuum, (n1 c1 + lr n2 c2) / (c1 + lr c2) with
    lr = light_ratio mean(c1) / mean(c2), each star shifted by its own RV."""
    rng = np.random.default_rng(seed)
    lm = LineModel(spec)
    wl = spec.wl()
    n1 = _broadened(spec, label1, resolution, lm)
    n2 = _broadened(spec, label2, resolution, lm)
    c1 = continuum_shape(wl, *label1[:3])
    c2 = continuum_shape(wl, *label2[:3])
    lr = light_ratio * c1.mean() / c2.mean()
    lo, hi = observed_window(spec, rv_max, vsini_max, resolution)
    wl_obs = np.geomspace(lo, hi, n_obs)

    def at(arr, rv):
        return np.interp(np.log10(wl_obs * (1.0 - rv / C_KMS)), np.log10(wl), arr)

    a1, k1, a2, k2 = at(n1, label1[4]), at(c1, label1[4]), at(n2, label2[4]), at(c2, label2[4])
    model = (a1 * k1 + lr * a2 * k2) / (k1 + lr * k2)
    x = np.linspace(-1.0, 1.0, n_obs)
    b1, b2 = rng.uniform(-0.2, 0.2, 2)
    signal = model * (1.0 + b1 * x + b2 * x * x)
    sigma = np.abs(signal) / snr + 1e-6
    flux = signal + sigma * rng.standard_normal(n_obs)
    lab = np.concatenate([np.asarray(label1, np.float64), np.asarray(label2, np.float64), [light_ratio]])
    return Star(wl_obs, flux.astype(np.float32), (sigma ** 2).astype(np.float32), lab, snr)
