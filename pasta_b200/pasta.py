"""Drop-in replacement for PASTA's PyO3 module ``pasta`` (src/lib.rs:1971-1993).

Same class and function names, arguments, defaults and error behaviour as the
reference for the single-star path.  Every compute call goes through
libpasta_b200.so (include/pasta_b200.h) to the sm_100a kernels; the grid is
uploaded to HBM once when an interpolator is constructed.

Usage::

    import pasta_b200.pasta as pasta
    interp = pasta.InMemInterpolator(grid_dir, False, pasta.WlGrid(np.log10(4000), 2e-6, 76145, log=True))
    fitter = interp.get_fitter(pasta.FixedResolutionDispersion(wl, 85000, wl_grid),
                               pasta.ChunkContinuumFitter(wl), pasta.PSOSettings(40, 100), (0, 300), (-150, 150))
    result = fitter.fit(interp, flux, var)

Differences that are intrinsic to a GPU build are documented on each method;
the random draws of the particle swarm come from a seeded counter-based
stream (``seed=`` keyword, random when omitted, like StdRng::from_entropy).
"""
from __future__ import annotations

import ctypes as C
import glob
import io
import json
import os
import tarfile
from typing import Optional, Sequence

import numpy as np

from . import _ffi
from ._ffi import check, f32, f64, lib, ptr

__all__ = [
    "WlGrid", "PSOSettings", "Label", "OptimizationResult", "NoConvolutionDispersion",
    "FixedResolutionDispersion", "VariableResolutionDispersion", "ChunkContinuumFitter",
    "LinearModelContinuumFitter", "FixedContinuum", "ConstantContinuum", "FixConstraint",
    "RangeConstraint", "get_vsini_kernel", "InMemInterpolator", "OnDiskInterpolator",
    "CachedInterpolator", "PyWavelengthDispersion", "PyContinuumFitter", "SingleFitter",
    "Server", "PastaError", "LabelUncertainties", "BinaryFitter", "BinaryOptimizationResult",
]

PastaError = _ffi.PastaError
C_KMS = 299792.0


# ------------------------------------------------------------------ values
class WlGrid:
    """lib.rs:632-653.  log=True: (log10 of first wavelength, log10 step, length)."""

    def __init__(self, min: float, step: float, len: int, log: Optional[bool] = None):
        self.kind = _ffi.WL_LOGSPACE if log else _ffi.WL_LINSPACE
        self.a, self.b, self.n = float(min), float(step), int(len)
        self.values = None

    @staticmethod
    def non_uniform(wl) -> "WlGrid":
        g = WlGrid(0.0, 0.0, 0)
        g.kind = _ffi.WL_NONUNIFORM
        g.values = f64(wl)
        g.n = len(g.values)
        return g

    def get_array(self) -> list:
        if self.kind == _ffi.WL_LINSPACE:
            return [self.a + self.b * i for i in range(self.n)]
        if self.kind == _ffi.WL_LOGSPACE:
            return list(10.0 ** (self.a + self.b * np.arange(self.n, dtype=np.float64)))
        return list(self.values)

    def _c(self):
        return self.kind, self.a, self.b, self.n, self.values


class PSOSettings:
    """lib.rs:42-72."""

    def __init__(self, num_particles: int, max_iters: int, inertia_factor: Optional[float] = None,
                 cognitive_factor: Optional[float] = None, social_factor: Optional[float] = None,
                 delta: Optional[float] = None):
        self.num_particles = int(num_particles)
        self.max_iters = int(max_iters)
        self.inertia_factor = 0.7213475204 if inertia_factor is None else float(inertia_factor)
        self.cognitive_factor = 1.1931471806 if cognitive_factor is None else float(cognitive_factor)
        self.social_factor = 1.1931471806 if social_factor is None else float(social_factor)
        self.delta = 1e-7 if delta is None else float(delta)


class Label:
    """lib.rs:81-166."""

    __slots__ = ("teff", "m", "logg", "vsini", "rv")

    def __init__(self, teff, m, logg, vsini, rv):
        self.teff, self.m, self.logg, self.vsini, self.rv = map(float, (teff, m, logg, vsini, rv))

    def as_list(self):
        return [self.teff, self.m, self.logg, self.vsini, self.rv]

    def to_dict(self):
        return dict(teff=self.teff, m=self.m, logg=self.logg, vsini=self.vsini, rv=self.rv)

    @staticmethod
    def from_dict(d):
        return Label(d["teff"], d["m"], d["logg"], d["vsini"], d["rv"])

    def __repr__(self):
        return "Label(teff=%g, m=%g, logg=%g, vsini=%g, rv=%g)" % tuple(self.as_list())


class LabelUncertainties:
    """lib.rs:168-210: per label the (below, above) distances of the chi2
    landscape crossing; None where the search failed."""

    __slots__ = ("teff", "m", "logg", "vsini", "rv")

    def __init__(self, teff, m, logg, vsini, rv):
        self.teff, self.m, self.logg, self.vsini, self.rv = teff, m, logg, vsini, rv

    def to_dict(self):
        return dict(teff=self.teff, m=self.m, logg=self.logg, vsini=self.vsini, rv=self.rv)

    def to_json(self):
        return json.dumps({k: list(v) for k, v in self.to_dict().items()}, separators=(",", ":"))

    def __repr__(self):
        return "LabelUncertainties(%s)" % ", ".join("%s=%r" % kv for kv in self.to_dict().items())


class OptimizationResult:
    """lib.rs:212-294."""

    def __init__(self, label: Label, continuum_params, chi2: float, iterations: int, time: float):
        self.label = label
        self.continuum_params = [float(x) for x in continuum_params]
        self.chi2 = float(chi2)
        self.iterations = int(iterations)
        self.time = float(time)

    def to_dict(self):
        return dict(label=self.label.to_dict(), continuum_params=list(self.continuum_params), chi2=self.chi2,
                    iterations=self.iterations, time=self.time)

    def to_json(self):
        return json.dumps(self.to_dict(), separators=(",", ":"))

    @staticmethod
    def from_dict(d):
        return OptimizationResult(Label.from_dict(d["label"]), d["continuum_params"], d["chi2"], d["iterations"],
                                  d["time"])


class BinaryOptimizationResult:
    """lib.rs:296-360."""

    def __init__(self, label1: Label, label2: Label, light_ratio: float, continuum_params, chi2: float,
                 iterations: int, time: float):
        self.label1 = label1
        self.label2 = label2
        self.light_ratio = float(light_ratio)
        self.continuum_params = [float(x) for x in continuum_params]
        self.chi2 = float(chi2)
        self.iterations = int(iterations)
        self.time = float(time)

    def to_dict(self):
        return dict(label1=self.label1.to_dict(), label2=self.label2.to_dict(), light_ratio=self.light_ratio,
                    continuum_params=list(self.continuum_params), chi2=self.chi2, iterations=self.iterations,
                    time=self.time)

    def to_json(self):
        return json.dumps(self.to_dict(), separators=(",", ":"))

    @staticmethod
    def from_dict(d):
        return BinaryOptimizationResult(Label.from_dict(d["label1"]), Label.from_dict(d["label2"]),
                                        d["light_ratio"], d["continuum_params"], d["chi2"], d["iterations"],
                                        d["time"])


# ------------------------------------------------------------ dispersions
class PyWavelengthDispersion:
    """lib.rs:664-756: wraps one of the dispersion kinds, resident on the device."""

    def __init__(self, kind, wl, synth_wl: WlGrid, resolution=0.0, disp=None):
        self.kind = kind
        self.wl = f64(wl)
        self.synth_wl = synth_wl
        k, a, b, n, vals = synth_wl._c()
        h = C.c_void_p()
        dd = None if disp is None else f32(disp)
        check(lib().pasta_dispersion_create(k, a, b, n, ptr(vals), kind, ptr(self.wl), len(self.wl),
                                            float(resolution), ptr(dd), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _ffi._lib is not None:
            lib().pasta_dispersion_destroy(h)

    def convolve(self, flux) -> np.ndarray:
        """Instrument broadening of a synthetic spectrum (lib.rs:671-680)."""
        x = f32(flux)
        out = np.empty_like(x)
        check(lib().pasta_dispersion_convolve(self._h, ptr(x), len(x), ptr(out)))
        return out

    def wavelength(self) -> list:
        return list(self.wl)

    def convolve_and_resample_spectra(self, spectra, input_wavelength: WlGrid) -> np.ndarray:
        """Instrument broadening and resampling at RV 0 to this dispersion's
        wavelengths of many dequantised grid spectra at once (M x n_synth -> M x n_obs)."""
        x = np.ascontiguousarray(np.atleast_2d(spectra), dtype=np.float32)
        out = np.empty((x.shape[0], len(self.wl)), np.float32)
        k, a, b, n, _ = input_wavelength._c()
        check(lib().pasta_dispersion_convolve_resample(self._h, k, a, b, x.shape[1], ptr(x), x.shape[0], ptr(out)))
        return out

    def convolve_and_resample_directory(self, input_directory: str, output_directory: str, includes_factor: bool,
                                        input_wavelength: WlGrid, batch: int = 256) -> None:
        """Pre-convolve a grid directory (lib.rs:686-755): every model file is
        convolved with this dispersion and resampled to its wavelengths, then
        written under the same name, requantised to uint16 (with the f32
        maximum prefix when includes_factor).  Existing outputs are kept.
        The arithmetic runs on the GPU, ``batch`` files per launch."""
        files = sorted(os.listdir(input_directory))
        todo = [f for f in files if not os.path.exists(os.path.join(output_directory, f))]
        for i0 in range(0, len(todo), batch):
            names = todo[i0:i0 + batch]
            rows, facs = [], []
            for name in names:
                arr = np.load(os.path.join(input_directory, name))
                u, mx = _split_factor(arr, includes_factor)
                x = u.astype(np.float32) / np.float32(65535.0)
                if includes_factor:
                    x = x * np.float32(mx)
                rows.append(x)
            res = self.convolve_and_resample_spectra(np.stack(rows), input_wavelength)
            for name, r in zip(names, res):
                if includes_factor:
                    mx = np.float32(r.max())
                    q = _as_u16(np.maximum(r, np.float32(0.0)) / mx * np.float32(65535.0))
                    out = np.concatenate([np.frombuffer(mx.astype("<f4").tobytes(), dtype="<u2"), q])
                else:
                    out = _as_u16(np.clip(r, np.float32(0.0), np.float32(1.0)) * np.float32(65535.0))
                np.save(os.path.join(output_directory, name), out.astype(np.uint16))

    def kernels(self) -> np.ndarray:
        w = C.c_int64()
        check(lib().pasta_dispersion_kernels(self._h, C.byref(w), None))
        if self.kind == _ffi.DISP_NONE or w.value == 0:
            return np.zeros((0, 0), np.float32)
        if self.kind == _ffi.DISP_FIXED and self.synth_wl.kind == _ffi.WL_LOGSPACE:
            out = np.empty(w.value, np.float32)
        else:
            out = np.empty((w.value, self.synth_wl.n), np.float32)
        check(lib().pasta_dispersion_kernels(self._h, C.byref(w), ptr(out)))
        return out


def NoConvolutionDispersion(wl, wl_grid: WlGrid) -> PyWavelengthDispersion:
    """lib.rs:791-797."""
    return PyWavelengthDispersion(_ffi.DISP_NONE, wl, wl_grid)


def FixedResolutionDispersion(wl, resolution: float, synth_wl: WlGrid) -> PyWavelengthDispersion:
    """lib.rs:773-789."""
    return PyWavelengthDispersion(_ffi.DISP_FIXED, wl, synth_wl, resolution=resolution)


def VariableResolutionDispersion(wl, disp, synth_wl: WlGrid) -> PyWavelengthDispersion:
    """lib.rs:758-771.  ``disp`` is used as a Gaussian sigma in Angstrom per
    observed pixel, as the reference computes it (convolve_rv.rs:363)."""
    return PyWavelengthDispersion(_ffi.DISP_VARIABLE, wl, synth_wl, disp=disp)


# -------------------------------------------------------------- continuum
class PyContinuumFitter:
    """lib.rs:853-940."""

    def __init__(self, kind, wl=None, n_chunks=5, p_order=8, overlap=0.2, design=None, continuum=None,
                 ignore=0):
        self.kind = kind
        self.wl = None if wl is None else f64(wl)
        self.design = None if design is None else f32(design)
        self.continuum = None if continuum is None else f32(continuum)
        if kind == _ffi.CONT_CHUNK:
            n = len(self.wl)
        elif kind == _ffi.CONT_LINEAR:
            n = self.design.shape[0]
        elif kind == _ffi.CONT_FIXED:
            n = len(self.continuum)
        else:
            n = 0
        self.n = n
        k = 0 if self.design is None else self.design.shape[1]
        h = C.c_void_p()
        check(lib().pasta_continuum_create(kind, ptr(self.wl), n, int(n_chunks), int(p_order), float(overlap),
                                           ptr(self.design), k, ptr(self.continuum), int(ignore), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _ffi._lib is not None:
            lib().pasta_continuum_destroy(h)

    def nparams(self) -> int:
        return lib().pasta_continuum_nparams(self._h)

    def _fit(self, model, observed, observed_var):
        m, y, v = f32(model), f32(observed), f32(observed_var)
        if len(y) != len(v):
            raise ValueError("Flux and variance vectors must have the same length")
        params = np.empty(max(self.nparams(), 1), np.float32)
        chi2 = C.c_double()
        check(lib().pasta_continuum_fit(self._h, ptr(m), ptr(y), ptr(v), len(y), ptr(params), C.byref(chi2)))
        return params, chi2.value

    def fit_continuum(self, model, observed, observed_var):
        """Fit observed/model; returns (params, chi2) (lib.rs:862-874)."""
        return self._fit(model, observed, observed_var)

    def fit_and_return_chi2(self, synth, y, yerr) -> float:
        return self._fit(synth, y, yerr)[1]

    def build_continuum(self, params) -> np.ndarray:
        p = f32(params)
        n = 1 if self.kind == _ffi.CONT_CONSTANT else self.n
        out = np.empty(n, np.float32)
        check(lib().pasta_continuum_build(self._h, ptr(p), len(p), ptr(out)))
        return out

    def fit_and_return_continuum(self, synth, observed, observed_var) -> np.ndarray:
        params, _ = self._fit(synth, observed, observed_var)
        return self.build_continuum(params)

    def fit_continuum_and_return_normalized_spec(self, synth, observed, observed_var) -> np.ndarray:
        cont = self.fit_and_return_continuum(synth, observed, observed_var)
        y = f32(observed)
        if len(cont) != len(y):
            raise ValueError("continuum and observed spectrum have different lengths")
        return y / cont


def ChunkContinuumFitter(wl, n_chunks: Optional[int] = None, p_order: Optional[int] = None,
                         overlap: Optional[float] = None) -> PyContinuumFitter:
    """lib.rs:942-960 (defaults 5 chunks, order 8, overlap 0.2)."""
    return PyContinuumFitter(_ffi.CONT_CHUNK, wl=wl, n_chunks=5 if n_chunks is None else n_chunks,
                             p_order=8 if p_order is None else p_order, overlap=0.2 if overlap is None else overlap)


def LinearModelContinuumFitter(design_matrix) -> PyContinuumFitter:
    """lib.rs:962-966."""
    d = np.asarray(design_matrix, dtype=np.float32)
    if d.ndim != 2:
        raise ValueError("design_matrix must be 2-D")
    return PyContinuumFitter(_ffi.CONT_LINEAR, design=d)


def FixedContinuum(continuum, ignore_first_and_last: Optional[int] = None) -> PyContinuumFitter:
    """lib.rs:968-977."""
    return PyContinuumFitter(_ffi.CONT_FIXED, continuum=continuum,
                             ignore=0 if ignore_first_and_last is None else ignore_first_and_last)


def ConstantContinuum() -> PyContinuumFitter:
    """lib.rs:979-983."""
    return PyContinuumFitter(_ffi.CONT_CONSTANT)


class _Constraint:
    def __init__(self, parameter, kind, a, b):
        self.parameter, self.kind, self.a, self.b = int(parameter), kind, float(a), float(b)


def FixConstraint(parameter: int, value: float) -> _Constraint:
    """lib.rs:814-823."""
    return _Constraint(parameter, 1, value, value)


def RangeConstraint(parameter: int, lower: float, upper: float) -> _Constraint:
    """lib.rs:825-835."""
    return _Constraint(parameter, 2, lower, upper)


def get_vsini_kernel(vsini: float, synth_wl: WlGrid) -> list:
    """Rotation kernel (lib.rs:1962-1969, convolve_rv.rs:438-475): f64 values
    cast to f32 and normalised by their f32 sum."""
    if synth_wl.kind != _ffi.WL_LOGSPACE:
        raise ValueError("Only logspace is supported")
    dvelo = np.log(10.0) * synth_wl.b
    eps = 0.6
    vrot = vsini / C_KMS
    n = max(1, int(np.ceil(2.0 * vrot / dvelo * np.sqrt(1.0 + (4.0 * (eps - 1.0) / (np.pi * eps)) ** 2.0))) + 2)
    n = n + 1 - n % 2
    velo = np.arange(n, dtype=np.float64) * dvelo
    velo = velo - velo[-1] / 2.0
    k = np.zeros(n, np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = velo / vrot
        y = 1.0 - r * r
    for i in range(n):
        if y[i] > 0.0:
            k[i] = np.float32((2.0 * (1.0 - eps) * np.sqrt(y[i]) + np.pi * eps / 2.0 * y[i])
                              / (np.pi * vrot * (1.0 - eps / 3.0)))
    s = np.float32(0.0)
    for v in k:
        s = np.float32(s + v)
    return list((k / s).astype(np.float32))


def _settings_c(settings: PSOSettings, vsini_range, rv_range, constraints) -> _ffi.PsoSettingsC:
    st = _ffi.PsoSettingsC()
    st.num_particles, st.max_iters = settings.num_particles, settings.max_iters
    st.inertia_factor, st.cognitive_factor = settings.inertia_factor, settings.cognitive_factor
    st.social_factor, st.delta = settings.social_factor, settings.delta
    st.vsini_lo, st.vsini_hi = map(float, vsini_range)
    st.rv_lo, st.rv_hi = map(float, rv_range)
    for c in constraints or ():
        if not 0 <= c.parameter < 5:
            raise IndexError("constraint parameter index out of range")
        st.ckind[c.parameter], st.ca[c.parameter], st.cb[c.parameter] = c.kind, c.a, c.b
    return st


def _seed(seed):
    if seed is None:
        return int.from_bytes(os.urandom(8), "little")
    return int(seed) & 0xFFFFFFFFFFFFFFFF


# ------------------------------------------------------------ interpolators
def _label_from_filename(filename: str):
    """model_fetchers.rs:23-38."""
    parts = filename.split(".")[0].split("_")
    if len(parts) != 3 or len(parts[0]) != 6 or len(parts[1]) != 5 or len(parts[2]) != 4:
        raise ValueError("Invalid filename: %s" % filename)
    sign = -1.0 if parts[0].startswith("lm") else 1.0
    return float(parts[1]), sign * float(parts[0][2:]) / 100.0, float(parts[2]) / 100.0


def _as_u16(x: np.ndarray) -> np.ndarray:
    """Rust's `f32 as u16`: truncation toward zero, saturating at 0 and 65535, NaN -> 0."""
    x = np.nan_to_num(np.asarray(x, np.float32), nan=0.0, posinf=65535.0, neginf=0.0)
    return np.trunc(np.clip(x, 0.0, 65535.0)).astype(np.uint16)


def _split_factor(arr: np.ndarray, includes_factor: bool):
    """model_fetchers.rs:48-67: the first two uint16 hold the f32 maximum."""
    arr = np.asarray(arr, dtype=np.uint16)
    if includes_factor:
        mx = np.frombuffer(arr[:2].tobytes(), dtype="<f4")[0]
        if mx < 0:
            raise ValueError("Negative factor: %g" % mx)
        return arr[2:], np.float32(mx)
    return arr, None


class _Grid:
    """Resident grid handle (pasta_grid_create)."""

    def __init__(self, labels, spectra, maxima, wavelength: WlGrid):
        labels = f64(labels)
        spectra = np.ascontiguousarray(spectra, dtype=np.uint16)
        mx = None if maxima is None else f32(maxima)
        if wavelength.n != spectra.shape[1]:
            raise ValueError("Length of model and wavelength grid don't match. model: %d, synth_wl: %d"
                             % (spectra.shape[1], wavelength.n))
        k, a, b, n, vals = wavelength._c()
        h = C.c_void_p()
        check(lib().pasta_grid_create(ptr(labels), ptr(spectra), ptr(mx), len(labels), spectra.shape[1], k, a, b,
                                      ptr(vals), C.byref(h)))
        self._h = h
        self.wl = wavelength
        shape = np.zeros(5, np.int64)
        check(lib().pasta_grid_shape(h, ptr(shape)))
        self.nt, self.nm, self.nl, self.npx, self.nmodels = map(int, shape)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _ffi._lib is not None:
            lib().pasta_grid_destroy(h)


class _Interpolator:
    """Methods shared by the interpolator classes (lib.rs:987-1466)."""

    _grid: _Grid

    # ---- construction helpers
    def _init_arrays(self, labels, spectra, maxima, wavelength: WlGrid):
        self._grid = _Grid(labels, spectra, maxima, wavelength)
        self.synth_wl = wavelength

    def _init_dir(self, dir: str, includes_factor: bool, wavelength: WlGrid):
        if not os.path.isdir(dir):
            raise FileNotFoundError("Not found %r" % dir)
        names = sorted(os.listdir(dir))
        labels = [_label_from_filename(n) for n in names]
        specs, maxima = [], []
        for n in names:
            s, mx = _split_factor(np.load(os.path.join(dir, n)), includes_factor)
            specs.append(s)
            maxima.append(mx)
        if not specs:
            raise ValueError("empty grid directory %r" % dir)
        self._init_arrays(np.array(labels), np.stack(specs), np.array(maxima, np.float32) if includes_factor else None,
                          wavelength)

    # ---- model production
    def _labels(self, labels, ncols):
        lab = f64(np.atleast_2d(np.asarray(labels, dtype=np.float64)))
        if lab.shape[1] != ncols:
            raise ValueError("labels must have %d columns" % ncols)
        return lab

    def _produce(self, dispersion: PyWavelengthDispersion, lab) -> tuple:
        out = np.empty((len(lab), len(dispersion.wl)), np.float32)
        st = np.zeros(len(lab), np.int32)
        check(lib().pasta_produce_model(self._grid._h, dispersion._h, ptr(lab), len(lab), ptr(out), ptr(st)))
        return out, st

    @staticmethod
    def _raise_status(st, what="model production"):
        bad = np.nonzero(st)[0]
        if len(bad):
            raise PastaError(int(st[bad[0]]), "%s failed for label %d (status %d)" % (what, bad[0], st[bad[0]]))

    def produce_model(self, dispersion, teff, m, logg, vsini, rv) -> np.ndarray:
        """interpolate -> rotation -> instrument -> RV shift + resample (lib.rs:993-1011)."""
        out, st = self._produce(dispersion, self._labels([teff, m, logg, vsini, rv], 5))
        self._raise_status(st)
        return out[0]

    def produce_model_bulk(self, dispersion, labels, progress: Optional[bool] = None) -> np.ndarray:
        """All labels in one batched device pass (lib.rs:1064-1089)."""
        out, st = self._produce(dispersion, self._labels(labels, 5))
        self._raise_status(st)
        return out

    def produce_model_on_grid(self, dispersion, teff, mh, logg, vsini, rv) -> np.ndarray:
        """Model straight from a grid node (lib.rs:1093-1107).  The reference
        scales the node spectrum by 1/65535 twice (interpolate.rs:1129); the
        same scale is applied here."""
        t = self._snap(0, teff, self.teffs())
        m = self._snap(1, mh, self.ms())
        g = self._snap(2, logg, self.loggs())
        return self.produce_model(dispersion, t, m, g, vsini, rv) / np.float32(65535.0)

    @staticmethod
    def _snap(axis, x, values):
        values = np.asarray(values)
        i = int(np.argmin(np.abs(values - x)))
        if abs(values[i] - x) >= 0.001:
            raise PastaError(-10, ["Teff", "m", "logg"][axis] + " not in grid")
        return float(values[i])

    def interpolate(self, teff, m, logg) -> np.ndarray:
        """Cubic interpolation only (lib.rs:1111-1123)."""
        lab = self._labels([teff, m, logg], 3)
        out = np.empty((1, self._grid.npx), np.float32)
        st = np.zeros(1, np.int32)
        check(lib().pasta_interpolate(self._grid._h, ptr(lab), 1, ptr(out), ptr(st)))
        self._raise_status(st, "interpolation")
        return out[0]

    def interpolate_bulk(self, labels) -> np.ndarray:
        lab = self._labels(labels, 3)
        out = np.empty((len(lab), self._grid.npx), np.float32)
        st = np.zeros(len(lab), np.int32)
        check(lib().pasta_interpolate(self._grid._h, ptr(lab), len(lab), ptr(out), ptr(st)))
        self._raise_status(st, "interpolation")
        return out

    def interpolate_and_convolve(self, dispersion, teff, m, logg, vsini) -> np.ndarray:
        """Interpolation + rotation + instrument broadening (lib.rs:1141-1157)."""
        lab = self._labels([teff, m, logg, vsini], 4)
        out = np.empty((1, self._grid.npx), np.float32)
        st = np.zeros(1, np.int32)
        check(lib().pasta_interpolate_and_convolve(self._grid._h, dispersion._h, ptr(lab), 1, ptr(out), ptr(st)))
        self._raise_status(st)
        return out[0]

    @property
    def direct_max(self) -> int:
        """Widest combined broadening kernel (rotation taps + 2 x instrument
        half width) convolved directly instead of by FFT blocks; measured on
        this device when the grid was loaded (no counterpart in the reference)."""
        v = C.c_int32()
        check(lib().pasta_grid_direct_max(self._grid._h, C.byref(v)))
        return int(v.value)

    @direct_max.setter
    def direct_max(self, taps: int):
        check(lib().pasta_grid_set_direct_max(self._grid._h, int(taps)))

    @property
    def tc_min(self) -> int:
        """Members from which a group of one star's evaluations sharing their 64
        neighbour rows is interpolated on the tensor cores (65: never); measured
        on this device when the grid was loaded (no counterpart in the reference)."""
        v = C.c_int32()
        check(lib().pasta_grid_tc_min(self._grid._h, C.byref(v)))
        return int(v.value)

    @tc_min.setter
    def tc_min(self, members: int):
        check(lib().pasta_grid_set_tc_min(self._grid._h, int(members)))

    def interpolate_linear(self, teff, m, logg) -> np.ndarray:
        """Trilinear interpolation over the 8 surrounding models
        (interpolate.rs:985-1028; lib.rs:1127-1139)."""
        lab = self._labels([teff, m, logg], 3)
        out = np.empty((1, self._grid.npx), np.float32)
        st = np.zeros(1, np.int32)
        check(lib().pasta_interpolate_linear(self._grid._h, ptr(lab), 1, ptr(out), ptr(st)))
        self._raise_status(st, "linear interpolation")
        return out[0]

    def produce_binary_model_norm(self, continuum_interpolator, dispersion, labels1, labels2,
                                  light_ratio: float) -> np.ndarray:
        """Normalised model of a binary (lib.rs:1013-1041): each star's
        normalised model weighted by its continuum from the continuum
        interpolator (a grid of unnormalised models), light ratio
        light_ratio * mean(c1) / mean(c2) (interpolate.rs:822-893)."""
        lab = f64(np.concatenate([np.asarray(labels1, np.float64).reshape(5),
                                  np.asarray(labels2, np.float64).reshape(5), [float(light_ratio)]])[None, :])
        out = np.empty((1, len(dispersion.wl)), np.float32)
        st = np.zeros(1, np.int32)
        check(lib().pasta_binary_model(self._grid._h, continuum_interpolator._grid._h, dispersion._h, ptr(lab), 1,
                                       ptr(out), ptr(st)))
        self._raise_status(st, "binary model production")
        return out[0]

    def get_binary_fitter(self, dispersion, continuum_fitter, settings: PSOSettings, vsini_range,
                          rv_range) -> "BinaryFitter":
        """lib.rs:1177-1193."""
        return BinaryFitter(dispersion, continuum_fitter, settings, vsini_range, rv_range)

    def get_kernels(self, wl, disp) -> np.ndarray:
        """Variable-resolution kernels, width x n_synth (lib.rs:1043-1060)."""
        return VariableResolutionDispersion(wl, disp, self.synth_wl).kernels()

    # ---- fitting
    def get_fitter(self, dispersion, continuum_fitter, settings: PSOSettings, vsini_range, rv_range) -> "SingleFitter":
        """lib.rs:1159-1175."""
        return SingleFitter(dispersion, continuum_fitter, settings, vsini_range, rv_range)

    def fit_continuum(self, fitter: PyContinuumFitter, dispersion, observed_flux, observed_var, label) -> np.ndarray:
        """Continuum of observed vs model at label (lib.rs:1234-1261).  Like the
        reference, label[2] (logg) is passed as vsini (lib.rs:1249)."""
        lab = list(map(float, label))
        synth = self.produce_model(dispersion, lab[0], lab[1], lab[2], lab[2], lab[4])
        return fitter.fit_and_return_continuum(synth, observed_flux, observed_var)

    def fit_continuum_and_return_model(self, fitter: PyContinuumFitter, dispersion, observed_flux, observed_var,
                                       label) -> np.ndarray:
        """Continuum x model at label (lib.rs:1266-1293)."""
        lab = list(map(float, label))
        synth = self.produce_model(dispersion, *lab)
        cont = fitter.fit_and_return_continuum(synth, observed_flux, observed_var)
        if len(cont) != len(synth):
            raise ValueError("continuum and model have different lengths")
        return cont * synth

    def chi2_bulk(self, observed_wavelength, observed_flux, observed_var, labels, progress=None,
                  allow_nan=None) -> list:
        """Chi2 of many spectra, each with its own wavelengths, a pre-convolved
        grid and a 5 x 8 x 0.2 chunk fitter (lib.rs:1297-1338), all in one
        batched device pass (pasta_chi2_many)."""
        wls = [f64(w) for w in observed_wavelength]
        fl = [f32(x) for x in observed_flux]
        vr = [f32(x) for x in observed_var]
        S = len(wls)
        if not (len(fl) == len(vr) == S == len(labels)):
            raise ValueError("wavelengths, fluxes, variances and labels must have the same count")
        for w, f, v in zip(wls, fl, vr):
            if not (len(w) == len(f) == len(v)):
                raise ValueError("Flux and variance vectors must have the same length")
        if S == 0:
            return []
        disps = [NoConvolutionDispersion(w, self.synth_wl) for w in wls]
        conts = [ChunkContinuumFitter(w, 5, 8, 0.2) for w in wls]
        lab = f64(np.asarray(labels, dtype=np.float64).reshape(S, 5))
        out = np.empty(S)
        st = np.zeros(S, np.int32)
        Pp = C.c_void_p
        dh = (Pp * S)(*[d._h.value for d in disps])
        ch = (Pp * S)(*[c._h.value for c in conts])
        fp = (Pp * S)(*[x.ctypes.data for x in fl])
        vp = (Pp * S)(*[x.ctypes.data for x in vr])
        n = np.array([len(x) for x in fl], np.int64)
        check(lib().pasta_chi2_many(self._grid._h, S, dh, ch, fp, vp, ptr(n), ptr(lab), ptr(out), ptr(st)))
        if not allow_nan:
            self._raise_status(st, "chi2")
        return [float(x) for x in out]

    def ccf(self, vs, teff, m, logg, dispersion, observed_flux) -> np.ndarray:
        """Cross-correlation of the unbroadened model with the flux (lib.rs:1340-1371)."""
        flux = f32(observed_flux)
        if len(dispersion.wl) != len(flux):
            raise ValueError("Dispersion and observed flux must have the same length.")
        nd = NoConvolutionDispersion(dispersion.wl, self.synth_wl)
        v = np.ascontiguousarray(vs, np.float64).reshape(-1)
        out = np.empty(len(v), np.float32)
        st = np.zeros(len(v), np.int32)
        # the shifted models stay on the device; their dot products with the flux are summed there
        check(lib().pasta_ccf(self._grid._h, nd._h, ptr(v), len(v), float(teff), float(m), float(logg), ptr(flux),
                              len(flux), ptr(out), ptr(st)))
        self._raise_status(st)
        return out

    # ---- grid getters (lib.rs:1373-1465)
    def clamp_1d(self, teff, m, logg, index) -> float:
        out = C.c_double()
        check(lib().pasta_grid_clamp_1d(self._grid._h, teff, m, logg, int(index), C.byref(out)))
        return out.value

    def _coeffs(self, teff, m, logg):
        cols = np.zeros(64, np.int64)
        w = np.zeros(64, np.float32)
        t16, l16, m4 = np.zeros(16), np.zeros(16), np.zeros(4)
        check(lib().pasta_grid_coefficients(self._grid._h, teff, m, logg, ptr(cols), ptr(w), ptr(t16), ptr(l16),
                                            ptr(m4)))
        return cols, w, t16.reshape(4, 4), l16.reshape(4, 4), m4

    def calculate_interpolation_coefficients_flat(self, teff, m, logg):
        """(teff factors [logg row][teff col], logg factors, m factors) (lib.rs:1388-1397)."""
        _, _, t, l, mm = self._coeffs(teff, m, logg)
        # nalgebra matrices convert to nested lists column by column
        return t.T.tolist(), l.T.tolist(), mm.tolist()

    def calculate_interpolation_coefficients(self, teff, m, logg) -> list:
        return self._coeffs(teff, m, logg)[1].tolist()

    def get_neighbor_indices(self, teff, m, logg) -> list:
        """(teff, m, logg) indices of the 64 neighbours, (0, 0, 0) if missing (lib.rs:1414-1433)."""
        cols = self._coeffs(teff, m, logg)[0]
        pts = self._colmap()
        return [pts[c] if c >= 0 else (0, 0, 0) for c in cols]

    def _colmap(self):
        if getattr(self, "_cm", None) is None:
            lo, hi = self._limits()
            cm = []
            for i in range(self._grid.nt):
                for k in range(lo[i], hi[i] + 1):
                    for j in range(self._grid.nm):
                        cm.append((i, j, k))
            self._cm = cm
        return self._cm

    def _axis(self, a, n):
        v = np.zeros(n)
        check(lib().pasta_grid_axis(self._grid._h, a, ptr(v)))
        return v

    def teffs(self) -> list:
        return list(self._axis(0, self._grid.nt))

    def ms(self) -> list:
        return list(self._axis(1, self._grid.nm))

    def loggs(self) -> list:
        return list(self._axis(2, self._grid.nl))

    def _limits(self):
        lo, hi = np.zeros(self._grid.nt, np.int64), np.zeros(self._grid.nt, np.int64)
        check(lib().pasta_grid_logg_limits(self._grid._h, ptr(lo), ptr(hi)))
        return lo, hi

    def logg_limits(self) -> list:
        lo, hi = self._limits()
        return [(int(a), int(b)) for a, b in zip(lo, hi)]

    def cumulative_grid_size(self) -> list:
        v = np.zeros(self._grid.nt, np.int64)
        check(lib().pasta_grid_cumulative_size(self._grid._h, ptr(v)))
        return [int(x) for x in v]

    def list_gridpoints(self) -> list:
        t, m, g = self.teffs(), self.ms(), self.loggs()
        return [[t[i], m[j], g[k]] for (i, j, k) in self._colmap()]

    def is_teff_logg_between_bounds(self, teff, logg) -> bool:
        out = C.c_int()
        check(lib().pasta_grid_is_teff_logg_between_bounds(self._grid._h, teff, logg, C.byref(out)))
        return bool(out.value)


ZSTD_MAGIC = b"\x28\xb5\x2f\xfd"


def _tar_bytes(file_path: str) -> bytes:
    """The tar archive inside a .tar.zst file (model_fetchers.rs:168-180).  A
    zstd frame is decoded by the zstandard module or the zstd program; a
    file that is not zstd-compressed is read as a plain tar archive."""
    raw = open(file_path, "rb").read()
    if raw[:4] != ZSTD_MAGIC:
        return raw
    try:
        import zstandard  # type: ignore
        return zstandard.ZstdDecompressor().decompress(raw, max_output_size=1 << 40)
    except ImportError:
        pass
    import shutil
    import subprocess
    exe = shutil.which("zstd") or shutil.which("unzstd")
    if exe is None:
        raise RuntimeError("%s is zstd-compressed, and neither the 'zstandard' Python module nor a zstd program is "
                           "available to decode it; decompress it to a plain .tar (which from_tar_zstd also reads) "
                           "or install one of them" % file_path)
    return subprocess.run([exe, "-dc", file_path], check=True, capture_output=True).stdout


def _read_tar_models(file_path: str, includes_factor: bool):
    """(labels, spectra, maxima or None) of the archive's grid models."""
    labels, specs, maxima = [], [], []
    with tarfile.open(fileobj=io.BytesIO(_tar_bytes(file_path))) as tf:
        for mem in tf.getmembers():
            name = os.path.basename(mem.name)
            if not mem.isfile() or not name.startswith("l"):
                continue
            labels.append(_label_from_filename(name))
            sp, mx = _split_factor(np.load(io.BytesIO(tf.extractfile(mem).read())), includes_factor)
            specs.append(sp)
            maxima.append(mx)
    if not specs:
        raise ValueError("no grid models in %r" % file_path)
    return np.array(labels), np.stack(specs), np.array(maxima, np.float32) if includes_factor else None


class InMemInterpolator(_Interpolator):
    """lib.rs:1881-1908: the whole grid resident in HBM."""

    def __init__(self, dir: str, includes_factor: bool, wavelength: WlGrid):
        self._init_dir(dir, includes_factor, wavelength)

    @staticmethod
    def from_tar_zstd(file_path: str, includes_factor: bool, wavelength: WlGrid) -> "InMemInterpolator":
        """model_fetchers.rs:168-226: members starting with 'l' are grid models."""
        labels, specs, maxima = _read_tar_models(file_path, includes_factor)
        self = InMemInterpolator.__new__(InMemInterpolator)
        self._init_arrays(labels, specs, maxima, wavelength)
        return self

    @staticmethod
    def from_arrays(labels, spectra, maxima, wavelength: WlGrid) -> "InMemInterpolator":
        """Grid from in-memory arrays: labels n x (teff, m, logg), spectra n x npx uint16,
        maxima (includes_factor) or None."""
        self = InMemInterpolator.__new__(InMemInterpolator)
        self._init_arrays(labels, spectra, maxima, wavelength)
        return self


class OnDiskInterpolator(_Interpolator):
    """lib.rs:1867-1879.  The GPU build keeps the grid resident, so this loads it into HBM once."""

    def __init__(self, dir: str, includes_factor: bool, wavelength: WlGrid):
        self._init_dir(dir, includes_factor, wavelength)


class CachedInterpolator(_Interpolator):
    """lib.rs:1909-1935.  Loads the whole grid into HBM; lrucap/n_shards are accepted for API compatibility."""

    def __init__(self, dir: str, includes_factor: bool, wavelength: WlGrid, lrucap: Optional[int] = None,
                 n_shards: Optional[int] = None):
        self._init_dir(dir, includes_factor, wavelength)
        self.lrucap = 4000 if lrucap is None else int(lrucap)
        self.n_shards = 4 if n_shards is None else int(n_shards)

    def cache_size(self) -> int:
        return self._grid.nmodels


# ------------------------------------------------------------------- fitter
class SingleFitter:
    """InMemSingleFitter / OnDiskSingleFitter / CachedSingleFitter (lib.rs:1468-1628)."""

    def __init__(self, dispersion, continuum_fitter, settings: PSOSettings, vsini_range, rv_range):
        self.dispersion = dispersion
        self.continuum_fitter = continuum_fitter
        self.settings = settings
        self.vsini_range = tuple(map(float, vsini_range))
        self.rv_range = tuple(map(float, rv_range))

    def _st(self, constraints):
        return _settings_c(self.settings, self.vsini_range, self.rv_range, constraints)

    def _run(self, interpolator, fluxes, vars_, constraints, seeds, mode, trace=False):
        fl = f32(np.atleast_2d(fluxes))
        vr = f32(np.atleast_2d(vars_))
        if fl.shape != vr.shape:
            raise ValueError("Flux and variance vectors must have the same length")
        S, n = fl.shape
        if n != len(self.dispersion.wl):
            raise PastaError(-1, "Observed spectrum and target dispersion must have the same length")
        st = self._st(constraints)
        res = (_ffi.FitResultC * S)()
        npar = self.continuum_fitter.nparams()
        params = np.zeros((S, max(npar, 1)), np.float32)
        seeds = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64))
        tr = np.zeros((st.max_iters + 1, st.num_particles, 6)) if trace else None
        check(lib().pasta_fit(interpolator._grid._h, self.dispersion._h, self.continuum_fitter._h, C.byref(st),
                              ptr(fl), ptr(vr), n, S, ptr(seeds), mode, res, ptr(params), ptr(tr)))
        return res, params, tr

    @staticmethod
    def _result(r, params) -> OptimizationResult:
        if r.status:
            raise PastaError(int(r.status), "fit failed (status %d)" % r.status)
        return OptimizationResult(Label(*r.label), params[:r.n_params], r.chi2, r.iterations, r.time)

    def fit(self, interpolator, observed_flux, observed_var, trace_directory: Optional[str] = None,
            best_particle_file: Optional[str] = None, parallelize: Optional[bool] = None, constraints=None,
            seed: Optional[int] = None, mode: int = _ffi.FIT_BATCHED) -> OptimizationResult:
        """PSO fit of one star (lib.rs:1478-1507).  ``parallelize`` is accepted for
        API compatibility (the device always evaluates all particles at once)."""
        if trace_directory is not None and best_particle_file is not None:
            raise RuntimeError("Cannot specify both trace_directory and best_particle_file")
        want_trace = trace_directory is not None or best_particle_file is not None
        res, params, tr = self._run(interpolator, observed_flux, observed_var, constraints, [_seed(seed)], mode,
                                    trace=want_trace)
        out = self._result(res[0], params[0])
        if want_trace:
            _write_trace(tr, trace_directory, best_particle_file)
        return out

    def fit_bulk(self, interpolator, observed_fluxes, observed_vars, constraints=None, seeds=None,
                 mode: int = _ffi.FIT_BATCHED) -> list:
        """All stars in one batched device run (lib.rs:1511-1540)."""
        S = len(observed_fluxes)
        seeds = [_seed(None) for _ in range(S)] if seeds is None else list(seeds)
        res, params, _ = self._run(interpolator, observed_fluxes, observed_vars, constraints, seeds, mode)
        return [self._result(res[i], params[i]) for i in range(S)]

    def chi2(self, interpolator, observed_flux, observed_var, labels, allow_nan: Optional[bool] = None) -> list:
        """Chi2 at fixed labels with the continuum fitted (lib.rs:1603-1627);
        failures give NaN unless allow_nan is False."""
        fl, vr = f32(observed_flux), f32(observed_var)
        if len(fl) != len(vr):
            raise ValueError("Flux and variance vectors must have the same length")
        lab = f64(np.atleast_2d(np.asarray(labels, dtype=np.float64)))
        out = np.empty(len(lab))
        st = np.zeros(len(lab), np.int32)
        check(lib().pasta_chi2(interpolator._grid._h, self.dispersion._h, self.continuum_fitter._h, ptr(fl),
                               ptr(vr), len(fl), ptr(lab), len(lab), ptr(out), ptr(st)))
        if allow_nan is False:
            _Interpolator._raise_status(st, "chi2")
        return [float(x) for x in out]


    def compute_uncertainty(self, interpolator, observed_flux, observed_var, spec_res: float, label,
                            search_radius=None) -> LabelUncertainties:
        """Chi2-landscape uncertainties at a best-fit label (lib.rs:1545-1566,
        fitting.rs:480-568); raises when chi2 at the label itself fails."""
        return self.compute_uncertainty_bulk(interpolator, [observed_flux], [observed_var], spec_res, [label],
                                             search_radius)[0]

    def compute_uncertainty_bulk(self, interpolator, observed_fluxes, observed_vars, spec_res: float, labels,
                                 search_radius=None) -> list:
        """compute_uncertainty for many spectra of this fitter's wavelength
        grid (lib.rs:1570-1600); every search of every spectrum shares one
        batched chi2 evaluation per Brent step."""
        fl = np.ascontiguousarray(np.stack([f32(x) for x in observed_fluxes]), dtype=np.float32)
        vr = np.ascontiguousarray(np.stack([f32(x) for x in observed_vars]), dtype=np.float32)
        if fl.shape != vr.shape:
            raise ValueError("Flux and variance vectors must have the same length")
        S, n = fl.shape
        lab = f64(np.asarray(labels, dtype=np.float64).reshape(S, 5))
        sr = None if search_radius is None else f64(np.asarray(search_radius, dtype=np.float64).reshape(5))
        out = np.empty((S, 5, 2))
        bst = np.zeros((S, 5, 2), np.int32)
        sst = np.zeros(S, np.int32)
        check(lib().pasta_compute_uncertainty(interpolator._grid._h, self.dispersion._h, self.continuum_fitter._h,
                                              S, ptr(fl), ptr(vr), n, float(spec_res), ptr(lab),
                                              ptr(sr) if sr is not None else None, ptr(out), ptr(bst), ptr(sst)))
        _Interpolator._raise_status(sst, "compute_uncertainty")
        res = []
        for i in range(S):
            pairs = [tuple(None if bst[i, k, j] else float(out[i, k, j]) for j in range(2)) for k in range(5)]
            res.append(LabelUncertainties(*pairs))
        return res


class BinaryFitter:
    """InMemBinaryFitter / OnDiskBinaryFitter / CachedBinaryFitter
    (lib.rs:1630-1699; fitting.rs:571-717): 11 parameters, star 1
    (teff, m, logg, vsini, rv), star 2 (the same) and the light ratio."""

    def __init__(self, dispersion, continuum_fitter, settings: PSOSettings, vsini_range, rv_range):
        self.dispersion = dispersion
        self.continuum_fitter = continuum_fitter
        self.settings = settings
        self.vsini_range = tuple(map(float, vsini_range))
        self.rv_range = tuple(map(float, rv_range))

    def _st(self, constraints) -> _ffi.BinarySettingsC:
        st = _ffi.BinarySettingsC()
        s = self.settings
        st.num_particles, st.max_iters = s.num_particles, s.max_iters
        st.inertia_factor, st.cognitive_factor = s.inertia_factor, s.cognitive_factor
        st.social_factor, st.delta = s.social_factor, s.delta
        st.vsini_lo, st.vsini_hi = self.vsini_range
        st.rv_lo, st.rv_hi = self.rv_range
        for c in constraints or ():
            if not 0 <= c.parameter < 11:
                raise IndexError("constraint parameter index out of range")
            st.ckind[c.parameter], st.ca[c.parameter], st.cb[c.parameter] = c.kind, c.a, c.b
        return st

    def fit(self, interpolator, continuum_interpolator, observed_flux, observed_var,
            trace_directory: Optional[str] = None, best_particle_file: Optional[str] = None,
            parallelize: Optional[bool] = None, constraints=None, seed: Optional[int] = None,
            _trace: bool = False) -> BinaryOptimizationResult:
        """PSO fit of a binary (lib.rs:1636-1671).  ``parallelize`` is accepted
        for API compatibility (every particle of an iteration is evaluated in
        one device batch)."""
        if trace_directory is not None and best_particle_file is not None:
            raise RuntimeError("Cannot specify both trace_directory and best_particle_file")
        fl, vr = f32(observed_flux), f32(observed_var)
        if fl.shape != vr.shape:
            raise ValueError("Flux and variance vectors must have the same length")
        if len(fl) != len(self.dispersion.wl):
            raise PastaError(-1, "Observed spectrum and target dispersion must have the same length")
        st = self._st(constraints)
        res = _ffi.BinaryResultC()
        params = np.zeros(max(self.continuum_fitter.nparams(), 1), np.float32)
        want_trace = _trace or trace_directory is not None or best_particle_file is not None
        tr = np.zeros((st.max_iters + 1, st.num_particles, 12)) if want_trace else None
        check(lib().pasta_binary_fit(interpolator._grid._h, continuum_interpolator._grid._h, self.dispersion._h,
                                     self.continuum_fitter._h, C.byref(st), ptr(fl), ptr(vr), len(fl),
                                     _seed(seed), C.byref(res), ptr(params), ptr(tr)))
        if res.status:
            raise PastaError(int(res.status), "binary fit failed (status %d)" % res.status)
        if trace_directory is not None or best_particle_file is not None:
            _write_trace(tr, trace_directory, best_particle_file)
        out = BinaryOptimizationResult(Label(*res.label1), Label(*res.label2), res.light_ratio,
                                       params[:res.n_params], res.chi2, res.iterations, res.time)
        if _trace:
            out._trace = tr
        return out

    def chi2(self, interpolator, continuum_interpolator, observed_flux, observed_var, labels,
             allow_nan: Optional[bool] = None) -> list:
        """Chi2 at fixed 11-parameter labels (lib.rs:1673-1698); failures give
        NaN unless allow_nan is False."""
        fl, vr = f32(observed_flux), f32(observed_var)
        if len(fl) != len(vr):
            raise ValueError("Flux and variance vectors must have the same length")
        lab = f64(np.atleast_2d(np.asarray(labels, dtype=np.float64)))
        if lab.shape[1] != 11:
            raise ValueError("binary labels have 11 columns")
        out = np.empty(len(lab))
        st = np.zeros(len(lab), np.int32)
        check(lib().pasta_binary_chi2(interpolator._grid._h, continuum_interpolator._grid._h, self.dispersion._h,
                                      self.continuum_fitter._h, ptr(fl), ptr(vr), len(fl), ptr(lab), len(lab),
                                      ptr(out), ptr(st)))
        if allow_nan is False:
            _Interpolator._raise_status(st, "chi2")
        return [float(x) for x in out]


def _write_trace(tr, trace_directory, best_particle_file):
    """PSOobserver / BestParticleObserver output (fitting.rs:217-296)."""
    if tr is None:
        return
    n_it = tr.shape[0] - 1
    if trace_directory is not None:
        os.makedirs(trace_directory, exist_ok=True)
        for it in range(n_it):
            vals = [{"position": list(map(float, p[:-1])), "cost": float(p[-1])} for p in tr[it + 1]]
            with open(os.path.join(trace_directory, "it_%d.json" % it), "w") as f:
                json.dump(vals, f, separators=(",", ":"))
    if best_particle_file is not None:
        best = tr[0][0]
        hist = []
        for it in range(n_it):
            for p in tr[it + 1]:
                if p[-1] < best[-1]:
                    best = p
            hist.append({"position": list(map(float, best[:-1])), "cost": float(best[-1])})
            with open(best_particle_file, "w") as f:
                json.dump(hist, f, separators=(",", ":"))


# ----------------------------------------------------- batched / served
def fit_many(interpolator, dispersions, continuum_fitters, settings, fluxes, vars_, vsini_range, rv_range,
             seeds=None, constraints=None, mode: int = _ffi.FIT_BATCHED) -> list:
    """Batched fit of stars with their own wavelength grids (ragged pixel counts)."""
    S = len(fluxes)
    sts = (_ffi.PsoSettingsC * S)()
    for i in range(S):
        s = settings[i] if isinstance(settings, (list, tuple)) else settings
        sts[i] = _settings_c(s, vsini_range, rv_range, constraints)
    fl = [f32(x) for x in fluxes]
    vr = [f32(x) for x in vars_]
    n = np.array([len(x) for x in fl], np.int64)
    seeds = np.asarray([_seed(None) for _ in range(S)] if seeds is None else seeds, np.uint64)
    P = C.c_void_p
    dh = (P * S)(*[d._h.value for d in dispersions])
    ch = (P * S)(*[c._h.value for c in continuum_fitters])
    fp = (P * S)(*[x.ctypes.data for x in fl])
    vp = (P * S)(*[x.ctypes.data for x in vr])
    params = [np.zeros(max(c.nparams(), 1), np.float32) for c in continuum_fitters]
    pp = (P * S)(*[p.ctypes.data for p in params])
    res = (_ffi.FitResultC * S)()
    check(lib().pasta_fit_many(interpolator._grid._h, S, dh, ch, sts, fp, vp, ptr(n), ptr(seeds), mode, res, pp))
    return [SingleFitter._result(res[i], params[i]) for i in range(S)]


class Server:
    """Continuous-batching fit service on one GPU (pasta_server_*)."""

    def __init__(self, interpolator, max_slots: int = 256, hbm_budget_bytes: int = 0):
        h = C.c_void_p()
        check(lib().pasta_server_create(interpolator._grid._h, int(max_slots), int(hbm_budget_bytes), C.byref(h)))
        self._h = h
        self._keep = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _ffi._lib is not None:
            lib().pasta_server_destroy(h)

    def submit(self, dispersion, continuum_fitter, settings: PSOSettings, flux, var, vsini_range, rv_range,
               seed=None, constraints=None) -> int:
        st = _settings_c(settings, vsini_range, rv_range, constraints)
        fl, vr = f32(flux), f32(var)
        rid = C.c_int64()
        check(lib().pasta_server_submit(self._h, dispersion._h, continuum_fitter._h, C.byref(st), ptr(fl), ptr(vr),
                                        len(fl), _seed(seed), C.byref(rid)))
        self._keep[rid.value] = (dispersion, continuum_fitter)
        return rid.value

    def step(self) -> int:
        return check(lib().pasta_server_step(self._h))

    def poll(self, max_results: int = 1024, max_params: int = 512):
        ids = np.zeros(max_results, np.int64)
        res = (_ffi.FitResultC * max_results)()
        params = np.zeros((max_results, max_params), np.float32)
        n = C.c_int()
        check(lib().pasta_server_poll(self._h, ptr(ids), res, ptr(params), max_params, max_results, C.byref(n)))
        out = []
        for i in range(n.value):
            r = res[i]
            self._keep.pop(int(ids[i]), None)
            out.append((int(ids[i]), int(r.status), OptimizationResult(Label(*r.label), params[i][:r.n_params],
                                                                        r.chi2, r.iterations, r.time)))
        return out

    def run(self, steps: int) -> float:
        """``steps`` steps back to back; returns the milliseconds between CUDA
        events around them on the library's stream."""
        ms = C.c_double()
        check(lib().pasta_server_run(self._h, int(steps), C.byref(ms)))
        return ms.value

    def stats(self) -> dict:
        out = np.zeros(7, np.int64)
        check(lib().pasta_server_stats(self._h, ptr(out)))
        return dict(zip(["evals", "steps", "particles_per_slot", "admit_us", "device_us", "retire_us", "refit_us"],
                        out.tolist()))

    def memory(self):
        """(HBM budget, bytes held by the running requests)."""
        b, u = C.c_int64(), C.c_int64()
        check(lib().pasta_server_memory(self._h, C.byref(b), C.byref(u)))
        return b.value, u.value

    def pending(self):
        q, a, d = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().pasta_server_pending(self._h, C.byref(q), C.byref(a), C.byref(d)))
        return q.value, a.value, d.value


class BatchFit:
    """Step-wise batched fit of many stars (pasta_batch_*): the object the
    benchmark times.  ``step(n)`` advances every swarm n PSO steps (the first
    step evaluates the initial swarm) and returns the device milliseconds."""

    def __init__(self, interpolator, dispersions, continuum_fitters, settings, fluxes, vars_, vsini_range, rv_range,
                 seeds=None, constraints=None):
        S = len(fluxes)
        self.S = S
        self._st = (_ffi.PsoSettingsC * S)()
        for i in range(S):
            s = settings[i] if isinstance(settings, (list, tuple)) else settings
            self._st[i] = _settings_c(s, vsini_range, rv_range, constraints)
        self._fl = [f32(x) for x in fluxes]
        self._vr = [f32(x) for x in vars_]
        n = np.array([len(x) for x in self._fl], np.int64)
        seeds = np.asarray([_seed(None) for _ in range(S)] if seeds is None else seeds, np.uint64)
        P = C.c_void_p
        self._keep = (dispersions, continuum_fitters, interpolator)
        dh = (P * S)(*[d._h.value for d in dispersions])
        ch = (P * S)(*[c._h.value for c in continuum_fitters])
        fp = (P * S)(*[x.ctypes.data for x in self._fl])
        vp = (P * S)(*[x.ctypes.data for x in self._vr])
        h = C.c_void_p()
        check(lib().pasta_batch_create(interpolator._grid._h, S, dh, ch, self._st, fp, vp, ptr(n), ptr(seeds),
                                       C.byref(h)))
        self._h = h
        self._nparams = [max(c.nparams(), 1) for c in continuum_fitters]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _ffi._lib is not None:
            lib().pasta_batch_destroy(h)

    def step(self, n: int = 1) -> float:
        ms = C.c_double()
        check(lib().pasta_batch_step(self._h, int(n), C.byref(ms)))
        return ms.value

    def profile_step(self) -> dict:
        out = np.zeros(12)
        check(lib().pasta_batch_profile_step(self._h, ptr(out)))
        names = ["update_ms", "prep_ms", "rotker_ms", "interp_ms", "broaden_ms", "direct_unfused_ms", "chi2_ms", "best_ms",
                 "interp_px", "evals", "obs_px", "broaden_blocks"]
        return dict(zip(names, out.tolist()))

    def info(self) -> dict:
        out = np.zeros(6, np.int64)
        check(lib().pasta_batch_info(self._h, ptr(out)))
        return dict(zip(["stars", "particles", "evals_per_step", "iterations", "steps_done", "kernels_per_step"],
                        out.tolist()))

    def finish(self) -> list:
        res = (_ffi.FitResultC * self.S)()
        params = [np.zeros(k, np.float32) for k in self._nparams]
        pp = (C.c_void_p * self.S)(*[p.ctypes.data for p in params])
        check(lib().pasta_batch_finish(self._h, res, pp))
        return [(int(res[i].status), OptimizationResult(Label(*res[i].label), params[i][:res[i].n_params],
                                                         res[i].chi2, res[i].iterations, res[i].time))
                for i in range(self.S)]
