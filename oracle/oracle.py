"""ctypes wrapper of the CPU oracle (liboracle): TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
The product (pasta_b200) never does.  Parity status: unpinned by reference
outputs (see pasta_oracle.h); pinned by analytic known-answer tests.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpasta_oracle.so")

F32, F64 = 0, 1
WL_LINSPACE, WL_LOGSPACE, WL_NONUNIFORM = 0, 1, 2
DISP_NONE, DISP_FIXED, DISP_VARIABLE = 0, 1, 2
CONT_CHUNK, CONT_LINEAR, CONT_FIXED, CONT_CONSTANT = 0, 1, 2, 3

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "pasta_oracle.cpp")):
        subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


class PsoSettings(C.Structure):
    _fields_ = [("num_particles", C.c_int), ("max_iters", C.c_int), ("inertia", C.c_double),
                ("cognitive", C.c_double), ("social", C.c_double), ("delta", C.c_double),
                ("vsini_lo", C.c_double), ("vsini_hi", C.c_double), ("rv_lo", C.c_double),
                ("rv_hi", C.c_double), ("ckind", C.c_int * 5), ("ca", C.c_double * 5),
                ("cb", C.c_double * 5)]


class FitResult(C.Structure):
    _fields_ = [("label", C.c_double * 5), ("chi2", C.c_double), ("iterations", C.c_int),
                ("status", C.c_int), ("n_params", C.c_int), ("params", C.c_double * 512)]


class BinarySettings(C.Structure):
    _fields_ = [("num_particles", C.c_int), ("max_iters", C.c_int), ("inertia", C.c_double),
                ("cognitive", C.c_double), ("social", C.c_double), ("delta", C.c_double),
                ("vsini_lo", C.c_double), ("vsini_hi", C.c_double), ("rv_lo", C.c_double),
                ("rv_hi", C.c_double), ("ckind", C.c_int * 11), ("ca", C.c_double * 11),
                ("cb", C.c_double * 11)]


class BinaryResult(C.Structure):
    _fields_ = [("label1", C.c_double * 5), ("label2", C.c_double * 5), ("light_ratio", C.c_double),
                ("chi2", C.c_double), ("iterations", C.c_int), ("status", C.c_int), ("n_params", C.c_int),
                ("params", C.c_double * 512)]


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        P, d, i64, i = C.c_void_p, C.c_double, C.c_int64, C.c_int
        sig = {
            "or_last_error": (C.c_char_p, []),
            "or_grid_create": (P, [P, P, P, i64, i64, i, d, d, P]),
            "or_grid_free": (None, [P]),
            "or_grid_axes": (i, [P, P, P, P]),
            "or_grid_axis_values": (i, [P, i, P]),
            "or_grid_logg_limits": (i, [P, P, P]),
            "or_local_grid": (i, [P, d, d, d, P, P]),
            "or_is_within_bounds": (i, [P, d, d, d]),
            "or_limits_at": (i, [P, P, i, P, P]),
            "or_interpolate": (i, [P, i, d, d, d, P]),
            "or_rotation_kernel": (i, [d, d, P, i]),
            "or_convolve_rotation": (i, [P, i, P, d, P]),
            "or_disp_create": (P, [P, i, P, i64, d, P]),
            "or_disp_free": (None, [P]),
            "or_disp_convolve": (i, [P, i, P, P]),
            "or_disp_kernel_width": (i, [P]),
            "or_produce_model": (i, [P, P, i, P, P]),
            "or_cont_create": (P, [i, P, i64, i, i, d, P, i, P, i]),
            "or_cont_free": (None, [P]),
            "or_cont_nparams": (i, [P]),
            "or_cont_chunk_bounds": (i, [P, P]),
            "or_fit_continuum": (i, [P, i, P, P, P, i64, P, P]),
            "or_build_continuum": (i, [P, i, P, P]),
            "or_chi2": (i, [P, P, P, i, P, P, i64, P, i64, P, P, i]),
            "or_fit": (i, [P, P, P, i, P, P, P, i64, i64, P, i, i, P, P]),
            "or_draw_u01": (d, [C.c_uint64] * 5),
            "or_local_grid_linear": (i, [P, d, d, d, P, P]),
            "or_interpolate_linear": (i, [P, i, d, d, d, P]),
            "or_binary_model": (i, [P, P, P, i, P, P]),
            "or_binary_chi2": (i, [P, P, P, P, i, P, P, i64, P, i64, P, P, i]),
            "or_binary_fit": (i, [P, P, P, P, i, P, P, P, i64, C.c_uint64, i, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


class OracleError(RuntimeError):
    pass


def _err():
    return OracleError(lib().or_last_error().decode())


def _p(a):
    return None if a is None else a.ctypes.data


class Grid:
    def __init__(self, labels, spectra, factors=None, wl_kind=WL_LOGSPACE, wl_a=0.0, wl_b=0.0,
                 wl_values=None):
        self.labels = np.ascontiguousarray(labels, dtype=np.float64)
        self.spectra = np.ascontiguousarray(spectra, dtype=np.uint16)
        self.factors = None if factors is None else np.ascontiguousarray(factors, dtype=np.float32)
        self.npx = self.spectra.shape[1]
        wv = None if wl_values is None else np.ascontiguousarray(wl_values, dtype=np.float64)
        self.h = lib().or_grid_create(_p(self.labels), _p(self.spectra), _p(self.factors),
                                      len(self.labels), self.npx, wl_kind, wl_a, wl_b, _p(wv))
        if not self.h:
            raise _err()
        self.wl_kind, self.wl_a, self.wl_b = wl_kind, wl_a, wl_b

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_grid_free(self.h)

    def axes(self):
        n = (C.c_int * 3)()
        lib().or_grid_axes(self.h, C.byref(n, 0), C.byref(n, 4), C.byref(n, 8))
        out = []
        for ax in range(3):
            v = np.zeros(n[ax])
            lib().or_grid_axis_values(self.h, ax, _p(v))
            out.append(v)
        return out

    def local_grid(self, t, m, g):
        cols = np.zeros(64, dtype=np.int64)
        w = np.zeros(64)
        if lib().or_local_grid(self.h, t, m, g, _p(cols), _p(w)):
            raise _err()
        return cols, w

    def interpolate(self, t, m, g, prec=F32):
        out = np.zeros(self.npx)
        if lib().or_interpolate(self.h, prec, t, m, g, _p(out)):
            raise _err()
        return out

    def local_grid_linear(self, t, m, g):
        cols = np.zeros(8, dtype=np.int64)
        w = np.zeros(8)
        if lib().or_local_grid_linear(self.h, t, m, g, _p(cols), _p(w)):
            raise _err()
        return cols, w

    def interpolate_linear(self, t, m, g, prec=F32):
        out = np.zeros(self.npx)
        if lib().or_interpolate_linear(self.h, prec, t, m, g, _p(out)):
            raise _err()
        return out

    def convolve_rotation(self, x, vsini, prec=F32):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(self.npx)
        if lib().or_convolve_rotation(self.h, prec, _p(x), vsini, _p(out)):
            raise _err()
        return out

    def within(self, t, m, g):
        return bool(lib().or_is_within_bounds(self.h, t, m, g))


def rotation_kernel(vsini, dvelo, cap=4096):
    out = np.zeros(cap)
    n = lib().or_rotation_kernel(vsini, dvelo, _p(out), cap)
    if n < 0:
        raise _err()
    return out[:n]


class Disp:
    def __init__(self, grid: Grid, kind, wl_obs, resolution=0.0, disp=None):
        self.grid = grid
        self.wl = np.ascontiguousarray(wl_obs, dtype=np.float64)
        dd = None if disp is None else np.ascontiguousarray(disp, dtype=np.float32)
        self.h = lib().or_disp_create(grid.h, kind, _p(self.wl), len(self.wl), float(resolution), _p(dd))
        if not self.h:
            raise _err()

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_disp_free(self.h)

    def convolve(self, x, prec=F32):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(self.grid.npx)
        if lib().or_disp_convolve(self.h, prec, _p(x), _p(out)):
            raise _err()
        return out

    def produce_model(self, label, prec=F32):
        lab = np.ascontiguousarray(label, dtype=np.float64)
        out = np.zeros(len(self.wl))
        if lib().or_produce_model(self.grid.h, self.h, prec, _p(lab), _p(out)):
            raise _err()
        return out


class Cont:
    def __init__(self, kind, wl=None, n_chunks=5, p_order=8, overlap=0.2, design=None,
                 continuum=None, ignore=0, n=None):
        self.wl = None if wl is None else np.ascontiguousarray(wl, dtype=np.float64)
        self.design = None if design is None else np.ascontiguousarray(design, dtype=np.float32)
        self.cont = None if continuum is None else np.ascontiguousarray(continuum, dtype=np.float32)
        if n is None:
            n = len(self.wl) if self.wl is not None else (
                self.design.shape[0] if self.design is not None else len(self.cont))
        self.n = n
        k = 0 if self.design is None else self.design.shape[1]
        self.h = lib().or_cont_create(kind, _p(self.wl), n, n_chunks, p_order, overlap,
                                      _p(self.design), k, _p(self.cont), ignore)
        if not self.h:
            raise _err()
        self.kind = kind

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_cont_free(self.h)

    def nparams(self):
        return lib().or_cont_nparams(self.h)

    def chunk_bounds(self):
        ss = np.zeros(2 * 64, dtype=np.int64)
        nc = lib().or_cont_chunk_bounds(self.h, _p(ss))
        return ss[:2 * nc].reshape(nc, 2)

    def fit(self, flux, var, model, prec=F32):
        flux = np.ascontiguousarray(flux, dtype=np.float32)
        var = np.ascontiguousarray(var, dtype=np.float32)
        model = np.ascontiguousarray(model, dtype=np.float64)
        params = np.zeros(max(self.nparams(), 1))
        chi2 = C.c_double()
        if lib().or_fit_continuum(self.h, prec, _p(flux), _p(var), _p(model), len(flux), _p(params),
                                  C.byref(chi2)):
            raise _err()
        return params, chi2.value

    def build(self, params, prec=F32):
        params = np.ascontiguousarray(params, dtype=np.float64)
        out = np.zeros(self.n)
        if lib().or_build_continuum(self.h, prec, _p(params), _p(out)):
            raise _err()
        return out


def chi2(grid, disp, cont, flux, var, labels, prec=F32, nthreads=0):
    flux = np.ascontiguousarray(flux, dtype=np.float32)
    var = np.ascontiguousarray(var, dtype=np.float32)
    labels = np.ascontiguousarray(np.atleast_2d(labels), dtype=np.float64)
    out = np.zeros(len(labels))
    st = np.zeros(len(labels), dtype=np.int32)
    nt = nthreads or os.cpu_count()
    if lib().or_chi2(grid.h, disp.h, cont.h, prec, _p(flux), _p(var), len(flux), _p(labels), len(labels),
                     _p(out), _p(st), nt):
        raise _err()
    return out, st


def settings(num_particles, max_iters, vsini_range, rv_range, inertia=0.7213475204,
             cognitive=1.1931471806, social=1.1931471806, delta=1e-7, constraints=()):
    s = PsoSettings()
    s.num_particles, s.max_iters = num_particles, max_iters
    s.inertia, s.cognitive, s.social, s.delta = inertia, cognitive, social, delta
    s.vsini_lo, s.vsini_hi = vsini_range
    s.rv_lo, s.rv_hi = rv_range
    for (idx, kind, a, b) in constraints:
        s.ckind[idx], s.ca[idx], s.cb[idx] = kind, a, b
    return s


def fit(grid, disp, cont, st, fluxes, vars_, seeds, prec=F32, nthreads=0, over_stars=True,
        trace=False):
    fluxes = np.ascontiguousarray(np.atleast_2d(fluxes), dtype=np.float32)
    vars_ = np.ascontiguousarray(np.atleast_2d(vars_), dtype=np.float32)
    S, n = fluxes.shape
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    res = (FitResult * S)()
    tr = np.zeros((st.max_iters + 1, st.num_particles, 6)) if trace else None
    nt = nthreads or os.cpu_count()
    rc = lib().or_fit(grid.h, disp.h, cont.h, prec, C.byref(st), _p(fluxes), _p(vars_), n, S, _p(seeds),
                      nt, 1 if over_stars else 0, res, _p(tr))
    out = []
    for r in res:
        out.append(dict(label=np.array(r.label[:]), chi2=r.chi2, iterations=r.iterations, status=r.status,
                        params=np.array(r.params[:r.n_params])))
    if trace:
        return out, rc, tr
    return out, rc


def draw_u01(seed, phase, a, b, c):
    return lib().or_draw_u01(seed, phase, a, b, c)


def limits_at(grid, tml, index):
    """Grid::get_limits_at (interpolate.rs:645-663) for index 0..2."""
    p = np.ascontiguousarray(tml[:3], dtype=np.float64)
    lo, hi = C.c_double(), C.c_double()
    if lib().or_limits_at(grid.h, _p(p), index, C.byref(lo), C.byref(hi)):
        raise _err()
    return lo.value, hi.value


def _brent(f, a, b, tol=1e-3, max_iter=500):
    """Brent's zero finder (Brent 1973, ch. 4; Numerical Recipes' zbrent) on
    [a, b]; f raises on a failed evaluation.  Returns the root estimate."""
    fa, fb = f(a), f(b)
    if fa * fb > 0:
        raise ValueError("f(min) and f(max) must have different signs")
    c, fc = b, fb
    d = e = b - a
    eps = np.finfo(np.float64).eps
    for _ in range(max_iter):
        if (fb > 0 and fc > 0) or (fb < 0 and fc < 0):
            c, fc = a, fa
            d = e = b - a
        if abs(fc) < abs(fb):
            a, b, c = b, c, b
            fa, fb, fc = fb, fc, fb
        tol1 = 2.0 * eps * abs(b) + 0.5 * tol
        xm = 0.5 * (c - b)
        if abs(xm) <= tol1 or fb == 0.0:
            return b
        if abs(e) >= tol1 and abs(fa) > abs(fb):
            s = fb / fa
            if a == c:
                p, q = 2.0 * xm * s, 1.0 - s
            else:
                qq, r = fa / fc, fb / fc
                p = s * (2.0 * xm * qq * (qq - r) - (b - a) * (r - 1.0))
                q = (qq - 1.0) * (r - 1.0) * (s - 1.0)
            if p > 0:
                q = -q
            p = abs(p)
            if 2.0 * p < min(3.0 * xm * q - abs(tol1 * q), abs(e * q)):
                e, d = d, p / q
            else:
                d = e = xm
        else:
            d = e = xm
        a, fa = b, fb
        b += d if abs(d) > tol1 else math.copysign(tol1, xm)
        fb = f(b)
    raise ValueError("no convergence")


def compute_uncertainty(grid, disp, cont, flux, var, spec_res, label, search_radius=None, prec=F64):
    """SingleFitter::compute_uncertainty (fitting.rs:480-568) on the oracle's
    chi2: {label index: (below, above)} with None for a failed search."""
    sr = np.array(search_radius if search_radius is not None else [2000.0, 0.3, 0.3, 40.0, 40.0], float)
    lab = np.asarray(label, dtype=np.float64)
    sr[0] *= lab[0]
    sr[3] = max(lab[3] * sr[3], 100.0)
    c0, s0 = chi2(grid, disp, cont, flux, var, lab, prec)
    if s0[0]:
        raise OracleError("chi2 at the label failed")
    n = 4.0 * spec_res * (disp.wl[-1] - disp.wl[0]) / (disp.wl[0] + disp.wl[-1])
    target = c0[0] * (1.0 + math.sqrt(2.0 / n))
    outer = {3: (0.0, 1e4), 4: (-1e3, 1e3)}
    res = {}
    for i in range(5):
        pair = []
        for right in (False, True):
            try:
                bl = lab.copy()
                bl[i] += sr[i] if right else -sr[i]
                lo, hi = outer[i] if i in outer else limits_at(grid, bl, i)
                bound = min(max(bl[i], lo), hi)
                resc = (bound - lab[i]) / sr[i]

                def f(x, i=i):
                    l2 = lab.copy()
                    l2[i] += x * sr[i]
                    c, s = chi2(grid, disp, cont, flux, var, l2, prec)
                    if s[0]:
                        raise ValueError("chi2 failed")
                    return c[0] - target

                sol = _brent(f, 0.0, min(resc, 1.0)) if right else _brent(f, resc, 0.0)
                pair.append(sol * sr[i] if right else -sol * sr[i])
            except (ValueError, OracleError):
                pair.append(None)
        res[i] = tuple(pair)
    return res


# ------------------------------------------------------------------ binaries
def binary_model(grid, cont_grid, disp, lab, prec=F32):
    """produce_binary_model_norm (interpolate.rs:868): lab = star 1 [5],
    star 2 [5], light ratio."""
    lab = np.ascontiguousarray(lab, dtype=np.float64)
    out = np.zeros(len(disp.wl))
    if lib().or_binary_model(grid.h, cont_grid.h, disp.h, prec, _p(lab), _p(out)):
        raise _err()
    return out


def binary_chi2(grid, cont_grid, disp, cont, flux, var, labels, prec=F32, nthreads=0):
    flux = np.ascontiguousarray(flux, dtype=np.float32)
    var = np.ascontiguousarray(var, dtype=np.float32)
    labels = np.ascontiguousarray(np.atleast_2d(labels), dtype=np.float64)
    out = np.zeros(len(labels))
    st = np.zeros(len(labels), dtype=np.int32)
    nt = nthreads or os.cpu_count()
    if lib().or_binary_chi2(grid.h, cont_grid.h, disp.h, cont.h, prec, _p(flux), _p(var), len(flux),
                            _p(labels), len(labels), _p(out), _p(st), nt):
        raise _err()
    return out, st


def binary_settings(num_particles, max_iters, vsini_range, rv_range, inertia=0.7213475204,
                    cognitive=1.1931471806, social=1.1931471806, delta=1e-7, constraints=()):
    s = BinarySettings()
    s.num_particles, s.max_iters = num_particles, max_iters
    s.inertia, s.cognitive, s.social, s.delta = inertia, cognitive, social, delta
    s.vsini_lo, s.vsini_hi = vsini_range
    s.rv_lo, s.rv_hi = rv_range
    for (idx, kind, a, b) in constraints:
        s.ckind[idx], s.ca[idx], s.cb[idx] = kind, a, b
    return s


def binary_fit(grid, cont_grid, disp, cont, st, flux, var, seed, prec=F32, nthreads=0, trace=False):
    """BinaryFitter::fit (fitting.rs:633-697) on the shared draw stream."""
    flux = np.ascontiguousarray(flux, dtype=np.float32)
    var = np.ascontiguousarray(var, dtype=np.float32)
    res = BinaryResult()
    tr = np.zeros((st.max_iters + 1, st.num_particles, 12)) if trace else None
    nt = nthreads or os.cpu_count()
    rc = lib().or_binary_fit(grid.h, cont_grid.h, disp.h, cont.h, prec, C.byref(st), _p(flux), _p(var),
                             len(flux), seed, nt, C.byref(res), _p(tr))
    out = dict(label1=np.array(res.label1[:]), label2=np.array(res.label2[:]), light_ratio=res.light_ratio,
               chi2=res.chi2, iterations=res.iterations, status=res.status,
               params=np.array(res.params[:res.n_params]),
               error=lib().or_last_error().decode() if rc else "")
    if trace:
        return out, rc, tr
    return out, rc
