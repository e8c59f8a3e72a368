#!/usr/bin/env python
"""Benchmark: batched PSO fits of synthetic stars on B200 (one process per GPU).

Workload (the reference's batched configuration): a 60 x 21 x 11 grid of
80,000-pixel uint16 models (13,860 models, 2.2 GB resident in HBM); 1,024
synthetic stars per GPU with labels uniform in the grid, vsini 0-300 km/s, RV
-150..150 km/s, 10k-60k observed pixels and SNR 20-200; R = 85,000 Gaussian
instrument profile; 8-chunk degree-5 continuum with 0.2 overlap; PSO with 64
particles x 200 iterations.  Data are synthetic and seeded (there is no
public dataset for this path).

A step is one PSO iteration over the whole batch: every star's 64
particles are evaluated (interpolate -> rotation -> instrument ->
shift/resample -> continuum -> chi2) and every swarm is updated.
value = star fits/s = chi2 evals/s / evals per fit (64 x 201).  e2e =
the same metric for a complete fit of the batch through the public API
(host arrays in, results out).

--impl reference times the CPU restatement of the reference's path (the
oracle, FP32 mirror, all host threads, stars in parallel like fit_bulk) on
a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "star fits/s & χ² evals/s vs plain GPU path at equal label error; p99 latency"
PARTICLES, ITERS = 64, 200
EVALS_PER_FIT = PARTICLES * (ITERS + 1)
RESOLUTION = 85000.0
# Algorithmic work per unit (the bases of the roofline fields):
# interpolation: 64 neighbours x 2 B read + 4 B written per interpolated pixel
INTERP_BYTES_PER_PX = 64 * 2 + 4
# broadening: per 2048-point overlap-save block a forward and an inverse real
# FFT (2.5 N log2 N flops each) plus the complex product on 1025 bins
BROADEN_FLOPS_PER_BLOCK = 2 * 2.5 * 2048 * 11 + 6 * 1025
# broadening bytes: 2048 f32 inputs per block, the rotation spectrum per
# evaluation, and per observed pixel its f64 float index read + f32 model written
BROADEN_BYTES_PER_BLOCK, BROADEN_BYTES_PER_EVAL, BROADEN_BYTES_PER_OBS = 2048 * 4, 1025 * 8, 8 + 4
# whole path, per chi2 evaluation: B_eval = 128 N_win + 8 N_obs (grid rows + flux/var)
PATH_BYTES_PER_WIN_PX, PATH_BYTES_PER_OBS = 128, 8
# nominal FP32 CUDA-core peak of a B200: 148 SMs x 128 FMA/clk x 2 flops x 1.965 GHz
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
# DRAM bytes per evaluation (dram__bytes_read.sum + dram__bytes_write.sum)
# from one ncu capture of a mid-fit step of 256 stars (16,384 evaluations,
# --clock-control none), divided by its evaluations: the traffic of a launch
# grows in proportion to the evaluations it runs, so a full launch's traffic
# is this figure times its evaluations.  The interpolation is the
# tensor-core kernel plus the CUDA-core kernel (groups below the tuned
# size); k_broaden includes its block-bound search; chi2 is k_chunk_fit.
DRAM_BYTES_PER_EVAL = {"k_interp": 142447 + 308582 + 23127 + 2459, "k_broaden": 387851 + 133902 + 852,
                       "chi2": 246046 + 5488}
DRAM_SOURCE = "ncu capture, mid-fit step of 256 config-1 stars (16,384 evaluations), scaled per evaluation"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ workload
def make_grid(spec, use_gpu):
    """Config-1 grid; the matrix product runs on the GPU when present (same model as synth.make_grid)."""
    from pasta_b200 import synth as S
    if not use_gpu:
        return S.make_grid(spec)
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    labels = S.gridpoints(spec)
    lm = S.LineModel(spec)
    prof = torch.from_numpy(lm.profiles(spec.wl(), dtype=np.float32)).cuda()
    spectra = np.empty((len(labels), spec.n_px), np.uint16)
    for s in range(0, len(labels), 2048):
        d = torch.from_numpy(lm.depths(labels[s:s + 2048]).astype(np.float32)).cuda()
        f = (1.0 - d @ prof).clamp_(min=0.0)
        spectra[s:s + 2048] = torch.clamp(torch.round(f * 65535.0), 0, 65535).to(torch.int32).cpu().numpy().astype(np.uint16)
    del prof
    torch.cuda.empty_cache()
    return labels, spectra, None


def make_grid_factor_gpu(spec):
    """includes_factor grid (blackbody x line spectrum, f32 maximum per model) with the products on the GPU
    (the same model as synth.make_grid)."""
    import torch
    from pasta_b200 import synth as S
    torch.backends.cuda.matmul.allow_tf32 = False
    labels = S.gridpoints(spec)
    lm = S.LineModel(spec)
    wl = spec.wl()
    prof = torch.from_numpy(lm.profiles(wl, dtype=np.float32)).cuda()
    wlt = torch.from_numpy(wl).cuda()
    spectra = np.empty((len(labels), spec.n_px), np.uint16)
    factors = np.empty(len(labels), np.float32)
    hc_k = 1.4387769e8
    for s0 in range(0, len(labels), 1024):
        lab = labels[s0:s0 + 1024]
        d = torch.from_numpy(lm.depths(lab).astype(np.float32)).cuda()
        f = (1.0 - d @ prof).clamp_(min=0.0)
        t = torch.from_numpy(lab[:, 0]).cuda()[:, None]
        bb = (1.0 / (wlt[None, :] ** 5 * torch.expm1(hc_k / (wlt[None, :] * t))) / S.BB_REF).to(torch.float32)
        f = f * bb
        mx = f.max(dim=1).values
        factors[s0:s0 + 1024] = mx.cpu().numpy()
        q = torch.clamp(torch.round(f / mx[:, None] * 65535.0), 0, 65535).to(torch.int32)
        spectra[s0:s0 + 1024] = q.cpu().numpy().astype(np.uint16)
    del prof
    torch.cuda.empty_cache()
    return labels, spectra, factors


def make_workload(n_stars, seed, spec):
    from pasta_b200 import synth as S
    rng = np.random.default_rng(seed)
    labels = S.random_labels(spec, n_stars, seed=seed, vsini=(0.0, 300.0), rv=(-150.0, 150.0))
    n_obs = rng.integers(10000, 60001, n_stars)
    snr = rng.uniform(20.0, 200.0, n_stars)
    return S.make_stars(spec, labels, n_obs, snr, RESOLUTION, seed=seed)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region, every
    500 ms: its queries can delay the served step's host-side CUDA calls, so
    they are kept sparse."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "500"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ served latency
def serve_latency(P, interp, stars, settings, seeds, rate, n_req, seed):
    """Submit n_req requests at Poisson arrival times (rate per second) to a
    server stepping continuously; time-to-fit is submission to retirement."""
    rng = np.random.default_rng(seed)
    arrive = np.cumsum(rng.exponential(1.0 / rate, n_req))
    pick = rng.integers(0, len(stars), n_req)
    chunks = rng.integers(4, 13, n_req)
    degree = rng.integers(3, 9, n_req)
    conts = [P.ChunkContinuumFitter(stars[j].wl, int(d), int(c), 0.2) for j, c, d in zip(pick, chunks, degree)]
    disps = {}
    for j in set(pick.tolist()):
        disps[j] = P.FixedResolutionDispersion(stars[j].wl, RESOLUTION, interp.synth_wl)
    srv = P.Server(interp, max_slots=len(stars))
    t0 = time.perf_counter()
    i = 0
    ttf = []
    while len(ttf) < n_req:
        now = time.perf_counter() - t0
        while i < n_req and arrive[i] <= now:
            j = int(pick[i])
            srv.submit(disps[j], conts[i], settings, stars[j].flux, stars[j].var, (0.0, 300.0), (-150.0, 150.0),
                       seed=seeds[j] + 104729 * (i + 1))
            i += 1
        q, active, _ = srv.pending()
        if q + active > 0:
            srv.step()
        elif i < n_req:
            time.sleep(max(0.0, min(arrive[i] - now, 0.01)))
        for _, st, res in srv.poll(4096):
            ttf.append(res.time)
    wall = time.perf_counter() - t0
    del srv
    ttf = np.array(ttf)
    return {"p50": float(np.percentile(ttf, 50)), "p99": float(np.percentile(ttf, 99)),
            "mean": float(ttf.mean()), "requests": n_req, "arrival_rate_per_s": rate,
            "fits_per_s": n_req / wall,
            "what": "served form: Poisson arrivals, config-1 stars, own continuum settings per request "
                    "(4-12 chunks, degree 3-8), time from submission to result"}


# ------------------------------------------------------------------ our arm
def binary_leg(P, S, n_stars, cpu, seed):
    """BinaryFitter on the config-0 grid (9 x 11 x 5 x 20,000 px) with a
    continuum grid of unnormalised models on the same axes: n_stars synthetic
    binaries (15,000 observed pixels, SNR 100, R = 85,000), 5 chunks of degree
    8, PSO 40 x 100, each fit through the public API (BinaryFitter.fit, the
    reference's per-star call).  cpu: the oracle's binary fit (FP32 mirror,
    particles on all host threads as with parallelize=true) on a bounded
    sample: one star, initial swarm + 2 iterations, scaled to 101 rounds."""
    import torch
    spec0 = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec0)
    cl, cs, cf = S.make_continuum_grid(spec0)
    wl = P.WlGrid(spec0.log_first, spec0.log_step, spec0.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    cint = P.InMemInterpolator.from_arrays(cl, cs, cf, wl)
    rng = np.random.default_rng(seed)

    def lab():
        return [rng.uniform(6000.0, 8000.0), rng.uniform(-0.5, 0.5), rng.uniform(3.5, 4.5),
                rng.uniform(0.0, 100.0), rng.uniform(-100.0, 100.0)]

    stars = [S.make_binary_star(spec0, lab(), lab(), rng.uniform(0.2, 0.9), 15000, 100.0, RESOLUTION, seed=seed + i,
                                rv_max=100.0, vsini_max=100.0) for i in range(n_stars)]
    fitters = [interp.get_binary_fitter(P.FixedResolutionDispersion(s.wl, RESOLUTION, wl),
                                        P.ChunkContinuumFitter(s.wl, 5, 8, 0.2), P.PSOSettings(40, 100),
                                        (0.0, 100.0), (-100.0, 100.0)) for s in stars]
    warm = interp.get_binary_fitter(fitters[0].dispersion, fitters[0].continuum_fitter, P.PSOSettings(40, 3),
                                    (0.0, 100.0), (-100.0, 100.0))
    warm.fit(interp, cint, stars[0].flux, stars[0].var, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = [f.fit(interp, cint, s.flux, s.var, seed=seed + 17 * i) for i, (f, s) in enumerate(zip(fitters, stars))]
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    evals = n_stars * 40 * 101
    out = {"workload": "binary fits (BinaryFitter.fit per star): config-0 grid 9x11x5 x 20000 px + continuum grid, "
                       "N_obs 15000, 5 chunks deg 8, PSO 40x100 over 11 parameters",
           "stars": n_stars, "fits_per_s": n_stars / t, "chi2_evals_per_s": evals / t, "seconds": t,
           "median_chi2": float(np.median([r.chi2 for r in res]))}
    if cpu:
        O = _oracle()
        og = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec0.log_first, spec0.log_step)
        ogc = O.Grid(cl, cs, cf, O.WL_LOGSPACE, spec0.log_first, spec0.log_step)
        s = stars[0]
        od = O.Disp(og, O.DISP_FIXED, s.wl, RESOLUTION)
        oc = O.Cont(O.CONT_CHUNK, s.wl, 5, 8, 0.2)
        st = O.binary_settings(40, 2, (0.0, 100.0), (-100.0, 100.0))
        nthreads = os.cpu_count() or 1
        t0 = time.perf_counter()
        r, rc = O.binary_fit(og, ogc, od, oc, st, s.flux, s.var, seed, O.F32, nthreads=nthreads)
        tc = time.perf_counter() - t0
        per_fit = tc / 3 * 101
        out["cpu_baseline"] = {"value": 1.0 / per_fit, "unit": "binary fits/s", "cores": nthreads, "kind": "port",
                               "sample": "1 star, initial swarm + 2 iterations (3 x 40 binary chi2 evals) in %.2fs, "
                                         "scaled to 101 rounds" % tc}
        out["gpu_over_cpu"] = out["fits_per_s"] * per_fit
    return out


def linear_leg(P, S, n_labels, k, reps=5):
    """Linear-model continuum (design of k Legendre columns) on the config-0
    grid (20,000 px), one star of 15,000 observed pixels: chi2 of n_labels
    random labels per call through SingleFitter.chi2, with the tensor-core
    path and with the CUDA-core path (best of reps calls each, host clock,
    host arrays in and out)."""
    from pasta_b200 import _ffi
    spec0 = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec0)
    wl = P.WlGrid(spec0.log_first, spec0.log_step, spec0.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    star = S.make_star(spec0, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, RESOLUTION, seed=11)
    d = P.FixedResolutionDispersion(star.wl, RESOLUTION, wl)
    cont = P.LinearModelContinuumFitter(S.legendre_design(star.wl, k))
    fitter = interp.get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    rng = np.random.default_rng(5)
    labs = np.stack([rng.uniform(6000, 8000, n_labels), rng.uniform(-0.5, 0.5, n_labels),
                     rng.uniform(3.5, 4.5, n_labels), rng.uniform(0, 200, n_labels),
                     rng.uniform(-100, 100, n_labels)], axis=1)
    out = {"workload": "chi2 of %d labels, linear-model continuum with %d Legendre columns, config-0 grid, "
                       "N_obs 15000" % (n_labels, k)}
    for name, on in (("tensor_cores", 1), ("cuda_cores", 0)):
        _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(on))
        fitter.chi2(interp, star.flux, star.var, labs)
        best = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            fitter.chi2(interp, star.flux, star.var, labs)
            best = min(best, time.perf_counter() - t0)
        out[name] = {"chi2_evals_per_s": n_labels / best, "seconds": best}
    _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(1))
    return out


def variable_sigma(wl):
    """R(lambda) linear 60,000 -> 90,000 over the observed range, as the Gaussian
    sigma in Angstrom the reference's VariableTargetDispersion takes
    (convolve_rv.rs:363 uses disp as a sigma)."""
    return (wl / np.linspace(60000.0, 90000.0, len(wl)) / 2.355).astype(np.float32)


def precision_leg(args):
    """Precision study on the config-1 grid: n_stars stars with R(lambda) 60k
    -> 90k, rotation through the FFT blocks, the FP32 path (compensated f64
    continuum sums, FP64 Cholesky) against the FP64 oracle over n_labels
    seeded label vectors (half uniform in the grid and the vsini/RV ranges,
    half near each star's own labels, as a contracted swarm): model flux
    (max |d| / max |ref| per label) and chi2 (relative), with the oracle's
    FP32 mirror of the reference's arithmetic beside it; then label errors of
    seeded fits (64 x 200) replayed on the FP64 oracle."""
    import concurrent.futures as cf
    import torch
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    torch.cuda.set_device(0)
    O = _oracle()
    spec = S.config1_grid(n_px=args.npx)
    labels, spectra, factors = make_grid(spec, use_gpu=True)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    interp.direct_max = 0  # rotation through the FFT path
    og = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    ns = args.precision_stars
    stars = make_workload(ns, 2000, spec)
    rng = np.random.default_rng(2024)
    per = -(-args.precision_labels // ns)
    nthreads = os.cpu_count() or 1
    fl_err, fl_err32, c_err, c_err32, chi_ref = [], [], [], [], []
    t0 = time.perf_counter()
    for i, st in enumerate(stars):
        n_here = min(per, args.precision_labels - i * per)
        if n_here <= 0:
            break
        uni = S.random_labels(spec, n_here - n_here // 2, seed=int(rng.integers(1 << 30)), vsini=(0.0, 300.0),
                              rv=(-150.0, 150.0))
        near = st.label + rng.normal(0, 1, (n_here // 2, 5)) * np.array([0.01 * st.label[0], 0.05, 0.05, 5.0, 3.0])
        near[:, 3] = np.clip(near[:, 3], 0.0, 300.0)
        lo = [spec.teffs.min(), spec.ms.min(), spec.loggs.min()]
        hi = [spec.teffs.max(), spec.ms.max(), spec.loggs.max()]
        near[:, :3] = np.clip(near[:, :3], lo, hi)
        labs = np.vstack([uni, near])
        sig = variable_sigma(st.wl)
        d = P.VariableResolutionDispersion(st.wl, sig, wl)
        cont = P.ChunkContinuumFitter(st.wl, 8, 5, 0.2)
        fitter = interp.get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
        gm = interp.produce_model_bulk(d, labs)
        gc = np.array(fitter.chi2(interp, st.flux, st.var, labs))
        od = O.Disp(og, O.DISP_VARIABLE, st.wl, disp=sig)
        oc = O.Cont(O.CONT_CHUNK, st.wl, 8, 5, 0.2)
        r64, s64 = O.chi2(og, od, oc, st.flux, st.var, labs, O.F64, nthreads=nthreads)
        r32, s32 = O.chi2(og, od, oc, st.flux, st.var, labs, O.F32, nthreads=nthreads)

        def models(k):
            m64 = od.produce_model(labs[k], O.F64)
            m32 = od.produce_model(labs[k], O.F32)
            mx = np.abs(m64).max()
            return np.abs(gm[k] - m64).max() / mx, np.abs(m32 - m64).max() / mx

        with cf.ThreadPoolExecutor(nthreads) as ex:
            for a, b in ex.map(models, range(len(labs))):
                fl_err.append(a)
                fl_err32.append(b)
        ok = (s64 == 0) & np.isfinite(r64)
        c_err.extend((np.abs(gc[ok] - r64[ok]) / r64[ok]).tolist())
        c_err32.extend((np.abs(r32[ok] - r64[ok]) / r64[ok]).tolist())
        chi_ref.extend(r64[ok].tolist())
        del od, oc
    t_models = time.perf_counter() - t0

    def stats(x):
        x = np.asarray(x)
        return {"max": float(x.max()), "p99": float(np.percentile(x, 99)), "median": float(np.median(x))}

    chi_ref = np.array(chi_ref)
    c_err, c_err32 = np.array(c_err), np.array(c_err32)
    good = chi_ref < 10.0
    out = {"workload": "precision study: config-1 grid (60x21x11 x %d px), %d stars with R(lambda) 60k->90k "
                       "(VariableResolutionDispersion), rotation by FFT blocks, 8 chunks deg 5; %d label vectors"
                       % (spec.n_px, ns, len(fl_err)),
           "model_flux_rel_err": {"gpu_vs_fp64": stats(fl_err), "fp32_mirror_vs_fp64": stats(fl_err32),
                                  "basis": "max |model - FP64| / max |FP64| per label"},
           "chi2_rel_err": {"gpu_vs_fp64": stats(c_err), "fp32_mirror_vs_fp64": stats(c_err32),
                            "gpu_vs_fp64_chi2_below_10": stats(c_err[good]) if good.any() else None,
                            "labels": int(len(c_err))},
           "seconds_models_chi2": t_models}
    if args.replay_stars > 0:
        k = args.replay_stars
        disps = [P.VariableResolutionDispersion(s.wl, variable_sigma(s.wl), wl) for s in stars[:k]]
        conts = [P.ChunkContinuumFitter(s.wl, 8, 5, 0.2) for s in stars[:k]]
        seeds = [int(77 + i) for i in range(k)]
        res = P.fit_many(interp, disps, conts, P.PSOSettings(PARTICLES, ITERS), [s.flux for s in stars[:k]],
                         [s.var for s in stars[:k]], (0.0, 300.0), (-150.0, 150.0), seeds=seeds)
        out["label_error_vs_fp64_oracle"] = label_replay(
            O, og, stars[:k], seeds, res, disp=lambda s: O.Disp(og, O.DISP_VARIABLE, s.wl, disp=variable_sigma(s.wl)))
    return out


def config4_leg(args):
    """Config 4: the includes_factor grid (80 x 26 x 13 models x 120,000 px,
    6.5 GB u16 + f32 maxima), stars fitted with a 40-column Legendre
    linear-model continuum (tensor cores) and PSO 128 x 300, served (slots
    refilled as fits finish, steady state) and batched (fit_many)."""
    import torch
    from pasta_b200 import _ffi
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    spec = S.config4_grid(n_px=120000)
    t = time.time()
    labels, spectra, factors = make_grid_factor_gpu(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    log(f"[config4] grid {spectra.shape} in {time.time() - t:.1f}s")
    ns = args.c4_stars
    rng = np.random.default_rng(4096)
    lab = S.random_labels(spec, ns, seed=4096, vsini=(0.0, 300.0), rv=(-150.0, 150.0))
    t = time.time()
    stars = S.make_stars(spec, lab, rng.integers(10000, 60001, ns), rng.uniform(20.0, 200.0, ns), RESOLUTION,
                         seed=4096)
    log(f"[config4] {ns} stars in {time.time() - t:.1f}s")
    disps = [P.FixedResolutionDispersion(s.wl, RESOLUTION, wl) for s in stars]
    conts = [P.LinearModelContinuumFitter(S.legendre_design(s.wl, 40)) for s in stars]
    Pn, It = 128, 300
    settings = P.PSOSettings(Pn, It)
    seeds = [int(11 + i) for i in range(ns)]
    fl = [s.flux for s in stars]
    vr = [s.var for s in stars]
    srv = P.Server(interp, max_slots=ns)
    per_step = -(-ns // (It + 1))
    cursor = [0]

    def feed(k):
        for _ in range(k):
            i = cursor[0] % ns
            srv.submit(disps[i], conts[i], settings, fl[i], vr[i], (0.0, 300.0), (-150.0, 150.0),
                       seed=seeds[i] + 7919 * (cursor[0] // ns))
            cursor[0] += 1

    t = time.time()
    for _ in range(It + 1):
        feed(per_step)
        srv.step()
        srv.poll(4096)
    log(f"[config4] served ramp-up in {time.time() - t:.1f}s")
    feed(per_step * (args.warmup + 2))
    srv.run(args.warmup)
    srv.poll(4096)
    feed(per_step * (args.steps + 2))
    torch.cuda.synchronize(dev)
    st0 = srv.stats()
    with ClockSampler(0) as clk:
        ms = srv.run(args.steps)
    torch.cuda.synchronize(dev)
    st1 = srv.stats()
    del srv
    evals = st1["evals"] - st0["evals"]
    served = evals / (ms / 1000.0) / (Pn * (It + 1))
    # stage profile of a batched mid-fit step (roofline of the dominant kernel)
    nb = min(ns, args.c4_batch)
    b = P.BatchFit(interp, disps[:nb], conts[:nb], settings, fl[:nb], vr[:nb], (0.0, 300.0), (-150.0, 150.0),
                   seeds=seeds[:nb])
    b.step(It // 2)
    prof = [b.profile_step() for _ in range(3)]
    stage = {k: float(np.mean([p[k] for p in prof])) for k in prof[0]}
    b.finish()
    del b
    # batched form end to end (fit_many from host arrays) on nb stars
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = P.fit_many(interp, disps[:nb], conts[:nb], settings, fl[:nb], vr[:nb], (0.0, 300.0), (-150.0, 150.0),
                     seeds=seeds[:nb])
    torch.cuda.synchronize(dev)
    t_e2e = time.perf_counter() - t0
    peak, peak_kind = measured_peaks()
    br_s = stage["broaden_ms"] / 1000.0
    br_bytes = (stage["broaden_blocks"] * BROADEN_BYTES_PER_BLOCK + stage["evals"] * BROADEN_BYTES_PER_EVAL
                + stage["obs_px"] * BROADEN_BYTES_PER_OBS)
    br_tf = stage["broaden_blocks"] * BROADEN_FLOPS_PER_BLOCK / br_s / 1e12
    err = np.array([np.abs(np.array(r.label.as_list()) - s.label) for r, s in zip(res, stars[:nb])])
    return {"config4": True, "metric": METRIC, "value": served, "unit": "fits/s",
            "workload": "config 4: includes_factor grid 80x26x13 x 120000 px (%.1f GB), %d stars served in steady "
                        "state (slots refilled), 40-column Legendre linear-model continuum, PSO %dx%d, R=85000"
                        % (spectra.nbytes / 1e9, ns, Pn, It),
            "served": {"fits_per_s": served, "evals_per_s": evals / (ms / 1000.0), "ms_per_step": ms / args.steps,
                       "steps": args.steps},
            "batched_e2e": {"stars": nb, "fits_per_s": nb / t_e2e, "seconds": t_e2e},
            "stage_ms": {k: v for k, v in stage.items() if k.endswith("_ms")},
            "roofline": {"bound": "hbm", "kernel": "k_broaden", "algorithmic_rate": br_bytes / br_s / 1e9,
                         "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
                         "fp32": {"achieved": br_tf, "peak": FP32_PEAK_TFLOPS, "frac": br_tf / FP32_PEAK_TFLOPS}},
            "label_error_vs_truth": {"median_abs": np.median(err, axis=0).tolist()},
            "clocks": clk.summary(), "linear_tensor_cores": True,
            "kernel_launches": int(_ffi.lib().pasta_kernel_launch_count())}


def run_ours(args):
    import torch
    import torch.distributed as dist

    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    from pasta_b200.dist import gather_to_rank0, max_over_ranks, sum_over_ranks

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    from pasta_b200 import _ffi
    _ffi.check(_ffi.lib().pasta_set_device(local))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    n_stars = args.stars
    spec = S.config1_grid(n_px=args.npx)
    t = time.time()
    labels, spectra, factors = make_grid(spec, use_gpu=True)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    log(f"[rank {rank}] grid {spectra.shape} in {time.time() - t:.1f}s")
    t = time.time()
    stars = make_workload(n_stars, 1000 + rank, spec)
    disps = [P.FixedResolutionDispersion(s.wl, RESOLUTION, wl) for s in stars]
    conts = [P.ChunkContinuumFitter(s.wl, 8, 5, 0.2) for s in stars]
    settings = P.PSOSettings(PARTICLES, ITERS)
    seeds = [int(7 + 100003 * rank + i) for i in range(n_stars)]
    log(f"[rank {rank}] {n_stars} stars in {time.time() - t:.1f}s")
    if args.stages_only:
        # one mid-fit step run stage by stage inside an NVTX range "stages"
        # (what ncu --nvtx --nvtx-include "stages/" captures)
        b = P.BatchFit(interp, disps, conts, settings, [s.flux for s in stars], [s.var for s in stars],
                       (0.0, 300.0), (-150.0, 150.0), seeds=seeds)
        b.step(ITERS // 2)
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_push("stages")
        st = b.profile_step()
        torch.cuda.nvtx.range_pop()
        b.finish()
        return {"stages_only": True, "stars": n_stars, "stage": st} if rank == 0 else None

    fl = [s.flux for s in stars]
    vr = [s.var for s in stars]

    # -------- timed region: the served form in steady state.  n_stars slots,
    # refilled as fits finish, so the slots sit at every PSO iteration of the
    # fit and a step costs what the average step of a whole fit costs.  The
    # ramp-up that spreads the slots over the iterations is set-up, untimed.
    srv = P.Server(interp, max_slots=n_stars)
    per_step = -(-n_stars // (ITERS + 1))  # fits that finish per step in steady state
    cursor = [0]

    def feed(k):
        for _ in range(k):
            i = cursor[0] % n_stars
            srv.submit(disps[i], conts[i], settings, fl[i], vr[i], (0.0, 300.0), (-150.0, 150.0),
                       seed=seeds[i] + 7919 * (cursor[0] // n_stars))
            cursor[0] += 1

    t = time.time()
    for _ in range(ITERS + 1):
        feed(per_step)
        srv.step()
        srv.poll(4096)
    log(f"[rank {rank}] served ramp-up in {time.time() - t:.1f}s, {srv.pending()[1]} slots active")
    feed(per_step * (args.warmup + 2))
    srv.run(args.warmup)
    srv.poll(4096)
    feed(per_step * (args.steps + 2))
    barrier()
    torch.cuda.synchronize(dev)
    st0 = srv.stats()
    launches0 = _ffi.lib().pasta_kernel_launch_count()
    with ClockSampler(local) as clk:
        dev_ms = srv.run(args.steps)
    torch.cuda.synchronize(dev)
    barrier()
    launches = _ffi.lib().pasta_kernel_launch_count() - launches0
    st1 = srv.stats()
    fits_done = len(srv.poll(1 << 16))
    del srv
    t_max = max_over_ranks(dev_ms / 1000.0, dev)
    evals_step = (st1["evals"] - st0["evals"]) / args.steps
    evals_total = sum_over_ranks(st1["evals"] - st0["evals"], dev)
    evals_per_s = evals_total / t_max
    fits_per_s = evals_per_s / EVALS_PER_FIT

    # -------- per-stage breakdown (CUDA events between the stages, live) on a
    # batch advanced to the middle of its fit
    b = P.BatchFit(interp, disps, conts, settings, fl, vr, (0.0, 300.0), (-150.0, 150.0), seeds=seeds)
    b.step(ITERS // 2)
    prof = [b.profile_step() for _ in range(3)]
    stage = {k: float(np.mean([p[k] for p in prof])) for k in prof[0]}
    b.finish()
    del b

    # -------- end to end: one complete fit of the batch through the public API
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = P.fit_many(interp, disps, conts, settings, fl, vr, (0.0, 300.0), (-150.0, 150.0), seeds=seeds)
    torch.cuda.synchronize(dev)
    t_e2e = max_over_ranks(time.perf_counter() - t0, dev)
    barrier()
    e2e_fits = sum_over_ranks(len(res), dev) / t_e2e
    h2d = int(sum(x.nbytes + y.nbytes for x, y in zip(fl, vr)))
    d2h = int(sum(8 * 8 + 4 * len(r.continuum_params) for r in res))
    err = np.array([np.abs(np.array(r.label.as_list()) - s.label) for r, s in zip(res, stars)])

    # -------- plain one-star-at-a-time GPU path on a sample of the workload
    n_plain = min(args.plain_stars, n_stars)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    plain = P.fit_many(interp, disps[:n_plain], conts[:n_plain], settings, fl[:n_plain], vr[:n_plain],
                       (0.0, 300.0), (-150.0, 150.0), seeds=seeds[:n_plain], mode=1)
    torch.cuda.synchronize(dev)
    t_plain = time.perf_counter() - t0
    same = all(a.label.as_list() == r.label.as_list() and a.chi2 == r.chi2 for a, r in zip(plain, res[:n_plain]))
    plain_fits = n_plain / t_plain

    # -------- binary fits (BinaryFitter, config-0 sizes)
    binary = binary_leg(P, S, args.binary_stars, rank == 0 and world == 1 and not args.no_cpu,
                        seed=5150 + rank) if args.binary_stars > 0 else None
    torch.cuda.synchronize(dev)

    # -------- linear-model continuum: tensor-core vs CUDA-core path (config-0 sizes)
    linear = linear_leg(P, S, args.linear_labels, args.linear_k) if args.linear_labels > 0 and rank == 0 else None
    torch.cuda.synchronize(dev)

    # -------- served time-to-fit: Poisson arrivals at each rate, each request
    # its own continuum settings (4-12 chunks, degree 3-8), stars of the workload
    lat = None
    if args.serve_requests > 0:
        lat = [serve_latency(P, interp, stars, settings, seeds, rate=r, n_req=args.serve_requests,
                             seed=4242 + rank) for r in args.serve_rates]
    torch.cuda.synchronize(dev)

    # -------- CPU legs (oracle, rank 0 at N=1): the baseline and the label
    # errors of a sample of the timed workload against the FP64 oracle
    cpu = replay = None
    if rank == 0 and world == 1 and not args.no_cpu:
        O = _oracle()
        og = cpu_setup(O, labels, spectra, factors, spec)
        cpu = cpu_baseline(O, og, stars, seeds, budget_s=args.cpu_seconds)
        if args.replay_stars > 0:
            replay = label_replay(O, og, stars[:args.replay_stars], seeds[:args.replay_stars],
                                  res[:args.replay_stars])
        del og

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    ev = stage["evals"]
    step_ms = dev_ms / args.steps

    def traffic(k):
        return DRAM_BYTES_PER_EVAL[k] * ev

    def hbm_view(kernel, bytes_alg, ms, tkey, note=None):
        """algorithmic rate and measured-DRAM fraction of one kernel (per mid-fit launch)"""
        s_ = ms / 1000.0
        tr = traffic(tkey)
        d = {"bound": "hbm", "kernel": kernel, "achieved": tr / s_ / 1e9, "peak": peak, "unit": "GB/s",
             "frac": tr / s_ / 1e9 / peak, "traffic": tr, "basis": "measured DRAM bytes per launch / launch time",
             "peak_kind": peak_kind, "ms": ms, "algorithmic_bytes_per_launch": bytes_alg,
             "algorithmic_rate": {"value": bytes_alg / s_ / 1e9, "unit": "GB/s",
                                  "over_peak": bytes_alg / s_ / 1e9 / peak}}
        if note:
            d["note"] = note
        return d

    # the dominant kernel: fused broadening.  Its work is FP32 FFT arithmetic;
    # its HBM view is measured DRAM bytes (and algorithmic bytes) per launch
    br_flops = stage["broaden_blocks"] * BROADEN_FLOPS_PER_BLOCK
    br_bytes = (stage["broaden_blocks"] * BROADEN_BYTES_PER_BLOCK + ev * BROADEN_BYTES_PER_EVAL
                + stage["obs_px"] * BROADEN_BYTES_PER_OBS)
    roofline = hbm_view("k_broaden", br_bytes, stage["broaden_ms"], "k_broaden")
    br_tf = br_flops / (stage["broaden_ms"] / 1000.0) / 1e12
    roofline["fp32"] = {"achieved": br_tf, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": br_tf / FP32_PEAK_TFLOPS,
                        "algorithmic_flops_per_launch": br_flops,
                        "peak_kind": "nominal FP32 CUDA-core peak (148 SMs x 128 FMA/clk x 1.965 GHz)"}
    interp_bytes = stage["interp_px"] * INTERP_BYTES_PER_PX
    # chunk continuum + chi2: per observed pixel the model, flux and chunk
    # coordinate (moments) and the model, flux, var and coordinate (residuals)
    chi2_bytes = stage["obs_px"] * (12 + 16)
    # the path as a whole on the per-evaluation byte basis B_eval (no reuse)
    path_bytes = stage["interp_px"] * PATH_BYTES_PER_WIN_PX + stage["obs_px"] * PATH_BYTES_PER_OBS
    path_gbs = path_bytes / ev * evals_per_s / 1e9
    step_dram = sum(DRAM_BYTES_PER_EVAL.values()) * evals_step
    line = {
        "metric": METRIC, "value": fits_per_s, "unit": "fits/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (u16 grid, f64 continuum solves)", "data": "synthetic (seeded)",
        "config": {**workload_config(n_stars, spec, spectra.nbytes, world),
                   "evals_per_step": evals_step, "fits_finished_in_timed_steps": fits_done,
                   "host_ms_per_step": {k: (st1[k + "_us"] - st0[k + "_us"]) / 1000.0 / args.steps
                                        for k in ("admit", "device", "retire", "refit")},
                   "step": "one served step: PSO update, chi2 of every active particle, best update, "
                           "admissions and retirements (final refit)",
                   "l2": "inputs larger than L2 (%.1f GB grid, ~%.0f GB of interpolation reads per step)"
                         % (spectra.nbytes / 1e9, interp_bytes / 1e9)},
        "evals_per_s": evals_per_s,
        "e2e": {"value": e2e_fits, "unit": "fits/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "seconds": t_e2e, "what": "batched form: fit_many of %d stars from host arrays to results "
                                          "(201 PSO steps + final refit); bytes are per call" % n_stars},
        "latency_s": lat,
        "binary": binary,
        "linear_continuum": linear,
        "plain_gpu": {"fits_per_s": plain_fits, "stars": n_plain, "identical_results": same,
                      "what": "plain form: stars 0..%d of the workload one at a time, swarm on the host, "
                              "eager launches, costs read back every iteration" % (n_plain - 1),
                      "served_over_plain": fits_per_s / (plain_fits * world),
                      "batched_e2e_over_plain": e2e_fits / (plain_fits * world),
                      "served_p99_s": lat[-1]["p99"] if lat else None},
        "label_error_vs_truth": {"median_abs": np.median(err, axis=0).tolist(),
                                 "order": ["teff", "m", "logg", "vsini", "rv"]},
        "label_error_vs_fp64_oracle": replay,
        "stage_ms": {k: v for k, v in stage.items() if k.endswith("_ms")},
        "roofline": roofline,
        "roofline_path": {"basis": "B_eval = 128 B x window px + 8 B x observed px per evaluation (no reuse)",
                          "algorithmic_rate": {"value": path_gbs, "unit": "GB/s", "over_peak": path_gbs / peak},
                          "measured_dram": {"value": step_dram / (step_ms / 1000.0) / 1e9, "unit": "GB/s",
                                            "frac": step_dram / (step_ms / 1000.0) / 1e9 / peak,
                                            "bytes_per_step": step_dram},
                          "peak": peak, "peak_kind": peak_kind, "bytes_per_eval": path_bytes / ev},
        "roofline_kernels": [
            hbm_view("k_interp_tc+k_interp", interp_bytes, stage["interp_ms"], "k_interp",
                     "neighbour rows shared by a star's particles are read once per group and hit in L2, so the "
                     "algorithmic rate exceeds the DRAM rate"),
            hbm_view("k_chunk_fit", chi2_bytes, stage["chi2_ms"], "chi2"),
        ],
        "dram_source": DRAM_SOURCE,
        "tuned": {"direct_max_taps": interp.direct_max, "interp_tc_min_members": interp.tc_min,
                  "what": "measured on this device at grid load: widest combined broadening kernel convolved "
                          "directly, and the group size from which the interpolation runs on the tensor cores "
                          "(65: never, the CUDA cores win at every size)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    return line


# ------------------------------------------------------------ CPU baseline
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    return O


def cpu_setup(O, labels, spectra, factors, spec):
    return O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)


def cpu_sample(O, og, stars, seeds, n_stars, iters, nthreads):
    """Fit n_stars stars (threads over stars) with `iters` PSO iterations; returns (seconds, evals)."""
    st = O.settings(PARTICLES, iters, (0.0, 300.0), (-150.0, 150.0))
    t0 = time.perf_counter()
    evals = 0
    # stars with different wavelength grids: one oracle call per group of nthreads stars
    import concurrent.futures as cf

    def one(i):
        s = stars[i]
        od = O.Disp(og, O.DISP_FIXED, s.wl, RESOLUTION)
        oc = O.Cont(O.CONT_CHUNK, s.wl, 8, 5, 0.2)
        res, rc = O.fit(og, od, oc, st, s.flux[None], s.var[None], [seeds[i]], O.F32, nthreads=1, over_stars=True)
        return PARTICLES * (iters + 1)

    with cf.ThreadPoolExecutor(nthreads) as ex:
        for e in ex.map(one, range(n_stars)):
            evals += e
    return time.perf_counter() - t0, evals


def cpu_baseline(O, og, stars, seeds, budget_s=20.0):
    nthreads = os.cpu_count() or 1
    t1, e1 = cpu_sample(O, og, stars, seeds, 1, 0, 1)  # calibration: one star, initial swarm only
    per_eval = t1 / e1
    n = max(nthreads, int(budget_s * nthreads / (per_eval * PARTICLES)))
    n = min(n, len(stars))
    t, e = cpu_sample(O, og, stars, seeds, n, 0, nthreads)
    evals_s = e / t
    return {"value": evals_s / EVALS_PER_FIT, "unit": "fits/s", "cores": nthreads, "kind": "port",
            "evals_per_s": evals_s,
            "sample": "%d stars x %d particles (initial swarm evaluation, %d chi2 evals) in %.1fs on %d threads; "
                      "fits/s = evals/s / %d" % (n, PARTICLES, e, t, nthreads, EVALS_PER_FIT)}


def label_replay(O, og, stars, seeds, results, disp=None):
    """Label errors of the device fits of a sample of the timed workload
    against the FP64 oracle replayed on the same draw stream (64 x 200, the
    same seeds), beside the error of the oracle's FP32 mirror of the
    reference's arithmetic on the same replay.  Tolerance: dTeff <= 1 K,
    d[M/H], dlogg <= 1e-3, dvsini, dRV <= 0.01 km/s."""
    tol = np.array([1.0, 1e-3, 1e-3, 0.01, 0.01])
    st = O.settings(PARTICLES, ITERS, (0.0, 300.0), (-150.0, 150.0))
    nthreads = os.cpu_count() or 1
    gpu_err, f32_err, per = [], [], []
    t0 = time.perf_counter()
    for s, sd, r in zip(stars, seeds, results):
        od = disp(s) if disp else O.Disp(og, O.DISP_FIXED, s.wl, RESOLUTION)
        oc = O.Cont(O.CONT_CHUNK, s.wl, 8, 5, 0.2)
        r64, rc64 = O.fit(og, od, oc, st, s.flux[None], s.var[None], [sd], O.F64, nthreads=nthreads,
                          over_stars=False)
        r32, rc32 = O.fit(og, od, oc, st, s.flux[None], s.var[None], [sd], O.F32, nthreads=nthreads,
                          over_stars=False)
        ref = r64[0]["label"]
        g = np.abs(np.array(r.label.as_list()) - ref)
        f = np.abs(r32[0]["label"] - ref)
        gpu_err.append(g)
        f32_err.append(f)
        per.append({"gpu": g.tolist(), "fp32_mirror": f.tolist(), "within_tolerance": bool((g <= tol).all()),
                    "chi2_rel": abs(r.chi2 - r64[0]["chi2"]) / r64[0]["chi2"]})
    gpu_err, f32_err = np.array(gpu_err), np.array(f32_err)
    return {"stars": len(stars), "order": ["teff", "m", "logg", "vsini", "rv"],
            "gpu_max_abs": gpu_err.max(axis=0).tolist(), "fp32_mirror_max_abs": f32_err.max(axis=0).tolist(),
            "tolerance": tol.tolist(), "gpu_within_tolerance": int(sum(p["within_tolerance"] for p in per)),
            "per_star": per, "seconds": time.perf_counter() - t0,
            "what": "stars 0..%d of the timed workload: device fit (fit_many, the e2e run) and the oracle's FP32 "
                    "mirror of the reference, each against the FP64 oracle on the same seeded draws (64 x 200)"
                    % (len(stars) - 1)}


def workload_config(n_stars, spec, grid_bytes, world):
    """The workload both arms of the bench name in their `config`."""
    return {"workload": "config-1 fits in steady state: %d slots/GPU refilled as fits finish (slots spread "
                        "over all PSO iterations); grid 60x21x11 x %d px uint16 (%.1f GB), N_obs 10k-60k, "
                        "vsini 0-300, RV +-150, R=85000, 8 chunks deg 5, PSO %dx%d"
                        % (n_stars, spec.n_px, grid_bytes / 1e9, PARTICLES, ITERS),
            "stars_per_gpu": n_stars, "particles": PARTICLES, "iterations": ITERS,
            "parallelism": "replicas x%d (stars sharded, no collective)" % world}


def run_reference(args):
    rank, world, local = env_rank()
    if rank != 0:
        return None
    from pasta_b200 import synth as S
    O = _oracle()
    spec = S.config1_grid(n_px=args.npx)
    t = time.time()
    labels, spectra, factors = S.make_grid(spec)
    log(f"[reference] grid in {time.time() - t:.1f}s")
    stars = make_workload(args.stars, 1000, spec)
    seeds = [int(7 + i) for i in range(args.stars)]
    og = cpu_setup(O, labels, spectra, factors, spec)
    nthreads = os.cpu_count() or 1
    per_step = nthreads  # one star per thread per step, initial swarm evaluated
    times, evals = [], []
    cursor = 0
    for k in range(args.warmup + args.steps):
        idx = [(cursor + j) % len(stars) for j in range(per_step)]
        cursor += per_step
        sub = [stars[i] for i in idx]
        sd = [seeds[i] for i in idx]
        t, e = cpu_sample(O, og, sub, sd, len(sub), 0, nthreads)
        if k >= args.warmup:
            times.append(t)
            evals.append(e)
    tot_t, tot_e = float(np.sum(times)), float(np.sum(evals))
    evals_s = tot_e / tot_t
    value = evals_s / EVALS_PER_FIT
    sample = ("per step %d stars x %d particles (initial swarm, %d chi2 evals) on %d threads; fits/s = evals/s / %d"
              % (per_step, PARTICLES, per_step * PARTICLES, nthreads, EVALS_PER_FIT))
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_t / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": workload_config(args.stars, spec, spectra.nbytes, world),
            "implementation": "C++ restatement of the reference CPU path (oracle FP32 mirror, stars on all host "
                              "threads like fit_bulk); the Rust reference cannot be built here",
            "evals_per_s": evals_s,
            "cpu_baseline": {"value": value, "unit": "fits/s", "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--stars", type=int, default=1024)
    ap.add_argument("--npx", type=int, default=80000)
    ap.add_argument("--plain-stars", type=int, default=16, help="plain-form leg: stars of the workload")
    ap.add_argument("--replay-stars", type=int, default=4,
                    help="label errors against the FP64 oracle: stars of the workload replayed on the CPU (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-rates", type=lambda x: [float(v) for v in x.split(",")], default=[50.0, 500.0, 2000.0],
                    help="served latency runs: arrivals per second, comma separated")
    ap.add_argument("--serve-requests", type=int, default=300, help="served latency runs: requests each (0: skip)")
    ap.add_argument("--binary-stars", type=int, default=16, help="binary-fit leg: stars (0: skip)")
    ap.add_argument("--linear-only", action="store_true",
                    help="time chi2 with a linear-model continuum, tensor-core and CUDA-core paths, and print it")
    ap.add_argument("--linear-labels", type=int, default=1024, help="linear-continuum leg: labels per call (0: skip)")
    ap.add_argument("--linear-k", type=int, default=40)
    ap.add_argument("--binary-only", action="store_true",
                    help="run only the binary-fit leg (with its CPU baseline unless --no-cpu) and print it")
    ap.add_argument("--precision", action="store_true",
                    help="run the precision study (R(lambda) 60k->90k, FFT rotation, FP32 path vs the FP64 oracle) "
                         "and print it")
    ap.add_argument("--precision-stars", type=int, default=256)
    ap.add_argument("--precision-labels", type=int, default=10000)
    ap.add_argument("--config4", action="store_true",
                    help="run the config-4 workload (includes_factor grid at 120,000 px, 40-column linear-model "
                         "continuum, PSO 128 x 300) served and batched, and print it")
    ap.add_argument("--c4-stars", type=int, default=512, help="config-4 leg: served slots (stars)")
    ap.add_argument("--c4-batch", type=int, default=256, help="config-4 leg: stars in the batched fit")
    ap.add_argument("--stages-only", action="store_true",
                    help="profiling aid: one mid-fit batched step, stage by stage, in an NVTX range 'stages'")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torch.distributed.run
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % args.gpus,
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        raise SystemExit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world != args.gpus:
        raise SystemExit("--gpus %d but %d ranks were launched" % (args.gpus, world))
    if args.linear_only:
        from pasta_b200 import pasta as P
        from pasta_b200 import synth as S
        print(json.dumps(linear_leg(P, S, args.linear_labels, args.linear_k)), flush=True)
        return
    if args.precision:
        print(json.dumps(precision_leg(args)), flush=True)
        return
    if args.config4:
        print(json.dumps(config4_leg(args)), flush=True)
        return
    if args.binary_only:
        from pasta_b200 import pasta as P
        from pasta_b200 import synth as S
        print(json.dumps(binary_leg(P, S, max(args.binary_stars, 1), not args.no_cpu, seed=5150)), flush=True)
        return
    line = run_reference(args) if args.impl == "reference" else run_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    if args.impl == "ours":
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
