"""GPU parity on the grid shapes the benchmark workloads use, against the
CPU oracle on the same seeded inputs.

* config-1 shape: the non-uniform Teff axis of the 60 x 21 x 11 grid (a
  run of 16 consecutive Teff values, 5 [M/H] x 5 logg), 80,000 pixels.
  Rotation kernels up to ~945 taps (vsini 300 km/s), RV +-150 km/s, both
  broadening paths, the unfused path above 1,920 combined taps, variable
  resolution R(lambda) 60k -> 90k, and seeded fits replayed against the
  FP64 oracle at the benchmark's PSO size (64 x 200).
* config-4 shape: an includes_factor grid (blackbody x lines, f32 maximum
  per model) at 120,000 pixels (the last 64 pixels carry the reference's
  extra 1/65535, interpolate.rs:978), rotation kernels up to ~1,415 taps,
  and a 40-column linear-model continuum on the tensor cores.
* staircase grid: per-Teff logg limits (interpolate.rs:267-331) with
  labels on the stair edges, where the quadratic fallback and the PSO
  clamps change (interpolate.rs:378-421, 647-664).
* single-star FixConstraint / RangeConstraint fits through the device
  swarm (bounds.rs:69-130).

Tolerances: model flux vs the FP32 mirror max|gpu - ref| <= 1e-5 max|ref|;
chi2 vs FP64 relative 1e-5; replayed fits dTeff <= 1 K, d[M/H], dlogg <=
1e-3, dvsini, dRV <= 0.01 km/s against the FP64 oracle.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLUX_TOL = 1e-5
CHI2_TOL = 1e-5
LABEL_TOL = np.array([1.0, 1e-3, 1e-3, 0.01, 0.01])
R = 85000.0


def relmax(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


def _env(spec):
    import oracle as O
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    labels, spectra, factors = S.make_grid(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    og = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    return dict(O=O, P=P, S=S, spec=spec, labels=labels, spectra=spectra, factors=factors, interp=interp, og=og,
                wl=wl)


def config1_shape():
    from pasta_b200 import synth as S
    spec = S.config1_grid(n_px=80000)
    return dataclasses.replace(spec, teffs=spec.teffs[18:34], ms=spec.ms[::5], loggs=spec.loggs[2:7])


def config4_shape():
    from pasta_b200 import synth as S
    spec = S.config4_grid(n_px=120000)
    return dataclasses.replace(spec, teffs=spec.teffs[30:38], ms=spec.ms[::5], loggs=spec.loggs[4:8])


@pytest.fixture(scope="module")
def c1():
    e = _env(config1_shape())
    S = e["S"]
    e["star"] = S.make_star(e["spec"], [9000.0, -0.3, 3.6, 150.0, 40.0], 40000, 120.0, R, seed=21)
    return e


@pytest.fixture(scope="module")
def c4():
    e = _env(config4_shape())
    S = e["S"]
    spec = e["spec"]
    t = float(np.mean(spec.teffs[2:4]))
    e["star"] = S.make_star(spec, [t, -0.6, 3.3, 120.0, -30.0], 30000, 150.0, R, seed=41)
    return e


def _disp(e, star, kind):
    O, P = e["O"], e["P"]
    if kind == "fixed":
        return P.FixedResolutionDispersion(star.wl, R, e["wl"]), O.Disp(e["og"], O.DISP_FIXED, star.wl, R)
    # R(lambda) linear 60k -> 90k, passed as a Gaussian sigma in Angstrom (the
    # reference's disp is a sigma, convolve_rv.rs:363)
    sig = (star.wl / np.linspace(60000.0, 90000.0, len(star.wl)) / 2.355).astype(np.float32)
    return (P.VariableResolutionDispersion(star.wl, sig, e["wl"]),
            O.Disp(e["og"], O.DISP_VARIABLE, star.wl, disp=sig))


def _models_both_paths(interp, d, lab):
    keep = interp.direct_max
    try:
        interp.direct_max = 512
        direct = interp.produce_model(d, *lab)
        interp.direct_max = 0
        fft = interp.produce_model(d, *lab)
    finally:
        interp.direct_max = keep
    return direct, fft


# ------------------------------------------------------------ config-1 shape
@pytest.mark.parametrize("kind", ["fixed", "variable"])
@pytest.mark.parametrize("vsini,rv", [(0.0, 0.0), (6.0, -150.0), (40.0, 150.0), (150.0, -75.0), (300.0, 149.0),
                                      (300.0, -150.0)])
def test_config1_produce_model(c1, kind, vsini, rv):
    """80,000-pixel non-uniform-Teff grid: both broadening paths against the FP32 mirror."""
    O = c1["O"]
    d, od = _disp(c1, c1["star"], kind)
    lab = [9150.0, -0.41, 3.72, vsini, rv]
    direct, fft = _models_both_paths(c1["interp"], d, lab)
    ref = od.produce_model(lab, O.F32)
    assert relmax(fft, ref) <= FLUX_TOL
    assert relmax(direct, ref) <= FLUX_TOL


def test_config1_kernel_widths(c1):
    """The widest kernel of the benchmark (vsini 300 km/s) on this grid."""
    P = c1["P"]
    k = P.get_vsini_kernel(300.0, c1["wl"])
    assert 941 <= len(k) <= 947
    k4 = P.get_vsini_kernel(300.0, c1["P"].WlGrid(config4_shape().log_first, config4_shape().log_step, 120000,
                                                   log=True))
    assert 1409 <= len(k4) <= 1419


@pytest.mark.parametrize("vsini", [620.0, 645.0])
def test_config1_unfused_wide_kernel(c1, vsini):
    """Rotation kernels wider than 1,920 taps with the instrument profile take
    the unfused rotation FFT + instrument pass (model and chi2)."""
    O, P = c1["O"], c1["P"]
    star = c1["star"]
    m = len(P.get_vsini_kernel(vsini, c1["wl"]))
    assert 1920 < m <= 2048
    d, od = _disp(c1, star, "fixed")
    lab = [9150.0, -0.41, 3.72, vsini, 25.0]
    gpu = c1["interp"].produce_model(d, *lab)
    ref = od.produce_model(lab, O.F32)
    assert relmax(gpu, ref) <= FLUX_TOL
    cont = P.ChunkContinuumFitter(star.wl, 8, 5, 0.2)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 8, 5, 0.2)
    fitter = c1["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 800.0), (-150.0, 150.0))
    g = fitter.chi2(c1["interp"], star.flux, star.var, [lab])[0]
    r, st = O.chi2(c1["og"], od, oc, star.flux, star.var, np.array([lab]), O.F64)
    assert st[0] == 0
    assert abs(g - r[0]) <= CHI2_TOL * r[0]


def test_config1_chi2_matches_fp64(c1):
    """8 chunks of degree 5 (the benchmark's continuum) at the star and around it."""
    O, P, star = c1["O"], c1["P"], c1["star"]
    d, od = _disp(c1, star, "fixed")
    cont = P.ChunkContinuumFitter(star.wl, 8, 5, 0.2)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 8, 5, 0.2)
    labs = np.array([star.label, [9100.0, -0.25, 3.65, 140.0, 38.0], [8800.0, -0.5, 3.5, 160.0, 45.0],
                     [9300.0, -0.2, 3.8, 300.0, 40.0], [9000.0, -0.3, 3.6, 0.0, 40.0]])
    fitter = c1["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    for dm in (0, 512):
        keep = c1["interp"].direct_max
        try:
            c1["interp"].direct_max = dm
            gpu = np.array(fitter.chi2(c1["interp"], star.flux, star.var, labs))
        finally:
            c1["interp"].direct_max = keep
        ref, st = O.chi2(c1["og"], od, oc, star.flux, star.var, labs, O.F64)
        assert (st == 0).all()
        np.testing.assert_allclose(gpu, ref, rtol=CHI2_TOL)


def _replay(e, stars, P_, I_, seed):
    """GPU fits of stars (batched) and the FP64 oracle's replay on the same draw stream."""
    O, P = e["O"], e["P"]
    disps = [P.FixedResolutionDispersion(s.wl, R, e["wl"]) for s in stars]
    conts = [P.ChunkContinuumFitter(s.wl, 8, 5, 0.2) for s in stars]
    res = P.fit_many(e["interp"], disps, conts, P.PSOSettings(P_, I_), [s.flux for s in stars],
                     [s.var for s in stars], (0.0, 300.0), (-150.0, 150.0), seeds=[seed + i for i in range(len(stars))])
    out = []
    for i, (s, r) in enumerate(zip(stars, res)):
        od = O.Disp(e["og"], O.DISP_FIXED, s.wl, R)
        oc = O.Cont(O.CONT_CHUNK, s.wl, 8, 5, 0.2)
        st = O.settings(P_, I_, (0.0, 300.0), (-150.0, 150.0))
        ref, rc = O.fit(e["og"], od, oc, st, s.flux[None], s.var[None], [seed + i], O.F64, over_stars=False)
        assert rc == 0
        out.append((np.array(r.label.as_list()), r.chi2, ref[0]["label"], ref[0]["chi2"]))
    return out


def test_config1_fit_replay_matches_fp64(c1):
    """Seeded fits of two config-1-shaped stars (64 x 200, 8 chunks of degree
    5, as the benchmark) against the FP64 oracle on the same draws."""
    S = c1["S"]
    labs = np.array([[7820.6, -0.9129, 3.3101, 63.01, -59.33], [9744.5, -0.7158, 3.9645, 31.12, 102.74]])
    stars = S.make_stars(c1["spec"], labs, [45000, 50000], [150.0, 120.0], R, seed=31)
    for lab, chi2, rl, rchi2 in _replay(c1, stars, 64, 200, seed=99):
        assert (np.abs(lab - rl) <= LABEL_TOL).all(), (lab, rl)
        assert abs(chi2 - rchi2) <= 1e-5 * rchi2


# ------------------------------------------------------------ config-4 shape
@pytest.mark.parametrize("tml", [(None, -0.6, 3.3), (None, -1.5, 3.1), (None, 0.4, 3.7)])
def test_config4_interpolate_includes_factor(c4, tml):
    """Cubic interpolation on an includes_factor grid (f32 maximum per model)
    at 120,000 pixels, the 64-pixel tail included."""
    O, spec = c4["O"], c4["spec"]
    t = float(spec.teffs[3] + 0.37 * (spec.teffs[4] - spec.teffs[3]))
    gpu = c4["interp"].interpolate(t, tml[1], tml[2])
    ref = c4["og"].interpolate(t, tml[1], tml[2], O.F32)
    assert relmax(gpu, ref) <= FLUX_TOL
    tail = spec.n_px % 128
    assert tail == 64
    np.testing.assert_allclose(gpu[-tail:], ref[-tail:], rtol=1e-5, atol=1e-5 * np.abs(ref).max())


@pytest.mark.parametrize("vsini,rv", [(0.0, 10.0), (8.0, -120.0), (120.0, -30.0), (300.0, 150.0)])
def test_config4_produce_model(c4, vsini, rv):
    """includes_factor models broadened by kernels up to ~1,415 taps."""
    O = c4["O"]
    d, od = _disp(c4, c4["star"], "fixed")
    lab = [float(np.mean(c4["spec"].teffs[2:4])), -0.6, 3.3, vsini, rv]
    direct, fft = _models_both_paths(c4["interp"], d, lab)
    ref = od.produce_model(lab, O.F32)
    assert relmax(fft, ref) <= FLUX_TOL
    assert relmax(direct, ref) <= FLUX_TOL


def test_config4_linear_continuum_tensor_cores(c4):
    """chi2 with the 40-column Legendre linear-model continuum (tensor-core
    path and CUDA-core path) against the FP64 oracle."""
    from pasta_b200 import _ffi
    O, P, S, star = c4["O"], c4["P"], c4["S"], c4["star"]
    d, od = _disp(c4, star, "fixed")
    D = S.legendre_design(star.wl, 40)
    cont, oc = P.LinearModelContinuumFitter(D), O.Cont(O.CONT_LINEAR, design=D)
    fitter = c4["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    rng = np.random.default_rng(4)
    base = np.array(star.label)
    labs = np.array([base + [rng.normal(0, 60), rng.normal(0, 0.05), rng.normal(0, 0.05), rng.normal(0, 5),
                             rng.normal(0, 2)] for _ in range(150)])
    labs[:, 3] = np.clip(labs[:, 3], 0.0, 300.0)
    gpu = np.array(fitter.chi2(c4["interp"], star.flux, star.var, labs))
    _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(0))
    try:
        cc = np.array(fitter.chi2(c4["interp"], star.flux, star.var, labs))
    finally:
        _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(1))
    ref, st = O.chi2(c4["og"], od, oc, star.flux, star.var, labs, O.F64)
    assert (st == 0).all()
    np.testing.assert_allclose(gpu, ref, rtol=CHI2_TOL)
    np.testing.assert_allclose(cc, ref, rtol=CHI2_TOL)
    np.testing.assert_allclose(gpu, cc, rtol=CHI2_TOL)


# ------------------------------------------------------------ staircase
STAIRS = [(0, 2), (0, 3), (0, 4), (1, 4), (1, 4), (2, 4), (2, 4), (0, 4), (1, 3)]


@pytest.fixture(scope="module")
def stair():
    from pasta_b200 import synth as S
    spec = dataclasses.replace(S.config0_grid(n_px=20000), logg_limits=STAIRS)
    e = _env(spec)
    e["star"] = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, R, seed=11)
    return e


def _stair_points(spec, n, seed):
    rng = np.random.default_rng(seed)
    t = rng.uniform(spec.teffs[0], spec.teffs[-1], n)
    m = rng.uniform(spec.ms[0], spec.ms[-1], n)
    g = rng.uniform(spec.loggs[0], spec.loggs[-1], n)
    # points on the stair edges and node lines
    edge_t = np.repeat(spec.teffs[1:-1], 3)
    edge_g = np.tile(spec.loggs[[1, 2, 3]], len(spec.teffs) - 2)
    t = np.concatenate([t, edge_t, edge_t + 17.0])
    g = np.concatenate([g, edge_g, edge_g - 0.06])
    m = np.concatenate([m, np.zeros(len(edge_t)), np.full(len(edge_t), 0.23)])
    return np.stack([t, m, g], axis=1)


def test_staircase_geometry(stair):
    """Grid getters of a staircase grid: logg limits, cumulative sizes, bounds and clamps."""
    O, interp, og, spec = stair["O"], stair["interp"], stair["og"], stair["spec"]
    assert interp.logg_limits() == STAIRS
    sizes = [hi - lo + 1 for lo, hi in STAIRS]
    assert interp.cumulative_grid_size() == [int(x) for x in np.concatenate([[0], np.cumsum(sizes)[:-1]])]
    for (t, m, g) in _stair_points(spec, 300, 2):
        assert interp.is_teff_logg_between_bounds(t, g) == og.within(t, m, g)
        if og.within(t, m, g):
            for i in range(3):
                lo, hi = O.limits_at(og, np.array([t, m, g]), i)
                x = [t, m, g][i]
                assert interp.clamp_1d(t, m, g, i) == min(max(x, lo), hi)


def test_staircase_interpolation_matches_oracle(stair):
    """Device neighbour search and cubic weights on a staircase, stair edges
    included: every label inside the grid against the FP32 mirror; labels
    the oracle rejects are rejected."""
    O, interp, og, spec = stair["O"], stair["interp"], stair["og"], stair["spec"]
    from pasta_b200 import _ffi
    pts = _stair_points(spec, 200, 3)
    out = np.empty((len(pts), spec.n_px), np.float32)
    st = np.zeros(len(pts), np.int32)
    lab = np.ascontiguousarray(pts)
    _ffi.check(_ffi.lib().pasta_interpolate(interp._grid._h, _ffi.ptr(lab), len(lab), _ffi.ptr(out), _ffi.ptr(st)))
    n_ok = 0
    for i, (t, m, g) in enumerate(pts):
        try:
            ref = og.interpolate(t, m, g, O.F32)
        except O.OracleError:
            assert st[i] != 0, (t, m, g)
            continue
        assert st[i] == 0, (t, m, g, st[i])
        assert relmax(out[i], ref) <= FLUX_TOL
        n_ok += 1
    assert n_ok >= 80


# a milder staircase (reduced logg ranges at the two coolest and the two
# hottest Teff values) on which a swarm stays inside the interpolation stencil
STAIRS_FIT = [(0, 2), (0, 3), (0, 4), (0, 4), (0, 4), (0, 4), (0, 4), (1, 4), (2, 4)]


def test_staircase_fit_replay(stair):
    """Seeded fits on staircase grids (the swarm clamps at the per-Teff logg
    limits on the device) against the FP64 oracle.  On the harsher staircase
    a particle lands where a neighbour is missing and the reference aborts
    the fit (particleswarm.rs:117, 281); the device fit must fail the same way."""
    import oracle as O
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    for stairs, lab, ok in ((STAIRS_FIT, [6400.0, 0.07, 3.8, 50.0, 20.0], True),
                            (STAIRS, [7130.0, 0.07, 4.02, 50.0, 20.0], False)):
        spec = dataclasses.replace(S.config0_grid(n_px=20000), logg_limits=stairs)
        e = _env(spec) if stairs != STAIRS else stair
        star = S.make_star(spec, lab, 15000, 100.0, R, seed=11)
        d = P.FixedResolutionDispersion(star.wl, R, e["wl"])
        cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
        fitter = e["interp"].get_fitter(d, cont, P.PSOSettings(40, 60), (0.0, 300.0), (-150.0, 150.0))
        od = O.Disp(e["og"], O.DISP_FIXED, star.wl, R)
        oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
        st = O.settings(40, 60, (0.0, 300.0), (-150.0, 150.0))
        ref, rc = O.fit(e["og"], od, oc, st, star.flux[None], star.var[None], [1234], O.F64, over_stars=False)
        if not ok:
            assert rc != 0 and "neighbor" in O.lib().or_last_error().decode()
            with pytest.raises(P.PastaError):
                fitter.fit(e["interp"], star.flux, star.var, seed=1234)
            continue
        assert rc == 0
        r = fitter.fit(e["interp"], star.flux, star.var, seed=1234)
        assert (np.abs(np.array(r.label.as_list()) - ref[0]["label"]) <= LABEL_TOL).all()
        assert abs(r.chi2 - ref[0]["chi2"]) <= 1e-5 * ref[0]["chi2"]


# ------------------------------------------------------------ constraints
@pytest.mark.parametrize("cons", [[("fix", 1, 0.07)], [("range", 3, 30.0, 70.0)],
                                  [("fix", 2, 4.0), ("range", 4, 10.0, 30.0)]])
def test_constrained_fit_replay(stair, cons):
    """Single-star fits with FixConstraint / RangeConstraint (bounds.rs:69-130)
    through the device swarm, against the FP64 oracle on the same draws."""
    import oracle as O
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    spec = S.config0_grid(n_px=20000)
    e = stair.get("rect")
    if e is None:
        e = stair["rect"] = _env(spec)
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, R, seed=11)
    pc, oc_ = [], []
    for c in cons:
        if c[0] == "fix":
            pc.append(P.FixConstraint(c[1], c[2]))
            oc_.append((c[1], 1, c[2], c[2]))
        else:
            pc.append(P.RangeConstraint(c[1], c[2], c[3]))
            oc_.append((c[1], 2, c[2], c[3]))
    d = P.FixedResolutionDispersion(star.wl, R, e["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = e["interp"].get_fitter(d, cont, P.PSOSettings(32, 50), (0.0, 300.0), (-150.0, 150.0))
    r = fitter.fit(e["interp"], star.flux, star.var, constraints=pc, seed=4321)
    od = O.Disp(e["og"], O.DISP_FIXED, star.wl, R)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    st = O.settings(32, 50, (0.0, 300.0), (-150.0, 150.0), constraints=oc_)
    ref, rc = O.fit(e["og"], od, oc, st, star.flux[None], star.var[None], [4321], O.F64, over_stars=False)
    assert rc == 0
    lab = np.array(r.label.as_list())
    assert (np.abs(lab - ref[0]["label"]) <= LABEL_TOL).all(), (lab, ref[0]["label"])
    for c in cons:
        if c[0] == "fix":
            assert lab[c[1]] == c[2]
        else:
            assert c[2] <= lab[c[1]] <= c[3]
