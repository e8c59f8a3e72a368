"""GPU parity of the binary-star path (BinaryFitter, produce_binary_model_norm,
interpolate_linear) through the drop-in module against the CPU oracle.

Tolerances (stated per test):
* interpolate_linear: bit-identical to the oracle's FP32 mirror (the same f32
  operations in the same order).
* binary model: vs the FP32 mirror, max |gpu - ref| <= 1e-5 * max |ref|
  (FFT roundoff of the broadening; continuum means summed in f64 on the GPU
  and in f32 order in the mirror).
* chi2: vs the oracle's FP64 mode, relative 1e-5.
* seeded PSO replay: the same initial swarm as the oracle on the shared draw
  stream; final labels vs the FP64 oracle within dTeff <= 1 K, d[M/H],
  dlogg <= 1e-3, dvsini, dRV <= 0.01 km/s, dlight ratio <= 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLUX_TOL = 1e-5
CHI2_TOL = 1e-5
L1 = [7600.0, 0.1, 4.1, 30.0, -40.0]
L2 = [6300.0, -0.2, 3.8, 10.0, 45.0]


@pytest.fixture(scope="module")
def benv():
    import oracle as O
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S

    spec = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec)
    cl, cs, cf = S.make_continuum_grid(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    cinterp = P.InMemInterpolator.from_arrays(cl, cs, cf, wl)
    og = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    ogc = O.Grid(cl, cs, cf, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    star = S.make_binary_star(spec, L1, L2, 0.6, 15000, 150.0, 85000.0, seed=21)
    d = P.FixedResolutionDispersion(star.wl, 85000.0, wl)
    od = O.Disp(og, O.DISP_FIXED, star.wl, 85000.0)
    return dict(O=O, P=P, S=S, spec=spec, interp=interp, cinterp=cinterp, og=og, ogc=ogc, star=star, d=d,
                od=od, cl=cl, cs=cs, cf=cf, wl=wl)


LIN_LABELS = [(7130.0, 0.07, 4.02), (6000.0, -0.5, 3.5), (8000.0, 0.5, 4.5), (6250.0, 0.0, 3.75),
              (6010.0, -0.49, 4.49), (7999.0, 0.41, 3.61)]


@pytest.mark.parametrize("tml", LIN_LABELS)
def test_interpolate_linear_is_bit_identical(benv, tml):
    gpu = benv["cinterp"].interpolate_linear(*tml)
    ref = benv["ogc"].interpolate_linear(*tml, benv["O"].F32)
    np.testing.assert_array_equal(gpu, ref.astype(np.float32))


def test_interpolate_linear_outside_grid_raises(benv):
    with pytest.raises(benv["P"].PastaError):
        benv["cinterp"].interpolate_linear(9000.0, 0.0, 4.0)


@pytest.mark.parametrize("l1,l2,lr", [
    (L1, L2, 0.6),
    ([7130.0, 0.07, 4.02, 0.0, 0.0], [6500.0, -0.1, 3.9, 0.0, 0.0], 0.3),
    ([7900.0, 0.45, 4.45, 250.0, 120.0], [6100.0, -0.45, 3.55, 3.0, -140.0], 0.95),
    (L1, L1, 0.4),
    (L1, L2, 0.0),
])
def test_binary_model_matches_oracle(benv, l1, l2, lr):
    O = benv["O"]
    gpu = benv["interp"].produce_binary_model_norm(benv["cinterp"], benv["d"], l1, l2, lr)
    ref = O.binary_model(benv["og"], benv["ogc"], benv["od"], list(l1) + list(l2) + [lr], O.F32)
    assert gpu.shape == ref.shape
    assert np.abs(gpu - ref).max() / np.abs(ref).max() <= FLUX_TOL


def test_binary_of_identical_stars_is_the_single_model(benv):
    P = benv["P"]
    single = benv["interp"].produce_model(benv["d"], *L1)
    binary = benv["interp"].produce_binary_model_norm(benv["cinterp"], benv["d"], L1, L1, 0.7)
    assert np.abs(binary - single).max() <= 2e-6 * np.abs(single).max()


def _fitters(benv, kind):
    O, P, S, star = benv["O"], benv["P"], benv["S"], benv["star"]
    if kind == "chunk":
        return P.ChunkContinuumFitter(star.wl, 5, 8, 0.2), O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    if kind == "linear":
        D = S.legendre_design(star.wl, 12)
        return P.LinearModelContinuumFitter(D), O.Cont(O.CONT_LINEAR, design=D)
    return P.ConstantContinuum(), O.Cont(O.CONT_CONSTANT, n=len(star.wl))


@pytest.mark.parametrize("kind", ["chunk", "linear", "constant"])
def test_binary_chi2_matches_oracle_f64(benv, kind):
    O, P, star = benv["O"], benv["P"], benv["star"]
    cont, oc = _fitters(benv, kind)
    fitter = benv["interp"].get_binary_fitter(benv["d"], cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    labs = np.array([list(star.label),
                     L1 + [6400.0, -0.1, 3.9, 15.0, 40.0] + [0.55],
                     [7000.0, 0.0, 4.0, 120.0, -60.0, 7900.0, 0.4, 4.4, 0.0, 0.0, 0.2],
                     [6100.0, -0.4, 3.6, 5.0, 100.0, 6200.0, -0.3, 3.7, 250.0, -100.0, 0.9]])
    gpu = np.array(fitter.chi2(benv["interp"], benv["cinterp"], star.flux, star.var, labs))
    ref, st = O.binary_chi2(benv["og"], benv["ogc"], benv["od"], oc, star.flux, star.var, labs, O.F64)
    assert (st == 0).all()
    np.testing.assert_allclose(gpu, ref, rtol=CHI2_TOL)


def test_binary_chi2_errors_are_nan(benv):
    P, star = benv["P"], benv["star"]
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = benv["interp"].get_binary_fitter(benv["d"], cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    ok = list(star.label)
    labs = []
    for k, v in [(5, 9000.0), (3, -1.0), (8, -1.0), (4, 9000.0), (9, -9000.0), (2, 9.0)]:
        x = list(ok)
        x[k] = v
        labs.append(x)
    labs.append(ok)
    out = fitter.chi2(benv["interp"], benv["cinterp"], star.flux, star.var, labs)
    assert np.isnan(out[:-1]).all() and np.isfinite(out[-1])
    with pytest.raises(P.PastaError):
        fitter.chi2(benv["interp"], benv["cinterp"], star.flux, star.var, labs, allow_nan=False)


def test_binary_fit_replay_matches_oracle(benv):
    """Seeded binary PSO on the shared draw stream: the same initial swarm as
    the oracle, and the same best labels as the FP64 oracle."""
    O, P, star = benv["O"], benv["P"], benv["star"]
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    settings = P.PSOSettings(24, 12)
    fitter = benv["interp"].get_binary_fitter(benv["d"], cont, settings, (0.0, 100.0), (-100.0, 100.0))
    r = fitter.fit(benv["interp"], benv["cinterp"], star.flux, star.var, seed=99, _trace=True)
    st = O.binary_settings(24, 12, (0.0, 100.0), (-100.0, 100.0))
    ref, rc, rtr = O.binary_fit(benv["og"], benv["ogc"], benv["od"], oc, st, star.flux, star.var, 99, O.F64,
                                trace=True)
    assert rc == 0, ref["error"]
    # initial positions (sorted by cost) are the same draws
    np.testing.assert_array_equal(np.sort(r._trace[0][:, :11], axis=0), np.sort(rtr[0][:, :11], axis=0))
    tol = np.array([1.0, 1e-3, 1e-3, 0.01, 0.01])
    assert (np.abs(np.array(r.label1.as_list()) - ref["label1"]) <= tol).all(), (r.label1, ref["label1"])
    assert (np.abs(np.array(r.label2.as_list()) - ref["label2"]) <= tol).all(), (r.label2, ref["label2"])
    assert abs(r.light_ratio - ref["light_ratio"]) <= 1e-4
    assert abs(r.chi2 - ref["chi2"]) <= CHI2_TOL * ref["chi2"]
    assert len(r.continuum_params) == 45 and r.iterations == 12


def test_binary_fit_constraints(benv):
    P, star = benv["P"], benv["star"]
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = benv["interp"].get_binary_fitter(benv["d"], cont, P.PSOSettings(12, 3), (0.0, 100.0),
                                              (-100.0, 100.0))
    r = fitter.fit(benv["interp"], benv["cinterp"], star.flux, star.var, seed=5,
                   constraints=[P.FixConstraint(10, 0.6), P.RangeConstraint(0, 7500.0, 7700.0),
                                P.FixConstraint(8, 10.0)])
    assert r.light_ratio == 0.6 and r.label2.vsini == 10.0
    assert 7500.0 <= r.label1.teff <= 7700.0
    d = r.to_dict()
    r2 = P.BinaryOptimizationResult.from_dict(d)
    assert r2.to_json() == r.to_json()


def test_binary_fit_graph_replay_equals_eager(benv, monkeypatch):
    """Each binary fit captures its per-iteration evaluation once as a CUDA
    graph and replays it; with PASTA_NO_GRAPH set the same launches run
    eagerly.  Same kernels in the same order: bit-identical trajectories."""
    P, star = benv["P"], benv["star"]
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = benv["interp"].get_binary_fitter(benv["d"], cont, P.PSOSettings(16, 6), (0.0, 100.0),
                                              (-100.0, 100.0))
    graph = fitter.fit(benv["interp"], benv["cinterp"], star.flux, star.var, seed=31, _trace=True)
    monkeypatch.setenv("PASTA_NO_GRAPH", "1")
    eager = fitter.fit(benv["interp"], benv["cinterp"], star.flux, star.var, seed=31, _trace=True)
    np.testing.assert_array_equal(graph._trace, eager._trace)
    assert graph.label1.as_list() == eager.label1.as_list() and graph.label2.as_list() == eager.label2.as_list()
    assert graph.light_ratio == eager.light_ratio and graph.chi2 == eager.chi2
    np.testing.assert_array_equal(graph.continuum_params, eager.continuum_params)
