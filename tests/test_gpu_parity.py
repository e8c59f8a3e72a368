"""GPU parity: the CUDA path (through the C ABI / drop-in module) against the
CPU oracle on the same seeded inputs.

Tolerances (stated per test):
* model flux (interpolate, produce_model): vs the oracle's FP32 mirror,
  max |gpu - ref| <= 1e-5 * max |ref| over the spectrum.
* chi2: vs the oracle's FP64 mode, relative 1e-5.
* seeded PSO replay: vs the oracle on the same draw stream, dTeff <= 1 K,
  d[M/H], dlogg <= 1e-3, dvsini, dRV <= 0.01 km/s.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLUX_TOL = 1e-5
CHI2_TOL = 1e-5


@pytest.fixture(scope="module")
def env():
    import oracle as O
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S

    spec = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    og = O.Grid(labels, spectra, factors, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, 85000.0, seed=11)
    return dict(O=O, P=P, S=S, spec=spec, labels=labels, spectra=spectra, interp=interp, og=og, star=star, wl=wl)


def relmax(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


LABELS3 = [(7130.0, 0.07, 4.02), (6000.0, -0.5, 3.5), (8000.0, 0.5, 4.5), (6250.0, 0.0, 3.75),
           (6010.0, -0.49, 4.49), (7999.0, 0.41, 3.61), (7000.0, 0.1, 4.0)]


@pytest.mark.parametrize("tml", LABELS3)
def test_interpolate_matches_oracle(env, tml):
    gpu = env["interp"].interpolate(*tml)
    ref = env["og"].interpolate(*tml, env["O"].F32)
    assert gpu.shape == ref.shape
    assert relmax(gpu, ref) <= FLUX_TOL


def test_interpolate_at_node_is_the_model(env):
    i = 200
    t, m, g = env["labels"][i]
    gpu = env["interp"].interpolate(t, m, g)
    n = len(gpu) - len(gpu) % 128
    assert np.abs(gpu[:n] - env["spectra"][i][:n] / 65535.0).max() < 1e-6


@pytest.mark.parametrize("disp_kind", ["fixed", "none", "variable"])
@pytest.mark.parametrize("vsini,rv", [(0.0, 0.0), (3.0, -40.0), (50.0, 20.0), (180.0, 120.0), (300.0, -149.0)])
def test_produce_model_matches_oracle(env, disp_kind, vsini, rv):
    O, P, star = env["O"], env["P"], env["star"]
    if disp_kind == "fixed":
        d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
        od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    elif disp_kind == "none":
        d = P.NoConvolutionDispersion(star.wl, env["wl"])
        od = O.Disp(env["og"], O.DISP_NONE, star.wl)
    else:
        sig = (star.wl / np.linspace(60000.0, 90000.0, len(star.wl)) / 2.355).astype(np.float32)
        d = P.VariableResolutionDispersion(star.wl, sig, env["wl"])
        od = O.Disp(env["og"], O.DISP_VARIABLE, star.wl, disp=sig)
    lab = [7130.0, 0.07, 4.02, vsini, rv]
    gpu = env["interp"].produce_model(d, *lab)
    ref = od.produce_model(lab, O.F32)
    assert relmax(gpu, ref) <= FLUX_TOL


@pytest.mark.parametrize("disp_kind", ["fixed", "none", "variable"])
@pytest.mark.parametrize("vsini,rv", [(0.0, 0.0), (3.0, -40.0), (20.0, 10.0), (50.0, 20.0), (140.0, -90.0)])
def test_direct_broadening_matches_fft_and_oracle(env, disp_kind, vsini, rv):
    """The direct-convolution path (narrow kernels) and the FFT path give the
    same model: forced on and off, both against the oracle's FP32 mirror."""
    O, P, star = env["O"], env["P"], env["star"]
    if disp_kind == "fixed":
        d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
        od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    elif disp_kind == "none":
        d = P.NoConvolutionDispersion(star.wl, env["wl"])
        od = O.Disp(env["og"], O.DISP_NONE, star.wl)
    else:
        sig = (star.wl / np.linspace(60000.0, 90000.0, len(star.wl)) / 2.355).astype(np.float32)
        d = P.VariableResolutionDispersion(star.wl, sig, env["wl"])
        od = O.Disp(env["og"], O.DISP_VARIABLE, star.wl, disp=sig)
    lab = [7130.0, 0.07, 4.02, vsini, rv]
    interp = env["interp"]
    keep = interp.direct_max
    try:
        interp.direct_max = 512
        direct = interp.produce_model(d, *lab)
        interp.direct_max = 0
        fft = interp.produce_model(d, *lab)
    finally:
        interp.direct_max = keep
    ref = od.produce_model(lab, O.F32)
    assert relmax(direct, ref) <= FLUX_TOL
    assert relmax(fft, ref) <= FLUX_TOL
    assert relmax(direct, fft) <= FLUX_TOL


def test_direct_crossover_is_measured(env):
    v = env["interp"].direct_max
    assert 0 <= v <= 512
    print("direct/FFT crossover on this device: %d taps" % v)


def _fitters(env, kind):
    O, P, star, S = env["O"], env["P"], env["star"], env["S"]
    n = len(star.wl)
    if kind == "chunk":
        return P.ChunkContinuumFitter(star.wl, 5, 8, 0.2), O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    if kind == "chunk12":
        return P.ChunkContinuumFitter(star.wl, 12, 3, 0.25), O.Cont(O.CONT_CHUNK, star.wl, 12, 3, 0.25)
    if kind == "linear":
        D = S.legendre_design(star.wl, 40)
        return P.LinearModelContinuumFitter(D), O.Cont(O.CONT_LINEAR, design=D)
    if kind == "fixed":
        c = (1.0 + 0.1 * np.linspace(-1, 1, n)).astype(np.float32)
        return P.FixedContinuum(c, 10), O.Cont(O.CONT_FIXED, continuum=c, ignore=10)
    return P.ConstantContinuum(), O.Cont(O.CONT_CONSTANT, n=n)


@pytest.mark.parametrize("kind", ["chunk", "chunk12", "linear", "fixed", "constant"])
def test_chi2_matches_oracle_f64(env, kind):
    O, P, star = env["O"], env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    cont, oc = _fitters(env, kind)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0, 300), (-150, 150))
    labs = np.array([list(star.label), [7100.0, 0.0, 4.1, 40.0, 15.0], [6600.0, -0.3, 3.8, 120.0, -60.0],
                     [7900.0, 0.45, 4.45, 0.0, 0.0]])
    gpu = np.array(fitter.chi2(env["interp"], star.flux, star.var, labs))
    ref, st = O.chi2(env["og"], od, oc, star.flux, star.var, labs, O.F64)
    assert (st == 0).all()
    np.testing.assert_allclose(gpu, ref, rtol=CHI2_TOL)


def test_chi2_errors_are_nan(env):
    O, P, star = env["O"], env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0, 300), (-150, 150))
    labs = [[9000.0, 0.0, 4.0, 10.0, 0.0],   # outside the grid
            [7000.0, 0.0, 4.0, -1.0, 0.0],   # vsini < 0
            [7000.0, 0.0, 4.0, 10.0, 9000.0],  # RV leaves the synthetic grid
            [7000.0, 0.0, 4.0, 10.0, 0.0]]
    out = fitter.chi2(env["interp"], star.flux, star.var, labs)
    assert np.isnan(out[:3]).all() and np.isfinite(out[3])
    with pytest.raises(P.PastaError):
        fitter.chi2(env["interp"], star.flux, star.var, labs, allow_nan=False)


def test_fit_replay_matches_oracle(env):
    """Seeded PSO on the shared draw stream: GPU batched vs oracle (FP64 and FP32 mirror)."""
    O, P, star = env["O"], env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    settings = P.PSOSettings(40, 60)
    fitter = env["interp"].get_fitter(d, cont, settings, (0.0, 300.0), (-150.0, 150.0))
    r = fitter.fit(env["interp"], star.flux, star.var, seed=1234)
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    st = O.settings(40, 60, (0.0, 300.0), (-150.0, 150.0))
    ref, rc = O.fit(env["og"], od, oc, st, star.flux[None], star.var[None], [1234], O.F64, over_stars=False)
    assert rc == 0
    lab = np.array(r.label.as_list())
    rl = ref[0]["label"]
    tol = np.array([1.0, 1e-3, 1e-3, 0.01, 0.01])
    assert (np.abs(lab - rl) <= tol).all(), (lab, rl)
    assert abs(r.chi2 - ref[0]["chi2"]) <= 1e-5 * ref[0]["chi2"]
    assert r.iterations == 60 and len(r.continuum_params) == 45


def test_plain_and_batched_agree(env):
    P, star = env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(24, 15), (0.0, 300.0), (-150.0, 150.0))
    a = fitter.fit(env["interp"], star.flux, star.var, seed=99, mode=0)
    b = fitter.fit(env["interp"], star.flux, star.var, seed=99, mode=1)
    assert a.label.as_list() == b.label.as_list()
    assert a.chi2 == b.chi2


def test_fit_bulk_is_each_star_alone(env):
    P, S, spec = env["P"], env["S"], env["spec"]
    star = env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(16, 8), (0.0, 300.0), (-150.0, 150.0))
    labs = S.random_labels(spec, 3, seed=5, vsini=(0, 100), rv=(-50, 50))
    stars = [S.make_star(spec, l, len(star.wl), 80.0, 85000.0, seed=20 + i) for i, l in enumerate(labs)]
    # same wavelengths for all (fit_bulk shares the fitter)
    fl = np.stack([s.flux for s in stars])
    vr = np.stack([s.var for s in stars])
    bulk = fitter.fit_bulk(env["interp"], fl, vr, seeds=[1, 2, 3])
    for i in range(3):
        one = fitter.fit(env["interp"], fl[i], vr[i], seed=i + 1)
        assert bulk[i].label.as_list() == one.label.as_list()
        assert bulk[i].chi2 == one.chi2


def test_server_result_same_alone_and_in_mix(env):
    P, S, spec = env["P"], env["S"], env["spec"]
    interp = env["interp"]
    labs = S.random_labels(spec, 5, seed=8, vsini=(0, 150), rv=(-80, 80))
    reqs = []
    for i, l in enumerate(labs):
        n = 6000 + 1500 * i
        st = S.make_star(spec, l, n, 60.0, 85000.0, seed=40 + i)
        d = P.FixedResolutionDispersion(st.wl, 85000.0, env["wl"])
        c = P.ChunkContinuumFitter(st.wl, 4 + i, 3 + i % 4, 0.2)
        reqs.append((d, c, st))
    settings = P.PSOSettings(16, 10)
    # alone
    alone = []
    for (d, c, st) in reqs:
        fitter = interp.get_fitter(d, c, settings, (0.0, 300.0), (-150.0, 150.0))
        alone.append(fitter.fit(interp, st.flux, st.var, seed=77))
    # in the mix, staggered arrivals
    srv = P.Server(interp, max_slots=3)
    ids = []
    done = {}
    pending = list(range(len(reqs)))
    step = 0
    while len(done) < len(reqs):
        if pending and step % 3 == 0:
            i = pending.pop(0)
            d, c, st = reqs[i]
            ids.append(srv.submit(d, c, settings, st.flux, st.var, (0.0, 300.0), (-150.0, 150.0), seed=77))
        srv.step()
        for rid, status, res in srv.poll():
            assert status == 0
            done[rid] = res
        step += 1
        assert step < 1000
    for i, rid in enumerate(ids):
        assert done[rid].label.as_list() == alone[i].label.as_list()
        assert done[rid].chi2 == alone[i].chi2
        # the server refits inside its step graph, the batched fit after its last step
        assert done[rid].continuum_params == alone[i].continuum_params


def test_continuum_utilities(env):
    O, P, star = env["O"], env["P"], env["star"]
    og = env["og"]
    od = O.Disp(og, O.DISP_FIXED, star.wl, 85000.0)
    model = od.produce_model(star.label, O.F32).astype(np.float32)
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    params, chi2 = cont.fit_continuum(model, star.flux, star.var)
    rp, rchi2 = oc.fit(star.flux, star.var, model, O.F64)
    assert abs(chi2 - rchi2) <= CHI2_TOL * rchi2
    c_gpu = cont.build_continuum(params)
    c_ref = oc.build(rp, O.F64)
    assert relmax(c_gpu, c_ref) < 1e-4


def test_dispersion_convolve_matches_oracle(env):
    O, P, star = env["O"], env["P"], env["star"]
    x = env["og"].interpolate(7130.0, 0.07, 4.02, O.F32)
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    assert relmax(d.convolve(x), od.convolve(x, O.F32)) <= FLUX_TOL


def test_compute_uncertainty_matches_oracle(env):
    """Chi2-landscape bounds (fitting.rs:480-568): batched GPU Brent vs the oracle's sequential one."""
    O, P, star = env["O"], env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(8, 2), (0.0, 300.0), (-150.0, 150.0))
    sr = np.array([0.05, 0.3, 0.3, 0.5, 40.0])
    u = fitter.compute_uncertainty(env["interp"], star.flux, star.var, 85000.0, star.label, sr)
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    ref = O.compute_uncertainty(env["og"], od, oc, star.flux, star.var, 85000.0, star.label, sr)
    radius = sr * np.array([star.label[0], 1, 1, 1, 1])
    radius[3] = max(star.label[3] * sr[3], 100.0)
    got = [u.teff, u.m, u.logg, u.vsini, u.rv]
    for i in range(5):
        for a, b in zip(got[i], ref[i]):
            assert (a is None) == (b is None), (i, got[i], ref[i])
            if a is not None:
                assert abs(a - b) <= 5e-3 * radius[i], (i, a, b)
    # the bulk form runs every search of every spectrum together; each result
    # is the one computed alone
    other = env["S"].make_star(env["spec"], [6900.0, -0.1, 4.1, 30.0, -10.0], 15000, 100.0, 85000.0, seed=12)
    assert len(other.flux) == len(star.flux)
    bulk = fitter.compute_uncertainty_bulk(env["interp"], [star.flux, other.flux], [star.var, other.var], 85000.0,
                                           [star.label, other.label], sr)
    assert bulk[0].to_dict() == u.to_dict()
    alone = fitter.compute_uncertainty(env["interp"], other.flux, other.var, 85000.0, other.label, sr)
    assert bulk[1].to_dict() == alone.to_dict()
    assert set(u.to_dict()) == {"teff", "m", "logg", "vsini", "rv"}


def test_server_run_counts_steps_and_evaluations(env):
    P, star = env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    srv = P.Server(env["interp"], max_slots=4)
    for k in range(2):
        srv.submit(d, cont, P.PSOSettings(8, 30), star.flux, star.var, (0.0, 300.0), (-150.0, 150.0), seed=5 + k)
    ms = srv.run(3)
    st = srv.stats()
    assert ms > 0.0
    assert st["steps"] == 3 and st["evals"] == 3 * 2 * 8


def test_grouped_interpolation_is_each_label_alone(env):
    """Labels in one grid cube share their neighbour rows (grouped in k_interp on the
    CUDA cores); each model must be bit-identical to the label evaluated alone, and
    match the oracle.  The tensor-core groups (a different summation order) are
    held off here; their own tests compare them with this path."""
    O, P, star = env["O"], env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    rng = np.random.default_rng(3)
    lab = np.array([[7100.0 + 20 * rng.random(), 0.05 + 0.02 * rng.random(), 4.0 + 0.03 * rng.random(),
                     40.0 + 20 * rng.random(), 15.0 + 10 * rng.random()] for _ in range(9)])
    lab = np.vstack([lab, [[6600.0, -0.2, 3.8, 10.0, -30.0], [7600.0, 0.3, 4.3, 120.0, 60.0]]])
    keep = env["interp"].tc_min
    env["interp"].tc_min = 65
    try:
        bulk = env["interp"].produce_model_bulk(d, lab)
        alones = [env["interp"].produce_model(d, *l) for l in lab]
    finally:
        env["interp"].tc_min = keep
    for i, l in enumerate(lab):
        alone = alones[i]
        np.testing.assert_array_equal(bulk[i], alone)
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    for i in (0, 4, 9):
        assert relmax(bulk[i], od.produce_model(lab[i], O.F32)) <= FLUX_TOL


def _resample_rv0(x, wl_obs, log_first, log_step):
    """shift_and_resample at RV 0 on a Logspace grid (convolve_rv.rs:569-590), numpy."""
    idx = (np.log10(wl_obs) - log_first) / log_step
    j = np.floor(idx).astype(np.int64)
    w = idx.astype(np.float32) - j.astype(np.float32)
    x = np.asarray(x, np.float32)
    return (np.float32(1.0) - w) * x[j] + w * x[j + 1]


def test_convolve_and_resample_directory(env, tmp_path):
    """Grid pre-convolution (lib.rs:686-755) with and without the f32 maximum prefix."""
    O, P, S, star = env["O"], env["P"], env["S"], env["star"]
    spec = env["spec"]
    labels, spectra = env["labels"][:3], env["spectra"][:3]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    for with_factor in (False, True):
        src, dst = tmp_path / ("in%d" % with_factor), tmp_path / ("out%d" % with_factor)
        os.makedirs(dst)
        maxima = np.array([1.5, 0.8, 2.25], np.float32) if with_factor else None
        S.write_grid_dir(str(src), labels, spectra, maxima)
        d.convolve_and_resample_directory(str(src), str(dst), with_factor, env["wl"])
        for i, (t, m, g) in enumerate(labels):
            name = S.filename_from_labels(t, m, g)
            got = np.load(os.path.join(dst, name))
            x = spectra[i].astype(np.float32) / np.float32(65535.0)
            if with_factor:
                x = x * maxima[i]
            ref = _resample_rv0(od.convolve(x, O.F32), star.wl, spec.log_first, spec.log_step).astype(np.float32)
            assert relmax(d.convolve_and_resample_spectra(x[None], env["wl"])[0], ref) <= FLUX_TOL
            if with_factor:
                mx = np.frombuffer(got[:2].tobytes(), dtype="<f4")[0]
                assert abs(mx - ref.max()) <= 1e-5 * ref.max()
                expect = np.trunc(np.maximum(ref, 0) / ref.max() * np.float32(65535.0))
                body = got[2:]
            else:
                expect = np.trunc(np.clip(ref, 0, 1) * np.float32(65535.0))
                body = got
            assert body.dtype == np.uint16 and len(body) == len(star.wl)
            assert np.abs(body.astype(np.int64) - expect.astype(np.int64)).max() <= 2
        # existing outputs are kept
        before = os.path.getmtime(os.path.join(dst, S.filename_from_labels(*labels[0])))
        d.convolve_and_resample_directory(str(src), str(dst), with_factor, env["wl"])
        assert os.path.getmtime(os.path.join(dst, S.filename_from_labels(*labels[0]))) == before


@pytest.mark.parametrize("k", [12, 40, 64])
def test_linear_continuum_tensor_core_many_labels(env, k):
    """Linear-model continua run as tcgen05 tf32 (split hi/lo) products per
    group of 128 evaluations: chi2 of 300 random labels (three groups).

    The broadening path is pinned (the timed direct/FFT crossover can fall
    either way on this small grid).  Direct convolution for every kernel:
    against the CUDA-core path on the same models relative 5e-6, against the
    FP64 oracle relative 3e-5 (NaN where the oracle's 64-column solve
    breaks down), good fits (chi2 < 1000) 1e-5.  FFT blocks for every
    kernel: good fits 1e-5.  The narrow-kernel labels that fit badly (chi2
    up to 1e9) are ill-conditioned in the model: the FFT's f32 roundoff of
    4e-7 in the flux moves their chi2 by up to 1e-2 at 12-40 columns and 0.3
    at 64, and the oracle's own FP32 mirror of the reference deviates from
    its FP64 mode by up to 2.4% (7e12 where FP64 gives NaN), so they carry
    no tolerance on that path beyond being finite."""
    from pasta_b200 import _ffi
    O, P, S, star, interp = env["O"], env["P"], env["S"], env["star"], env["interp"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    D = S.legendre_design(star.wl, k)
    cont, oc = P.LinearModelContinuumFitter(D), O.Cont(O.CONT_LINEAR, design=D)
    rng = np.random.default_rng(k)
    labs = np.stack([rng.uniform(6000, 8000, 300), rng.uniform(-0.5, 0.5, 300), rng.uniform(3.5, 4.5, 300),
                     rng.uniform(0, 200, 300), rng.uniform(-100, 100, 300)], axis=1)
    fitter = interp.get_fitter(d, cont, P.PSOSettings(8, 2), (0, 300), (-150, 150))
    saved = interp.direct_max
    try:
        interp.direct_max = 512  # every kernel of the test (at most 512 taps) convolved directly
        gpu = np.array(fitter.chi2(interp, star.flux, star.var, labs))
        _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(0))
        try:
            cuda_cores = np.array(fitter.chi2(interp, star.flux, star.var, labs))
        finally:
            _ffi.check(_ffi.lib().pasta_set_linear_tensor_cores(1))
        interp.direct_max = 0  # every kernel through the FFT blocks
        gpu_fft = np.array(fitter.chi2(interp, star.flux, star.var, labs))
    finally:
        interp.direct_max = saved
    np.testing.assert_allclose(gpu, cuda_cores, rtol=5e-6)
    ref, st = O.chi2(env["og"], od, oc, star.flux, star.var, labs, O.F64)
    assert (st == 0).all()
    np.testing.assert_allclose(gpu, ref, rtol=3e-5)
    good = ref < 1000.0
    np.testing.assert_allclose(gpu[good], ref[good], rtol=CHI2_TOL)
    np.testing.assert_allclose(gpu_fft[good], ref[good], rtol=CHI2_TOL)
    assert (np.isfinite(gpu_fft) | ~np.isfinite(ref)).all()


def test_linear_continuum_fit_params(env):
    """A fit with a linear-model continuum: the continuum parameters of the
    result against the oracle's fit at the returned label."""
    O, P, S, star = env["O"], env["P"], env["S"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    od = O.Disp(env["og"], O.DISP_FIXED, star.wl, 85000.0)
    D = S.legendre_design(star.wl, 40)
    cont, oc = P.LinearModelContinuumFitter(D), O.Cont(O.CONT_LINEAR, design=D)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(16, 4), (0, 300), (-150, 150))
    r = fitter.fit(env["interp"], star.flux, star.var, seed=77)
    lab = r.label.as_list()
    mdl = od.produce_model(lab, O.F64)
    params, chi2 = oc.fit(star.flux, star.var, mdl, O.F64)
    assert len(r.continuum_params) == 40
    np.testing.assert_allclose(r.continuum_params, params, rtol=1e-3, atol=1e-4 * np.abs(params).max())
    assert abs(r.chi2 - chi2) <= 1e-4 * chi2


def test_server_budget_makes_requests_wait(env):
    """Admission by HBM budget: with room for two running requests, the third
    and fourth wait in the queue until earlier ones retire, never more than
    two run at once, and every result is the one the star gets alone."""
    P, S, spec = env["P"], env["S"], env["spec"]
    interp = env["interp"]
    labs = S.random_labels(spec, 4, seed=19, vsini=(0, 150), rv=(-80, 80))
    reqs = []
    for i, l in enumerate(labs):
        st = S.make_star(spec, l, 8000, 60.0, 85000.0, seed=60 + i)
        reqs.append((P.FixedResolutionDispersion(st.wl, 85000.0, env["wl"]),
                     P.ChunkContinuumFitter(st.wl, 5, 4, 0.2), st))
    settings = P.PSOSettings(16, 6)
    probe = P.Server(interp, max_slots=4)
    budget0, used0 = probe.memory()
    assert budget0 > 0 and used0 == 0
    d, c, st = reqs[0]
    probe.submit(d, c, settings, st.flux, st.var, (0.0, 300.0), (-150.0, 150.0), seed=3)
    probe.step()
    per_request = probe.memory()[1]
    assert per_request > 16 * 20000 * 4  # the particles' evaluation workspace is counted
    del probe
    srv = P.Server(interp, max_slots=4, hbm_budget_bytes=int(2.5 * per_request))
    ids = [srv.submit(d, c, settings, st.flux, st.var, (0.0, 300.0), (-150.0, 150.0), seed=300 + i)
           for i, (d, c, st) in enumerate(reqs)]
    done, waited, steps = {}, False, 0
    while len(done) < len(reqs):
        srv.step()
        q, a, _ = srv.pending()
        assert a <= 2
        waited |= q > 0 and a == 2
        assert srv.memory()[1] <= int(2.5 * per_request)
        for rid, status, res in srv.poll():
            assert status == 0
            done[rid] = res
        steps += 1
        assert steps < 200
    assert waited
    for i, (d, c, st) in enumerate(reqs):
        alone = interp.get_fitter(d, c, settings, (0.0, 300.0), (-150.0, 150.0)).fit(interp, st.flux, st.var,
                                                                                    seed=300 + i)
        assert done[ids[i]].label.as_list() == alone.label.as_list()
        assert done[ids[i]].chi2 == alone.chi2


def test_interpolation_tensor_cores(env):
    """Labels of one star that share their 64 neighbour rows (16 or more)
    are interpolated on the tensor cores: each model against the oracle's
    FP32 mirror (1e-5 of the maximum) and against the CUDA-core path (2e-6),
    the reference's 1/65535 tail included; a member's result does not depend
    on the other members of its group; scattered labels stay exact."""
    from pasta_b200 import _ffi
    O, S, interp, og, spec = env["O"], env["S"], env["interp"], env["og"], env["spec"]
    rng = np.random.default_rng(9)
    cube = np.stack([rng.uniform(7010.0, 7240.0, 40), rng.uniform(0.01, 0.09, 40), rng.uniform(4.01, 4.24, 40)], 1)
    scat = S.random_labels(spec, 8, seed=3)[:, :3]
    lab = np.vstack([cube, scat])
    keep = interp.tc_min
    assert 8 <= keep <= 65
    interp.tc_min = 16
    try:
        tc = interp.interpolate_bulk(lab)
        half = interp.interpolate_bulk(cube[:20])
        _ffi.check(_ffi.lib().pasta_set_interp_tensor_cores(0))
        try:
            cc = interp.interpolate_bulk(lab)
        finally:
            _ffi.check(_ffi.lib().pasta_set_interp_tensor_cores(1))
    finally:
        interp.tc_min = keep
    for i in range(len(lab)):
        ref = og.interpolate(*lab[i], O.F32)
        assert relmax(tc[i], ref) <= FLUX_TOL, i
    assert np.abs(tc - cc).max() <= 2e-6 * np.abs(cc).max()
    np.testing.assert_array_equal(tc[40:], cc[40:])  # scattered labels: CUDA cores either way
    np.testing.assert_array_equal(half, tc[:20])
    print("tensor-core group threshold measured on this device: %d members" % keep)


def test_tensor_core_groups_with_own_windows(env):
    """A 64-member tensor-core group (one star's whole swarm in one grid cube)
    whose members have their own RV shifts and so their own interpolation
    windows: each model against the CUDA-core path (2e-6 of the maximum) and
    the oracle (1e-5), the window edges included."""
    from pasta_b200 import _ffi
    O, P, star, og, interp = env["O"], env["P"], env["star"], env["og"], env["interp"]
    rng = np.random.default_rng(21)
    lab = np.stack([rng.uniform(7010.0, 7240.0, 64), rng.uniform(0.01, 0.09, 64), rng.uniform(4.01, 4.24, 64),
                    rng.uniform(0.0, 60.0, 64), rng.uniform(-140.0, 140.0, 64)], 1)
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    keep = interp.tc_min
    interp.tc_min = 16
    try:
        tc = interp.produce_model_bulk(d, lab)
        _ffi.check(_ffi.lib().pasta_set_interp_tensor_cores(0))
        try:
            cc = interp.produce_model_bulk(d, lab)
        finally:
            _ffi.check(_ffi.lib().pasta_set_interp_tensor_cores(1))
    finally:
        interp.tc_min = keep
    assert np.abs(tc - cc).max() <= 2e-6 * np.abs(cc).max()
    od = O.Disp(og, O.DISP_FIXED, star.wl, resolution=85000.0)
    for i in range(0, 64, 7):
        ref = od.produce_model(lab[i], O.F32)
        assert relmax(tc[i], ref) <= FLUX_TOL, i


def test_ccf_matches_oracle(env):
    """ccf (lib.rs:1340-1371): the unbroadened model shifted to each velocity
    and resampled onto the observed wavelengths, dotted with the flux on the
    device; against the oracle's FP64 model at each velocity and an FP64 dot
    product (1e-5), a failing velocity raises, and the length check."""
    O, P, star, og = env["O"], env["P"], env["star"], env["og"]
    vs = np.linspace(-120.0, 120.0, 25)
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    got = env["interp"].ccf(vs, 7130.0, 0.07, 4.02, d, star.flux)
    od = O.Disp(og, O.DISP_NONE, star.wl)
    ref = np.array([np.dot(od.produce_model([7130.0, 0.07, 4.02, 0.0, v], O.F64).astype(np.float64),
                           star.flux.astype(np.float64)) for v in vs])
    np.testing.assert_allclose(got, ref, rtol=1e-5)
    assert np.argmax(got) == np.argmax(ref)
    with pytest.raises(ValueError):
        env["interp"].ccf(vs, 7130.0, 0.07, 4.02, d, star.flux[:-1])
    with pytest.raises(P.PastaError):
        env["interp"].ccf([0.0, 5.0e5], 7130.0, 0.07, 4.02, d, star.flux)


def test_chi2_bulk_one_batched_pass(env):
    """chi2_bulk (lib.rs:1297-1338): spectra with their own wavelength grids,
    a no-convolution dispersion and a 5 x 8 x 0.2 chunk fitter each, in one
    batched pass; against the FP64 oracle and against each spectrum alone."""
    O, P, S, spec, interp = env["O"], env["P"], env["S"], env["spec"], env["interp"]
    labs = np.array([[7130.0, 0.07, 4.02, 30.0, 20.0], [6600.0, -0.3, 3.8, 0.0, -40.0],
                     [7700.0, 0.3, 4.3, 120.0, 60.0]])
    stars = [S.make_star(spec, l, n, 90.0, 0.0, seed=70 + i) for i, (l, n) in enumerate(zip(labs, [9000, 12000, 7000]))]
    got = interp.chi2_bulk([s.wl for s in stars], [s.flux for s in stars], [s.var for s in stars], labs)
    for i, s in enumerate(stars):
        od = O.Disp(env["og"], O.DISP_NONE, s.wl)
        oc = O.Cont(O.CONT_CHUNK, s.wl, 5, 8, 0.2)
        ref, st = O.chi2(env["og"], od, oc, s.flux, s.var, labs[i][None], O.F64)
        assert st[0] == 0
        assert abs(got[i] - ref[0]) <= CHI2_TOL * ref[0]
        d = P.NoConvolutionDispersion(s.wl, env["wl"])
        f = interp.get_fitter(d, P.ChunkContinuumFitter(s.wl, 5, 8, 0.2), P.PSOSettings(8, 2), (0, 300), (-150, 150))
        alone = f.chi2(interp, s.flux, s.var, [labs[i]])[0]
        assert abs(got[i] - alone) <= 1e-12 * alone
    bad = labs.copy()
    bad[1, 0] = 9000.0  # outside the grid
    out = interp.chi2_bulk([s.wl for s in stars], [s.flux for s in stars], [s.var for s in stars], bad, allow_nan=True)
    assert np.isnan(out[1]) and np.isfinite(out[0]) and np.isfinite(out[2])
    with pytest.raises(P.PastaError):
        interp.chi2_bulk([s.wl for s in stars], [s.flux for s in stars], [s.var for s in stars], bad)


def test_grid_ingest_directory_and_tar(env, tmp_path):
    """InMemInterpolator(dir) / OnDiskInterpolator / CachedInterpolator from a
    directory of .npy models (model_fetchers.rs:136-166) and from a tar
    archive (model_fetchers.rs:168-226), with and without the f32 maximum
    prefix, interpolate exactly like the same grid given as arrays."""
    import tarfile
    P, S = env["P"], env["S"]
    spec = S.config0_grid(n_px=4000)
    for with_factor in (False, True):
        spec.includes_factor = with_factor
        labels, spectra, factors = S.make_grid(spec)
        d = tmp_path / ("grid%d" % with_factor)
        S.write_grid_dir(str(d), labels, spectra, factors)
        wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
        ref = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
        tar = tmp_path / ("grid%d.tar" % with_factor)
        with tarfile.open(tar, "w") as tf:
            tf.add(str(d), arcname="models")
        grids = [P.InMemInterpolator(str(d), with_factor, wl), P.OnDiskInterpolator(str(d), with_factor, wl),
                 P.CachedInterpolator(str(d), with_factor, wl), P.InMemInterpolator.from_tar_zstd(str(tar), with_factor, wl)]
        tml = [(7130.0, 0.07, 4.02), (6010.0, -0.49, 3.51)]
        for g in grids:
            assert g.list_gridpoints() == ref.list_gridpoints()
            for x in tml:
                np.testing.assert_array_equal(g.interpolate(*x), ref.interpolate(*x))


def test_fit_trace_output(env, tmp_path):
    """PSOobserver / BestParticleObserver files (fitting.rs:217-296; lib.rs:837-851):
    one it_<i>.json per iteration with every particle's position and cost, and
    the best particle after every iteration, consistent with the fit result."""
    import json
    P, star = env["P"], env["star"]
    d = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(d, cont, P.PSOSettings(12, 5), (0.0, 300.0), (-150.0, 150.0))
    tdir = tmp_path / "trace"
    r = fitter.fit(env["interp"], star.flux, star.var, trace_directory=str(tdir), seed=31)
    files = sorted(os.listdir(tdir))
    assert files == ["it_%d.json" % i for i in range(5)]
    last = json.load(open(tdir / "it_4.json"))
    assert len(last) == 12 and set(last[0]) == {"position", "cost"} and len(last[0]["position"]) == 5
    best_file = tmp_path / "best.json"
    r2 = fitter.fit(env["interp"], star.flux, star.var, best_particle_file=str(best_file), seed=31)
    hist = json.load(open(best_file))
    assert len(hist) == 5
    costs = [h["cost"] for h in hist]
    assert all(b <= a for a, b in zip(costs, costs[1:]))
    assert r2.label.as_list() == r.label.as_list()
    assert abs(costs[-1] - r2.chi2) <= 1e-9 * r2.chi2 or costs[-1] >= r2.chi2
    with pytest.raises(RuntimeError):
        fitter.fit(env["interp"], star.flux, star.var, trace_directory=str(tdir), best_particle_file=str(best_file))


@pytest.mark.parametrize("run_len", ["1", "3", "16"])
def test_broadening_independent_of_item_runs(env, monkeypatch, run_len):
    """k_broaden hands each CTA runs of consecutive block pairs (their length
    is chosen from the batch size; PASTA_BR_RUN fixes it).  Every block pair
    is computed and resampled by exactly one CTA whatever the runs, so chi2
    and the models are bit-identical for every run length."""
    P, star = env["P"], env["star"]
    disp = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(disp, cont, P.PSOSettings(16, 5), (0.0, 300.0), (-150.0, 150.0))
    rng = np.random.default_rng(23)
    n = 300
    lab = np.stack([rng.uniform(6050, 7950, n), rng.uniform(-0.45, 0.45, n), rng.uniform(3.55, 4.45, n),
                    rng.uniform(0, 300, n), rng.uniform(-140, 140, n)], axis=1)
    monkeypatch.setenv("PASTA_BR_RUN", "1")
    c_ref = np.array(fitter.chi2(env["interp"], star.flux, star.var, lab.tolist()))
    m_ref = env["interp"].produce_model_bulk(disp, lab[:40])
    monkeypatch.setenv("PASTA_BR_RUN", run_len)
    c = np.array(fitter.chi2(env["interp"], star.flux, star.var, lab.tolist()))
    m = env["interp"].produce_model_bulk(disp, lab[:40])
    assert np.isfinite(c_ref).all()
    np.testing.assert_array_equal(c, c_ref)
    np.testing.assert_array_equal(m, m_ref)


def test_merged_interpolation_groups_are_bit_identical(env, monkeypatch):
    """Evaluations alone in their segment (chunks of 64 labels) but with the
    same neighbour columns as evaluations of other segments are interpolated
    together (k_merge / k_interp_merged).  Every member keeps its own
    accumulators and row order, so chi2 and the models are bit-identical with
    the merging switched off (PASTA_INTERP_MERGE=0), and match the oracle."""
    O, P, star = env["O"], env["P"], env["star"]
    disp = P.FixedResolutionDispersion(star.wl, 85000.0, env["wl"])
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = env["interp"].get_fitter(disp, cont, P.PSOSettings(16, 5), (0.0, 300.0), (-150.0, 150.0))
    rng = np.random.default_rng(31)
    n = 512
    lab = np.stack([rng.uniform(6050, 7950, n), rng.uniform(-0.45, 0.45, n), rng.uniform(3.55, 4.45, n),
                    rng.uniform(0, 300, n), rng.uniform(-140, 140, n)], axis=1)
    # one label per segment in the same grid cell (and a second cell), the rest spread
    for k in range(8):
        lab[64 * k + 5] = [7130.0 + 10 * k, 0.07 - 0.01 * k, 4.02 + 0.01 * k, 50.0 + k, 20.0 - k]
        lab[64 * k + 9, :3] = [6310.0 + 5 * k, -0.31, 3.66]
    monkeypatch.setenv("PASTA_INTERP_MERGE", "0")
    c_off = np.array(fitter.chi2(env["interp"], star.flux, star.var, lab.tolist()))
    m_off = env["interp"].produce_model_bulk(disp, lab[:192])
    monkeypatch.setenv("PASTA_INTERP_MERGE", "1")
    c_on = np.array(fitter.chi2(env["interp"], star.flux, star.var, lab.tolist()))
    m_on = env["interp"].produce_model_bulk(disp, lab[:192])
    assert np.isfinite(c_on).all()
    np.testing.assert_array_equal(c_on, c_off)
    np.testing.assert_array_equal(m_on, m_off)
    og = env["og"]
    od = O.Disp(og, O.DISP_FIXED, star.wl, 85000.0)
    oc = O.Cont(O.CONT_CHUNK, star.wl, 5, 8, 0.2)
    idx = [5, 69, 133]
    ref = O.chi2(og, od, oc, star.flux, star.var, lab[idx], O.F64)[0]
    np.testing.assert_allclose(c_on[idx], ref, rtol=CHI2_TOL)
