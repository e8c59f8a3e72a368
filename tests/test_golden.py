"""Committed fixtures (tests/golden/pasta_small.npz, made by make_golden.py with
the oracle): the oracle must keep reproducing them (CPU), and the CUDA path
must match them (GPU) within the stated tolerances."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "pasta_small.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_oracle_reproduces_fixtures(gold):
    import oracle as O
    g = O.Grid(gold["grid_labels"], gold["grid_spectra"], None, O.WL_LOGSPACE, float(gold["wl_a"]),
               float(gold["wl_b"]))
    d = O.Disp(g, O.DISP_FIXED, gold["obs_wl"], float(gold["resolution"]))
    c = O.Cont(O.CONT_CHUNK, gold["obs_wl"], int(gold["n_chunks"]), int(gold["p_order"]), float(gold["overlap"]))
    model = np.stack([d.produce_model(l, O.F32) for l in gold["eval_labels"]])
    assert np.abs(model - gold["model_f32"]).max() <= 1e-6 * np.abs(gold["model_f32"]).max()
    chi2, st = O.chi2(g, d, c, gold["obs_flux"], gold["obs_var"], gold["eval_labels"], O.F64)
    np.testing.assert_allclose(chi2, gold["chi2_f64"], rtol=1e-9)
    sett = O.settings(int(gold["fit_particles"]), int(gold["fit_iters"]), tuple(gold["vsini_range"]),
                      tuple(gold["rv_range"]))
    res, rc = O.fit(g, d, c, sett, gold["obs_flux"][None], gold["obs_var"][None], [int(gold["fit_seed"])], O.F64,
                    over_stars=False)
    assert rc == 0
    np.testing.assert_allclose(res[0]["label"], gold["fit_label"], rtol=0, atol=1e-9)


@pytest.mark.gpu
def test_cuda_path_matches_fixtures(gold):
    from pasta_b200 import pasta as P
    wl = P.WlGrid(float(gold["wl_a"]), float(gold["wl_b"]), gold["grid_spectra"].shape[1], log=True)
    interp = P.InMemInterpolator.from_arrays(gold["grid_labels"], gold["grid_spectra"], None, wl)
    d = P.FixedResolutionDispersion(gold["obs_wl"], float(gold["resolution"]), wl)
    c = P.ChunkContinuumFitter(gold["obs_wl"], int(gold["n_chunks"]), int(gold["p_order"]), float(gold["overlap"]))
    model = interp.produce_model_bulk(d, gold["eval_labels"])
    assert np.abs(model - gold["model_f32"]).max() <= 1e-5 * np.abs(gold["model_f32"]).max()
    sett = P.PSOSettings(int(gold["fit_particles"]), int(gold["fit_iters"]))
    fitter = interp.get_fitter(d, c, sett, tuple(gold["vsini_range"]), tuple(gold["rv_range"]))
    chi2 = fitter.chi2(interp, gold["obs_flux"], gold["obs_var"], gold["eval_labels"])
    np.testing.assert_allclose(chi2, gold["chi2_f64"], rtol=1e-5)
    r = fitter.fit(interp, gold["obs_flux"], gold["obs_var"], seed=int(gold["fit_seed"]))
    tol = np.array([1.0, 1e-3, 1e-3, 0.01, 0.01])
    assert (np.abs(np.array(r.label.as_list()) - gold["fit_label"]) <= tol).all()
