"""Generates tests/golden/pasta_small.npz with the CPU oracle.

The reference (Rust) cannot be built or run here and ships no golden vectors,
so these fixtures come from the oracle's restatement of its algorithm.  They
pin the oracle and the CUDA path against regressions.  They do not pin either
to the reference's own outputs.

Contents (small: a 5 x 4 x 4 grid of 1,536-pixel models):
  grid_labels, grid_spectra, wl_a, wl_b         the grid (log-uniform)
  obs_wl, obs_flux, obs_var                     one synthetic star
  eval_labels                                   label vectors evaluated
  model_f32                                     produce_model, FP32 mirror, R = 60,000
  chi2_f64                                      chi2, FP64, 4 chunks deg 5
  fit_label, fit_chi2                           seeded PSO (16 x 12), FP64
Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from pasta_b200 import synth as S  # noqa: E402

R = 60000.0


def spec_small():
    return S.GridSpec(teffs=np.array([6000.0, 6500.0, 7000.0, 7500.0, 8000.0]),
                      ms=np.array([-0.4, -0.1, 0.2, 0.5]), loggs=np.array([3.5, 3.8, 4.1, 4.4]),
                      n_px=1536, wl_lo=4400.0, wl_hi=4500.0, n_lines=40, seed=21)


def main():
    spec = spec_small()
    labels, spectra, _ = S.make_grid(spec)
    g = O.Grid(labels, spectra, None, O.WL_LOGSPACE, spec.log_first, spec.log_step)
    star = S.make_star(spec, [6830.0, 0.05, 3.97, 25.0, 12.0], 900, 150.0, R, seed=4, rv_max=60.0,
                       vsini_max=60.0)
    d = O.Disp(g, O.DISP_FIXED, star.wl, R)
    c = O.Cont(O.CONT_CHUNK, star.wl, 4, 5, 0.2)
    ev = np.array([[6830.0, 0.05, 3.97, 25.0, 12.0], [6100.0, -0.3, 3.6, 0.0, 0.0],
                   [7900.0, 0.45, 4.35, 55.0, -40.0], [6500.0, 0.2, 4.1, 10.0, 30.0],
                   [7250.0, -0.05, 3.75, 40.0, -10.0]])
    model = np.stack([d.produce_model(l, O.F32) for l in ev])
    chi2, st = O.chi2(g, d, c, star.flux, star.var, ev, O.F64)
    assert (st == 0).all()
    sett = O.settings(16, 12, (0.0, 60.0), (-60.0, 60.0))
    res, rc = O.fit(g, d, c, sett, star.flux[None], star.var[None], [2024], O.F64, over_stars=False)
    assert rc == 0
    np.savez_compressed(os.path.join(HERE, "pasta_small.npz"), grid_labels=labels, grid_spectra=spectra,
                        wl_a=spec.log_first, wl_b=spec.log_step, obs_wl=star.wl, obs_flux=star.flux,
                        obs_var=star.var, eval_labels=ev, model_f32=model, chi2_f64=chi2,
                        fit_label=res[0]["label"], fit_chi2=res[0]["chi2"], resolution=R, n_chunks=4,
                        p_order=5, overlap=0.2, fit_particles=16, fit_iters=12, fit_seed=2024,
                        vsini_range=[0.0, 60.0], rv_range=[-60.0, 60.0])
    print("wrote", os.path.join(HERE, "pasta_small.npz"))


if __name__ == "__main__":
    main()
