"""pasta_chi2_noalloc: chi2 for callers that cannot allocate device memory
(a host that gives the GPU's whole memory to its own pool, a real-time loop
that may not call cudaMalloc, a service with a fixed footprint).  The caller
owns every input and output buffer on the device; the library's workspace is
a static device array of fixed size.

Checked against the regular entry point pasta_chi2 (same tolerance as the
other chi2 tests: relative 1e-5) on two calls in a row, and the size limit is
enforced.  This file runs last so that a failure here cannot hide another
test's result; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHI2_TOL = 1e-5


def test_chi2_without_allocation_matches_pasta_chi2():
    import torch

    from pasta_b200 import _ffi
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S

    spec = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, 85000.0, seed=11)
    disp = P.FixedResolutionDispersion(star.wl, 85000.0, wl)
    cont = P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    fitter = interp.get_fitter(disp, cont, P.PSOSettings(8, 2), (0, 300), (-150, 150))
    labs = np.array([list(star.label), [7100.0, 0.0, 4.1, 40.0, 15.0], [6600.0, -0.3, 3.8, 120.0, -60.0],
                     [7900.0, 0.45, 4.45, 0.0, 0.0], [9000.0, 0.0, 4.0, 10.0, 0.0]])
    expect = np.array(fitter.chi2(interp, star.flux, star.var, labs))

    dev = torch.device("cuda", 0)
    flux = torch.from_numpy(star.flux).to(dev)
    var = torch.from_numpy(star.var).to(dev)
    lab = torch.from_numpy(labs).to(dev)
    out = torch.full((len(labs),), -1.0, dtype=torch.float64, device=dev)
    status = torch.full((len(labs),), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = _ffi.lib()

    def call(L=len(labs)):
        return lib.pasta_chi2_noalloc(interp._grid._h, disp._h, cont._h, flux.data_ptr(), var.data_ptr(),
                                      len(star.flux), lab.data_ptr(), L, out.data_ptr(), status.data_ptr(),
                                      C.c_void_p(stream.cuda_stream))

    for attempt in range(2):
        out.fill_(-1.0)
        status.fill_(7)
        free_before = torch.cuda.mem_get_info(dev)[0]
        assert call() == 0, lib.pasta_last_error().decode()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        st = status.cpu().numpy()
        assert (st[:4] == 0).all() and st[4] != 0
        np.testing.assert_allclose(got[:4], expect[:4], rtol=CHI2_TOL)
        assert np.isnan(got[4]) and np.isnan(expect[4])
        if attempt == 1:  # set-up done by the first call: nothing more is taken from the device
            assert torch.cuda.mem_get_info(dev)[0] == free_before

    # more labels than the static workspace holds are rejected with a clear error
    rc = call(L=100000)
    assert rc == -1  # PASTA_E_ARG
    assert b"exceed the allocation-free scratch" in lib.pasta_last_error()
