"""pasta_chi2_noalloc: chi2 for callers that cannot allocate device memory
(a host that gives the GPU's whole memory to its own pool, a real-time loop
that may not call cudaMalloc, a service with a fixed footprint).  The caller
owns every input and output buffer on the device; the library's workspace is
a static device array of fixed size.

Checked against the regular entry point pasta_chi2 (same tolerance as the
other chi2 tests: relative 1e-5) on two calls in a row, for a chunk, a
linear-model and a constant continuum, with a narrow rotation kernel among
the labels and at the largest label count the array holds.  The entry point
always takes the FFT broadening path, so pasta_chi2 is pinned to it for the
comparison.  The size limit is enforced.  This file runs last so that a
failure here cannot hide another test's result; it also passes alone in a
fresh process."""
import ctypes as C
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHI2_TOL = 1e-5


@pytest.fixture(scope="module")
def env():
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S

    spec = S.config0_grid(n_px=20000)
    labels, spectra, factors = S.make_grid(spec)
    wl = P.WlGrid(spec.log_first, spec.log_step, spec.n_px, log=True)
    interp = P.InMemInterpolator.from_arrays(labels, spectra, factors, wl)
    star = S.make_star(spec, [7130.0, 0.07, 4.02, 50.0, 20.0], 15000, 100.0, 85000.0, seed=11)
    disp = P.FixedResolutionDispersion(star.wl, 85000.0, wl)
    return dict(P=P, S=S, interp=interp, star=star, disp=disp)


def _cont(env, kind):
    P, S, star = env["P"], env["S"], env["star"]
    if kind == "chunk":
        return P.ChunkContinuumFitter(star.wl, 5, 8, 0.2)
    if kind == "linear":
        return P.LinearModelContinuumFitter(S.legendre_design(star.wl, 12))
    return P.ConstantContinuum()


def _expected(env, cont, labs):
    """pasta_chi2 on the FFT broadening path (the one the entry point takes)."""
    P, interp, star = env["P"], env["interp"], env["star"]
    fitter = interp.get_fitter(env["disp"], cont, P.PSOSettings(8, 2), (0, 300), (-150, 150))
    keep = interp.direct_max
    try:
        interp.direct_max = 0
        return np.array(fitter.chi2(interp, star.flux, star.var, labs))
    finally:
        interp.direct_max = keep


class _Call:
    def __init__(self, env, cont, labs):
        import torch
        from pasta_b200 import _ffi
        self.torch, self.env, self.cont = torch, env, cont
        self.dev = torch.device("cuda", 0)
        star = env["star"]
        self.flux = torch.from_numpy(star.flux).to(self.dev)
        self.var = torch.from_numpy(star.var).to(self.dev)
        self.lab = torch.from_numpy(np.ascontiguousarray(labs)).to(self.dev)
        self.out = torch.full((len(labs),), -1.0, dtype=torch.float64, device=self.dev)
        self.status = torch.full((len(labs),), 7, dtype=torch.int32, device=self.dev)
        self.stream = torch.cuda.current_stream(self.dev)
        self.lib = _ffi.lib()

    def __call__(self, L=None):
        L = len(self.lab) if L is None else L
        self.out.fill_(-1.0)
        self.status.fill_(7)
        return self.lib.pasta_chi2_noalloc(self.env["interp"]._grid._h, self.env["disp"]._h, self.cont._h,
                                           self.flux.data_ptr(), self.var.data_ptr(), len(self.env["star"].flux),
                                           self.lab.data_ptr(), L, self.out.data_ptr(), self.status.data_ptr(),
                                           C.c_void_p(self.stream.cuda_stream))

    def results(self):
        self.torch.cuda.synchronize(self.dev)
        return self.out.cpu().numpy(), self.status.cpu().numpy()


@pytest.mark.parametrize("kind", ["chunk", "linear", "constant"])
def test_chi2_without_allocation_matches_pasta_chi2(env, kind):
    import torch
    star = env["star"]
    cont = _cont(env, kind)
    labs = np.array([list(star.label), [7100.0, 0.0, 4.1, 40.0, 15.0], [6600.0, -0.3, 3.8, 120.0, -60.0],
                     [7900.0, 0.45, 4.45, 0.0, 0.0], [7130.0, 0.07, 4.02, 5.0, 20.0], [9000.0, 0.0, 4.0, 10.0, 0.0]])
    expect = _expected(env, cont, labs)
    call = _Call(env, cont, labs)
    for attempt in range(2):
        free_before = torch.cuda.mem_get_info(call.dev)[0]
        assert call() == 0, call.lib.pasta_last_error().decode()
        got, st = call.results()
        assert (st[:5] == 0).all() and st[5] != 0
        np.testing.assert_allclose(got[:5], expect[:5], rtol=CHI2_TOL)
        assert np.isnan(got[5]) and np.isnan(expect[5])
        if attempt == 1:  # set-up done by the first call: nothing more is taken from the device
            assert torch.cuda.mem_get_info(call.dev)[0] == free_before
    # no labels: nothing to do, like pasta_chi2
    assert call(L=0) == 0


def test_chi2_without_allocation_at_the_size_limit(env):
    """The largest label count the static array holds is evaluated like
    pasta_chi2; one more is rejected with a clear error."""
    star = env["star"]
    cont = _cont(env, "chunk")
    probe = _Call(env, cont, np.array([list(star.label)]))
    assert probe(L=100000) == -1  # PASTA_E_ARG
    msg = probe.lib.pasta_last_error().decode()
    assert "exceed the allocation-free scratch" in msg
    max_labels = int(re.search(r"at most (\d+) labels", msg).group(1))
    assert 100 <= max_labels <= 400
    rng = np.random.default_rng(17)
    labs = np.stack([rng.uniform(6100, 7900, max_labels), rng.uniform(-0.45, 0.45, max_labels),
                     rng.uniform(3.6, 4.4, max_labels), rng.uniform(20, 200, max_labels),
                     rng.uniform(-100, 100, max_labels)], axis=1)
    expect = _expected(env, cont, labs)
    call = _Call(env, cont, labs)
    for _ in range(2):
        assert call() == 0, call.lib.pasta_last_error().decode()
        got, st = call.results()
        assert (st == 0).all()
        np.testing.assert_allclose(got, expect, rtol=CHI2_TOL)
    assert call(L=max_labels + 1) == -1
    assert "exceed the allocation-free scratch" in call.lib.pasta_last_error().decode()
