"""CPU tests of the host side: the C ABI library exports, the drop-in module's
host logic, the synthetic data, and the replica sharding over gloo ranks."""
import os
import re
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    from pasta_b200 import _ffi
    lib = _ffi.lib()
    hdr = open(os.path.join(ROOT, "include", "pasta_b200.h")).read()
    names = re.findall(r"^\s*(?:int|int64_t|const char \*)\s*\*?\s*(pasta_\w+)\s*\(", hdr, re.M)
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in _ffi.SIGNATURES, n
    assert lib.pasta_abi_version() == 1


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from pasta_b200 import _ffi
    monkeypatch.setattr(_ffi, "_lib", None)
    monkeypatch.setattr(_ffi, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        _ffi.lib()


def test_filename_labels_roundtrip():
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    for t, m, g in [(7100.0, -0.3, 3.9), (25000.0, 0.5, 4.25), (4000.0, 0.0, 2.5)]:
        name = S.filename_from_labels(t, m, g)
        assert P._label_from_filename(name) == (t, m, g)
    assert S.filename_from_labels(7100, -0.3, 3.9) == "lm0030_07100_0390.npy"
    with pytest.raises(ValueError):
        P._label_from_filename("foo_bar.npy")


def test_includes_factor_prefix(tmp_path):
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    spec = S.config0_grid(n_px=512)
    spec.includes_factor = True
    labels, spectra, factors = S.make_grid(spec)
    S.write_grid_dir(str(tmp_path), labels[:3], spectra[:3], factors[:3])
    for i in range(3):
        arr = np.load(tmp_path / S.filename_from_labels(*labels[i]))
        s, mx = P._split_factor(arr, True)
        np.testing.assert_array_equal(s, spectra[i])
        assert mx == factors[i]


def test_settings_conversion_and_constraints():
    from pasta_b200 import pasta as P
    s = P.PSOSettings(46, 60, inertia_factor=-0.3085, cognitive_factor=0, social_factor=2.0273)
    st = P._settings_c(s, (1, 500), (-150, 150), [P.FixConstraint(1, 0.0), P.RangeConstraint(0, 6000, 7000)])
    assert st.num_particles == 46 and st.max_iters == 60
    assert st.cognitive_factor == 0.0 and st.delta == 1e-7
    assert list(st.ckind) == [2, 1, 0, 0, 0]
    assert st.ca[0] == 6000 and st.cb[0] == 7000 and st.ca[1] == 0.0
    d = P.PSOSettings(10, 5)
    assert d.inertia_factor == 0.7213475204 and d.social_factor == 1.1931471806


def test_vsini_kernel_matches_oracle():
    import oracle as O
    from pasta_b200 import pasta as P
    wl = P.WlGrid(np.log10(4000), 2e-6, 1000, log=True)
    for v in (5.0, 60.0, 250.0):
        a = np.array(P.get_vsini_kernel(v, wl))
        b = O.rotation_kernel(v, np.log(10.0) * 2e-6)
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-9)


def test_result_serialisation():
    from pasta_b200 import pasta as P
    r = P.OptimizationResult(P.Label(7000, 0.1, 4.0, 20, -5), [1.0, 2.0], 1.5, 100, 0.3)
    d = r.to_dict()
    r2 = P.OptimizationResult.from_dict(d)
    assert r2.to_json() == r.to_json()
    assert r2.label.as_list() == [7000.0, 0.1, 4.0, 20.0, -5.0]


def test_synthetic_grid_is_seeded():
    from pasta_b200 import synth as S
    spec = S.config0_grid(n_px=300)
    a = S.make_grid(spec)[1]
    b = S.make_grid(spec)[1]
    np.testing.assert_array_equal(a, b)
    assert a.shape == (495, 300)
    c1 = S.config1_grid(n_px=8)
    assert len(c1.teffs) * len(c1.ms) * len(c1.loggs) == 13860
    c4 = S.config4_grid(n_px=8)
    assert len(c4.teffs) * len(c4.ms) * len(c4.loggs) == 27040


def test_shard_partitions_everything():
    from pasta_b200.dist import shard
    for n in (0, 1, 7, 1024):
        for w in (1, 2, 3, 8):
            got = [i for r in range(w) for i in shard(n, r, w)]
            assert got == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
from pasta_b200.dist import shard, max_over_ranks, sum_over_ranks, gather_to_rank0
dist.init_process_group("gloo", init_method="env://")
r, w = dist.get_rank(), dist.get_world_size()
mine = list(shard(10, r, w))
t = max_over_ranks(float(r + 1))
s = sum_over_ranks(float(len(mine)))
g = gather_to_rank0(mine)
if r == 0:
    assert t == float(w), t
    assert s == 10.0, s
    assert sum(g, []) == list(range(10)), g
    print("OK", flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def test_replica_sharding_over_two_gloo_ranks(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2")
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    assert "OK" in outs[0]


def test_rust_style_u16_cast():
    """`f32 as u16` truncates toward zero and saturates; NaN becomes 0."""
    from pasta_b200.pasta import _as_u16
    x = np.array([-3.0, 0.0, 0.99, 1.0, 65534.9, 65535.0, 70000.0, np.nan, np.inf], np.float32)
    np.testing.assert_array_equal(_as_u16(x), [0, 0, 0, 1, 65534, 65535, 65535, 0, 65535])


def test_tar_grid_reader(tmp_path):
    """Grid archives (model_fetchers.rs:168-226): models are the members whose
    name starts with 'l'; a plain tar is read directly, and a zstd frame
    without a decoder installed gives a clear error."""
    import tarfile
    from pasta_b200 import pasta as P
    from pasta_b200 import synth as S
    spec = S.config0_grid(n_px=256)
    spec.includes_factor = True
    labels, spectra, factors = S.make_grid(spec)
    d = tmp_path / "grid"
    S.write_grid_dir(str(d), labels[:6], spectra[:6], factors[:6])
    (d / "readme.txt").write_text("not a model")
    tar = tmp_path / "grid.tar"
    with tarfile.open(tar, "w") as tf:
        tf.add(str(d), arcname="grid")
    lab, sp, mx = P._read_tar_models(str(tar), True)
    order = np.lexsort((lab[:, 2], lab[:, 1], lab[:, 0]))
    ref = np.lexsort((labels[:6, 2], labels[:6, 1], labels[:6, 0]))
    np.testing.assert_allclose(lab[order], labels[:6][ref])
    np.testing.assert_array_equal(sp[order], spectra[:6][ref])
    np.testing.assert_array_equal(mx[order], factors[:6][ref])
    zst = tmp_path / "grid.tar.zst"
    zst.write_bytes(P.ZSTD_MAGIC + b"\x00" * 64)
    import importlib.util
    import shutil
    if importlib.util.find_spec("zstandard") is None and not (shutil.which("zstd") or shutil.which("unzstd")):
        with pytest.raises(RuntimeError, match="zstd"):
            P._read_tar_models(str(zst), True)
