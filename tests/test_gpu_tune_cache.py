"""The autotuner's optional on-disk cache (environment variable
CGFDM_TUNE_CACHE): a process whose tuner has no choice for a grid in memory
takes it from the file before timing anything, and writes the choices it
times back.  Each run here is a fresh process (the in-memory choices of this
one would otherwise answer first)."""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

TESTS = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(TESTS), "cgfdm-fp16_sve_sme_b200")
CHILD = r"""
import json, sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
out = sys.argv[1]
import numpy as np
import cgfdm
from test_gpu_batch import _synthetic
nx, ny, nz, npml = 96, 80, 30, 6
sc = _synthetic(nx, ny, nz, npml, seed=nx + ny)
d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, 4, cgfdm.FP32, cgfdm.KERNEL_AUTO)
with cgfdm.Simulation(d) as sim:
    sim.set_model(sc["cjm"], sc["rdz"])
    sim.set_point_source(*sc["src"], 6.0)
    sim.set_stations(sc["sta"])
    sim.run(4)
    np.save(out, np.asarray(sim.wavefield()))
    print(json.dumps({"tuning": list(sim.tuning3())}))
""" % (PKG, TESTS)


def _child(cache):
    env = dict(os.environ, CGFDM_TUNE_CACHE=cache)
    wave = cache + ".wave.npy"
    out = subprocess.run([sys.executable, "-c", CHILD, wave], env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    res["wave"] = np.load(wave)
    return res


def test_tuning_cache_is_written_and_read(gpu_available):
    d = tempfile.mkdtemp(prefix="cgfdm_tune_")
    try:
        _check(os.path.join(d, "tune.json"))
    finally:
        shutil.rmtree(d, ignore_errors=True)


def _check(cache):
    first = _child(cache)
    entries = json.load(open(cache))
    assert len(entries) == 1
    (key, val), = entries.items()
    assert val == first["tuning"]
    assert "96x80x30" in key and "npml6" in key
    # another valid choice in the file: a fresh process takes it as it stands
    form, chunk, top = val
    other = [8 if form != 8 else 16, 32 if chunk != 32 else 64, 1 - top]
    json.dump({key: other}, open(cache, "w"))
    second = _child(cache)
    assert second["tuning"] == other
    # the two choices agree to rounding (the fast path's bar: relative L2
    # 1e-5 on the wavefield)
    a, b = first["wave"].astype(np.float64), second["wave"].astype(np.float64)
    assert np.abs(a).max() > 0
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(a)
    # a malformed file is ignored: the tuner times and writes a valid file
    open(cache, "w").write("{not json")
    third = _child(cache)
    assert json.load(open(cache)) == {key: third["tuning"]}
