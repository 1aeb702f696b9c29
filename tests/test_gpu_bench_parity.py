"""The fast path against the reference's FP32 CPU build at the benchmark
configurations (fixtures made by tests/golden/make_golden.py from the
reference run on 8 MPI ranks, the rank files merged):

* c2_hill.npz: the Gaussian-hill configuration, 401 x 401 x 201, 20-cell
  PML, 121 surface stations, explosive source, 400 steps (3.2 s);
* c3_201.npz: the 201 x 201 x 401 PerformanceTest shape with random terrain,
  a layered medium and the 80 x 40 finite fault, 700 steps (5.6 s).

Each run goes through cgfdm_run_directory (the reference's run directory in,
its output files out).  The bar on the streaming kernels (KERNEL_AUTO, the
path every reported number comes from): relative L2 <= 1e-5 on each of the
Vx, Vy, Vz station seismograms, on the PGV map and on the last two
free-surface velocity snapshots, taken while the wave is in the domain.  The
exact-order kernel reproduces all of them bit for bit.
"""
import json
import os
import tempfile

import numpy as np
import pytest

import scenarios

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"c2_hill.npz": scenarios.c2_parity, "c3_201.npz": scenarios.c3_201_parity}
BAR = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _fixture(name):
    fn = os.path.join(GOLDEN, name)
    if not os.path.exists(fn):
        pytest.skip("%s not generated" % name)
    g = np.load(fn)
    sc = CASES[name]()
    # the inputs are regenerated from the seeded scenario; they must be the
    # ones the fixture was made from
    assert json.loads(str(g["params_json"])) == json.loads(json.dumps(sc["params"]))
    assert json.loads(str(g["stations_json"])) == json.loads(json.dumps(sc["stations"]))
    return sc, g


def _run(sc, kernel):
    d = tempfile.mkdtemp(prefix="cgfdm_parity_")
    scenarios.write_inputs(sc, d)
    cgfdm.run_directory(d, cgfdm.FP32, kernel)
    return scenarios.read_outputs(sc, os.path.join(d, sc["params"]["out"]))


def _snapshots(got, g):
    its = list(got["freesurf_its"])
    return np.stack([got["freesurf"][its.index(it)] for it in g["out_freesurf_its"]])


@pytest.mark.parametrize("name", sorted(CASES))
def test_streaming_kernels_within_1e5_of_reference(gpu_available, name):
    sc, g = _fixture(name)
    got = _run(sc, cgfdm.KERNEL_AUTO)
    ref_v = g["out_station_v"]
    # the wave has reached the stations and the surface
    assert np.abs(ref_v).max() > 0 and np.abs(g["out_freesurf"][-1]).max() > 0
    errs = {}
    for v, comp in enumerate("xyz"):
        errs["V" + comp] = rel_l2(got["station_wave"][:, :, v], ref_v[:, :, v])
    errs["pgv"] = rel_l2(got["pgv"], g["out_pgv"])
    snaps = _snapshots(got, g)
    for q, it in enumerate(g["out_freesurf_its"]):
        errs["freesurf_%d" % it] = rel_l2(snaps[q], g["out_freesurf"][q])
    print("\n%s streaming kernels vs reference FP32 CPU build: %s" % (
        name, ", ".join("%s %.2e" % kv for kv in errs.items())))
    for key, err in errs.items():
        assert err <= BAR, (key, err)


@pytest.mark.parametrize("name", sorted(CASES))
def test_exact_kernel_bitwise_reference(gpu_available, name):
    sc, g = _fixture(name)
    got = _run(sc, cgfdm.KERNEL_EXACT)
    np.testing.assert_array_equal(got["station_wave"][:, :, :3], g["out_station_v"])
    np.testing.assert_array_equal(got["pgv"], g["out_pgv"])
    np.testing.assert_array_equal(_snapshots(got, g), g["out_freesurf"])
