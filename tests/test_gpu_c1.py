"""The half-space benchmark configuration end to end (161 x 161 x 101, 1000
RK4 steps, 12-cell PML, double-couple point source through the multi-source
path, 25 surface stations): the reference program on one GPU
(cgfdm_run_directory) against the reference's own FP32 CPU build
(tests/golden/c1_halfspace.npz).  The exact-order kernel reproduces every
seismogram sample, the PGV map and the free-surface snapshots bit for bit;
the streaming kernel stays within relative L2 1e-5 on the seismograms, the
PGV map and the free-surface snapshot taken while the wave crosses the
surface (the later ones hold only the residual the wave leaves behind and are
held to 1e-5 of the peak)."""
import os
import tempfile

import numpy as np
import pytest

import scenarios

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_halfspace.npz")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def c1_ref(gpu_available):
    if not os.path.exists(FIXTURE):
        pytest.skip("c1 fixture not generated")
    return np.load(FIXTURE)


def _run(kernel):
    sc = scenarios.c1()
    d = tempfile.mkdtemp()
    scenarios.write_inputs(sc, d)
    cgfdm.run_directory(d, cgfdm.FP32, kernel)
    return scenarios.read_outputs(sc, os.path.join(d, sc["params"]["out"]))


def _snap(got, it):
    return got["freesurf"][list(got["freesurf_its"]).index(it)]


def test_c1_exact_kernel_bitwise(c1_ref):
    got = _run(cgfdm.KERNEL_EXACT)
    np.testing.assert_array_equal(got["station_wave"], c1_ref["out_station_wave"])
    np.testing.assert_array_equal(got["pgv"], c1_ref["out_pgv"])
    for q, it in enumerate(c1_ref["out_freesurf_its"]):
        np.testing.assert_array_equal(_snap(got, int(it)), c1_ref["out_freesurf"][q])


def test_c1_streaming_kernel_within_1e5(c1_ref):
    got = _run(cgfdm.KERNEL_AUTO)
    for v in range(3):
        err = rel_l2(got["station_wave"][:, :, v], c1_ref["out_station_wave"][:, :, v])
        assert err <= 1e-5, (v, err)
    assert rel_l2(got["pgv"], c1_ref["out_pgv"]) <= 1e-5
    # free-surface snapshots every 333 steps.  Those taken while the wave is
    # in the domain (peak at least 1 % of the largest snapshot's: step 333,
    # t = 2.7 s): plain relative L2.  Those that hold only the residual the
    # wave leaves behind after it has gone out through the PML (steps 666 and
    # 999, peaks 2e-4 and 2e-6 of it), where a relative L2 divides rounding
    # differences by a near-zero field: the largest difference against the
    # peak of the run's snapshots.
    its = [int(x) for x in c1_ref["out_freesurf_its"]]
    ref = {it: c1_ref["out_freesurf"][q] for q, it in enumerate(its)}
    peak = max(float(np.abs(f).max()) for f in ref.values())
    live = [it for it in its if 0 < it and np.abs(ref[it]).max() >= 1e-2 * peak]
    if not live:
        pytest.skip("the C1 fixture holds no snapshot taken while the wave crosses the surface")
    for it in its:
        if it == 0:
            continue
        got_it = _snap(got, it)
        if it in live:
            err = rel_l2(got_it, ref[it])
            assert err <= 1e-5, (it, err)
        else:
            diff = float(np.abs(got_it.astype(np.float64) - ref[it]).max())
            assert diff <= 1e-5 * peak, (it, diff, peak)
