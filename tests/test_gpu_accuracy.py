"""Accuracy of the storage forms against an FP64 run on the GPU, on the
Gaussian-hill configuration (401 x 401 x 201, 20-cell PML, 121 surface
stations, explosive source), capped at 800 of its 2000 steps so that the FP64
run (the exact-order kernel on double) fits the test budget.

The error measure is the reference's own comparison of two seismogram sets
(plotXY.py:144): the relative L2 norm of the difference of the Vx, Vy, Vz
seismograms of every station over all steps.  Scaled FP16 must stay within
1e-2 of FP64; FP32 within 1e-5.  Scaled BF16 (an 8-bit mantissa) does not meet
the 1e-2 bar; its error is reported beside the others and held to 1e-1.
"""
import shutil
import tempfile

import numpy as np
import pytest

from cgfdm import scenarios as S

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

STEPS = 800


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _seismograms(prec):
    w = S.c2_workload(STEPS + 2)
    d = tempfile.mkdtemp(prefix="cgfdm_acc_")
    try:
        S.write_run_dir(d, w["params"], stations=w["stations"], terrain=w["terrain"],
                        layers=w["layers"])
        st = cgfdm.setup_from_directory(d, prec)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    d0 = st["desc"]
    desc = cgfdm.make_desc(d0.nx, d0.ny, d0.nz, d0.npml, d0.dh, d0.dt, STEPS, prec,
                           cgfdm.KERNEL_AUTO, 0)
    sta, _, fs = cgfdm.propagate(desc, st["cjm"], st["rdz"], point=st["point"],
                                 rickerfc=st["rickerfc"], stations=st["stations"])
    return sta.reshape(len(st["stations"]), -1, 9)[:, :STEPS, :3], fs


@pytest.fixture(scope="module")
def fp64(gpu_available):
    return _seismograms(cgfdm.FP64)


def test_fp64_run_has_signal_at_the_stations(fp64):
    sta, _ = fp64
    assert np.isfinite(sta).all()
    # the wave has reached most of the surface lattice by step 800
    peak = np.abs(sta).max(axis=(1, 2))
    assert (peak > 1e-3 * peak.max()).mean() > 0.5


@pytest.mark.parametrize("prec,bar", [("fp32", 1e-5), ("fp16", 1e-2), ("bf16", 1e-1)])
def test_storage_form_against_fp64(fp64, prec, bar):
    sta64, _ = fp64
    sta, fs = _seismograms({"fp32": cgfdm.FP32, "fp16": cgfdm.FP16, "bf16": cgfdm.BF16}[prec])
    assert np.isfinite(sta).all() and np.isfinite(fs).all()
    err = rel_l2(sta, sta64)
    print("\n%s: rel L2 of the seismograms against FP64 over %d steps = %.3e" % (prec, STEPS, err))
    assert err <= bar, (prec, err)
