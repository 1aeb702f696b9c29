"""The scaled-FP16 path against the reference's own scalar FP16 build
(tests/golden/run_point_fp16.npz: the flat half-space point-source run) and
against our FP32 path.

The exact-order FP16 kernel follows the reference's FP16 roundings and must
reproduce the reference FP16 build bit for bit; the streaming FP16 kernel
(FMA contraction, reordered sums) is held to a relative L2 error of the
seismograms (Vx, Vy, Vz of all stations) stated per test."""
import os
import tempfile

import numpy as np
import pytest

import scenarios

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _run(precision, kernel):
    sc = scenarios.run_point()
    d = tempfile.mkdtemp()
    scenarios.write_inputs(sc, d)
    s = cgfdm.setup_from_directory(d, precision)
    d0 = s["desc"]
    with cgfdm.Simulation(cgfdm.make_desc(d0.nx, d0.ny, d0.nz, d0.npml, d0.dh, d0.dt, d0.nt,
                                          precision, kernel)) as sim:
        sim.set_model(s["cjm"], s["rdz"])
        sim.set_point_source(*s["point"], s["rickerfc"])
        sim.set_stations(s["stations"])
        sim.run(d0.nt)
        return sim.stations()


def test_fp16_exact_kernel_is_bitwise_the_reference_fp16_build(gpu_available):
    g = scenarios.load_golden("run_point_fp16.npz")
    got = _run(cgfdm.FP16, cgfdm.KERNEL_EXACT)
    np.testing.assert_array_equal(got, g["out_station_wave"])


def test_fp16_streaming_kernel_close_to_reference_fp16_build(gpu_available):
    g = scenarios.load_golden("run_point_fp16.npz")
    got = _run(cgfdm.FP16, cgfdm.KERNEL_AUTO)
    assert np.isfinite(got).all()
    err = rel_l2(got[:, :, :3], g["out_station_wave"][:, :, :3])
    print("FP16 streaming vs reference FP16 build: rel L2 %.3e" % err)  # 1.06e-3 measured
    assert err <= 5e-3


def test_fp16_close_to_fp32(gpu_available):
    g = scenarios.load_golden("run_point.npz")
    got = _run(cgfdm.FP16, cgfdm.KERNEL_AUTO)
    err = rel_l2(got[:, :, :3], g["out_station_wave"][:, :, :3])
    print("FP16 vs reference FP32: rel L2 %.3e" % err)
    assert err <= 5e-3
