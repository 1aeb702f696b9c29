"""Real terrain from SRTM90 DEM tiles (terrain.cpp:217-940) against the
reference's own reader (tests/golden/srtm_run.npz, made by the reference's
terrain.cpp with the spherical projection stand-in of oracle/ref_shim/proj.h,
the same projection the library uses in place of PROJ).

The seeded DEM tile carries steep single-point spikes and SRTM void values
near the model, so the void reset, the gradient calibration, both Gaussian
smoothings and the bilinear interpolation (with the reference's corner
order) all act on the result.  Host setup: bit for bit.  The run on this
terrain through cgfdm_run_directory: the exact-order kernel bit for bit,
the streaming kernels within relative L2 1e-5.
"""
import json
import os
import shutil
import tempfile

import numpy as np
import pytest

import scenarios

cgfdm = pytest.importorskip("cgfdm")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def srtm_dir():
    sc = scenarios.srtm_run()
    d = tempfile.mkdtemp(prefix="cgfdm_srtm_")
    scenarios.write_srtm_inputs(sc, d)
    yield sc, d
    shutil.rmtree(d, ignore_errors=True)


@pytest.fixture(scope="module")
def golden():
    g = scenarios.load_golden("srtm_run.npz")
    assert g["params"] == json.loads(json.dumps(scenarios.srtm_run()["params"]))
    return g


def test_terrain_is_bitwise_the_reference_reader(srtm_dir, golden):
    sc, d = srtm_dir
    st = cgfdm.setup_from_directory(d)
    np.testing.assert_array_equal(st["terrain"][3:-3, 3:-3], golden["out_terrain"])


def test_calibration_and_void_reset_act_on_the_model(srtm_dir):
    """Without the spikes and voids the same tile gives a different surface:
    the reader's clean-up steps are exercised by the fixture."""
    sc, d = srtm_dir
    clean = tempfile.mkdtemp(prefix="cgfdm_srtm_clean_")
    try:
        scenarios.write_inputs(sc, clean)
        tile = cgfdm.scenarios.synthetic_dem_tile(100, 30, seed=41)
        cgfdm.scenarios.write_dem_tile(os.path.join(clean, "dem"), 100, 30, tile)
        a = cgfdm.setup_from_directory(d)["terrain"]
        b = cgfdm.setup_from_directory(clean)["terrain"]
        assert not np.array_equal(a, b)
        # a void left at zero in 5 km high terrain would dent the surface by
        # kilometres; after the reset, calibration and smoothing the dents
        # stay a fraction of that
        assert np.isfinite(a).all() and np.abs(a - b).max() < 500.0
    finally:
        shutil.rmtree(clean, ignore_errors=True)


def test_missing_tile_and_model_outside_the_dem_are_errors(srtm_dir):
    sc, d = srtm_dir
    bad = tempfile.mkdtemp(prefix="cgfdm_srtm_bad_")
    try:
        p = dict(sc["params"], TerrainDir="nowhere")
        scenarios.write_inputs(dict(sc, params=p), bad)
        with pytest.raises(cgfdm.CgfdmError) as e:
            cgfdm.setup_from_directory(bad)
        assert "DEM tile" in str(e.value)
        # the model centred at the tile's corner: its window leaves the DEM
        os.symlink(os.path.join(d, "dem"), os.path.join(bad, "dem"))
        p = dict(sc["params"], centerLongitude=100.0, centerLatitude=30.0)
        scenarios.write_inputs(dict(sc, params=p), bad)
        with pytest.raises(cgfdm.CgfdmError) as e:
            cgfdm.setup_from_directory(bad)
        assert "DEM" in str(e.value)
    finally:
        shutil.rmtree(bad, ignore_errors=True)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["exact", "auto"])
def test_run_on_dem_terrain_matches_reference(gpu_available, srtm_dir, golden, kernel):
    sc, d = srtm_dir
    run = tempfile.mkdtemp(prefix="cgfdm_srtm_run_")
    try:
        for name in os.listdir(d):
            src = os.path.join(d, name)
            if name != sc["params"]["out"]:
                os.symlink(src, os.path.join(run, name))
        cgfdm.run_directory(run, cgfdm.FP32,
                            cgfdm.KERNEL_EXACT if kernel == "exact" else cgfdm.KERNEL_AUTO)
        got = scenarios.read_outputs(sc, os.path.join(run, sc["params"]["out"]))
    finally:
        shutil.rmtree(run, ignore_errors=True)
    if kernel == "exact":
        np.testing.assert_array_equal(got["station_wave"], golden["out_station_wave"])
        np.testing.assert_array_equal(got["pgv"], golden["out_pgv"])
        np.testing.assert_array_equal(got["freesurf"], golden["out_freesurf"])
    else:
        for v in range(9):
            err = rel_l2(got["station_wave"][:, :, v], golden["out_station_wave"][:, :, v])
            assert err <= 1e-5, (v, err)
        assert rel_l2(got["pgv"], golden["out_pgv"]) <= 1e-5
        assert rel_l2(got["freesurf"], golden["out_freesurf"]) <= 1e-5
