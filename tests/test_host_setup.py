"""Host setup (C++, no GPU needed) against the reference's own setup products:
params parsing, coordinates, layered medium, metrics/Jacobian (CJM), the
free-surface matrices, the PML profiles and the finite-fault source table
must equal the reference's bit for bit."""
import json
import os

import numpy as np
import pytest

import scenarios

cgfdm = pytest.importorskip("cgfdm")


def _setup(tmp_path, sc):
    d = str(tmp_path)
    scenarios.write_inputs(sc, d)
    return cgfdm.setup_from_directory(d)


@pytest.fixture(scope="module")
def stage_golden():
    return scenarios.load_golden("stage_small.npz")


def _scenario_from_golden(g):
    return {"params": g["params"], "stations": {}, "terrain": g["terrain_input"],
            "layers": g["layers"]}


def test_setup_matches_reference_bitwise(tmp_path, stage_golden):
    g = stage_golden
    s = _setup(tmp_path, _scenario_from_golden(g))
    np.testing.assert_array_equal(s["coord"], g["coord"])
    np.testing.assert_array_equal(s["medium"], g["medium"])
    np.testing.assert_array_equal(s["cjm"], g["cjm"])
    np.testing.assert_array_equal(s["rdz"], g["rdz"])
    np.testing.assert_array_equal(s["pml"], g["pml"])


@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_run_setup_matches_reference(tmp_path, name):
    g = scenarios.load_golden(name)
    sc = {"params": g["params"], "stations": g["stations"], "terrain": g.get("terrain"),
          "layers": g.get("layers"), "source": g.get("source")}
    s = _setup(tmp_path, sc)
    np.testing.assert_array_equal(s["cjm"], g["cjm"])
    np.testing.assert_array_equal(s["rdz"], g["rdz"])
    p = g["params"]
    assert s["desc"].nt == scenarios.S.nt_of(p)
    exp = np.array([[x + 3, y + 3, z + 3] for x, y, z in g["stations"].values()], np.int32)
    np.testing.assert_array_equal(s["stations"], exp)
    if p["useMultiSource"]:
        np.testing.assert_array_equal(s["src_index"], g["src_index"])
        assert s["src_nt"] == int(g["src_nt"])
        np.testing.assert_array_equal(s["moment_rate"], g["src_rate"])
    else:
        assert s["point"] == (p["sourceX"] + 3, p["sourceY"] + 3, p["sourceZ"] + 3)


def _write(tmp_path, params, stations=None):
    d = str(tmp_path)
    scenarios.S.write_run_dir(d, params, stations=stations or {})
    return d


def _code(fn):
    with pytest.raises(cgfdm.CgfdmError) as e:
        fn()
    return e.value.code


def test_missing_params_is_an_error(tmp_path):
    assert _code(lambda: cgfdm.setup_from_directory(str(tmp_path))) == 100


def test_malformed_params_is_an_error(tmp_path):
    (tmp_path / "params.json").write_text('{"NX": 10, "NY": ')
    assert _code(lambda: cgfdm.setup_from_directory(str(tmp_path))) == 100


def test_cfl_violation(tmp_path):
    p = scenarios.S.params(NX=16, NY=16, NZ=12, nPML=4, DT=0.05)
    assert _code(lambda: cgfdm.setup_from_directory(_write(tmp_path, p))) == 110


def test_pml_bigger_than_grid(tmp_path):
    p = scenarios.S.params(NX=16, NY=16, NZ=12, nPML=20)
    assert _code(lambda: cgfdm.setup_from_directory(_write(tmp_path, p))) == 130


def test_no_source(tmp_path):
    p = scenarios.S.params(NX=16, NY=16, NZ=12, nPML=4, **{"useSingleSource(ricker)": 0})
    assert _code(lambda: cgfdm.setup_from_directory(_write(tmp_path, p))) == 180


def test_missing_source_file(tmp_path):
    p = scenarios.S.params(NX=16, NY=16, NZ=12, nPML=4, useMultiSource=1,
                           **{"useSingleSource(ricker)": 0})
    assert _code(lambda: cgfdm.setup_from_directory(_write(tmp_path, p))) == 181


def test_keys_are_case_insensitive(tmp_path):
    p = scenarios.S.params(NX=16, NY=14, NZ=12, nPML=4)
    q = {k.upper() if k in ("NX", "nPML", "DT") else k: v for k, v in p.items()}
    q["npml"] = q.pop("NPML")
    s = cgfdm.setup_from_directory(_write(tmp_path, q))
    assert (s["desc"].nx, s["desc"].ny, s["desc"].npml) == (16, 14, 4)


def test_station_outside_grid_is_dropped(tmp_path):
    p = scenarios.S.params(NX=16, NY=14, NZ=12, nPML=4)
    s = cgfdm.setup_from_directory(_write(tmp_path, p, {"A": [3, 3, 11], "B": [40, 3, 11]}))
    np.testing.assert_array_equal(s["stations"], [[6, 6, 14]])


def test_point_source_outside_grid_is_skipped(tmp_path):
    p = scenarios.S.params(NX=16, NY=14, NZ=12, nPML=4, sourceX=99)
    assert cgfdm.setup_from_directory(_write(tmp_path, p))["point"] is None
