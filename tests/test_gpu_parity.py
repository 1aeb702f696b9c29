"""CUDA path against the reference (through the C ABI).

The exact-order kernel must reproduce the reference's FP32 CPU results bit
for bit: one RK stage on seeded state (all four stages, mixed MacCormack
signs, PML slabs and free surface included) and complete runs (stations,
PGV, free-surface snapshots).  Fixtures: tests/golden/ (made by the
reference itself, see tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

import scenarios

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

HALO = 3


def _desc(p, nt, precision=None, kernel=None):
    return cgfdm.make_desc(p["NX"], p["NY"], p["NZ"], p["nPML"], p["DH"], p["DT"], nt,
                           cgfdm.FP32 if precision is None else precision,
                           cgfdm.KERNEL_EXACT if kernel is None else kernel)


@pytest.fixture(scope="module")
def stage_golden(gpu_available):
    return scenarios.load_golden("stage_small.npz")


def _split_aux_out(flat, p):
    """golden aux out: per slab {h, Aux, t, m} -> per slab {Aux, t, m}."""
    out, off = [], 0
    for n in scenarios.slab_points(p):
        n9 = 9 * n
        out.append(flat[off + n9: off + 4 * n9])
        off += 4 * n9
    return np.concatenate(out)


@pytest.mark.parametrize("case", range(len(scenarios.STAGE_CASES)))
def test_stage_bitwise(stage_golden, case):
    g = stage_golden
    p = g["params"]
    irk, fb = scenarios.STAGE_CASES[case]
    with cgfdm.Simulation(_desc(p, 1)) as sim:
        sim.set_model(g["cjm"], g["rdz"])
        sim.set_state(irk, W=g["in_W"], t=g["in_t"], m=g["in_m"], aux=g["in_aux"])
        sim.stage(irk, fb)
        st = sim.get_state()
    np.testing.assert_array_equal(st["W"], g["case%d_W" % case])
    if irk < 3:
        np.testing.assert_array_equal(st["t"], g["case%d_t" % case])
        np.testing.assert_array_equal(st["m"], g["case%d_m" % case])
    ref_aux = _split_aux_out(g["case%d_aux" % case], p)
    got_aux = st["aux"]
    # per slab: compare Aux (always) and t (stages 0-2); m is the step state
    off = 0
    for n in scenarios.slab_points(p):
        n9 = 9 * n
        np.testing.assert_array_equal(got_aux[off:off + n9], ref_aux[off:off + n9])
        if irk < 3:
            np.testing.assert_array_equal(got_aux[off + n9:off + 2 * n9],
                                          ref_aux[off + n9:off + 2 * n9])
        off += 3 * n9


def _run_sim(g, precision=None, kernel=None, steps=None, tile_rows=0):
    p = g["params"]
    nt = scenarios.S.nt_of(p)
    steps = nt if steps is None else steps
    sim = cgfdm.Simulation(_desc(p, nt, precision, kernel))
    sim.set_tile_rows(tile_rows)
    sim.set_model(g["cjm"], g["rdz"])
    if p["useMultiSource"]:
        dt = float(np.frombuffer(g["source"][8:12].tobytes(), np.float32)[0])
        sim.set_fault_source(g["src_index"], g["src_rate"], int(g["src_nt"]), dt, scaled=True)
    else:
        sim.set_point_source(p["sourceX"] + HALO, p["sourceY"] + HALO, p["sourceZ"] + HALO,
                             p["rickerfc"])
    xyz = np.array([[x + HALO, y + HALO, z + HALO] for x, y, z in g["stations"].values()])
    sim.set_stations(xyz)
    snaps = []
    for it in range(steps):
        sim.run(1)
        if it % p["IT_SKIP"] == 0:
            snaps.append(sim.free_surface())
    out = {"station_wave": sim.stations(), "pgv": sim.pgv(), "freesurf": np.stack(snaps),
           "W": sim.wavefield()}
    sim.close()
    return out


@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_full_run_bitwise(gpu_available, name):
    g = scenarios.load_golden(name)
    res = _run_sim(g)
    np.testing.assert_array_equal(res["station_wave"], g["out_station_wave"])
    np.testing.assert_array_equal(res["pgv"], g["out_pgv"])
    np.testing.assert_array_equal(res["freesurf"], g["out_freesurf"])


@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_run_directory_writes_reference_files(gpu_available, tmp_path, name):
    g = scenarios.load_golden(name)
    sc = {"params": g["params"], "stations": g["stations"], "terrain": g.get("terrain"),
          "layers": g.get("layers"), "source": g.get("source")}
    d = str(tmp_path)
    scenarios.write_inputs(sc, d)
    cgfdm.run_directory(d, kernel=cgfdm.KERNEL_EXACT)
    res = scenarios.read_outputs(sc, os.path.join(d, g["params"]["out"]))
    np.testing.assert_array_equal(res["station_xyz"], g["out_station_xyz"])
    np.testing.assert_array_equal(res["station_wave"], g["out_station_wave"])
    np.testing.assert_array_equal(res["pgv"], g["out_pgv"])
    np.testing.assert_array_equal(res["freesurf"], g["out_freesurf"])


def test_propagate_dropin_matches_reference(gpu_available):
    g = scenarios.load_golden("run_fault.npz")
    p = g["params"]
    nt = scenarios.S.nt_of(p)
    dt = float(np.frombuffer(g["source"][8:12].tobytes(), np.float32)[0])
    xyz = np.array([[x + HALO, y + HALO, z + HALO] for x, y, z in g["stations"].values()])
    sta, pgv, fs = cgfdm.propagate(_desc(p, nt), g["cjm"], g["rdz"], src_index=g["src_index"],
                                   moment_rate=g["src_rate"], src_nt=int(g["src_nt"]),
                                   src_dt=dt, stations=xyz)
    np.testing.assert_array_equal(sta, g["out_station_wave"])
    np.testing.assert_array_equal(pgv, g["out_pgv"])


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def test_fp64_oracle_run_close_to_fp32(gpu_available):
    """The FP64 GPU run solves the same discrete problem; FP32's rounding
    error against it on the seismograms stays far below 1e-5."""
    g = scenarios.load_golden("run_fault.npz")
    r64 = _run_sim(g, precision=cgfdm.FP64)
    err = _rel_l2(g["out_station_wave"][:, :, :3], r64["station_wave"][:, :, :3])
    assert err < 1e-5, err
