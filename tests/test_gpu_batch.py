"""Step graphs and batches.

* A step replayed as a CUDA graph runs the same kernels on the same data:
  results are bit-identical to launching them one by one, and with the
  exact-order kernel still bit-identical to the reference's fixtures.
* A batch advances several scenarios (uneven grids, own sources and
  stations, different phases of the MacCormack schedule) with one persistent
  streaming launch per stage spanning all of them: every member's results
  are bit-identical to running it alone.
"""
import numpy as np
import pytest

import scenarios

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")

NT = 24


def _synthetic(nx, ny, nz, npml, seed):
    rng = np.random.default_rng(seed)
    cjm = np.zeros((13, nz + 6, ny + 6, nx + 6), np.float32)
    inner = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))
    base = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 1e6, 3.2e10, 3.2e10, 1 / 2670.0], np.float32)
    cjm[inner] = base[:, None, None, None] * (
        1 + 0.05 * rng.standard_normal((13, nz, ny, nx)).astype(np.float32))
    for f in (1, 2, 3, 5, 6, 7):
        cjm[f][inner[1:]] = 0.02 * rng.standard_normal((nz, ny, nx)).astype(np.float32)
    rdz = (0.1 * rng.standard_normal(18 * (nx + 6) * (ny + 6))).astype(np.float32)
    sta = np.array([[4, 4, nz + 2], [nx // 2, ny // 2, nz + 1], [nx, ny, nz // 2 + 3]])
    return {"dims": (nx, ny, nz, npml), "cjm": cjm.reshape(-1), "rdz": rdz, "sta": sta,
            "src": (nx // 2 + 3, ny // 2 + 3, nz // 2 + 3)}


def _scaled(sc):
    """The coefficient form of the FP16 / BF16 setup: mu and lambda times
    Cs/Cv, buoyancy divided by Cs/Cv and by Crho."""
    c = sc["cjm"].reshape(13, -1)
    c[9] *= 1e-6  # a Jacobian of order one, as the setup's (half tops out at 65504)
    c[10:12] *= 1e-6 / 5e3
    c[12] *= 5e3 / 1e-6 / 1e6
    return sc


SHAPES = [(71, 45, 40, 6), (40, 33, 30, 4), (96, 64, 48, 8), (33, 70, 36, 5), (50, 50, 60, 0)]


def _sim(sc, precision=cgfdm.FP32, kernel=cgfdm.KERNEL_AUTO):
    nx, ny, nz, npml = sc["dims"]
    s = cgfdm.Simulation(cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, NT, precision, kernel))
    s.set_tile_rows(16)
    s.set_model(sc["cjm"], sc["rdz"])
    s.set_point_source(*sc["src"], 4.0)
    s.set_stations(sc["sta"])
    return s


def _results(s):
    out = s.stations(), s.pgv(), s.wavefield()
    assert all(np.isfinite(x).all() for x in out)
    return out


def _same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_graph_exact_path_still_matches_reference_bitwise(gpu_available, name):
    g = scenarios.load_golden(name)
    p = g["params"]
    nt = scenarios.S.nt_of(p)
    sim = cgfdm.Simulation(cgfdm.make_desc(p["NX"], p["NY"], p["NZ"], p["nPML"], p["DH"], p["DT"],
                                           nt, cgfdm.FP32, cgfdm.KERNEL_EXACT))
    sim.set_graph(True)
    sim.set_model(g["cjm"], g["rdz"])
    if p["useMultiSource"]:
        dt = float(np.frombuffer(g["source"][8:12].tobytes(), np.float32)[0])
        sim.set_fault_source(g["src_index"], g["src_rate"], int(g["src_nt"]), dt, scaled=True)
    else:
        sim.set_point_source(p["sourceX"] + 3, p["sourceY"] + 3, p["sourceZ"] + 3, p["rickerfc"])
    sim.set_stations(np.array([[x + 3, y + 3, z + 3] for x, y, z in g["stations"].values()]))
    sim.run(nt)
    np.testing.assert_array_equal(sim.stations(), g["out_station_wave"])
    np.testing.assert_array_equal(sim.pgv(), g["out_pgv"])
    sim.close()


@pytest.mark.parametrize("precision", [cgfdm.FP32, cgfdm.FP16])
def test_graph_replay_is_bitwise_identical(gpu_available, precision):
    sc = _synthetic(*SHAPES[0], seed=1)
    if precision != cgfdm.FP32:
        sc = _scaled(sc)
    out = []
    for graph in (False, True):
        s = _sim(sc, precision)
        s.set_graph(graph)
        for _ in range(4):  # several run() calls: phases recur, graphs are replayed
            s.run(NT // 4)
        out.append(_results(s))
        s.close()
    _same(out[0], out[1])


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_members_alone(gpu_available, graph):
    scs = [_synthetic(*d, seed=10 + q) for q, d in enumerate(SHAPES)]
    # alone
    alone = []
    for q, sc in enumerate(scs):
        s = _sim(sc)
        s.run(NT)
        alone.append(_results(s))
        s.close()
    # together: members start at different steps (phases of the MacCormack
    # schedule), advanced alone first, then as one batch
    sims = [_sim(sc) for sc in scs]
    for q, s in enumerate(sims):
        if q:
            s.run(q)
    b = cgfdm.Batch(sims, graph=graph)
    for _ in range(3):
        b.run(4)
    b.synchronize()
    b.close()
    for q, s in enumerate(sims):
        s.run(NT - q - 12)  # the rest alone again
        _same(_results(s), alone[q])
        s.close()


def test_batch_fp16_matches_alone(gpu_available):
    scs = [_scaled(_synthetic(*d, seed=30 + q)) for q, d in enumerate(SHAPES[:3])]
    alone = []
    for sc in scs:
        s = _sim(sc, cgfdm.FP16)
        s.run(NT)
        alone.append(_results(s))
        s.close()
    sims = [_sim(sc, cgfdm.FP16) for sc in scs]
    with cgfdm.Batch(sims, graph=True) as b:
        b.run(NT)
        b.synchronize()
    for q, s in enumerate(sims):
        _same(_results(s), alone[q])
        s.close()


def test_batch_rejects_mixed_precision(gpu_available):
    a = _sim(_synthetic(*SHAPES[1], seed=3))
    h = _sim(_synthetic(*SHAPES[1], seed=3), cgfdm.FP16)
    with pytest.raises(cgfdm.CgfdmError):
        cgfdm.Batch([a, h])
    a.close()
    h.close()
