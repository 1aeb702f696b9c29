"""Small test configurations shared by the golden generator and the tests.

Each scenario is a dict with ``params`` (params.json content), ``stations``
(station.json content), and optionally ``terrain`` (float32 array of the
padded (NY+6, NX+6) grid), ``layers`` (layered-model file bytes as uint8)
and ``source`` (finite-fault file bytes as uint8).
"""
import json
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "cgfdm-fp16_sve_sme_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)
from cgfdm import scenarios as S  # noqa: E402

HALO = 3
# (irk, (FB1, FB2, FB3)) of the stage fixtures: every RK stage, mixed sign
# triples from the MacCormack schedule (propagate.cpp:107-117).
STAGE_CASES = [(0, (-1, -1, -1)), (1, (1, 1, 1)), (2, (-1, 1, -1)), (3, (1, -1, 1))]

TWO_LAYERS = [(0.5, 2.0, 3.5, 2.2), (1000.0, 3.464, 6.0, 2.67)]
THREE_LAYERS = [(0.6, 2.6, 4.5, 2.3), (1.2, 3.35, 5.8, 2.6), (1000.0, 3.75, 6.5, 2.8)]


def as_u8(b):
    return np.frombuffer(bytes(b), dtype=np.uint8).copy()


def grid_dims(p):
    return S.grid_dims(p)


def stage_small():
    """12 x 10 x 10 curvilinear grid: Gaussian-hill terrain, two layers,
    3-cell PML (bottom, four sides) and the free surface on top."""
    p = S.params(NX=12, NY=10, NZ=10, nPML=3, DH=100.0, DT=0.008, TMAX=0.0161,
                 **{"Depth(km)": 1.0}, centerX=6, centerY=5, useTerrain=1, useMedium=1,
                 LayeredModel=1, sourceX=6, sourceY=5, sourceZ=5, out="out")
    terrain = S.gaussian_hill(p, amp=300.0, x0=100.0, y0=-50.0, width=400.0)
    return {"params": p, "stations": {}, "terrain": terrain,
            "layers": as_u8(S.layered_bytes(TWO_LAYERS))}


def run_point():
    """Flat half-space, homogeneous medium, smoothed explosive point source
    (the single-source path), 24 x 20 x 16 grid, 40 steps."""
    p = S.params(NX=24, NY=20, NZ=16, nPML=4, DH=100.0, DT=0.008, TMAX=0.3201,
                 centerX=12, centerY=10, IT_SKIP=13, sliceFreeSurf=1,
                 sourceX=11, sourceY=9, sourceZ=8, rickerfc=6.0, out="out")
    stations = {"A": [5, 5, 15], "B": [11, 9, 15], "C": [18, 14, 15], "D": [11, 9, 12],
                "E": [4, 16, 10]}
    return {"params": p, "stations": stations}


def run_fault():
    """Gaussian-hill terrain, layered medium, finite-fault source through
    the multi-source path, 24 x 22 x 18 grid, 40 steps."""
    p = S.params(NX=24, NY=22, NZ=18, nPML=4, DH=100.0, DT=0.006, TMAX=0.2401,
                 **{"Depth(km)": 1.6}, centerX=12, centerY=11, IT_SKIP=13,
                 sliceFreeSurf=1, useTerrain=1, useMedium=1, LayeredModel=1,
                 useMultiSource=1, **{"useSingleSource(ricker)": 0}, out="out")
    terrain = S.gaussian_hill(p, amp=250.0, x0=-200.0, y0=100.0, width=600.0)
    nt = 60
    src = S.finite_fault(cx=0.0, cy=0.0, cz=-700.0, length=600.0, width=300.0, nl=4, nw=2,
                         strike=90.0, dip=30.0, rake=60.0, mean_slip=1.5, vs_rupture=2400.0,
                         stf_width=0.02, nt=nt, dt=0.006, seed=7)
    stations = {"A": [5, 5, 17], "B": [12, 11, 17], "C": [19, 16, 17], "D": [12, 11, 12],
                "E": [6, 17, 9]}
    return {"params": p, "stations": stations, "terrain": terrain,
            "layers": as_u8(S.layered_bytes(TWO_LAYERS)), "source": as_u8(src)}


def write_inputs(sc, dirpath):
    S.write_run_dir(dirpath, sc["params"], stations=sc.get("stations") or {},
                    terrain=sc.get("terrain"), layers=sc.get("layers"),
                    source=sc.get("source"))


def c1():
    """The homogeneous half-space benchmark configuration: 161 x 161 x 101
    at DH = 100 m (Vp 6000, Vs 3464, rho 2670, the reference's homogeneous
    medium), DT = 0.008 s, 1000 steps, 12-cell PML; one double-couple point
    source (strike 0, dip 90, rake 0, M0 = 1e16) at x = y = 8 km, 2 km deep,
    through the multi-source path, with the moment-rate time function of the
    reference's single source (singleSource.cpp:47-53: the derivative of a
    Ricker wavelet, f0 = 1.5 Hz) centred at t0 = 1.0 s; 25 surface stations
    on a 5 x 5 lattice, 3 km apart; free-surface snapshots every 333 steps
    (mid-run while the wave crosses the surface, and the last step)."""
    nt = 1000
    dt = 0.008
    p = S.params(NX=161, NY=161, NZ=101, DH=100.0, DT=dt, TMAX=8.0001, nPML=12,
                 centerX=0, centerY=0, useMultiSource=1, **{"useSingleSource(ricker)": 0},
                 IT_SKIP=333, sliceFreeSurf=1, out="out")
    f0, t0 = 1.5, 1.0

    def stf(t):
        r = np.pi * f0 * (t - t0)
        return np.pi * f0 * 2.0 * r * (2.0 * r * r - 3.0) * np.exp(-r * r)

    src = S.double_couple_point(8000.0, 8000.0, -2000.0, m0=1e16, mu=2670.0 * 3464.0 ** 2,
                                strike=0.0, dip=90.0, rake=0.0, nt=nt + 2, dt=dt, stf=stf)
    stations = {"S%d%d" % (a, b): [20 + 30 * a, 20 + 30 * b, 100]
                for a in range(5) for b in range(5)}
    return {"params": p, "stations": stations, "source": src}


def c2_parity():
    """The Gaussian-hill benchmark configuration (401 x 401 x 201, nPML 20,
    121 stations, explosive source) for 400 steps (3.2 s: the wave is at
    the surface and still in the domain), free-surface snapshots every 133
    steps."""
    w = S.c2_workload(400, it_skip=133, slice_free_surf=1)
    w["params"]["TMAX"] = 400 * 0.008 + 0.0001
    return {"params": w["params"], "stations": w["stations"], "terrain": w["terrain"],
            "layers": as_u8(w["layers"])}


def c3_201_parity():
    """The 201 x 201 x 401 PerformanceTest shape (random terrain, layered
    medium, 80 x 40 finite fault, nPML 12) for 700 steps (5.6 s: the
    rupture's waves reach the surface), free-surface snapshots every 233
    steps; without the per-cell medium perturbation, which the reference's
    medium reader cannot express."""
    w = S.c3_workload(201, 700, perturbation=0.0, it_skip=233, slice_free_surf=1)
    w["params"]["TMAX"] = 700 * 0.008 + 0.0001
    return {"params": w["params"], "stations": w["stations"], "terrain": w["terrain"],
            "layers": as_u8(w["layers"]), "source": as_u8(w["source"])}


def srtm_run():
    """Real-terrain configuration through the SRTM90 reader: one 5 x 5 degree
    DEM tile (100-105 E, 30-35 N, seeded, with steep spikes and void points
    near the model), a 64 x 56 x 24 grid at 100 m centred on 102.5 E, 32.5 N,
    two layers, an explosive point source three cells below the surface, 120
    steps (the wave crosses the surface stations).  The tile is 144 MB and is
    written next to the run by write_srtm_inputs."""
    p = S.params(NX=64, NY=56, NZ=24, nPML=6, DH=100.0, DT=0.008, TMAX=120 * 0.008 + 0.0001,
                 **{"Depth(km)": 2.4}, centerX=32, centerY=28, useTerrain=1, useMedium=1,
                 LayeredModel=1, SRTM90=1, TerrainDir="dem", lonStart=100, latStart=30,
                 blockX=1, blockY=1, centerLongitude=102.5, centerLatitude=32.5,
                 sourceX=32, sourceY=28, sourceZ=20, rickerfc=4.0, IT_SKIP=40, sliceFreeSurf=1,
                 out="out")
    stations = {"A": [10, 10, 23], "B": [32, 28, 23], "C": [50, 40, 23], "D": [20, 45, 12]}
    return {"params": p, "stations": stations, "layers": as_u8(S.layered_bytes(TWO_LAYERS))}


# the grid centre lies at DEM index (3000, 3000); spikes and voids within the
# model's window (about +-50 points)
SRTM_SPIKES = [(3010, 2995, 400.0), (2980, 3020, -350.0), (3025, 3012, 600.0)]
SRTM_HOLES = [(2990, 2990), (3015, 2985)]


def write_srtm_inputs(sc, dirpath):
    write_inputs(sc, dirpath)
    tile = S.synthetic_dem_tile(100, 30, seed=41, spikes=SRTM_SPIKES, holes=SRTM_HOLES)
    S.write_dem_tile(os.path.join(dirpath, sc["params"]["TerrainDir"]), 100, 30, tile)


def read_outputs(sc, outdir):
    """Reads the reference's single-rank outputs (station.cpp:382-405,
    PGV.cpp:103-111, data_io.cpp:323-495)."""
    p = sc["params"]
    g = grid_dims(p)
    nt = S.nt_of(p)
    res = {}
    fn = os.path.join(outdir, "station_mpi_0_0_0.bin")
    if os.path.exists(fn):
        raw = np.fromfile(fn, dtype=np.uint8)
        nsta = len(sc["stations"])
        res["station_xyz"] = raw[: 12 * nsta].view(np.int32).reshape(nsta, 3)
        res["station_wave"] = raw[12 * nsta:].view(np.float32).reshape(nsta, nt, 9)
    fn = os.path.join(outdir, "PGV_Z_mpi_0_0_0.bin")
    if os.path.exists(fn):
        res["pgv"] = np.fromfile(fn, np.float32).reshape(g["ny"], g["nx"], 2)
    snaps = []
    for it in range(0, nt, p["IT_SKIP"]):
        fn = os.path.join(outdir, "FreeSurfVz_%d_Z_mpi_0_0_0.bin" % it)
        if os.path.exists(fn):
            v = [np.fromfile(os.path.join(outdir, "FreeSurfV%s_%d_Z_mpi_0_0_0.bin" % (c, it)),
                             np.float32).reshape(g["ny"], g["nx"]) for c in "xyz"]
            snaps.append(np.stack(v))
    if snaps:
        res["freesurf"] = np.stack(snaps)
        res["freesurf_its"] = np.arange(0, nt, p["IT_SKIP"])[: len(snaps)]
    return res


def slab_points(p):
    nx, ny, nz, n = p["NX"], p["NY"], p["NZ"], p["nPML"]
    return [n * ny * nz, nx * n * nz, nx * ny * n, n * ny * nz, nx * n * nz]


def random_state(p, seed):
    """Seeded input state of one stage: wavefield W, RK accumulators t and m
    (each 9 x num, zero in the halo like the reference's, velocities ~1e-2,
    stresses ~1e5) and the PML auxiliaries (5 slabs x [Aux, t, m])."""
    rng = np.random.default_rng(seed)
    g = grid_dims(p)
    scale = np.array([1e-2] * 3 + [1e5] * 6, np.float32)[:, None, None, None]

    def wave():
        w = np.zeros((9, g["nz_"], g["ny_"], g["nx_"]), np.float32)
        inner = rng.standard_normal((9, g["nz"], g["ny"], g["nx"])).astype(np.float32)
        w[:, HALO:-HALO, HALO:-HALO, HALO:-HALO] = inner * scale
        return w.reshape(-1)

    st = {"W": wave(), "t": wave(), "m": wave()}
    aux = []
    sc = np.array([1e-2] * 3 + [1e5] * 6, np.float32)
    for n in slab_points(p):
        for _ in range(3):
            aux.append((rng.standard_normal((n, 9)).astype(np.float32) * sc).reshape(-1))
    st["aux"] = np.concatenate(aux)
    return st


def load_golden(name):
    d = np.load(os.path.join(REPO, "tests", "golden", name))
    out = {k: d[k] for k in d.files}
    out["params"] = json.loads(str(out.pop("params_json")))
    if "stations_json" in out:
        out["stations"] = json.loads(str(out.pop("stations_json")))
    return out
