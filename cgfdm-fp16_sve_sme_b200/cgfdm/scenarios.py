"""Synthetic model inputs in the reference's own file formats.

The reference reads its run from ``params.json`` (src-new-FP32-SVE/
getParams.cpp:55-242), ``station.json`` (station.cpp:83-187), a layered
medium file (medium.cpp:98-130), a finite-fault source file
(multiSource.cpp:14-87, 362-418) and, for real terrain, DEM tiles.  The
public datasets behind those inputs are not available here, so the model
shapes of the benchmark configurations are synthesised with seeded
generators and written in exactly those formats:

* terrain: an analytic Gaussian hill or a seeded Gaussian random field over
  the padded grid (NX+6)x(NY+6), x fastest, heights in metres;
* layered medium: ``int32 layers`` then per layer ``float32`` bottom depth
  (km), Vs, Vp (km/s), rho (g/cc);
* source: ``int32 npts, int32 nt, float32 dt`` then per point
  ``float32 x, y, z, area, strike, dip, rake[nt], slip_rate[nt]``; x and y
  are metres from the grid centre (the reader's map projection is the
  identity on them), z is negative down.
"""
import json
import math
import os
import struct

import numpy as np

HALO = 3

DEFAULT_PARAMS = {
    "TMAX": 1.0001, "DT": 0.008, "DH": 100.0, "NX": 64, "NY": 64, "NZ": 48,
    "Depth(km)": 4.8, "centerX": 0, "centerY": 0, "IT_SKIP": 100000,
    "sliceX": -1, "sliceY": -1, "sliceZ": -1, "sliceFreeSurf": 0,
    "PX": 1, "PY": 1, "PZ": 1, "sourceX": 32, "sourceY": 32, "sourceZ": 24,
    "centerLatitude": 0.0, "centerLongitude": 0.0,
    "nPML": 12, "Non-Uniform": 0, "gauss_hill": 0, "useTerrain": 0, "useMedium": 0,
    "useMultiSource": 0, "useSingleSource(ricker)": 1, "rickerfc": 1.5,
    "ShenModel": 0, "Crust_1Medel": 0, "LayeredModel": 0, "LayeredFileName": "layers.bin",
    "out": "output", "sourceDir": ".", "sourceFile": "source.bin", "SRTM90": 0,
}


def params(**over):
    p = dict(DEFAULT_PARAMS)
    p.update(over)
    return p


def nt_of(p):
    """NT = (int)(TMAX / DT) with DT stored as double (propagate.cpp:35-36)."""
    return int(p["TMAX"] / np.float32(p["DT"]))


def grid_dims(p):
    nx, ny, nz = p["NX"], p["NY"], p["NZ"]
    d = {"nx": nx, "ny": ny, "nz": nz, "nx_": nx + 2 * HALO, "ny_": ny + 2 * HALO,
         "nz_": nz + 2 * HALO}
    d["num"] = d["nx_"] * d["ny_"] * d["nz_"]
    return d


def xy_axes(p):
    """Global x, y coordinates of the padded grid (coord.cpp:137-138)."""
    I = np.arange(p["NX"] + 2 * HALO)
    J = np.arange(p["NY"] + 2 * HALO)
    DH = np.float32(p["DH"])
    x = (I - HALO) * DH - p["centerX"] * DH
    y = (J - HALO) * DH - p["centerY"] * DH
    return x.astype(np.float64), y.astype(np.float64)


def gaussian_hill(p, amp, x0, y0, width):
    """h = amp * exp(-((x-x0)^2 + (y-y0)^2) / width^2) on the padded grid."""
    x, y = xy_axes(p)
    X, Y = np.meshgrid(x, y)
    return (amp * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / width ** 2)).astype(np.float32)


def random_terrain(p, rms, corr, seed):
    """Seeded Gaussian random field with a Gaussian spectrum of correlation
    length ``corr`` (m), rescaled to RMS height ``rms`` (m), made
    non-negative-mean by shifting its minimum to zero."""
    rng = np.random.default_rng(seed)
    ny, nx = p["NY"] + 2 * HALO, p["NX"] + 2 * HALO
    white = rng.standard_normal((ny, nx))
    kx = np.fft.fftfreq(nx, d=p["DH"]) * 2 * np.pi
    ky = np.fft.fftfreq(ny, d=p["DH"]) * 2 * np.pi
    KX, KY = np.meshgrid(kx, ky)
    filt = np.exp(-(KX ** 2 + KY ** 2) * corr ** 2 / 8.0)
    field = np.real(np.fft.ifft2(np.fft.fft2(white) * filt))
    field -= field.mean()
    field *= rms / max(field.std(), 1e-12)
    return field.astype(np.float32)


def layered_bytes(layers):
    """layers: [(bottom_depth_km, vs_kms, vp_kms, rho_gcc), ...]."""
    out = struct.pack("<i", len(layers))
    for row in layers:
        out += struct.pack("<4f", *row)
    return out


def ricker_rate(t, f0, t0):
    """Ricker wavelet (1 - 2 r^2) exp(-r^2), r = pi f0 (t - t0)."""
    r = np.pi * f0 * (t - t0)
    return (1.0 - 2.0 * r ** 2) * np.exp(-r ** 2)


def gaussian_rate(t, width, t0):
    """Unit-area Gaussian slip-rate function of standard deviation ``width``."""
    return np.exp(-0.5 * ((t - t0) / width) ** 2) / (width * math.sqrt(2 * math.pi))


def source_bytes(points, nt, dt):
    """points: list of dicts x, y, z, area, strike, dip, rake[nt], rate[nt]."""
    out = struct.pack("<iif", len(points), nt, dt)
    for q in points:
        out += struct.pack("<6f", q["x"], q["y"], q["z"], q["area"], q["strike"], q["dip"])
        out += np.asarray(q["rake"], np.float32).tobytes()
        out += np.asarray(q["rate"], np.float32).tobytes()
    return out


def double_couple_point(x, y, z, m0, mu, strike, dip, rake, nt, dt, stf):
    """One double-couple point source through the finite-fault path: area is
    M0/mu (unit slip), rate is the slip-rate time function ``stf`` sampled at
    dt.  A zero-area anchor at z=0 keeps the reader's depth shift
    (z - max z, multiSource.cpp:211-225) from moving the source."""
    t = np.arange(nt) * dt
    pts = [dict(x=x, y=y, z=z, area=m0 / mu, strike=strike, dip=dip,
                rake=np.full(nt, rake, np.float32), rate=stf(t).astype(np.float32)),
           dict(x=x, y=y, z=0.0, area=0.0, strike=strike, dip=dip,
                rake=np.full(nt, rake, np.float32), rate=np.zeros(nt, np.float32))]
    return source_bytes(pts, nt, dt)


def finite_fault(cx, cy, cz, length, width, nl, nw, strike, dip, rake, mean_slip,
                 vs_rupture, stf_width, nt, dt, seed, mu=3.2e10, surface_z=0.0):
    """Planar fault of nl x nw point sources centred at (cx, cy, cz) with
    seeded log-normal slip of mean ``mean_slip``; rupture starts at the
    centre and spreads at ``vs_rupture``; each point's slip rate is a Gaussian
    of width ``stf_width`` (s) delayed by its rupture time, scaled by its
    slip.  Returns the source file bytes."""
    rng = np.random.default_rng(seed)
    sigma = 0.5
    slip = rng.lognormal(mean=math.log(mean_slip) - sigma ** 2 / 2, sigma=sigma, size=(nw, nl))
    s, d = math.radians(strike), math.radians(dip)
    us = np.array([math.sin(s), math.cos(s), 0.0])             # along strike
    ud = np.array([math.cos(d) * math.cos(s), -math.cos(d) * math.sin(s),
                   -math.sin(d)])                               # down dip
    t = np.arange(nt) * dt
    area = (length / nl) * (width / nw)
    pts = []
    for iw in range(nw):
        for il in range(nl):
            a = (il + 0.5) / nl * length - length / 2
            b = (iw + 0.5) / nw * width - width / 2
            pos = np.array([cx, cy, cz]) + a * us + b * ud
            delay = math.hypot(a, b) / vs_rupture
            rate = slip[iw, il] * gaussian_rate(t, stf_width, delay + 3 * stf_width)
            pts.append(dict(x=pos[0], y=pos[1], z=pos[2], area=area, strike=strike, dip=dip,
                            rake=np.full(nt, rake, np.float32), rate=rate.astype(np.float32)))
    pts.append(dict(x=cx, y=cy, z=surface_z, area=0.0, strike=strike, dip=dip,
                    rake=np.full(nt, rake, np.float32), rate=np.zeros(nt, np.float32)))
    return source_bytes(pts, nt, dt)


def write_run_dir(dirpath, p, stations=None, terrain=None, layers=None, source=None):
    """Writes params.json, station.json, terrain_input.bin, the layered file
    and the source file of a run into ``dirpath``."""
    os.makedirs(dirpath, exist_ok=True)
    with open(os.path.join(dirpath, "params.json"), "w") as f:
        json.dump(p, f, indent=1)
    if stations is not None:
        with open(os.path.join(dirpath, "station.json"), "w") as f:
            json.dump({"station(point)": stations}, f, indent=1)
    if terrain is not None:
        np.asarray(terrain, np.float32).tofile(os.path.join(dirpath, "terrain_input.bin"))
    if layers is not None:
        with open(os.path.join(dirpath, p["LayeredFileName"]), "wb") as f:
            f.write(_as_bytes(layers))
    if source is not None:
        os.makedirs(os.path.join(dirpath, p["sourceDir"]), exist_ok=True)
        with open(os.path.join(dirpath, p["sourceDir"], p["sourceFile"]), "wb") as f:
            f.write(_as_bytes(source))


def _as_bytes(x):
    return x.tobytes() if isinstance(x, np.ndarray) else bytes(x)


def sample_scenario(seed, nx_range=(121, 401), nz_range=(101, 201), points=None,
                    nsteps=100, dt=0.008, npml=12):
    """One seeded scenario of the batched-serving workloads: grid sizes
    uniform in the ranges (or, with ``points`` given, NX = NY chosen so that
    NX * NY * NZ is close to it), a Gaussian hill of amplitude U[0, 2000] m,
    a three-layer medium with seeded layer depths and velocities (+-5 %), a
    double-couple point source of random strike / dip / rake at 1-10 km depth
    with a Ricker source time function of f0 U[0.5, 3] Hz, and a 5 x 5
    station lattice on the surface.  Returns dict(params, terrain, layers,
    source, stations)."""
    rng = np.random.default_rng(seed)
    nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
    if points is None:
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        ny = int(rng.integers(nx_range[0], nx_range[1] + 1))
    else:
        nx = ny = max(40, int(round(math.sqrt(points / nz))))
    dh = 100.0
    depth_km = (nz - 1) * dh / 1000.0
    p = params(NX=nx, NY=ny, NZ=nz, DH=dh, DT=dt, TMAX=(nsteps + 0.5) * dt,
               **{"Depth(km)": depth_km}, centerX=0, centerY=0, nPML=npml, useTerrain=1,
               useMedium=1, LayeredModel=1, useMultiSource=1,
               **{"useSingleSource(ricker)": 0}, IT_SKIP=10 ** 7, out="out")
    amp = float(rng.uniform(0.0, 2000.0))
    terrain = gaussian_hill(p, amp=amp, x0=nx * dh / 2, y0=ny * dh / 2,
                            width=max(nx, ny) * dh / 8)
    j = lambda: float(rng.uniform(0.95, 1.05))
    d1, d2 = float(rng.uniform(1.5, 2.5)), float(rng.uniform(6.0, 10.0))
    layers = layered_bytes([(d1, 2.6 * j(), 4.5 * j(), 2.3), (d2, 3.35 * j(), 5.8 * j(), 2.6),
                            (1000.0, 3.75 * j(), 6.5 * j(), 2.8)])
    f0 = float(rng.uniform(0.5, 3.0))
    zdepth = float(rng.uniform(1000.0, min(10000.0, 0.6 * depth_km * 1000.0)))
    x = float(rng.uniform(0.3, 0.7)) * nx * dh
    y = float(rng.uniform(0.3, 0.7)) * ny * dh
    nt_src = nsteps + 8
    src = double_couple_point(x, y, -zdepth, m0=1e16, mu=3.2e10,
                              strike=float(rng.uniform(0, 360)), dip=float(rng.uniform(10, 90)),
                              rake=float(rng.uniform(-180, 180)), nt=nt_src, dt=dt,
                              stf=lambda t: ricker_rate(t, f0, 1.2 / f0))
    stations = {"S%02d" % (a * 5 + b): [int(nx * (a + 1) / 6), int(ny * (b + 1) / 6), nz - 1]
                for a in range(5) for b in range(5)}
    return {"params": p, "terrain": terrain, "layers": layers, "source": src,
            "stations": stations}



# --------------------------------------------------------------------------
# the benchmark configurations
# --------------------------------------------------------------------------
C2_LAYERS = [(2.0, 2.6, 4.5, 2.3), (8.0, 3.35, 5.8, 2.6), (1000.0, 3.75, 6.5, 2.8)]


def c2_workload(nsteps_total, it_skip=10 ** 7, slice_free_surf=0):
    """401 x 401 x 201 Gaussian hill (1500 m at x = y = 20 km, 5 km width),
    bottom at -20 km, three layers, 20-cell PML, explosive Ricker source
    (f0 = 2 Hz, the single-source path) 3 km under the hill flank, 121
    surface stations on an 11 x 11 lattice 3 km apart.  ``it_skip`` and
    ``slice_free_surf`` ask for free-surface snapshots every it_skip steps."""
    NX, NY, NZ, DH = 401, 401, 201, 100.0
    dt = 0.008
    p = params(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=dt, TMAX=(nsteps_total + 0.5) * dt,
               **{"Depth(km)": 20.0}, centerX=0, centerY=0, nPML=20, useTerrain=1,
               useMedium=1, LayeredModel=1, rickerfc=2.0, IT_SKIP=it_skip,
               sliceFreeSurf=slice_free_surf, out="out")
    terrain = gaussian_hill(p, amp=1500.0, x0=20000.0, y0=20000.0, width=5000.0)
    # source at i=170, j=200, 3 km below the local surface
    h = float(terrain[200 + HALO, 170 + HALO])
    dz = (h + 20000.0) / (NZ - 1)
    p.update(sourceX=170, sourceY=200, sourceZ=int(round(NZ - 1 - 3000.0 / dz)))
    stations = {"S%03d" % (a * 11 + b): [50 + 30 * a, 50 + 30 * b, NZ - 1]
                for a in range(11) for b in range(11)}
    return {"name": "c2-gaussian-hill-401x401x201", "params": p, "stations": stations,
            "terrain": terrain, "layers": layered_bytes(C2_LAYERS)}


def c3_workload(n, nsteps_total, perturbation=0.05, it_skip=10 ** 7, slice_free_surf=0):
    """n x n x 401 PerformanceTest shape (PerformanceTest/params.json_*):
    seeded random terrain (500 m RMS, 10 km correlation), the C2 layers with
    a seeded +-``perturbation`` velocity perturbation per cell (a host-setup
    extension; the reference's own medium reader has none), a finite fault
    of 80 x 40 points (40 x 20 km where the grid allows, strike 90, dip 30,
    log-normal slip of mean 1.5 m, rupture at 0.8 Vs, Gaussian slip rate of
    1 s), 121 surface stations."""
    NZ, DH, dt = 401, 100.0, 0.008
    extra = dict(mediumPerturbation=perturbation, mediumSeed=3) if perturbation else {}
    p = params(NX=n, NY=n, NZ=NZ, DH=DH, DT=dt, TMAX=(nsteps_total + 0.5) * dt,
               **{"Depth(km)": 40.0}, centerX=n // 2, centerY=n // 2, nPML=12,
               useTerrain=1, useMedium=1, LayeredModel=1, useMultiSource=1,
               **{"useSingleSource(ricker)": 0}, IT_SKIP=it_skip,
               sliceFreeSurf=slice_free_surf, out="out", **extra)
    terrain = random_terrain(p, rms=500.0, corr=10000.0, seed=11)
    fault_len = min(40000.0, (n - 40) * DH * 0.6)
    fault_wid = fault_len / 2
    nt_src = nsteps_total + 8
    src = finite_fault(cx=0.0, cy=0.0, cz=-12000.0, length=fault_len, width=fault_wid,
                       nl=80, nw=40, strike=90.0, dip=30.0, rake=90.0, mean_slip=1.5,
                       vs_rupture=0.8 * 3350.0, stf_width=1.0, nt=nt_src, dt=dt, seed=5,
                       surface_z=float(terrain.max()))
    stations = {"S%03d" % (a * 11 + b): [n // 12 * (a + 1), n // 12 * (b + 1), NZ - 1]
                for a in range(11) for b in range(11)}
    return {"name": "c3-perftest-%dx%dx401" % (n, n), "params": p, "stations": stations,
            "terrain": terrain, "layers": layered_bytes(C2_LAYERS), "source": src}


# --------------------------------------------------------------------------
# SRTM90 DEM tiles (terrain.cpp:217-307): 6000 x 6000 float heights per 5 x 5
# degree tile, x (longitude) fastest, file srtm_<lat>N<lon>E.bin
# --------------------------------------------------------------------------
DEM_POINTS = 6000


def synthetic_dem_tile(lon0, lat0, seed, spikes=(), holes=()):
    """A seeded smooth DEM tile (heights in metres, float32, shape (6000,
    6000), row = latitude index): a few broad Gaussian mountains on a gentle
    slope.  ``spikes`` (i, j, metres) add single-point peaks, the steep local
    gradients the reader smooths away; ``holes`` (i, j) set the SRTM void
    value -32768, which the reader resets to zero."""
    rng = np.random.default_rng(seed)
    ax = np.arange(DEM_POINTS, dtype=np.float64) / DEM_POINTS
    X, Y = np.meshgrid(ax, ax)
    h = 300.0 + 400.0 * X + 200.0 * Y
    for _ in range(6):
        cx, cy = rng.uniform(0.2, 0.8, 2)
        w = rng.uniform(0.05, 0.3)
        h += rng.uniform(500.0, 2500.0) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / w ** 2)
    t = h.astype(np.float32)
    for i, j, dz in spikes:
        t[j, i] += np.float32(dz)
    for i, j in holes:
        t[j, i] = np.float32(-32768.0)
    return t


def write_dem_tile(dirpath, lon0, lat0, tile):
    os.makedirs(dirpath, exist_ok=True)
    fn = os.path.join(dirpath, "srtm_%dN%dE.bin" % (lat0, lon0))
    np.ascontiguousarray(tile, np.float32).tofile(fn)
    return fn
