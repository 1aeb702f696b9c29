"""ctypes binding of the ORACLE (liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, as the checker.  It wraps the C restatement in cgfdm_oracle.c
with numpy arrays in the reference's memory layout and adds a small driver
(``run``) that strings the per-step pieces together exactly as
src-new-FP32-SVE/propagate.cpp:142-198 does on a single rank.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
HALO = 3

_lib = None


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "cgfdm_oracle.c")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nPML", C.c_int),
                ("DH", C.c_float), ("rDH", C.c_float)]


class Aux(C.Structure):
    _fields_ = [("h", C.c_void_p), ("a", C.c_void_p), ("t", C.c_void_p), ("m", C.c_void_p)]


class Aux5(C.Structure):
    _fields_ = [("slab", Aux * 5)]


class Pml(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("alpha_x", "beta_x", "d_x", "alpha_y", "beta_y", "d_y", "alpha_z", "beta_z", "d_z")]


def _declare(L):
    P, I, F, LL = C.c_void_p, C.c_int, C.c_float, C.c_longlong
    G = C.POINTER(Grid)
    L.oracle_num.restype = LL
    L.oracle_num.argtypes = [G]
    L.oracle_slab_points.restype = LL
    L.oracle_slab_points.argtypes = [G, I]
    L.oracle_pml_params.argtypes = [G, C.POINTER(Pml)]
    L.oracle_stage.argtypes = [G, I, I, I, I, F, P, P, P, P, P, P, P, C.POINTER(Pml),
                               C.POINTER(Aux5)]
    L.oracle_ricker_moment.restype = F
    L.oracle_ricker_moment.argtypes = [F, I, F]
    L.oracle_smooth_source.argtypes = [G, P, P, I, I, I, I, F, F]
    L.oracle_add_moment_rate.restype = I
    L.oracle_add_moment_rate.argtypes = [G, P, P, P, LL, I, F, I, F]
    L.oracle_scale_moment_rate.argtypes = [G, P, P, P, LL, I]
    L.oracle_station.argtypes = [G, P, P, I, I, I, P]
    L.oracle_pgv.argtypes = [G, P, P]


def _p(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def make_grid(nx, ny, nz, nPML, DH):
    return Grid(nx, ny, nz, nPML, np.float32(DH), np.float32(1.0 / np.float32(DH)))


class PmlProfiles:
    """alpha/beta/d profiles along x, y, z (init_pml_para.cpp layout order)."""

    def __init__(self, g):
        n_ = [g.nx + 2 * HALO, g.ny + 2 * HALO, g.nz + 2 * HALO]
        self.block = np.zeros(3 * sum(n_), np.float32)
        views, off = [], 0
        for n in n_:
            for _ in range(3):
                views.append(self.block[off: off + n])
                off += n
        self.views = views  # ax, bx, dx, ay, by, dy, az, bz, dz
        self.struct = Pml(*[v.ctypes.data for v in views])
        lib().oracle_pml_params(C.byref(g), C.byref(self.struct))


class AuxState:
    """PML auxiliaries: 5 slabs x 4 buffers of [npos][9] float32."""

    def __init__(self, g):
        self.bufs = []
        self.struct = Aux5()
        for s in range(5):
            n = lib().oracle_slab_points(C.byref(g), s)
            b = [np.zeros(n * 9, np.float32) for _ in range(4)]
            self.bufs.append(b)
            self.struct.slab[s] = Aux(*[x.ctypes.data for x in b])


class State:
    """Wavefield buffers h, W, t, m (each 9 * num float32) plus PML aux."""

    def __init__(self, g):
        num = lib().oracle_num(C.byref(g))
        self.num = num
        self.h = np.zeros(9 * num, np.float32)
        self.W = np.zeros(9 * num, np.float32)
        self.t = np.zeros(9 * num, np.float32)
        self.m = np.zeros(9 * num, np.float32)
        self.aux = AuxState(g)


def stage(g, irk, fb, DT, st, cjm, rdz, pml):
    nsurf = (g.nx + 2 * HALO) * (g.ny + 2 * HALO)
    lib().oracle_stage(C.byref(g), irk, fb[0], fb[1], fb[2], np.float32(DT), _p(st.h), _p(st.W),
                       _p(st.t), _p(st.m), _p(cjm), _p(rdz), rdz.ctypes.data + 4 * 9 * nsurf,
                       C.byref(pml.struct), C.byref(st.aux.struct))


FB_TABLE = [(-1, -1, -1), (1, 1, -1), (1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1),
            (1, -1, 1), (-1, 1, 1)]


def run(g, DT, NT, cjm, rdz, *, point=None, rickerfc=1.5, fault=None, stations=None,
        snapshot_every=None, steps=None):
    """Runs ``steps`` (default NT) time steps from rest, like propagate.cpp.

    point:    (sx, sy, sz) padded indices of the smoothed single source
    fault:    dict(srcIndex int64[npts], momentRate float32[nt*npts*6] (scaled),
              nt, dt) for the multi-source path
    stations: int32[nsta, 3] padded indices
    Returns dict with station_wave [nsta, NT, 9], pgv [ny, nx, 2], snapshots.
    """
    L = lib()
    st = State(g)
    pml = PmlProfiles(g)
    steps = NT if steps is None else steps
    out = {}
    nsta = 0 if stations is None else len(stations)
    if nsta:
        xyz = np.ascontiguousarray(stations, np.int32)
        wave = np.zeros(nsta * NT * 9, np.float32)
    pgv = np.zeros(g.ny * g.nx * 2, np.float32)
    snaps, snap_its = [], []
    fault_on = fault is not None
    num = st.num
    for it in range(steps):
        fb = list(FB_TABLE[it % 8])
        if point is not None:
            L.oracle_smooth_source(C.byref(g), _p(st.W), _p(cjm), point[0], point[1], point[2],
                                   it, np.float32(DT), np.float32(rickerfc))
        if fault_on:
            fault_on = bool(L.oracle_add_moment_rate(
                C.byref(g), _p(st.W), _p(fault["srcIndex"]), _p(fault["momentRate"]),
                len(fault["srcIndex"]), fault["nt"], np.float32(fault["dt"]), it,
                np.float32(DT)))
        for irk in range(4):
            stage(g, irk, fb, DT, st, cjm, rdz, pml)
            fb = [-f for f in fb]
        if nsta:
            L.oracle_station(C.byref(g), _p(st.W), _p(xyz), nsta, NT, it, _p(wave))
        L.oracle_pgv(C.byref(g), _p(st.W), _p(pgv))
        if snapshot_every and it % snapshot_every == 0:
            k = g.nz + HALO - 1
            W = st.W.reshape(9, g.nz + 6, g.ny + 6, g.nx + 6)
            snaps.append(W[0:3, k, HALO:-HALO, HALO:-HALO].copy())
            snap_its.append(it)
    if nsta:
        out["station_wave"] = wave.reshape(nsta, NT, 9)
    out["pgv"] = pgv.reshape(g.ny, g.nx, 2)
    if snaps:
        out["freesurf"] = np.stack(snaps)
        out["freesurf_its"] = np.array(snap_its)
    out["W"] = st.W
    return out


def scale_moment_rate(g, cjm, momentRate, srcIndex, nt):
    mr = np.ascontiguousarray(momentRate, np.float32).copy()
    lib().oracle_scale_moment_rate(C.byref(g), _p(cjm), _p(mr), _p(srcIndex), len(srcIndex), nt)
    return mr
