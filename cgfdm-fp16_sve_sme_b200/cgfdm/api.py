"""Python host API over the C ABI (numpy arrays in, numpy arrays out).

Mirrors the reference's hot-path interface: ``Simulation`` is the state that
propagate() (src-new-FP32-SVE/propagate.cpp:24-228) owns on one rank,
``propagate`` is the one-call drop-in, ``setup_from_directory`` is the host
setup of run.cpp:56-131 and ``run_directory`` the whole program.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import CgfdmError, Desc, check, lib

HALO = 3


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, np.float32)


def make_desc(nx, ny, nz, npml, dh, dt, nt, precision=_lib.FP32, kernel=_lib.KERNEL_AUTO,
              device=0):
    return Desc(nx, ny, nz, npml, np.float32(dh), np.float32(dt), nt, precision, kernel, device)


def device_bytes(desc):
    n = C.c_int64()
    check(lib().cgfdm_device_bytes(C.byref(desc), C.byref(n)))
    return n.value


class Simulation:
    """One simulation resident on one GPU (a C-ABI handle)."""

    def __init__(self, desc):
        self.desc = desc
        self.nx_, self.ny_, self.nz_ = desc.nx + 2 * HALO, desc.ny + 2 * HALO, desc.nz + 2 * HALO
        self.num = self.nx_ * self.ny_ * self.nz_
        self.nsurf = self.nx_ * self.ny_
        h = C.c_void_p()
        check(lib().cgfdm_create(C.byref(desc), C.byref(h)))
        self._h = h
        self.nsta = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().cgfdm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- inputs -----------------------------------------------------------
    def set_model(self, cjm, rdz):
        cjm, rdz = _f32(cjm), _f32(rdz)
        assert cjm.size == 13 * self.num and rdz.size == 18 * self.nsurf
        check(lib().cgfdm_set_model(self._h, _ptr(cjm), _ptr(rdz)))

    def set_point_source(self, sx, sy, sz, rickerfc):
        check(lib().cgfdm_set_point_source(self._h, sx, sy, sz, np.float32(rickerfc)))

    def set_fault_source(self, src_index, moment_rate, nt, dt, scaled=True):
        idx = np.ascontiguousarray(src_index, np.int64)
        mr = _f32(moment_rate)
        assert mr.size == idx.size * nt * 6
        check(lib().cgfdm_set_fault_source(self._h, _ptr(idx), _ptr(mr), idx.size, nt,
                                           np.float32(dt), int(scaled)))

    def set_stations(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
        check(lib().cgfdm_set_stations(self._h, _ptr(xyz), len(xyz)))
        self.nsta = len(xyz)

    # ---- execution --------------------------------------------------------
    def run(self, nsteps, stream=None):
        check(lib().cgfdm_run(self._h, nsteps, stream))

    def stage(self, irk, fb, stream=None):
        check(lib().cgfdm_stage(self._h, irk, fb[0], fb[1], fb[2], stream))

    def synchronize(self):
        check(lib().cgfdm_synchronize(self._h))

    def steps_done(self):
        it = C.c_int32()
        check(lib().cgfdm_steps_done(self._h, C.byref(it)))
        return it.value

    def set_timing(self, on=True):
        check(lib().cgfdm_set_timing(self._h, int(on)))

    def timing_ms(self):
        ms = np.zeros(3, np.float32)
        check(lib().cgfdm_get_timing(self._h, _ptr(ms)))
        return ms

    def checkpoint(self):
        """The handle's state at the current step boundary (bytes)."""
        n = C.c_int64()
        check(lib().cgfdm_checkpoint_bytes(self._h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        check(lib().cgfdm_checkpoint_save(self._h, _ptr(buf), n.value))
        return buf

    def restore(self, buf):
        """Continue from a checkpoint of a handle with the same descriptor,
        sources and stations."""
        buf = np.ascontiguousarray(buf, np.uint8)
        check(lib().cgfdm_checkpoint_load(self._h, _ptr(buf), buf.size))

    def inject_fault(self, kind=1):
        """Failure-detection tests: the next streaming launch leaves one load
        unissued so that a bounded device wait expires (CGFDM_ERR_TIMEOUT)."""
        check(lib().cgfdm_inject_fault(self._h, int(kind)))

    def set_graph(self, on=True):
        """Replay each step of run() as a CUDA graph (results are identical)."""
        check(lib().cgfdm_set_graph(self._h, int(on)))

    def set_chunk(self, planes):
        """Planes per streaming work item in z (0: automatic)."""
        check(lib().cgfdm_set_chunk(self._h, int(planes)))

    def tuning(self):
        """(tile form, planes per work item) of the streaming kernel."""
        return self.tuning3()[:2]

    def tuning3(self):
        """(tile form, planes per work item, tiled free-surface kernel 0/1)."""
        v = np.zeros(3, np.int32)
        check(lib().cgfdm_get_tuning(self._h, _ptr(v)))
        return int(v[0]), int(v[1]), int(v[2])

    def set_tile_rows(self, rows):
        """Streaming-kernel tile height: 16, 8, or 0 to autotune at the first run."""
        check(lib().cgfdm_set_tile_rows(self._h, int(rows)))

    def kernel_stats(self):
        """Per-kernel device view of the last run (cgfdm_get_kernel_stats)."""
        v = np.zeros(8, np.float64)
        check(lib().cgfdm_get_kernel_stats(self._h, _ptr(v)))
        return {"stream_ms": v[0], "stream_launches": int(v[1]), "stream_bytes": v[2],
                "launches": int(v[3]), "gap_ms": v[4], "exact_ms": v[5],
                "stages": int(v[6]), "tile_rows": int(v[7])}

    # ---- outputs ----------------------------------------------------------
    def stations(self):
        out = np.zeros((self.nsta, self.desc.nt, 9), np.float32)
        if self.nsta:
            check(lib().cgfdm_get_stations(self._h, _ptr(out)))
        return out

    def pgv(self):
        out = np.zeros((self.desc.ny, self.desc.nx, 2), np.float32)
        check(lib().cgfdm_get_pgv(self._h, _ptr(out)))
        return out

    def wavefield(self):
        out = np.zeros(9 * self.num, np.float32)
        check(lib().cgfdm_get_wavefield(self._h, _ptr(out)))
        return out

    def free_surface(self):
        out = np.zeros((3, self.desc.ny, self.desc.nx), np.float32)
        check(lib().cgfdm_get_free_surface(self._h, _ptr(out)))
        return out

    def aux_floats(self):
        n = C.c_int64()
        check(lib().cgfdm_aux_floats(self._h, C.byref(n)))
        return n.value

    def set_state(self, irk, W=None, t=None, m=None, aux=None):
        W, t, m, aux = _f32(W), _f32(t), _f32(m), _f32(aux)
        check(lib().cgfdm_set_state(self._h, irk, _ptr(W), _ptr(t), _ptr(m), _ptr(aux)))

    def get_state(self):
        W = np.zeros(9 * self.num, np.float32)
        t = np.zeros_like(W)
        m = np.zeros_like(W)
        aux = np.zeros(3 * self.aux_floats(), np.float32)
        check(lib().cgfdm_get_state(self._h, _ptr(W), _ptr(t), _ptr(m), _ptr(aux)))
        return {"W": W, "t": t, "m": m, "aux": aux}


class Batch:
    """Several Simulations of one precision advanced together (cgfdm_batch):
    one persistent streaming launch per stage spans all members.  The
    members must outlive the batch; read results from the members after
    synchronize()."""

    def __init__(self, sims, graph=False):
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s._h.value for s in self.sims])
        b = C.c_void_p()
        check(lib().cgfdm_batch_create(arr, len(self.sims), C.byref(b)))
        self._b = b
        if graph:
            check(lib().cgfdm_batch_set_graph(self._b, 1))

    def run(self, nsteps, stream=None):
        check(lib().cgfdm_batch_run(self._b, int(nsteps), stream))

    def synchronize(self):
        check(lib().cgfdm_batch_synchronize(self._b))

    def close(self):
        if getattr(self, "_b", None):
            lib().cgfdm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Server:
    """The library's request loop with continuous batching (cgfdm_server_*).

    submit() queues a simulation and returns its id at once; the server's
    worker admits requests by free HBM, advances all admitted requests of a
    precision as one batch, and streams seismogram rows back every `chunk`
    steps.  wait(id) returns (seismograms, pgv, (ms to first chunk, ms to
    completion))."""

    def __init__(self, hbm_budget_bytes=0, chunk=100, device=0, graph=True):
        o = _lib.ServerOpts(int(hbm_budget_bytes), int(chunk), int(device), int(graph))
        sv = C.c_void_p()
        check(lib().cgfdm_server_create(C.byref(o), C.byref(sv)))
        self._s = sv
        self._shape = {}

    def submit(self, desc, cjm, rdz, *, point=None, rickerfc=0.0, src_index=None,
               moment_rate=None, src_nt=0, src_dt=0.0, stations=None):
        cjm, rdz = _f32(cjm), _f32(rdz)
        pxyz = None if point is None else np.ascontiguousarray(point, np.int32)
        idx = None if src_index is None else np.ascontiguousarray(src_index, np.int64)
        mr = _f32(moment_rate)
        sta = None if stations is None else np.ascontiguousarray(stations, np.int32).reshape(-1, 3)
        nsta = 0 if sta is None else len(sta)
        rid = C.c_int64()
        check(lib().cgfdm_server_submit(
            self._s, C.byref(desc), _ptr(cjm), _ptr(rdz), int(point is not None), _ptr(pxyz),
            np.float32(rickerfc), _ptr(idx), _ptr(mr), 0 if idx is None else idx.size, src_nt,
            np.float32(src_dt), _ptr(sta), nsta, C.byref(rid)))
        self._shape[rid.value] = (nsta, desc.nt, desc.ny, desc.nx)
        return rid.value

    def poll(self, rid):
        st, steps = C.c_int32(), C.c_int32()
        check(lib().cgfdm_server_poll(self._s, rid, C.byref(st), C.byref(steps)))
        return st.value, steps.value

    def read_rows(self, rid, out, start=0):
        """Copies the rows streamed back so far (from `start`) into out
        ([nsta][nt][9] float32); returns the row count available."""
        upto = C.c_int32()
        check(lib().cgfdm_server_read_rows(self._s, rid, start, _ptr(out), C.byref(upto)))
        return upto.value

    def wait(self, rid):
        nsta, nt, ny, nx = self._shape.pop(rid, (0, 0, 0, 0))
        wave = np.zeros((nsta, nt, 9), np.float32)
        pgv = np.zeros((ny, nx, 2), np.float32)
        lat = np.zeros(2, np.float64)
        check(lib().cgfdm_server_wait(self._s, rid, _ptr(wave), _ptr(pgv), _ptr(lat)))
        return wave, pgv, (float(lat[0]), float(lat[1]))

    def cancel(self, rid):
        check(lib().cgfdm_server_cancel(self._s, rid))

    def stats(self):
        v = np.zeros(8, np.float64)
        check(lib().cgfdm_server_stats(self._s, _ptr(v)))
        return {"first_p50_ms": v[0], "first_p99_ms": v[1], "done_p50_ms": v[2],
                "done_p99_ms": v[3], "gpts": v[4], "completed": int(v[5]), "busy_s": v[6],
                "peak_bytes": v[7]}

    def close(self):
        if getattr(self, "_s", None):
            lib().cgfdm_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def propagate(desc, cjm, rdz, *, point=None, rickerfc=0.0, src_index=None, moment_rate=None,
              src_nt=0, src_dt=0.0, stations=None):
    """propagate() drop-in with host buffers; returns (stations, pgv, free_surface)."""
    cjm, rdz = _f32(cjm), _f32(rdz)
    pxyz = None if point is None else np.ascontiguousarray(point, np.int32)
    idx = None if src_index is None else np.ascontiguousarray(src_index, np.int64)
    mr = _f32(moment_rate)
    sta = None if stations is None else np.ascontiguousarray(stations, np.int32).reshape(-1, 3)
    nsta = 0 if sta is None else len(sta)
    out_sta = np.zeros((nsta, desc.nt, 9), np.float32)
    out_pgv = np.zeros((desc.ny, desc.nx, 2), np.float32)
    out_fs = np.zeros((3, desc.ny, desc.nx), np.float32)
    check(lib().cgfdm_propagate(C.byref(desc), _ptr(cjm), _ptr(rdz), int(point is not None),
                                _ptr(pxyz), np.float32(rickerfc), _ptr(idx), _ptr(mr),
                                0 if idx is None else idx.size, src_nt, np.float32(src_dt),
                                _ptr(sta), nsta, _ptr(out_sta) if nsta else None,
                                _ptr(out_pgv), _ptr(out_fs)))
    return out_sta, out_pgv, out_fs


class _SetupOwner:
    """Releases a library-built setup once no array views it any more."""

    def __init__(self, s):
        self.s = s

    def __del__(self):
        try:
            lib().cgfdm_free_setup(C.byref(self.s))
        except Exception:  # noqa: BLE001  (interpreter shutdown)
            pass


def _view(ptr, n, ctype, dtype, owner):
    if n == 0:
        return np.zeros(0, dtype)
    buf = (ctype * n).from_address(C.addressof(ptr.contents))
    buf._owner = owner  # keeps the library storage alive while viewed
    return np.frombuffer(buf, dtype=dtype)


def setup_from_directory(run_dir, precision=_lib.FP32):
    """Host setup (params.json, station.json, model files) -> dict of arrays.

    precision selects the storage scaling of cjm and the moment rates
    (FP16/BF16: the reference's Cv, Cs, Crho).  The arrays are views of the
    library's own buffers (no copies), released when the last view goes.
    """
    s = _lib.Setup()
    check(lib().cgfdm_setup_from_directory_ex(run_dir.encode(), int(precision), C.byref(s)))
    owner = _SetupOwner(s)
    d = s.desc
    nx_, ny_, nz_ = d.nx + 6, d.ny + 6, d.nz + 6
    num, nsurf = nx_ * ny_ * nz_, nx_ * ny_
    f32 = lambda p, n: _view(p, n, C.c_float, np.float32, owner)
    return {
        "desc": Desc(*[getattr(d, f) for f, _ in Desc._fields_]),
        "cjm": f32(s.cjm, 13 * num), "rdz": f32(s.rdz, 18 * nsurf),
        "coord": f32(s.coord, 3 * num), "medium": f32(s.medium, 3 * num),
        "pml": f32(s.pml, 3 * (nx_ + ny_ + nz_)),
        "point": tuple(s.point_xyz) if s.point_src else None, "rickerfc": s.rickerfc,
        "src_index": _view(s.src_index, s.npts, C.c_int64, np.int64, owner),
        "moment_rate": f32(s.moment_rate, s.npts * s.src_nt * 6),
        "src_nt": s.src_nt, "src_dt": s.src_dt,
        "stations": _view(s.sta_xyz, 3 * s.nsta, C.c_int32, np.int32, owner).reshape(-1, 3),
        "terrain": f32(s.terrain, nsurf).reshape(ny_, nx_),
        "precision": int(precision),
    }


def hbm_layout(nx, ny, nz, elem_bytes):
    """The device layout of wavefield and coefficient buffers (the formula in
    include/cgfdm_b200.h beside cgfdm_stage_buffers): field f of padded point
    (i, j, k) at element f * fs + xoff + i + j * px + k * plane."""
    nx_, ny_, nz_ = nx + 6, ny + 6, nz + 6
    xoff = 128 // elem_bytes - 3
    px = (nx_ + xoff + 31) // 32 * 32
    plane = px * ny_
    fs = (plane * nz_ + 31) // 32 * 32
    return {"nx_": nx_, "ny_": ny_, "nz_": nz_, "xoff": xoff, "px": px, "plane": plane,
            "fs": fs}


def stage_noalloc(buffers, stream=None, wait=True):
    """cgfdm_stage_noalloc: one RK stage on device buffers the caller already
    owns (a StageBuffers of device pointers), for hosts that cannot allocate
    device memory while running.  Allocates nothing."""
    check(lib().cgfdm_stage_noalloc(C.byref(buffers), stream, int(wait)))


def run_directory(run_dir, precision=_lib.FP32, kernel=_lib.KERNEL_AUTO, device=0):
    """The reference program on one GPU: reads run_dir, writes its outputs."""
    check(lib().cgfdm_run_directory(run_dir.encode(), precision, kernel, device))


__all__ = ["Simulation", "Batch", "Server", "propagate", "setup_from_directory", "run_directory", "make_desc",
           "device_bytes", "CgfdmError", "hbm_layout", "stage_noalloc"]
