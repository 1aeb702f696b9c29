"""ctypes binding of lib/libcgfdm_b200.so (the C ABI of include/cgfdm_b200.h).

There is no CPU fallback: if the shared library is missing or cannot be
loaded, every entry point raises.  The library is built in-tree by
``make -C cgfdm-fp16_sve_sme_b200`` (or ``__graft_entry__.build()``).
"""
import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libcgfdm_b200.so")

OK = 0
ERR = {1: "ARG", 100: "PARAMS", 110: "CFL", 130: "PML", 180: "NO_SOURCE", 181: "SOURCE",
       200: "IO", 300: "CUDA", 301: "NOMEM", 302: "NO_KERNEL", 303: "TIMEOUT", 304: "STATE",
       305: "CANCELLED"}
FP32, FP16, BF16, FP64 = 0, 1, 2, 3
KERNEL_AUTO, KERNEL_EXACT, KERNEL_STREAM = 0, 1, 2
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4


class CgfdmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cgfdm error %d (%s): %s" % (code, ERR.get(code, "?"), msg))
        self.code = code


class Desc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("npml", C.c_int32),
                ("dh", C.c_float), ("dt", C.c_float), ("nt", C.c_int32),
                ("precision", C.c_int32), ("kernel", C.c_int32), ("device", C.c_int32)]


class Setup(C.Structure):
    _fields_ = [("desc", Desc),
                ("cjm", C.POINTER(C.c_float)), ("rdz", C.POINTER(C.c_float)),
                ("coord", C.POINTER(C.c_float)), ("medium", C.POINTER(C.c_float)),
                ("pml", C.POINTER(C.c_float)),
                ("point_src", C.c_int32), ("point_xyz", C.c_int32 * 3), ("rickerfc", C.c_float),
                ("npts", C.c_int64), ("src_nt", C.c_int32), ("src_dt", C.c_float),
                ("src_index", C.POINTER(C.c_int64)), ("moment_rate", C.POINTER(C.c_float)),
                ("nsta", C.c_int32), ("sta_xyz", C.POINTER(C.c_int32)),
                ("owner", C.c_void_p), ("terrain", C.POINTER(C.c_float))]


class StageBuffers(C.Structure):
    """cgfdm_stage_buffers: device pointers of one no-allocation stage."""
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("npml", C.c_int32),
                ("dh", C.c_float), ("dt", C.c_float), ("precision", C.c_int32),
                ("irk", C.c_int32), ("fb1", C.c_int32), ("fb2", C.c_int32), ("fb3", C.c_int32),
                ("w_in", C.c_void_p), ("w_out", C.c_void_p), ("w_m", C.c_void_p),
                ("t", C.c_void_p), ("cjm", C.c_void_p), ("rdz", C.c_void_p),
                ("aux_in", C.c_void_p), ("aux_out", C.c_void_p), ("aux_m", C.c_void_p),
                ("aux_t", C.c_void_p)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("chunk_steps", C.c_int32),
                ("device", C.c_int32), ("use_graph", C.c_int32)]


_lib = None

# name -> (restype, argtypes); every entry point returns int unless noted
P, I32, I64, F = C.c_void_p, C.c_int32, C.c_int64, C.c_float
SIGNATURES = {
    "cgfdm_version": (C.c_char_p, []),
    "cgfdm_last_error": (C.c_char_p, []),
    "cgfdm_device_bytes": (C.c_int, [C.POINTER(Desc), C.POINTER(I64)]),
    "cgfdm_create": (C.c_int, [C.POINTER(Desc), C.POINTER(P)]),
    "cgfdm_destroy": (C.c_int, [P]),
    "cgfdm_set_model": (C.c_int, [P, P, P]),
    "cgfdm_set_point_source": (C.c_int, [P, I32, I32, I32, F]),
    "cgfdm_set_fault_source": (C.c_int, [P, P, P, I64, I32, F, I32]),
    "cgfdm_set_stations": (C.c_int, [P, P, I32]),
    "cgfdm_run": (C.c_int, [P, I32, P]),
    "cgfdm_stage": (C.c_int, [P, I32, I32, I32, I32, P]),
    "cgfdm_synchronize": (C.c_int, [P]),
    "cgfdm_steps_done": (C.c_int, [P, C.POINTER(I32)]),
    "cgfdm_get_stations": (C.c_int, [P, P]),
    "cgfdm_get_pgv": (C.c_int, [P, P]),
    "cgfdm_get_wavefield": (C.c_int, [P, P]),
    "cgfdm_get_free_surface": (C.c_int, [P, P]),
    "cgfdm_set_state": (C.c_int, [P, I32, P, P, P, P]),
    "cgfdm_get_state": (C.c_int, [P, P, P, P, P]),
    "cgfdm_aux_floats": (C.c_int, [P, C.POINTER(I64)]),
    "cgfdm_set_timing": (C.c_int, [P, I32]),
    "cgfdm_get_timing": (C.c_int, [P, P]),
    "cgfdm_get_kernel_stats": (C.c_int, [P, P]),
    "cgfdm_set_tile_rows": (C.c_int, [P, I32]),
    "cgfdm_set_chunk": (C.c_int, [P, I32]),
    "cgfdm_get_tuning": (C.c_int, [P, P]),
    "cgfdm_set_graph": (C.c_int, [P, I32]),
    "cgfdm_inject_fault": (C.c_int, [P, I32]),
    "cgfdm_checkpoint_bytes": (C.c_int, [P, C.POINTER(I64)]),
    "cgfdm_checkpoint_save": (C.c_int, [P, P, I64]),
    "cgfdm_checkpoint_load": (C.c_int, [P, P, I64]),
    "cgfdm_batch_create": (C.c_int, [P, I32, C.POINTER(P)]),
    "cgfdm_batch_run": (C.c_int, [P, I32, P]),
    "cgfdm_batch_set_graph": (C.c_int, [P, I32]),
    "cgfdm_batch_synchronize": (C.c_int, [P]),
    "cgfdm_batch_destroy": (C.c_int, [P]),
    "cgfdm_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(P)]),
    "cgfdm_server_submit": (C.c_int, [P, C.POINTER(Desc), P, P, I32, P, F, P, P, I64, I32, F, P,
                                      I32, C.POINTER(I64)]),
    "cgfdm_server_poll": (C.c_int, [P, I64, C.POINTER(I32), C.POINTER(I32)]),
    "cgfdm_server_read_rows": (C.c_int, [P, I64, I32, P, C.POINTER(I32)]),
    "cgfdm_server_wait": (C.c_int, [P, I64, P, P, P]),
    "cgfdm_server_stats": (C.c_int, [P, P]),
    "cgfdm_server_cancel": (C.c_int, [P, I64]),
    "cgfdm_server_destroy": (C.c_int, [P]),
    "cgfdm_propagate": (C.c_int, [C.POINTER(Desc), P, P, I32, P, F, P, P, I64, I32, F, P, I32,
                                  P, P, P]),
    "cgfdm_run_directory": (C.c_int, [C.c_char_p, I32, I32, I32]),
    "cgfdm_setup_from_directory": (C.c_int, [C.c_char_p, C.POINTER(Setup)]),
    "cgfdm_setup_from_directory_ex": (C.c_int, [C.c_char_p, I32, C.POINTER(Setup)]),
    "cgfdm_free_setup": (C.c_int, [C.POINTER(Setup)]),
    "cgfdm_stage_noalloc": (C.c_int, [C.POINTER(StageBuffers), P, I32]),
}


def lib():
    """Loads the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CgfdmError(302, "CUDA extension not built: %s is missing "
                                  "(run make -C cgfdm-fp16_sve_sme_b200)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != OK:
        raise CgfdmError(rc, lib().cgfdm_last_error().decode(errors="replace"))
    return rc
