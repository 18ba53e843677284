"""ctypes binding of ``libcvfes_b200.so`` (declared in ``include/cvfes_b200.h``).

The library is loaded from this package directory only.  There is no fallback:
if the shared object is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcvfes_b200.so")

CVFES_OK = 0
CVFES_ERR_ARG = -1
CVFES_ERR_CUDA = -2
CVFES_ERR_NONFINITE = -3
CVFES_ERR_TIMEOUT = -4
CVFES_ERR_UNSUPPORTED = -5
CVFES_ERR_MESH = -6


class CvfesError(RuntimeError):
    """A libcvfes_b200 entry point returned a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class NonFiniteError(CvfesError):
    """The FP64 watchdog found NaN/Inf in the solid state (CFL violation or bad input)."""


class SolidMeshDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("n_elems", C.c_int64),
        ("n_samples", C.c_int64),
        ("n_clamped", C.c_int64),
        ("clamp_value", C.c_double),
        ("node_ptr", C.c_void_p),
        ("slot_rec", C.c_void_p),
        ("slot_k", C.c_void_p),
        ("fhat", C.c_void_p),
        ("max_degree", C.c_int64),
        ("status", C.c_void_p),
        ("tile_win", C.c_void_p),
        ("tile_rec", C.c_void_p),
        ("node_loc", C.c_void_p),
        ("tile_p", C.c_int32),
        ("tile_h", C.c_int32),
        ("tile_w", C.c_int32),
        ("tile_eh", C.c_int32),
        ("tile_we", C.c_int32),
        ("tile_pad", C.c_int32),
        ("bandwidth", C.c_int64),
        ("state_form", C.c_int32),
        ("damping_form", C.c_int32),
    ]


class BatchItem(C.Structure):
    _fields_ = [
        ("mesh", SolidMeshDesc),
        ("coef", C.c_void_p),
        ("invm", C.c_void_p),
        ("buf", C.c_void_p * 3),
        ("p_sched", C.c_void_p),
        ("dt", C.c_double),
        ("damp", C.c_double),
    ]


class AdjointDesc(C.Structure):
    _fields_ = [
        ("mesh", SolidMeshDesc),
        ("precision", C.c_int32),
        ("record", C.c_int32),
        ("coef", C.c_void_p),
        ("invm", C.c_void_p),
        ("owner_blocks", C.c_void_p),
        ("state", C.c_void_p * 3),
        ("adj", C.c_void_p * 2),
        ("ckpt", C.c_void_p),
        ("p_sched", C.c_void_p),
        ("clock", C.c_void_p),
        ("n_steps", C.c_int64),
        ("ckpt_every", C.c_int64),
        ("n_obs", C.c_int32),
        ("obs_every", C.c_int32),
        ("obs_nodes", C.c_void_p),
        ("obs", C.c_void_p),
        ("jpart", C.c_void_p),
        ("J", C.c_void_p),
        ("gamma", C.c_void_p),
        ("gmass", C.c_void_p),
        ("dt", C.c_double),
        ("damp", C.c_double),
    ]


P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32
D = C.c_double
DESC = C.POINTER(SolidMeshDesc)

# name -> (restype, argtypes)
SIGNATURES = {
    "cvfes_last_error": (C.c_char_p, []),
    "cvfes_version": (C.c_int, []),
    "cvfes_mesh_incidence": (C.c_int, [I64, I64, P, P, P, P]),
    "cvfes_mesh_color_greedy": (C.c_int, [I64, I64, P, I32, P]),
    "cvfes_gmrf_selected_inverse_diag": (C.c_int, [I64, P, P, P, P, P]),
    "cvfes_gmrf_solve_lt": (C.c_int, [I64, P, P, P, I64, P]),
    "cvfes_solid_templates_f64": (C.c_int, [I64, I64, P, P, P, P, P, P, P, P, P, P, P]),
    "cvfes_solid_mass_load_f64": (C.c_int, [I64, I64, I64, P, P, P, P, P, I32, P, P, P, P, P, P, P]),
    "cvfes_solid_assemble_bsr_f64": (C.c_int, [I64, I64, P, P, P, I32, P, P, P, P]),
    "cvfes_bsr_spmv_f64": (C.c_int, [I64, I64, P, P, P, P, P, P]),
    "cvfes_solid_kmul_f64": (C.c_int, [DESC, P, P, P, I32, P]),
    "cvfes_solid_kmul_f32": (C.c_int, [DESC, P, P, P, I32, P]),
    "cvfes_solid_step_f64": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, P, D, D, P]),
    "cvfes_solid_step_f32": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, P, D, D, P]),
    "cvfes_solid_step_norms_f64": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, P, D, D, P, P,
                                             P, I32, P]),
    "cvfes_solid_step_norms_f32": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, P, D, D, P, P,
                                             P, I32, P]),
    "cvfes_solid_advance_f64": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, D, P, P, P]),
    "cvfes_solid_advance_f32": (C.c_int, [DESC, P, P, P, P, P, P, P, I64, D, D, P, P, P]),
    "cvfes_solid_init_f64": (C.c_int, [DESC, P, P, P, P, P, P, D, D, D, P]),
    "cvfes_solid_init_f32": (C.c_int, [DESC, P, P, P, P, P, P, D, D, D, P]),
    "cvfes_norms_work_size": (C.c_int64, [I64, I64]),
    "cvfes_solid_norms_f64": (C.c_int, [I64, I64, P, P, P, P, P, I32, P]),
    "cvfes_solid_norms_f32": (C.c_int, [I64, I64, P, P, P, P, P, I32, P]),
    "cvfes_solid_norms_noalloc_f32": (C.c_int, [I64, I64, P, P, P, P, I32, P]),
    "cvfes_solid_norms_vel_f64": (C.c_int, [I64, I64, P, P, P, P, P, I32, P]),
    "cvfes_solid_norms_vel_f32": (C.c_int, [I64, I64, P, P, P, P, P, I32, P]),
    "cvfes_graph_capture_advance": (C.c_int, [DESC, I32, P, P, P, P, P, P, P, I64, D, D, P,
                                              C.POINTER(C.c_void_p)]),
    "cvfes_graph_launch": (C.c_int, [P, P]),
    "cvfes_graph_destroy": (C.c_int, [P]),
    "cvfes_set_step_tuning": (C.c_int, [I32, I32, I32, I32, I32]),
    "cvfes_get_step_tuning": (C.c_int, [I32, P, P, P, P]),
    "cvfes_set_step_prefetch": (C.c_int, [I32, I32, I32]),
    "cvfes_get_step_prefetch": (C.c_int, [I32, P, P]),
    "cvfes_status_read": (C.c_int, [P, P]),
    "cvfes_set_wait_probe": (C.c_int, [I32]),
    "cvfes_set_norms_memory": (C.c_int, [I32]),
    "cvfes_batch_table_bytes": (C.c_int64, [I32]),
    "cvfes_batch_pack": (C.c_int, [C.POINTER(BatchItem), I32, I32, I32, P, P]),
    "cvfes_batch_step": (C.c_int, [P, I32, P, I32, I32, I32, I32, P, I64, I32, P]),
    "cvfes_batch_advance": (C.c_int, [P, I32, P, I32, I32, I32, I32, P, I64, I32,
                                      C.POINTER(C.c_int32), P]),
    "cvfes_batch_graph_capture": (C.c_int, [P, I32, P, I32, I32, I32, P, I64, I32,
                                            C.POINTER(C.c_void_p)]),
    "cvfes_mesh_tiles": (C.c_int, [I64, I64, P, P, I64, I32, I32, I32, I32, I32, P, P, P, P]),
    "cvfes_set_geo_tuning": (C.c_int, [I32, I32, I32]),
    "cvfes_get_geo_tuning": (C.c_int, [I32, P, P]),
    "cvfes_solid_slot_geometry_f64": (C.c_int, [I64, P, P, P, P, P, P]),
    "cvfes_solid_step_geo_f64": (C.c_int, [DESC, P, P, P, P, P, P, P, P, P, I64, D, P, D, D, D,
                                           P]),
    "cvfes_solid_step_geo_f32": (C.c_int, [DESC, P, P, P, P, P, P, P, P, P, I64, D, P, D, D, D,
                                           P]),
    "cvfes_solid_advance_geo_f64": (C.c_int, [DESC, P, P, P, P, P, P, P, P, P, I64, I64, P, I32,
                                              D, D, D, P, P, P, P]),
    "cvfes_solid_advance_geo_f32": (C.c_int, [DESC, P, P, P, P, P, P, P, P, P, I64, I64, P, I32,
                                              D, D, D, P, P, P, P]),
    "cvfes_solid_stress_f64": (C.c_int, [I64, I64, P, P, P, P, P, D, P, P]),
    "cvfes_solid_stress_f32": (C.c_int, [I64, I64, P, P, P, P, P, D, P, P]),
    "cvfes_set_adjoint_tuning": (C.c_int, [I32, I32, I32, I32, I32]),
    "cvfes_get_adjoint_tuning": (C.c_int, [I32, P, P, P, P]),
    "cvfes_adjoint_ckpt_count": (C.c_int64, [I64, I64]),
    "cvfes_adjoint_jpart_size": (C.c_int64, [I64, I32, I32, I64]),
    "cvfes_adjoint_owner_blocks": (C.c_int, [DESC, I32, P, P, P, P]),
    "cvfes_adjoint_material": (C.c_int, [I64, I64, P, P, P, P, P, P]),
    "cvfes_adjoint_forward": (C.c_int, [C.POINTER(AdjointDesc), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32), P]),
    "cvfes_adjoint_reverse": (C.c_int, [C.POINTER(AdjointDesc), I32, I32, P]),
    "cvfes_adjoint_gradients": (C.c_int, [C.POINTER(AdjointDesc), P, P, P, P, P, P, P, P, P]),
    "cvfes_adjoint_capture": (C.c_int, [C.POINTER(AdjointDesc), I32, I32, I32,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_void_p)]),
}


def get_step_tuning(precision: int) -> dict:
    vals = [C.c_int32() for _ in range(4)]
    call("cvfes_get_step_tuning", precision, *[C.byref(v) for v in vals])
    return dict(zip(("vec", "npb", "staged", "minb"), (v.value for v in vals)))


def set_step_tuning(precision: int, vec: int, npb: int, staged: int, minb: int) -> None:
    call("cvfes_set_step_tuning", precision, vec, npb, staged, minb)


def get_step_prefetch(precision: int) -> dict:
    d, p = C.c_int32(), C.c_int32()
    call("cvfes_get_step_prefetch", precision, C.byref(d), C.byref(p))
    return dict(distance=d.value, parts=p.value)


def set_step_prefetch(precision: int, distance: int = -1, parts: int = -1) -> None:
    call("cvfes_set_step_prefetch", precision, distance, parts)


def get_adjoint_tuning(precision: int) -> dict:
    vals = [C.c_int32() for _ in range(4)]
    call("cvfes_get_adjoint_tuning", precision, *[C.byref(v) for v in vals])
    return dict(zip(("vec", "npb", "variant", "minb"), (v.value for v in vals)))


def set_adjoint_tuning(precision: int, vec: int, npb: int, variant: int, minb: int) -> None:
    call("cvfes_set_adjoint_tuning", precision, vec, npb, variant, minb)

_lock = threading.Lock()
_lib = None


def load():
    """Load the shared library (once) and declare every signature."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise CvfesError(CVFES_ERR_UNSUPPORTED,
                             f"{LIB_PATH} is not built; run `python -m cvfes_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().cvfes_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> int:
    """Raise on a negative status, return it otherwise."""
    if rc < 0:
        cls = NonFiniteError if rc == CVFES_ERR_NONFINITE else CvfesError
        raise cls(rc, f"{what}: {last_error()}" if what else last_error())
    return rc


def call(name: str, *args) -> int:
    return check(getattr(load(), name)(*args), name)


def ptr(t) -> int | None:
    """Raw address of a torch tensor / numpy array (None stays None)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
