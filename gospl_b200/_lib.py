"""ctypes binding of libgospl_b200.so (the C ABI in include/gospl_b200.h).

The library is built in-tree (gospl_b200/build.py); importing this module never
falls back to anything else: if the shared object is missing or a CUDA device
is absent, calls fail loudly.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libgospl_b200.so")

GS_OK = 0
# slots of gs_sed_budget's output (GS_LED_* in the header)
LED_SLOTS = ("eroded", "pit_sinks", "kept", "dropped", "outlets", "sea", "retained", "excess", "zero_excess",
             "inflow", "placed", "routed", "realised", "kept_deposit")
ERRORS = {1: "GS_EINVAL", 2: "GS_ECUDA", 3: "GS_EMAXITER", 4: "GS_ENONFINITE", 5: "GS_ECYCLE",
          6: "GS_ETIMEOUT", 7: "GS_ENOMEM"}

EXPORTS = ("gs_version", "gs_last_error", "gs_plan_create", "gs_plan_destroy", "gs_plan_set_members",
           "gs_plan_tune", "gs_plan_tuning", "gs_plan_set_precision", "gs_plan_set_deposition",
           "gs_plan_set_stream",
           "gs_plan_launches", "gs_mfdreceivers", "gs_fill_elevation", "gs_build_flow_direction", "gs_pit_tables",
           "gs_flow_accumulation", "gs_erodep_spl", "gs_sed_change", "gs_sed_budget", "gs_sea_change", "gs_plan_set_lake_diffusion", "gs_hillslope", "gs_apply_forces", "gs_output_fields", "gs_mesh_geometry", "gs_plan_profile",
           "gs_plan_profile_report", "gs_plan_profile_trace", "gs_plan_record", "gs_plan_record_slot",
           "gs_adjoint_step", "gs_flow_solve_noalloc")


class GsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


class GsStats(ctypes.Structure):
    _fields_ = [("npits", ctypes.c_int32), ("cascade_passes", ctypes.c_int32),
                ("cascade_solves", ctypes.c_int32), ("fill_rounds", ctypes.c_int32),
                ("flat_rounds", ctypes.c_int32), ("cycle_nodes", ctypes.c_int32),
                ("cg_iters", ctypes.c_int32), ("status", ctypes.c_int32), ("cg_relres", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path=None):
    """Load (once) and type the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIBPATH
    if not os.path.exists(path):
        raise ImportError("libgospl_b200.so not built (run gospl_b200/build.py): %s" % path)
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    i32 = ctypes.c_int32
    i64 = ctypes.c_int64
    d = ctypes.c_double
    L.gs_version.restype = ctypes.c_int
    L.gs_last_error.argtypes = [ctypes.c_char_p, i64]
    L.gs_plan_create.argtypes = [i64, P, P, P, P, P, P, P, i64, P, i64, i32, i32, ctypes.POINTER(P)]
    L.gs_plan_destroy.argtypes = [P]
    L.gs_plan_set_members.argtypes = [P, i32, P, P]
    L.gs_plan_tune.argtypes = [P, i32, i32]
    L.gs_plan_tuning.argtypes = [P, i32]
    L.gs_plan_set_precision.argtypes = [P, i32, d]
    L.gs_plan_set_deposition.argtypes = [P, d]
    L.gs_plan_set_stream.argtypes = [P, P]
    L.gs_plan_launches.argtypes = [P]
    L.gs_plan_launches.restype = i64
    L.gs_mfdreceivers.argtypes = [P, i32, d, P, d, P, P, P, P]
    L.gs_fill_elevation.argtypes = [P, P, d, d, i32, P, P, P, P]
    L.gs_build_flow_direction.argtypes = [P, P, i32, d, P, P, P, P, P, P, P, P]
    L.gs_pit_tables.argtypes = [P, P, P, P, P]
    L.gs_flow_accumulation.argtypes = [P, P, P, d, d, d, P, P, P, P, P, P, P, P, P, P, P,
                                       ctypes.POINTER(GsStats)]
    L.gs_erodep_spl.argtypes = [P, P, P, P, P, P, d, P, d, d, d, P, P, P, P, P, ctypes.POINTER(GsStats)]
    L.gs_plan_set_lake_diffusion.argtypes = [P, d, d, i32, i32]
    L.gs_sed_change.argtypes = [P, P, P, P, P, d, d, d, d, d, P, P, P, P, P, P, P, P, ctypes.POINTER(GsStats)]
    L.gs_sed_budget.argtypes = [P, P]
    L.gs_sea_change.argtypes = [P, P, P, P, P, P, P, i64, d, d, d, d, d, d, d, P, P, P, ctypes.POINTER(GsStats)]
    L.gs_hillslope.argtypes = [P, P, P, P, d, d, d, d, d, i32, ctypes.POINTER(GsStats)]
    L.gs_apply_forces.argtypes = [P, P, P, P, d, d, P]
    L.gs_output_fields.argtypes = [P, P, P, P, P, P, P, P, P, P, P, P]
    L.gs_plan_profile.argtypes = [P, i32]
    L.gs_flow_solve_noalloc.argtypes = [i64, i32, P, P, P, P, P]
    L.gs_plan_profile_report.argtypes = [P, ctypes.c_char_p, i64]
    L.gs_plan_profile_trace.argtypes = [P, ctypes.c_char_p, i64]
    L.gs_plan_record.argtypes = [P, i32]
    L.gs_plan_record_slot.argtypes = [P, i32]
    L.gs_adjoint_step.argtypes = [P, i32, P, P, d, P, d, d, d, d, d, d, d, i32, P, P, P, P]
    L.gs_mesh_geometry.argtypes = [i64, P, i64, P, P, P, i64, P, P, P, P, i32, P, P, P, P, P, P, P]
    for name in EXPORTS:
        if name not in ("gs_version", "gs_plan_launches"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(code):
    if code != GS_OK:
        buf = ctypes.create_string_buffer(512)
        load().gs_last_error(buf, 512)
        raise GsError(code, buf.value.decode(errors="replace"))


def ptr(t):
    """Raw device/host address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return t.ctypes.data_as(ctypes.c_void_p)
