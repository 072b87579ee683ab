"""ctypes bindings of the in-tree library liboctlb_b200.so.

Everything here is a thin marshalling layer over the C ABI declared in
include/octlb_gpu.h and include/octlb_forest.h.  The library is loaded from
the package directory; a missing library is an ImportError, never a silent
fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboctlb_b200.so")

OCTLB_OK = 0
OCTLB_EINVAL = -1
OCTLB_ENOMEM = -2
OCTLB_ECUDA = -3
OCTLB_ENAN = -4
OCTLB_ETIMEOUT = -5
OCTLB_ESTATE = -6

FP32 = 0
FP16_SHIFTED = 1
STREAM_ROTATE = 0
STREAM_LINKS = 1
COUPLER_REFERENCE = 0
COUPLER_PHYSICAL = 1
ORDER_AB = 0
ORDER_AA = 1
TB_NONE = 0
TB_WALL = 1
TB_OUTFLOW = 2

# BcKind (src/solver/lbm/bc_kind.h:14-23)
BULK, SOLID, BOUNCE_BACK, MOVING_BOUNCE_BACK, BOUZIDI, VELOCITY_DIRICHLET, PRESSURE_DIRICHLET, OUTFLOW = range(8)

P = ctypes.c_void_p
I32P = ctypes.POINTER(ctypes.c_int)
F64P = ctypes.POINTER(ctypes.c_double)
U8P = ctypes.POINTER(ctypes.c_uint8)


class Tables(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("n_blocks", ctypes.c_int),
        ("levels", I32P), ("bounds", F64P), ("kinds", U8P),
        ("n_same_level", ctypes.c_int), ("same_level", I32P),
        ("n_coarse_fine", ctypes.c_int), ("coarse_fine", I32P), ("coarse_fine_bounds", F64P),
        ("n_tree_boundary", ctypes.c_int), ("tree_boundary", I32P), ("tree_boundary_spec", F64P),
        ("n_links", ctypes.c_int), ("link_cells", I32P), ("link_q", F64P),
        ("moving", U8P), ("wall_u", F64P), ("obstacle", U8P),
        ("periodic", ctypes.c_int),
    ]


class AdjParams(ctypes.Structure):
    """octlb_adj_params."""
    _fields_ = [("coarse_steps", ctypes.c_int), ("window", ctypes.c_int),
                ("checkpoint_interval", ctypes.c_int), ("component", ctypes.c_int)]


VTK_VELOCITY, VTK_DENSITY, VTK_PRESSURE = 1, 2, 4

INLET_NONE, INLET_UNIFORM, INLET_POISEUILLE, INLET_CHANNEL_POISEUILLE = 0, 1, 2, 3


class FdInlet(ctypes.Structure):
    """octlb_fd_inlet: one face's inlet velocity field."""
    _fields_ = [("kind", ctypes.c_int), ("n_inplane", ctypes.c_int * 2), ("u", ctypes.c_double * 3),
                ("u_peak", ctypes.c_double), ("patch", ctypes.c_double * 4), ("ramp_end_t", ctypes.c_double)]


class Partition(ctypes.Structure):
    """octlb_partition."""
    _fields_ = [("rank", ctypes.c_int), ("nranks", ctypes.c_int), ("owner", ctypes.POINTER(ctypes.c_int)),
                ("comm", ctypes.c_void_p)]


class Params(ctypes.Structure):
    _fields_ = [
        ("omega", ctypes.c_double), ("precision", ctypes.c_int), ("stream_mode", ctypes.c_int),
        ("drag", ctypes.c_int), ("fp16_scale", ctypes.c_double * 32),
        ("coupler_mode", ctypes.c_int), ("omega_level", ctypes.c_double * 32),
        ("stream_order", ctypes.c_int),
    ]


_lib = None


def lib():
    """The loaded library; raises ImportError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"octlb_b200: {LIB_PATH} is missing; run octlb_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "octlb_gpu_create": (ctypes.c_int, [ctypes.POINTER(Tables), ctypes.POINTER(Params), F64P, ctypes.POINTER(P)]),
        "octlb_gpu_create_part": (ctypes.c_int, [ctypes.POINTER(Tables), ctypes.POINTER(Params), F64P,
                                                 ctypes.POINTER(Partition), ctypes.POINTER(P)]),
        "octlb_gpu_partition": (ctypes.c_int, [ctypes.POINTER(Tables), ctypes.c_int, I32P]),
        "octlb_gpu_plan_part": (ctypes.c_int, [ctypes.POINTER(Tables), ctypes.POINTER(Params), ctypes.c_int,
                                               ctypes.c_int, I32P, ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.c_longlong]),
        "octlb_comm_create_local": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(P)]),
        "octlb_comm_nccl_unique_id": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ubyte)]),
        "octlb_comm_create_nccl": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(P)]),
        "octlb_comm_destroy": (None, [P]),
        "octlb_comm_last_error": (ctypes.c_char_p, []),
        "octlb_gpu_destroy": (None, [P]),
        "octlb_gpu_last_error": (ctypes.c_char_p, [P]),
        "octlb_gpu_set_stream": (ctypes.c_int, [P, P]),
        "octlb_gpu_advance": (ctypes.c_int, [P, ctypes.c_int]),
        "octlb_gpu_synchronize": (ctypes.c_int, [P]),
        "octlb_gpu_set_populations": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_set_equilibrium": (ctypes.c_int, [P, F64P, F64P]),
        "octlb_gpu_set_body_force": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_set_const_rho": (ctypes.c_int, [P, ctypes.c_int]),
        "octlb_gpu_set_fd_boundary": (ctypes.c_int, [P, I32P, F64P, F64P, F64P, ctypes.c_double]),
        "octlb_fd_stamp_kinds": (ctypes.c_int, [ctypes.POINTER(Tables), I32P, U8P]),
        "octlb_fd_plan": (ctypes.c_int, [ctypes.POINTER(Tables), I32P, F64P, F64P, F64P, ctypes.c_double, P,
                                         ctypes.c_int]),
        "octlb_fd_record_bytes": (ctypes.c_int, []),
        "octlb_gpu_set_fd_boundary_inlets": (ctypes.c_int, [P, I32P, F64P, F64P, ctypes.POINTER(FdInlet)]),
        "octlb_fd_plan_inlets": (ctypes.c_int, [ctypes.POINTER(Tables), I32P, F64P, F64P, ctypes.POINTER(FdInlet),
                                                P, ctypes.c_int]),
        "octlb_gpu_write_vtk": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int]),
        "octlb_vtk_write_block": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, F64P,
                                                 ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), I32P,
                                                 ctypes.POINTER(F64P)]),
        "octlb_vtk_write_index": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_char_p)]),
        "octlb_gpu_average_rho": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_adjoint": (ctypes.c_int, [P, ctypes.POINTER(AdjParams), F64P, F64P, F64P]),
        "octlb_gpu_get_populations": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_get_fields": (ctypes.c_int, [P, F64P, F64P]),
        "octlb_gpu_force": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_force_sum": (ctypes.c_int, [P, F64P, ctypes.POINTER(ctypes.c_longlong)]),
        "octlb_gpu_force_reset": (ctypes.c_int, [P]),
        "octlb_gpu_audit": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_audit_noalloc": (ctypes.c_int, [P, F64P]),
        "octlb_gpu_counters": (ctypes.c_int, [P, I32P, I32P, ctypes.c_int]),
        "octlb_gpu_max_level": (ctypes.c_int, [P]),
        "octlb_gpu_step_stats": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "octlb_gpu_debug_fastdiv": (ctypes.c_uint, [ctypes.c_uint, ctypes.c_uint]),
        "octlb_gpu_plan": (ctypes.c_int, [ctypes.POINTER(Tables), ctypes.POINTER(Params),
                                           ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
        "octlb_forest_new": (P, [ctypes.c_int] * 6 + [F64P]),
        "octlb_forest_free": (None, [P]),
        "octlb_forest_refine_uniform": (ctypes.c_int, [P, ctypes.c_int]),
        "octlb_forest_refine_box": (ctypes.c_int, [P, F64P, ctypes.c_int]),
        "octlb_forest_balance": (ctypes.c_int, [P]),
        "octlb_forest_build": (ctypes.c_int, [P]),
        "octlb_forest_num_leaves": (ctypes.c_int, [P]),
        "octlb_forest_leaves": (ctypes.c_int, [P, I32P, F64P]),
        "octlb_forest_num_same_level": (ctypes.c_int, [P]),
        "octlb_forest_same_level": (ctypes.c_int, [P, I32P]),
        "octlb_forest_num_coarse_fine": (ctypes.c_int, [P]),
        "octlb_forest_coarse_fine": (ctypes.c_int, [P, I32P, F64P]),
        "octlb_forest_num_tree_boundary": (ctypes.c_int, [P]),
        "octlb_forest_tree_boundary": (ctypes.c_int, [P, I32P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class OctlbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"octlb error {code}: {msg}")
        self.code = code
