"""ctypes binding of libpfsht_b200.so (include/pfsht_b200.h).

The shared library is built in-tree (``make -C partialfsht.jl_b200/csrc``). There is no
fallback: if the library is missing or fails to load, importing the package raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpfsht_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "pfsht_b200.h")

OK, ERR_ARGUMENT, ERR_DIMENSION, ERR_REFUSED, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_UNSUPPORTED = range(8)
METHODS = {"auto": 0, "stretch": 1, "direct": 2, "multibox": 3}
PRECISIONS = {"fp64": 0, "mixed": 1}
KINDS = {0: "pole", 1: "interior", 2: "full", 3: "direct", 4: "multibox"}


class Opts(C.Structure):
    _fields_ = [("method", C.c_int32), ("points_on_device", C.c_int32), ("device", C.c_int32),
                ("ring_rings_per_lane", C.c_int32), ("nufft_bin_rows", C.c_int32),
                ("nufft_bin_cols", C.c_int32), ("oversample_theta", C.c_double),
                ("oversample_phi", C.c_double), ("eps_apo_max", C.c_double),
                ("ring_segment_degrees", C.c_int32), ("nufft_fft_lengths", C.c_int32),
                ("nufft_nf1", C.c_int32), ("nufft_nf2", C.c_int32), ("maxboxes", C.c_int32),
                ("spin", C.c_int32), ("nufft_transpose", C.c_int32), ("deterministic", C.c_int32),
                ("nufft_spread", C.c_int32)]


class Box(C.Structure):
    """pfsht_box: SphereBox (src/Box.jl:23-30)."""
    _fields_ = [("theta_lo", C.c_double), ("theta_hi", C.c_double), ("phi_start", C.c_double),
                ("phi_extent", C.c_double), ("touches_north", C.c_int32),
                ("touches_south", C.c_int32)]


class PlanInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("flip", C.c_int32), ("lmax", C.c_int32),
                ("ntrans", C.c_int32), ("precision", C.c_int32), ("nth_half", C.c_int32),
                ("nth", C.c_int32), ("nph", C.c_int32), ("mmax", C.c_int32),
                ("nrings", C.c_int32), ("npts", C.c_int64), ("K", C.c_int64),
                ("ring_work", C.c_int64), ("tol", C.c_double), ("beta", C.c_double),
                ("h", C.c_double), ("theta_lo", C.c_double), ("theta_hi", C.c_double),
                ("eps_apo", C.c_double), ("Theta1", C.c_double), ("sigma", C.c_double),
                ("ThetaT", C.c_double), ("nufft_w", C.c_int32), ("nf1", C.c_int32),
                ("nf2", C.c_int32), ("row0", C.c_int32), ("nrows", C.c_int32),
                ("ncols", C.c_int32), ("nufft_beta", C.c_double), ("device_bytes", C.c_int64),
                ("spin", C.c_int32), ("pad_", C.c_int32)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
SIGNATURES = {
    "pfsht_opts_default": (C.c_int, [C.POINTER(Opts)]),
    "pfsht_plan_create": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                    C.c_int32, C.POINTER(Opts), C.POINTER(_vp)]),
    "pfsht_plan_destroy": (C.c_int, [_vp]),
    "pfsht_forward": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_adjoint": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_forward_host": (C.c_int, [_vp, _vp, _vp]),
    "pfsht_adjoint_host": (C.c_int, [_vp, _vp, _vp]),
    "pfsht_forward_host_async": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_adjoint_host_async": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_host_sync": (C.c_int, [_vp]),
    "pfsht_wait_timeouts": (C.c_int, [C.POINTER(C.c_int32)]),
    "pfsht_ring_forward": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_ring_adjoint": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_ring_work": (C.c_int64, [_vp]),
    "pfsht_host_bytes": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "pfsht_plan_get_info": (C.c_int, [_vp, C.POINTER(PlanInfo)]),
    "pfsht_workspace_bytes": (C.c_int64, [_vp]),
    "pfsht_plan_geometry": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                      C.POINTER(Opts), C.POINTER(PlanInfo)]),
    "pfsht_dfs_double": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "pfsht_dfs_fold": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "pfsht_nufft_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                     C.c_double, _vp, _vp, C.c_int64, C.POINTER(_vp)]),
    "pfsht_nufft_exec": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pfsht_nufft_destroy": (C.c_int, [_vp]),
    "pfsht_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "pfsht_version": (C.c_char_p, []),
    "pfsht_fma_peak": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "pfsht_launch_count": (C.c_int64, []),
    "pfsht_direct_forward_noalloc": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, _vp, _vp, _vp]),
    "pfsht_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "pfsht_batch_forward": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    "pfsht_batch_adjoint": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    "pfsht_batch_info": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "pfsht_batch_destroy": (C.c_int, [_vp]),
    "pfsht_server_create": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, C.POINTER(_vp)]),
    "pfsht_server_add_plan": (C.c_int, [_vp, _vp, C.POINTER(C.c_int32)]),
    "pfsht_server_submit": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, C.POINTER(C.c_int64)]),
    "pfsht_server_wait": (C.c_int, [_vp, C.c_int64, C.c_double, C.POINTER(C.c_double)]),
    "pfsht_server_request_times": (C.c_int, [_vp, C.c_int64, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "pfsht_server_release": (C.c_int, [_vp, C.c_int64]),
    "pfsht_server_stats": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "pfsht_server_destroy": (C.c_int, [_vp]),
    "pfsht_bounding_box": (C.c_int, [_vp, _vp, C.c_int64, C.POINTER(Box)]),
    "pfsht_cost_direct": (C.c_double, [C.c_int64, C.c_int32, C.c_int32]),
    "pfsht_cost_stretch": (C.c_double, [C.POINTER(Box), C.c_int64, C.c_int32, C.c_int32, C.c_double]),
    "pfsht_partition_boxes": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                        C.c_int32, _vp, C.POINTER(C.c_int32), C.POINTER(Box), _dp]),
    "pfsht_select_method": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                      C.POINTER(C.c_int32)]),
    "pfsht_bounding_box_device": (C.c_int, [_vp, _vp, C.c_int64, C.POINTER(Box), _vp]),
    "pfsht_partition_boxes_device": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                               C.c_int32, _vp, C.POINTER(C.c_int32), C.POINTER(Box),
                                               _dp, _vp]),
    "pfsht_select_method_device": (C.c_int, [_vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                             C.POINTER(C.c_int32), _vp]),
    "pfsht_solve": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_double, C.c_int32, _vp, _vp, _vp,
                              C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "pfsht_set_cost_constants": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double]),
    "pfsht_get_cost_constants": (C.c_int, [_dp, _dp, _dp, _dp, C.POINTER(C.c_int32)]),
    "pfsht_plan_num_boxes": (C.c_int32, [_vp]),
    "pfsht_plan_box": (C.c_int, [_vp, C.c_int32, C.POINTER(PlanInfo), _vp]),
    "pfsht_profile_start": (C.c_int, [_vp, C.c_int32]),
    "pfsht_profile_stop": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "pfsht_num_stages": (C.c_int32, []),
    "pfsht_stage_name": (C.c_char_p, [C.c_int32]),
}

_lib = None


def load():
    """Load libpfsht_b200.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C partialfsht.jl_b200/csrc` "
            "(or __graft_entry__.build()). There is no CPU fallback.")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class PFSHTError(RuntimeError):
    pass


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch (src/Layout.jl:35-56)."""


class RefusedGeometry(ValueError):
    """The stretched construction is degenerate here (src/Windows.jl:66-75)."""


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().pfsht_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, what: str = ""):
    if status == OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if status == ERR_ARGUMENT:
        raise ValueError(msg)
    if status == ERR_DIMENSION:
        raise DimensionMismatch(msg)
    if status == ERR_REFUSED:
        raise RefusedGeometry(msg)
    if status == ERR_OOM:
        raise MemoryError(msg)
    if status == ERR_TIMEOUT:
        raise TimeoutError(msg)
    if status == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise PFSHTError(msg)


def default_opts() -> Opts:
    o = Opts()
    check(load().pfsht_opts_default(C.byref(o)))
    return o
