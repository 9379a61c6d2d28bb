"""ctypes binding of libgear_b200.so (the C ABI declared in include/gear_b200.h)."""
import ctypes
import os

from . import build as _build

_LIB = None
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_dblp = ctypes.POINTER(ctypes.c_double)


class GearError(RuntimeError):
    pass


class LowerArgs(ctypes.Structure):
    """gear_lower_args: one instance of a gear_crown_lower_multi call."""
    _fields_ = [("dag", ctypes.c_void_p), ("x_L", ctypes.c_void_p), ("x_U", ctypes.c_void_p),
                ("batch", ctypes.c_int64), ("C", ctypes.c_void_p), ("lb", ctypes.c_void_p),
                ("lA", ctypes.c_void_p), ("lbias", ctypes.c_void_p), ("lb_ibp", ctypes.c_void_p)]


def lib():
    """Load the in-tree extension; raise if it is missing (there is no CPU fallback)."""
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not os.path.exists(path):
            raise GearError(f"libgear_b200.so not built ({path}); run gear_b200.build.build()")
        L = ctypes.CDLL(path)
        L.gear_dag_create.argtypes = [c_i32p, ctypes.c_int64, c_i32p, ctypes.c_int64, c_i32p, ctypes.c_int64,
                                      c_i32p, ctypes.c_int64, c_i32p, ctypes.c_int64, c_i32p, ctypes.c_int64,
                                      c_dblp, ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
        L.gear_dag_create.restype = ctypes.c_int
        L.gear_dag_destroy.argtypes = [ctypes.c_void_p]
        L.gear_dag_destroy.restype = ctypes.c_int
        L.gear_crown_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        L.gear_crown_workspace_bytes.restype = ctypes.c_int64
        L.gear_crown_lower.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        L.gear_crown_lower.restype = ctypes.c_int
        L.gear_crown_lower_ibp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        L.gear_crown_lower_ibp.restype = ctypes.c_int
        L.gear_last_error.argtypes = []
        L.gear_last_error.restype = ctypes.c_char_p
        L.gear_last_launch_count.argtypes = []
        L.gear_last_launch_count.restype = ctypes.c_int
        vp, i64, i32, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
        L.gear_crown_lower_static.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp]
        L.gear_crown_lower_static.restype = i32
        L.gear_crown_static_scratch_bytes.argtypes = []
        L.gear_crown_static_scratch_bytes.restype = i64
        L.gear_queue_create.argtypes = [i32, i32, i64, i64, vp, vp, ctypes.POINTER(ctypes.c_void_p)]
        L.gear_queue_create.restype = i32
        L.gear_queue_destroy.argtypes = [vp]
        L.gear_queue_destroy.restype = i32
        L.gear_queue_push.argtypes = [vp, vp, vp, vp, i64, vp]
        L.gear_queue_push.restype = i32
        L.gear_queue_pop.argtypes = [vp, vp, vp, vp]
        L.gear_queue_pop.restype = i32
        L.gear_queue_size.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), vp]
        L.gear_queue_size.restype = i32
        L.gear_queue_counters.argtypes = [vp, vp, vp, vp]
        L.gear_queue_counters.restype = i32
        L.gear_queue_reserve.argtypes = [vp, i64, vp]
        L.gear_queue_reserve.restype = i32
        L.gear_queue_capacity.argtypes = [vp]
        L.gear_queue_capacity.restype = i64
        L.gear_bab_step_workspace_bytes.argtypes = [vp, i64]
        L.gear_bab_step_workspace_bytes.restype = i64
        L.gear_bab_step.argtypes = [vp, vp, vp, vp, vp, vp, dbl, dbl, i32, vp, i64, vp]
        L.gear_bab_step.restype = i32
        L.gear_bab_step_bounded.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, dbl, dbl, vp]
        L.gear_bab_step_bounded.restype = i32
        L.gear_crown_multi_prepare.argtypes = [ctypes.POINTER(LowerArgs), i32, vp, i64, ctypes.POINTER(ctypes.c_void_p)]
        L.gear_crown_multi_prepare.restype = i32
        L.gear_crown_multi_launch.argtypes = [vp, vp]
        L.gear_crown_multi_launch.restype = i32
        L.gear_crown_multi_plan_destroy.argtypes = [vp]
        L.gear_crown_multi_plan_destroy.restype = i32
        L.gear_crown_fold_vectors.argtypes = [vp, vp, vp, i64, vp, vp, vp, i64, vp]
        L.gear_crown_fold_vectors.restype = i32
        L.gear_crown_fold_workspace_bytes.argtypes = [vp, i64]
        L.gear_crown_fold_workspace_bytes.restype = i64
        L.gear_bab_workspace_bytes.argtypes = [i64]
        L.gear_bab_workspace_bytes.restype = i64
        L.gear_bab_prune.argtypes = [vp, vp, i64, i32, vp, vp, vp, vp, vp, i64, vp]
        L.gear_bab_prune.restype = i32
        L.gear_bab_branch.argtypes = [vp, vp, vp, vp, vp, i64, i32, i32, vp, dbl, dbl, vp, vp, i64, vp]
        L.gear_bab_branch.restype = i32
        L.gear_bab_split.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, vp, i32, vp, vp, vp, vp]
        L.gear_bab_split.restype = i32
        L.gear_queue_order.argtypes = [vp, vp, vp, i64, vp, i64, vp]
        L.gear_queue_order.restype = i32
        L.gear_queue_merge.argtypes = [vp, vp, vp, i64, vp, i64, vp, vp]
        L.gear_queue_merge.restype = i32
        L.gear_gather_rows.argtypes = [vp, vp, i64, i64, vp, vp]
        L.gear_gather_rows.restype = i32
        L.gear_scatter_rows.argtypes = [vp, vp, i64, i64, vp, vp]
        L.gear_scatter_rows.restype = i32
        L.gear_constrained_workspace_bytes.argtypes = [i64, i32]
        L.gear_constrained_workspace_bytes.restype = i64
        L.gear_constrained_lower.argtypes = [vp, vp, i64, i32, vp, i32, vp, vp, i32, i32, vp, vp, vp, i64, vp]
        L.gear_constrained_lower.restype = i32
        L.gear_clip_domains.argtypes = [vp, vp, vp, vp, vp, vp, i64, i32, i32, i32, vp, vp]
        L.gear_clip_domains.restype = i32
        L.gear_bab_child_keys.argtypes = [vp, vp, vp, vp, vp, vp, i64, i32, i32, vp, vp]
        L.gear_bab_child_keys.restype = i32
        L.gear_bab_compact.argtypes = [vp, i64, vp, vp, vp, i64, vp]
        L.gear_bab_compact.restype = i32
        L.gear_dual_lower_bound.argtypes = [vp, vp, vp, vp, i32, i64, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                            i32, vp, vp, vp, vp]
        L.gear_dual_lower_bound.restype = i32
        L.gear_crown_plain_workspace_bytes.argtypes = [vp, i64]
        L.gear_crown_plain_workspace_bytes.restype = i64
        L.gear_crown_lower_plain.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp, i64, vp]
        L.gear_crown_lower_plain.restype = i32
        L.gear_crown_lower_plain_ibp.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, i64, vp]
        L.gear_crown_lower_plain_ibp.restype = i32
        L.gear_crown_cuts_workspace_bytes.argtypes = [vp, i64, i32]
        L.gear_crown_cuts_workspace_bytes.restype = i64
        L.gear_crown_lower_cuts.argtypes = [vp, vp, vp, i64, vp, vp, vp, i32, i32, vp, vp, vp, vp, vp, i64, vp]
        L.gear_crown_lower_cuts.restype = i32
        L.gear_crown_multi_workspace_bytes.argtypes = [ctypes.POINTER(LowerArgs), i32]
        L.gear_crown_multi_workspace_bytes.restype = i64
        L.gear_crown_lower_multi.argtypes = [ctypes.POINTER(LowerArgs), i32, vp, i64, vp]
        L.gear_crown_lower_multi.restype = i32
        _LIB = L
    return _LIB


def check(status, what):
    if status != 0:
        msg = lib().gear_last_error().decode(errors="replace")
        if status == -2:
            import torch
            raise torch.OutOfMemoryError(f"{what}: {msg}")
        raise GearError(f"{what} failed ({status}): {msg}")


def ptr_i32(a):
    return a.ctypes.data_as(c_i32p)


def ptr_dbl(a):
    return a.ctypes.data_as(c_dblp)


EXPORTED = ("gear_dag_create", "gear_dag_destroy", "gear_crown_workspace_bytes", "gear_crown_lower",
            "gear_last_launch_count", "gear_last_error", "gear_bab_workspace_bytes", "gear_bab_prune",
            "gear_bab_branch", "gear_bab_split", "gear_queue_order", "gear_gather_rows", "gear_scatter_rows",
            "gear_crown_lower_static", "gear_crown_static_scratch_bytes", "gear_constrained_workspace_bytes",
            "gear_constrained_lower", "gear_clip_domains", "gear_bab_child_keys", "gear_bab_compact",
            "gear_dual_lower_bound", "gear_crown_lower_ibp", "gear_crown_multi_workspace_bytes",
            "gear_crown_lower_multi", "gear_crown_plain_workspace_bytes", "gear_crown_lower_plain",
            "gear_queue_merge", "gear_crown_fold_vectors", "gear_crown_fold_workspace_bytes",
            "gear_crown_lower_plain_ibp", "gear_queue_create", "gear_queue_destroy", "gear_queue_push",
            "gear_queue_pop", "gear_queue_size", "gear_queue_counters", "gear_bab_step_workspace_bytes",
            "gear_bab_step", "gear_bab_step_bounded", "gear_crown_multi_prepare", "gear_crown_multi_launch",
            "gear_crown_multi_plan_destroy", "gear_queue_reserve", "gear_queue_capacity",
            "gear_crown_cuts_workspace_bytes", "gear_crown_lower_cuts")
