"""ctypes binding of libflsp_dg.so.

The library is the product: there is no CPU fallback.  Importing this
module does not need a GPU, but ``load()`` raises if the shared library
is missing, and every call that reaches the device raises ``FlspError``
when the library reports a failure (for example FLSP_ERR_NO_DEVICE).
"""
import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflsp_dg.so")

_lib = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p

# every symbol include/flsp_dg.h declares, with its ctypes signature
PROTOTYPES = {
    "flsp_create": (C.c_int, [C.POINTER(abi.MeshDesc), C.POINTER(abi.DGOpts), C.POINTER(_vp)]),
    "flsp_destroy": (None, [_vp]),
    "flsp_last_error": (C.c_char_p, []),
    "flsp_version": (C.c_int, []),
    "flsp_n_dofs": (C.c_int, [_vp, _i64p]),
    "flsp_dofs_per_cell": (C.c_int, [_vp, _ip]),
    "flsp_set_velocity": (C.c_int, [_vp, C.POINTER(abi.VelocityDesc)]),
    "flsp_set_velocity_fe": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double), C.c_int64]),
    "flsp_project_ic": (C.c_int, [_vp, C.POINTER(abi.ICDesc)]),
    "flsp_set_state": (C.c_int, [_vp, _dp, C.c_int64]),
    "flsp_get_state": (C.c_int, [_vp, _dp, C.c_int64]),
    "flsp_set_time": (C.c_int, [_vp, C.c_double]),
    "flsp_get_time": (C.c_int, [_vp, _dp]),
    "flsp_get_step_count": (C.c_int, [_vp, _i64p]),
    "flsp_snapshot": (C.c_int, [_vp]),
    "flsp_set_dirichlet": (C.c_int, [_vp, C.c_int, C.c_double]),
    "flsp_clear_dirichlet": (C.c_int, [_vp]),
    "flsp_advect_rhs": (C.c_int, [_vp, C.c_double, _dp, C.c_int64]),
    "flsp_advance": (C.c_int, [_vp, C.c_double, C.c_int, _dp]),
    "flsp_advance_steps": (C.c_int, [_vp, C.c_int, C.c_double]),
    "flsp_reinit": (C.c_int, [_vp, C.POINTER(abi.ReinitOpts), _ip]),
    "flsp_hj_gradients": (C.c_int, [_vp, _dp, C.c_int64]),
    "flsp_weno_limit": (C.c_int, [_vp, _ip]),
    "flsp_ls_advance": (C.c_int, [_vp, C.POINTER(abi.LSOpts), C.c_double, C.c_int, _dp]),
    "flsp_ls_run_steps": (C.c_int, [_vp, C.POINTER(abi.LSOpts), C.c_int]),
    "flsp_sync": (C.c_int, [_vp]),
    "flsp_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "flsp_time_kernel": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "flsp_reduce": (C.c_int, [_vp, C.c_int, C.POINTER(abi.ICDesc), _dp]),
    "flsp_autotune": (C.c_int, [_vp, C.c_int, _ip, _ip, _dp, _ip]),
    "flsp_stage_tile": (C.c_int, [_vp, _ip]),
    "flsp_curvature": (C.c_int, [_vp, C.c_int, _dp, C.c_int64]),
    "flsp_material_mix": (C.c_int, [C.POINTER(_vp), C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int64]),
    "flsp_eval_patches": (C.c_int, [_vp, C.c_int, _dp, C.c_int64]),
    "flsp_export_solutions": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "flsp_write_vtu": (C.c_int, [C.POINTER(abi.MeshDesc), C.c_int, _dp, C.c_char_p, C.c_char_p]),
    "flsp_write_pvd": (C.c_int, [C.c_char_p, C.c_int, _dp, C.POINTER(C.c_char_p)]),
    "flsp_reduce_noalloc": (C.c_int, [C.POINTER(abi.MeshDesc), C.c_int, C.c_int, C.c_int, _vp, _vp,
                                      C.c_int, C.POINTER(abi.ICDesc), _vp, _vp]),
    "flsp_default_dg_opts": (None, [C.POINTER(abi.DGOpts)]),
    "flsp_default_reinit_opts": (None, [C.POINTER(abi.ReinitOpts)]),
    "flsp_default_ls_opts": (None, [C.POINTER(abi.LSOpts)]),
    "flsp_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "flsp_mlp_create_patch": (C.c_int, [C.c_int, C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "flsp_mlp_info": (C.c_int, [_vp, _ip, _ip, _i64p]),
    "flsp_mlp_destroy": (None, [_vp]),
    "flsp_mlp_n_params": (C.c_int, [_i64p]),
    "flsp_mlp_get_params": (C.c_int, [_vp, _fp, C.c_int64]),
    "flsp_mlp_set_params": (C.c_int, [_vp, _fp, C.c_int64]),
    "flsp_mlp_forward": (C.c_int, [_vp, _fp, C.c_int64, _fp]),
    "flsp_mlp_backward": (C.c_int, [_vp, _fp, _fp, C.c_int64, _fp]),
    "flsp_mlp_collect": (C.c_int, [_vp, _vp, C.c_double, C.POINTER(abi.ReinitOpts), _i64p]),
    "flsp_mlp_n_pairs": (C.c_int, [_vp, _i64p]),
    "flsp_mlp_clear_pairs": (C.c_int, [_vp]),
    "flsp_mlp_train": (C.c_int, [_vp, C.POINTER(abi.TrainOpts), _dp]),
    "flsp_mlp_eval": (C.c_int, [_vp, _dp]),
    "flsp_reinit_learned": (C.c_int, [_vp, _vp, C.POINTER(abi.LearnedOpts), C.POINTER(abi.LearnedStats)]),
    "flsp_ls_run_steps_learned": (C.c_int, [_vp, _vp, C.POINTER(abi.LearnedOpts), C.c_int, C.c_int]),
    "flsp_learned_totals": (C.c_int, [_vp, _i64p, _i64p, C.c_int]),
    "flsp_default_train_opts": (None, [C.POINTER(abi.TrainOpts)]),
    "flsp_default_learned_opts": (None, [C.POINTER(abi.LearnedOpts)]),
    "flsp_batch_create": (C.c_int, [C.c_int, C.POINTER(abi.MeshDesc), C.POINTER(abi.DGOpts), C.POINTER(_vp)]),
    "flsp_batch_destroy": (None, [_vp]),
    "flsp_batch_size": (C.c_int, [_vp, _ip]),
    "flsp_batch_problem": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "flsp_batch_autotune": (C.c_int, [_vp, C.POINTER(abi.BatchTuning)]),
    "flsp_batch_run_steps": (C.c_int, [_vp, C.POINTER(abi.LSOpts), C.c_int]),
    "flsp_batch_sync": (C.c_int, [_vp]),
    "flsp_batch_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "flsp_group_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(_vp)]),
    "flsp_group_destroy": (None, [_vp]),
    "flsp_group_run_periods": (C.c_int, [_vp, C.POINTER(abi.LSOpts), C.c_int]),
    "flsp_group_run_periods_learned": (C.c_int, [_vp, _vp, C.POINTER(abi.LearnedOpts), C.c_int, C.c_int]),
    "flsp_group_sync": (C.c_int, [_vp]),
    "flsp_group_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
}


class FlspError(RuntimeError):
    def __init__(self, code, msg):
        self.code = code
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")


def load():
    """Load libflsp_dg.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing; build it with `python -m felspa_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code):
    if code != abi.FLSP_OK:
        msg = load().flsp_last_error()
        raise FlspError(code, msg.decode() if msg else "")
    return code


def fp(a):
    return a.ctypes.data_as(_fp)


def dp(a):
    return a.ctypes.data_as(_dp)
