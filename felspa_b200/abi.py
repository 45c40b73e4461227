"""ctypes mirror of include/flsp_dg.h (the C ABI of libflsp_dg.so).

The structure layouts here must match the header field for field; the
test suite checks sizes against the library (``flsp_abi_sizes``).
"""
import ctypes as C

FLSP_OK = 0
FLSP_ERR_CUDA = 1
FLSP_ERR_NONFINITE = 2
FLSP_ERR_BAD_ARG = 3
FLSP_ERR_BAD_MESH = 4
FLSP_ERR_TIMEOUT = 5
FLSP_ERR_BAND_NOT_REACHED = 6
FLSP_ERR_UNSUPPORTED = 7
FLSP_ERR_NO_DEVICE = 8
FLSP_ERR_OOM = 9

STATUS_NAMES = {
    0: "FLSP_OK", 1: "FLSP_ERR_CUDA", 2: "FLSP_ERR_NONFINITE", 3: "FLSP_ERR_BAD_ARG",
    4: "FLSP_ERR_BAD_MESH", 5: "FLSP_ERR_TIMEOUT", 6: "FLSP_ERR_BAND_NOT_REACHED",
    7: "FLSP_ERR_UNSUPPORTED", 8: "FLSP_ERR_NO_DEVICE", 9: "FLSP_ERR_OOM",
}

BASIS_P = 0
BASIS_Q = 1
FP64 = 0
FP32 = 1

F_ONE, F_LIN, F_SIN, F_COS, F_SINSQ, F_SINPI, F_COSPI, F_SINPISQ = range(8)
T_ONE, T_COS, T_COSPI, T_ONE_MINUS_EXP = range(4)
IC_SPHERE, IC_RECT, IC_HEIGHT, IC_UNION, IC_DIFF, IC_INTERSECT = range(6)
REINIT_BAND, REINIT_GLOBAL, REINIT_FIXED = range(3)
CURV_REFERENCE, CURV_NEIGHBOUR = range(2)
(RED_MASS, RED_MASS_ERROR, RED_L1_INTERFACE, RED_MEAN_ABS_DIFF, RED_GRAD_DEVIATION,
 RED_MAX_ABS, RED_L2_ERROR_IC, RED_L1_INTERFACE_IC, RED_MASS_SHARP) = range(9)
NOALLOC_MAX_CELLS = 65536 * 128   # flsp_reduce_noalloc scratch limit (cells)
MAX_MATERIALS = 8                 # level sets of a material stack
MAX_MIX_QPTS = 8                  # Gauss points per axis of the mixing
HEAVISIDE_NONE, HEAVISIDE_LINEAR, HEAVISIDE_SINE = 0, 1, 2

MAX_VEL_TERMS = 24
MAX_IC_NODES = 32
MAX_IC_WAVES = 32


class MeshDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("host_cell_order", C.POINTER(C.c_int64)),
        ("boundary_ids", C.POINTER(C.c_int32)),
    ]


class DGOpts(C.Structure):
    _fields_ = [
        ("degree", C.c_int),
        ("basis", C.c_int),
        ("precision", C.c_int),
        ("rk_order", C.c_int),
        ("cfl_max", C.c_double),
        ("device", C.c_int),
    ]


class Factor(C.Structure):
    _fields_ = [("kind", C.c_int), ("a", C.c_double), ("b", C.c_double)]


class VelTerm(C.Structure):
    _fields_ = [("comp", C.c_int), ("coeff", C.c_double), ("f", Factor * 3)]


class VelocityDesc(C.Structure):
    _fields_ = [
        ("n_terms", C.c_int),
        ("terms", VelTerm * MAX_VEL_TERMS),
        ("time_kind", C.c_int),
        ("ta", C.c_double),
        ("tb", C.c_double),
    ]


class ICNode(C.Structure):
    _fields_ = [("kind", C.c_int), ("a", C.c_int), ("b", C.c_int), ("p", C.c_double * 6)]


class ICDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int),
        ("root", C.c_int),
        ("exact", C.c_int),
        ("nodes", ICNode * MAX_IC_NODES),
        ("n_waves", C.c_int),
        ("waves", (C.c_double * 4) * MAX_IC_WAVES),
    ]


class ReinitOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int),
        ("n_pseudo_steps", C.c_int),
        ("band_width_coeff", C.c_double),
        ("max_iter", C.c_int),
        ("cfl_max", C.c_double),
        ("viscosity", C.c_double),
        ("rk_order", C.c_int),
        ("limiter", C.c_int),
        ("narrow_band", C.c_int),
        ("band_cells", C.c_double),
    ]


class TrainOpts(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("batch", C.c_int),
        ("lr", C.c_double),
        ("beta1", C.c_double),
        ("beta2", C.c_double),
        ("eps", C.c_double),
        ("seed", C.c_uint64),
    ]


class LearnedOpts(C.Structure):
    _fields_ = [
        ("band_cells", C.c_double),
        ("max_residual", C.c_double),
        ("fallback", ReinitOpts),
    ]


class LearnedStats(C.Structure):
    _fields_ = [
        ("n_band", C.c_int64),
        ("n_fallback", C.c_int64),
        ("hj_ran", C.c_int),
    ]


class BatchTuning(C.Structure):
    _fields_ = [
        ("adv_tile", C.c_int * 2),
        ("hj_tile", C.c_int * 2),
        ("n_adv", C.c_int),
        ("n_hj", C.c_int),
        ("adv_cand", (C.c_int * 2) * 8),
        ("hj_cand", (C.c_int * 2) * 8),
        ("adv_ms", C.c_double * 8),
        ("hj_ms", C.c_double * 8),
    ]


MLP_IN, MLP_HIDDEN, MLP_OUT = 82, 256, 9
MLP3_IN, MLP3_OUT = 730, 27
PATCH_2D_Q2, PATCH_3D_Q2 = 0, 1


class LSOpts(C.Structure):
    _fields_ = [
        ("reinit_frequency", C.c_int),
        ("execute_reinit", C.c_int),
        ("reinit", ReinitOpts),
    ]


def default_reinit_opts(**kw):
    """ReinitControl / AdditionalControl defaults (reinit.h:276-341)."""
    o = ReinitOpts(mode=REINIT_BAND, n_pseudo_steps=5, band_width_coeff=4.0,
                   max_iter=1000, cfl_max=0.2, viscosity=0.0, rk_order=1,
                   limiter=-1, narrow_band=0, band_cells=6.0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_ls_opts(reinit=None, **kw):
    """LevelSetControl defaults (level_set.h:108-166)."""
    o = LSOpts(reinit_frequency=10, execute_reinit=1,
               reinit=reinit if reinit is not None else default_reinit_opts())
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def mesh_desc(dim, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), host_cell_order=None, boundary_ids=None):
    m = MeshDesc()
    m.dim = dim
    n = list(n) + [1] * (3 - len(n))
    lo = list(lo) + [0.0] * (3 - len(lo))
    hi = list(hi) + [1.0] * (3 - len(hi))
    for d in range(3):
        m.n[d] = int(n[d])
        m.lo[d] = float(lo[d])
        m.hi[d] = float(hi[d])
    m.host_cell_order = host_cell_order
    m.boundary_ids = boundary_ids
    return m
