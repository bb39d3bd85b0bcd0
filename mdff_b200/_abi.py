"""ctypes mirror of ``include/mdff_gpu.h`` and the loader of ``libmdff_gpu.so``.

The structures here are byte-for-byte the C structs of the boundary; the
layout test (tests/test_abi.py) checks their sizes against the compiled
library.  Per-type tables use C indexing ``[it][jt]`` = namelist entry
``(it+1, jt+1)`` of the reference (e.g. ``Abmhftd(1,2)`` in
``non_bonded.f90:135-150``).
"""
import ctypes
import os

NKCLASS = 7      # MDFF_NKCLASS
KCLASS_NAMES = ("list_build", "short_range", "real_space_field", "real_space_force",
                "structure_factor", "reciprocal_field", "other")
NT = 16          # MDFF_NTYPEMAX (config.f90:42 ntypemax)
ASPC_DEPTH = 5   # dipia_ind_t(5,3,natm) (coulomb.f90:435)
ABI_VERSION = 1

MDFF_OK = 0
MDFF_ERR_BAD_ARGS = 1
MDFF_ERR_CUDA = 2
MDFF_ERR_CATASTROPHE = 3
MDFF_ERR_LIST_OVERFLOW = 4
MDFF_ERR_NOT_CONVERGED = 5
MDFF_ERR_TIMEOUT = 6
MDFF_ERR_NO_DEVICE = 7
MDFF_ERR_UNSUPPORTED = 8
MDFF_ERR_NOMEM = 9

CALC_MD, CALC_OPT, CALC_OTHER = 0, 1, 2
TRUNC_NONE, TRUNC_LINEAR, TRUNC_QUADRATIC = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
SOLVER_SCF, SOLVER_CG = 0, 1
THOLE_NONE, THOLE_LINEAR, THOLE_EXPON1, THOLE_EXPON2, THOLE_GAUSS = 0, 1, 2, 3, 4
ALGO_SCF, ALGO_KO_V1, ALGO_KO_V2, ALGO_KO_V3, ALGO_KO_V4_1, ALGO_KO_V4_2 = 0, 1, 2, 3, 4, 5
EXT_ASPC, EXT_POLY = 0, 1

_d = ctypes.c_double
_i = ctypes.c_int


class MdffParams(ctypes.Structure):
    _fields_ = [
        ("natm", _i), ("ntype", _i), ("natmi", _i * NT),
        ("lcoulomb", _i), ("lbmhft", _i), ("lbmhftd", _i), ("lnmlj", _i),
        ("lsurf", _i), ("lreduced", _i), ("calc", _i),
        ("cutshortrange", _d), ("cutlongrange", _d), ("skindiff", _d),
        ("qch", _d * NT), ("dip", (_d * 3) * NT),
        ("trunc", _i), ("symmetric_pot_nb", _i),
        ("epslj", (_d * NT) * NT), ("sigmalj", (_d * NT) * NT),
        ("plj", (_d * NT) * NT), ("qlj", (_d * NT) * NT),
        ("Abmhftd", (_d * NT) * NT), ("Bbmhftd", (_d * NT) * NT),
        ("Cbmhftd", (_d * NT) * NT), ("Dbmhftd", (_d * NT) * NT),
        ("BDbmhftd", (_d * NT) * NT),
        ("alphaES", _d), ("kES", _i * 3), ("lautoES", _i), ("epsw", _d),
        ("ldip_polar", _i * NT), ("poldip", ((_d * 3) * 3) * NT),
        ("ldip_damping", ((_i * NT) * NT) * NT),
        ("pol_damp_b", ((_d * NT) * NT) * NT),
        ("pol_damp_c", ((_d * NT) * NT) * NT),
        ("pol_damp_k", ((_i * NT) * NT) * NT),
        ("conv_tol_ind", _d), ("min_scf_pol_iter", _i), ("max_scf_pol_iter", _i),
        ("extrapolate_order", _i), ("symmetric_pot_pim", _i),
        ("precision", _i), ("solver", _i), ("cg_tol", _d), ("cg_max_iter", _i),
        ("fail_on_nonconvergence", _i), ("device", _i),
        ("wall24", (_d * NT) * NT),
        ("thole_type", _i), ("thole_param", (_d * NT) * NT),
        ("algo_moment_from_pola", _i), ("algo_ext_dipole", _i), ("omegakO", _d),
        ("lwfc", _i * NT), ("ldip_wfc", _i), ("rcut_wfc", _d),
    ]


class MdffResult(ctypes.Structure):
    _fields_ = [
        ("fx", ctypes.POINTER(_d)), ("fy", ctypes.POINTER(_d)), ("fz", ctypes.POINTER(_d)),
        ("mu", ctypes.POINTER(_d)), ("ef", ctypes.POINTER(_d)),
        ("u_lj", _d), ("vir_lj", _d), ("u_bmhft", _d), ("vir_bmhft", _d),
        ("u_coul", _d), ("u_pol", _d), ("pvirial_coul", _d),
        ("tau_nonb", (_d * 3) * 3), ("tau_coul", (_d * 3) * 3), ("tau", (_d * 3) * 3),
    ]


class MdffStats(ctypes.Structure):
    _fields_ = [
        ("n_pol_iter", _i), ("converged", _i), ("rmsd", _d),
        ("list_rebuilds", _i), ("list_capacity", _i), ("list_needed", _i),
        ("nk", _i), ("alphaES", _d), ("kES", _i * 3), ("cutlongrange", _d),
        ("n_launches", _i), ("ms_last", _d), ("rmsd_initial", _d), ("n_fp64_residuals", _i),
        ("n_kardir", _i),
    ]


BATCH_MAXTYPES = 4
BATCH_MAXATM = 2048


class MdffBatchDesc(ctypes.Structure):
    _fields_ = [("nconf", _i), ("pset", ctypes.POINTER(_i)), ("natmi", ctypes.POINTER(_i)),
                ("cell_A", ctypes.POINTER(_d))]


class MdffBatchConf(ctypes.Structure):
    _fields_ = [
        ("u_lj", _d), ("vir_lj", _d), ("u_bmhft", _d), ("vir_bmhft", _d),
        ("u_coul", _d), ("u_pol", _d), ("pvirial_coul", _d),
        ("tau_nonb", (_d * 3) * 3), ("tau_coul", (_d * 3) * 3), ("tau", (_d * 3) * 3),
        ("rmsd", _d), ("n_pol_iter", _i), ("converged", _i), ("catastrophe", _i), ("nk", _i),
        ("alphaES", _d), ("cutlongrange", _d), ("kES", _i * 3), ("pad", _i),
    ]


# every symbol include/mdff_gpu.h declares, with its ctypes signature
_P = ctypes.c_void_p
_DP = ctypes.POINTER(_d)
_IP = ctypes.POINTER(_i)
SIGNATURES = {
    "mdff_gpu_abi_version": (_i, []),
    "mdff_gpu_struct_size": (_i, [_i]),
    "mdff_gpu_strerror": (ctypes.c_char_p, [_i]),
    "mdff_gpu_last_error": (ctypes.c_char_p, [_P]),
    "mdff_gpu_create": (_i, [ctypes.POINTER(MdffParams), _DP, ctypes.POINTER(_P)]),
    "mdff_gpu_set_cell": (_i, [_P, _DP]),
    "mdff_gpu_engforce": (_i, [_P, _DP, _DP, _DP, _i, ctypes.POINTER(MdffResult)]),
    "mdff_gpu_engforce_device": (_i, [_P, _P, _i, _P, _P, _P, ctypes.POINTER(MdffResult)]),
    "mdff_gpu_get_aspc_history": (_i, [_P, _DP]),
    "mdff_gpu_set_aspc_history": (_i, [_P, _DP]),
    "mdff_gpu_kardir_roundtrips": (_i, [_P, _DP, _DP, _DP, _i]),
    "mdff_gpu_get_stats": (_i, [_P, ctypes.POINTER(MdffStats)]),
    "mdff_gpu_verlet_half_list": (_i, [_P, _i, _DP, _DP, _DP, _IP, _IP, _i, _IP]),
    "mdff_gpu_verlet_half_list_noalloc": (_i, [ctypes.POINTER(MdffParams), _DP, _i, _DP, _DP, _DP,
                                                _IP, _IP, _i, _IP]),
    "mdff_gpu_md_nve": (_i, [_P, _P, _P, _P, _d, _i, _i, _DP]),
    "mdff_gpu_profile": (_i, [_P, _i]),
    "mdff_gpu_set_tc_wait_limit": (_i, [_P, _i]),
    "mdff_gpu_kernel_times": (_i, [_P, _DP, ctypes.POINTER(ctypes.c_longlong), _DP]),
    "mdff_gpu_peak_flops": (_i, [_i, _i, _DP]),
    "mdff_gpu_efg": (_i, [_P, _DP]),
    "mdff_gpu_destroy": (None, [_P]),
    "mdff_gpu_batch_create": (_i, [ctypes.POINTER(MdffParams), _i, ctypes.POINTER(MdffBatchDesc),
                                   ctypes.POINTER(_P)]),
    "mdff_gpu_batch_engforce": (_i, [_P, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP,
                                     ctypes.POINTER(MdffBatchConf)]),
    "mdff_gpu_batch_engforce_device": (_i, [_P, _P, _P, _P, _P, ctypes.POINTER(MdffBatchConf)]),
    "mdff_gpu_batch_tune": (_i, [_P, _IP, _IP, _DP]),
    "mdff_gpu_batch_set_shape": (_i, [_P, _i, _i]),
    "mdff_gpu_batch_info": (_i, [_P, _IP, _IP, _IP, _IP, _DP]),
    "mdff_gpu_batch_last_error": (ctypes.c_char_p, [_P]),
    "mdff_gpu_batch_destroy": (None, [_P]),
    "mdff_gpu_batch_fit_define": (_i, [_P, _i, _IP, _IP, _IP]),
    "mdff_gpu_batch_fit_set": (_i, [_P, _DP]),
    "mdff_gpu_batch_fit_get": (_i, [_P, _DP]),
    "mdff_gpu_batch_adjoint": (_i, [_P, _P, _P, _P, _i, _DP, _DP]),
}

FIT_A, FIT_RHO, FIT_C, FIT_POL, FIT_TTB, FIT_TTC, FIT_QSCALE = range(7)
FIT_MAX = 16

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdff_gpu.so")
_lib = None


class MdffError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"mdff status {status}: {msg}")


def load_library(path=None):
    """Load libmdff_gpu.so (built in-tree by mdff_b200.build).  There is no
    fallback: a missing library is an error."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libmdff_gpu.so not built at {p}; run mdff_b200.build.build()")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_DP)


def iptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_IP)
