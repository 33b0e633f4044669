"""ctypes binding of libpmc_coag_gpu.so (the C ABI in include/pmc_coag_gpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmc_coag_gpu.so")

PMC_OK = 0
PMC_ERR_CAPACITY = 3
STATUS_NAMES = {
    0: "PMC_OK",
    1: "PMC_ERR_INVALID_ARG",
    2: "PMC_ERR_OUT_OF_GRID",
    3: "PMC_ERR_CAPACITY",
    4: "PMC_ERR_CUDA",
    5: "PMC_ERR_TIMEOUT",
    6: "PMC_ERR_RNG_EXHAUSTED",
    7: "PMC_ERR_ASSERT",
    8: "PMC_ERR_NO_DEVICE",
}

MODE_FP64, MODE_MIXED, MODE_REPLAY = 0, 1, 2

# every symbol the header declares, with (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_LP = ctypes.POINTER(ctypes.c_int64)
_ULP = ctypes.POINTER(ctypes.c_uint64)
_PP = ctypes.POINTER(ctypes.c_void_p)

SIGNATURES = {
    "pmc_coag_gpu_init": (_I, [_I, _DP, _I, _I, _I, _IP, _DP, _DP, ctypes.c_uint64, _PP]),
    "pmc_coag_gpu_init_batch": (_I, [_I, _I, _DP, _I, _I, _I, _IP, _DP, _DP, _ULP, _PP]),
    "pmc_coag_gpu_destroy": (_I, [_P]),
    "pmc_coag_gpu_upload": (_I, [_P, _I, _I, _DP, _IP, _IP, _LP, _IP]),
    "pmc_coag_gpu_upload_components": (_I, [_P, _I, _I, _IP, _IP, _DP]),
    "pmc_coag_gpu_step": (_I, [_P, _I, _D, _D, _D, _D, _IP, _IP]),
    "pmc_coag_gpu_step_batch": (_I, [_P, _I, _DP, _DP, _D, _D, _I, _LP, _LP]),
    "pmc_coag_gpu_n_part": (_I, [_P, _I, _IP]),
    "pmc_coag_gpu_download": (_I, [_P, _I, _I, _DP, _IP, _IP, _LP, _IP, _IP]),
    "pmc_coag_gpu_download_components": (_I, [_P, _I, _I, _IP, _IP, _DP]),
    "pmc_coag_gpu_sync_host": (_I, [_P, _I, _I, _DP, _IP, _IP, _LP, _IP, ctypes.POINTER(ctypes.c_uint8), _IP, _IP,
                                    _IP]),
    "pmc_coag_gpu_set_weight": (_I, [_P, _IP, _DP, _DP]),
    "pmc_coag_gpu_set_weight_pop": (_I, [_P, _I, _IP, _DP, _DP]),
    "pmc_coag_gpu_set_next_id": (_I, [_P, _I, ctypes.c_int64]),
    "pmc_coag_gpu_get_next_id": (_I, [_P, _I, _LP]),
    "pmc_coag_gpu_set_mode": (_I, [_P, _I]),
    "pmc_coag_gpu_set_graphs": (_I, [_P, _I]),
    "pmc_coag_gpu_set_seed": (_I, [_P, _I, ctypes.c_uint64]),
    "pmc_coag_gpu_rebalance": (_I, [_P, _I, _DP, _I, _I]),
    "pmc_coag_gpu_autotune": (_I, [_P, _I]),
    "pmc_coag_gpu_tune_state": (_I, [_P, _IP, _IP, ctypes.POINTER(ctypes.c_float)]),
    "pmc_coag_gpu_set_tune": (_I, [_P, _IP]),
    "pmc_coag_gpu_add_dist_sample": (_I, [_P, _I, _I, _IP, _DP, _DP, _DP, _DP, _DP, _IP, _IP, _DP, _DP, _D, _D, _D,
                                          _DP, _I, _I, _LP]),
    "pmc_coag_gpu_get_weight": (_I, [_P, _I, _DP]),
    "pmc_coag_gpu_size_dist": (_I, [_P, _I, _I, _D, _D, _DP, _DP]),
    "pmc_coag_gpu_replay_set": (_I, [_P, _DP, ctypes.c_int64]),
    "pmc_coag_gpu_replay_open": (_I, [_P, ctypes.c_char_p]),
    "pmc_coag_gpu_replay_used": (_I, [_P, _LP]),
    "pmc_coag_gpu_stats": (_I, [_P, _LP, _LP, _LP]),
    "pmc_coag_gpu_sort": (_I, [_P, _I, _IP, _DP, _I, _IP, _IP]),
    "pmc_coag_gpu_kmax_table": (_I, [_P, _I, _D, _D, _D, _DP, _I]),
    "pmc_coag_gpu_eval_kernel": (_I, [_P, _I, _D, _D, _D, _I, _DP, _IP, _DP, _IP, _IP, _DP]),
    "pmc_coag_gpu_status_string": (ctypes.c_char_p, [_I]),
    "pmc_coag_gpu_profile": (_I, [_P, _I]),
    "pmc_coag_gpu_profile_read": (_I, [_P, _I, _DP, _LP, _LP]),
    "pmc_coag_gpu_launch_count": (_I, [_LP]),
    "pmc_coag_gpu_conflicts": (_I, [_P, _LP, _LP, _LP, _LP]),
    "pmc_coag_gpu_exact_tests": (_I, [_P, _LP]),
    "pmc_coag_gpu_set_fractal": (_I, [_P, _D, _D, _D]),
    "pmc_coag_gpu_set_record_removals": (_I, [_P, _I]),
    "pmc_coag_gpu_removals": (_I, [_P, _I, ctypes.c_int64, _LP, _IP, _LP, _LP]),
    "pmc_coag_gpu_bin_sort_noalloc": (_I, [_I, _P, _P, _I, _I, _D, _D, _P, _P, _P, _P, _P]),
}

_lib = None


class PmcError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        name = STATUS_NAMES.get(code, str(code))
        msg = ""
        try:
            msg = lib().pmc_coag_gpu_status_string(code).decode()
        except Exception:
            pass
        super().__init__(f"{where}: {name} ({msg})")


def lib():
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} not found: build it with `python -m partmc_b200.build` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, where):
    if code != PMC_OK:
        raise PmcError(code, where)


def dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


def ip(a):
    return a.ctypes.data_as(_IP) if a is not None else None


def lp(a):
    return a.ctypes.data_as(_LP) if a is not None else None
