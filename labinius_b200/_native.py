"""ctypes binding of the C ABI in include/labinius_gpu.h (``liblabinius_gpu.so``, built in-tree).

The library is loaded from this package directory only; there is no fallback: if it is missing
or fails to load, every call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblabinius_gpu.so")

LBG_OK = 0
LBG_ERR_INVALID = -1
LBG_ERR_PARAMS = -2
LBG_ERR_CUDA = -3
LBG_ERR_OOM = -4
LBG_ERR_UNSUPPORTED = -5
LBG_ERR_WITNESS = -6


class lbg_params(ctypes.Structure):
    _fields_ = [
        ("witness_log_len", ctypes.c_uint32),
        ("column_log_len", ctypes.c_uint32),
        ("n_moduli", ctypes.c_uint32),
        ("moduli", ctypes.c_uint32 * 7),
        ("opening", ctypes.c_uint32),
        ("dropped_bits", ctypes.c_uint32),
    ]


# Every symbol the header declares, with its signature: (restype, argtypes).
_vp, _sz, _u32, _u64, _int, _dbl = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64,
                                    ctypes.c_int, ctypes.c_double)
_P = ctypes.POINTER(lbg_params)
SIGNATURES = {
    "lbg_last_error": (ctypes.c_char_p, []),
    "lbg_version": (_int, []),
    "lbg_params_check": (_int, [_P]),
    "lbg_public_parameters_from_seed": (_int, [_P, _vp, ctypes.POINTER(_vp)]),
    "lbg_public_parameters_free": (None, [_vp]),
    "lbg_key_download": (_int, [_vp, _vp]),
    "lbg_prover_new": (_int, [_vp, ctypes.POINTER(_vp)]),
    "lbg_prover_free": (None, [_vp]),
    "lbg_witness_from_host": (_int, [_vp, _vp, _sz, ctypes.POINTER(_vp)]),
    "lbg_witness_random": (_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    "lbg_witness_lifted": (_int, [_vp, _vp, _sz, ctypes.POINTER(_vp)]),
    "lbg_witness_download": (_int, [_vp, _vp, _sz]),
    "lbg_witness_free": (None, [_vp]),
    "lbg_commit": (_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "lbg_opening_matrix": (_int, [_vp, _vp]),
    "lbg_opening_dropped": (_int, [_vp, _vp, _vp]),
    "lbg_opening_free": (None, [_vp]),
    "lbg_opening_pack_commitment": (ctypes.c_longlong, [_vp, _vp, _sz]),
    "lbg_row_evaluate_packed": (ctypes.c_longlong, [_vp, _vp, _vp, _sz, _vp, _vp, _sz]),
    "lbg_batch_arena_bytes": (_sz, [_vp, _sz, _sz]),
    "lbg_device_memory": (_int, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
    "lbg_row_evaluate": (_int, [_vp, _vp, _vp, _sz, _vp]),
    "lbg_mle_evaluate": (_int, [_vp, _vp, _vp, _sz, _vp, _sz, _vp]),
    "lbg_fold": (_int, [_vp, _vp, _vp, _sz, _vp]),
    "lbg_prover_folded": (_int, [_vp, _vp]),
    "lbg_fold_commitment": (_int, [_vp, _vp, _sz, _vp, _sz, _vp]),
    "lbg_transcript_new": (_vp, [_vp, _sz]),
    "lbg_transcript_clone": (_vp, [_vp]),
    "lbg_transcript_free": (None, [_vp]),
    "lbg_transcript_absorb_bytes": (None, [_vp, _vp, _sz]),
    "lbg_transcript_absorb_u64": (None, [_vp, _u64]),
    "lbg_transcript_fill": (None, [_vp, ctypes.c_char_p, _vp, _sz]),
    "lbg_sample_short_challenge": (_int, [_vp, _u32, _dbl, _vp, _vp]),
    "lbg_derive_evaluation_point": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "lbg_derive_folding_challenges": (_int, [_vp, _vp, _vp, _vp]),
    "lbg_pack_dropped": (_sz, [_vp, _vp, _vp, _vp, _sz]),
    "lbg_pp_columns": (_sz, [_vp]),
    "lbg_pp_len_ring": (_sz, [_vp]),
    "lbg_pp_witness_len": (_sz, [_vp]),
    "lbg_pp_limbs": (_u32, [_vp]),
    "lbg_prover_stream": (_vp, [_vp]),
    "lbg_prover_sync": (_int, [_vp]),
    "lbg_prover_profile": (_int, [_vp, _int]),
    "lbg_prover_kernel_stats": (_int, [_vp, ctypes.c_char_p, _vp, _vp]),
    "lbg_prover_launch_count": (_u64, [_vp]),
    "lbg_params_derive_evaluation_point": (_int, [_P, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "lbg_params_derive_folding_challenges": (_int, [_P, _vp, _vp, _vp]),
    "lbg_params_pack_dropped": (_sz, [_P, _vp, _vp, _vp, _sz]),
    "lbg_fold_static": (_int, [_u32, _u32, _u32, _vp, _vp, _sz, _vp, _vp]),
    "lbg_batch_new": (_int, [_vp, _vp, _sz, ctypes.POINTER(_vp)]),
    "lbg_batch_new_capacity": (_int, [_vp, _sz, _sz, ctypes.POINTER(_vp)]),
    "lbg_batch_assign": (_int, [_vp, _vp, _sz]),
    "lbg_batch_witness_generate": (_int, [_vp, _vp, _vp]),
    "lbg_batch_free": (None, [_vp]),
    "lbg_batch_columns": (_sz, [_vp]),
    "lbg_batch_witness_random": (_int, [_vp, _vp]),
    "lbg_batch_witness_upload": (_int, [_vp, _sz, _vp, _sz]),
    "lbg_batch_witness_download": (_int, [_vp, _sz, _vp, _sz]),
    "lbg_batch_use_graphs": (_int, [_vp, _int]),
    "lbg_batch_autotune": (_int, [_vp, _vp, _vp]),
    "lbg_batch_commit": (_int, [_vp, _vp, _vp, _vp]),
    "lbg_batch_row_evaluate": (_int, [_vp, _vp, _vp]),
    "lbg_batch_mle_evaluate": (_int, [_vp, _vp, _vp, _vp]),
    "lbg_batch_fold": (_int, [_vp, _vp, _sz, _vp]),
    "lbg_batch_round": (_int, [_vp, _vp, _sz, _vp]),
    "lbg_batch_set_switch": (_int, [_vp, _vp, _vp, _vp]),
    "lbg_commit_host": (_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "lbg_wire_encode": (ctypes.c_longlong, [_vp, _sz, ctypes.c_uint32, _vp, _sz]),
    "lbg_wire_encode_bound": (_sz, [_sz]),
    "lbg_prover_encode_folded": (ctypes.c_longlong, [_vp, _vp, _sz]),
    "lbg_verify_folded_opening_bd": (_int, [_vp, _vp, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _vp, _vp]),
    "lbg_batch_switch_outputs": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "lbg_prover_set_kept_transform": (_int, [_vp, _int]),
    "lbg_batch_set_kept_transform": (_int, [_vp, _int]),
    "lbg_fold_row_evaluation": (_int, [_vp, _vp, _vp, _sz, _vp]),
    "lbg_verify_evaluation": (_int, [_vp, _vp, _sz, _vp, _vp, _sz, _vp]),
    "lbg_verify_folded_opening": (_int, [_vp, _vp, _vp, _vp, _sz, _vp, _vp]),
    "lbg_switch_prove": (_int, [_vp, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "lbg_ntt648_forward": (_int, [ctypes.c_uint32, _vp, _vp, _sz, _vp]),
    "lbg_ntt648_inverse": (_int, [ctypes.c_uint32, _vp, _vp, _sz, _vp]),
    "lbg_batch_stream": (_vp, [_vp]),
    "lbg_batch_set_priority": (_int, [_vp, _int]),
    "lbg_batch_schedule": (_int, [_vp, _vp, _vp]),
    "lbg_opening_residues": (_int, [_vp, _sz, _vp]),
    "lbg_left_expansion": (_int, [_vp, _vp, _sz, _sz, _vp]),
    "lbg_batch_set_sm_limit": (_int, [_vp, _int]),
    "lbg_batch_launch_count": (_u64, [_vp]),
}

_lib = None


class lbg_batch_outputs(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in
                ("matrix", "top", "digits", "p0", "p1", "mle", "u", "challenges", "v")]


class NativeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"labinius_gpu error {code}: {msg}")
        self.code = code


def lib():
    """The loaded library; raises if it is absent (build with labinius_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m labinius_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != LBG_OK:
        raise NativeError(rc, lib().lbg_last_error().decode(errors="replace"))
    return rc


def ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)
