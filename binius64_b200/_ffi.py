"""ctypes binding of libbinius_gpu.so (declarations in include/binius_gpu.h).

The CUDA library is the product path: if it is missing this module raises instead of falling back
to any CPU implementation.
"""
from __future__ import annotations

import ctypes
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libbinius_gpu.so")
HEADER_PATHS = [os.path.join(ROOT, "include", "binius_gpu.h")]

BINIUS_OK = 0
BINIUS_E_ARG = 1
BINIUS_E_OOM = 2
BINIUS_E_CUDA = 3
BINIUS_E_TIMEOUT = 4
BINIUS_E_UNSUPPORTED = 5

_STATUS_NAMES = {0: "OK", 1: "ArgumentError", 2: "OutOfMemory", 3: "CudaError", 4: "Timeout",
                 5: "Unsupported"}


class BiniusError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class ArgumentError(BiniusError, ValueError):
    """Mirrors binius_prover::Error::ArgumentError (prover/prover/src/error.rs:9-24)."""


class OutOfMemoryError(BiniusError, MemoryError):
    """BINIUS_E_OOM: a device allocation was refused, or a proving queue refused a request that
    needs more device memory than its budget."""


_c = ctypes
_vp = _c.c_void_p
_u32 = _c.c_uint32
_u64 = _c.c_uint64
_int = _c.c_int

# name -> (restype, argtypes)
_SIGS = {
    "binius_last_error": (_c.c_char_p, []),
    "binius_version": (_c.c_char_p, []),
    "binius_launch_count": (_u64, []),
    "binius_ntt_create": (_int, [_int, _vp, _u32, _c.POINTER(_vp)]),
    "binius_ntt_destroy": (_int, [_vp]),
    "binius_ntt_log_domain": (_u32, [_vp]),
    "binius_domain_subspace": (_int, [_vp, _u32, _u32, _vp]),
    "binius_ntt_twiddles": (_vp, [_vp]),
    "binius_ntt_forward": (_int, [_vp, _vp, _u32, _u32, _u32, _vp]),
    "binius_ntt_inverse": (_int, [_vp, _vp, _u32, _u32, _u32, _vp]),
    "binius_rs_encode_batch": (_int, [_vp, _vp, _u32, _u32, _u32, _vp, _vp]),
    "binius_merkle_commit": (_int, [_vp, _u32, _u32, _vp, _vp]),
    "binius_merkle_branch": (_int, [_vp, _u32, _u64, _u32, _vp, _vp]),
    "binius_merkle_layer": (_int, [_vp, _u32, _u32, _vp, _vp]),
    "binius_fri_fold_interleaved": (_int, [_vp, _u32, _u32, _vp, _vp, _vp]),
    "binius_fri_fold_codeword": (_int, [_vp, _vp, _u32, _vp, _u32, _vp, _vp]),
    "binius_fri_fold_codeword_noalloc": (_int, [_vp, _vp, _u32, _vp, _u32, _vp, _vp]),
    "binius_fri_commit_interleaved": (_int, [_vp, _vp, _u32, _u32, _u32, _vp, _vp, _vp, _vp]),
    "binius_transcript_create": (_int, [_c.POINTER(_vp)]),
    "binius_transcript_destroy": (_int, [_vp]),
    "binius_transcript_message": (_int, [_vp, _vp, _c.c_size_t]),
    "binius_transcript_decommitment": (_int, [_vp, _vp, _c.c_size_t]),
    "binius_transcript_observe": (_int, [_vp, _vp, _c.c_size_t]),
    "binius_transcript_sample": (_int, [_vp, _vp, _c.c_size_t]),
    "binius_transcript_sample_bits": (_u32, [_vp, _u32]),
    "binius_transcript_len": (_c.c_size_t, [_vp]),
    "binius_transcript_finalize": (_int, [_vp, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t)]),
    "binius_pcs_create": (_int, [_vp, _u32, _u32, _u32, _vp, _u32, _u32, _c.POINTER(_vp)]),
    "binius_pcs_destroy": (_int, [_vp]),
    "binius_pcs_commit": (_int, [_vp, _vp, _c.POINTER(_vp), _vp, _vp]),
    "binius_pcs_committed_destroy": (_int, [_vp]),
    "binius_pcs_committed_codeword": (_vp, [_vp]),
    "binius_pcs_prove": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "binius_cs_from_bytes": (_int, [_int, _c.c_char_p, _c.c_size_t, _c.POINTER(_vp)]),
    "binius_cs_destroy": (_int, [_vp]),
    "binius_cs_info": (_int, [_vp, _vp]),
    "binius_values_data_encode": (_int, [_vp, _c.c_size_t, _vp, _c.c_size_t,
                                         _c.POINTER(_c.c_size_t)]),
    "binius_values_data_decode": (_int, [_vp, _c.c_size_t, _vp, _c.c_size_t,
                                         _c.POINTER(_c.c_size_t)]),
    "binius_proof_encode": (_int, [_vp, _c.c_size_t, _c.c_char_p, _vp, _c.c_size_t,
                                   _c.POINTER(_c.c_size_t)]),
    "binius_proof_decode": (_int, [_vp, _c.c_size_t, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t),
                                   _c.c_char_p, _c.c_size_t]),
    "binius_value_vec_from_data": (_int, [_vp, _vp, _c.c_size_t, _vp, _c.c_size_t, _vp]),
    "binius_key_collection_from_cs_bytes": (_int, [_c.c_char_p, _c.c_size_t, _vp, _c.c_size_t,
                                                   _c.POINTER(_c.c_size_t)]),
    "binius_cs_key_collection": (_int, [_vp, _vp, _c.c_size_t, _c.POINTER(_c.c_size_t)]),
    "binius_cs_load_key_collection": (_int, [_vp, _c.c_char_p, _c.c_size_t]),
    "binius_prover_setup_with_key_collection": (_int, [_vp, _u32, _c.c_char_p, _c.c_size_t,
                                                       _vp]),
    "binius_vision4_permute": (_int, [_vp, _u64, _vp]),
    "binius_eval_form_create": (_int, [_c.c_char_p, _c.c_size_t, _u64, _vp]),
    "binius_eval_form_info": (_int, [_vp, _vp]),
    "binius_eval_form_evaluate": (_int, [_vp, _vp, _u32, _vp, _vp, _vp]),
    "binius_eval_form_destroy": (_int, [_vp]),
    "binius_values_transpose": (_int, [_vp, _u64, _u64, _vp, _vp]),
    "binius_merkle_commit_vision4": (_int, [_vp, _u32, _u32, _vp, _vp]),
    "binius_pcs_set_merkle_hash": (_int, [_vp, _u32]),
    "binius_prover_set_merkle_hash": (_int, [_vp, _u32]),
    "binius_eval_operands": (_int, [_vp, _vp, _int, _vp, _vp]),
    "binius_and_reduction_prove": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "binius_shift_reduction_prove": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "binius_intmul_reduction_prove": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "binius_prover_setup": (_int, [_vp, _u32, _vp]),
    "binius_setup": (_int, [_int, _c.c_char_p, _c.c_size_t, _u32, _c.c_char_p, _c.c_size_t,
                            _vp]),
    "binius_prove": (_int, [_vp, _vp, _c.c_size_t, _vp, _vp, _c.c_size_t,
                            _c.POINTER(_c.c_size_t), _vp]),
    "binius_prover_destroy": (_int, [_vp]),
    "binius_prover_info": (_int, [_vp, _vp]),
    "binius_prover_prove": (_int, [_vp, _vp, _vp, _vp]),
    "binius_prover_phase_ms": (_int, [_vp, _vp]),
    "binius_prover_committed_words": (_u64, [_vp]),
    "binius_prover_workspace_bytes": (_u64, [_vp]),
    "binius_prover_get_tuning": (_int, [_vp, _vp]),
    "binius_prover_set_tuning": (_int, [_vp, _vp]),
    "binius_prover_autotune": (_int, [_vp, _vp, _u32, _vp, _vp]),
    "binius_queue_create": (_int, [_int, _u32, _u64, _vp]),
    "binius_queue_destroy": (_int, [_vp]),
    "binius_queue_submit": (_int, [_vp, _vp, _vp, _int, _vp]),
    "binius_queue_poll": (_int, [_vp, _u64, _vp]),
    "binius_queue_wait": (_int, [_vp, _u64, _vp, _c.c_size_t, _vp, _vp]),
    "binius_queue_stats": (_int, [_vp, _vp]),
    "binius_debug_fail_allocs": (None, [_c.c_int64]),
    "binius_fri_n_test_queries": (_u32, [_u32, _u32]),
    "binius_fri_estimate_optimal_arity": (_u32, [_u32, _u32, _u32]),
    "binius_gf_mul_batch": (_int, [_vp, _vp, _vp, _u64, _vp]),
    "binius_bivariate_round_evals": (_int, [_vp, _vp, _u32, _vp, _vp]),
    "binius_bivariate_fold_round_evals": (_int, [_vp, _vp, _u32, _vp, _vp, _vp]),
    "binius_sumcheck_bivariate_create": (_int, [_vp, _vp, _u32, _vp, _vp, _vp]),
    "binius_sumcheck_bivariate_execute": (_int, [_vp, _vp, _vp]),
    "binius_sumcheck_bivariate_fold": (_int, [_vp, _vp]),
    "binius_sumcheck_bivariate_finish": (_int, [_vp, _vp]),
    "binius_sumcheck_quadratic_mle_create": (_int, [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp]),
    "binius_sumcheck_quadratic_mle_execute": (_int, [_vp, _vp, _vp]),
    "binius_sumcheck_quadratic_mle_fold": (_int, [_vp, _vp]),
    "binius_sumcheck_quadratic_mle_finish": (_int, [_vp, _vp]),
    "binius_sumcheck_quadratic_mle_eval_point": (_int, [_vp, _vp]),
    "binius_sumcheck_inout_create": (_int, [_vp, _u32, _vp, _u32, _vp, _vp]),
    "binius_sumcheck_inout_execute": (_int, [_vp, _vp, _vp]),
    "binius_sumcheck_inout_fold": (_int, [_vp, _vp]),
    "binius_sumcheck_inout_finish": (_int, [_vp, _vp]),
    "binius_sumcheck_inout_eval_point": (_int, [_vp, _vp]),
    "binius_sumcheck_n_vars": (_u32, [_vp]),
    "binius_sumcheck_destroy": (_int, [_vp]),
}

_lib = None


def declared_functions() -> list[str]:
    """Function names declared in include/*.h (used by the export test)."""
    names = []
    for path in HEADER_PATHS:
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(binius_[a-z0-9_]+)\s*\(", text):
            if m.group(1) not in names:
                names.append(m.group(1))
    return names


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                f"g.build()'` (there is no CPU fallback for the GPU prover path)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != BINIUS_OK:
        msg = lib().binius_last_error().decode(errors="replace")
        if rc == BINIUS_E_ARG:
            raise ArgumentError(rc, msg)
        if rc == BINIUS_E_OOM:
            raise OutOfMemoryError(rc, msg)
        raise BiniusError(rc, msg)
