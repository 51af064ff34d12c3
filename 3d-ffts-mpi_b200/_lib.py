"""ctypes binding of ``liba2afft_b200.so`` (declarations in
``include/a2afft_b200.h``).  Loading fails loudly when the library has not been
built: there is no fallback implementation."""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "liba2afft_b200.so")

# a2a_status
SUCCESS = 0
STATUS_NAMES = {
    0: "A2A_SUCCESS",
    1: "A2A_ERROR_INVALID_VALUE",
    2: "A2A_ERROR_DECOMPOSITION",
    3: "A2A_ERROR_UNSUPPORTED",
    4: "A2A_ERROR_NO_PLANS",
    5: "A2A_ERROR_MISALIGNED",
    6: "A2A_ERROR_CUDA",
    7: "A2A_ERROR_OUT_OF_MEMORY",
    8: "A2A_ERROR_TIMEOUT",
    9: "A2A_ERROR_NOT_IMPLEMENTED",
}
# a2a_precision
C128, C64 = 0, 1
# a2a_method
METHOD_PLAIN, METHOD_SPLIT_BF16, METHOD_SPLIT_FP16 = 0, 1, 2


class Desc(ctypes.Structure):
    """``a2a_distribution_desc``."""

    _fields_ = [
        ("ndims", ctypes.c_int),
        ("ng", ctypes.c_int * 3),
        ("world_size", ctypes.c_int),
        ("dims", ctypes.c_int * 3),
        ("local_grid_size", ctypes.c_int * 3),
        ("nlocal", ctypes.c_int64),
        ("nsends", ctypes.c_int64),
        ("block_size", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("element_bytes", ctypes.c_size_t),
        ("buffer_bytes", ctypes.c_size_t),
        ("first_rank", ctypes.c_int),
        ("local_ranks", ctypes.c_int),
    ]


_P = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
_I = ctypes.c_int
_I3 = ctypes.c_int * 3

# name -> argtypes (every function returns a2a_status unless listed in _RET)
SIGNATURES = {
    "a2a_distribution_create": [_I, _I, _I, _I, ctypes.POINTER(_P)],
    "a2a_distribution_create_box": [_I, _I, _I, _I, _I, _I, ctypes.POINTER(_P)],
    "a2a_distribution_describe": [_P, ctypes.POINTER(Desc)],
    "a2a_rank_coords": [_P, _I, _I3, _I3],
    "a2a_distribution_set_stream": [_P, _P],
    "a2a_distribution_set_rank_range": [_P, _I, _I],
    "a2a_get_z_pencils": [_P, _PP, _PP],
    "a2a_return_z_pencils": [_P, _PP, _PP],
    "a2a_get_x_pencils": [_P, _PP, _PP],
    "a2a_return_x_pencils": [_P, _PP, _PP],
    "a2a_get_y_pencils": [_P, _PP, _PP],
    "a2a_return_y_pencils": [_P, _PP, _PP],
    "a2a_distribution_finalize": [_P],
    "a2a_alltoall": [_P, _PP, _PP],
    "a2a_d_z_a2a_to_z_pencils": [_P, _PP, _PP],
    "a2a_d_z_pencils_to_z_a2a": [_P, _PP, _PP],
    "a2a_d_x_a2a_to_x_pencils": [_P, _PP, _PP],
    "a2a_d_x_pencils_to_x_a2a": [_P, _PP, _PP],
    "a2a_d_y_a2a_to_y_pencils": [_P, _PP, _PP],
    "a2a_d_y_pencils_to_y_a2a": [_P, _PP, _PP],
    "a2a_d_fast_z_to_x": [_P, _PP, _PP],
    "a2a_d_fast_x_to_y": [_P, _PP, _PP],
    "a2a_d_fast_y_to_z": [_P, _PP, _PP],
    "a2a_forward_1d_fft": [_P, _PP],
    "a2a_inverse_1d_fft": [_P, _PP],
    "a2a_scale_fft": [_P, _PP, _PP],
    "a2a_fast_copy_fft": [_P, _PP, _PP],
    "a2a_dfft_create": [_P, ctypes.POINTER(_P)],
    "a2a_dfft_set_method": [_P, _I],
    "a2a_dfft_make_plans": [_P, _PP],
    "a2a_dfft_set_autotune": [_P, _I],
    "a2a_dfft_variant_count": [_P, _I, ctypes.POINTER(_I)],
    "a2a_dfft_check_device": [_P],
    "a2a_dfft_select_variant": [_P, _I, _I],
    "a2a_dfft_plan_report": [_P, ctypes.c_char_p, ctypes.c_size_t],
    "a2a_dfft_forward": [_P, _PP],
    "a2a_dfft_inverse": [_P, _PP],
    "a2a_dfft_backward": [_P, _PP],
    "a2a_dfft_forward_async": [_P, _PP, _P],
    "a2a_dfft_inverse_async": [_P, _PP, _P],
    "a2a_dfft_execute_pass_async": [_P, _PP, _I, _I, _P],
    "a2a_dfft_launches_per_transform": [_P, ctypes.POINTER(_I)],
    "a2a_dfft_destroy": [_P],
    "a2a_dfft_forward_host": [_P, _P, _PP],
    "a2a_dfft_inverse_host": [_P, _P, _PP],
    "a2a_decompose": [_I, _I, _I3, _I3, ctypes.POINTER(ctypes.c_int64)],
    "a2a_write_dims": [_I, _I, ctypes.c_char_p],
    "a2a_write_rank_dumps": [_I, _I, _I, ctypes.c_char_p, _P, _P, _P],
    "a2a_lines_fft_noalloc": [_P, _I, ctypes.c_int64, _I, _I, _P],
    "a2a_dfft_execute_pass_blocks": [_P, _PP, _I, _I, _I, _I, _I, _P],
    "a2a_dfft_set_blocks_kernel": [_P, _I],
    "a2a_ipc_export": [_P, _P, ctypes.POINTER(ctypes.c_uint64)],
    "a2a_ipc_import": [_P, ctypes.c_uint64, ctypes.POINTER(_P)],
    "a2a_ipc_release": [_P],
    "a2a_batch_create": [_I, ctypes.POINTER(_I), _I, _I, ctypes.POINTER(_P)],
    "a2a_batch_box_elements": [_P, _I, ctypes.POINTER(ctypes.c_int64)],
    "a2a_batch_make_plans": [_P, _PP],
    "a2a_batch_set_schedule": [_P, _I, _I, _I],
    "a2a_batch_select_variant": [_P, _I, _I, _I],
    "a2a_batch_set_graph": [_P, _I],
    "a2a_batch_inject_stall": [_P, _I],
    "a2a_batch_plan_report": [_P, ctypes.c_char_p, ctypes.c_size_t],
    "a2a_batch_forward": [_P, _PP],
    "a2a_batch_inverse": [_P, _PP],
    "a2a_batch_forward_async": [_P, _PP, _P],
    "a2a_batch_inverse_async": [_P, _PP, _P],
    "a2a_batch_check_device": [_P],
    "a2a_batch_launches_per_transform": [_P, ctypes.POINTER(_I)],
    "a2a_batch_destroy": [_P],
    "a2a_status_string": [_I],
    "a2a_last_error": [],
    "a2a_version": [],
}
_RET = {"a2a_status_string": ctypes.c_char_p, "a2a_last_error": ctypes.c_char_p, "a2a_version": ctypes.c_int}

_lib = None


class A2AError(RuntimeError):
    """A non-success ``a2a_status`` with the library's detail message."""

    def __init__(self, status: int, func: str, detail: str):
        self.status = status
        self.func = func
        self.detail = detail
        super().__init__(f"{func}: {STATUS_NAMES.get(status, status)}: {detail}")


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C {os.path.join(PKG_DIR, 'csrc')}` "
                "or __graft_entry__.build(); there is no fallback implementation"
            )
        handle = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = _RET.get(name, ctypes.c_int)
        _lib = handle
    return _lib


def call(name: str, *args) -> None:
    """Call ``name`` and raise ``A2AError`` unless it returned A2A_SUCCESS."""
    st = getattr(lib(), name)(*args)
    if st != SUCCESS:
        detail = lib().a2a_last_error().decode(errors="replace")
        raise A2AError(st, name, detail)


def bufptr(ptr: int):
    """``void**`` holding one device pointer (the reference's ``fftPrecision**``)."""
    return (ctypes.c_void_p * 1)(ptr)
