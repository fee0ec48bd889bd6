"""ctypes binding of ``libtenet_b200.so`` (the C ABI in ``include/tenet_b200.h``).

The library is built in-tree (``python -m tenet_b200.build``).  Loading fails
loudly when it is missing: there is no fallback implementation.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtenet_b200.so"

TNT_OK = 0
STATUS_NAMES = {
    0: "TNT_OK",
    1: "TNT_INVALID_ARGUMENT",
    2: "TNT_OUT_OF_MEMORY",
    3: "TNT_UNSUPPORTED",
    4: "TNT_CUDA_ERROR",
    5: "TNT_DEVICE_TIMEOUT",
    6: "TNT_INTERNAL",
}

U1, SU2, FZ2, Z2 = 0, 1, 2, 3
CODEC_PACKED, CODEC_CANTOR = 0, 1
PREC_FP64, PREC_BF16X, PREC_CUBLAS_FP64, PREC_INT8X = 0, 1, 2, 3
TRUNC_FULL, TRUNC_RANK, TRUNC_TOL, TRUNC_DISCARD, TRUNC_SPACE = 0, 1, 2, 3, 4


class TenetError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


vp = C.c_void_p
i32, i64, u64, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double
P = C.POINTER

# name -> argtypes (restype is tnt_status = int unless listed in _RESTYPES)
_SIGS = {
    "tnt_last_error": [C.c_char_p, C.c_size_t],
    "tnt_version": [],
    "tnt_rule_create": [i32, P(i32), i32, P(vp)],
    "tnt_rule_create_table": [i32, P(i32), P(C.c_uint8), P(f64), P(f64), P(f64), P(f64), f64, P(vp)],
    "tnt_rule_destroy": [vp],
    "tnt_rule_sector_id": [vp, P(i32), P(u64)],
    "tnt_rule_fsymbol": [vp, P(i32), P(f64)],
    "tnt_rule_rsymbol": [vp, P(i32), P(f64)],
    "tnt_rule_dim": [vp, P(i32), P(f64)],
    "tnt_space_create": [vp, i32, i32, P(i32), P(i32), P(i64), P(C.c_uint8), P(vp)],
    "tnt_space_destroy": [vp],
    "tnt_space_info": [vp, P(i64), P(i32), P(i32), P(i32), P(i32)],
    "tnt_space_sectors": [vp, P(i32), P(i64), P(i64), P(i64)],
    "tnt_space_blocks": [vp, P(i64), P(i64), P(i64), P(i32)],
    "tnt_space_block_keys": [vp, P(i32), i64, P(i64)],
    "tnt_space_leg": [vp, i32, P(i32), P(i32), P(i64), P(C.c_uint8)],
    "tnt_permute_plan": [vp, i32, P(i32), i32, P(i32), P(vp)],
    "tnt_braid_plan": [vp, i32, P(i32), i32, P(i32), P(i32), P(vp)],
    "tnt_repartition_plan": [vp, i32, P(vp)],
    "tnt_adjoint_plan": [vp, P(vp)],
    "tnt_twist_plan": [vp, i32, P(i32), i32, P(vp)],
    "tnt_transform_chain_plan": [vp, i32, P(i32), i64, P(vp)],
    "tnt_xplan_from_tables": [i32, i64, P(i64), i64, P(i64), i64, P(i64), i64, P(f64), i64, i64, P(vp)],
    "tnt_network_plan": [i32, P(vp), P(C.c_uint8), i32, P(i32), i64, i32, P(i32), i64, P(vp)],
    "tnt_nplan_destroy": [vp],
    "tnt_nplan_output_space": [vp, P(vp)],
    "tnt_nplan_info": [vp, P(i64), P(i64), P(C.c_double), P(i64), P(i64)],
    "tnt_nplan_workspace_bytes": [vp, i32, i32, P(C.c_size_t)],
    "tnt_network_execute": [vp, vp, i32, P(vp), vp, vp, C.c_size_t, i32, i32, vp],
    "tnt_contract_rhs_plan": [vp, i32, P(i32), i32, P(i32), P(vp)],
    "tnt_xplan_destroy": [vp],
    "tnt_xplan_dst_space": [vp, P(vp)],
    "tnt_xplan_info": [vp, P(i64), P(i64), P(i64)],
    "tnt_xplan_entries": [vp, P(i64), P(i64)],
    "tnt_xplan_export": [vp, P(i64), P(i64), P(i64), P(f64)],
    "tnt_compose_plan": [vp, vp, P(vp)],
    "tnt_cplan_destroy": [vp],
    "tnt_cplan_dst_space": [vp, P(vp)],
    "tnt_cplan_info": [vp, P(i64), P(f64)],
    "tnt_cplan_export": [vp, P(i64)],
    "tnt_cplan_from_jobs": [i64, P(i64), i64, i64, i64, P(vp)],
    "tnt_factor_plan": [vp, P(vp)],
    "tnt_fplan_destroy": [vp],
    "tnt_fplan_info": [vp, P(i32), P(i64), P(i64), P(i64)],
    "tnt_fplan_export": [vp, P(i64), P(f64)],
    "tnt_ctx_create": [i32, P(vp)],
    "tnt_ctx_destroy": [vp],
    "tnt_transform": [vp, vp, vp, vp, f64, f64, vp],
    "tnt_compose": [vp, vp, i64, vp, i64, vp, i64, vp, i64, f64, f64, i32, i32, vp],
    "tnt_compose_host": [vp, vp, i64, vp, vp, vp, i32, i32, vp],
    "tnt_svd": [vp, vp, vp, vp, vp, vp, vp],
    "tnt_svd_static": [vp, vp, vp, vp, vp, vp],
    "tnt_truncate": [vp, vp, vp, i32, f64, f64, P(i64), vp, vp, vp],
    "tnt_xplan_concat": [i32, P(vp), P(i64), P(i64), P(vp)],
    "tnt_cplan_concat": [i32, P(vp), P(i64), P(i64), P(i64), P(vp)],
    "tnt_fplan_concat": [i32, P(vp), P(i64), P(i64), P(i64), P(i64), P(i64), P(vp)],
    "tnt_fplan_work": [vp, P(i64)],
    "tnt_svd_ws": [vp, vp, vp, vp, vp, vp, vp, vp],
    "tnt_qr": [vp, vp, vp, vp, vp, vp],
    "tnt_svd_ws_async": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
    "tnt_truncate_async": [vp, vp, vp, i32, f64, f64, vp, vp, vp, vp],
    "tnt_copy_segments_async": [vp, i64, vp, vp, vp, vp, vp],
    "tnt_ctx_svd_sweeps": [vp, P(i32)],
    "tnt_ctx_sync": [vp, vp],
    "tnt_cplan_scratch_bytes": [vp, i64, i32, i32, P(C.c_size_t)],
    "tnt_compose_ws": [vp, vp, i64, vp, i64, vp, i64, vp, i64, f64, f64, i32, i32, vp, C.c_size_t, vp],
    "tnt_split_operand_bytes": [vp, i32, i32, i32, P(C.c_size_t)],
    "tnt_split_pack_operand": [vp, vp, i32, vp, i32, i32, vp, C.c_size_t, vp],
    "tnt_compose_packed": [vp, vp, vp, vp, vp, vp, vp, f64, f64, i32, i32, vp],
    "tnt_cplan_tile_shapes": [vp, P(f64), P(i32)],
    "tnt_tuning_info": [i32, P(f64), P(i32), P(f64), P(i32)],
    "tnt_eigh": [vp, vp, vp, vp, vp, vp, vp],
    "tnt_truncate_segments": [vp, vp, i32, P(i32), vp, i32, f64, f64, P(i64), vp, vp, vp],
    "tnt_copy_segments": [vp, i64, P(i64), vp, vp, vp, vp],
    "tnt_wdot": [vp, vp, i32, vp, i64, vp, vp, vp],
    "tnt_axpy_many": [vp, i64, i32, vp, i64, vp, f64, vp, vp, vp],
    "tnt_symeig": [vp, i32, vp, vp, vp, vp],
}
_RESTYPES = {
    "tnt_version": C.c_char_p,
    "tnt_rule_destroy": None,
    "tnt_space_destroy": None,
    "tnt_xplan_destroy": None,
    "tnt_cplan_destroy": None,
    "tnt_fplan_destroy": None,
    "tnt_ctx_destroy": None,
    "tnt_nplan_destroy": None,
}

_lib = None


def lib():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m tenet_b200.build` "
                "(the package has no CPU fallback)"
            )
        handle = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
        for name, args in _SIGS.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = handle
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().tnt_last_error(buf, len(buf))
    return buf.value.decode()


def check(status: int):
    if status != TNT_OK:
        raise TenetError(status, last_error())


def call(name, *args):
    check(getattr(lib(), name)(*args))


def arr(ctype, values):
    values = list(values)
    return (ctype * max(1, len(values)))(*values)
