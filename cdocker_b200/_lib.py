"""ctypes binding of libcdock_b200.so (the C-ABI declared in include/cdock_b200.h).

The library is loaded from the package directory. There is no fallback: if the shared
library is missing the import fails with an explicit error, and if no GPU is present the
GPU entry points return CDK_ERR_CUDA.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcdock_b200.so")

CDK_OK = 0
CDK_ERR_INVALID = 1
CDK_ERR_CUDA = 2
CDK_ERR_NOMEM = 3
CDK_ERR_UNSUPPORTED = 4
CDK_ERR_OVERFLOW = 5
CDK_ERR_IO = 6
CDK_ERR_BUSY = 7

CDK_FORM_FP32 = 0
CDK_FORM_BF16X3 = 1
CDK_FORM_FP16X2 = 2


class CdkOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("form", C.c_int),
        ("wave_rotations", C.c_int),
        ("max_atoms", C.c_int),
        ("col_tile", C.c_int),
        ("use_graphs", C.c_int),
        ("reserved", C.c_int * 8),
    ]


class CdkServerOpts(C.Structure):
    _fields_ = [
        ("arena_bytes", C.c_size_t),
        ("wave_rotations", C.c_int),
        ("max_box", C.c_int),
        ("max_atoms", C.c_int),
        ("max_conformers", C.c_int),
        ("max_waiting", C.c_int),
        ("reserved", C.c_int * 4),
    ]


class CdkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cdk error {code}: {msg}")
        self.code = code


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_vp = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "cdk_version": (C.c_char_p, []),
    "cdk_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "cdk_opts_default": (None, [C.POINTER(CdkOpts)]),
    "cdk_ctx_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _fp,
                                 C.POINTER(CdkOpts), C.POINTER(_vp)]),
    "cdk_ctx_destroy": (C.c_int, [_vp]),
    "cdk_search": (C.c_int, [_vp, C.c_int, C.c_int, _fp, _fp, _fp, _ip, C.c_int, _fp, _fp, _ip,
                             _vp]),
    "cdk_search_device": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp,
                                    _vp, _vp]),
    "cdk_search_device_noalloc": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int,
                                            _vp, _vp, _vp, _vp]),
    "cdk_rescore_fp64": (C.c_int, [_vp, C.c_int, C.c_int, _fp, _fp, _fp, _ip, C.c_int, _ip, _fp,
                                   _ip, _dp, _vp]),
    "cdk_fill_ligand_grid": (C.c_int, [C.c_int, C.c_int, _fp, _fp, _fp, _fp, _ip, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_float, _fp]),
    "cdk_conj_mult": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp]),
    "cdk_sum_grids": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "cdk_quaternion_uniform_sampling": (C.c_int, [C.c_uint64, C.c_int, C.c_int, _fp]),
    "cdk_filter_quaternions": (C.c_int, [_fp, C.c_int, C.c_int, _fp, C.c_float, C.c_float,
                                         C.c_float, C.c_int, _fp, _ip]),
    "cdk_vdw_slots": (C.c_int, [C.c_int, _fp, C.c_int, _fp, _ip, _ip, _ip]),
    "cdk_read_grids": (C.c_int, [C.c_char_p, _ip, _fp, _fp, C.c_long, _fp, C.c_long]),
    "cdk_write_grids": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp,
                                  C.c_float, C.c_float, _fp, _fp]),
    "cdk_synth_receptor_grids": (C.c_int, [C.c_int, C.c_float, _fp, C.c_int, _fp, _fp, _fp, _fp,
                                           C.c_int, _fp, C.c_float, C.c_float, C.c_float, _fp]),
    "cdk_receptor_grids_gpu": (C.c_int, [C.c_int, C.c_int, C.c_float, _fp, C.c_int, _fp, _fp, _fp,
                                         _fp, C.c_int, _fp, C.c_float, C.c_float, C.c_float, _fp]),
    "cdk_ctx_stats": (C.c_int, [_vp, _dp, C.c_int]),
    "cdk_server_opts_default": (None, [C.POINTER(CdkServerOpts)]),
    "cdk_server_create": (C.c_int, [_vp, C.POINTER(CdkServerOpts), C.POINTER(_vp)]),
    "cdk_server_submit": (C.c_int, [_vp, C.c_int, C.c_int, _fp, _fp, _fp, _ip, C.c_int, _fp,
                                    C.POINTER(C.c_uint64)]),
    "cdk_server_poll": (C.c_int, [_vp, C.c_uint64, C.c_int, _fp, _ip, _dp]),
    "cdk_server_stats": (C.c_int, [_vp, _dp, C.c_int]),
    "cdk_server_destroy": (C.c_int, [_vp]),
    "cdk_pose_coordinates": (C.c_int, [C.c_int, _fp, _fp, _dp, C.c_float, _ip, _dp]),
    "cdk_sort_index": (C.c_int, [_fp, C.c_long, C.POINTER(C.c_long)]),
    "cdk_ctx_top_poses": (C.c_int, [_vp, C.c_int, _ip, _fp, _ip, _dp, _ip]),
    "cdk_cluster_conformers": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _vp, C.c_double, C.c_int,
                                         _ip, _ip]),
    "cdk_pair_rmsd": (C.c_int, [C.c_int, C.c_int, _dp, _vp, _dp]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libcdock_b200.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cdocker_b200.build` "
                "(there is no CPU fallback for the search path)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().cdk_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != CDK_OK:
        raise CdkError(rc, last_error())
