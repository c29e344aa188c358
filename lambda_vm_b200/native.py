"""ctypes binding of libstarkgpu.so (the C ABI in include/starkgpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstarkgpu.so")

SG_OK, SG_ERR_INVALID, SG_ERR_CUDA, SG_ERR_OOM, SG_ERR_BUDGET, SG_ERR_UNSUPPORTED = range(6)
_ERR_NAMES = {1: "SG_ERR_INVALID", 2: "SG_ERR_CUDA", 3: "SG_ERR_OOM", 4: "SG_ERR_BUDGET", 5: "SG_ERR_UNSUPPORTED"}


class SgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class LeafLayout(C.Structure):
    _fields_ = [("rows_per_leaf", C.c_uint32), ("little_endian", C.c_uint32),
                ("col_start", C.c_uint64), ("col_end", C.c_uint64)]


class LdeInfo(C.Structure):
    _fields_ = [("d_lde", C.c_void_p), ("lde_rows", C.c_uint64), ("row_u64", C.c_uint64),
                ("d_nodes", C.c_void_p), ("leaves_len", C.c_uint64), ("root", C.c_uint8 * 32)]


u64, u32, i32, vp = C.c_uint64, C.c_uint32, C.c_int, C.c_void_p
PROTOTYPES = {
    "sg_ctx_create": (i32, [i32, u64, C.POINTER(vp)]),
    "sg_ctx_destroy": (None, [vp]),
    "sg_last_error": (C.c_char_p, []),
    "sg_ctx_memory": (i32, [vp, C.POINTER(u64), C.POINTER(u64)]),
    "sg_ctx_launches": (u64, [vp]),
    "sg_ctx_fail_alloc_after": (i32, [vp, C.c_int64]),
    "sg_dev_alloc": (i32, [vp, vp, u64, C.POINTER(vp)]),
    "sg_dev_free": (i32, [vp, vp, vp, u64]),
    "sg_memcpy_h2d": (i32, [vp, vp, vp, vp, u64]),
    "sg_memcpy_d2h": (i32, [vp, vp, vp, vp, u64]),
    "sg_stream_sync": (i32, [vp, vp]),
    "sg_host_alloc": (i32, [u64, C.POINTER(vp)]),
    "sg_host_free": (i32, [vp]),
    "sg_ntt_forward": (i32, [vp, vp, vp, u64, u64]),
    "sg_ntt_inverse": (i32, [vp, vp, vp, u64, u64]),
    "sg_coset_lde": (i32, [vp, vp, vp, u64, u64, u32, vp, vp]),
    "sg_keccak_leaves": (i32, [vp, vp, vp, u64, u64, C.POINTER(LeafLayout), vp]),
    "sg_merkle_build": (i32, [vp, vp, vp, u64, vp, vp]),
    "sg_merkle_leaves_len": (u64, [u64]),
    "sg_merkle_gather_paths": (i32, [vp, vp, vp, u64, vp, u32, vp]),
    "sg_lde_commit": (i32, [vp, vp, vp, i32, u64, u64, u32, vp, C.POINTER(LeafLayout), vp, C.POINTER(vp), vp]),
    "sg_lde_get_info": (i32, [vp, C.POINTER(LdeInfo)]),
    "sg_lde_free": (None, [vp, vp]),
    "sg_grind": (i32, [vp, vp, vp, C.c_uint8, C.POINTER(u64)]),
    "sg_coset_lde_static": (i32, [vp, vp, u64, u64, u32, vp, vp]),
}
SG_STATIC_SCRATCH_BYTES = 32 << 20

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python lambda_vm_b200/build.py` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != SG_OK:
        msg = lib().sg_last_error()
        raise SgError(rc, msg.decode() if msg else "")
    return rc
